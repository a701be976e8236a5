"""Table loader: the reference's TransactionManager::Transaction::load over
libahead_b200.so (include/ahead_ingest.h).

``load(ops, path, ...)`` keeps the reference's arguments
(include/column_storage/TransactionManager.h:129-135: path, tableName,
prefix, size, delim, ignoreMoreData) plus the two configuration switches it
reads (AHEAD_Config.cpp:33-40: ``--AN-minbfw`` and ``--convert-table-files``)
as keywords.  It reads ``<path>_header.csv``, then each column from
``<path>_<column>.ahead`` where that file exists (re-encoding AN columns to
the min-BFW A on the device) and the rest from ``<path>.tbl`` (parsed on the
device), and writes the ``.ahead`` files of the parsed columns.  Columns stay
in device memory; integer and AN columns come back as BATs.

``write_tbl`` / ``format_tbl`` turn columns into `.tbl` text and a header
file (the dbgen layout: every field followed by the delimiter); they make
the synthetic tables the tests and the bench load.
"""
from __future__ import annotations

import ctypes
import sys
import os
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .gpu import AheadError, GpuOps, load_library
from .model import OK, WIDTH, Bat, Col, void_col

TINYINT, SHORTINT, INT, LARGEINT, STRING, FIXED, CHAR, RESTINY, RESSHORT, RESINT, RESBIGINT = range(11)
TYPE_NAMES = {TINYINT: "TINYINT", SHORTINT: "SHORTINT", INT: "INTEGER", LARGEINT: "LARGEINT", STRING: "STRING",
              FIXED: "FIXED", CHAR: "CHAR", RESTINY: "RESTINY", RESSHORT: "RESSHORT", RESINT: "RESINT",
              RESBIGINT: "RESBIGINT"}
# parse kinds (ahead_tbl_kind)
KIND_SKIP, KIND_INT, KIND_RES, KIND_STRING, KIND_FIXED, KIND_CHAR = range(6)
KIND_OF = {TINYINT: KIND_INT, SHORTINT: KIND_INT, INT: KIND_INT, LARGEINT: KIND_INT, STRING: KIND_STRING,
           FIXED: KIND_FIXED, CHAR: KIND_CHAR, RESTINY: KIND_RES, RESSHORT: KIND_RES, RESINT: KIND_RES}
SIGNED = {1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}
UNSIGNED = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}


class CTblHeaderCol(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 256), ("tbl_type", ctypes.c_int32), ("width", ctypes.c_uint32)]


class CTblCol(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("width", ctypes.c_uint32), ("A", ctypes.c_uint64),
                ("data", ctypes.c_void_p)]


class CLoadOpts(ctypes.Structure):
    _fields_ = [("prefix", ctypes.c_char_p), ("size", ctypes.c_uint64), ("delim", ctypes.c_char_p),
                ("ignore_more_data", ctypes.c_int32), ("min_bfw", ctypes.c_uint32),
                ("convert_table_files", ctypes.c_int32), ("block_mb", ctypes.c_uint32)]


class CTableCol(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("tbl_type", ctypes.c_int32), ("type", ctypes.c_int32),
                ("width", ctypes.c_uint32), ("from_file", ctypes.c_int32), ("A", ctypes.c_uint64),
                ("Ainv", ctypes.c_uint64), ("unenc_max", ctypes.c_uint64), ("data", ctypes.c_void_p),
                ("count", ctypes.c_uint64)]


class CLoadStats(ctypes.Structure):
    _fields_ = [("text_bytes", ctypes.c_uint64), ("binary_bytes", ctypes.c_uint64),
                ("written_bytes", ctypes.c_uint64), ("blocks", ctypes.c_uint64), ("reencoded", ctypes.c_uint64),
                ("total_ms", ctypes.c_double), ("file_ms", ctypes.c_double), ("parse_ms", ctypes.c_double),
                ("reencode_ms", ctypes.c_double)]


def _bind(lib):
    if getattr(lib, "_ingest_bound", False):
        return lib
    vp, u64 = ctypes.c_void_p, ctypes.c_uint64
    lib.ahead_tbl_read_header.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                          ctypes.POINTER(CTblHeaderCol), ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                          ctypes.c_char_p, ctypes.c_size_t]
    lib.ahead_tbl_load_a.argtypes = [ctypes.c_int]
    lib.ahead_tbl_load_a.restype = u64
    lib.ahead_tbl_minbfw_a.argtypes = [ctypes.c_int, ctypes.c_uint32]
    lib.ahead_tbl_minbfw_a.restype = u64
    lib.ahead_gpu_tbl_parse.argtypes = [vp, vp, u64, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(CTblCol),
                                        ctypes.c_int, u64, u64, u64, ctypes.POINTER(u64), ctypes.POINTER(u64)]
    lib.ahead_gpu_reencode.argtypes = [vp, vp, u64, ctypes.c_int, u64, u64]
    lib.ahead_table_load.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(CLoadOpts), ctypes.POINTER(vp)]
    lib.ahead_table_ncols.argtypes = [vp]
    lib.ahead_table_rows.argtypes = [vp]
    lib.ahead_table_rows.restype = u64
    lib.ahead_table_column.argtypes = [vp, ctypes.c_int, ctypes.POINTER(CTableCol)]
    lib.ahead_table_stats.argtypes = [vp, ctypes.POINTER(CLoadStats)]
    lib.ahead_table_destroy.argtypes = [vp]
    lib.ahead_table_destroy.restype = None
    lib._ingest_bound = True
    return lib


def read_header(path: str, prefix: Optional[str] = None, delim: Optional[str] = None) -> List[Tuple[str, int, int]]:
    """Columns of ``<path>_header.csv`` as (name, type, width); needs no GPU."""
    lib = _bind(load_library())
    cap = 512
    cols = (CTblHeaderCol * cap)()
    n = ctypes.c_int(0)
    err = ctypes.create_string_buffer(512)
    rc = lib.ahead_tbl_read_header(path.encode(), prefix.encode() if prefix else None,
                                   delim.encode() if delim else None, cols, cap, ctypes.byref(n), err, 512)
    if rc != OK:
        raise AheadError(rc, "read_header", err.value.decode())
    return [(cols[i].name.decode(), int(cols[i].tbl_type), int(cols[i].width)) for i in range(min(n.value, cap))]


def load_a(tbl_type: int) -> int:
    return int(_bind(load_library()).ahead_tbl_load_a(tbl_type))


def minbfw_a(tbl_type: int, min_bfw: int) -> int:
    return int(_bind(load_library()).ahead_tbl_minbfw_a(tbl_type, min_bfw))


# ------------------------------------------------------------------ tables
class _Handle:
    """Owns one ahead_table; device views of its columns keep it alive."""

    def __init__(self, lib, ptr):
        self.lib, self.ptr = lib, ptr

    def __del__(self, _finalizing=sys.is_finalizing):  # bound now: module globals may be gone at exit
        if self.ptr and not _finalizing():  # the CUDA runtime may be gone at exit
            self.lib.ahead_table_destroy(self.ptr)
            self.ptr = None


class _DeviceView:
    def __init__(self, owner, ptr: int, nbytes: int):
        self.owner = owner
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3, "strides": None}


@dataclass
class Column:
    name: str
    tbl_type: int
    type: int          # BAT tail type (model.*); -1 for STRING / FIXED / CHAR
    width: int
    from_file: bool
    A: int
    Ainv: int
    unenc_max: int
    count: int
    data: object       # torch uint8 tensor on the device, count * width bytes

    def col(self) -> Col:
        if self.type < 0:
            raise TypeError(f"column {self.name} ({TYPE_NAMES[self.tbl_type]}) is not a BAT type")
        return Col(self.type, self.data, self.A, self.Ainv, self.unenc_max, 0)

    def bat(self) -> Bat:
        """(void, tail) BAT over the device column."""
        return Bat(void_col(0), self.col(), self.count)

    def host(self) -> np.ndarray:
        """Values on the host: signed integers, AN codes, float64, or byte strings."""
        raw = self.data.cpu().numpy() if self.count else np.zeros(0, np.uint8)
        if self.tbl_type in (TINYINT, SHORTINT, INT, LARGEINT):
            return raw.view(SIGNED[self.width])
        if self.tbl_type in (RESTINY, RESSHORT, RESINT):
            return raw.view(UNSIGNED[self.width])
        if self.tbl_type == FIXED:
            return raw.view(np.float64)
        return raw.view(f"S{self.width}")


class Table:
    """A loaded table: its columns in device memory, in header order."""

    def __init__(self, name: Optional[str], path: str, handle: _Handle, columns: List[Column], rows: int,
                 stats: Dict[str, float]):
        self.name, self.path, self._handle = name, path, handle
        self.columns, self.rows, self.stats = columns, rows, stats
        self._by_name = {c.name: c for c in columns}

    def __getitem__(self, name: str) -> Column:
        return self._by_name[name]

    def __contains__(self, name: str) -> bool:
        return name in self._by_name

    def names(self) -> List[str]:
        return [c.name for c in self.columns]


def load(ops: GpuOps, path: str, table_name: Optional[str] = None, prefix: Optional[str] = None,
         size: Optional[int] = None, delim: Optional[str] = None, ignore_more_data: bool = True, *,
         min_bfw: int = 0, convert_table_files: bool = True, block_mb: int = 0) -> Table:
    """Load table ``path`` (Transaction.cpp:66-648) into the device of ``ops``.

    ``table_name`` names the result (the reference also registers it in its
    catalog, which this library does not have)."""
    lib = _bind(ops.lib)
    torch = ops.torch
    opts = CLoadOpts(prefix.encode() if prefix else None, (1 << 64) - 1 if size is None else int(size),
                     delim.encode() if delim else None, int(bool(ignore_more_data)), int(min_bfw),
                     int(bool(convert_table_files)), int(block_mb))
    h = ctypes.c_void_p()
    rc = lib.ahead_table_load(ops.ctx, path.encode(), ctypes.byref(opts), ctypes.byref(h))
    if rc != OK:
        raise AheadError(rc, "load", lib.ahead_ctx_last_error(ops.ctx).decode())
    handle = _Handle(lib, h.value)
    cols: List[Column] = []
    for i in range(lib.ahead_table_ncols(h)):
        c = CTableCol()
        lib.ahead_table_column(h, i, ctypes.byref(c))
        nbytes = int(c.count) * int(c.width)
        if nbytes:
            data = torch.as_tensor(_DeviceView(handle, int(c.data), nbytes), device="cuda")
        else:
            data = torch.empty(0, dtype=torch.uint8, device="cuda")
        cols.append(Column(c.name.decode(), int(c.tbl_type), int(c.type), int(c.width), bool(c.from_file),
                           int(c.A), int(c.Ainv), int(c.unenc_max), int(c.count), data))
    st = CLoadStats()
    lib.ahead_table_stats(h, ctypes.byref(st))
    stats = {k: getattr(st, k) for k, _ in CLoadStats._fields_}
    return Table(table_name, path, handle, cols, int(lib.ahead_table_rows(h)), stats)


def tbl_parse(ops: GpuOps, text, kinds: Sequence[int], widths: Sequence[int], As: Sequence[int], outs,
              row0: int = 0, cap: Optional[int] = None, max_lines: Optional[int] = None, delim: Optional[str] = None,
              ignore_more_data: bool = True) -> int:
    """Parse device text (uint8 tensor, 16-byte aligned, whole lines) into the
    device columns ``outs`` (uint8 tensors, None for skipped columns);
    returns the number of lines in the text."""
    lib = _bind(ops.lib)
    ops.torch.cuda.current_stream().synchronize()  # the library's stream does not wait for torch's
    n = len(kinds)
    cc = (CTblCol * n)()
    for i in range(n):
        cc[i].kind, cc[i].width, cc[i].A = int(kinds[i]), int(widths[i]), int(As[i])
        cc[i].data = outs[i].data_ptr() if outs[i] is not None else None
    if cap is None:
        cap = min(int(o.numel()) // int(w) for o, w in zip(outs, widths) if o is not None) if any(
            o is not None for o in outs) else 0
    lines, bad = ctypes.c_uint64(0), ctypes.c_uint64(0)
    rc = lib.ahead_gpu_tbl_parse(ops.ctx, text.data_ptr(), text.numel(), delim.encode() if delim else None,
                                 int(bool(ignore_more_data)), cc, n, row0, cap,
                                 (1 << 64) - 1 if max_lines is None else int(max_lines), ctypes.byref(lines),
                                 ctypes.byref(bad))
    if rc != OK:
        err = AheadError(rc, "tbl_parse", lib.ahead_ctx_last_error(ops.ctx).decode())
        err.bad_line = int(bad.value)
        err.lines = int(lines.value)
        raise err
    return int(lines.value)


def reencode(ops: GpuOps, col: Col, count: int, a_new: int) -> Col:
    """Re-encode an AN column in place to ``a_new`` (ColumnManager.cpp:320-371);
    returns the column with its new A / A^-1."""
    lib = _bind(ops.lib)
    ops.torch.cuda.current_stream().synchronize()  # the library's stream does not wait for torch's
    w = WIDTH[col.type]
    rc = lib.ahead_gpu_reencode(ops.ctx, col.data.data_ptr() if count else None, count, w, col.A, a_new)
    if rc != OK:
        raise AheadError(rc, "reencode", lib.ahead_ctx_last_error(ops.ctx).decode())
    inv = pow(int(a_new), -1, 1 << (8 * w))
    return Col(col.type, col.data, int(a_new), inv, col.unenc_max, col.seqbase)


# ------------------------------------------------------------------ text
_FILL = 0xFF  # a byte no formatted field holds; dropped when the rows are packed


def _int_block(v: np.ndarray) -> np.ndarray:
    """Signed 64-bit values -> [n, 1 + digits] bytes, right-aligned, padded with _FILL."""
    v = v.astype(np.int64)
    neg = v < 0
    mag = np.where(neg, -(v + 1), v).astype(np.uint64) + neg.astype(np.uint64)  # |v| without overflow
    top = int(mag.max()) if len(mag) else 0
    nd_max = max(len(str(top)), 1)
    pw = np.array([10 ** k for k in range(nd_max - 1, -1, -1)], dtype=np.uint64)
    d = (mag[:, None] // pw[None, :]) % np.uint64(10)
    nd = np.ones(len(v), dtype=np.int64)
    for k in range(1, nd_max):
        nd += mag >= np.uint64(10 ** k)
    keep = np.arange(nd_max)[None, :] >= (nd_max - nd)[:, None]
    out = np.full((len(v), nd_max + 1), _FILL, dtype=np.uint8)
    out[:, 1:] = np.where(keep, d.astype(np.uint8) + 48, _FILL)
    out[neg, 0] = ord("-")
    return out


def _bytes_block(c: np.ndarray) -> np.ndarray:
    b = c.astype("S") if c.dtype.kind != "S" else c
    w = max(b.dtype.itemsize, 1)
    m = np.frombuffer(np.ascontiguousarray(b).tobytes(), dtype=np.uint8).reshape(len(b), w).copy()
    if (m == _FILL).any():
        raise ValueError("string fields may not hold byte 0xFF")
    m[m == 0] = _FILL
    return m


def _float_block(c: np.ndarray) -> np.ndarray:
    return _bytes_block(np.array([repr(float(x)).encode() for x in c]))


def format_tbl(columns: Sequence, delim: str = "|", rows_per_chunk: int = 1 << 18) -> bytes:
    """Rows of `.tbl` text, each field followed by ``delim`` (dbgen layout).
    A column is an integer numpy array, a float64 array (written with repr),
    or an array of byte strings (no NUL or 0xFF bytes inside)."""
    cols = [np.asarray(c) for c in columns]
    n = len(cols[0])
    d = np.full((1, 1), ord(delim), dtype=np.uint8)
    parts = []
    for r0 in range(0, n, rows_per_chunk):
        r1 = min(n, r0 + rows_per_chunk)
        blocks = []
        for c in cols:
            x = c[r0:r1]
            if x.dtype.kind in "iu":
                blocks.append(_int_block(x))
            elif x.dtype.kind == "f":
                blocks.append(_float_block(x))
            else:
                blocks.append(_bytes_block(x))
            blocks.append(np.broadcast_to(d, (r1 - r0, 1)))
        blocks.append(np.full((r1 - r0, 1), ord("\n"), dtype=np.uint8))
        m = np.hstack(blocks)
        parts.append(m[m != _FILL].tobytes())
    return b"".join(parts)


def write_tbl(path: str, names: Sequence[str], types: Sequence[str], columns: Sequence, delim: str = "|"):
    """Write ``<path>_header.csv`` and ``<path>.tbl``."""
    with open(path + "_header.csv", "w") as f:
        f.write(delim.join(names) + "\n" + delim.join(types) + "\n")
    with open(path + ".tbl", "wb") as f:
        f.write(format_tbl(columns, delim))


def remove_binaries(path: str, names: Sequence[str]):
    """Delete the ``.ahead`` files of a table (forces the next load to parse)."""
    for n in names:
        p = f"{path}_{n}.ahead"
        if os.path.exists(p):
            os.remove(p)
