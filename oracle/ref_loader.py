"""TEST INFRASTRUCTURE ONLY: the reference's own table loader, compiled from
the reference sources (oracle/_ref/libahead_ref_load.so, ``make refload``;
oracle/ref/ref_load.cpp is its C entry).  It is the checker that pins the
loader restatement (oracle/tbl_oracle.c) and, through fixtures it writes, the
GPU loader: ``load_table`` runs AHEAD::loadTable
(lib/AHEAD.cpp:96-128 -> lib/column_storage/Transaction.cpp:66-648) on
``<directory>/<table>`` and returns every column as raw bytes, ``width`` bytes
per row in the column's own type.  The reference always converts: a column
without its ``.ahead`` file is parsed from the ``.tbl`` text and written; with
every file present the columns are read from them (re-encoded to the minimum
bit-flip weight's A when one is given).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REFLOAD_LIB = os.path.join(HERE, "_ref", "libahead_ref_load.so")


class RefLoadError(RuntimeError):
    """An exception the reference's loader raised (its text)."""


def build_refload() -> Optional[str]:
    """Compile the reference's loader (only where the reference tree exists)."""
    ref = os.environ.get("AHEAD_REFERENCE", "/root/reference")
    if not os.path.isdir(os.path.join(ref, "lib", "column_storage")):
        return REFLOAD_LIB if os.path.exists(REFLOAD_LIB) else None
    subprocess.run(["make", "-s", "-C", HERE, "refload", f"REFERENCE={ref}"], check=True)
    return REFLOAD_LIB


_lib = None


def _load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(REFLOAD_LIB)
        u64 = ctypes.c_uint64
        lib.refl_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, u64, ctypes.c_char_p,
                                  ctypes.c_int, ctypes.POINTER(u64), ctypes.c_char_p, ctypes.c_size_t]
        lib.refl_column.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p,
                                    u64, ctypes.POINTER(u64), ctypes.c_char_p, ctypes.c_size_t]
        lib.refl_reset.restype = None
        _lib = lib
    return _lib


def load_table(directory: str, table: str, columns: Sequence[Tuple[str, int, int]], min_bfw: int = 0,
               size: Optional[int] = None, delim: Optional[str] = None, ignore_more_data: bool = True
               ) -> Tuple[int, Dict[str, np.ndarray]]:
    """(rows, {name: raw bytes}) of ``<directory>/<table>`` loaded by the
    reference; ``columns`` = (name, header type code of include/ahead_ingest.h,
    width in bytes), e.g. from ahead_b200.ingest.read_header.  The reference's
    managers are process-wide singletons that cannot be created again once
    destroyed, so every load runs in a fresh child process."""
    import json
    import sys
    out = os.path.join(directory, f".{table}.refload.npz")
    args = json.dumps({"directory": directory, "table": table, "columns": [list(c) for c in columns],
                       "min_bfw": min_bfw, "size": size, "delim": delim, "ignore_more_data": ignore_more_data,
                       "out": out})
    proc = subprocess.run([sys.executable, "-m", "oracle.ref_loader", args], cwd=os.path.dirname(HERE),
                          capture_output=True, text=True)
    if proc.returncode == 3:
        raise RefLoadError(proc.stdout.strip())
    if proc.returncode:
        raise RuntimeError(f"reference loader child failed ({proc.returncode}): {proc.stderr[-2000:]}")
    with np.load(out) as z:
        rows = int(z["__rows__"])
        cols = {c[0]: z[c[0]] for c in columns}
    os.remove(out)
    return rows, cols


def _load_here(directory: str, table: str, columns: Sequence[Tuple[str, int, int]], min_bfw: int,
               size: Optional[int], delim: Optional[str], ignore_more_data: bool
               ) -> Tuple[int, Dict[str, np.ndarray]]:
    lib = _load()
    err = ctypes.create_string_buffer(1024)
    rows = ctypes.c_uint64(0)
    try:
        rc = lib.refl_load(directory.encode(), table.encode(), int(min_bfw), 1,
                           ctypes.c_uint64((1 << 64) - 1 if size is None else size),
                           delim.encode() if delim else None, int(ignore_more_data), ctypes.byref(rows), err,
                           len(err))
        if rc:
            raise RefLoadError(err.value.decode(errors="replace"))
        n = int(rows.value)
        out = {}
        for name, tbl_type, width in columns:
            buf = np.zeros(max(n, 1) * int(width), np.uint8)
            cnt = ctypes.c_uint64(0)
            rc = lib.refl_column(table.encode(), name.encode(), int(tbl_type), int(width), buf.ctypes.data,
                                 ctypes.c_uint64(n), ctypes.byref(cnt), err, len(err))
            if rc:
                raise RefLoadError(err.value.decode(errors="replace"))
            out[name] = buf[: int(cnt.value) * int(width)]
        return n, out
    finally:
        lib.refl_reset()


if __name__ == "__main__":  # the child of load_table
    import json
    import sys
    a = json.loads(sys.argv[1])
    try:
        n, cols = _load_here(a["directory"], a["table"], [tuple(c) for c in a["columns"]], a["min_bfw"], a["size"],
                             a["delim"], a["ignore_more_data"])
    except RefLoadError as ex:
        print(ex)
        sys.exit(3)
    np.savez(a["out"], __rows__=np.array(n), **cols)
