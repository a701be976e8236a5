"""TEST INFRASTRUCTURE ONLY: numpy access to the loader restatement
(oracle/tbl_oracle.c) -- the checker of the GPU table loader.

``tbl_parse`` runs the line loop of TransactionManager::Transaction::load
(lib/column_storage/Transaction.cpp:485-590 of the reference) on an
in-memory text with the C library's strtok/atoi/atol/atoll/strncpy/atof;
``reencode`` is ColumnIterator::read0<true>'s re-encode
(lib/column_storage/ColumnManager.cpp:320-343).  The A tables below restate
include/util/resilience.hpp:56-109 and Transaction.cpp:357-376, 424-456.
Parity of the loader is pinned against the reference's own loader, compiled
from its sources (oracle/ref_loader.py, ``make refload``).
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

import numpy as np

from .oracle import PORT_LIB, build_port

# header type names -> (tbl type code of include/ahead_ingest.h, width); STRING is sized per header
TBL_TINYINT, TBL_SHORTINT, TBL_INT, TBL_LARGEINT, TBL_STRING, TBL_FIXED, TBL_CHAR = range(7)
TBL_RESTINY, TBL_RESSHORT, TBL_RESINT, TBL_RESBIGINT = range(7, 11)
# load A of a fresh AN column: As[7] (restiny), As[15] (resshort, resint)
LOAD_A = {TBL_RESTINY: 233, TBL_RESSHORT: 63877, TBL_RESINT: 65117}
# AsBFW of v2_restiny_t (u16), v2_resshort_t (u32), v2_resint_t (u64)
AS_BFW = {TBL_RESTINY: (1, 3, 29, 233), TBL_RESSHORT: (1, 3, 61, 463, 7785, 63877),
          TBL_RESINT: (1, 3, 125, 881, 16089)}
KIND_SKIP, KIND_INT, KIND_RES, KIND_STRING, KIND_FIXED, KIND_CHAR = range(6)


def minbfw_a(tbl_type: int, min_bfw: int) -> Optional[int]:
    """AsBFW->at(min(AsBFW->size(), minBFW)); None where at() throws."""
    tab = AS_BFW[tbl_type]
    i = min(len(tab), min_bfw)
    return tab[i] if i < len(tab) else None


_lib = None


def _load():
    global _lib
    if _lib is None:
        import os
        path = PORT_LIB if os.path.exists(PORT_LIB) else build_port()
        lib = ctypes.CDLL(path)
        lib.orc_tbl_parse.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_uint32),
                                      ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_void_p),
                                      ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64),
                                      ctypes.POINTER(ctypes.c_uint64)]
        lib.orc_reencode.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64,
                                     ctypes.c_uint64]
        lib.orc_reencode.restype = None
        _lib = lib
    return _lib


def tbl_parse(text: bytes, kinds: Sequence[int], widths: Sequence[int], As: Sequence[int], delim: str = "|",
              ignore_more_data: bool = True, max_lines: Optional[int] = None
              ) -> Tuple[int, int, int, List[np.ndarray]]:
    """Parse ``text``; returns (status, lines, bad_line, raw column bytes)."""
    lib = _load()
    n = len(kinds)
    rows = text.count(b"\n") + (1 if text and not text.endswith(b"\n") else 0)
    outs = [np.zeros(max(rows, 1) * int(w), dtype=np.uint8) for w in widths]
    ptrs = (ctypes.c_void_p * n)(*[o.ctypes.data for o in outs])
    lines, bad = ctypes.c_uint64(0), ctypes.c_uint64(0)
    rc = lib.orc_tbl_parse(text, len(text), delim.encode(), int(ignore_more_data), n,
                           (ctypes.c_int32 * n)(*kinds), (ctypes.c_uint32 * n)(*widths),
                           (ctypes.c_uint64 * n)(*[int(a) for a in As]), ptrs,
                           ctypes.c_uint64(rows if max_lines is None else max_lines), ctypes.byref(lines),
                           ctypes.byref(bad))
    stored = min(int(lines.value), rows if max_lines is None else max_lines)
    return rc, int(lines.value), int(bad.value), [o[: stored * int(w)] for o, w in zip(outs, widths)]


def reencode(values: np.ndarray, width: int, a_old: int, a_new: int) -> np.ndarray:
    """Re-encoded copy of ``values`` (unsigned, ``width`` bytes each)."""
    out = np.ascontiguousarray(values, dtype={2: np.uint16, 4: np.uint32, 8: np.uint64}[width]).copy()
    _load().orc_reencode(out.ctypes.data, out.size, width, a_old, a_new)
    return out
