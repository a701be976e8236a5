"""BAT data model and AN-code parameters.

A BAT is a pair of equally long columns (head, tail).  Each column carries an
AHEAD value type and the AN metadata of the reference's ColumnMetaData
(include/column_storage/ColumnMetaData.hpp:150-200).  ``Col.data`` is a numpy
array for host columns or a torch tensor for device columns; it is ``None``
for a VOID column, whose value at row i is the oid_t ``(seqbase + i) mod 2^32``.

The ctypes mirror of ``include/ahead_types.h`` lives here too, so the GPU
library wrapper and the CPU oracle share one description of the ABI.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Any, Optional

import numpy as np

# ---------------------------------------------------------------- value types
VOID, TINYINT, SHORTINT, INT, BIGINT, OID = 0, 1, 2, 3, 4, 5
RESTINY, RESSHORT, RESINT, RESBIGINT, RESOID = 6, 7, 8, 9, 10
# fixed-width string slots (v2_str_t), taken and returned only by the string selections
STR = 16

TYPE_NAMES = {
    VOID: "void", TINYINT: "tinyint", SHORTINT: "shortint", INT: "int", BIGINT: "bigint",
    OID: "oid", RESTINY: "restiny", RESSHORT: "resshort", RESINT: "resint",
    RESBIGINT: "resbigint", RESOID: "resoid",
}
# storage width in bytes (include/util/v2types.hpp:242-253, resilience.hpp:36-42)
WIDTH = {VOID: 4, TINYINT: 1, SHORTINT: 2, INT: 4, BIGINT: 8, OID: 4,
         RESTINY: 2, RESSHORT: 4, RESINT: 8, RESBIGINT: 8, RESOID: 8}
NP_DTYPE = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}
ENCODED = {RESTINY, RESSHORT, RESINT, RESBIGINT, RESOID}
# TypeMap<T>::v2_encoded_t (resilience.hpp:278-432)
ENCODED_TYPE = {VOID: RESOID, TINYINT: RESTINY, SHORTINT: RESSHORT, INT: RESINT,
                BIGINT: RESBIGINT, OID: RESOID, RESTINY: RESTINY, RESSHORT: RESSHORT,
                RESINT: RESINT, RESBIGINT: RESBIGINT, RESOID: RESOID}
UNENCODED_TYPE = {RESTINY: TINYINT, RESSHORT: SHORTINT, RESINT: INT, RESBIGINT: BIGINT,
                  RESOID: OID}

# predicates / combiners / hash side / arithmetic (include/ahead_types.h)
CMP_NONE, LT, LE, EQ, NE, GE, GT = 0, 1, 2, 3, 4, 5, 6
AND, OR = 0, 1
HASH_LEFT, HASH_RIGHT = 0, 1
ADD, SUB, MUL, DIV = 0, 1, 2, 3

# status codes
OK, BAD_ARG, SIZE_MISMATCH, CAPACITY, TIMEOUT, CUDA_ERROR, NO_MEMORY, UNSUPPORTED = range(8)
STATUS_NAMES = ["OK", "BAD_ARG", "SIZE_MISMATCH", "CAPACITY", "TIMEOUT", "CUDA_ERROR",
                "NO_MEMORY", "UNSUPPORTED"]

# ---------------------------------------------------------- AN parameters
# A tables of the reference (include/util/resilience.hpp:56-109); the
# inverses are recomputed here with Python's modular inverse.
AS_RESTINY = (1, 3, 7, 13, 29, 59, 115, 233)
AS_RESSHORT = (1, 3, 7, 13, 29, 61, 119, 233, 463, 947, 1939, 3349, 7785, 14781, 28183, 63877)
AS_RESINT = (1, 3, 7, 13, 29, 61, 125, 225, 445, 881, 2029, 3973, 7841, 16089, 32417, 65117)
AS_RESOID = AS_RESINT
AS_BFW_RESOID = (AS_RESINT[0], AS_RESINT[1], AS_RESINT[6], AS_RESINT[9], AS_RESINT[13])
# default A_OID of the operators: last entry of v2_resoid_t::AsBFW (OperatorsAN.hpp:38)
AOID_DEFAULT = AS_BFW_RESOID[-1]  # 16089
# default AOID of groupbyAN / aggregate: largest resoid A (OperatorsAN.hpp:113-136)
A_RESOID_MAX = AS_RESINT[-1]  # 65117
# UNENC_MAX_U (lib/util/resilience.cpp:47-71)
UNENC_MAX = {RESTINY: 0xFF, RESSHORT: 0xFFFF, RESINT: 0xFFFFFFFF,
             RESBIGINT: 0x00FFFFFFFFFFFFFF, RESOID: 0x00FFFFFFFFFFFFFF}
# A per width chosen at table load (lib/column_storage/Transaction.cpp:357-376)
A_LOAD = {RESTINY: 233, RESSHORT: 63877, RESINT: 65117}


def ainv(a: int, bits: int) -> int:
    """Inverse of odd ``a`` modulo 2**bits."""
    return pow(a, -1, 1 << bits)


def an_meta(t: int, A: Optional[int] = None) -> dict:
    """AN metadata dict for encoded type ``t`` with multiplier ``A``."""
    if t not in ENCODED:
        return dict(A=1, Ainv=1, unenc_max=0)
    if A is None:
        A = A_LOAD.get(t, A_RESOID_MAX)
    return dict(A=A, Ainv=ainv(A, 8 * WIDTH[t]), unenc_max=UNENC_MAX[t])


# ---------------------------------------------------------------- BATs
@dataclass
class Col:
    type: int
    data: Any = None
    A: int = 1
    Ainv: int = 1
    unenc_max: int = 0
    seqbase: int = 0
    # string columns (STR): the slot width in bytes, and the dictionary that
    # maps an attribute's integer code to its string (thresholds given as codes)
    width: int = 0
    names: Any = None

    def meta(self) -> dict:
        return dict(A=self.A, Ainv=self.Ainv, unenc_max=self.unenc_max, seqbase=self.seqbase)


@dataclass
class Bat:
    head: Col
    tail: Col
    count: int

    def mirror_head(self) -> "Bat":
        return Bat(self.head, self.head, self.count)

    def reverse(self) -> "Bat":
        return Bat(self.tail, self.head, self.count)

    def clear_head(self) -> "Bat":
        return Bat(Col(VOID), self.tail, self.count)


def void_col(seqbase: int = 0) -> Col:
    return Col(VOID, None, 1, 1, 0, seqbase)


def host_bat(tail_type: int, values, seqbase: int = 0, A: Optional[int] = None) -> Bat:
    """A (void, tail) BAT over host values, AN metadata filled for encoded tails."""
    arr = np.ascontiguousarray(values, dtype=NP_DTYPE[WIDTH[tail_type]])
    m = an_meta(tail_type, A)
    return Bat(void_col(seqbase), Col(tail_type, arr, m["A"], m["Ainv"], m["unenc_max"], 0), len(arr))


@dataclass
class ErrVec:
    """An error-position vector; ``None``-like when ``present`` is False."""
    values: Optional[np.ndarray]
    present: bool = True

    def __len__(self):
        return 0 if self.values is None else len(self.values)


# ------------------------------------------------------------ ctypes mirror
class CCol(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("type", ctypes.c_int32), ("A", ctypes.c_uint32),
                ("Ainv", ctypes.c_uint64), ("unenc_max", ctypes.c_uint64),
                ("seqbase", ctypes.c_uint64)]


class CBat(ctypes.Structure):
    _fields_ = [("head", CCol), ("tail", CCol), ("count", ctypes.c_uint64)]


class CErrVec(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("capacity", ctypes.c_uint64),
                ("count", ctypes.c_uint64), ("present", ctypes.c_int32),
                ("_pad", ctypes.c_int32)]


def ccol(c: Col, ptr: int) -> CCol:
    return CCol(ptr or None, c.type, c.A & 0xFFFFFFFF, c.Ainv & 0xFFFFFFFFFFFFFFFF,
                c.unenc_max & 0xFFFFFFFFFFFFFFFF, c.seqbase & 0xFFFFFFFFFFFFFFFF)


def col_from_c(c: CCol, data) -> Col:
    return Col(c.type, data, c.A, c.Ainv, c.unenc_max, c.seqbase)
