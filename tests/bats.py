"""Seeded synthetic BATs for the parity tests (host numpy arrays)."""
from __future__ import annotations

import numpy as np

from ahead_b200.model import (ENCODED, NP_DTYPE, RESOID, UNENC_MAX, VOID, WIDTH, Bat, Col, an_meta,
                              void_col)

BASE_MAX = {6: 0xFF, 7: 0xFFFF, 8: 0xFFFFFFFF, 9: 0x00FFFFFFFFFFFFFF, 10: 0xFFFFFFFF}


def flip_bits(arr: np.ndarray, nflips: int, rng: np.random.Generator) -> np.ndarray:
    """Flip one seeded bit in each of ``nflips`` distinct seeded rows (in place)."""
    n = len(arr)
    if n == 0 or nflips == 0:
        return np.zeros(0, dtype=np.int64)
    rows = rng.choice(n, size=min(nflips, n), replace=False)
    bits = rng.integers(0, arr.dtype.itemsize * 8, size=len(rows))
    one = np.array(1, dtype=arr.dtype)
    for r, b in zip(rows, bits):
        arr[r] ^= (one << np.array(b, dtype=arr.dtype))
    return np.sort(rows)


def encoded_col(t: int, values, A=None, seqbase: int = 0) -> Bat:
    m = an_meta(t, A)
    vals = np.asarray(values, dtype=np.uint64)
    codes = (vals * np.uint64(m["A"])) & np.uint64((1 << (8 * WIDTH[t])) - 1 if WIDTH[t] < 8 else 0xFFFFFFFFFFFFFFFF)
    arr = codes.astype(NP_DTYPE[WIDTH[t]])
    return Bat(void_col(seqbase), Col(t, arr, m["A"], m["Ainv"], m["unenc_max"], 0), len(arr))


def random_encoded(t: int, n: int, lo: int, hi: int, rng, nflips: int = 0, A=None, seqbase: int = 0):
    vals = rng.integers(lo, hi, size=n, dtype=np.uint64) if n else np.zeros(0, np.uint64)
    b = encoded_col(t, vals, A, seqbase)
    rows = flip_bits(b.tail.data, nflips, rng)
    return b, vals, rows


def oid_list(oids, A: int = 65117, seqbase: int = 0) -> Bat:
    """A (void, resoid) BAT of AN-coded OIDs (a selection vector)."""
    m = an_meta(RESOID, A)
    o = (np.asarray(oids, dtype=np.uint64) * np.uint64(A)).astype(np.uint64)
    return Bat(void_col(seqbase), Col(RESOID, o, m["A"], m["Ainv"], m["unenc_max"], 0), len(o))
