"""TEST INFRASTRUCTURE ONLY: numpy-level access to the CPU oracle.

``Oracle("port")`` loads the plain-C restatement (oracle/liban_oracle.so);
``Oracle("reference")`` loads the reference's own scalar operators compiled
from the reference sources (oracle/_ref/libahead_ref.so).  Both implement
oracle/an_oracle.h.  Only tests, the smoke check and the CPU-baseline leg of
bench.py use this module, and only to check or time the CPU path.

Each method mirrors one reference operator and returns host ``Bat`` objects
and ``ErrVec`` error-position vectors.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import List, Optional, Tuple

import numpy as np

from ahead_b200.model import (NP_DTYPE, VOID, WIDTH, Bat, CBat, CErrVec, Col, ErrVec, ccol,
                              col_from_c, CAPACITY, OK, STATUS_NAMES)

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "liban_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libahead_ref.so")


class OracleError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what}: {STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else status}")
        self.status = status


def build_port() -> str:
    subprocess.run(["make", "-s", "-C", HERE, "liban_oracle.so"], check=True)
    return PORT_LIB


def build_reference() -> Optional[str]:
    """Compile the reference's scalar operators (only where the reference tree exists)."""
    ref = os.environ.get("AHEAD_REFERENCE", "/root/reference")
    if not os.path.isdir(os.path.join(ref, "lib", "column_operators")):
        return REF_LIB if os.path.exists(REF_LIB) else None
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE={ref}"], check=True)
    return REF_LIB


def _ptr(a) -> int:
    return 0 if a is None else a.ctypes.data


class _Keep:
    """Keeps numpy buffers alive while a C call runs."""

    def __init__(self):
        self.items = []

    def __call__(self, x):
        self.items.append(x)
        return x


def _in_bat(b: Bat, keep: _Keep) -> CBat:
    h = b.head.data if b.head.type != VOID else None
    t = b.tail.data if b.tail.type != VOID else None
    if h is not None:
        h = keep(np.ascontiguousarray(h, dtype=NP_DTYPE[WIDTH[b.head.type]]))
    if t is not None:
        t = keep(np.ascontiguousarray(t, dtype=NP_DTYPE[WIDTH[b.tail.type]]))
    return CBat(ccol(b.head, _ptr(h)), ccol(b.tail, _ptr(t)), b.count)


class _Out:
    def __init__(self, cap: int):
        self.cap = max(int(cap), 1)
        self.h = np.zeros(self.cap, dtype=np.uint64)
        self.t = np.zeros(self.cap, dtype=np.uint64)
        self.c = CBat()
        self.c.head.data = self.h.ctypes.data
        self.c.tail.data = self.t.ctypes.data

    def bat(self) -> Bat:
        n = int(self.c.count)

        def col(cc, buf):
            if cc.type == VOID or not cc.data:
                return col_from_c(cc, None)
            dt = NP_DTYPE[WIDTH[cc.type]]
            return col_from_c(cc, buf.view(dt)[:n].copy())

        return Bat(col(self.c.head, self.h), col(self.c.tail, self.t), n)


class _Errs:
    def __init__(self, k: int, cap: int):
        self.bufs = [np.zeros(max(int(cap), 1), dtype=np.uint64) for _ in range(k)]
        self.c = (CErrVec * k)()
        for i in range(k):
            self.c[i].data = self.bufs[i].ctypes.data
            self.c[i].capacity = len(self.bufs[i])

    def need(self) -> int:
        return max(int(e.count) for e in self.c)

    def vecs(self) -> List[ErrVec]:
        out = []
        for i, e in enumerate(self.c):
            if not e.present:
                out.append(ErrVec(None, False))
            else:
                out.append(ErrVec(self.bufs[i][: int(e.count)].copy(), True))
        return out


class Oracle:
    def __init__(self, kind: str = "port"):
        self.kind = kind
        path = PORT_LIB if kind == "port" else REF_LIB
        if not os.path.exists(path):
            path = build_port() if kind == "port" else build_reference()
        if not path or not os.path.exists(path):
            raise FileNotFoundError(f"oracle library '{kind}' is not built")
        self.lib = ctypes.CDLL(path)
        self.lib.orc_ainv.restype = ctypes.c_uint64
        self.lib.orc_ainv.argtypes = [ctypes.c_uint64, ctypes.c_int]

    # -- generic driver: retry with the exact capacity when an output overflowed
    def _run(self, what, call, cap: int, nerr: int, nout: int = 1):
        while True:
            keep = _Keep()
            outs = [_Out(cap) for _ in range(nout)]
            errs = _Errs(nerr, cap)
            rc = call(keep, outs, errs)
            need = max([int(o.c.count) for o in outs] + [errs.need() if nerr else 0])
            if rc == CAPACITY or need > cap:
                cap = max(need, 1)
                continue
            if rc != OK:
                raise OracleError(rc, what)
            return outs, errs

    def ainv(self, a: int, bits: int) -> int:
        return int(self.lib.orc_ainv(a, bits))

    # -- selection
    def select_an(self, b: Bat, op1, th1, op2=0, th2=0, comb=0, aoid=16089) -> Tuple[Bat, ErrVec]:
        def call(keep, outs, errs):
            cb = _in_bat(b, keep)
            return self.lib.orc_select_an(ctypes.byref(cb), op1, ctypes.c_uint64(th1), op2, ctypes.c_uint64(th2), comb,
                                          ctypes.c_uint64(aoid), ctypes.byref(outs[0].c), ctypes.c_uint64(outs[0].cap),
                                          ctypes.byref(errs.c[0]))
        outs, errs = self._run("selectAN", call, b.count, 1)
        return outs[0].bat(), errs.vecs()[0]

    def select(self, b: Bat, op1, th1, op2=0, th2=0, comb=0) -> Bat:
        def call(keep, outs, errs):
            cb = _in_bat(b, keep)
            return self.lib.orc_select(ctypes.byref(cb), op1, ctypes.c_uint64(th1), op2, ctypes.c_uint64(th2), comb,
                                       ctypes.byref(outs[0].c), ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("select", call, b.count, 0)
        return outs[0].bat()

    # -- string selection: `strs` is a uint8 array of rows of `width` bytes
    def _select_str(self, fn, what, strs, width, seqbase, op1, th1, op2, th2, comb, dtype) -> np.ndarray:
        strs = np.ascontiguousarray(strs, dtype=np.uint8)
        count = len(strs) // width if width else 0

        def call(keep, outs, errs):
            return fn(ctypes.c_void_p(strs.ctypes.data), ctypes.c_uint64(width), ctypes.c_uint64(count),
                      ctypes.c_uint64(seqbase), op1, ctypes.c_char_p(th1), op2, ctypes.c_char_p(th2), comb,
                      ctypes.byref(outs[0].c), ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run(what, call, count, 0)
        return outs[0].h.view(dtype)[: int(outs[0].c.count)].copy()

    def select_str_an(self, strs, width, seqbase, op1, th1: bytes, op2=0, th2: bytes = b"", comb=0) -> np.ndarray:
        """selectAN over a string tail: the kept rows' resoid codes (u64)."""
        return self._select_str(self.lib.orc_select_str_an, "selectAN(str)", strs, width, seqbase, op1, th1, op2,
                                th2, comb, np.uint64)

    def select_str(self, strs, width, seqbase, op1, th1: bytes, op2=0, th2: bytes = b"", comb=0) -> np.ndarray:
        """select over a string tail: the kept rows' oid_t (u32)."""
        return self._select_str(self.lib.orc_select_str, "select(str)", strs, width, seqbase, op1, th1, op2, th2,
                                comb, np.uint32)

    # -- check / decode
    def check_an(self, b: Bat, ainv, unenc_max, aoid=16089) -> ErrVec:
        def call(keep, outs, errs):
            cb = _in_bat(b, keep)
            return self.lib.orc_check_an(ctypes.byref(cb), ctypes.c_uint64(ainv), ctypes.c_uint64(unenc_max),
                                         ctypes.c_uint64(aoid), ctypes.byref(errs.c[0]))
        _, errs = self._run("checkAN", call, b.count, 1, nout=0)
        return errs.vecs()[0]

    def decode_an(self, b: Bat, aoid=16089) -> Tuple[Bat, ErrVec]:
        def call(keep, outs, errs):
            cb = _in_bat(b, keep)
            return self.lib.orc_decode_an(ctypes.byref(cb), ctypes.c_uint64(aoid), ctypes.byref(outs[0].c),
                                          ctypes.c_uint64(outs[0].cap), ctypes.byref(errs.c[0]))
        outs, errs = self._run("decodeAN", call, b.count, 1)
        return outs[0].bat(), errs.vecs()[0]

    def check_and_decode_an(self, b: Bat, aoid=16089) -> Tuple[Bat, ErrVec, ErrVec]:
        def call(keep, outs, errs):
            cb = _in_bat(b, keep)
            return self.lib.orc_check_and_decode_an(ctypes.byref(cb), ctypes.c_uint64(aoid), ctypes.byref(outs[0].c),
                                                    ctypes.c_uint64(outs[0].cap), ctypes.byref(errs.c[0]),
                                                    ctypes.byref(errs.c[1]))
        outs, errs = self._run("checkAndDecodeAN", call, b.count, 2)
        v = errs.vecs()
        return outs[0].bat(), v[0], v[1]

    def encode_an(self, b: Bat, A) -> Bat:
        def call(keep, outs, errs):
            cb = _in_bat(b, keep)
            return self.lib.orc_encode_an(ctypes.byref(cb), ctypes.c_uint64(A), ctypes.byref(outs[0].c),
                                          ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("encodeAN", call, b.count, 0)
        return outs[0].bat()

    # -- joins
    def hashjoin_an(self, l: Bat, r: Bat, reenc_head=False, ah1r=1, ah1invr=1, reenc_tail=False, at2r=1,
                    at2invr=1, side=1, aoid=16089) -> Tuple[Bat, List[ErrVec]]:
        def call(keep, outs, errs):
            cl, cr = _in_bat(l, keep), _in_bat(r, keep)
            return self.lib.orc_hashjoin_an(ctypes.byref(cl), ctypes.byref(cr), int(reenc_head), ctypes.c_uint64(ah1r),
                                            ctypes.c_uint64(ah1invr), int(reenc_tail), ctypes.c_uint64(at2r),
                                            ctypes.c_uint64(at2invr), side, ctypes.c_uint64(aoid),
                                            ctypes.byref(outs[0].c), ctypes.c_uint64(outs[0].cap), errs.c)
        outs, errs = self._run("hashjoinAN", call, max(l.count, r.count), 4)
        return outs[0].bat(), errs.vecs()

    def hashjoin_str_an(self, l: Bat, r: Bat, r_strs, width: int, reenc_head=False, ah1r=1, ah1invr=1, side=1,
                        aoid=16089):
        """hashjoinAN with a string right tail: (head column, the matched
        `width`-byte slots as an (n, width) uint8 array, [H1, T1, H2, T2]
        error vectors)."""
        r_strs = np.ascontiguousarray(r_strs, dtype=np.uint8)
        cap = max(1, l.count * max(1, r.count))
        cap = min(cap, 1 << 20)
        while True:
            keep = _Keep()
            out = _Out(cap)
            sbuf = np.zeros(cap * width + 1, np.uint8)
            out.c.tail.data = sbuf.ctypes.data
            errs = _Errs(4, max(l.count, r.count, 1))
            rc = self.lib.orc_hashjoin_str_an(ctypes.byref(_in_bat(l, keep)), ctypes.byref(_in_bat(r, keep)),
                                              ctypes.c_void_p(r_strs.ctypes.data), ctypes.c_uint64(width),
                                              int(bool(reenc_head)), ctypes.c_uint64(ah1r), ctypes.c_uint64(ah1invr),
                                              side, ctypes.c_uint64(aoid), ctypes.byref(out.c), ctypes.c_uint64(cap),
                                              errs.c)
            n = int(out.c.count)
            if rc == CAPACITY or n > cap:
                cap = max(n, 1)
                continue
            if rc != OK:
                raise OracleError(rc, "hashjoinAN(str)")
            head = col_from_c(out.c.head, out.h.view(NP_DTYPE[WIDTH[out.c.head.type]])[:n].copy())
            return head, sbuf[: n * width].reshape(n, width).copy(), errs.vecs()

    def hashjoin(self, l: Bat, r: Bat, side=1) -> Bat:
        def call(keep, outs, errs):
            cl, cr = _in_bat(l, keep), _in_bat(r, keep)
            return self.lib.orc_hashjoin(ctypes.byref(cl), ctypes.byref(cr), side, ctypes.byref(outs[0].c),
                                         ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("hashjoin", call, max(l.count, r.count), 0)
        return outs[0].bat()

    def matchjoin_an(self, a: Bat, b: Bat, reenc=False, ah1r=0, ah1invr=0, at2r=0, at2invr=0,
                     aoid=16089) -> Tuple[Bat, List[ErrVec]]:
        def call(keep, outs, errs):
            ca, cb = _in_bat(a, keep), _in_bat(b, keep)
            return self.lib.orc_matchjoin_an(ctypes.byref(ca), ctypes.byref(cb), int(reenc), ctypes.c_uint64(ah1r),
                                             ctypes.c_uint64(ah1invr), ctypes.c_uint64(at2r), ctypes.c_uint64(at2invr),
                                             ctypes.c_uint64(aoid), ctypes.byref(outs[0].c),
                                             ctypes.c_uint64(outs[0].cap), errs.c)
        outs, errs = self._run("matchjoinAN", call, max(a.count, b.count) * 2 + 1, 4)
        return outs[0].bat(), errs.vecs()

    def matchjoin(self, a: Bat, b: Bat) -> Bat:
        def call(keep, outs, errs):
            ca, cb = _in_bat(a, keep), _in_bat(b, keep)
            return self.lib.orc_matchjoin(ctypes.byref(ca), ctypes.byref(cb), ctypes.byref(outs[0].c),
                                          ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("matchjoin", call, max(a.count, b.count), 0)
        return outs[0].bat()

    def fetchjoin_an(self, a: Bat, b: Bat, reenc=False, atr=1, atrinv=1, aoid=16089) -> Tuple[Bat, List[ErrVec]]:
        def call(keep, outs, errs):
            ca, cb = _in_bat(a, keep), _in_bat(b, keep)
            return self.lib.orc_fetchjoin_an(ctypes.byref(ca), ctypes.byref(cb), int(reenc), ctypes.c_uint64(atr),
                                             ctypes.c_uint64(atrinv), ctypes.c_uint64(aoid), ctypes.byref(outs[0].c),
                                             ctypes.c_uint64(outs[0].cap), errs.c)
        outs, errs = self._run("fetchjoinAN", call, a.count, 2)
        return outs[0].bat(), errs.vecs()

    def fetchjoin(self, a: Bat, b: Bat) -> Bat:
        def call(keep, outs, errs):
            ca, cb = _in_bat(a, keep), _in_bat(b, keep)
            return self.lib.orc_fetchjoin(ctypes.byref(ca), ctypes.byref(cb), ctypes.byref(outs[0].c),
                                          ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("fetchjoin", call, a.count, 0)
        return outs[0].bat()

    # -- grouping and aggregation
    def groupby_an(self, b: Bat, aoid=65117, aoidinv=0x3E36D3BC8D9BC5F5) -> Tuple[Bat, Bat, List[ErrVec]]:
        def call(keep, outs, errs):
            cb = _in_bat(b, keep)
            return self.lib.orc_groupby_an(ctypes.byref(cb), ctypes.c_uint64(aoid), ctypes.c_uint64(aoidinv),
                                           ctypes.byref(outs[0].c), ctypes.byref(outs[1].c),
                                           ctypes.c_uint64(outs[0].cap), errs.c)
        outs, errs = self._run("groupbyAN", call, b.count, 2, nout=2)
        return outs[0].bat(), outs[1].bat(), errs.vecs()

    def groupby2_an(self, b: Bat, grouping: Bat, ngroups: int, aoid=65117,
                    aoidinv=0x3E36D3BC8D9BC5F5) -> Tuple[Bat, Bat, List[ErrVec]]:
        def call(keep, outs, errs):
            cb, cg = _in_bat(b, keep), _in_bat(grouping, keep)
            return self.lib.orc_groupby2_an(ctypes.byref(cb), ctypes.byref(cg), ctypes.c_uint64(ngroups),
                                            ctypes.c_uint64(aoid), ctypes.c_uint64(aoidinv), ctypes.byref(outs[0].c),
                                            ctypes.byref(outs[1].c), ctypes.c_uint64(outs[0].cap), errs.c)
        outs, errs = self._run("groupbyAN2", call, b.count, 3, nout=2)
        return outs[0].bat(), outs[1].bat(), errs.vecs()

    def fetchjoin_str_an(self, a: Bat, strs, width: int, aoid=16089) -> Tuple[np.ndarray, List[ErrVec]]:
        """fetchjoinAN with a string tail: the fetched slots as an (n, width)
        uint8 array, and [vec1, vec2] (vec2 not present)."""
        strs = np.ascontiguousarray(strs, dtype=np.uint8)
        count = len(strs) if strs.ndim == 2 else len(strs) // width
        cap = max(a.count, 1)
        while True:
            keep = _Keep()
            out = np.zeros(cap * width, np.uint8)
            n = ctypes.c_uint64(0)
            errs = _Errs(2, max(a.count, 1))
            rc = self.lib.orc_fetchjoin_str_an(ctypes.byref(_in_bat(a, keep)), ctypes.c_void_p(strs.ctypes.data),
                                               ctypes.c_uint64(width), ctypes.c_uint64(count), ctypes.c_uint64(aoid),
                                               ctypes.c_void_p(out.ctypes.data), ctypes.c_uint64(cap),
                                               ctypes.byref(n), errs.c)
            if rc == CAPACITY:
                cap = max(int(n.value), 1)
                continue
            if rc != OK:
                raise OracleError(rc, "fetchjoinAN(str)")
            return out[: int(n.value) * width].reshape(int(n.value), width).copy(), errs.vecs()

    def groupby2_str_an(self, strs, width: int, grouping: Bat, ngroups: int, aoid=65117,
                        aoidinv=0x3E36D3BC8D9BC5F5, seqbase: int = 0) -> Tuple[Bat, Bat, List[ErrVec]]:
        """groupbyAN binary over a string tail (a void head with `seqbase`)."""
        strs = np.ascontiguousarray(strs, dtype=np.uint8)
        count = len(strs) if strs.ndim == 2 else len(strs) // width

        def call(keep, outs, errs):
            cg = _in_bat(grouping, keep)
            return self.lib.orc_groupby2_str_an(ctypes.c_void_p(strs.ctypes.data), ctypes.c_uint64(width),
                                                ctypes.c_uint64(count), ctypes.c_uint64(seqbase), ctypes.byref(cg),
                                                ctypes.c_uint64(ngroups), ctypes.c_uint64(aoid),
                                                ctypes.c_uint64(aoidinv), ctypes.byref(outs[0].c),
                                                ctypes.byref(outs[1].c), ctypes.c_uint64(outs[0].cap), errs.c)
        outs, errs = self._run("groupbyAN2(str)", call, count, 3, nout=2)
        return outs[0].bat(), outs[1].bat(), errs.vecs()

    def fetchjoin_str(self, a: Bat, strs, width: int) -> np.ndarray:
        """fetchjoin over a string tail (unencoded): the fetched slots."""
        strs = np.ascontiguousarray(strs, dtype=np.uint8)
        count = len(strs) if strs.ndim == 2 else len(strs) // width
        cap = max(a.count, 1)
        while True:
            keep = _Keep()
            out = np.zeros(cap * width, np.uint8)
            n = ctypes.c_uint64(0)
            rc = self.lib.orc_fetchjoin_str(ctypes.byref(_in_bat(a, keep)), ctypes.c_void_p(strs.ctypes.data),
                                            ctypes.c_uint64(width), ctypes.c_uint64(count),
                                            ctypes.c_void_p(out.ctypes.data), ctypes.c_uint64(cap), ctypes.byref(n))
            if rc == CAPACITY:
                cap = max(int(n.value), 1)
                continue
            if rc != OK:
                raise OracleError(rc, "fetchjoin(str)")
            return out[: int(n.value) * width].reshape(int(n.value), width).copy()

    def groupby2_str(self, strs, width: int, grouping: Bat, ngroups: int, seqbase: int = 0) -> Tuple[Bat, Bat]:
        """groupby binary over a string tail (unencoded)."""
        strs = np.ascontiguousarray(strs, dtype=np.uint8)
        count = len(strs) if strs.ndim == 2 else len(strs) // width

        def call(keep, outs, errs):
            cg = _in_bat(grouping, keep)
            return self.lib.orc_groupby2_str(ctypes.c_void_p(strs.ctypes.data), ctypes.c_uint64(width),
                                             ctypes.c_uint64(count), ctypes.c_uint64(seqbase), ctypes.byref(cg),
                                             ctypes.c_uint64(ngroups), ctypes.byref(outs[0].c),
                                             ctypes.byref(outs[1].c), ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("groupby2(str)", call, count, 0, nout=2)
        return outs[0].bat(), outs[1].bat()

    def aggregate_sum_grouped_an(self, b: Bat, grouping: Bat, ngroups: int, result_type=9, ar=65117,
                                 arinv=0x3E36D3BC8D9BC5F5, aoid=65117) -> Tuple[Bat, List[ErrVec]]:
        def call(keep, outs, errs):
            cb, cg = _in_bat(b, keep), _in_bat(grouping, keep)
            return self.lib.orc_aggregate_sum_grouped_an(ctypes.byref(cb), ctypes.byref(cg), ctypes.c_uint64(ngroups),
                                                         result_type, ctypes.c_uint64(ar), ctypes.c_uint64(arinv),
                                                         ctypes.c_uint64(aoid), ctypes.byref(outs[0].c), errs.c)
        outs, errs = self._run("aggregate_sum_groupedAN", call, max(b.count, ngroups, 1), 3)
        return outs[0].bat(), errs.vecs()

    def aggregate_mul_sum_an(self, a: Bat, b: Bat, result_type=9, init=0, ra=65117,
                             rainv=0x3E36D3BC8D9BC5F5, aoid=16089) -> Tuple[int, List[ErrVec]]:
        tot = ctypes.c_uint64(0)

        def call(keep, outs, errs):
            ca, cb = _in_bat(a, keep), _in_bat(b, keep)
            return self.lib.orc_aggregate_mul_sum_an(ctypes.byref(ca), ctypes.byref(cb), result_type,
                                                     ctypes.c_uint64(init), ctypes.c_uint64(ra), ctypes.c_uint64(rainv),
                                                     ctypes.c_uint64(aoid), ctypes.byref(tot), errs.c)
        _, errs = self._run("aggregate_mul_sumAN", call, max(a.count, b.count), 2, nout=0)
        return int(tot.value), errs.vecs()

    def aggregate_mul_sum(self, a: Bat, b: Bat, result_type=4, init=0) -> int:
        tot = ctypes.c_uint64(0)
        keep = _Keep()
        ca, cb = _in_bat(a, keep), _in_bat(b, keep)
        rc = self.lib.orc_aggregate_mul_sum(ctypes.byref(ca), ctypes.byref(cb), result_type, ctypes.c_uint64(init),
                                            ctypes.byref(tot))
        if rc != OK:
            raise OracleError(rc, "aggregate_mul_sum")
        return int(tot.value)

    # -- unencoded twins
    def groupby(self, b: Bat) -> Tuple[Bat, Bat]:
        def call(keep, outs, errs):
            cb = _in_bat(b, keep)
            return self.lib.orc_groupby(ctypes.byref(cb), ctypes.byref(outs[0].c), ctypes.byref(outs[1].c),
                                        ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("groupby", call, b.count, 0, nout=2)
        return outs[0].bat(), outs[1].bat()

    def groupby2(self, b: Bat, grouping: Bat, ngroups: int) -> Tuple[Bat, Bat]:
        def call(keep, outs, errs):
            cb, cg = _in_bat(b, keep), _in_bat(grouping, keep)
            return self.lib.orc_groupby2(ctypes.byref(cb), ctypes.byref(cg), ctypes.c_uint64(ngroups),
                                         ctypes.byref(outs[0].c), ctypes.byref(outs[1].c), ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("groupby2", call, b.count, 0, nout=2)
        return outs[0].bat(), outs[1].bat()

    def aggregate_sum_grouped(self, b: Bat, grouping: Bat, ngroups: int, result_type=4) -> Bat:
        def call(keep, outs, errs):
            cb, cg = _in_bat(b, keep), _in_bat(grouping, keep)
            return self.lib.orc_aggregate_sum_grouped(ctypes.byref(cb), ctypes.byref(cg), ctypes.c_uint64(ngroups),
                                                      result_type, ctypes.byref(outs[0].c))
        outs, _ = self._run("aggregate_sum_grouped", call, max(b.count, ngroups, 1), 0)
        return outs[0].bat()

    def aggregate_sum(self, b: Bat, result_type=4) -> int:
        tot = ctypes.c_uint64(0)
        keep = _Keep()
        cb = _in_bat(b, keep)
        rc = self.lib.orc_aggregate_sum(ctypes.byref(cb), result_type, ctypes.byref(tot))
        if rc != OK:
            raise OracleError(rc, "aggregate_sum")
        return int(tot.value)

    def arithmetic(self, op, result_type, a: Bat, b: Bat) -> Bat:
        def call(keep, outs, errs):
            ca, cb = _in_bat(a, keep), _in_bat(b, keep)
            return self.lib.orc_arithmetic(op, result_type, ctypes.byref(ca), ctypes.byref(cb), ctypes.byref(outs[0].c))
        outs, _ = self._run("arithmetic", call, max(a.count, 1), 0)
        return outs[0].bat()

    def arithmetic_an(self, op, result_type, a: Bat, b: Bat, ar, arinv, aoid=16089) -> Tuple[Bat, List[ErrVec]]:
        def call(keep, outs, errs):
            ca, cb = _in_bat(a, keep), _in_bat(b, keep)
            return self.lib.orc_arithmetic_an(op, result_type, ctypes.byref(ca), ctypes.byref(cb), ctypes.c_uint64(ar),
                                              ctypes.c_uint64(arinv), ctypes.c_uint64(aoid), ctypes.byref(outs[0].c),
                                              errs.c)
        outs, errs = self._run("arithmeticAN", call, max(a.count, 1), 4)
        return outs[0].bat(), errs.vecs()
