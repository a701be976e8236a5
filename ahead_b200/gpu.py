"""Host-side mirror of the reference's operator API over libahead_b200.so.

Every method calls one ``ahead_gpu_*`` entry point of ``include/ahead_gpu.h``
and keeps the reference operator's name and argument meaning
(include/column_operators/OperatorsAN.hpp, Operators.hpp of the reference):
BATs in; BATs, sums and error-position vectors out.  Device memory comes from
torch (plumbing only); all computation happens in the library's sm_100a
kernels.  There is no CPU path: without the library or a CUDA device every
call raises.
"""
from __future__ import annotations

import ctypes
import sys
import os
from typing import List, Optional, Tuple

import numpy as np

from .model import (CAPACITY, NP_DTYPE, OK, STATUS_NAMES, STR, VOID, WIDTH, Bat, CBat, CErrVec, Col, ErrVec,
                    ccol, col_from_c)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libahead_b200.so")

_lib = None


class AheadError(RuntimeError):
    def __init__(self, status: int, what: str, detail: str = ""):
        name = STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else str(status)
        super().__init__(f"{what}: {name}{(' (' + detail + ')') if detail else ''}")
        self.status = status


def load_library():
    """Load libahead_b200.so (built in-tree by __graft_entry__.build())."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build the CUDA library first (no CPU fallback exists)")
    lib = ctypes.CDLL(LIB_PATH)
    lib.ahead_ctx_create.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    lib.ahead_ctx_destroy.argtypes = [ctypes.c_void_p]
    lib.ahead_ctx_last_error.argtypes = [ctypes.c_void_p]
    lib.ahead_ctx_last_error.restype = ctypes.c_char_p
    lib.ahead_ctx_launches.argtypes = [ctypes.c_void_p]
    lib.ahead_ctx_launches.restype = ctypes.c_uint64
    lib.ahead_ctx_stream.argtypes = [ctypes.c_void_p]
    lib.ahead_ctx_stream.restype = ctypes.c_void_p
    lib.ahead_ctx_stream.argtypes = [ctypes.c_void_p]
    lib.ahead_ctx_stream.restype = ctypes.c_void_p
    _lib = lib
    return lib


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("no CUDA device: ahead_b200 has no CPU fallback")
    return torch


def to_device(b: Bat, device: str = "cuda") -> Bat:
    """Copy a host BAT (numpy columns) into device memory."""
    torch = _torch()

    def col(c: Col) -> Col:
        if c.type == VOID or c.data is None:
            return Col(c.type, None, c.A, c.Ainv, c.unenc_max, c.seqbase)
        if c.type == STR:  # fixed-width string slots
            t = torch.from_numpy(np.ascontiguousarray(c.data, dtype=np.uint8).reshape(-1).copy()).to(device)
            return Col(STR, t, c.A, c.Ainv, c.unenc_max, c.seqbase, c.width, c.names)
        a = np.ascontiguousarray(c.data, dtype=NP_DTYPE[WIDTH[c.type]])
        t = torch.from_numpy(a.view(np.uint8).copy()).to(device)
        return Col(c.type, t, c.A, c.Ainv, c.unenc_max, c.seqbase)

    return Bat(col(b.head), col(b.tail), b.count)


def to_host(b: Bat) -> Bat:
    """Copy a device BAT back into numpy arrays of the column types."""

    def col(c: Col) -> Col:
        if c.type == VOID or c.data is None:
            return Col(c.type, None, c.A, c.Ainv, c.unenc_max, c.seqbase)
        w = WIDTH[c.type]
        raw = c.data[: b.count * w].cpu().numpy() if hasattr(c.data, "cpu") else np.asarray(c.data)
        return Col(c.type, raw.view(NP_DTYPE[w])[: b.count].copy(), c.A, c.Ainv, c.unenc_max, c.seqbase)

    return Bat(col(b.head), col(b.tail), b.count)


def err_to_host(e: ErrVec) -> ErrVec:
    if not e.present or e.values is None:
        return ErrVec(None, e.present) if not e.present else ErrVec(np.zeros(0, np.uint64), True)
    v = e.values
    if hasattr(v, "cpu"):
        v = v.cpu().numpy().view(np.uint64)
    return ErrVec(np.asarray(v, dtype=np.uint64).copy(), True)


def _ptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


def _in_bat(b: Bat) -> CBat:
    return CBat(ccol(b.head, _ptr(b.head.data) if b.head.type != VOID else 0),
                ccol(b.tail, _ptr(b.tail.data) if b.tail.type != VOID else 0), b.count)


class _Out:
    def __init__(self, torch, cap: int):
        self.cap = max(int(cap), 1)
        self.h = torch.empty(self.cap * 8, dtype=torch.uint8, device="cuda")
        self.t = torch.empty(self.cap * 8, dtype=torch.uint8, device="cuda")
        self.c = CBat()
        self.c.head.data = self.h.data_ptr()
        self.c.tail.data = self.t.data_ptr()

    def bat(self) -> Bat:
        n = int(self.c.count)

        def col(cc, buf):
            if cc.type == VOID or not cc.data:
                return col_from_c(cc, None)
            used = buf[: n * WIDTH[cc.type]]
            # a result far below its capacity is moved out, so the capacity-sized
            # buffer does not stay alive with it
            return col_from_c(cc, used.clone() if 4 * used.numel() < buf.numel() else used)

        return Bat(col(self.c.head, self.h), col(self.c.tail, self.t), n)


class _Errs:
    def __init__(self, torch, k: int, cap: int):
        self.bufs = [torch.empty(max(int(cap), 1) * 8, dtype=torch.uint8, device="cuda") for _ in range(k)]
        self.c = (CErrVec * k)()
        for i in range(k):
            self.c[i].data = self.bufs[i].data_ptr()
            self.c[i].capacity = max(int(cap), 1)

    def need(self) -> int:
        return max([int(e.count) for e in self.c] + [0])

    def vecs(self) -> List[ErrVec]:
        out = []
        for i, e in enumerate(self.c):
            if not e.present:
                out.append(ErrVec(None, False))
            else:
                out.append(ErrVec(self.bufs[i][: int(e.count) * 8], True))
        return out


class GpuOps:
    """One library context (device + stream + scratch arena)."""

    def __init__(self, device: int = 0):
        self.torch = _torch()
        self.lib = load_library()
        self.torch.cuda.set_device(device)
        stream = self.torch.cuda.current_stream(device)
        self.ctx = ctypes.c_void_p()
        rc = self.lib.ahead_ctx_create(device, ctypes.c_void_p(stream.cuda_stream), ctypes.byref(self.ctx))
        if rc != OK:
            raise AheadError(rc, "ahead_ctx_create")

    def close(self):
        if self.ctx:
            self.lib.ahead_ctx_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self, _finalizing=sys.is_finalizing):  # bound now: module globals may be gone at exit
        if _finalizing():  # the CUDA runtime may be gone; the process frees everything
            return
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self) -> int:
        return int(self.lib.ahead_ctx_launches(self.ctx))

    def stream(self):
        """The CUDA stream this context launches on, as a torch stream (for
        events that time the library's kernels)."""
        return self.torch.cuda.ExternalStream(int(self.lib.ahead_ctx_stream(self.ctx) or 0))

    def _check(self, rc: int, what: str):
        if rc != OK:
            raise AheadError(rc, what, self.lib.ahead_ctx_last_error(self.ctx).decode())

    def _run(self, what, call, cap: int, nerr: int, nout: int = 1):
        """Run an operator with outputs of `cap` rows and error vectors of a
        small first capacity (detected errors are rare); on AHEAD_CAPACITY the
        call is repeated with the sizes it reported."""
        torch = self.torch
        ecap = min(max(int(cap), 1), 1 << 16)
        while True:
            outs = [_Out(torch, cap) for _ in range(nout)]
            errs = _Errs(torch, nerr, ecap) if nerr else None
            rc = call(outs, errs)
            need_o = max([int(o.c.count) for o in outs] + [0])
            need_e = errs.need() if errs else 0
            if rc == CAPACITY or need_o > cap or need_e > ecap:
                if need_o <= cap and need_e <= ecap:
                    self._check(rc, what)
                cap, ecap = max(cap, need_o, 1), max(ecap, need_e)
                continue
            self._check(rc, what)
            return outs, errs

    # -- selection
    def select_an(self, b: Bat, op1, th1, op2=0, th2=0, comb=0, aoid=16089) -> Tuple[Bat, ErrVec]:
        def call(outs, errs):
            cb = _in_bat(b)
            return self.lib.ahead_gpu_select_an(self.ctx, ctypes.byref(cb), op1, ctypes.c_uint64(th1), op2,
                                                ctypes.c_uint64(th2), comb, ctypes.c_uint64(aoid),
                                                ctypes.byref(outs[0].c), ctypes.c_uint64(outs[0].cap),
                                                ctypes.byref(errs.c[0]))
        outs, errs = self._run("selectAN", call, b.count, 1)
        return outs[0].bat(), errs.vecs()[0]

    def select(self, b: Bat, op1, th1, op2=0, th2=0, comb=0) -> Bat:
        def call(outs, errs):
            cb = _in_bat(b)
            return self.lib.ahead_gpu_select(self.ctx, ctypes.byref(cb), op1, ctypes.c_uint64(th1), op2,
                                             ctypes.c_uint64(th2), comb, ctypes.byref(outs[0].c),
                                             ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("select", call, b.count, 0)
        return outs[0].bat()

    # -- string selection over fixed-width string slots
    def _select_str(self, fn, what, strs, width: int, seqbase, op1, th1, op2, th2, comb, an: bool) -> Col:
        torch = self.torch
        if strs.dtype != torch.uint8 or not strs.is_cuda or not strs.is_contiguous():
            raise ValueError("strs must be a contiguous uint8 CUDA tensor of rows of `width` bytes")
        count = strs.numel() // width if width else 0
        torch.cuda.current_stream().synchronize()  # the library launches on its own stream

        def call(outs, errs):
            return fn(self.ctx, ctypes.c_void_p(strs.data_ptr()), ctypes.c_uint64(width), ctypes.c_uint64(count),
                      ctypes.c_uint64(seqbase), op1, ctypes.c_char_p(th1), op2, ctypes.c_char_p(th2), comb,
                      ctypes.byref(outs[0].c), ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run(what, call, count, 0)
        o = outs[0]
        n = int(o.c.count)
        used = o.h[: n * (8 if an else 4)]
        return col_from_c(o.c.head, used.clone() if 4 * used.numel() < o.h.numel() else used)

    def select_str_an(self, strs, width: int, seqbase, op1, th1: bytes, op2=0, th2: bytes = b"", comb=0) -> Col:
        """selectAN over a string tail (selectAN_scalar.tcc:98-131, 185-222):
        the kept rows' resoid codes as a device column of u64 bytes."""
        return self._select_str(self.lib.ahead_gpu_select_str_an, "selectAN(str)", strs, width, seqbase, op1, th1,
                                op2, th2, comb, True)

    def select_str(self, strs, width: int, seqbase, op1, th1: bytes, op2=0, th2: bytes = b"", comb=0) -> Col:
        """select over a string tail (Normal/select_scalar.tcc:78-101, 137-165):
        the kept rows' oid_t as a device column of u32 bytes."""
        return self._select_str(self.lib.ahead_gpu_select_str, "select(str)", strs, width, seqbase, op1, th1, op2,
                                th2, comb, False)

    def hashjoin_str_an(self, l: Bat, r: Bat, r_strs, width: int, reenc_head=False, ah1r=1, ah1invr=1, side=1,
                        aoid=16089):
        """hashjoinAN with a string right tail (hashjoinAN.tcc:225-367):
        (head column, the matched `width`-byte slots as an (n, width) uint8
        device tensor, [H1, T1, H2, T2] error vectors)."""
        torch = self.torch
        if r_strs.dtype != torch.uint8 or not r_strs.is_cuda or not r_strs.is_contiguous():
            raise ValueError("r_strs must be a contiguous uint8 CUDA tensor of rows of `width` bytes")
        torch.cuda.current_stream().synchronize()  # the library launches on its own stream
        cap = max(l.count, 1)
        ecap = min(max(l.count, r.count, 1), 1 << 16)
        while True:
            head = torch.empty(cap * 8, dtype=torch.uint8, device="cuda")
            strs = torch.empty(cap * width + 1, dtype=torch.uint8, device="cuda")
            c = CBat()
            c.head.data = head.data_ptr()
            c.tail.data = strs.data_ptr()
            errs = _Errs(torch, 4, ecap)
            rc = self.lib.ahead_gpu_hashjoin_str_an(
                self.ctx, ctypes.byref(_in_bat(l)), ctypes.byref(_in_bat(r)), ctypes.c_void_p(r_strs.data_ptr()),
                ctypes.c_uint64(width), int(bool(reenc_head)), ctypes.c_uint64(ah1r), ctypes.c_uint64(ah1invr), side,
                ctypes.c_uint64(aoid), ctypes.byref(c), ctypes.c_uint64(cap), errs.c)
            n, need_e = int(c.count), errs.need()
            if rc == CAPACITY or n > cap or need_e > ecap:
                if n <= cap and need_e <= ecap:
                    self._check(rc, "hashjoinAN(str)")
                cap, ecap = max(cap, n, 1), max(ecap, need_e)
                continue
            self._check(rc, "hashjoinAN(str)")
            hcol = col_from_c(c.head, head[: n * WIDTH[c.head.type]].clone())
            return hcol, strs[: n * width].view(n, width).clone(), errs.vecs()

    def fetchjoin_str_an(self, a: Bat, strs, width: int, aoid=16089):
        """fetchjoinAN with a string tail (matchjoinAN.tcc:304-354): the
        fetched slots as an (n, width) uint8 device tensor and [vec1, vec2]
        (vec2 never present)."""
        torch = self.torch
        if strs.dtype != torch.uint8 or not strs.is_cuda or not strs.is_contiguous():
            raise ValueError("strs must be a contiguous uint8 CUDA tensor of rows of `width` bytes")
        count = strs.numel() // width
        torch.cuda.current_stream().synchronize()  # the library launches on its own stream
        cap = max(a.count, 1)
        ecap = min(cap, 1 << 16)
        while True:
            out = torch.empty(cap * width + 1, dtype=torch.uint8, device="cuda")
            n = ctypes.c_uint64(0)
            errs = _Errs(torch, 2, ecap)
            rc = self.lib.ahead_gpu_fetchjoin_str_an(self.ctx, ctypes.byref(_in_bat(a)), ctypes.c_void_p(strs.data_ptr()),
                                                     ctypes.c_uint64(width), ctypes.c_uint64(count),
                                                     ctypes.c_uint64(aoid), ctypes.c_void_p(out.data_ptr()),
                                                     ctypes.c_uint64(cap), ctypes.byref(n), errs.c)
            need_e = errs.need()
            if rc == CAPACITY or need_e > ecap:
                cap, ecap = max(cap, int(n.value), 1), max(ecap, need_e)
                continue
            self._check(rc, "fetchjoinAN(str)")
            k = int(n.value)
            return out[: k * width].view(k, width).clone(), errs.vecs()

    def groupby2_str_an(self, strs, width: int, grouping: Bat, ngroups: int, aoid=65117,
                        aoidinv=0x3E36D3BC8D9BC5F5, seqbase: int = 0) -> Tuple[Bat, Bat, List[ErrVec]]:
        """groupbyAN binary over a string tail (a void head with `seqbase`;
        the reference's Java-style string hash)."""
        torch = self.torch
        if strs.dtype != torch.uint8 or not strs.is_cuda or not strs.is_contiguous():
            raise ValueError("strs must be a contiguous uint8 CUDA tensor of rows of `width` bytes")
        count = strs.numel() // width
        torch.cuda.current_stream().synchronize()

        def call(outs, errs):
            cg = _in_bat(grouping)
            return self.lib.ahead_gpu_groupby2_str_an(self.ctx, ctypes.c_void_p(strs.data_ptr()),
                                                      ctypes.c_uint64(width), ctypes.c_uint64(count),
                                                      ctypes.c_uint64(seqbase), ctypes.byref(cg),
                                                      ctypes.c_uint64(ngroups), ctypes.c_uint64(aoid),
                                                      ctypes.c_uint64(aoidinv), ctypes.byref(outs[0].c),
                                                      ctypes.byref(outs[1].c), ctypes.c_uint64(outs[0].cap), errs.c)
        outs, errs = self._run("groupbyAN2(str)", call, count, 3, nout=2)
        return outs[0].bat(), outs[1].bat(), errs.vecs()

    def fetchjoin_str(self, a: Bat, strs, width: int):
        """fetchjoin over a string tail (Normal/matchjoin.tcc:144-160): the
        fetched slots as an (n, width) uint8 device tensor."""
        torch = self.torch
        if strs.dtype != torch.uint8 or not strs.is_cuda or not strs.is_contiguous():
            raise ValueError("strs must be a contiguous uint8 CUDA tensor of rows of `width` bytes")
        count = strs.numel() // width
        torch.cuda.current_stream().synchronize()
        cap = max(a.count, 1)
        while True:
            out = torch.empty(cap * width + 1, dtype=torch.uint8, device="cuda")
            n = ctypes.c_uint64(0)
            rc = self.lib.ahead_gpu_fetchjoin_str(self.ctx, ctypes.byref(_in_bat(a)), ctypes.c_void_p(strs.data_ptr()),
                                                  ctypes.c_uint64(width), ctypes.c_uint64(count),
                                                  ctypes.c_void_p(out.data_ptr()), ctypes.c_uint64(cap), ctypes.byref(n))
            if rc == CAPACITY:
                cap = max(cap, int(n.value), 1)
                continue
            self._check(rc, "fetchjoin(str)")
            k = int(n.value)
            return out[: k * width].view(k, width).clone()

    def groupby2_str(self, strs, width: int, grouping: Bat, ngroups: int, seqbase: int = 0) -> Tuple[Bat, Bat]:
        """groupby binary over a string tail (Normal/groupby.tcc:85-121)."""
        torch = self.torch
        if strs.dtype != torch.uint8 or not strs.is_cuda or not strs.is_contiguous():
            raise ValueError("strs must be a contiguous uint8 CUDA tensor of rows of `width` bytes")
        count = strs.numel() // width
        torch.cuda.current_stream().synchronize()

        def call(outs, errs):
            return self.lib.ahead_gpu_groupby2_str(self.ctx, ctypes.c_void_p(strs.data_ptr()), ctypes.c_uint64(width),
                                                   ctypes.c_uint64(count), ctypes.c_uint64(seqbase),
                                                   ctypes.byref(_in_bat(grouping)), ctypes.c_uint64(ngroups),
                                                   ctypes.byref(outs[0].c), ctypes.byref(outs[1].c),
                                                   ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("groupby2(str)", call, count, 0, nout=2)
        return outs[0].bat(), outs[1].bat()

    # -- check / decode
    def check_an(self, b: Bat, ainv, unenc_max, aoid=16089) -> ErrVec:
        def call(outs, errs):
            cb = _in_bat(b)
            return self.lib.ahead_gpu_check_an(self.ctx, ctypes.byref(cb), ctypes.c_uint64(ainv),
                                               ctypes.c_uint64(unenc_max), ctypes.c_uint64(aoid),
                                               ctypes.byref(errs.c[0]))
        _, errs = self._run("checkAN", call, b.count, 1, nout=0)
        return errs.vecs()[0]

    def decode_an(self, b: Bat, aoid=16089) -> Tuple[Bat, ErrVec]:
        def call(outs, errs):
            cb = _in_bat(b)
            return self.lib.ahead_gpu_decode_an(self.ctx, ctypes.byref(cb), ctypes.c_uint64(aoid),
                                                ctypes.byref(outs[0].c), ctypes.c_uint64(outs[0].cap),
                                                ctypes.byref(errs.c[0]))
        outs, errs = self._run("decodeAN", call, b.count, 1)
        return outs[0].bat(), errs.vecs()[0]

    def check_and_decode_an(self, b: Bat, aoid=16089) -> Tuple[Bat, ErrVec, ErrVec]:
        def call(outs, errs):
            cb = _in_bat(b)
            return self.lib.ahead_gpu_check_and_decode_an(self.ctx, ctypes.byref(cb), ctypes.c_uint64(aoid),
                                                          ctypes.byref(outs[0].c), ctypes.c_uint64(outs[0].cap),
                                                          ctypes.byref(errs.c[0]), ctypes.byref(errs.c[1]))
        outs, errs = self._run("checkAndDecodeAN", call, b.count, 2)
        v = errs.vecs()
        return outs[0].bat(), v[0], v[1]

    def encode_an(self, b: Bat, A) -> Bat:
        def call(outs, errs):
            cb = _in_bat(b)
            return self.lib.ahead_gpu_encode_an(self.ctx, ctypes.byref(cb), ctypes.c_uint64(A),
                                                ctypes.byref(outs[0].c), ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("encodeAN", call, b.count, 0)
        return outs[0].bat()

    # -- joins
    def hashjoin_an(self, l: Bat, r: Bat, reenc_head=False, ah1r=1, ah1invr=1, reenc_tail=False, at2r=1,
                    at2invr=1, side=1, aoid=16089) -> Tuple[Bat, List[ErrVec]]:
        def call(outs, errs):
            cl, cr = _in_bat(l), _in_bat(r)
            return self.lib.ahead_gpu_hashjoin_an(self.ctx, ctypes.byref(cl), ctypes.byref(cr), int(reenc_head),
                                                  ctypes.c_uint64(ah1r), ctypes.c_uint64(ah1invr), int(reenc_tail),
                                                  ctypes.c_uint64(at2r), ctypes.c_uint64(at2invr), side,
                                                  ctypes.c_uint64(aoid), ctypes.byref(outs[0].c),
                                                  ctypes.c_uint64(outs[0].cap), errs.c)
        outs, errs = self._run("hashjoinAN", call, max(l.count, r.count), 4)
        return outs[0].bat(), errs.vecs()

    def hashjoin(self, l: Bat, r: Bat, side=1) -> Bat:
        def call(outs, errs):
            cl, cr = _in_bat(l), _in_bat(r)
            return self.lib.ahead_gpu_hashjoin(self.ctx, ctypes.byref(cl), ctypes.byref(cr), side,
                                               ctypes.byref(outs[0].c), ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("hashjoin", call, max(l.count, r.count), 0)
        return outs[0].bat()

    def matchjoin_an(self, a: Bat, b: Bat, reenc=False, ah1r=0, ah1invr=0, at2r=0, at2invr=0,
                     aoid=16089) -> Tuple[Bat, List[ErrVec]]:
        def call(outs, errs):
            ca, cb = _in_bat(a), _in_bat(b)
            return self.lib.ahead_gpu_matchjoin_an(self.ctx, ctypes.byref(ca), ctypes.byref(cb), int(reenc),
                                                   ctypes.c_uint64(ah1r), ctypes.c_uint64(ah1invr),
                                                   ctypes.c_uint64(at2r), ctypes.c_uint64(at2invr),
                                                   ctypes.c_uint64(aoid), ctypes.byref(outs[0].c),
                                                   ctypes.c_uint64(outs[0].cap), errs.c)
        # at most one output row per row of the smaller input (a retry covers the rest)
        outs, errs = self._run("matchjoinAN", call, max(min(a.count, b.count), 1), 4)
        return outs[0].bat(), errs.vecs()

    def matchjoin(self, a: Bat, b: Bat) -> Bat:
        def call(outs, errs):
            ca, cb = _in_bat(a), _in_bat(b)
            return self.lib.ahead_gpu_matchjoin(self.ctx, ctypes.byref(ca), ctypes.byref(cb),
                                                ctypes.byref(outs[0].c), ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("matchjoin", call, max(a.count, b.count), 0)
        return outs[0].bat()

    def fetchjoin_an(self, a: Bat, b: Bat, reenc=False, atr=1, atrinv=1, aoid=16089) -> Tuple[Bat, List[ErrVec]]:
        def call(outs, errs):
            ca, cb = _in_bat(a), _in_bat(b)
            return self.lib.ahead_gpu_fetchjoin_an(self.ctx, ctypes.byref(ca), ctypes.byref(cb), int(reenc),
                                                   ctypes.c_uint64(atr), ctypes.c_uint64(atrinv),
                                                   ctypes.c_uint64(aoid), ctypes.byref(outs[0].c),
                                                   ctypes.c_uint64(outs[0].cap), errs.c)
        outs, errs = self._run("fetchjoinAN", call, a.count, 2)
        return outs[0].bat(), errs.vecs()

    def fetchjoin(self, a: Bat, b: Bat) -> Bat:
        def call(outs, errs):
            ca, cb = _in_bat(a), _in_bat(b)
            return self.lib.ahead_gpu_fetchjoin(self.ctx, ctypes.byref(ca), ctypes.byref(cb),
                                                ctypes.byref(outs[0].c), ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("fetchjoin", call, a.count, 0)
        return outs[0].bat()

    # -- grouping and aggregation
    def groupby_an(self, b: Bat, aoid=65117, aoidinv=0x3E36D3BC8D9BC5F5) -> Tuple[Bat, Bat, List[ErrVec]]:
        def call(outs, errs):
            cb = _in_bat(b)
            return self.lib.ahead_gpu_groupby_an(self.ctx, ctypes.byref(cb), ctypes.c_uint64(aoid),
                                                 ctypes.c_uint64(aoidinv), ctypes.byref(outs[0].c),
                                                 ctypes.byref(outs[1].c), ctypes.c_uint64(outs[0].cap), errs.c)
        outs, errs = self._run("groupbyAN", call, b.count, 2, nout=2)
        return outs[0].bat(), outs[1].bat(), errs.vecs()

    def groupby2_an(self, b: Bat, grouping: Bat, ngroups: int, aoid=65117,
                    aoidinv=0x3E36D3BC8D9BC5F5) -> Tuple[Bat, Bat, List[ErrVec]]:
        def call(outs, errs):
            cb, cg = _in_bat(b), _in_bat(grouping)
            return self.lib.ahead_gpu_groupby2_an(self.ctx, ctypes.byref(cb), ctypes.byref(cg),
                                                  ctypes.c_uint64(ngroups), ctypes.c_uint64(aoid),
                                                  ctypes.c_uint64(aoidinv), ctypes.byref(outs[0].c),
                                                  ctypes.byref(outs[1].c), ctypes.c_uint64(outs[0].cap), errs.c)
        outs, errs = self._run("groupbyAN2", call, b.count, 3, nout=2)
        return outs[0].bat(), outs[1].bat(), errs.vecs()

    def aggregate_sum_grouped_an(self, b: Bat, grouping: Bat, ngroups: int, result_type=9, ar=65117,
                                 arinv=0x3E36D3BC8D9BC5F5, aoid=65117) -> Tuple[Bat, List[ErrVec]]:
        def call(outs, errs):
            cb, cg = _in_bat(b), _in_bat(grouping)
            return self.lib.ahead_gpu_aggregate_sum_grouped_an(self.ctx, ctypes.byref(cb), ctypes.byref(cg),
                                                               ctypes.c_uint64(ngroups), result_type,
                                                               ctypes.c_uint64(ar), ctypes.c_uint64(arinv),
                                                               ctypes.c_uint64(aoid), ctypes.byref(outs[0].c),
                                                               errs.c)
        outs, errs = self._run("aggregate_sum_groupedAN", call, max(b.count, ngroups, 1), 3)
        return outs[0].bat(), errs.vecs()

    def aggregate_mul_sum_an(self, a: Bat, b: Bat, result_type=9, init=0, ra=65117,
                             rainv=0x3E36D3BC8D9BC5F5, aoid=16089) -> Tuple[int, List[ErrVec]]:
        tot = ctypes.c_uint64(0)

        def call(outs, errs):
            ca, cb = _in_bat(a), _in_bat(b)
            return self.lib.ahead_gpu_aggregate_mul_sum_an(self.ctx, ctypes.byref(ca), ctypes.byref(cb), result_type,
                                                           ctypes.c_uint64(init), ctypes.c_uint64(ra),
                                                           ctypes.c_uint64(rainv), ctypes.c_uint64(aoid),
                                                           ctypes.byref(tot), errs.c)
        _, errs = self._run("aggregate_mul_sumAN", call, max(a.count, b.count), 2, nout=0)
        return int(tot.value), errs.vecs()

    def aggregate_mul_sum(self, a: Bat, b: Bat, result_type=4, init=0) -> int:
        tot = ctypes.c_uint64(0)
        ca, cb = _in_bat(a), _in_bat(b)
        rc = self.lib.ahead_gpu_aggregate_mul_sum(self.ctx, ctypes.byref(ca), ctypes.byref(cb), result_type,
                                                  ctypes.c_uint64(init), ctypes.byref(tot))
        self._check(rc, "aggregate_mul_sum")
        return int(tot.value)

    # -- unencoded twins
    def groupby(self, b: Bat) -> Tuple[Bat, Bat]:
        def call(outs, errs):
            cb = _in_bat(b)
            return self.lib.ahead_gpu_groupby(self.ctx, ctypes.byref(cb), ctypes.byref(outs[0].c),
                                              ctypes.byref(outs[1].c), ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("groupby", call, b.count, 0, nout=2)
        return outs[0].bat(), outs[1].bat()

    def groupby2(self, b: Bat, grouping: Bat, ngroups: int) -> Tuple[Bat, Bat]:
        def call(outs, errs):
            cb, cg = _in_bat(b), _in_bat(grouping)
            return self.lib.ahead_gpu_groupby2(self.ctx, ctypes.byref(cb), ctypes.byref(cg), ctypes.c_uint64(ngroups),
                                               ctypes.byref(outs[0].c), ctypes.byref(outs[1].c),
                                               ctypes.c_uint64(outs[0].cap))
        outs, _ = self._run("groupby2", call, b.count, 0, nout=2)
        return outs[0].bat(), outs[1].bat()

    def aggregate_sum_grouped(self, b: Bat, grouping: Bat, ngroups: int, result_type=4) -> Bat:
        def call(outs, errs):
            cb, cg = _in_bat(b), _in_bat(grouping)
            return self.lib.ahead_gpu_aggregate_sum_grouped(self.ctx, ctypes.byref(cb), ctypes.byref(cg),
                                                            ctypes.c_uint64(ngroups), result_type,
                                                            ctypes.byref(outs[0].c))
        outs, _ = self._run("aggregate_sum_grouped", call, max(ngroups, 1), 0)
        return outs[0].bat()

    def aggregate_sum(self, b: Bat, result_type=4) -> int:
        tot = ctypes.c_uint64(0)
        cb = _in_bat(b)
        self._check(self.lib.ahead_gpu_aggregate_sum(self.ctx, ctypes.byref(cb), result_type, ctypes.byref(tot)),
                    "aggregate_sum")
        return int(tot.value)

    def arithmetic(self, op, result_type, a: Bat, b: Bat) -> Bat:
        def call(outs, errs):
            ca, cb = _in_bat(a), _in_bat(b)
            return self.lib.ahead_gpu_arithmetic(self.ctx, op, result_type, ctypes.byref(ca), ctypes.byref(cb),
                                                 ctypes.byref(outs[0].c))
        outs, _ = self._run("arithmetic", call, max(a.count, 1), 0)
        return outs[0].bat()

    def arithmetic_an(self, op, result_type, a: Bat, b: Bat, ar, arinv, aoid=16089) -> Tuple[Bat, List[ErrVec]]:
        def call(outs, errs):
            ca, cb = _in_bat(a), _in_bat(b)
            return self.lib.ahead_gpu_arithmetic_an(self.ctx, op, result_type, ctypes.byref(ca), ctypes.byref(cb),
                                                    ctypes.c_uint64(ar), ctypes.c_uint64(arinv),
                                                    ctypes.c_uint64(aoid), ctypes.byref(outs[0].c), errs.c)
        outs, errs = self._run("arithmeticAN", call, max(a.count, 1), 4)
        return outs[0].bat(), errs.vecs()
