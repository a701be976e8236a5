"""Fused star joins (ahead_sj_* in include/ahead_gpu.h) from Python.

`StarJoinEngine` prepares a device-resident schema once and answers batches
of up to 64 `StarQuery`s in one fused pass over the fact table (optionally by
replaying a CUDA graph).  A query the fused path cannot answer (its inputs
leave the fused path's domain, e.g. duplicate or corrupt dimension keys) comes
back with status UNSUPPORTED; `answer()` then runs the operator-at-a-time
composition on the same GPU library.
"""
from __future__ import annotations

import ctypes
import sys
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from .gpu import AheadError, GpuOps, load_library
from .model import CAPACITY, CCol, CErrVec, OK, UNSUPPORTED, ccol
from .ssb import ENGINE_ATTRS, FACT_COLS, FK, KEY, MEASURES, StarQuery, StarSchema

DIM_INDEX = {"date": 0, "customer": 1, "part": 2, "supplier": 3}
PACKED_SLOTS = 3  # ahead_sj_cube_variant_slots of a shape that reads the packed join index
NCOL = len(FACT_COLS)
FACT_COL_INDEX = {c: i for i, c in enumerate(FACT_COLS)}


def engine_attrs(schema: StarSchema) -> Dict[str, List[str]]:
    """The dimension attributes an engine over `schema` registers, in order:
    those of ENGINE_ATTRS the schema holds."""
    return {d: [a for a in ENGINE_ATTRS[d] if a in schema.tables[d]] for d in ENGINE_ATTRS}


class CSjDim(ctypes.Structure):
    _fields_ = [("key", CCol), ("attr", CCol * 4), ("rows", ctypes.c_uint64), ("nattr", ctypes.c_int32),
                ("_pad", ctypes.c_int32)]


class CSjSchema(ctypes.Structure):
    _fields_ = [("fk", CCol * 4), ("price", CCol), ("discount", CCol), ("fact_rows", ctypes.c_uint64),
                ("dim", CSjDim * 4), ("quantity", CCol), ("revenue", CCol), ("supplycost", CCol)]


class CSjPred(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int32), ("attr", ctypes.c_int32), ("op1", ctypes.c_int32), ("op2", ctypes.c_int32),
                ("comb", ctypes.c_int32), ("_pad", ctypes.c_int32), ("th1", ctypes.c_uint64),
                ("th2", ctypes.c_uint64)]


class CSjFPred(ctypes.Structure):
    _fields_ = [("col", ctypes.c_int32), ("op1", ctypes.c_int32), ("op2", ctypes.c_int32), ("comb", ctypes.c_int32),
                ("th1", ctypes.c_uint64), ("th2", ctypes.c_uint64)]


class CSjQuery(ctypes.Structure):
    _fields_ = [("fact_rows", ctypes.c_uint64), ("npred", ctypes.c_int32), ("ngroup", ctypes.c_int32),
                ("pred", CSjPred * 4), ("gdim", ctypes.c_int32 * 3), ("gattr", ctypes.c_int32 * 3),
                ("measure", ctypes.c_int32), ("nfpred", ctypes.c_int32), ("fpred", CSjFPred * 2)]


class CSjResult(ctypes.Structure):
    _fields_ = [("ngroups", ctypes.c_uint64), ("capacity", ctypes.c_uint64),
                ("keys", ctypes.POINTER(ctypes.c_uint64) * 3), ("sums", ctypes.POINTER(ctypes.c_uint64)),
                ("total", ctypes.c_uint64), ("status", ctypes.c_int32), ("_pad", ctypes.c_int32),
                ("fact_err", CErrVec * NCOL)]


class CSjStats(ctypes.Structure):
    _fields_ = [("batch_ms", ctypes.c_float), ("fact_ms", ctypes.c_float), ("fact_rows", ctypes.c_uint64),
                ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64), ("errors_logged", ctypes.c_uint64),
                ("strategy", ctypes.c_uint32), ("unseen_sigs", ctypes.c_uint32), ("exception_rows", ctypes.c_uint64),
                ("cube_variant", ctypes.c_int32), ("pad", ctypes.c_uint32)]


class CSjXchg(ctypes.Structure):
    _fields_ = [("sums", ctypes.c_void_p), ("firsts", ctypes.c_void_p), ("flags", ctypes.c_void_p),
                ("log", ctypes.c_void_p), ("groups", ctypes.c_uint64), ("log_cap", ctypes.c_uint64)]


@dataclass
class Xchg:
    """The exchange area of a fact-sharded batch's local half (device
    addresses and sizes): group sums and first rows (int64 each), 4 status
    flags, the error log (1 + log_cap words)."""
    sums: int
    firsts: int
    flags: int
    log: int
    groups: int
    log_cap: int


@dataclass
class FusedResult:
    status: int
    keys: List[np.ndarray]
    sums: Optional[np.ndarray]
    total: Optional[int]
    fact_errors: Dict[str, np.ndarray] = field(default_factory=dict)


def _col(b, which="tail") -> CCol:
    c = getattr(b, which)
    return ccol(c, int(c.data.data_ptr()) if c.data is not None else 0)


def c_query(q: StarQuery, schema: StarSchema) -> CSjQuery:
    ai = {d: {a: i for i, a in enumerate(v)} for d, v in engine_attrs(schema).items()}
    cq = CSjQuery()
    cq.fact_rows = q.fact_rows or schema.sizes["fact"]
    cq.npred = len(q.preds)
    for k, p in enumerate(q.preds):
        A = schema.tables[p.dim][p.attr].tail.A
        cq.pred[k] = CSjPred(DIM_INDEX[p.dim], ai[p.dim][p.attr], p.op1, p.op2, p.comb, 0, p.v1 * A, p.v2 * A)
    cq.ngroup = len(q.group)
    for j, (d, a) in enumerate(q.group):
        cq.gdim[j] = DIM_INDEX[d]
        cq.gattr[j] = ai[d][a]
    cq.measure = MEASURES.index(q.measure)
    cq.nfpred = len(q.fpreds)
    for k, f in enumerate(q.fpreds):
        A = schema.tables["lineorder"][f.col].tail.A
        cq.fpred[k] = CSjFPred(FACT_COL_INDEX[f.col], f.op1, f.op2, f.comb, f.v1 * A, f.v2 * A)
    return cq


def index_packing(krange, nrec):
    """(A, payload bits) of the packed join index for two dimensions with key
    ranges `krange` and `nrec` distinct attribute records, or None when it does
    not fit 64 bits (ahead_sj_index_packing; host arithmetic, no device)."""
    lib = load_library()
    u64p = ctypes.POINTER(ctypes.c_uint64)
    lib.ahead_sj_index_packing.argtypes = [u64p, u64p, u64p, ctypes.POINTER(ctypes.c_uint32)]
    kr = (ctypes.c_uint64 * 2)(*krange)
    nr = (ctypes.c_uint64 * 2)(*nrec)
    a, bits = ctypes.c_uint64(), ctypes.c_uint32()
    rc = lib.ahead_sj_index_packing(kr, nr, ctypes.byref(a), ctypes.byref(bits))
    if rc == UNSUPPORTED:
        return None
    if rc != OK:
        raise AheadError(rc, "ahead_sj_index_packing", "")
    return int(a.value), int(bits.value)


class StarJoinEngine:
    """A device-resident star schema prepared for fused batches."""

    def __init__(self, gpu: GpuOps, schema: StarSchema, max_groups: int = 4096, err_cap: int = 1 << 16):
        self.gpu = gpu
        self.lib = load_library()
        self.schema = schema
        self.max_groups = max_groups
        self.err_cap = err_cap
        T = schema.tables
        s = CSjSchema()
        attrs = engine_attrs(schema)
        for d, i in DIM_INDEX.items():
            s.fk[i] = _col(T["lineorder"][FK[d]])
            dim = CSjDim()
            dim.key = _col(T[d][KEY[d]])
            for j, a in enumerate(attrs[d]):
                dim.attr[j] = _col(T[d][a])
            dim.nattr = len(attrs[d])
            dim.rows = T[d][KEY[d]].count
            s.dim[i] = dim
        s.price = _col(T["lineorder"]["price"])
        s.discount = _col(T["lineorder"]["discount"])
        for c in ("quantity", "revenue", "supplycost"):  # the programs' measures and fact predicates
            if c in T["lineorder"]:
                setattr(s, c, _col(T["lineorder"][c]))
        s.fact_rows = T["lineorder"]["price"].count
        self._schema = s
        self.eng = ctypes.c_void_p()
        L = self.lib
        L.ahead_sj_create.argtypes = [ctypes.c_void_p, ctypes.POINTER(CSjSchema), ctypes.POINTER(ctypes.c_void_p)]
        L.ahead_sj_destroy.argtypes = [ctypes.c_void_p]
        for f in (L.ahead_sj_run, L.ahead_sj_run_graph):
            f.argtypes = [ctypes.c_void_p, ctypes.POINTER(CSjQuery), ctypes.c_int, ctypes.POINTER(CSjResult)]
        L.ahead_sj_submit.argtypes = [ctypes.c_void_p, ctypes.POINTER(CSjQuery), ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_uint64)]
        L.ahead_sj_wait.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(CSjResult)]
        L.ahead_sj_fetch.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(CSjResult)]
        L.ahead_sj_last_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(CSjStats)]
        L.ahead_sj_tune.argtypes = [ctypes.c_void_p, ctypes.POINTER(CSjQuery), ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_int)]
        L.ahead_sj_set_variant.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ahead_sj_set_strategy.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ahead_sj_set_cube_variant.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ahead_sj_set_cube_split.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
        L.ahead_sj_cube_variant_count.argtypes = []
        L.ahead_sj_set_shard.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64]
        L.ahead_sj_submit_local.argtypes = [ctypes.c_void_p, ctypes.POINTER(CSjQuery), ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(CSjXchg)]
        L.ahead_sj_submit_final.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_int]
        L.ahead_sj_cube_variant_is_indexed.argtypes = [ctypes.c_int]
        L.ahead_sj_cube_variant_slots.argtypes = [ctypes.c_int]
        L.ahead_sj_set_index.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ahead_sj_index_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                          ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                          ctypes.POINTER(ctypes.c_uint32)]
        L.ahead_sj_last_ms.restype = ctypes.c_float
        L.ahead_sj_last_ms.argtypes = [ctypes.c_void_p]
        rc = self.lib.ahead_sj_create(gpu.ctx, ctypes.byref(s), ctypes.byref(self.eng))
        if rc != OK:
            raise AheadError(rc, "ahead_sj_create", self.lib.ahead_ctx_last_error(gpu.ctx).decode())
        self._bufs = None

    def close(self):
        if self.eng:
            self.lib.ahead_sj_destroy(self.eng)
            self.eng = ctypes.c_void_p()

    def __del__(self, _finalizing=sys.is_finalizing):  # bound now: module globals may be gone at exit
        if _finalizing():  # the CUDA runtime may be gone; the process frees everything
            return
        try:
            self.close()
        except Exception:
            pass

    @property
    def last_ms(self) -> float:
        return float(self.lib.ahead_sj_last_ms(self.eng))

    def tune(self, queries: Sequence[StarQuery]) -> int:
        """Time the fact-kernel shapes on this batch and keep the fastest."""
        cqs = (CSjQuery * len(queries))(*[c_query(q, self.schema) for q in queries])
        v = ctypes.c_int()
        self._check(self.lib.ahead_sj_tune(self.eng, cqs, len(queries), ctypes.byref(v)), "ahead_sj_tune")
        return v.value

    def set_strategy(self, strategy: int):
        """-1: chosen per batch; 0: per-row pass; 1: signature cube (when the batch fits)."""
        self._check(self.lib.ahead_sj_set_strategy(self.eng, strategy), "ahead_sj_set_strategy")

    def set_cube_variant(self, variant: int):
        self._check(self.lib.ahead_sj_set_cube_variant(self.eng, variant), "ahead_sj_set_cube_variant")

    def cube_variants(self) -> int:
        """Number of compiled cube-scan shapes."""
        return int(self.lib.ahead_sj_cube_variant_count())

    def cube_variant_is_indexed(self, variant: int) -> bool:
        """Whether cube-scan shape `variant` reads the engine's join index."""
        return self.lib.ahead_sj_cube_variant_is_indexed(variant) == 1

    def cube_variant_slots(self, variant: int) -> int:
        """Index arrays cube-scan shape `variant` reads (0, 1 or 2; 3: both
        dimensions from the packed index)."""
        return int(self.lib.ahead_sj_cube_variant_slots(variant))

    def set_index(self, fmt: int):
        """Rebuild the join index: -1 packed when it fits, else two words
        (the default); 0 none; 1 two words per row; 2 packed."""
        self._check(self.lib.ahead_sj_set_index(self.eng, fmt), "ahead_sj_set_index")

    def cube_variant_reads_index(self, variant: int) -> bool:
        """Whether shape `variant` reads the engine's current join index (its
        format included)."""
        ptr, bpr, _, _ = self.index_info()
        slots = self.cube_variant_slots(variant)
        return bool(ptr) and self.cube_variant_is_indexed(variant) and slots > 0 and \
            (slots == PACKED_SLOTS) == (bpr == 8)

    def index_info(self):
        """(device address or None, bytes per row, rows, indexed-dimension bit set) of the join index."""
        p, bpr, rows, dims = ctypes.c_void_p(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint32()
        self._check(self.lib.ahead_sj_index_info(self.eng, ctypes.byref(p), ctypes.byref(bpr), ctypes.byref(rows),
                                                 ctypes.byref(dims)), "ahead_sj_index_info")
        return p.value, bpr.value, rows.value, dims.value



    def set_cube_split(self, rows: int):
        """Rows of the cube scan's first phase (0: automatic)."""
        self._check(self.lib.ahead_sj_set_cube_split(self.eng, rows), "ahead_sj_set_cube_split")

    def set_variant(self, variant: int):
        self._check(self.lib.ahead_sj_set_variant(self.eng, variant), "ahead_sj_set_variant")

    def last_stats(self) -> CSjStats:
        st = CSjStats()
        self._check(self.lib.ahead_sj_last_stats(self.eng, ctypes.byref(st)), "ahead_sj_last_stats")
        return st

    def _results(self, slot: int):
        """Host result buffers of one slot (two batches may be in flight)."""
        if self._bufs is None:
            self._bufs = [None, None]
        if self._bufs[slot] is None:
            cap, ecap = self.max_groups, self.err_cap
            keys = [[np.zeros(cap, np.uint64) for _ in range(3)] for _ in range(64)]
            sums = [np.zeros(cap, np.uint64) for _ in range(64)]
            errs = [[np.zeros(ecap, np.uint64) for _ in range(NCOL)] for _ in range(64)]
            arr = (CSjResult * 64)()
            for q in range(64):
                arr[q].capacity = cap
                for j in range(3):
                    arr[q].keys[j] = keys[q][j].ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
                arr[q].sums = sums[q].ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
                for c in range(NCOL):
                    arr[q].fact_err[c].data = errs[q][c].ctypes.data
                    arr[q].fact_err[c].capacity = ecap
            self._bufs[slot] = (keys, sums, errs, arr)
        return self._bufs[slot]

    def _check(self, rc: int, what: str):
        if rc != OK:
            raise AheadError(rc, what, self.lib.ahead_ctx_last_error(self.gpu.ctx).decode())

    def submit(self, queries: Sequence[StarQuery], graph: bool = True) -> int:
        """Enqueue a batch of 1..64 queries; returns its ticket."""
        nq = len(queries)
        if not 1 <= nq <= 64:
            raise ValueError("a fused batch holds 1..64 queries")
        cqs = (CSjQuery * nq)(*[c_query(q, self.schema) for q in queries])
        t = ctypes.c_uint64()
        self._check(self.lib.ahead_sj_submit(self.eng, cqs, nq, int(graph), ctypes.byref(t)), "ahead_sj_submit")
        self._pending = getattr(self, "_pending", {})
        self._pending[t.value] = list(queries)
        return t.value

    def set_shard(self, first_row: int, table_rows: int):
        """This engine's fact columns are rows [first_row, first_row + rows) of
        a table of `table_rows` rows; batches then run as submit_local /
        exchange / submit_final."""
        self._check(self.lib.ahead_sj_set_shard(self.eng, first_row, table_rows), "ahead_sj_set_shard")

    def submit_local(self, queries: Sequence[StarQuery], graph: bool = True):
        """The local half of a fact-sharded batch; returns (ticket, Xchg)."""
        nq = len(queries)
        if not 1 <= nq <= 64:
            raise ValueError("a fused batch holds 1..64 queries")
        cqs = (CSjQuery * nq)(*[c_query(q, self.schema) for q in queries])
        t, x = ctypes.c_uint64(), CSjXchg()
        self._check(self.lib.ahead_sj_submit_local(self.eng, cqs, nq, int(graph), ctypes.byref(t), ctypes.byref(x)),
                    "ahead_sj_submit_local")
        self._pending = getattr(self, "_pending", {})
        self._pending[t.value] = list(queries)
        return t.value, Xchg(x.sums, x.firsts, x.flags, x.log, int(x.groups), int(x.log_cap))

    def submit_final(self, ticket: int, gathered_logs: int, world: int):
        """The final half, after the exchange: `gathered_logs` = device address
        of `world` areas of 1 + log_cap words (every engine's log, rank order)."""
        self._check(self.lib.ahead_sj_submit_final(self.eng, ticket, ctypes.c_void_p(gathered_logs), world),
                    "ahead_sj_submit_final")

    def wait(self, ticket: int) -> List[FusedResult]:
        """Results of a submitted batch, in query order."""
        queries = self._pending.pop(ticket)
        keys, sums, errs, arr = self._results(ticket % 2)
        self._check(self.lib.ahead_sj_wait(self.eng, ticket, arr), "ahead_sj_wait")
        out = []
        for i, q in enumerate(queries):
            r = arr[i]
            n = int(r.ngroups)
            if r.status == CAPACITY:  # more groups or errors than the buffers hold: fetch at full size
                r, big = self._fetch(ticket, i, n, [int(r.fact_err[c].count) for c in range(NCOL)])
                fe = {FACT_COLS[c]: big[4 + c][: int(r.fact_err[c].count)].copy() for c in range(NCOL)}
                if r.status == OK and q.group:
                    out.append(FusedResult(OK, [big[j][:n].copy() for j in range(len(q.group))], big[3][:n].copy(),
                                           None, fe))
                    continue
            else:
                fe = {FACT_COLS[c]: errs[i][c][: int(r.fact_err[c].count)].copy() for c in range(NCOL)}
            if r.status != OK:
                out.append(FusedResult(int(r.status), [], None, None, fe))
            elif not q.group:
                out.append(FusedResult(OK, [], None, int(r.total), fe))
            else:
                out.append(FusedResult(OK, [keys[i][j][:n].copy() for j in range(len(q.group))], sums[i][:n].copy(),
                                       None, fe))
        return out

    def _fetch(self, ticket: int, i: int, ngroups: int, nerr: List[int]):
        bufs = [np.zeros(max(ngroups, 1), np.uint64) for _ in range(4)] + [np.zeros(max(c, 1), np.uint64) for c in nerr]
        r = CSjResult()
        r.capacity = ngroups
        for j in range(3):
            r.keys[j] = bufs[j].ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
        r.sums = bufs[3].ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
        for c in range(NCOL):
            r.fact_err[c].data = bufs[4 + c].ctypes.data
            r.fact_err[c].capacity = nerr[c]
        self._check(self.lib.ahead_sj_fetch(self.eng, ticket, i, ctypes.byref(r)), "ahead_sj_fetch")
        return r, bufs

    def plain(self, q: StarQuery) -> FusedResult:
        """The same query operator at a time, composed in C++ from the AN
        operators (ahead_plain_starjoin; no engine state is used), as a
        FusedResult."""
        L = self.lib
        L.ahead_plain_starjoin.argtypes = [ctypes.c_void_p, ctypes.POINTER(CSjSchema), ctypes.POINTER(CSjQuery),
                                           ctypes.POINTER(CSjResult)]
        cq = c_query(q, self.schema)
        ngroups, nerr = self.max_groups, [self.err_cap] * NCOL
        while True:
            bufs = [np.zeros(max(ngroups, 1), np.uint64) for _ in range(4)] + \
                   [np.zeros(max(c, 1), np.uint64) for c in nerr]
            r = CSjResult()
            r.capacity = ngroups
            for j in range(3):
                r.keys[j] = bufs[j].ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
            r.sums = bufs[3].ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
            for c in range(NCOL):
                r.fact_err[c].data = bufs[4 + c].ctypes.data
                r.fact_err[c].capacity = nerr[c]
            rc = L.ahead_plain_starjoin(self.gpu.ctx, ctypes.byref(self._schema), ctypes.byref(cq), ctypes.byref(r))
            if rc == CAPACITY:
                ngroups = max(ngroups, int(r.ngroups))
                nerr = [max(a, int(r.fact_err[c].count)) for c, a in enumerate(nerr)]
                continue
            self._check(rc, "ahead_plain_starjoin")
            n = int(r.ngroups)
            fe = {FACT_COLS[c]: bufs[4 + c][: int(r.fact_err[c].count)].copy() for c in range(NCOL)}
            if not q.group:
                return FusedResult(OK, [], None, int(r.total), fe)
            return FusedResult(OK, [bufs[j][:n].copy() for j in range(len(q.group))], bufs[3][:n].copy(), None, fe)

    def run(self, queries: Sequence[StarQuery], graph: bool = False) -> List[FusedResult]:
        """One batch, synchronously (graph: replay the captured CUDA graph)."""
        return self.wait(self.submit(queries, graph))

    def answer(self, queries: Sequence[StarQuery], graph: bool = False) -> List[FusedResult]:
        """Fused results; a query outside the fused path's domain is answered
        by the operator-at-a-time composition on the same GPU library."""
        from .gpu import err_to_host, to_host
        from .pipelines import starjoin_continuous
        out = self.run(queries, graph)
        for i, (q, r) in enumerate(zip(queries, out)):
            if r.status != UNSUPPORTED:
                continue
            c = starjoin_continuous(self.gpu, self.schema, q)
            fe = {k: np.zeros(0, np.uint64) for k in FACT_COLS}
            for k, e in c.fact_errors.items():
                v = err_to_host(e).values
                fe[k] = np.zeros(0, np.uint64) if v is None else np.asarray(v, dtype=np.uint64)
            keys = [np.asarray(to_host(k).tail.data, dtype=np.uint64) for k in c.keys]
            sums = None if c.sums is None else np.asarray(to_host(c.sums).tail.data, dtype=np.uint64)
            out[i] = FusedResult(OK, keys, sums, c.total, fe)
        return out
