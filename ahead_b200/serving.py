"""The serving loop of the fused star-join engine (ahead_sj_server_* in
include/ahead_gpu.h) from Python: requests go in by `submit` or as an
open-loop `replay` of scheduled arrivals; completions come back with their
arrival, batch-start and done times on the server's clock."""
from __future__ import annotations

import ctypes
import sys
from dataclasses import dataclass
from typing import Dict, List, Sequence

import numpy as np

from .gpu import AheadError
from .model import OK
from .ssb import StarQuery
from .starjoin import FACT_COLS, CSjQuery, CSjResult, FusedResult, StarJoinEngine, c_query


class CSjServerCfg(ctypes.Structure):
    _fields_ = [("window_ms", ctypes.c_double), ("max_batch", ctypes.c_int32), ("use_graph", ctypes.c_int32),
                ("hbm_budget", ctypes.c_uint64), ("max_groups", ctypes.c_uint64), ("max_errors", ctypes.c_uint64)]


class CSjDone(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("arrival_us", ctypes.c_double), ("start_us", ctypes.c_double),
                ("done_us", ctypes.c_double), ("batch_size", ctypes.c_uint32), ("_pad", ctypes.c_int32),
                ("result", CSjResult)]


class CSjServerStats(ctypes.Structure):
    _fields_ = [("batches", ctypes.c_uint64), ("requests", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("busy_ms", ctypes.c_double), ("mean_batch", ctypes.c_double),
                ("max_inflight_bytes_frac_pct", ctypes.c_uint32), ("_pad", ctypes.c_uint32)]


@dataclass
class Completion:
    id: int
    arrival_us: float
    start_us: float
    done_us: float
    batch_size: int
    result: FusedResult

    @property
    def latency_ms(self) -> float:
        return (self.done_us - self.arrival_us) / 1e3


class StarJoinServer:
    def __init__(self, engine: StarJoinEngine, window_ms: float = 2.0, max_batch: int = 64, use_graph: bool = True,
                 hbm_budget: int = 150 << 30, max_groups: int = 4096, max_errors: int = 8192):
        self.engine = engine
        self.lib = engine.lib
        L = self.lib
        L.ahead_sj_server_create.argtypes = [ctypes.c_void_p, ctypes.POINTER(CSjServerCfg),
                                             ctypes.POINTER(ctypes.c_void_p)]
        L.ahead_sj_server_destroy.argtypes = [ctypes.c_void_p]
        L.ahead_sj_server_submit.argtypes = [ctypes.c_void_p, ctypes.POINTER(CSjQuery),
                                             ctypes.POINTER(ctypes.c_uint64)]
        L.ahead_sj_server_replay.argtypes = [ctypes.c_void_p, ctypes.POINTER(CSjQuery),
                                             ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_uint64)]
        L.ahead_sj_server_poll.argtypes = [ctypes.c_void_p, ctypes.POINTER(CSjDone), ctypes.c_int, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_int)]
        L.ahead_sj_server_release.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
        L.ahead_sj_server_stats_get.argtypes = [ctypes.c_void_p, ctypes.POINTER(CSjServerStats)]
        L.ahead_sj_server_now_us.argtypes = [ctypes.c_void_p]
        L.ahead_sj_server_now_us.restype = ctypes.c_double
        cfg = CSjServerCfg(window_ms, max_batch, int(use_graph), hbm_budget, max_groups, max_errors)
        self.srv = ctypes.c_void_p()
        self._check(L.ahead_sj_server_create(engine.eng, ctypes.byref(cfg), ctypes.byref(self.srv)),
                    "ahead_sj_server_create")
        self.queries: Dict[int, StarQuery] = {}
        self._done = (CSjDone * 256)()

    def _check(self, rc, what):
        if rc != OK:
            raise AheadError(rc, what, self.lib.ahead_ctx_last_error(self.engine.gpu.ctx).decode())

    def close(self):
        if self.srv:
            self.lib.ahead_sj_server_destroy(self.srv)
            self.srv = ctypes.c_void_p()

    def __del__(self, _finalizing=sys.is_finalizing):  # bound now: module globals may be gone at exit
        if _finalizing():  # the CUDA runtime may be gone; the process frees everything
            return
        try:
            self.close()
        except Exception:
            pass

    def now_us(self) -> float:
        return float(self.lib.ahead_sj_server_now_us(self.srv))

    def submit(self, q: StarQuery) -> int:
        cq = c_query(q, self.engine.schema)
        i = ctypes.c_uint64()
        self._check(self.lib.ahead_sj_server_submit(self.srv, ctypes.byref(cq), ctypes.byref(i)),
                    "ahead_sj_server_submit")
        self.queries[i.value] = q
        return i.value

    def replay(self, queries: Sequence[StarQuery], arrival_us: Sequence[float]) -> List[int]:
        n = len(queries)
        cqs = (CSjQuery * n)(*[c_query(q, self.engine.schema) for q in queries])
        arr = (ctypes.c_double * n)(*[float(a) for a in arrival_us])
        first = ctypes.c_uint64()
        self._check(self.lib.ahead_sj_server_replay(self.srv, cqs, arr, n, ctypes.byref(first)),
                    "ahead_sj_server_replay")
        ids = list(range(first.value, first.value + n))
        for i, q in zip(ids, queries):
            self.queries[i] = q
        return ids

    def poll(self, wait_ms: int = 100) -> List[Completion]:
        n = ctypes.c_int()
        self._check(self.lib.ahead_sj_server_poll(self.srv, self._done, len(self._done), wait_ms, ctypes.byref(n)),
                    "ahead_sj_server_poll")
        out = []
        for k in range(n.value):
            d = self._done[k]
            q = self.queries.pop(d.id)
            r = d.result
            fe = {FACT_COLS[c]: np.ctypeslib.as_array(ctypes.cast(r.fact_err[c].data, ctypes.POINTER(ctypes.c_uint64)),
                                                      (int(r.fact_err[c].capacity),)).copy()
                  if r.fact_err[c].capacity else np.zeros(0, np.uint64) for c in range(len(FACT_COLS))}
            if r.status != OK:
                res = FusedResult(int(r.status), [], None, None, fe)
            elif not q.group:
                res = FusedResult(OK, [], None, int(r.total), fe)
            else:
                ng = int(r.capacity)
                take = lambda p: (np.ctypeslib.as_array(p, (ng,)).copy() if ng else np.zeros(0, np.uint64))
                res = FusedResult(OK, [take(r.keys[j]) for j in range(len(q.group))], take(r.sums), None, fe)
            out.append(Completion(int(d.id), d.arrival_us, d.start_us, d.done_us, int(d.batch_size), res))
            self.lib.ahead_sj_server_release(self.srv, d.id)
        return out

    def collect(self, ids: Sequence[int], timeout_s: float = 120.0) -> Dict[int, Completion]:
        import time
        want = set(ids)
        got: Dict[int, Completion] = {}
        t_end = time.monotonic() + timeout_s
        while want - got.keys():
            if time.monotonic() > t_end:
                raise TimeoutError(f"{len(want - got.keys())} requests unfinished")
            for c in self.poll(100):
                got[c.id] = c
        return got

    def stats(self) -> CSjServerStats:
        st = CSjServerStats()
        self._check(self.lib.ahead_sj_server_stats_get(self.srv, ctypes.byref(st)), "ahead_sj_server_stats_get")
        return st


def poisson_arrivals(rate_qps: float, n: int, seed: int) -> np.ndarray:
    """Arrival times in microseconds of a Poisson stream (exponential gaps)."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1e6 / rate_qps, n))
