"""Fact-sharded star joins over the ranks of a job (one process per GPU).

Every rank holds the dimension tables whole and one contiguous range of the
lineorder rows: rank r of W holds rows [o_r, o_r + n_r), the ranges in rank
order and aligned to 4,096 rows.  A batch is answered by every rank over its
own rows -- a query over the prefix [0, P) reads the local prefix
[0, clamp(P - o_r, 0, n_r)) -- and one exchange step combines the per-rank
results into the result of the whole table:

* per-group AN-coded sums and ungrouped totals add modulo 2^64: the codes
  are linear in the rows (A * sum = sum of A * x, wrapping as the
  reference's u64 arithmetic wraps);
* groups come out in first-occurrence order: the ranks hold ascending row
  ranges, so the order of the whole table is rank 0's groups, then each later
  rank's groups not seen before, in that rank's order;
* error positions are row * A_OID: a rank's local positions move by
  o_r * A_OID (mod 2^64) and concatenate in rank order, which is ascending
  row order, as the single-table scan pushes them.

Every step of the composition the reference's programs run is local to one
fact row (the first join probes each row's key, the later joins and the
measure fetches are positional in row order, a corrupt value drops its own
row), so this combination is exact; tests/test_sharded.py checks it against
the unsharded result on the CPU (two gloo ranks) and on the GPU (shards of one
device).

The exchange is two all_gathers per batch (the packed sizes, then the packed
results padded to the largest) over the job's process group: NCCL on GPUs,
gloo on CPUs.  An all-reduce of per-group sums over a dense group index (the
survey's sketch) gives the same sums but not the group order or the error
lists; the gather carries all three in one step.
"""
from __future__ import annotations

import dataclasses
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from .model import AOID_DEFAULT, OK, Bat, Col
from .ssb import FACT_COLS, StarQuery, StarSchema

ALIGN = 4096
_M64 = (1 << 64) - 1


@dataclasses.dataclass
class Part:
    """One query's result over some rows (the fused engine's FusedResult
    fields): group attribute codes, AN-coded sums or total, error positions."""
    status: int
    keys: List[np.ndarray]
    sums: Optional[np.ndarray]
    total: Optional[int]
    fact_errors: dict


def shard_rows(total: int, world: int, rank: int, align: int = ALIGN) -> Tuple[int, int]:
    """(first row, rows) of `rank`'s contiguous range of `total` fact rows."""
    per = -(-total // world)
    per = -(-per // align) * align
    lo = min(total, rank * per)
    return lo, min(total, lo + per) - lo


def _slice(b: Bat, lo: int, n: int) -> Bat:
    from .model import WIDTH
    t = b.tail
    w = WIDTH[t.type]
    data = t.data[lo * w:(lo + n) * w] if hasattr(t.data, "data_ptr") else t.data[lo:lo + n]
    return Bat(b.head, Col(t.type, data, t.A, t.Ainv, t.unenc_max, t.seqbase), n)


def shard_schema(schema: StarSchema, lo: int, n: int) -> StarSchema:
    """The schema with lineorder cut to rows [lo, lo + n) (views, no copies)."""
    t = dict(schema.tables)
    t["lineorder"] = {c: _slice(b, lo, n) for c, b in schema.tables["lineorder"].items()}
    return StarSchema(t, {**schema.sizes, "fact": n})


def local_prefix(q: StarQuery, full: int, lo: int, n: int) -> int:
    """Rows of this shard inside the query's prefix."""
    p = q.fact_rows or full
    return max(0, min(p - lo, n))


def empty_part(q: StarQuery) -> Part:
    return Part(OK, [np.zeros(0, np.uint64) for _ in q.group], np.zeros(0, np.uint64) if q.group else None,
                None if q.group else 0, {c: np.zeros(0, np.uint64) for c in FACT_COLS})


# ------------------------------------------------------------------ packing
def pack(parts: Sequence[Part], queries: Sequence[StarQuery]) -> np.ndarray:
    """One uint64 buffer: per query [status, total, ngroups, an error count
    per fact column] then the key columns, the sums and the error vectors."""
    out = []
    for p, q in zip(parts, queries):
        ng = len(p.sums) if p.sums is not None else 0
        errs = [np.asarray(p.fact_errors.get(c, np.zeros(0)), dtype=np.uint64) for c in FACT_COLS]
        out.append(np.array([p.status & _M64, (p.total or 0) & _M64, ng] + [len(e) for e in errs], dtype=np.uint64))
        for k in range(len(q.group)):
            out.append(np.asarray(p.keys[k][:ng], dtype=np.uint64))
        if ng:
            out.append(np.asarray(p.sums, dtype=np.uint64))
        out.extend(errs)
    return np.concatenate(out) if out else np.zeros(0, np.uint64)


def unpack(buf: np.ndarray, queries: Sequence[StarQuery]) -> List[Part]:
    parts, i = [], 0
    for q in queries:
        nh = 3 + len(FACT_COLS)
        h = buf[i:i + nh]
        i += nh
        status, total, ng = int(h[0]), int(h[1]), int(h[2])
        cnt = [int(x) for x in h[3:nh]]
        keys = []
        for _ in q.group:
            keys.append(buf[i:i + ng].copy())
            i += ng
        sums = None
        if q.group:
            sums = buf[i:i + ng].copy()
            i += ng
        errs = {}
        for c, k in zip(FACT_COLS, cnt):
            errs[c] = buf[i:i + k].copy()
            i += k
        parts.append(Part(status, keys, sums, None if q.group else total, errs))
    return parts


# ------------------------------------------------------------------ combine
def combine(parts: Sequence[Part], offsets: Sequence[int], q: StarQuery, aoid: int = AOID_DEFAULT) -> Part:
    """The whole table's result from per-shard results in shard order."""
    bad = [p.status for p in parts if p.status != OK]
    errs = {}
    for c in FACT_COLS:
        vs = [(np.asarray(p.fact_errors.get(c, np.zeros(0)), dtype=np.uint64) + np.uint64((o * aoid) & _M64))
              for p, o in zip(parts, offsets)]
        errs[c] = np.concatenate(vs) if vs else np.zeros(0, np.uint64)
    if bad:
        return Part(bad[0], [], None, None, errs)
    if not q.group:
        return Part(OK, [], None, sum(int(p.total or 0) for p in parts) & _M64, errs)
    nk = len(q.group)
    keys = [np.concatenate([p.keys[k] for p in parts]) for k in range(nk)]
    sums = np.concatenate([p.sums for p in parts])
    if len(sums) == 0:
        return Part(OK, [np.zeros(0, np.uint64) for _ in range(nk)], np.zeros(0, np.uint64), None, errs)
    rec = np.stack(keys, axis=1)
    _, first, inv = np.unique(rec, axis=0, return_index=True, return_inverse=True)
    inv = inv.reshape(-1)
    order = np.argsort(first, kind="stable")          # groups by first occurrence
    rank_of = np.empty(len(order), dtype=np.int64)
    rank_of[order] = np.arange(len(order))
    out_sums = np.zeros(len(order), dtype=np.uint64)
    np.add.at(out_sums, rank_of[inv], sums)           # uint64 wraps modulo 2^64
    out_keys = [k[np.sort(first)] for k in keys]
    return Part(OK, out_keys, out_sums, None, errs)


class ShardedStarJoin:
    """Answers batches over this rank's fact rows and combines them with the
    other ranks' in one exchange.  `answer(local_queries)` returns the local
    Parts (the fused engine's `answer`, or any composition); `group` is the
    job's Replicas (None for one process)."""

    def __init__(self, answer: Callable[[List[StarQuery]], List[Part]], full_rows: int, lo: int, n: int,
                 group=None, device: str = "cpu", aoid: int = AOID_DEFAULT):
        self.answer_local, self.full, self.lo, self.n = answer, full_rows, lo, n
        self.group, self.device, self.aoid = group, device, aoid

    def local(self, queries: Sequence[StarQuery]) -> List[Part]:
        """This rank's part of every query (empty where its rows lie past a prefix)."""
        todo, where = [], []
        for i, q in enumerate(queries):
            p = local_prefix(q, self.full, self.lo, self.n)
            if p:
                todo.append(dataclasses.replace(q, fact_rows=p))
                where.append(i)
        parts = [empty_part(q) for q in queries]
        if todo:
            for i, r in zip(where, self.answer_local(todo)):
                parts[i] = Part(r.status, list(r.keys), r.sums, r.total, dict(r.fact_errors))
        return parts

    def exchange(self, parts: List[Part], queries: Sequence[StarQuery]) -> List[List[Part]]:
        """Every rank's parts, in rank order (two all_gathers)."""
        buf = pack(parts, queries)
        g = self.group
        if g is None or g.world == 1:
            return [parts]
        import torch
        dist = g._dist
        dev = self.device
        n = torch.tensor([len(buf)], dtype=torch.int64, device=dev)
        ns = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(g.world)]
        dist.all_gather(ns, n)
        ns = [int(x.item()) for x in ns]
        m = max(ns)
        mine = torch.zeros(m, dtype=torch.int64, device=dev)
        if len(buf):
            mine[:len(buf)] = torch.from_numpy(buf.view(np.int64)).to(dev)
        got = [torch.zeros(m, dtype=torch.int64, device=dev) for _ in range(g.world)]
        dist.all_gather(got, mine)
        return [unpack(t[:k].cpu().numpy().view(np.uint64), queries) for t, k in zip(got, ns)]

    def offsets(self) -> List[int]:
        g = self.group
        w = 1 if g is None else g.world
        return [shard_rows(self.full, w, r)[0] for r in range(w)]

    def run(self, queries: Sequence[StarQuery]) -> List[Part]:
        """The whole table's results, on every rank."""
        mine = self.local(queries)
        if self.group is None or self.group.world == 1:
            return mine  # one shard from row 0: its results are the table's
        everyone = self.exchange(mine, queries)
        offs = self.offsets()
        return [combine([ps[i] for ps in everyone], offs, q, self.aoid) for i, q in enumerate(queries)]


def star_to_part(c, to_host=None, err_to_host=None) -> Part:
    """A pipelines.StarResult (host or device BATs) as a Part."""
    h = to_host or (lambda b: b)
    e = err_to_host or (lambda x: x)
    fe = {k: np.zeros(0, np.uint64) for k in FACT_COLS}
    for k, v in c.fact_errors.items():
        vals = e(v).values
        fe[k] = np.zeros(0, np.uint64) if vals is None else np.asarray(vals, dtype=np.uint64)
    keys = [np.asarray(h(k).tail.data, dtype=np.uint64)[: h(k).count] for k in c.keys]
    sums = None if c.sums is None else np.asarray(h(c.sums).tail.data, dtype=np.uint64)[: c.ngroups]
    return Part(OK, keys, sums, c.total, fe)


# ------------------------------------------------------------------ device exchange
# The fused engine's form of the same combination (ahead_sj_submit_local /
# ahead_sj_submit_final): every engine exports its dense per-query group
# tables -- AN-coded sums and first rows (rows of the whole table), int64 --
# its status flags and its error log; one all-reduce SUM of the sums (int64
# adds wrap mod 2^64 like the reference's u64 sums), one MIN of the first rows,
# one MAX of the flags and one all-gather of the logs combine them, all on the
# device; each engine then orders groups and errors of the whole table
# itself.  The group slots are the same on every engine: the batch plan
# depends on the queries and the dimensions only.

def device_int64(ptr: int, n: int):
    """A torch int64 tensor aliasing `n` words of device memory at `ptr` (the
    engine owns the memory; the tensor only names it)."""
    import torch

    class _Area:
        pass

    a = _Area()
    a.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<i8", "data": (int(ptr), False), "version": 3,
                                  "strides": None}
    return torch.as_tensor(a, device="cuda")


def xchg_tensors(x):
    """(sums, firsts, flags, log) tensors of an engine's exchange area."""
    return (device_int64(x.sums, x.groups), device_int64(x.firsts, x.groups), device_int64(x.flags, 4),
            device_int64(x.log, 1 + x.log_cap))


def exchange(tensors, dist, world: int):
    """The collectives of one batch over a process group: in place on the
    sums (SUM), first rows (MIN) and flags (MAX); returns the gathered logs,
    `world` areas in rank order, as one contiguous tensor.  Every rank calls
    it with its own tensors, in the same batch order."""
    import torch
    sums, firsts, flags, log = tensors
    dist.all_reduce(sums, op=dist.ReduceOp.SUM)
    dist.all_reduce(firsts, op=dist.ReduceOp.MIN)
    dist.all_reduce(flags, op=dist.ReduceOp.MAX)
    parts = [torch.empty_like(log) for _ in range(world)]
    dist.all_gather(parts, log)
    return torch.cat(parts)


def exchange_on_one_device(areas):
    """The same combination for engines that share one device (each a shard
    of one table): the combined tables written back into every area; returns
    the gathered logs."""
    import torch
    ts = [xchg_tensors(x) for x in areas]
    sums = ts[0][0].clone()
    firsts = ts[0][1].clone()
    flags = ts[0][2].clone()
    for s, f, g, _ in ts[1:]:
        sums += s  # int64 wraps mod 2^64
        torch.minimum(firsts, f, out=firsts)
        torch.maximum(flags, g, out=flags)
    for s, f, g, _ in ts:
        s.copy_(sums)
        f.copy_(firsts)
        g.copy_(flags)
    return torch.cat([t[3] for t in ts])


class EngineShardedStarJoin:
    """Fact-sharded batches through the fused engine, the exchange on the
    device: `eng` holds this rank's rows [lo, lo + n) of a table of `full_rows`
    rows (set_shard is applied here); `group` is the job's Replicas.  Two
    batches are in flight (`step`): a batch's local half is queued before the
    previous batch's final half, so its scan overlaps that batch's exchange."""

    def __init__(self, eng, full_rows: int, lo: int, group=None):
        import torch
        self.eng, self.group = eng, group
        self.world = 1 if group is None else group.world
        eng.set_shard(lo, full_rows)
        self.stream = eng.gpu.stream()
        self._prev = None  # (ticket, gathered logs) whose final half is not submitted yet
        self._logs = {}  # ticket -> gathered logs, alive until the batch is collected
        self._inflight = []  # tickets submitted and not collected, oldest first
        self._torch = torch

    def _exchange(self, x):
        torch = self._torch
        ts = xchg_tensors(x)
        if self.world == 1:
            return ts[3]  # one engine: its own tables and log
        ready = torch.cuda.Event()
        ready.record(self.stream)
        cur = torch.cuda.current_stream()
        cur.wait_event(ready)
        gathered = exchange(ts, self.group._dist, self.world)
        done = torch.cuda.Event()
        done.record(cur)
        self.stream.wait_event(done)
        return gathered

    def step(self, queries):
        """Queue a batch: collect the batch two steps back (its slot is this
        batch's; its final half is already queued), then this batch's local
        half and exchange, then the previous batch's final half behind this
        scan.  Returns the collected batch's results (None while the pipeline
        fills).  The device then holds this scan and the previous final half
        while the caller works on the returned results."""
        done = None
        if len(self._inflight) == 2:
            done = self.wait(self._inflight.pop(0))
        t, x = self.eng.submit_local(queries, graph=True)
        g = self._exchange(x)
        prev, self._prev = self._prev, (t, g)
        self._final(prev)
        self._inflight.append(t)
        return done

    def drain(self):
        """The final half of the last batch, then every batch still in flight."""
        prev, self._prev = self._prev, None
        self._final(prev)
        out = [self.wait(t) for t in self._inflight]
        self._inflight = []
        return out

    def _final(self, prev):
        if prev is None:
            return None
        t, g = prev
        self._logs[t] = g  # alive until its final half has read it
        self.eng.submit_final(t, g.data_ptr(), self.world)
        return t

    def wait(self, ticket):
        out = self.eng.wait(ticket)
        self._logs.pop(ticket, None)
        return out

    def run(self, queries):
        """One batch, synchronously: the whole table's results on every rank."""
        if self._inflight:
            raise RuntimeError("run() with batches in flight")
        self.step(queries)
        return self.drain()[0]
