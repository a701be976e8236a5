"""Fact-sharded star joins (ahead_b200/sharded.py): per-shard results combined
in one exchange equal the result over the whole table.

CPU: shard ranges, the packed exchange format, the combination of per-shard
oracle results for 1-3 shards (bit flips, prefixes that end inside a shard,
grouped and ungrouped queries), and two gloo ranks running the exchange.
GPU: the fused engine on three shards of one device's schema, combined,
against the engine on the whole schema.
"""
import os
import socket
import sys

import numpy as np
import pytest

from ahead_b200.sharded import (FACT_COLS, ShardedStarJoin, combine, local_prefix, pack, shard_rows, shard_schema,
                                star_to_part, unpack)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SIZES = dict(fact=50_000, date=2556, customer=300, part=2000, supplier=40)
FACT = ("orderdate", "custkey", "partkey", "suppkey", "price", "discount")


def _schema(seed=4, flips=5):
    from ahead_b200.ssb import generate, inject_flips
    s = generate(SIZES, seed=seed)
    for i, c in enumerate(FACT):
        inject_flips(s, "lineorder", c, flips, seed=seed + 50 + i)
    return s


def _queries(seed=9, n=10):
    from ahead_b200.ssb import random_query
    rng = np.random.default_rng(seed)
    qs = [random_query(rng, fact_sizes=(7_000, 23_000, 41_000, 50_000), max_fact=50_000) for _ in range(n)]
    return qs


def _same(a, b):
    assert a.status == b.status
    assert (a.total is None) == (b.total is None) and (a.total is None or int(a.total) == int(b.total))
    assert (a.sums is None) == (b.sums is None)
    if a.sums is not None:
        assert np.array_equal(np.asarray(a.sums, np.uint64), np.asarray(b.sums, np.uint64))
        assert len(a.keys) == len(b.keys)
        for x, y in zip(a.keys, b.keys):
            assert np.array_equal(np.asarray(x, np.uint64), np.asarray(y, np.uint64))
    for c in FACT_COLS:
        assert np.array_equal(np.asarray(a.fact_errors[c], np.uint64), np.asarray(b.fact_errors[c], np.uint64)), c


def test_shard_rows_cover_the_table():
    for total in (0, 1, 4095, 4096, 50_000, 600_000_000):
        for world in (1, 2, 3, 8):
            got = [shard_rows(total, world, r) for r in range(world)]
            assert sum(n for _, n in got) == total
            pos = 0
            for lo, n in got:
                assert lo == pos or n == 0
                assert lo % 4096 == 0 or n == 0
                pos = lo + n


def test_pack_round_trip():
    from ahead_b200.sharded import Part
    from ahead_b200.ssb import StarQuery
    q1 = StarQuery(preds=[], group=[("date", "year"), ("part", "category")])
    q2 = StarQuery(preds=[], group=[])
    rng = np.random.default_rng(1)
    p1 = Part(0, [rng.integers(0, 2 ** 63, 5, dtype=np.uint64) for _ in range(2)],
              rng.integers(0, 2 ** 63, 5, dtype=np.uint64), None,
              {c: rng.integers(0, 2 ** 63, i, dtype=np.uint64) for i, c in enumerate(FACT_COLS)})
    p2 = Part(0, [], None, 2 ** 64 - 3, {c: np.zeros(0, np.uint64) for c in FACT_COLS})
    back = unpack(pack([p1, p2], [q1, q2]), [q1, q2])
    _same(back[0], p1)
    _same(back[1], p2)


@pytest.mark.parametrize("world", [1, 2, 3])
def test_combined_shards_equal_whole_table(world):
    """The oracle composition per shard, combined, against the oracle on the
    whole table."""
    from ahead_b200.pipelines import starjoin_continuous
    from oracle.oracle import Oracle
    port = Oracle("port")
    s = _schema()
    qs = _queries()
    full = [star_to_part(starjoin_continuous(port, s, q)) for q in qs]
    shards = [shard_rows(SIZES["fact"], world, r) for r in range(world)]

    def answer_on(lo, n):
        sub = shard_schema(s, lo, n)
        return lambda todo: [star_to_part(starjoin_continuous(port, sub, q)) for q in todo]

    per = [ShardedStarJoin(answer_on(lo, n), SIZES["fact"], lo, n).local(qs) for lo, n in shards]
    for i, q in enumerate(qs):
        assert any(local_prefix(q, SIZES["fact"], lo, n) for lo, n in shards)
        _same(combine([p[i] for p in per], [lo for lo, _ in shards], q), full[i])
    # the flips do reach the compared error vectors
    assert sum(len(f.fact_errors[c]) for f in full for c in FACT_COLS) > 0


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from test_sharded import SIZES as S, _queries as Q, _schema as SCH

    from ahead_b200.pipelines import starjoin_continuous
    from ahead_b200.replicas import Replicas
    from ahead_b200.sharded import ShardedStarJoin, pack, shard_rows, shard_schema, star_to_part
    from oracle.oracle import Oracle
    g = Replicas("gloo", timeout_s=120)
    port_ops = Oracle("port")
    lo, n = shard_rows(S["fact"], world, rank)
    sub = shard_schema(SCH(), lo, n)
    sj = ShardedStarJoin(lambda todo: [star_to_part(starjoin_continuous(port_ops, sub, x)) for x in todo],
                         S["fact"], lo, n, group=g)
    qs = Q()
    res = sj.run(qs)
    q.put((rank, pack(res, qs).tobytes()))
    g.close()


def test_two_ranks_over_gloo():
    import torch.multiprocessing as mp

    from ahead_b200.pipelines import starjoin_continuous
    from oracle.oracle import Oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    qs = _queries()
    s = _schema()
    ora = Oracle("port")
    full = [star_to_part(starjoin_continuous(ora, s, x)) for x in qs]
    assert got[0] == got[1]  # every rank holds the whole result
    back = unpack(np.frombuffer(got[0], dtype=np.uint64), qs)
    for a, b in zip(back, full):
        _same(a, b)


@pytest.mark.gpu
def test_gpu_shards_of_one_device_equal_whole_table():
    """Three engines over three row ranges of one device's schema, combined,
    against one engine over the whole schema (fused path, flips included)."""
    import torch

    from ahead_b200.gpu import GpuOps
    from ahead_b200.ssb import generate_device, random_query
    from ahead_b200.starjoin import StarJoinEngine
    sizes = dict(fact=3_000_000, date=2556, customer=30_000, part=200_000, supplier=2_000)
    s = generate_device(sizes, seed=3, flips=40, flip_seed=8)
    rng = np.random.default_rng(5)
    qs = [random_query(rng, fact_sizes=(300_000, 1_000_000, 2_100_000, 3_000_000), max_fact=3_000_000)
          for _ in range(24)]
    g = GpuOps(0)
    whole = StarJoinEngine(g, s)
    ref = whole.answer(qs)
    whole.close()
    world = 3
    per = []
    for r in range(world):
        lo, n = shard_rows(sizes["fact"], world, r)
        eng = StarJoinEngine(g, shard_schema(s, lo, n))
        per.append(ShardedStarJoin(lambda todo, e=eng: e.answer(todo), sizes["fact"], lo, n).local(qs))
        eng.close()
    offs = [shard_rows(sizes["fact"], world, r)[0] for r in range(world)]
    nerr = 0
    for i, q in enumerate(qs):
        c = combine([p[i] for p in per], offs, q)
        _same(c, ref[i])
        nerr += sum(len(c.fact_errors[k]) for k in FACT_COLS)
    assert nerr > 0
    torch.cuda.synchronize()
    g.close()


def test_combine_rules():
    """The exchange's combination on hand-made parts: sums and totals wrap
    modulo 2^64, groups keep first-occurrence order across shards, error
    positions move by the shard's first row times A_OID, a failed shard's
    status wins."""
    from ahead_b200.sharded import Part
    from ahead_b200.ssb import StarQuery
    M = 1 << 64
    none = {c: np.zeros(0, np.uint64) for c in FACT_COLS}
    q = StarQuery(preds=[], group=[])
    parts = [Part(0, [], None, M - 5, dict(none)), Part(0, [], None, 9, dict(none))]
    assert combine(parts, [0, 4096], q).total == 4
    g = StarQuery(preds=[], group=[("date", "year"), ("part", "category")])
    k = lambda *xs: np.array(xs, dtype=np.uint64)
    p0 = Part(0, [k(7, 3), k(1, 2)], k(M - 1, 10), None, {**none, "price": k(5 * 16089)})
    p1 = Part(0, [k(9, 7, 3), k(4, 1, 2)], k(1, 2, 3), None, {**none, "price": k(0, 16089)})
    c = combine([p0, p1], [0, 4096], g)
    assert [list(x) for x in c.keys] == [[7, 3, 9], [1, 2, 4]]       # (7,1), (3,2) from shard 0, then (9,4)
    assert list(c.sums) == [(M - 1 + 2) % M, 10 + 3, 1]
    assert list(c.fact_errors["price"]) == [5 * 16089, 4096 * 16089, 4097 * 16089]
    bad = Part(2, [], None, None, dict(none))
    assert combine([p0, bad], [0, 4096], g).status == 2


def _xchg_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    from ahead_b200.sharded import exchange
    dist.init_process_group("gloo", rank=rank, world_size=world)
    M = 1 << 64
    groups = 5
    # rank r: sums near the top of u64 (they wrap), first rows (INT64_MAX: none), flags, a log of r + 2 entries
    sums = torch.tensor([((M - 3 + 7 * rank + i) % M) - (M if ((M - 3 + 7 * rank + i) % M) >= M // 2 else 0)
                         for i in range(groups)], dtype=torch.int64)
    firsts = torch.tensor([100 * (world - rank) + i if i != 2 else 2 ** 63 - 1 for i in range(groups)],
                          dtype=torch.int64)
    flags = torch.tensor([rank == 1, 0, 0, rank == 0], dtype=torch.int64)
    cap = 6
    log = torch.zeros(1 + cap, dtype=torch.int64)
    log[0] = rank + 2
    log[1:rank + 3] = torch.arange(rank + 2) + 1000 * (rank + 1)
    g = exchange((sums, firsts, flags, log), dist, world)
    q.put((rank, sums.tolist(), firsts.tolist(), flags.tolist(), g.tolist()))
    dist.destroy_process_group()


def test_device_exchange_collectives_over_gloo():
    """The device exchange's collectives (ahead_b200.sharded.exchange) on two
    gloo ranks: group sums add with wrap-around mod 2^64, first rows take the
    minimum with INT64_MAX as "none", flags the maximum, and the error logs
    arrive in rank order on every rank."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 2
    procs = [ctx.Process(target=_xchg_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = {r: rest for r, *rest in (q.get(timeout=300) for _ in range(world))}
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    M = 1 << 64
    assert got[0] == got[1]
    sums, firsts, flags, gathered = got[0]
    assert [s % M for s in sums] == [((M - 3 + i) + (M - 3 + 7 + i)) % M for i in range(5)]
    assert firsts == [100 + i if i != 2 else 2 ** 63 - 1 for i in range(5)]
    assert flags == [1, 0, 0, 1]
    assert gathered[:7] == [2, 1000, 1001, 0, 0, 0, 0]
    assert gathered[7:] == [3, 2000, 2001, 2002, 0, 0, 0]


@pytest.mark.gpu
def test_gpu_engine_shards_exchange_on_the_device():
    """The fused engine's own sharded form: three engines over three row
    ranges of one device's schema (set_shard), local halves, the exchange
    combined on the device, final halves; every engine's results equal one
    engine over the whole schema -- groups in first-occurrence order of the
    whole table, error positions of the whole table -- in both strategies,
    launched directly and from graphs."""
    import torch

    from ahead_b200.gpu import GpuOps
    from ahead_b200.sharded import exchange_on_one_device
    from ahead_b200.ssb import generate_device, random_query
    from ahead_b200.starjoin import StarJoinEngine
    sizes = dict(fact=3_000_000, date=2556, customer=30_000, part=200_000, supplier=2_000)
    s = generate_device(sizes, seed=3, flips=400, flip_seed=8)
    rng = np.random.default_rng(5)
    qs = [random_query(rng, fact_sizes=(300_000, 1_000_000, 2_100_000, 3_000_000), max_fact=3_000_000)
          for _ in range(24)]
    g = GpuOps(0)
    whole = StarJoinEngine(g, s)
    world = 3
    engines = []
    for r in range(world):
        lo, n = shard_rows(sizes["fact"], world, r)
        e = StarJoinEngine(g, shard_schema(s, lo, n))
        e.set_shard(lo, sizes["fact"])
        engines.append(e)
    nerr = 0
    for strategy in (0, 1):
        for e in engines + [whole]:
            e.set_strategy(strategy)
        ref = whole.run(qs, graph=True)
        for graph in (False, True):
            halves = [e.submit_local(qs, graph=graph) for e in engines]
            torch.cuda.synchronize()
            logs = exchange_on_one_device([x for _, x in halves])
            torch.cuda.synchronize()
            for e, (t, _) in zip(engines, halves):
                e.submit_final(t, logs.data_ptr(), world)
                got = e.wait(t)
                for a, b in zip(got, ref):
                    assert a.status == b.status == 0
                    assert (a.total is None) == (b.total is None) and a.total == b.total
                    if b.sums is not None:
                        assert np.array_equal(a.sums, b.sums)
                        assert all(np.array_equal(x, y) for x, y in zip(a.keys, b.keys))
                    for c in FACT_COLS:
                        assert np.array_equal(a.fact_errors[c], b.fact_errors[c]), c
                        nerr += len(b.fact_errors[c])
    assert nerr > 0
    # a shard answers whole-table queries only through the exchange
    from ahead_b200.gpu import AheadError
    with pytest.raises(AheadError):
        engines[1].run(qs[:2])
    for e in engines + [whole]:
        e.close()
    g.close()


@pytest.mark.gpu
def test_gpu_engine_sharded_runner_pipelined():
    """EngineShardedStarJoin with one rank (the whole table) keeps two batches
    in flight -- a batch's local half ahead of the previous batch's final
    half -- and returns what the engine's ordinary path returns."""
    from ahead_b200.gpu import GpuOps
    from ahead_b200.sharded import EngineShardedStarJoin
    from ahead_b200.ssb import generate_device, random_query
    from ahead_b200.starjoin import StarJoinEngine
    sizes = dict(fact=2_000_000, date=2556, customer=30_000, part=200_000, supplier=2_000)
    s = generate_device(sizes, seed=6, flips=200, flip_seed=2)
    rng = np.random.default_rng(8)
    batches = [[random_query(rng, fact_sizes=(500_000, 2_000_000), max_fact=2_000_000) for _ in range(16)]
               for _ in range(4)]
    g = GpuOps(0)
    plain = StarJoinEngine(g, s)
    want = [plain.run(b, graph=True) for b in batches]
    plain.close()
    sj = EngineShardedStarJoin(StarJoinEngine(g, s), sizes["fact"], 0)
    got = []
    for b in batches:
        r = sj.step(b)
        if r is not None:
            got.append(r)
    got += sj.drain()
    assert len(got) == len(batches)
    assert len(sj.run(batches[0])) == 16
    for gb, wb in zip(got, want):
        for a, b in zip(gb, wb):
            assert a.status == b.status and a.total == b.total
            if b.sums is not None:
                assert np.array_equal(a.sums, b.sums)
            for c in FACT_COLS:
                assert np.array_equal(a.fact_errors[c], b.fact_errors[c])
    sj.eng.close()
    g.close()
