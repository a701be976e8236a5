"""Star-join pipelines: the reference composition of AN operators on the
CPU oracle (restatement and, where built, the reference itself), and the same
composition run operator by operator on the GPU library."""
import os

import numpy as np
import pytest

from ahead_b200.model import WIDTH, ErrVec
from ahead_b200.pipelines import starjoin_continuous
from ahead_b200.ssb import StarQuery, config2_query, generate, inject_flips, random_query
from oracle.oracle import REF_LIB, Oracle

TINY = dict(fact=20_000, date=2556, customer=300, part=2_000, supplier=40)


def _flipped_schema(seed=3):
    s = generate(TINY, seed=seed)
    for i, c in enumerate(("custkey", "suppkey", "partkey", "orderdate", "price", "discount", "quantity")):
        inject_flips(s, "lineorder", c, 6, seed=100 + i)
    return s


def _host_result(r, to_host=None, err_host=None):
    keys = [(to_host(k) if to_host else k).tail.data for k in r.keys]
    sums = None if r.sums is None else (to_host(r.sums) if to_host else r.sums).tail.data
    fe = {c: (err_host(e) if err_host else e) for c, e in r.fact_errors.items()}
    return keys, sums, r.total, fe


def _same(a, b):
    ka, sa, ta, fa = a
    kb, sb, tb, fb = b
    assert ta == tb
    assert len(ka) == len(kb)
    for x, y in zip(ka, kb):
        assert np.array_equal(np.asarray(x), np.asarray(y))
    if sa is None:
        assert sb is None
    else:
        assert np.array_equal(np.asarray(sa), np.asarray(sb))
    assert fa.keys() == fb.keys()
    for c in fa:
        assert fa[c].present == fb[c].present
        assert np.array_equal(np.asarray(fa[c].values), np.asarray(fb[c].values)), c


def _queries():
    rng = np.random.default_rng(11)
    qs = [config2_query()]
    qs += [random_query(rng, fact_sizes=(5_000, 20_000)) for _ in range(6)]
    qs.append(StarQuery(preds=config2_query().preds, group=[]))
    return qs


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference oracle not built")
def test_composition_restatement_matches_reference():
    s = _flipped_schema()
    port, ref = Oracle("port"), Oracle("reference")
    for q in _queries():
        _same(_host_result(starjoin_continuous(port, s, q)), _host_result(starjoin_continuous(ref, s, q)))


def test_config2_result_decodes_to_plain_sums():
    """Without flips the AN-coded group sums decode (x A^-1 twice: arithmeticAN
    multiplies two codes of A) to the plain sums of price*discount."""
    from ahead_b200.pipelines import AR_INV
    s = generate(TINY, seed=5)
    q = config2_query()
    keys, sums, _, _ = _host_result(starjoin_continuous(Oracle("port"), s, q))
    assert len(sums) > 50
    T = s.tables
    lo = {c: T["lineorder"][c].tail.data.astype(np.uint64) * np.uint64(T["lineorder"][c].tail.Ainv)
          for c in ("custkey", "suppkey", "partkey", "orderdate", "price", "discount")}
    dec = lambda d, c: (T[d][c].tail.data.astype(np.uint64) * np.uint64(T[d][c].tail.Ainv))
    m = lambda x, w: x & np.uint64((1 << (8 * w)) - 1)
    cr = m(dec("customer", "region"), 1)[m(lo["custkey"], 8).astype(np.int64) - 1]
    sr = m(dec("supplier", "region"), 1)[m(lo["suppkey"], 8).astype(np.int64) - 1]
    pm = m(dec("part", "mfgr"), 1)[m(lo["partkey"], 8).astype(np.int64) - 1]
    pc = m(dec("part", "category"), 1)[m(lo["partkey"], 8).astype(np.int64) - 1]
    yr = (m(lo["orderdate"], 8) // 10000)
    ok = (cr == 1) & (sr == 1) & (pm >= 1) & (pm <= 2)
    val = m(lo["price"], 8) * m(lo["discount"], 2)
    plain = {}
    for y, c, v in zip(yr[ok], pc[ok], val[ok]):
        plain[(int(y), int(c))] = plain.get((int(y), int(c)), 0) + int(v)
    ydec = m(keys[0].astype(np.uint64) * np.uint64(pow(63877, -1, 1 << 32)), 4)
    cat = T["part"]["category"].tail
    cdec = m(keys[1].astype(np.uint64) * np.uint64(cat.Ainv), WIDTH[cat.type])
    got = {(int(y), int(c)): int((int(v) * AR_INV * AR_INV) % (1 << 64)) for y, c, v in zip(ydec, cdec, sums)}
    assert got == plain


def test_packed_index_layout_detects_one_and_two_bit_flips():
    """The packed join index (one 64-bit word per fact row for two dimensions):
    payload = id 1 | id 2 << bits(records 1) | (offset 1 + (range 1 + 1) *
    offset 2) << (id bits).  ahead_sj_index_packing's layout for the SF100
    schema (customer: 3,000,000 keys and 40 attribute records, part: 1,400,000
    and 200) is 6 + 8 + 42 = 56 payload bits with A = 253 (no A of the AN code
    lists fits 8 bits and detects every two-bit flip: 233 misses flips 29 bits
    apart); with 25 records each the lists' 463 fits.  For these and other
    layouts: the code fits 64 bits, and every word with one or two bits flipped
    (all positions, brute force) is no multiple of A, so it decodes to a value
    at or above 2^payload bits.  Key ranges of 2^32 - 1 or more are refused."""
    from ahead_b200.starjoin import index_packing
    assert index_packing((3_000_000, 1_400_000), (40, 200)) == (253, 56)
    assert index_packing((3_000_000, 1_400_000), (25, 25)) == (463, 52)
    assert index_packing((61_131, 2_000), (371, 25)) == (65117, 41)
    assert index_packing((2**32, 2**31), (4095, 4095)) is None
    rng = np.random.default_rng(3)
    for kr, nr in (((3_000_000, 1_400_000), (40, 200)), ((3_000_000, 1_400_000), (25, 25)),
                   ((61_131, 2_000), (371, 25)), ((30_000_000, 2_200_000), (25, 25)), ((2**20, 2**20), (4095, 1))):
        got = index_packing(kr, nr)
        assert got is not None
        a, bits = got
        w = bits + a.bit_length()
        assert w <= 64 and a % 2 == 1 and a >= 3
        ib = sum(max(1, x.bit_length()) for x in nr)
        assert bits == ib + (kr[0] + (kr[0] + 1) * kr[1]).bit_length()
        ainv = pow(a, -1, 1 << 64)
        words = [int(p) * a for p in rng.integers(0, 1 << bits, 4, dtype=np.uint64)]
        words.append(((1 << bits) - 1) * a)
        for word in words:
            assert (word * ainv) % (1 << 64) < (1 << bits)
            for i in range(64):
                for j in range(i, 64):
                    bad = word ^ (1 << i) ^ ((1 << j) if j != i else 0)
                    assert (bad * ainv) % (1 << 64) >= (1 << bits), (a, bits, i, j)


@pytest.mark.gpu
def test_gpu_cube_roofs_measure_three_positive_times():
    """ahead_gpu_cube_roofs times the scan's column stream, one L2 reduction
    per row, and both, on 1,048,576 synthetic rows: three positive medians;
    rows below one 512-row tile are refused."""
    import ctypes
    from ahead_b200.gpu import GpuOps, load_library
    lib = load_library()
    lib.ahead_gpu_cube_roofs.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32,
                                         ctypes.POINTER(ctypes.c_float)]
    g = GpuOps(0)
    ms = (ctypes.c_float * 3)()
    assert lib.ahead_gpu_cube_roofs(g.ctx, 1 << 20, 4096, ms) == 0
    assert all(m > 0 for m in ms)
    assert lib.ahead_gpu_cube_roofs(g.ctx, 100, 4096, ms) != 0
    g.close()


@pytest.mark.gpu
def test_gpu_plain_path_matches_oracle():
    from ahead_b200.gpu import GpuOps, err_to_host, to_device, to_host
    s = _flipped_schema()
    ds = type(s)({t: {c: to_device(b) for c, b in cols.items()} for t, cols in s.tables.items()}, s.sizes)
    g = GpuOps(0)
    port = Oracle("port")
    for q in _queries():
        exp = _host_result(starjoin_continuous(port, s, q))
        got = _host_result(starjoin_continuous(g, ds, q), to_host, err_to_host)
        _same(got, exp)


def _fused_same(r, exp, q):
    """A fused result equals the composition's (host) result."""
    from ahead_b200.model import OK
    from ahead_b200.starjoin import FACT_COLS
    keys, sums, total, fe = exp
    assert r.status == OK
    if q.group:
        assert len(r.keys) == len(keys)
        for x, y in zip(r.keys, keys):
            assert np.array_equal(x, np.asarray(y).astype(np.uint64))
        assert np.array_equal(r.sums, np.asarray(sums).astype(np.uint64))
    else:
        assert r.total == total
    for c in FACT_COLS:
        want = np.asarray(fe[c].values, dtype=np.uint64) if c in fe else np.zeros(0, np.uint64)
        assert np.array_equal(r.fact_errors[c], want), c


def _device_schema(s):
    from ahead_b200.gpu import to_device
    return type(s)({t: {c: to_device(b) for c, b in cols.items()} for t, cols in s.tables.items()}, s.sizes)


def _fused_queries():
    rng = np.random.default_rng(21)
    qs = _queries()
    qs += [random_query(rng, fact_sizes=(1_000, 7_777, 20_000)) for _ in range(20)]
    return qs


@pytest.mark.gpu
def test_gpu_fused_matches_oracle_alone_batched_and_replayed():
    from ahead_b200.gpu import GpuOps
    from ahead_b200.starjoin import StarJoinEngine
    s = _flipped_schema()
    eng = StarJoinEngine(GpuOps(0), _device_schema(s))
    port = Oracle("port")
    qs = _fused_queries()
    exp = [_host_result(starjoin_continuous(port, s, q)) for q in qs]
    for q, e in zip(qs, exp):
        _fused_same(eng.run([q])[0], e, q)
    eng.set_strategy(0)
    for variant in (0, 1, 2):
        eng.set_variant(variant)
        for graph in (False, True, True):
            for r, q, e in zip(eng.run(qs, graph=graph), qs, exp):
                _fused_same(r, e, q)
    eng.set_strategy(1)
    assert any(eng.cube_variant_is_indexed(v) for v in range(eng.cube_variants()))
    assert not all(eng.cube_variant_is_indexed(v) for v in range(eng.cube_variants()))
    # every shape under each index format (a shape of the other format looks its codes up)
    for fmt, bpr in ((2, 8), (1, 16), (0, 0)):
        eng.set_index(fmt)
        assert eng.index_info()[1] == bpr if fmt else not eng.index_info()[0]
        for cube_variant in range(eng.cube_variants()):
            eng.set_cube_variant(cube_variant)
            for graph in (False, True, True):
                for r, q, e in zip(eng.run(qs, graph=graph), qs, exp):
                    _fused_same(r, e, q)
                st = eng.last_stats()
                assert st.strategy == 1 and st.exception_rows > 0
    eng.set_index(-1)
    for q, e in zip(qs, exp):  # single-query batches through the cube as well
        _fused_same(eng.run([q])[0], e, q)
    eng.set_strategy(-1)
    assert eng.tune(qs) in (0, 1, 2)
    for r, q, e in zip(eng.run(qs, graph=True), qs, exp):
        _fused_same(r, e, q)
    eng.close()


@pytest.mark.gpu
def test_gpu_cpp_plain_path_matches_oracle():
    """ahead_plain_starjoin, the operator-at-a-time star join composed in C++
    through the C ABI, equals the restatement's composition on every query
    of the fused tests (flips in every fact column, prefixes, 0-3 group
    attributes, the survey's config-2 query), and the fused engine on each."""
    from ahead_b200.gpu import GpuOps
    from ahead_b200.starjoin import StarJoinEngine
    s = _flipped_schema(seed=8)
    eng = StarJoinEngine(GpuOps(0), _device_schema(s))
    port = Oracle("port")
    qs = _fused_queries()
    exp = [_host_result(starjoin_continuous(port, s, q)) for q in qs]
    for q, e in zip(qs, exp):
        _fused_same(eng.plain(q), e, q)
    for r, q, e in zip(eng.run(qs), qs, exp):
        _fused_same(r, e, q)
    eng.close()


@pytest.mark.gpu
def test_gpu_fused_full_batch_of_64():
    from ahead_b200.gpu import GpuOps
    from ahead_b200.starjoin import StarJoinEngine
    s = _flipped_schema(seed=9)
    eng = StarJoinEngine(GpuOps(0), _device_schema(s))
    port = Oracle("port")
    rng = np.random.default_rng(5)
    qs = [random_query(rng, fact_sizes=(3_000, 20_000)) for _ in range(63)] + [config2_query()]
    res = eng.run(qs, graph=True)
    for r, q in zip(res, qs):
        _fused_same(r, _host_result(starjoin_continuous(port, s, q)), q)
    eng.close()


@pytest.mark.gpu
def test_gpu_fused_falls_back_on_duplicate_dimension_keys():
    """A dimension with a duplicate key leaves the fused path's domain: the
    engine reports UNSUPPORTED and answer() runs the composition."""
    from ahead_b200.gpu import GpuOps
    from ahead_b200.model import UNSUPPORTED
    from ahead_b200.starjoin import StarJoinEngine
    s = _flipped_schema(seed=4)
    key = s.tables["supplier"]["suppkey"].tail.data
    key[7] = key[3]
    eng = StarJoinEngine(GpuOps(0), _device_schema(s))
    port = Oracle("port")
    q = config2_query()
    assert eng.run([q])[0].status == UNSUPPORTED
    _fused_same(eng.answer([q])[0], _host_result(starjoin_continuous(port, s, q)), q)
    eng.close()


@pytest.mark.gpu
def test_gpu_fused_two_batches_in_flight():
    """submit/submit/wait/wait: each batch's results equal the oracle's, and a
    third submit before a wait is refused."""
    from ahead_b200.gpu import AheadError, GpuOps
    from ahead_b200.model import CAPACITY
    from ahead_b200.starjoin import StarJoinEngine
    s = _flipped_schema(seed=6)
    eng = StarJoinEngine(GpuOps(0), _device_schema(s))
    port = Oracle("port")
    rng = np.random.default_rng(8)
    a = [random_query(rng, fact_sizes=(4_000, 20_000)) for _ in range(10)]
    b = [random_query(rng, fact_sizes=(2_000, 20_000)) for _ in range(7)]
    ta, tb = eng.submit(a, graph=True), eng.submit(b, graph=False)
    with pytest.raises(AheadError) as ei:
        eng.submit(a)
    assert ei.value.status == CAPACITY
    rb, ra = eng.wait(tb), eng.wait(ta)
    for batch, res in ((a, ra), (b, rb)):
        for r, q in zip(res, batch):
            _fused_same(r, _host_result(starjoin_continuous(port, s, q)), q)
    st = eng.last_stats()
    assert st.h2d_bytes > 0 and st.d2h_bytes > 0 and st.fact_ms > 0
    eng.close()


@pytest.mark.gpu
def test_gpu_fused_many_groups():
    """Queries with more groups than one shared-memory sort holds (three
    40-value group attributes; ~38K groups over 60K rows) take the radix-sort
    finalize, a two-attribute query (~1.6K groups) the shared-memory sort, and
    both return results larger than the default buffers."""
    from ahead_b200.gpu import GpuOps
    from ahead_b200.ssb import DimPred
    from ahead_b200.model import GE
    from ahead_b200.starjoin import StarJoinEngine
    s = generate(dict(TINY, fact=60_000), seed=13)
    for i, c in enumerate(("custkey", "suppkey", "partkey", "orderdate", "price", "discount", "quantity")):
        inject_flips(s, "lineorder", c, 6, seed=500 + i)
    eng = StarJoinEngine(GpuOps(0), _device_schema(s))
    port = Oracle("port")
    big = StarQuery(preds=[DimPred("date", "year", GE, 1992)],
                    group=[("customer", "nation"), ("supplier", "nation"), ("part", "category")])
    mid = StarQuery(preds=[], group=[("customer", "nation"), ("part", "category")], fact_rows=12_000)
    qs = [big, mid, config2_query()]
    for strategy in (0, 1):
        eng.set_strategy(strategy)
        res = eng.run(qs, graph=True)
        for r, q in zip(res, qs):
            _fused_same(r, _host_result(starjoin_continuous(port, s, q)), q)
        assert len(res[0].sums) > 16384
    eng.close()


def _small_sig_queries():
    """Queries referencing only the date year and the supplier region: a cube
    of 8 x 6 signatures, so a short first phase leaves a few unseen."""
    from ahead_b200.ssb import GE, LE, DimPred
    yr = lambda a, b: DimPred("date", "year", GE, a, LE, b)
    rg = lambda a, b: DimPred("supplier", "region", GE, a, LE, b)
    return [StarQuery(preds=[yr(1993, 1996)], group=[("supplier", "region")]),
            StarQuery(preds=[rg(1, 3)], group=[("date", "year")], fact_rows=7_777),
            StarQuery(preds=[yr(1992, 1998), rg(0, 4)], group=[("date", "year"), ("supplier", "region")]),
            StarQuery(preds=[rg(2, 2)], group=[]),
            StarQuery(preds=[yr(1997, 1997)], group=[("supplier", "region")], fact_rows=1_000)]


@pytest.mark.gpu
def test_gpu_cube_split_phases():
    """The cube scan's two phases: whatever rows the first phase covers (one
    row, a few, all), the results are the composition's; the second phase's
    unseen set is exercised empty, partly filled and overflowing, in two scan
    shapes, launched directly and from a graph whose by-value descriptor is
    replaced per batch."""
    from ahead_b200.gpu import GpuOps
    from ahead_b200.starjoin import StarJoinEngine
    s = _flipped_schema(seed=4)
    eng = StarJoinEngine(GpuOps(0), _device_schema(s))
    port = Oracle("port")
    eng.set_strategy(1)
    seen = set()
    for qs in (_small_sig_queries(), _fused_queries()):
        exp = [_host_result(starjoin_continuous(port, s, q)) for q in qs]
        # shapes without the join index, with the two-word index (which the
        # packed index makes them look up) and with the packed index, with and
        # without the acceptance skip
        for cube_variant in (0, 2, 4, 6, 11, 13):
            eng.set_cube_variant(cube_variant)
            for split in (1, 3, 40, 700, 4096, 0, 1 << 30):
                eng.set_cube_split(split)
                for graph in (False, True):
                    for r, q, e in zip(eng.run(qs, graph=graph), qs, exp):
                        _fused_same(r, e, q)
                    st = eng.last_stats()
                    assert st.strategy == 1
                    u = st.unseen_sigs
                    seen.add("empty" if u == 0 else "set" if u <= 1024 else "overflow")
    assert seen == {"empty", "set", "overflow"}
    eng.close()


@pytest.mark.gpu
def test_gpu_cube_large_dimensions_in_global_memory():
    """Large dimensions (customer and part of 400,000 and 300,000 rows) with
    a 120,000-row fact table, in every cube-scan shape."""
    from ahead_b200.gpu import GpuOps
    from ahead_b200.starjoin import StarJoinEngine
    s = generate(dict(fact=120_000, date=2556, customer=400_000, part=300_000, supplier=2_000), seed=6)
    for i, c in enumerate(("custkey", "suppkey", "partkey", "orderdate", "price", "discount")):
        inject_flips(s, "lineorder", c, 4, seed=200 + i)
    eng = StarJoinEngine(GpuOps(0), _device_schema(s))
    port = Oracle("port")
    rng = np.random.default_rng(31)
    qs = [config2_query()] + [random_query(rng, fact_sizes=(30_000, 120_000)) for _ in range(15)]
    exp = [_host_result(starjoin_continuous(port, s, q)) for q in qs]
    eng.set_strategy(1)
    for cube_variant in range(eng.cube_variants()):
        eng.set_cube_variant(cube_variant)
        for r, q, e in zip(eng.run(qs, graph=True), qs, exp):
            _fused_same(r, e, q)
        assert eng.last_stats().strategy == 1
    eng.close()


@pytest.mark.gpu
def test_gpu_fused_equals_plain_path_random_batches_6m():
    """At 6M rows with 1,000 seeded flips, ten 64-query batches of the bench's
    random family: the fused engine (graph replay, tuned shapes) equals the
    operator-at-a-time GPU path query by query, error positions included; the
    batches log ~8-9K (query, column, row) error entries each."""
    import sys
    from ahead_b200.gpu import GpuOps
    from ahead_b200.pipelines import starjoin_continuous as plain
    from ahead_b200.ssb import generate_device
    from ahead_b200.starjoin import StarJoinEngine
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from bench import fused_vs_plain, make_batches
    sizes = dict(fact=6_000_000, date=2556, customer=30_000, part=200_000, supplier=2_000)
    s = generate_device(sizes, seed=4, flips=1000, flip_seed=9)
    g = GpuOps(0)
    eng = StarJoinEngine(g, s)
    batches = make_batches(6, 10, sizes["fact"])
    eng.tune(batches[0])
    checked, logged = 0, []
    for b in batches:
        for f, q in zip(eng.answer(b, graph=True), b):
            assert fused_vs_plain(f, plain(g, s, q)), q
            checked += 1
        logged.append(eng.last_stats().errors_logged)
    assert checked == 640
    assert min(logged) > 4096, logged
    eng.close()
    g.close()


KEYCOL = {"date": "datekey", "customer": "custkey", "part": "partkey", "supplier": "suppkey"}


def _cudart():
    import ctypes
    lib = ctypes.CDLL("libcudart.so.12")
    lib.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    return lib


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", [1, 2])
def test_gpu_join_index_follows_the_columns(fmt):
    """Indexed cube scans take a dimension's record from the join index only
    while a row's foreign key is still the one the index was built from and
    the index words pass their AN check.  After the engine is created (with
    the two-word index, fmt 1, or the packed one, fmt 2), some orderdate,
    partkey and custkey codes are replaced by codes of other valid keys (a
    change AN coding cannot detect) and some index words get one or two
    flipped bits; every indexed shape still equals the oracle on the changed
    columns, the rows of changed indexed keys and of corrupt index words
    taking the exact per-row path."""
    import ctypes

    import torch
    from ahead_b200.gpu import GpuOps
    from ahead_b200.starjoin import PACKED_SLOTS, StarJoinEngine
    s = _flipped_schema(seed=5)
    dev = _device_schema(s)
    eng = StarJoinEngine(GpuOps(0), dev)
    eng.set_index(fmt)
    n = s.sizes["fact"]
    ptr, bpr, rows, dims = eng.index_info()
    # the two dimensions with the largest key ranges: date (yyyymmdd keys) and part
    assert ptr and bpr == (16 if fmt == 1 else 8) and rows == n and dims == (1 << 0) | (1 << 2)
    indexed = [v for v in range(eng.cube_variants()) if eng.cube_variant_is_indexed(v)]
    reading = [v for v in indexed if eng.cube_variant_reads_index(v)]
    assert reading and all((eng.cube_variant_slots(v) == PACKED_SLOTS) == (fmt == 2) for v in reading)
    rng = np.random.default_rng(7)
    changed, changed_slot = set(), {1: set(), 2: set()}  # slot 1: date, slot 2: part
    for col, dim in (("orderdate", "date"), ("partkey", "part"), ("custkey", "customer")):
        rws = rng.choice(n, 40, replace=False)
        tail = s.tables["lineorder"][col].tail
        keys = s.tables[dim][KEYCOL[dim]].tail
        valid = (keys.data.astype(np.uint64) * np.uint64(keys.Ainv)) & np.uint64(0xFFFFFFFF)
        codes = rng.choice(valid, 40).astype(np.uint64) * np.uint64(tail.A)  # other keys of the dimension
        moved = rws[tail.data[rws] != codes]
        tail.data[rws] = codes
        if dim in ("date", "part"):
            changed_slot[1 if dim == "date" else 2] |= set(moved.tolist())
        dev.tables["lineorder"][col].tail.data.view(torch.int64)[torch.from_numpy(rws).cuda()] = \
            torch.from_numpy(codes.view(np.int64)).cuda()
        changed |= set(rws.tolist())
    torch.cuda.synchronize()
    # one or two flipped bits in an index word of 30 other rows
    cr = _cudart()
    words = n * bpr // 8
    host = np.zeros(words, np.uint64)
    assert cr.cudaMemcpy(host.ctypes.data, ptr, words * 8, 2) == 0  # device to host
    flip_rows = rng.choice(sorted(set(range(n)) - changed), 30, replace=False)
    flipped_slot = {1: set(), 2: set()}
    for r in flip_rows:  # two words: slot 1 at [0, n), slot 2 at [n, 2n); packed: one word per row
        sl = int(rng.integers(0, 2)) if fmt == 1 else 0
        for b in rng.choice(64, int(rng.integers(1, 3)), replace=False):
            host[sl * n + r] ^= np.uint64(1) << np.uint64(int(b))
        for k in ((sl + 1,) if fmt == 1 else (1, 2)):
            flipped_slot[k].add(int(r))
    assert cr.cudaMemcpy(ctypes.c_void_p(ptr), host.ctypes.data, words * 8, 1) == 0  # host to device
    port = Oracle("port")
    qs = _fused_queries()
    exp = [_host_result(starjoin_continuous(port, s, q)) for q in qs]
    eng.set_strategy(1)
    def key(h):
        keys, sums, total, _ = h
        return ([np.asarray(k).astype(np.uint64).tobytes() for k in keys],
                None if sums is None else np.asarray(sums).astype(np.uint64).tobytes(), total)

    clean = _flipped_schema(seed=5)  # the unchanged columns give other results for some queries
    assert any(key(_host_result(starjoin_continuous(port, clean, q))) != key(e) for q, e in zip(qs, exp))
    for v in indexed:
        eng.set_cube_variant(v)
        for graph in (False, True):
            for r, q, e in zip(eng.run(qs, graph=graph), qs, exp):
                _fused_same(r, e, q)
            st = eng.last_stats()
            assert st.strategy == 1 and st.cube_variant == v
            if v not in reading:
                continue
            slots = min(eng.cube_variant_slots(v), 2)  # the dimensions this shape takes from the index
            routed = set().union(*(changed_slot[k] | flipped_slot[k] for k in range(1, slots + 1)))
            scanned = {r for r in routed if r < st.fact_rows}
            assert st.exception_rows >= len(scanned) > 0
    eng.close()


@pytest.mark.gpu
def test_gpu_config2_query_on_the_full_config2_schema():
    """The survey's second configuration at its full size: config2_query on a
    6,000,000-row lineorder with dimensions of 2,556 / 30,000 / 200,000 /
    2,000 rows and seeded flips on every fact column it reads.  The operator-
    at-a-time GPU path and the fused engine (per-row pass and signature cube,
    with and without the join index, launched directly and from a graph) all
    equal the restatement, which the compiled reference pins."""
    from ahead_b200.gpu import GpuOps, err_to_host, to_host
    from ahead_b200.starjoin import StarJoinEngine
    s = generate(dict(fact=6_000_000, date=2556, customer=30_000, part=200_000, supplier=2_000), seed=12)
    for i, c in enumerate(("custkey", "suppkey", "partkey", "orderdate", "price", "discount", "quantity")):
        inject_flips(s, "lineorder", c, 12, seed=400 + i)
    q = config2_query()
    exp = _host_result(starjoin_continuous(Oracle("port"), s, q))
    assert exp[1] is not None and len(exp[1]) == 280
    assert sum(len(e.values) for e in exp[3].values() if e.present) > 0
    ds = _device_schema(s)
    g = GpuOps(0)
    _same(_host_result(starjoin_continuous(g, ds, q), to_host, err_to_host), exp)
    eng = StarJoinEngine(g, ds)
    assert eng.index_info()[0]
    for strategy in (0, 1):
        eng.set_strategy(strategy)
        for cv in range(eng.cube_variants()) if strategy else (0,):
            if strategy:
                eng.set_cube_variant(cv)
            for graph in (False, True):
                _fused_same(eng.run([q], graph=graph)[0], exp, q)
                assert eng.last_stats().strategy == strategy
    eng.close()
    g.close()


@pytest.mark.gpu
def test_gpu_fused_large_error_log():
    """A 64-query batch over a 20,000-row lineorder with 250 flips in each of
    six fact columns logs ~26,000 (query, column, row) errors, more than the
    pack kernel sorts on chip, so the log takes its radix sort; every query's
    error positions (and results) still equal the restatement's, in both
    strategies."""
    from ahead_b200.gpu import GpuOps
    from ahead_b200.starjoin import StarJoinEngine
    s = generate(TINY, seed=17)
    for i, c in enumerate(("custkey", "suppkey", "partkey", "orderdate", "price", "discount")):
        inject_flips(s, "lineorder", c, 250, seed=600 + i)
    rng = np.random.default_rng(23)
    qs = [random_query(rng, fact_sizes=(20_000,)) for _ in range(64)]
    port = Oracle("port")
    exp = [_host_result(starjoin_continuous(port, s, q)) for q in qs]
    eng = StarJoinEngine(GpuOps(0), _device_schema(s))
    for strategy in (0, 1):
        eng.set_strategy(strategy)
        for r, q, e in zip(eng.run(qs, graph=True), qs, exp):
            _fused_same(r, e, q)
        assert 16384 < eng.last_stats().errors_logged < 65536
    eng.close()
