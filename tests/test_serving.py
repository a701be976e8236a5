"""The serving loop: each request's result is the same alone and in the mix
(bit-exact: keys, AN-coded sums, totals and error positions), under Poisson
arrivals that put requests of different sizes into shared batches, with and
without admission limits."""
import numpy as np
import pytest

from test_starjoin import _device_schema, _flipped_schema

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert a.status == b.status
    assert a.total == b.total
    assert len(a.keys) == len(b.keys)
    for x, y in zip(a.keys, b.keys):
        assert np.array_equal(x, y)
    if a.sums is None:
        assert b.sums is None
    else:
        assert np.array_equal(a.sums, b.sums)
    for c in a.fact_errors:
        assert np.array_equal(a.fact_errors[c], b.fact_errors[c]), c


@pytest.fixture(scope="module")
def engine():
    from ahead_b200.gpu import GpuOps
    from ahead_b200.starjoin import StarJoinEngine
    eng = StarJoinEngine(GpuOps(0), _device_schema(_flipped_schema(seed=12)))
    yield eng
    eng.close()


def _queries(n, seed):
    from ahead_b200.ssb import random_query
    rng = np.random.default_rng(seed)
    return [random_query(rng, fact_sizes=(1_000, 5_000, 20_000)) for _ in range(n)]


@pytest.mark.parametrize("window_ms,budget", [(0.5, 150 << 30), (3.0, 150 << 30), (1.0, 300_000)])
def test_alone_equals_in_mix(engine, window_ms, budget):
    from ahead_b200.serving import StarJoinServer, poisson_arrivals
    qs = _queries(150, seed=int(window_ms * 10) + budget % 7)
    alone = [engine.run([q])[0] for q in qs]
    srv = StarJoinServer(engine, window_ms=window_ms, max_batch=64, hbm_budget=budget)
    ids = srv.replay(qs, poisson_arrivals(20_000, len(qs), seed=3))
    got = srv.collect(ids)
    st = srv.stats()
    srv.close()
    for i, a in zip(ids, alone):
        _same(got[i].result, a)
    assert st.completed == len(qs)
    if budget < (1 << 30):
        assert st.mean_batch < 8  # admission kept batches small
    else:
        assert st.mean_batch > 1.5  # arrivals shared batches
    lat = [got[i].latency_ms for i in ids]
    assert min(lat) > 0 and all(got[i].done_us >= got[i].start_us >= got[i].arrival_us for i in ids)


def test_submit_from_caller_thread(engine):
    from ahead_b200.serving import StarJoinServer
    qs = _queries(40, seed=9)
    alone = [engine.run([q])[0] for q in qs]
    srv = StarJoinServer(engine, window_ms=1.0, max_batch=16)
    ids = [srv.submit(q) for q in qs]
    got = srv.collect(ids)
    srv.close()
    for i, a in zip(ids, alone):
        _same(got[i].result, a)
        assert got[i].batch_size <= 16
