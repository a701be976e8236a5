"""The reference's DMR baseline (two replicas of the unencoded tables, the
normal placement on each, a vote) for all 13 SSB programs: equal replicas give
the normal placement's result; replicas that differ in lo_revenue and
lo_extendedprice raise where the vote looks (Q1.x totals, Q2.x revenue sums)
and pass where it does not (Q3.x and Q4.x compare their first result BAT
only).  CPU: the restatement against the compiled reference; GPU: sequential
and concurrent replicas against the restatement."""
import os

import numpy as np
import pytest

from ahead_b200 import ssb_programs as P
from ahead_b200.ssb import decoded, generate
from oracle.oracle import REF_LIB, Oracle

TINY = dict(fact=20_000, date=2556, customer=300, part=2_000, supplier=40)
PROGRAMS = (P.q11, P.q12, P.q13, P.q21, P.q22, P.q23, P.q31, P.q32, P.q33, P.q34, P.q41, P.q42, P.q43)


def _replicas(seed, differ):
    s = generate(TINY, seed=seed)
    a, b = decoded(s), decoded(s)
    if differ:
        for c in ("revenue", "price"):
            b.tables["lineorder"][c].tail.data[:] += 1
    return a, b


def _host_vals(bat, to_host):
    if bat is None:
        return None
    h = to_host(bat) if to_host else bat
    return (h.count, np.asarray(h.tail.data)[: h.count].astype(np.uint64).tobytes())


def _outcome(fn, to_host=None):
    try:
        r = fn()
    except P.ModularityError as e:
        return ("vote failed", str(e))
    return (r.total,) + tuple(_host_vals(getattr(r, k), to_host) for k in ("years", "nations", "profits", "snations")) \
        + tuple(_host_vals(r.extra[k], to_host) for k in sorted(r.extra))


def test_dmr_votes_as_the_reference_does():
    port = Oracle("port")
    for differ in (False, True):
        a, b = _replicas(7, differ)
        for prog in PROGRAMS:
            got = _outcome(lambda: P.dmr(prog, port, [a, b]))
            first = P.DMR_FIRST[prog.__name__]
            if not differ:
                assert got == _outcome(lambda: prog(port, None, "normal", a)), prog.__name__
            else:
                assert (got[0] == "vote failed") == (first in ("total", "profits")), (prog.__name__, got[:1])


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference oracle not built")
def test_dmr_restatement_matches_reference():
    port, ref = Oracle("port"), Oracle("reference")
    for differ in (False, True):
        a, b = _replicas(8, differ)
        for prog in PROGRAMS:
            assert _outcome(lambda: P.dmr(prog, port, [a, b])) == _outcome(lambda: P.dmr(prog, ref, [a, b])), \
                prog.__name__


@pytest.mark.gpu
def test_gpu_dmr_sequential_and_concurrent():
    from ahead_b200.gpu import GpuOps, to_device, to_host
    port = Oracle("port")
    dev = lambda sch: type(sch)({t: {c: to_device(x) for c, x in cols.items()} for t, cols in sch.tables.items()},
                                sch.sizes)
    g1, g2 = GpuOps(0), GpuOps(0)
    for differ in (False, True):
        a, b = _replicas(9, differ)
        da, db = dev(a), dev(b)
        for prog in PROGRAMS:
            want = _outcome(lambda: P.dmr(prog, port, [a, b]))
            assert _outcome(lambda: P.dmr(prog, g1, [da, db]), to_host) == want, prog.__name__
            assert _outcome(lambda: P.dmr(prog, [g1, g2], [da, db], concurrent=True), to_host) == want, prog.__name__
    g1.close()
    g2.close()


def _three(seed, bad):
    """Three replicas; `bad` lists the ones whose revenue and price differ
    (each bad replica by its own amount)."""
    s = generate(TINY, seed=seed)
    reps = [decoded(s) for _ in range(3)]
    for k in bad:
        for c in ("revenue", "price"):
            reps[k].tables["lineorder"][c].tail.data[:] += 1 + k
    return reps


def test_tmr_majority_vote():
    """TMR (ModularRedundant.hpp:155-200): one replica off is outvoted, which
    replica answers follows the reference's order; three different replicas
    fail where the vote looks (Q1.x totals, Q2.x revenue sums)."""
    port = Oracle("port")
    for bad in ((), (2,), (1,), (0,), (0, 1, 2)):
        reps = _three(11, bad)
        for prog in PROGRAMS:
            got = _outcome(lambda: P.tmr(prog, port, reps))
            first = P.DMR_FIRST[prog.__name__]
            looks = first in ("total", "profits")
            if len(bad) == 3 and looks:
                assert got[0] == "vote failed", prog.__name__
                continue
            # the answering replica: 0 unless it is the odd one out
            k = 1 if (bad == (0,) and looks) else 0
            assert got == _outcome(lambda: prog(port, None, "normal", reps[k])), (prog.__name__, bad)


@pytest.mark.gpu
def test_gpu_tmr_matches_oracle():
    from ahead_b200.gpu import GpuOps, to_device, to_host
    port = Oracle("port")
    dev = lambda sch: type(sch)({t: {c: to_device(x) for c, x in cols.items()} for t, cols in sch.tables.items()},
                                sch.sizes)
    gs = [GpuOps(0) for _ in range(3)]
    for bad in ((), (0,), (0, 1, 2)):
        reps = _three(12, bad)
        dreps = [dev(r) for r in reps]
        for prog in PROGRAMS:
            want = _outcome(lambda: P.tmr(prog, port, reps))
            assert _outcome(lambda: P.tmr(prog, gs[0], dreps), to_host) == want, (prog.__name__, bad)
            assert _outcome(lambda: P.tmr(prog, gs, dreps, concurrent=True), to_host) == want, (prog.__name__, bad)
    for g in gs:
        g.close()
