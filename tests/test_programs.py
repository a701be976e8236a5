"""The reference's SSB programs Q1.1-Q1.3, Q3.1 and Q4.1 in all five detection placements
(ahead_b200/ssb_programs.py):

- CPU: the restatement's operators and the reference's own operators give the
  same results and error vectors, or raise the same error, under bit flips;
- CPU: on clean data every placement yields the same decoded answer;
- GPU: the composition over the GPU operators equals the oracle's.
"""
import os

import numpy as np
import pytest

from ahead_b200.model import WIDTH, ainv
from ahead_b200.ssb import decoded, generate, inject_flips
from ahead_b200.ssb_programs import (NATION, PLACEMENTS, city_code, q11, q12, q13, q21, q22, q23, q31, q32, q33,
                                     q34, q41, q42, q43)

PROGRAMS = (q11, q12, q13, q21, q22, q23, q31, q32, q33, q34, q41, q42, q43)
GROUPED = (q21, q22, q23, q31, q32, q33, q34, q41, q42, q43)
from oracle.oracle import REF_LIB, Oracle

TINY = dict(fact=20_000, date=2556, customer=300, part=2_000, supplier=40)
FACT = ("custkey", "suppkey", "partkey", "orderdate", "price", "discount", "quantity", "revenue", "supplycost")


def _recode(b, values):
    """Overwrite a host column with the AN codes of `values`."""
    w = 8 * WIDTH[b.tail.type]
    b.tail.data[:] = ((values.astype(np.uint64) * np.uint64(b.tail.A)) & np.uint64((1 << w) - 1)).astype(
        b.tail.data.dtype)


def _skew(s):
    """Q3.2-Q3.4 select one nation or two cities: a quarter of the customers
    and suppliers get 'UNITED STATES', 40 % the cities 'UNITED KI1'/'UNITED KI5',
    so that those programs have rows to group on a 20,000-row fact table."""
    for dim in ("customer", "supplier"):
        n = s.tables[dim]["nation"].count
        i = np.arange(n)
        nat = np.where(i % 4 == 0, NATION["UNITED STATES"], (i * 7) % 40)
        city = np.where(i % 5 == 1, city_code("UNITED KI1"), np.where(i % 5 == 2, city_code("UNITED KI5"), nat * 10))
        _recode(s.tables[dim]["nation"], nat)
        _recode(s.tables[dim]["city"], city)


def _schema(seed, nflips):
    s = generate(TINY, seed=seed)
    _skew(s)
    plain = decoded(s)
    for i, c in enumerate(FACT):
        if nflips:
            inject_flips(s, "lineorder", c, nflips, seed=100 + i)
    return s, plain


def _host(b, to_host):
    return None if b is None else (to_host(b) if to_host else b)


def _outcome(fn, to_host=None, err_host=None):
    """Comparable form of a program run: its outputs, or the error it raised."""
    try:
        r = fn()
    except Exception as e:  # the reference raises on size mismatches; so must every implementation
        status = getattr(e, "status", None)
        return ("error", status)
    out = [r.total]
    for b in (r.years, r.nations, r.profits, r.snations) + tuple(r.extra[k] for k in sorted(r.extra)):
        h = _host(b, to_host)
        out.append(None if h is None else (h.count, h.tail.type, h.tail.A,
                                           np.asarray(h.tail.data)[: h.count].astype(np.uint64).tobytes()))
    errs = []
    for e in r.errors:
        e = err_host(e) if err_host else e
        errs.append(None if not e.present else np.asarray(e.values if e.values is not None else [],
                                                          dtype=np.uint64).tobytes())
    out.append(errs)
    return tuple(out[:-1]) + (tuple(errs),)


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference oracle not built")
@pytest.mark.parametrize("seed,nflips", [(3, 6), (4, 6), (5, 0)])
def test_programs_restatement_matches_reference(seed, nflips):
    s, plain = _schema(seed, nflips)
    port, ref = Oracle("port"), Oracle("reference")
    for prog in PROGRAMS:
        for pl in PLACEMENTS:
            a = _outcome(lambda: prog(port, s, pl, plain))
            b = _outcome(lambda: prog(ref, s, pl, plain))
            assert a == b, (prog.__name__, pl)


def _decoded_q11(r, placement):
    if placement in ("continuous", "continuous_reenc"):
        return (r.total * ainv(65117, 64)) % (1 << 64)  # aggregate_mul_sumAN codes with the largest A
    return r.total


def _decoded_groups(r):
    def dec(b):
        v = np.asarray(b.tail.data)[: b.count].astype(np.uint64)
        if b.tail.A != 1:
            w = 8 * WIDTH[b.tail.type]
            v = (v * np.uint64(b.tail.Ainv)) & np.uint64((1 << w) - 1 if w < 64 else 0xFFFFFFFFFFFFFFFF)
        return [int(x) for x in v]
    cols = [dec(b) for b in (r.years, r.nations, r.profits, r.snations) if b is not None]
    cols += [dec(r.extra[k]) for k in sorted(r.extra)]
    return sorted(zip(*cols))


def test_placements_agree_on_clean_data():
    s, plain = _schema(11, 0)
    port = Oracle("port")
    for prog in (q11, q12, q13):
        tot = {pl: _decoded_q11(prog(port, s, pl, plain), pl) for pl in PLACEMENTS}
        assert len(set(tot.values())) == 1 and list(tot.values())[0] > 0, (prog.__name__, tot)
    for prog in GROUPED:
        out = [_decoded_groups(prog(port, s, pl, plain)) for pl in PLACEMENTS]
        assert all(x == out[0] for x in out) and len(out[0]) >= 1, prog.__name__


@pytest.mark.gpu
@pytest.mark.parametrize("seed,nflips", [(3, 6), (5, 0)])
def test_gpu_programs_match_oracle(seed, nflips):
    from ahead_b200.gpu import GpuOps, err_to_host, to_device, to_host
    s, plain = _schema(seed, nflips)
    dev = lambda sch: type(sch)({t: {c: to_device(b) for c, b in cols.items()} for t, cols in sch.tables.items()},
                                sch.sizes)
    ds, dplain = dev(s), dev(plain)
    g = GpuOps(0)
    port = Oracle("port")
    for prog in PROGRAMS:
        for pl in PLACEMENTS:
            a = _outcome(lambda: prog(g, ds, pl, dplain), to_host, err_to_host)
            b = _outcome(lambda: prog(port, s, pl, plain))
            assert a == b, (prog.__name__, pl)
    g.close()
