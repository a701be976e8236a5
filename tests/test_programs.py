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


# ------------------------------------------------ the programs as fused star queries
NAMES = [p.__name__ for p in PROGRAMS]


def _dec_bat(b, to_host=None):
    b = to_host(b) if to_host else b
    v = np.asarray(b.tail.data)[: b.count].astype(np.uint64)
    if b.tail.A != 1:
        w = 8 * WIDTH[b.tail.type]
        v = (v * np.uint64(b.tail.Ainv)) & np.uint64((1 << w) - 1 if w < 64 else 0xFFFFFFFFFFFFFFFF)
    return [int(x) for x in v]


def _dec_sum(x):
    return (int(x) * ainv(65117, 64)) % (1 << 64)


def _program_answer(name, r):
    """{decoded group key tuple: decoded sum} of a program result (or its total)."""
    from ahead_b200.ssb_programs import PROGRAM_GROUP_FIELDS
    if name not in PROGRAM_GROUP_FIELDS:
        return _decoded_q11(r, "continuous")
    cols = [_dec_bat(getattr(r, f) if hasattr(r, f) else r.extra[f]) for f in PROGRAM_GROUP_FIELDS[name]]
    return dict(zip(zip(*cols), _dec_bat(r.profits)))


def _query_answer(s, q, keys, sums, total):
    """The same for a star query's result (keys: attribute codes; sums and
    total AN-coded with A = 65117)."""
    if not q.group:
        return _dec_sum(total)
    cols = []
    for (d, a), k in zip(q.group, keys):
        t = s.tables[d][a].tail
        w = 8 * WIDTH[t.type]
        cols.append([int(x) for x in (np.asarray(k, dtype=np.uint64) * np.uint64(t.Ainv)) & np.uint64((1 << w) - 1)])
    return dict(zip(zip(*cols), [_dec_sum(x) for x in sums]))


def test_program_queries_answer_as_the_programs():
    """Each program as one star query (ssb_programs.program_query): on clean
    data the composition that defines the fused engine's semantics gives the
    program's answer."""
    from ahead_b200.pipelines import starjoin_continuous
    from ahead_b200.ssb_programs import program_query
    s, plain = _schema(11, 0)
    port = Oracle("port")
    for prog in PROGRAMS:
        q = program_query(prog.__name__)
        c = starjoin_continuous(port, s, q)
        keys = [np.asarray(k.tail.data)[: k.count] for k in c.keys]
        sums = None if c.sums is None else np.asarray(c.sums.tail.data)[: c.sums.count]
        got = _query_answer(s, q, keys, sums, c.total)
        want = _program_answer(prog.__name__, prog(port, s, "continuous", plain))
        assert got == want, prog.__name__
        assert got, prog.__name__  # every program has rows on this schema


def _low_bit_flips(s, rows_per_col=300, seed=5):
    """Bit 0 of many quantity and discount codes flipped: a corrupt code then
    still passes the Q1.x predicates it passed before, so selectAN reports it
    and selects it."""
    rng = np.random.default_rng(seed)
    n = s.sizes["fact"]
    for c in ("quantity", "discount"):
        rows = rng.choice(n, rows_per_col, replace=False)
        s.tables["lineorder"][c].tail.data[rows] ^= 1
    return s


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference oracle not built")
def test_program_query_composition_restatement_matches_reference():
    """Under bit flips in every fact column the program queries' composition
    gives the same results and error positions over the restatement's and the
    reference's own operators."""
    from ahead_b200.pipelines import starjoin_continuous
    from ahead_b200.ssb_programs import program_query
    s, _ = _schema(3, 6)
    low = _low_bit_flips(_schema(4, 0)[0])
    port, ref = Oracle("port"), Oracle("reference")
    for sch, name in [(s, n) for n in NAMES] + [(low, n) for n in ("q11", "q12", "q13")]:
        q = program_query(name)
        a, b = starjoin_continuous(port, sch, q), starjoin_continuous(ref, sch, q)
        assert a.total == b.total, name
        for x, y in zip(a.keys + ([a.sums] if a.sums is not None else []),
                        b.keys + ([b.sums] if b.sums is not None else [])):
            assert np.array_equal(np.asarray(x.tail.data)[: x.count], np.asarray(y.tail.data)[: y.count]), name
        assert a.fact_errors.keys() == b.fact_errors.keys()
        for c in a.fact_errors:
            assert np.array_equal(np.asarray(a.fact_errors[c].values), np.asarray(b.fact_errors[c].values)), (name, c)


def _fused_equal(r, s, q, c, to_host, err_host):
    from ahead_b200.model import OK
    from ahead_b200.ssb import FACT_COLS
    assert r.status == OK
    if q.group:
        assert len(r.keys) == len(c.keys)
        for x, k in zip(r.keys, c.keys):
            assert np.array_equal(x, np.asarray(to_host(k).tail.data).astype(np.uint64))
        assert np.array_equal(r.sums, np.asarray(to_host(c.sums).tail.data).astype(np.uint64))
    else:
        assert r.total == c.total
    for col in FACT_COLS:
        want = np.zeros(0, np.uint64)
        if col in c.fact_errors:
            v = err_host(c.fact_errors[col]).values
            want = np.zeros(0, np.uint64) if v is None else np.asarray(v, dtype=np.uint64)
        assert np.array_equal(r.fact_errors[col], want), col


@pytest.mark.gpu
def test_gpu_program_queries_fused_prefilter():
    """Above 2^20 rows a per-row batch runs the prefilter first: Q1.x lists the
    rows their quantity / discount predicates can keep (and corrupt codes),
    Q2.x-Q4.x the rows their first joined dimension accepts (and corrupt
    foreign keys), and the per-row pass walks only those.  On a 1,500,000-row
    lineorder with 300 flips across the fact columns, each of the 13 programs
    (whole table and a 1,200,000-row prefix) equals the composition run
    operator by operator on the GPU, and the C++ operator path equals both."""
    from ahead_b200.gpu import GpuOps, err_to_host, to_host
    from ahead_b200.pipelines import starjoin_continuous
    from ahead_b200.ssb import generate_device
    from ahead_b200.ssb_programs import program_query
    from ahead_b200.starjoin import StarJoinEngine
    g = GpuOps(0)
    ds = generate_device(dict(fact=1_500_000, date=2556, customer=30_000, part=200_000, supplier=2_000), seed=5,
                         flips=300, flip_seed=9)
    eng = StarJoinEngine(g, ds)
    qs = [program_query(n) for n in NAMES] + [program_query(n, fact_rows=1_200_000) for n in ("q11", "q21", "q41")]
    comp = {}
    for q in qs:
        c = comp[id(q)] = starjoin_continuous(g, ds, q)
        _fused_equal(eng.run([q])[0], ds, q, c, to_host, err_to_host)
        _fused_equal(eng.plain(q), ds, q, c, to_host, err_to_host)
    # batches of several queries: two with fact predicates (one list for both), and
    # three whose first join is the customer dimension with selective predicates
    named = dict(zip(NAMES, qs[:13]))
    for names in (("q12", "q13"), ("q32", "q33", "q34")):
        batch = [named[n] for n in names]
        for r, q in zip(eng.run(batch), batch):
            _fused_equal(r, ds, q, comp[id(q)], to_host, err_to_host)
    eng.close()


@pytest.mark.gpu
def test_gpu_program_queries_fused():
    """The 13 programs on the fused engine (per-row strategy: fact predicates,
    two predicates on one dimension, revenue and revenue - supplycost
    measures, city / brand / yearmonth attributes joined in row mode): under
    flips in every fact column each equals the composition run operator by
    operator on the GPU library, alone and as one 13-query batch; on clean
    data each decodes to the program's own answer."""
    from ahead_b200.gpu import GpuOps, err_to_host, to_device, to_host
    from ahead_b200.pipelines import starjoin_continuous
    from ahead_b200.ssb_programs import program_query
    from ahead_b200.starjoin import StarJoinEngine
    dev = lambda sch: type(sch)({t: {c: to_device(b) for c, b in cols.items()} for t, cols in sch.tables.items()},
                                sch.sizes)
    g = GpuOps(0)
    s, _ = _schema(3, 6)
    ds = dev(s)
    eng = StarJoinEngine(g, ds)
    qs = [program_query(n) for n in NAMES] + [program_query(n, fact_rows=7_777) for n in ("q11", "q23", "q34", "q43")]
    comp = [starjoin_continuous(g, ds, q) for q in qs]
    for q, c in zip(qs, comp):
        _fused_equal(eng.run([q])[0], s, q, c, to_host, err_to_host)
        _fused_equal(eng.plain(q), s, q, c, to_host, err_to_host)  # the C++ operator-at-a-time path
    for r, q, c in zip(eng.run(qs[:13]), qs, comp):
        _fused_equal(r, s, q, c, to_host, err_to_host)
    eng.close()
    # corrupt quantity / discount codes that still pass the Q1.x predicates
    low = dev(_low_bit_flips(_schema(4, 0)[0]))
    eng = StarJoinEngine(g, low)
    for name in ("q11", "q12", "q13"):
        q = program_query(name)
        c = starjoin_continuous(g, low, q)
        assert len(err_to_host(c.fact_errors["quantity"]).values) > 100
        _fused_equal(eng.run([q])[0], low, q, c, to_host, err_to_host)
        _fused_equal(eng.plain(q), low, q, c, to_host, err_to_host)
    eng.close()
    clean, plain = _schema(11, 0)
    eng = StarJoinEngine(g, dev(clean))
    port = Oracle("port")
    for prog in PROGRAMS:
        q = program_query(prog.__name__)
        r = eng.run([q])[0]
        got = _query_answer(clean, q, r.keys, r.sums, r.total)
        assert got == _program_answer(prog.__name__, prog(port, clean, "continuous", plain)), prog.__name__
    eng.close()
    g.close()


# ------------------------------------------------ string attribute columns
STRING_PROGRAMS = (q21, q22, q23, q31, q32, q33, q34, q41, q42, q43)


def _str_outcome(fn, to_host=None, err_host=None):
    """As _outcome, with string result columns compared slot by slot."""
    from ahead_b200.model import STR
    try:
        r = fn()
    except Exception as e:
        return ("error", getattr(e, "status", None))
    out = [r.total]
    for b in (r.years, r.nations, r.profits, r.snations) + tuple(r.extra[k] for k in sorted(r.extra)):
        if b is None:
            out.append(None)
            continue
        if b.tail.type == STR:
            d = b.tail.data.cpu().numpy() if hasattr(b.tail.data, "cpu") else np.asarray(b.tail.data)
            out.append((b.count, STR, np.asarray(d, np.uint8).reshape(-1)[: b.count * b.tail.width].tobytes()))
            continue
        h = _host(b, to_host)
        out.append((h.count, h.tail.type, h.tail.A, np.asarray(h.tail.data)[: h.count].astype(np.uint64).tobytes()))
    errs = []
    for e in r.errors:
        e = err_host(e) if err_host else e
        errs.append(None if not e.present else np.asarray(e.values if e.values is not None else [],
                                                          dtype=np.uint64).tobytes())
    return tuple(out) + (tuple(errs),)


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference oracle not built")
@pytest.mark.parametrize("seed,nflips", [(3, 6), (5, 0)])
def test_string_programs_restatement_matches_reference(seed, nflips):
    """Q2.x-Q4.x on a schema whose region, nation, city, mfgr, category and
    brand are string columns (the reference's STRING:n layout): string
    selections, string fetch-joins and string group-bys in all five
    placements, the restatement against the reference's own operators under
    bit flips."""
    from ahead_b200.ssb import decoded, with_strings
    from ahead_b200.ssb_programs import StringOps
    s, _ = _schema(seed, nflips)
    ws = with_strings(s)
    wp = decoded(ws)
    port, ref = StringOps(Oracle("port")), StringOps(Oracle("reference"))
    for prog in STRING_PROGRAMS:
        for pl in PLACEMENTS:
            a = _str_outcome(lambda: prog(port, ws, pl, wp))
            b = _str_outcome(lambda: prog(ref, ws, pl, wp))
            assert a == b, (prog.__name__, pl)


def test_string_programs_answer_as_the_integer_programs():
    """On clean data every string program's groups, mapped back to the
    attributes' integer codes, carry the integer program's sums."""
    from ahead_b200.model import STR
    from ahead_b200.ssb import string_of, with_strings
    from ahead_b200.ssb_programs import PROGRAM_GROUP_FIELDS, StringOps
    s, plain = _schema(11, 0)
    ws = with_strings(s)
    port = Oracle("port")
    for prog in STRING_PROGRAMS:
        name = prog.__name__
        ri, rs = prog(port, s, "continuous"), prog(StringOps(port), ws, "continuous")
        want = _program_answer(name, ri)
        cols = []
        for f in PROGRAM_GROUP_FIELDS[name]:
            b = getattr(rs, f) if hasattr(rs, f) else rs.extra[f]
            if b.tail.type == STR:
                w = b.tail.width
                slots = np.asarray(b.tail.data, np.uint8).reshape(-1)[: b.count * w].reshape(b.count, w)
                cols.append([bytes(x).rstrip(b"\0").decode() for x in slots])
            else:
                cols.append(_dec_bat(b))
        got = dict(zip(zip(*cols), _dec_bat(rs.profits)))
        # the integer answer's keys as strings, attribute by attribute (program_query's group order)
        q = program_query_groups(name)
        want_s = {tuple(k if a == "year" else string_of(a, k) for k, a in zip(key, q)): v for key, v in want.items()}
        assert got == want_s and got, name


def program_query_groups(name):
    from ahead_b200.ssb_programs import program_query
    return [a for _, a in program_query(name).group]


@pytest.mark.gpu
def test_gpu_string_programs_match_oracle():
    """The same string programs through the GPU library's string operators
    against the restatement, all five placements, under bit flips."""
    from ahead_b200.gpu import GpuOps, err_to_host, to_device, to_host
    from ahead_b200.ssb import decoded, with_strings
    from ahead_b200.ssb_programs import StringOps
    s, _ = _schema(3, 6)
    ws = with_strings(s)
    wp = decoded(ws)
    dev = lambda sch: type(sch)({t: {c: to_device(b) for c, b in cols.items()} for t, cols in sch.tables.items()},
                                sch.sizes)
    dws, dwp = dev(ws), dev(wp)
    g = GpuOps(0)
    gs, port = StringOps(g), StringOps(Oracle("port"))
    for prog in STRING_PROGRAMS:
        for pl in PLACEMENTS:
            a = _str_outcome(lambda: prog(gs, dws, pl, dwp), to_host, err_to_host)
            b = _str_outcome(lambda: prog(port, ws, pl, wp))
            assert a == b, (prog.__name__, pl)
    g.close()
