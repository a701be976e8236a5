"""Star-join pipelines composed from the AN operators, in the reference's style.

`starjoin_continuous` builds a star join the way the reference's SSB query
programs do (tools/ssbm/ssbm-q41_continuous.cpp:97-216,
ssbm-q31_continuous.cpp:90-216): per dimension a selectAN on the predicate
attribute and a matchjoinAN onto the key column give a key -> OID map; the
first join probes the fact foreign-key column with hashjoinAN, every further
foreign key is fetched for the surviving rows with a positional matchjoinAN
and probed; the measures are fetched positionally, one after the other, so
that a row dropped for a corrupt value leaves all BATs aligned; group
attributes are fetched through the dimension OIDs; arithmeticAN<mul> forms
price * discount, groupbyAN (unary, then binary per further attribute)
numbers the groups by first occurrence, and aggregate_sum_groupedAN sums.
A query without group attributes ends in aggregate_mul_sumAN (the Q1.x shape,
ssbm-q11_continuous.cpp:67-124).

The SSB programs' further shapes: fact predicates (Q1.x) are selectANs over
the whole prefix of lo_quantity / lo_discount, intersected with matchjoinAN,
after which every foreign key is fetched positionally
(ssbm-q11_continuous.cpp:71-84); two predicates on one dimension are
intersected the same way before the key map (ssbm-q13_continuous.cpp); the
measure is price * discount, revenue (Q2.x, Q3.x: aggregate_sum_groupedAN of
the fetched codes) or revenue - supplycost (arithmeticAN<sub>, Q4.x,
ssbm-q41_continuous.cpp:176-182), its columns fetched one after the other.

`ops` is any object with the reference operator methods: the GPU library
(ahead_b200.gpu.GpuOps, the plain one-operator-per-launch GPU path) or a CPU
oracle used by the tests.  BATs are host or device accordingly.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, Callable, Dict, List, Optional

import numpy as np

from .model import (MUL, RESBIGINT, RESOID, SUB, VOID, WIDTH, A_RESOID_MAX, AOID_DEFAULT, Bat, Col, ErrVec,
                    ainv)
from .ssb import FK, KEY, StarQuery, StarSchema

AR = A_RESOID_MAX  # A of re-encoded OIDs and of AN-coded results (largest resint A)
AR_INV = ainv(AR, 64)


def prefix(b: Bat, n: int) -> Bat:
    """The first n rows of a (void, T) BAT, sharing its buffer."""
    if n >= b.count:
        return b
    t = b.tail
    data = t.data
    if data is not None:
        w = WIDTH[t.type]
        data = data[: n * w] if hasattr(data, "data_ptr") else data[:n]
    return Bat(b.head, Col(t.type, data, t.A, t.Ainv, t.unenc_max, t.seqbase), n)


@dataclass
class StarResult:
    """Group attribute codes (one array per group attribute, groups in first-
    occurrence order), the AN-coded u64 sums, or the single total of an
    ungrouped query; plus the fact-column error vectors in pipeline order."""
    keys: List[Any]
    sums: Any
    total: Optional[int]
    fact_errors: Dict[str, ErrVec] = field(default_factory=dict)
    ngroups: int = 0


def _host_values(e: ErrVec):
    v = e.values
    if v is None:
        return np.zeros(0, np.uint64)
    if hasattr(v, "cpu"):
        v = v.cpu().numpy().view(np.uint64)
    return np.asarray(v, dtype=np.uint64)


def _add_errors(fe: Dict[str, ErrVec], col: str, e: ErrVec):
    """A column read by two operators (a fact predicate's selectAN, then a
    positional fetch) reports the rows of both, in row order."""
    if col not in fe:
        fe[col] = e
        return
    fe[col] = ErrVec(np.sort(np.concatenate([_host_values(fe[col]), _host_values(e)])), True)


def _select_chain(ops, preds, col_of, aoid):
    """selectAN per predicate, the selections intersected in order with
    matchjoinAN (ssbm-q11_continuous.cpp:71-79, ssbm-q13_continuous.cpp);
    returns the mirrored OID list and each selection's errors."""
    sel, errs = None, []
    for p in preds:
        col = col_of(p)
        A = col.tail.A
        s, e = ops.select_an(col, p.op1, p.v1 * A, p.op2, p.v2 * A, p.comb, aoid)
        errs.append(e)
        sel = s.mirror_head() if sel is None else ops.matchjoin_an(sel, s.mirror_head(), aoid=aoid)[0].mirror_head()
    return sel, errs


def starjoin_continuous(ops, schema: StarSchema, q: StarQuery, aoid: int = AOID_DEFAULT) -> StarResult:
    T = schema.tables
    n = q.fact_rows or schema.sizes["fact"]
    lo = {c: prefix(b, n) for c, b in T["lineorder"].items()}
    fe: Dict[str, ErrVec] = {}
    if q.measure != "price_discount" and not q.group:
        raise ValueError("an ungrouped star query sums price * discount")

    # key -> OID maps of the dimensions (two predicates on one dimension: the
    # selections intersected first)
    km: Dict[str, Bat] = {}
    for d in q.dims():
        key = T[d][KEY[d]]
        preds = [p for p in q.preds if p.dim == d]
        if preds:
            sel, _ = _select_chain(ops, preds, lambda p: T[d][p.attr], aoid)
            km[d], _ = ops.matchjoin_an(key.reverse(), sel, aoid=aoid)
        else:
            km[d] = key.reverse()

    dims = q.dims()
    joined: Dict[str, Bat] = {}
    if q.fpreds:
        # fact predicates (Q1.x): selectAN over the whole prefix, then every
        # foreign key fetched positionally for the selected rows
        s, errs = _select_chain(ops, q.fpreds, lambda p: lo[p.col], aoid)
        for p, e in zip(q.fpreds, errs):
            _add_errors(fe, p.col, e)
        todo = dims
    else:
        # first join: probe the whole foreign-key column
        d0 = dims[0]
        void_tail = km[d0].tail.type == VOID
        j, errs = ops.hashjoin_an(lo[FK[d0]], km[d0], reenc_head=1, ah1r=AR, ah1invr=AR_INV,
                                  reenc_tail=int(void_tail), at2r=AR, at2invr=AR_INV, aoid=aoid)
        fe[FK[d0]] = errs[1]
        joined[d0] = j
        s = j.mirror_head()
        todo = dims[1:]
    for d in todo:
        f, errs = ops.matchjoin_an(s, lo[FK[d]], aoid=aoid)
        fe[FK[d]] = errs[3]
        void_tail = km[d].tail.type == VOID
        j, _ = ops.hashjoin_an(f, km[d], reenc_head=int(void_tail), ah1r=AR, ah1invr=AR_INV,
                               reenc_tail=int(void_tail), at2r=AR, at2invr=AR_INV, aoid=aoid)
        joined[d] = j
        s = j.mirror_head()

    # measures, dropped row-consistently: price then discount, or revenue then supplycost
    first, second = {"price_discount": ("price", "discount"), "revenue": ("revenue", None),
                     "profit": ("revenue", "supplycost")}[q.measure]
    m1, errs = ops.matchjoin_an(s, lo[first], aoid=aoid)
    _add_errors(fe, first, errs[3])
    s6 = m1.mirror_head()
    m2 = None
    mp = m1
    if second:
        m2, errs = ops.matchjoin_an(s6, lo[second], aoid=aoid)
        _add_errors(fe, second, errs[3])
        s6 = m2.mirror_head()
        mp, _ = ops.matchjoin_an(s6, m1, aoid=aoid)

    if not q.group:
        total, _ = ops.aggregate_mul_sum_an(mp, m2, aoid=aoid)
        return StarResult([], None, total, fe, 0)

    attrs = []
    for d, a in q.group:
        g, _ = ops.matchjoin_an(s6, joined[d], aoid=aoid)
        v, _ = ops.matchjoin_an(g, T[d][a], aoid=aoid)
        attrs.append(v)
    if q.measure == "price_discount":
        vals, _ = ops.arithmetic_an(MUL, RESBIGINT, mp.clear_head(), m2.clear_head(), AR, AR_INV, aoid=aoid)
    elif q.measure == "profit":
        vals, _ = ops.arithmetic_an(SUB, RESBIGINT, mp.clear_head(), m2.clear_head(), AR, AR_INV, aoid=aoid)
    else:
        vals = mp.clear_head()
    gids, firsts, _ = ops.groupby_an(attrs[0].clear_head())
    for v in attrs[1:]:
        gids, firsts, _ = ops.groupby2_an(v.clear_head(), gids, firsts.count)
    sums, _ = ops.aggregate_sum_grouped_an(vals, gids, firsts.count)
    keys = []
    for v in attrs:
        kv, _ = ops.matchjoin_an(firsts, v.clear_head(), aoid=aoid)
        keys.append(kv)
    return StarResult(keys, sums, None, fe, firsts.count)


@dataclass
class SelectSumResult:
    """The selected OIDs (AN-coded resoid, ascending), the AN-coded u64 sum of
    the selected values, and the error vectors of the three AN operators."""
    oids: Any
    total: int
    select_errors: ErrVec
    fetch_errors: List[ErrVec]
    decode_errors: List[ErrVec]


def select_sum_an(ops, col: Bat, lo: int, hi: int, aoid: int = AOID_DEFAULT) -> SelectSumResult:
    """The single-column select + sum path: selectAN<ge, lt, and> of
    [lo, hi) on codes (thresholds times A, as ssbm-q11_continuous.cpp:71-73
    passes them); the selected rows' values fetched by the positional
    matchjoinAN the SSB programs use for that step (mirror_head of the
    selection onto the column, ssbm-q11_continuous.cpp:80-83;
    matchjoinAN.tcc:226-302: a corrupt value is reported and dropped);
    checkAndDecodeAN of head and tail (encdecAN_scalar.tcc:129-176); the
    unencoded sum of the decoded values (Normal aggregate_sum, instantiated for
    OID heads) and its AN code with the largest resint A (65117), mod 2^64."""
    from .model import AND, BIGINT, GE, LT
    A = col.tail.A
    sel, e_sel = ops.select_an(col, GE, lo * A, LT, hi * A, AND, aoid=aoid)
    fetched, e_fetch = ops.matchjoin_an(sel.mirror_head(), col, aoid=aoid)
    dec, e1, e2 = ops.check_and_decode_an(fetched, aoid=aoid)
    total = ops.aggregate_sum(dec, BIGINT)
    return SelectSumResult(sel, (total * AR) % (1 << 64), e_sel, e_fetch, [e1, e2])
