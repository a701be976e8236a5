"""The reference's SSB query programs Q1.1, Q3.1 and Q4.1 in its five detection
placements, as operator compositions over any object with the operator API
(the GPU library `ahead_b200.gpu.GpuOps`, or a CPU oracle in the tests).

Each function follows the operator sequence of the reference program it
names, operator by operator:

  normal            unencoded tables, unencoded operators
                    (tools/ssbm/ssbm-q11_normal.cpp:69-117, ssbm-q31_normal.cpp,
                    ssbm-q41_normal.cpp:99-190)
  early             checkAndDecodeAN of every column first, then the unencoded
                    operators on the decoded BATs (ssbm-q11_early.cpp:70-131,
                    ssbm-q31_early.cpp, ssbm-q41_early.cpp:100-215)
  late              unencoded operators on the AN codes (thresholds times A),
                    checkAndDecodeAN of the results only
                    (ssbm-q11_late.cpp:70-117, ssbm-q31_late.cpp,
                    ssbm-q41_late.cpp:99-196)
  continuous        AN operators throughout (ssbm-q11_continuous.cpp:70-127,
                    ssbm-q31_continuous.cpp:88-207, ssbm-q41_continuous.cpp:99-215)
  continuous_reenc  AN operators that re-encode every intermediate result
                    with a different A (ssbm-q11_continuous_reenc.cpp:70-128,
                    ssbm-q31_continuous_reenc.cpp, ssbm-q41_continuous_reenc.cpp)

The reference's Q3.1 and Q4.1 filter and group on string columns (p_mfgr,
s_region, c_region, c_nation, s_nation); this schema carries those attributes as integer
dictionary codes (`mfgr` 1..5, `region` 0..4, `nation` 0..39), AN-coded like
every other column, so the string predicates become integer predicates
(mfgr in {1, 2}, region = 1) evaluated in each placement's representation.
`nation`, which Q4.1 fetches with fetchjoinAN, is a resshort column: the
reference's fetchjoinAN check misreports valid 16-bit codes (a restiny column)
as corrupt (matchjoinAN.tcc:342), which would drop rows of the fetched
attribute only and end the program with a size mismatch at the group-by.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional

from .model import (AND, AS_RESINT, AS_RESOID, AS_RESSHORT, AS_RESTINY, BIGINT, EQ, GE, INT, LE, LT, OR, RESBIGINT,
                    RESINT, SUB, ErrVec, ainv)
from .ssb import StarSchema

PLACEMENTS = ("normal", "early", "late", "continuous", "continuous_reenc")


def _A(table, i: int, bits: int):
    """(A, A^-1) of entry i of an A table (std::get<i>(*v2_x_t::As), Ainvs)."""
    a = table[i]
    return a, ainv(a, bits)


@dataclass
class ProgramResult:
    """Q1.1: the sum (as returned by the program); Q4.1: the group keys and
    profits (BATs, groups in first-occurrence order).  `errors` collects the
    error-position vectors of every AN operator, in program order."""
    total: Optional[int] = None
    years: Any = None
    nations: Any = None   # c_nation
    profits: Any = None   # Q4.1: lo_revenue - lo_supplycost; Q3.1: lo_revenue
    snations: Any = None  # Q3.1: s_nation
    errors: List[ErrVec] = field(default_factory=list)


def _cols(schema: StarSchema, names: Dict[str, tuple]):
    return {k: schema.tables[t][c] for k, (t, c) in names.items()}


Q11_COLS = {"LQ": ("lineorder", "quantity"), "LD": ("lineorder", "discount"), "LO": ("lineorder", "orderdate"),
            "LE": ("lineorder", "price"), "DY": ("date", "year"), "DD": ("date", "datekey")}


def q11(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema] = None) -> ProgramResult:
    """SSB Q1.1: sum(lo_extendedprice * lo_discount) where lo_quantity < 25,
    lo_discount between 1 and 3, d_year = 1993.  `plain` holds the unencoded
    tables (normal placement)."""
    res = ProgramResult()
    E = res.errors.extend
    if placement in ("normal", "early"):
        if placement == "normal":
            c = _cols(plain, Q11_COLS)
        else:  # 0) eager check (ssbm-q11_early.cpp:70-88)
            enc = _cols(schema, Q11_COLS)
            c = {}
            for k in ("DD", "DY", "LQ", "LD", "LO", "LE"):
                b, e1, e2 = ops.check_and_decode_an(enc[k])
                E([e1, e2])
                c[k] = b
        bat1 = ops.select(c["LQ"], LT, 25)
        bat2 = ops.select(c["LD"], GE, 1, LE, 3, AND)
        bat4 = ops.matchjoin(bat1.mirror_head(), bat2.mirror_head())
        bat5 = bat4.mirror_head()
        bat6 = ops.matchjoin(bat5, c["LO"])
        bat7 = ops.select(c["DY"], EQ, 1993)
        bat9 = ops.matchjoin(bat7.mirror_head(), c["DD"])
        batB = ops.hashjoin(bat6, bat9.reverse())
        batC = batB.mirror_head()
        batD = ops.matchjoin(batC, c["LE"])
        batE = ops.matchjoin(bat5, c["LD"])
        batF = ops.matchjoin(batC, batE)
        res.total = ops.aggregate_mul_sum(batD, batF, BIGINT, 0)
        return res
    c = _cols(schema, Q11_COLS)
    A = {k: c[k].tail.A for k in c}
    if placement == "late":
        bat1 = ops.select(c["LQ"], LT, 25 * A["LQ"])
        bat2 = ops.select(c["LD"], GE, 1 * A["LD"], LE, 3 * A["LD"], AND)
        bat4 = ops.matchjoin(bat1.mirror_head(), bat2.mirror_head())
        bat5 = bat4.mirror_head()
        bat6 = ops.matchjoin(bat5, c["LO"])
        bat7 = ops.select(c["DY"], EQ, 1993 * A["DY"])
        bat9 = ops.matchjoin(bat7.mirror_head(), c["DD"])
        batB = ops.hashjoin(bat6, bat9.reverse())
        batC = batB.mirror_head()
        batD = ops.matchjoin(batC, c["LE"])
        batE = ops.matchjoin(bat5, c["LD"])
        batF = ops.matchjoin(batC, batE)
        # 4) late check and decode
        batG, e1, e2 = ops.check_and_decode_an(batD)
        batH, e3, e4 = ops.check_and_decode_an(batF)
        E([e1, e2, e3, e4])
        res.total = ops.aggregate_mul_sum(batG, batH, BIGINT, 0)
        return res
    reenc = placement == "continuous_reenc"
    if placement not in ("continuous", "continuous_reenc"):
        raise ValueError(f"unknown placement {placement}")
    # the reenc program's selectAN overloads take an A that selectAN.tcc:51-70 ignores
    s1, e = ops.select_an(c["LQ"], LT, 25 * A["LQ"])
    E([e])
    s2, e = ops.select_an(c["LD"], GE, 1 * A["LD"], LE, 3 * A["LD"], AND)
    E([e])
    kw = lambda h, t: dict(reenc=True, ah1r=h[0], ah1invr=h[1], at2r=t[0], at2invr=t[1]) if reenc else {}
    t4, e = ops.matchjoin_an(s1.mirror_head(), s2.mirror_head(),
                             **kw(_A(AS_RESOID, 14, 64), _A(AS_RESTINY, 4, 16)))
    E(e)
    bat5 = t4.mirror_head()
    t6, e = ops.matchjoin_an(bat5, c["LO"], **kw(_A(AS_RESOID, 13, 64), _A(AS_RESINT, 14, 64)))
    E(e)
    s7, e = ops.select_an(c["DY"], EQ, 1993 * A["DY"])
    E([e])
    t9, e = ops.matchjoin_an(s7.mirror_head(), c["DD"], **kw(_A(AS_RESOID, 12, 64), _A(AS_RESINT, 13, 64)))
    E(e)
    if reenc:
        h, t = _A(AS_RESOID, 11, 64), _A(AS_RESOID, 10, 64)
        tB, e = ops.hashjoin_an(t6, t9.reverse(), reenc_head=True, ah1r=h[0], ah1invr=h[1], reenc_tail=True,
                                at2r=t[0], at2invr=t[1])
    else:
        tB, e = ops.hashjoin_an(t6, t9.reverse())
    E(e)
    batC = tB.mirror_head()
    tD, e = ops.matchjoin_an(batC, c["LE"], **kw(_A(AS_RESOID, 9, 64), _A(AS_RESINT, 12, 64)))
    E(e)
    tE, e = ops.matchjoin_an(bat5, c["LD"], **kw(_A(AS_RESOID, 8, 64), _A(AS_RESTINY, 3, 16)))
    E(e)
    tF, e = ops.matchjoin_an(batC, tE, **kw(_A(AS_RESOID, 7, 64), _A(AS_RESTINY, 2, 16)))
    E(e)
    total, e = ops.aggregate_mul_sum_an(tD, tF, RESBIGINT)
    E(e)
    res.total = total  # AN-coded with the result's A (the program multiplies by its inverse to print)
    return res


Q41_COLS = {"PM": ("part", "mfgr"), "PP": ("part", "partkey"), "LP": ("lineorder", "partkey"),
            "SR": ("supplier", "region"), "SS": ("supplier", "suppkey"), "LS": ("lineorder", "suppkey"),
            "CR": ("customer", "region"), "CC": ("customer", "custkey"), "LC": ("lineorder", "custkey"),
            "LR": ("lineorder", "revenue"), "LSC": ("lineorder", "supplycost"), "CN": ("customer", "nation"),
            "LO": ("lineorder", "orderdate"), "DD": ("date", "datekey"), "DY": ("date", "year")}


def q41(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema] = None) -> ProgramResult:
    """SSB Q4.1 with integer attributes: sum(lo_revenue - lo_supplycost) grouped
    by d_year, c_nation where c_region = 1, s_region = 1, p_mfgr in {1, 2}."""
    res = ProgramResult()
    E = res.errors.extend
    if placement in ("normal", "early", "late"):
        if placement == "normal":
            c = _cols(plain, Q41_COLS)
            A = {k: 1 for k in c}
        elif placement == "early":  # check and decode every AN column first (ssbm-q41_early.cpp:100-133)
            enc = _cols(schema, Q41_COLS)
            c = {}
            for k in ("CC", "DD", "DY", "LC", "LS", "LP", "LO", "LR", "LSC", "PP", "SS", "PM", "SR", "CR", "CN"):
                b, e1, e2 = ops.check_and_decode_an(enc[k])
                E([e1, e2])
                c[k] = b
            A = {k: 1 for k in c}
        else:
            c = _cols(schema, Q41_COLS)
            A = {k: c[k].tail.A for k in c}
        bat1 = ops.select(c["PM"], EQ, 1 * A["PM"], EQ, 2 * A["PM"], OR)
        bat4 = ops.matchjoin(c["PP"].reverse(), bat1.mirror_head())
        bat5 = ops.hashjoin(c["LP"], bat4)
        bat6 = bat5.mirror_head()
        bat7 = ops.select(c["SR"], EQ, 1 * A["SR"])
        bat10 = ops.matchjoin(c["SS"].reverse(), bat7.mirror_head())
        bat11 = ops.matchjoin(bat6, c["LS"])
        bat12 = ops.hashjoin(bat11, bat10)
        bat13 = bat12.mirror_head()
        bat14 = ops.select(c["CR"], EQ, 1 * A["CR"])
        bat17 = ops.matchjoin(c["CC"].reverse(), bat14.mirror_head())
        bat18 = ops.matchjoin(bat13, c["LC"])
        bat19 = ops.hashjoin(bat18, bat17)
        bat21 = bat19.mirror_head().clear_head()
        batAR = ops.fetchjoin(bat21, c["LR"])
        batAS = ops.fetchjoin(bat21, c["LSC"])
        batAP = ops.arithmetic(SUB, batAR.tail.type, batAR, batAS)
        bat22 = ops.fetchjoin(bat21, c["LC"])
        bat23 = ops.hashjoin(bat22, bat17)
        batAN = ops.fetchjoin(bat23.clear_head(), c["CN"])
        bat25 = ops.fetchjoin(bat21, c["LO"])
        bat30 = ops.hashjoin(bat25, c["DD"].reverse())
        batAY = ops.fetchjoin(bat30.clear_head(), c["DY"])
        if placement == "late":  # check and decode (ssbm-q41_late.cpp:176-184)
            batAP, e1, e2 = ops.check_and_decode_an(batAP)
            batAY, e3, e4 = ops.check_and_decode_an(batAY)
            E([e1, e2, e3, e4])
        gy, fy = ops.groupby(batAY)
        gn, fn = ops.groupby2(batAN, gy, fy.count)
        res.profits = ops.aggregate_sum_grouped(batAP, gn, fn.count, BIGINT)
        res.nations = ops.fetchjoin(fn, batAN)
        res.years = ops.fetchjoin(fn, batAY)
        return res
    if placement not in ("continuous", "continuous_reenc"):
        raise ValueError(f"unknown placement {placement}")
    reenc = placement == "continuous_reenc"
    c = _cols(schema, Q41_COLS)
    A = {k: c[k].tail.A for k in c}
    last = len(AS_RESOID) - 1
    mj = lambda a, b, h=None, t=None: ops.matchjoin_an(a, b, **(dict(reenc=True, ah1r=h[0], ah1invr=h[1], at2r=t[0],
                                                                     at2invr=t[1]) if reenc else {}))
    fj = lambda a, b, t=None: ops.fetchjoin_an(a, b, **(dict(reenc=True, atr=t[0], atrinv=t[1]) if reenc else {}))
    s1, e = ops.select_an(c["PM"], EQ, 1 * A["PM"], EQ, 2 * A["PM"], OR)
    E([e])
    t4, e = mj(c["PP"].reverse(), s1.mirror_head(), _A(AS_RESINT, 14, 64), _A(AS_RESOID, 14, 64))
    E(e)
    if reenc:
        h = _A(AS_RESOID, 13, 64)
        t5, e = ops.hashjoin_an(c["LP"], t4, reenc_head=True, ah1r=h[0], ah1invr=h[1])
    else:
        h = _A(AS_RESOID, last, 64)
        t5, e = ops.hashjoin_an(c["LP"], t4, reenc_head=True, ah1r=h[0], ah1invr=h[1], reenc_tail=True,
                                at2r=t4.tail.A, at2invr=t4.tail.Ainv)
    E(e)
    bat6 = t5.mirror_head()
    s7, e = ops.select_an(c["SR"], EQ, 1 * A["SR"])
    E([e])
    t10, e = mj(c["SS"].reverse(), s7.mirror_head(), _A(AS_RESINT, 13, 64), _A(AS_RESOID, 12, 64))
    E(e)
    t11, e = mj(bat6, c["LS"], _A(AS_RESOID, 11, 64), _A(AS_RESINT, 12, 64))
    E(e)
    if reenc:
        h, t = _A(AS_RESOID, 10, 64), _A(AS_RESOID, 9, 64)
        t12, e = ops.hashjoin_an(t11, t10, reenc_head=True, ah1r=h[0], ah1invr=h[1], reenc_tail=True, at2r=t[0],
                                 at2invr=t[1])
    else:
        t12, e = ops.hashjoin_an(t11, t10)
    E(e)
    bat13 = t12.mirror_head()
    s14, e = ops.select_an(c["CR"], EQ, 1 * A["CR"])
    E([e])
    t17, e = mj(c["CC"].reverse(), s14.mirror_head(), _A(AS_RESINT, 12, 64), _A(AS_RESOID, 8, 64))
    E(e)
    t18, e = mj(bat13, c["LC"], _A(AS_RESOID, 7, 64), _A(AS_RESINT, 11, 64))
    E(e)
    if reenc:
        h, t = _A(AS_RESOID, 6, 64), _A(AS_RESOID, 5, 64)
        t19, e = ops.hashjoin_an(t18, t17, reenc_head=True, ah1r=h[0], ah1invr=h[1], reenc_tail=True, at2r=t[0],
                                 at2invr=t[1])
    else:
        t19, e = ops.hashjoin_an(t18, t17)
    E(e)
    bat21 = t19.mirror_head().clear_head()
    tAR, e = fj(bat21, c["LR"], _A(AS_RESINT, 10, 64))
    E(e)
    tAS, e = fj(bat21, c["LSC"], _A(AS_RESINT, 9, 64))
    E(e)
    ar = _A(AS_RESINT, 8 if reenc else len(AS_RESINT) - 1, 64)
    tAP, e = ops.arithmetic_an(SUB, RESINT, tAR, tAS, ar[0], ar[1])
    E(e)
    t22, e = fj(bat21, c["LC"], _A(AS_RESOID, 4, 64))
    E(e)
    if reenc:
        h, t = _A(AS_RESOID, 3, 64), _A(AS_RESOID, 2, 64)
        t23, e = ops.hashjoin_an(t22, t17, reenc_head=True, ah1r=h[0], ah1invr=h[1], reenc_tail=True, at2r=t[0],
                                 at2invr=t[1])
    else:
        h = _A(AS_RESOID, last, 64)
        t23, e = ops.hashjoin_an(t22, t17, reenc_head=True, ah1r=h[0], ah1invr=h[1])
    E(e)
    tAN, e = ops.fetchjoin_an(t23.clear_head(), c["CN"])  # (c_nation is a string column there: no re-encoding)
    E(e)
    t25, e = fj(bat21, c["LO"], _A(AS_RESINT, 7, 64))
    E(e)
    h, t = (_A(AS_RESOID, 1, 64), _A(AS_RESOID, 15, 64)) if reenc else (_A(AS_RESOID, last, 64), _A(AS_RESOID, last, 64))
    t30, e = ops.hashjoin_an(t25, c["DD"].reverse(), reenc_head=True, ah1r=h[0], ah1invr=h[1], reenc_tail=True,
                             at2r=t[0], at2invr=t[1])
    E(e)
    tAY, e = fj(t30.clear_head(), c["DY"], _A(AS_RESSHORT, 14, 32))
    E(e)
    g1 = _A(AS_RESOID, 14, 64) if reenc else _A(AS_RESOID, last, 64)
    g2 = _A(AS_RESOID, 13, 64) if reenc else _A(AS_RESOID, last, 64)
    gy, fy, e = ops.groupby_an(tAY, g1[0], g1[1])
    E(e)
    gn, fn, e = ops.groupby2_an(tAN, gy, fy.count, g2[0], g2[1])
    E(e)
    rp, e = ops.aggregate_sum_grouped_an(tAP, gn, fn.count, RESBIGINT)
    E(e)
    rn, e = ops.fetchjoin_an(fn, tAN)
    E(e)
    ry, e = fj(fn, tAY, _A(AS_RESSHORT, 13, 32))
    E(e)
    res.profits, res.nations, res.years = rp, rn, ry
    return res


Q31_COLS = {"CC": ("customer", "custkey"), "CR": ("customer", "region"), "CN": ("customer", "nation"),
            "DD": ("date", "datekey"), "DY": ("date", "year"), "LC": ("lineorder", "custkey"),
            "LS": ("lineorder", "suppkey"), "LO": ("lineorder", "orderdate"), "LR": ("lineorder", "revenue"),
            "SS": ("supplier", "suppkey"), "SR": ("supplier", "region"), "SN": ("supplier", "nation")}
ASIA = 2  # region code of 'ASIA' (the dictionary order AFRICA, AMERICA, ASIA, EUROPE, MIDDLE EAST)


def q31(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema] = None) -> ProgramResult:
    """SSB Q3.1 with integer attributes: sum(lo_revenue) grouped by c_nation,
    s_nation, d_year where c_region = s_region = ASIA and d_year in
    [1992, 1997]; groups numbered by d_year, then s_nation, then c_nation
    (ssbm-q31_continuous.cpp:88-207 and its placement twins)."""
    res = ProgramResult()
    E = res.errors.extend
    if placement in ("normal", "early", "late"):
        if placement == "normal":
            c = _cols(plain, Q31_COLS)
            A = {k: 1 for k in c}
        elif placement == "early":  # check and decode every AN column first (ssbm-q31_early.cpp)
            enc = _cols(schema, Q31_COLS)
            c = {}
            for k in ("CC", "DD", "DY", "LC", "LS", "LO", "LR", "SS", "SR", "CR", "SN", "CN"):
                b, e1, e2 = ops.check_and_decode_an(enc[k])
                E([e1, e2])
                c[k] = b
            A = {k: 1 for k in c}
        else:
            c = _cols(schema, Q31_COLS)
            A = {k: c[k].tail.A for k in c}
        bat1 = ops.select(c["SR"], EQ, ASIA * A["SR"])
        bat4 = ops.matchjoin(c["SS"].reverse(), bat1.mirror_head())
        bat5 = ops.hashjoin(c["LS"], bat4)
        bat6 = bat5.mirror_head()
        bat7 = ops.select(c["CR"], EQ, ASIA * A["CR"])
        bat10 = ops.matchjoin(c["CC"].reverse(), bat7.mirror_head())
        bat11 = ops.matchjoin(bat6, c["LC"])
        bat12 = ops.hashjoin(bat11, bat10)
        bat13 = ops.select(c["DY"], GE, 1992 * A["DY"], LE, 1997 * A["DY"], AND)
        bat16 = ops.matchjoin(bat13.mirror_head(), c["DD"]).reverse()
        bat18 = ops.matchjoin(bat12.mirror_head(), c["LO"])
        bat19 = ops.hashjoin(bat18, bat16)
        bat21 = bat19.mirror_head().clear_head()
        batAR = ops.fetchjoin(bat21, c["LR"])
        bat23 = ops.hashjoin(ops.fetchjoin(bat21, c["LS"]), bat4)
        batAS = ops.fetchjoin(bat23.clear_head(), c["SN"])
        bat26 = ops.hashjoin(ops.fetchjoin(bat21, c["LC"]), bat10)
        batAC = ops.fetchjoin(bat26.clear_head(), c["CN"])
        bat29 = ops.hashjoin(ops.fetchjoin(bat21, c["LO"]), bat16)
        batAD = ops.fetchjoin(bat29.clear_head(), c["DY"])
        if placement == "late":  # check and decode (ssbm-q31_late.cpp)
            batAR, e1, e2 = ops.check_and_decode_an(batAR)
            batAD, e3, e4 = ops.check_and_decode_an(batAD)
            E([e1, e2, e3, e4])
        gd, fd = ops.groupby(batAD)
        gs, fs = ops.groupby2(batAS, gd, fd.count)
        gc, fc = ops.groupby2(batAC, gs, fs.count)
        res.profits = ops.aggregate_sum_grouped(batAR, gc, fc.count, BIGINT)
        res.years = ops.fetchjoin(fc, batAD)
        res.nations = ops.fetchjoin(fc, batAC)
        res.snations = ops.fetchjoin(fc, batAS)
        return res
    if placement not in ("continuous", "continuous_reenc"):
        raise ValueError(f"unknown placement {placement}")
    reenc = placement == "continuous_reenc"
    c = _cols(schema, Q31_COLS)
    A = {k: c[k].tail.A for k in c}
    last = len(AS_RESOID) - 1
    O = lambda i: _A(AS_RESOID, i, 64)
    I = lambda i: _A(AS_RESINT, i, 64)
    mj = lambda a, b, h=None, t=None: ops.matchjoin_an(a, b, **(dict(reenc=True, ah1r=h[0], ah1invr=h[1], at2r=t[0],
                                                                     at2invr=t[1]) if reenc else {}))
    fj = lambda a, b, t=None: ops.fetchjoin_an(a, b, **(dict(reenc=True, atr=t[0], atrinv=t[1]) if reenc else {}))

    def hj(l, r, h, t=None):
        """hashjoinAN with the head (and, given t, the tail) re-encoded."""
        if t is None:
            return ops.hashjoin_an(l, r, reenc_head=True, ah1r=h[0], ah1invr=h[1])
        return ops.hashjoin_an(l, r, reenc_head=True, ah1r=h[0], ah1invr=h[1], reenc_tail=True, at2r=t[0],
                               at2invr=t[1])

    s1, e = ops.select_an(c["SR"], EQ, ASIA * A["SR"])
    E([e])
    t4, e = mj(c["SS"].reverse(), s1.mirror_head(), I(14), O(14))
    E(e)
    t5, e = hj(c["LS"], t4, O(13), O(12)) if reenc else hj(c["LS"], t4, O(last), (t4.tail.A, t4.tail.Ainv))
    E(e)
    bat6 = t5.mirror_head()
    s7, e = ops.select_an(c["CR"], EQ, ASIA * A["CR"])
    E([e])
    t10, e = mj(c["CC"].reverse(), s7.mirror_head(), I(13), O(11))
    E(e)
    t11, e = mj(bat6, c["LC"], O(10), I(12))
    E(e)
    t12, e = hj(t11, t10, O(9), O(8)) if reenc else ops.hashjoin_an(t11, t10)
    E(e)
    # (the reenc program's selectAN overload takes an A that selectAN.tcc:51-70 ignores)
    s13, e = ops.select_an(c["DY"], GE, 1992 * A["DY"], LE, 1997 * A["DY"], AND)
    E([e])
    t15, e = mj(s13.mirror_head(), c["DD"], O(8), I(11))
    E(e)
    bat16 = t15.reverse()
    t18, e = mj(t12.mirror_head(), c["LO"], O(7), O(6))
    E(e)
    t19, e = hj(t18, bat16, O(5), O(4)) if reenc else ops.hashjoin_an(t18, bat16)
    E(e)
    bat21 = t19.mirror_head().clear_head()
    tAR, e = fj(bat21, c["LR"], I(10))
    E(e)
    t22, e = fj(bat21, c["LS"], I(9))
    E(e)
    t23, e = hj(t22, t4, O(3), O(2)) if reenc else hj(t22, t4, O(last))
    E(e)
    tAS, e = ops.fetchjoin_an(t23.clear_head(), c["SN"])  # (s_nation is a string column there: no re-encoding)
    E(e)
    t25, e = fj(bat21, c["LC"], I(8))
    E(e)
    t26, e = hj(t25, t10, O(1), O(0)) if reenc else hj(t25, t10, O(last))
    E(e)
    tAC, e = ops.fetchjoin_an(t26.clear_head(), c["CN"])
    E(e)
    t28, e = fj(bat21, c["LO"], I(7))
    E(e)
    t29, e = hj(t28, bat16, O(15), O(14)) if reenc else hj(t28, bat16, O(last))
    E(e)
    tAD, e = fj(t29.clear_head(), c["DY"], _A(AS_RESSHORT, 13, 32))
    E(e)
    g1, g2, g3 = (O(13), O(12), O(11)) if reenc else (O(last), O(last), O(last))
    gd, fd, e = ops.groupby_an(tAD, g1[0], g1[1])
    E(e)
    gs, fs, e = ops.groupby2_an(tAS, gd, fd.count, g2[0], g2[1])
    E(e)
    gc, fc, e = ops.groupby2_an(tAC, gs, fs.count, g3[0], g3[1])
    E(e)
    rr, e = ops.aggregate_sum_grouped_an(tAR, gc, fc.count, RESBIGINT)
    E(e)
    rd, e = fj(fc, tAD, _A(AS_RESSHORT, 12, 32))
    E(e)
    rc, e = ops.fetchjoin_an(fc, tAC)
    E(e)
    rs, e = ops.fetchjoin_an(fc, tAS)
    E(e)
    res.profits, res.years, res.nations, res.snations = rr, rd, rc, rs
    return res
