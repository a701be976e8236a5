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

from .model import (AND, CMP_NONE, AS_RESINT, AS_RESOID, AS_RESSHORT, AS_RESTINY, BIGINT, EQ, GE, INT, LE, LT, OR, RESBIGINT,
                    RESINT, RESOID, OID, STR, SUB, VOID, Bat, Col, ErrVec, ainv)
from .ssb import DimPred, FactPred, StarQuery, StarSchema

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
    extra: Dict[str, Any] = field(default_factory=dict)  # other group columns (p_brand, c_city, ...)
    errors: List[ErrVec] = field(default_factory=list)


def _cols(schema: StarSchema, names: Dict[str, tuple]):
    return {k: schema.tables[t][c] for k, (t, c) in names.items()}


Q1_COLS = {"LQ": ("lineorder", "quantity"), "LD": ("lineorder", "discount"), "LO": ("lineorder", "orderdate"),
           "LE": ("lineorder", "price"), "DD": ("date", "datekey")}


@dataclass
class Q1Spec:
    """The constants of one Q1.x program and the A-table indices its
    re-encoding variant passes to each operator (T: restiny table, O: resoid,
    I: resint; each index into the reference's v2_*_t::As)."""
    quantity: tuple        # selectAN arguments on lo_quantity (op1, v1, op2, v2, comb)
    discount: tuple        # lo_discount between lo and hi
    date: tuple            # (attribute, value) selections on date, intersected in order
    reenc: Dict[str, tuple]


Q1_SPECS = {
    # ssbm-q11_*.cpp: lo_quantity < 25, lo_discount 1..3, d_year = 1993
    "q11": Q1Spec((LT, 25, CMP_NONE, 0, AND), (1, 3), (("year", 1993),),
                  dict(t4=("O", 14, "T", 4), t6=("O", 13, "I", 14), t9=("O", 12, "I", 13), tB=("O", 11, "O", 10),
                       tD=("O", 9, "I", 12), tE=("O", 8, "T", 3), tF=("O", 7, "T", 2))),
    # ssbm-q12_*.cpp: lo_quantity 26..35, lo_discount 4..6, d_yearmonthnum = 199401
    "q12": Q1Spec((GE, 26, LE, 35, AND), (4, 6), (("yearmonthnum", 199401),),
                  dict(t4=("O", 14, "T", 4), t6=("O", 13, "O", 12), t9=("O", 11, "I", 14), tB=("O", 10, "O", 9),
                       tD=("O", 8, "I", 13), tE=("O", 7, "T", 2), tF=("O", 6, "T", 1))),
    # ssbm-q13_*.cpp: lo_quantity 26..35, lo_discount 5..7, d_year = 1994 and d_weeknuminyear = 6
    "q13": Q1Spec((GE, 26, LE, 35, AND), (5, 7), (("year", 1994), ("weeknuminyear", 6)),
                  dict(t4=("O", 14, "T", 4), t6=("O", 13, "O", 12), tA=("O", 11, "T", 3), t9=("O", 10, "I", 14),
                       tB=("O", 9, "I", 13), tD=("O", 8, "I", 12), tE=("O", 7, "T", 2), tF=("O", 6, "T", 1))),
}
_TABLES = {"T": (AS_RESTINY, 16), "S": (AS_RESSHORT, 32), "O": (AS_RESOID, 64), "I": (AS_RESINT, 64)}


def _ai(kind: str, i: int):
    table, bits = _TABLES[kind]
    return _A(table, i, bits)


def _q1(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema], spec: Q1Spec) -> ProgramResult:
    """SSB Q1.x: sum(lo_extendedprice * lo_discount) over the rows selected on
    lo_quantity, lo_discount and the date (ssbm-q11_continuous.cpp:70-127 and
    its twins; Q1.3 intersects two date selections with a matchjoin first,
    ssbm-q13_continuous.cpp).  `plain` holds the unencoded tables (normal
    placement)."""
    res = ProgramResult()
    E = res.errors.extend
    cols = dict(Q1_COLS, **{f"D{k}": ("date", a) for k, (a, _) in enumerate(spec.date)})
    dkeys = [f"D{k}" for k in range(len(spec.date))]
    q1, q2, q3, q4, q5 = spec.quantity
    dlo, dhi = spec.discount
    if placement in ("normal", "early", "late"):
        if placement == "normal":
            c = _cols(plain, cols)
        elif placement == "early":  # 0) eager check (ssbm-q11_early.cpp:70-88)
            enc = _cols(schema, cols)
            c = {}
            for k in ["DD", dkeys[0], "LQ", "LD", "LO", "LE"] + dkeys[1:]:
                if enc[k].tail.type == STR:  # string columns are not AN-coded: kept as they are
                    c[k] = enc[k]
                    continue
                b, e1, e2 = ops.check_and_decode_an(enc[k])
                E([e1, e2])
                c[k] = b
        else:
            c = _cols(schema, cols)
        A = {k: (c[k].tail.A if placement == "late" else 1) for k in c}
        bat1 = ops.select(c["LQ"], q1, q2 * A["LQ"], q3, q4 * A["LQ"], q5)
        bat2 = ops.select(c["LD"], GE, dlo * A["LD"], LE, dhi * A["LD"], AND)
        bat4 = ops.matchjoin(bat1.mirror_head(), bat2.mirror_head())
        bat5 = bat4.mirror_head()
        bat6 = ops.matchjoin(bat5, c["LO"])
        dsel = None
        for k, (_, v) in zip(dkeys, spec.date):
            s = ops.select(c[k], EQ, v * A[k]).mirror_head()
            dsel = s if dsel is None else ops.matchjoin(dsel, s).mirror_head()
        bat9 = ops.matchjoin(dsel, c["DD"])
        batB = ops.hashjoin(bat6, bat9.reverse())
        batC = batB.mirror_head()
        batD = ops.matchjoin(batC, c["LE"])
        batE = ops.matchjoin(bat5, c["LD"])
        batF = ops.matchjoin(batC, batE)
        if placement == "late":  # 4) late check and decode
            batD, e1, e2 = ops.check_and_decode_an(batD)
            batF, e3, e4 = ops.check_and_decode_an(batF)
            E([e1, e2, e3, e4])
        res.total = ops.aggregate_mul_sum(batD, batF, BIGINT, 0)
        return res
    reenc = placement == "continuous_reenc"
    if placement not in ("continuous", "continuous_reenc"):
        raise ValueError(f"unknown placement {placement}")
    c = _cols(schema, cols)
    A = {k: c[k].tail.A for k in c}

    def kw(step):
        if not reenc:
            return {}
        hk, hi, tk, ti = spec.reenc[step]
        h, t = _ai(hk, hi), _ai(tk, ti)
        return dict(reenc=True, ah1r=h[0], ah1invr=h[1], at2r=t[0], at2invr=t[1])

    # the reenc program's selectAN overloads take an A that selectAN.tcc:51-70 ignores
    s1, e = ops.select_an(c["LQ"], q1, q2 * A["LQ"], q3, q4 * A["LQ"], q5)
    E([e])
    s2, e = ops.select_an(c["LD"], GE, dlo * A["LD"], LE, dhi * A["LD"], AND)
    E([e])
    t4, e = ops.matchjoin_an(s1.mirror_head(), s2.mirror_head(), **kw("t4"))
    E(e)
    bat5 = t4.mirror_head()
    t6, e = ops.matchjoin_an(bat5, c["LO"], **kw("t6"))
    E(e)
    dsel = None
    for k, (_, v) in zip(dkeys, spec.date):
        s, e = ops.select_an(c[k], EQ, v * A[k])
        E([e])
        if dsel is None:
            dsel = s.mirror_head()
        else:
            tA, e = ops.matchjoin_an(dsel, s.mirror_head(), **kw("tA"))
            E(e)
            dsel = tA.mirror_head()
    t9, e = ops.matchjoin_an(dsel, c["DD"], **kw("t9"))
    E(e)
    if reenc:
        hk, hi, tk, ti = spec.reenc["tB"]
        h, t = _ai(hk, hi), _ai(tk, ti)
        tB, e = ops.hashjoin_an(t6, t9.reverse(), reenc_head=True, ah1r=h[0], ah1invr=h[1], reenc_tail=True,
                                at2r=t[0], at2invr=t[1])
    else:
        tB, e = ops.hashjoin_an(t6, t9.reverse())
    E(e)
    batC = tB.mirror_head()
    tD, e = ops.matchjoin_an(batC, c["LE"], **kw("tD"))
    E(e)
    tE, e = ops.matchjoin_an(bat5, c["LD"], **kw("tE"))
    E(e)
    tF, e = ops.matchjoin_an(batC, tE, **kw("tF"))
    E(e)
    total, e = ops.aggregate_mul_sum_an(tD, tF, RESBIGINT)
    E(e)
    res.total = total  # AN-coded with the result's A (the program multiplies by its inverse to print)
    return res


def q11(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema] = None) -> ProgramResult:
    """SSB Q1.1: lo_quantity < 25, lo_discount between 1 and 3, d_year = 1993."""
    return _q1(ops, schema, placement, plain, Q1_SPECS["q11"])


def q12(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema] = None) -> ProgramResult:
    """SSB Q1.2: lo_quantity between 26 and 35, lo_discount between 4 and 6,
    d_yearmonthnum = 199401."""
    return _q1(ops, schema, placement, plain, Q1_SPECS["q12"])


def q13(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema] = None) -> ProgramResult:
    """SSB Q1.3: lo_quantity between 26 and 35, lo_discount between 5 and 7,
    d_year = 1994, d_weeknuminyear = 6."""
    return _q1(ops, schema, placement, plain, Q1_SPECS["q13"])


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
                if enc[k].tail.type == STR:  # string columns are not AN-coded: kept as they are
                    c[k] = enc[k]
                    continue
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


# dictionary codes of the SSB strings the programs name
REGION = {"AFRICA": 0, "AMERICA": 1, "ASIA": 2, "EUROPE": 3, "MIDDLE EAST": 4}


def category_code(name: str) -> int:
    """'MFGR#mc' -> 5 (m - 1) + (c - 1)."""
    return 5 * (int(name[5]) - 1) + int(name[6]) - 1


def brand_code(name: str) -> int:
    """'MFGR#mcbb' -> 40 * category + bb - 1 (brands ordered as the strings)."""
    return 40 * category_code(name[:7]) + int(name[7:]) - 1


Q2_COLS = {"DD": ("date", "datekey"), "DY": ("date", "year"), "LP": ("lineorder", "partkey"),
           "LS": ("lineorder", "suppkey"), "LO": ("lineorder", "orderdate"), "LR": ("lineorder", "revenue"),
           "PP": ("part", "partkey"), "PC": ("part", "category"), "PB": ("part", "brand"),
           "SS": ("supplier", "suppkey"), "SR": ("supplier", "region")}
# per program: s_region, and the part selection (column, op1, v1, op2, v2, comb)
Q2_SPECS = {
    "q21": ("AMERICA", ("PC", EQ, category_code("MFGR#12"), CMP_NONE, 0, AND)),
    "q22": ("ASIA", ("PB", GE, brand_code("MFGR#2221"), LE, brand_code("MFGR#2228"), AND)),
    "q23": ("EUROPE", ("PB", EQ, brand_code("MFGR#2239"), CMP_NONE, 0, AND)),
}


def _q2(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema], spec) -> ProgramResult:
    """SSB Q2.x: sum(lo_revenue) grouped by d_year, p_brand for a supplier
    region and a part category or brand range (ssbm-q21_continuous.cpp and its
    twins; Q2.2 and Q2.3 differ in the two selections only)."""
    region, (pk, p1, pv1, p2, pv2, pc) = spec
    res = ProgramResult()
    E = res.errors.extend
    if placement in ("normal", "early", "late"):
        if placement == "normal":
            c = _cols(plain, Q2_COLS)
        elif placement == "early":  # check and decode every AN column first (ssbm-q21_early.cpp)
            enc = _cols(schema, Q2_COLS)
            c = {}
            for k in ("DD", "DY", "LP", "LS", "LO", "LR", "PP", "SS", "SR", "PC", "PB"):
                if enc[k].tail.type == STR:  # string columns are not AN-coded: kept as they are
                    c[k] = enc[k]
                    continue
                b, e1, e2 = ops.check_and_decode_an(enc[k])
                E([e1, e2])
                c[k] = b
        else:
            c = _cols(schema, Q2_COLS)
        A = {k: (c[k].tail.A if placement == "late" else 1) for k in c}
        bat1 = ops.select(c["SR"], EQ, REGION[region] * A["SR"])
        bat4 = ops.matchjoin(c["SS"].reverse(), bat1.mirror_head())
        bat6 = ops.hashjoin(c["LS"], bat4).mirror_head()
        bat7 = ops.matchjoin(bat6, c["LP"])
        bat8 = ops.select(c[pk], p1, pv1 * A[pk], p2, pv2 * A[pk], pc)
        batB = ops.matchjoin(c["PP"].reverse(), bat8.mirror_head())
        batE = ops.hashjoin(bat7, batB).mirror_head()
        batF = ops.matchjoin(batE, c["LO"])
        batI = ops.hashjoin(batF, c["DD"].reverse())
        batW = batI.mirror_head()
        batZ = ops.hashjoin(ops.matchjoin(batW, c["LP"]), c["PP"].reverse())
        batAY = ops.fetchjoin(batI.clear_head(), c["DY"])
        batAB = ops.fetchjoin(batZ.clear_head(), c["PB"])
        batAR = ops.fetchjoin(batW.clear_head(), c["LR"])
        if placement == "late":  # check and decode (ssbm-q21_late.cpp)
            batAY, e1, e2 = ops.check_and_decode_an(batAY)
            batAR, e3, e4 = ops.check_and_decode_an(batAR)
            E([e1, e2, e3, e4])
        gy, fy = ops.groupby(batAY)
        gb, fb = ops.groupby2(batAB, gy, fy.count)
        res.profits = ops.aggregate_sum_grouped(batAR, gb, fb.count, BIGINT)
        res.years = ops.fetchjoin(fb, batAY)
        res.extra["brand"] = ops.fetchjoin(fb, batAB)
        return res
    if placement not in ("continuous", "continuous_reenc"):
        raise ValueError(f"unknown placement {placement}")
    reenc = placement == "continuous_reenc"
    c = _cols(schema, Q2_COLS)
    A = {k: c[k].tail.A for k in c}
    last = len(AS_RESOID) - 1
    O = lambda i: _A(AS_RESOID, i, 64)
    I = lambda i: _A(AS_RESINT, i, 64)
    mj = lambda a, b, h=None, t=None: ops.matchjoin_an(a, b, **(dict(reenc=True, ah1r=h[0], ah1invr=h[1], at2r=t[0],
                                                                     at2invr=t[1]) if reenc else {}))
    fj = lambda a, b, t=None: ops.fetchjoin_an(a, b, **(dict(reenc=True, atr=t[0], atrinv=t[1]) if reenc else {}))

    def hj(l, r, h, t):
        return ops.hashjoin_an(l, r, reenc_head=True, ah1r=h[0], ah1invr=h[1], reenc_tail=True, at2r=t[0],
                               at2invr=t[1])

    s1, e = ops.select_an(c["SR"], EQ, REGION[region] * A["SR"])
    E([e])
    t4, e = mj(c["SS"].reverse(), s1.mirror_head(), I(14), O(14))
    E(e)
    t5, e = hj(c["LS"], t4, O(13), O(12)) if reenc else hj(c["LS"], t4, O(last), (t4.tail.A, t4.tail.Ainv))
    E(e)
    t7, e = mj(t5.mirror_head(), c["LP"], O(11), I(13))
    E(e)
    s8, e = ops.select_an(c[pk], p1, pv1 * A[pk], p2, pv2 * A[pk], pc)
    E([e])
    tB, e = mj(c["PP"].reverse(), s8.mirror_head(), I(12), O(10))
    E(e)
    tC, e = hj(t7, tB, O(9), O(8)) if reenc else ops.hashjoin_an(t7, tB)
    E(e)
    tF, e = mj(tC.mirror_head(), c["LO"], O(7), I(11))
    E(e)
    batH = c["DD"].reverse()
    tI, e = hj(tF, batH, O(6), O(5)) if reenc else hj(tF, batH, (tF.head.A, tF.head.Ainv), O(last))
    E(e)
    batW = tI.mirror_head()
    tX, e = mj(batW, c["LP"], O(4), I(10))
    E(e)
    batY = c["PP"].reverse()
    tZ, e = hj(tX, batY, O(3), O(2)) if reenc else hj(tX, batY, (tX.head.A, tX.head.Ainv), O(last))
    E(e)
    tAY, e = fj(tI.clear_head(), c["DY"], _A(AS_RESSHORT, 14, 32))
    E(e)
    tAB, e = ops.fetchjoin_an(tZ.clear_head(), c["PB"])  # (p_brand is a string column there: no re-encoding)
    E(e)
    tAR, e = fj(batW.clear_head(), c["LR"], I(9))
    E(e)
    gy, fy, e = ops.groupby_an(tAY)
    E(e)
    gb, fb, e = ops.groupby2_an(tAB, gy, fy.count)
    E(e)
    rr, e = ops.aggregate_sum_grouped_an(tAR, gb, fb.count, RESBIGINT)
    E(e)
    ry, e = fj(fb, tAY, _A(AS_RESSHORT, 13, 32))
    E(e)
    rb, e = ops.fetchjoin_an(fb, tAB)
    E(e)
    res.profits, res.years = rr, ry
    res.extra["brand"] = rb
    return res


def q21(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema] = None) -> ProgramResult:
    """SSB Q2.1: p_category = 'MFGR#12', s_region = 'AMERICA'."""
    return _q2(ops, schema, placement, plain, Q2_SPECS["q21"])


def q22(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema] = None) -> ProgramResult:
    """SSB Q2.2: p_brand between 'MFGR#2221' and 'MFGR#2228', s_region = 'ASIA'."""
    return _q2(ops, schema, placement, plain, Q2_SPECS["q22"])


def q23(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema] = None) -> ProgramResult:
    """SSB Q2.3: p_brand = 'MFGR#2239', s_region = 'EUROPE'."""
    return _q2(ops, schema, placement, plain, Q2_SPECS["q23"])


NATION = {"UNITED STATES": 12, "UNITED KINGDOM": 28}  # dictionary codes (region * 8 + 0..7)


def city_code(name: str) -> int:
    """'UNITED KIn' -> 10 * nation + n."""
    return 10 * NATION["UNITED KINGDOM" if name.startswith("UNITED KI") else "UNITED STATES"] + int(name[-1])


Q3_COLS = {"CK": ("customer", "custkey"), "CR": ("customer", "region"), "CN": ("customer", "nation"),
           "CCI": ("customer", "city"), "DD": ("date", "datekey"), "DY": ("date", "year"),
           "DM": ("date", "yearmonth"), "LC": ("lineorder", "custkey"), "LS": ("lineorder", "suppkey"),
           "LO": ("lineorder", "orderdate"), "LR": ("lineorder", "revenue"), "SS": ("supplier", "suppkey"),
           "SR": ("supplier", "region"), "SN": ("supplier", "nation"), "SCI": ("supplier", "city")}


@dataclass
class Q3Spec:
    """One Q3.x program: the supplier, customer and date selections (column,
    op1, v1, op2, v2, comb), the supplier and customer attributes it groups
    on, and the A-table indices of its re-encoding variant per step (None: the
    variant calls the plain overload there)."""
    supp: tuple
    cust: tuple
    date: tuple
    sgroup: str
    cgroup: str
    reenc: Dict[str, Any]


_YEARS = ("DY", GE, 1992, LE, 1997, AND)
_KI = lambda col: (col, EQ, city_code("UNITED KI1"), EQ, city_code("UNITED KI5"), OR)
Q3_SPECS = {
    # ssbm-q31_*.cpp: c_region = s_region = 'ASIA', d_year 1992..1997, by c_nation, s_nation, d_year
    "q31": Q3Spec(("SR", EQ, REGION["ASIA"], CMP_NONE, 0, AND), ("CR", EQ, REGION["ASIA"], CMP_NONE, 0, AND),
                  _YEARS, "SN", "CN",
                  dict(t4=("I", 14, "O", 14), t5=("O", 13, "O", 12), t10=("I", 13, "O", 11), t11=("O", 10, "I", 12),
                       t12=("O", 9, "O", 8), t15=("O", 8, "I", 11), t18=("O", 7, "O", 6), t19=("O", 5, "O", 4),
                       tAR=10, t22=9, t23=("O", 3, "O", 2), t25=8, t26=("O", 1, "O", 0), t28=7,
                       t29=("O", 15, "O", 14), tAD=13, groups=(13, 12, 11), rd=12)),
    # ssbm-q32_*.cpp: c_nation = s_nation = 'UNITED STATES', d_year 1992..1997, by c_city, s_city, d_year
    "q32": Q3Spec(("SN", EQ, NATION["UNITED STATES"], CMP_NONE, 0, AND),
                  ("CN", EQ, NATION["UNITED STATES"], CMP_NONE, 0, AND), _YEARS, "SCI", "CCI",
                  dict(t4=("I", 14, "O", 14), t5=("O", 13, "O", 12), t10=("I", 13, "O", 11), t11=("O", 10, "I", 12),
                       t12=("O", 9, "O", 8), t15=("O", 7, "I", 11), t18=("O", 6, "I", 10), t19=("O", 5, "O", 4),
                       tAR=9, t22=8, t23=("O", 3, "O", 2), t25=7, t26=("O", 1, "O", 0), t28=6,
                       t29=("O", 15), tAD=13, groups=None, rd=12)),
    # ssbm-q33_*.cpp: c_city, s_city in ('UNITED KI1', 'UNITED KI5'), d_year 1992..1997
    "q33": Q3Spec(_KI("SCI"), _KI("CCI"), _YEARS, "SCI", "CCI",
                  dict(t4=("I", 14, "O", 14), t5=("O", 13, "O", 12), t10=None, t11=("I", 13, "O", 11),
                       t12=("O", 10, "O", 9), t15=("O", 8, "I", 12), t18=("O", 7, "I", 11), t19=("O", 6, "O", 5),
                       tAR=10, t22=9, t23=("O", 4, "O", 3), t25=8, t26=("O", 2, "O", 1), t28=7,
                       t29=("O", 0, "O", 15), tAD=13, groups=(14, 13, 12), rd=12)),
    # ssbm-q34_*.cpp: as Q3.3 with d_yearmonth = 'Dec1997'
    "q34": Q3Spec(_KI("SCI"), _KI("CCI"), ("DM", EQ, 199712, CMP_NONE, 0, AND), "SCI", "CCI",
                  dict(t4=("I", 14, "O", 14), t5=("O", 13, "O", 12), t10=("I", 13, "O", 11), t11=("O", 10, "I", 12),
                       t12=("O", 9, "O", 8), t15=("O", 7, "I", 11), t18=("O", 6, "I", 10), t19=("O", 5, "O", 4),
                       tAR=9, t22=8, t23=("O", 3, "O", 2), t25=7, t26=("O", 1, "O", 14), t28=6,
                       t29=("O", 13, "O", 12), tAD=14, groups=(11, 10, 9), rd=13)),
}


def _q3(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema], spec: Q3Spec) -> ProgramResult:
    """SSB Q3.x: sum(lo_revenue) grouped by the customer and supplier
    attributes and d_year, for customer, supplier and date selections;
    groups numbered by d_year, then the supplier attribute, then the customer
    attribute (ssbm-q31_continuous.cpp:88-207 and its twins)."""
    res = ProgramResult()
    E = res.errors.extend
    strs = []
    for k in (spec.supp[0], spec.cust[0], spec.sgroup, spec.cgroup, spec.date[0]):
        if k not in ("DY",) and k not in strs:
            strs.append(k)

    def sel(sop, c, sp, A):
        k, o1, v1, o2, v2, cb = sp
        return sop(c[k], o1, v1 * A[k], o2, v2 * A[k], cb)

    if placement in ("normal", "early", "late"):
        if placement == "normal":
            c = _cols(plain, Q3_COLS)
        elif placement == "early":  # check and decode every AN column first (ssbm-q31_early.cpp)
            enc = _cols(schema, Q3_COLS)
            c = {}
            for k in ["CK", "DD", "DY", "LC", "LS", "LO", "LR", "SS"] + strs:
                if enc[k].tail.type == STR:  # string columns are not AN-coded: kept as they are
                    c[k] = enc[k]
                    continue
                b, e1, e2 = ops.check_and_decode_an(enc[k])
                E([e1, e2])
                c[k] = b
        else:
            c = _cols(schema, Q3_COLS)
        A = {k: (c[k].tail.A if placement == "late" else 1) for k in c}
        bat1 = sel(ops.select, c, spec.supp, A)
        bat4 = ops.matchjoin(c["SS"].reverse(), bat1.mirror_head())
        bat6 = ops.hashjoin(c["LS"], bat4).mirror_head()
        bat7 = sel(ops.select, c, spec.cust, A)
        bat10 = ops.matchjoin(c["CK"].reverse(), bat7.mirror_head())
        bat12 = ops.hashjoin(ops.matchjoin(bat6, c["LC"]), bat10)
        bat13 = sel(ops.select, c, spec.date, A)
        bat16 = ops.matchjoin(bat13.mirror_head(), c["DD"]).reverse()
        bat19 = ops.hashjoin(ops.matchjoin(bat12.mirror_head(), c["LO"]), bat16)
        bat21 = bat19.mirror_head().clear_head()
        batAR = ops.fetchjoin(bat21, c["LR"])
        bat23 = ops.hashjoin(ops.fetchjoin(bat21, c["LS"]), bat4)
        batAS = ops.fetchjoin(bat23.clear_head(), c[spec.sgroup])
        bat26 = ops.hashjoin(ops.fetchjoin(bat21, c["LC"]), bat10)
        batAC = ops.fetchjoin(bat26.clear_head(), c[spec.cgroup])
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
    R = spec.reenc
    c = _cols(schema, Q3_COLS)
    A = {k: c[k].tail.A for k in c}
    O = lambda i: _A(AS_RESOID, i, 64)
    last = len(AS_RESOID) - 1

    def mj(step, a, b):
        r = R[step] if reenc else None
        if r is None:
            return ops.matchjoin_an(a, b)
        h, t = _ai(r[0], r[1]), _ai(r[2], r[3])
        return ops.matchjoin_an(a, b, reenc=True, ah1r=h[0], ah1invr=h[1], at2r=t[0], at2invr=t[1])

    def hj(l, r, h, t=None):
        kw = dict(reenc_head=True, ah1r=h[0], ah1invr=h[1])
        if t is not None:
            kw.update(reenc_tail=True, at2r=t[0], at2invr=t[1])
        return ops.hashjoin_an(l, r, **kw)

    def hjs(step, l, r, plain_call):
        """A hashjoinAN step: the reenc variant's A indices, else the continuous call."""
        if not reenc:
            return plain_call()
        x = R[step]
        return hj(l, r, _ai(x[0], x[1]), _ai(x[2], x[3]) if len(x) > 2 else None)

    def fj(step, a, b, kind="I"):
        if not reenc:
            return ops.fetchjoin_an(a, b)
        t = _ai(kind, R[step])
        return ops.fetchjoin_an(a, b, reenc=True, atr=t[0], atrinv=t[1])

    s1, e = sel(ops.select_an, c, spec.supp, A)
    E([e])
    t4, e = mj("t4", c["SS"].reverse(), s1.mirror_head())
    E(e)
    t5, e = hjs("t5", c["LS"], t4, lambda: hj(c["LS"], t4, O(last), (t4.tail.A, t4.tail.Ainv)))
    E(e)
    bat6 = t5.mirror_head()
    s7, e = sel(ops.select_an, c, spec.cust, A)
    E([e])
    t10, e = mj("t10", c["CK"].reverse(), s7.mirror_head())
    E(e)
    t11, e = mj("t11", bat6, c["LC"])
    E(e)
    t12, e = hjs("t12", t11, t10, lambda: ops.hashjoin_an(t11, t10))
    E(e)
    # (the reenc programs' selectAN overload takes an A that selectAN.tcc:51-70 ignores)
    s13, e = sel(ops.select_an, c, spec.date, A)
    E([e])
    t15, e = mj("t15", s13.mirror_head(), c["DD"])
    E(e)
    bat16 = t15.reverse()
    t18, e = mj("t18", t12.mirror_head(), c["LO"])
    E(e)
    t19, e = hjs("t19", t18, bat16, lambda: ops.hashjoin_an(t18, bat16))
    E(e)
    bat21 = t19.mirror_head().clear_head()
    tAR, e = fj("tAR", bat21, c["LR"])
    E(e)
    t22, e = fj("t22", bat21, c["LS"])
    E(e)
    t23, e = hjs("t23", t22, t4, lambda: hj(t22, t4, O(last)))
    E(e)
    tAS, e = ops.fetchjoin_an(t23.clear_head(), c[spec.sgroup])  # (a string column there: no re-encoding)
    E(e)
    t25, e = fj("t25", bat21, c["LC"])
    E(e)
    t26, e = hjs("t26", t25, t10, lambda: hj(t25, t10, O(last)))
    E(e)
    tAC, e = ops.fetchjoin_an(t26.clear_head(), c[spec.cgroup])
    E(e)
    t28, e = fj("t28", bat21, c["LO"])
    E(e)
    t29, e = hjs("t29", t28, bat16, lambda: hj(t28, bat16, O(last)))
    E(e)
    tAD, e = fj("tAD", t29.clear_head(), c["DY"], "S")
    E(e)
    g = [O(i) for i in R["groups"]] if reenc and R["groups"] else [O(last)] * 3
    gd, fd, e = ops.groupby_an(tAD, g[0][0], g[0][1])
    E(e)
    gs, fs, e = ops.groupby2_an(tAS, gd, fd.count, g[1][0], g[1][1])
    E(e)
    gc, fc, e = ops.groupby2_an(tAC, gs, fs.count, g[2][0], g[2][1])
    E(e)
    rr, e = ops.aggregate_sum_grouped_an(tAR, gc, fc.count, RESBIGINT)
    E(e)
    rd, e = fj("rd", fc, tAD, "S")
    E(e)
    rc, e = ops.fetchjoin_an(fc, tAC)
    E(e)
    rs, e = ops.fetchjoin_an(fc, tAS)
    E(e)
    res.profits, res.years, res.nations, res.snations = rr, rd, rc, rs
    return res


def q31(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema] = None) -> ProgramResult:
    """SSB Q3.1: c_region = s_region = 'ASIA', d_year between 1992 and 1997;
    by c_nation, s_nation, d_year."""
    return _q3(ops, schema, placement, plain, Q3_SPECS["q31"])


def q32(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema] = None) -> ProgramResult:
    """SSB Q3.2: c_nation = s_nation = 'UNITED STATES', d_year between 1992 and
    1997; by c_city, s_city, d_year."""
    return _q3(ops, schema, placement, plain, Q3_SPECS["q32"])


def q33(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema] = None) -> ProgramResult:
    """SSB Q3.3: c_city and s_city in ('UNITED KI1', 'UNITED KI5'), d_year
    between 1992 and 1997; by c_city, s_city, d_year."""
    return _q3(ops, schema, placement, plain, Q3_SPECS["q33"])


def q34(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema] = None) -> ProgramResult:
    """SSB Q3.4: as Q3.3 with d_yearmonth = 'Dec1997'."""
    return _q3(ops, schema, placement, plain, Q3_SPECS["q34"])


Q4X_COLS = {"PM": ("part", "mfgr"), "PC": ("part", "category"), "PB": ("part", "brand"), "PP": ("part", "partkey"),
            "LP": ("lineorder", "partkey"), "SR": ("supplier", "region"), "SN": ("supplier", "nation"),
            "SCI": ("supplier", "city"), "SS": ("supplier", "suppkey"), "LS": ("lineorder", "suppkey"),
            "CR": ("customer", "region"), "CK": ("customer", "custkey"), "LC": ("lineorder", "custkey"),
            "LR": ("lineorder", "revenue"), "LSC": ("lineorder", "supplycost"), "DD": ("date", "datekey"),
            "DY": ("date", "year"), "LO": ("lineorder", "orderdate")}


@dataclass
class Q4Spec:
    """Q4.2 / Q4.3: part, supplier and (optional) customer selections, the two
    attributes grouped after d_year (supplier side, part side), and the
    A-table indices of the re-encoding variant per step."""
    part: tuple
    supp: tuple
    cust: Optional[tuple]
    sgroup: str
    pgroup: str
    reenc: Dict[str, Any]


Q4X_SPECS = {
    # ssbm-q42_*.cpp: p_mfgr in (MFGR#1, MFGR#2), s_region = c_region = 'AMERICA', d_year in (1997, 1998);
    # by d_year, s_nation, p_category
    "q42": Q4Spec(("PM", EQ, 1, EQ, 2, OR), ("SR", EQ, REGION["AMERICA"], CMP_NONE, 0, AND),
                  ("CR", EQ, REGION["AMERICA"], CMP_NONE, 0, AND), "SN", "PC",
                  dict(t4=("I", 14, "O", 14), t5=("O", 13, "O", 12), t10=("I", 13, "O", 12), t11=("O", 11, "I", 12),
                       t12=("O", 10, "O", 9), t17=("O", 11, "O", 8), t18=("O", 7, "I", 11), t19=("O", 6, "O", 5),
                       t24=("I", 10, "O", 4), t25=("O", 3, "I", 9), t26=("O", 2, "O", 1), tAR=9, tAS=8, tAP=14,
                       t29=7, t30=("O", 15, "O", 14), t32=6, t34=("O", 13, "O", 12), tAY=13, t36=5,
                       t38=("O", 11, "O", 10), groups=(13, 9, 8), ry=12)),
    # ssbm-q43_*.cpp: p_category = 'MFGR#14', s_nation = 'UNITED STATES', d_year in (1997, 1998);
    # by d_year, s_city, p_brand (the program joins no customer)
    "q43": Q4Spec(("PC", EQ, category_code("MFGR#14"), CMP_NONE, 0, AND),
                  ("SN", EQ, NATION["UNITED STATES"], CMP_NONE, 0, AND), None, "SCI", "PB",
                  dict(t4=("I", 14, "O", 14), t5=("O", 13, "O", 12), t10=("I", 13, "O", 12), t11=("O", 11, "I", 12),
                       t12=("O", 10, "O", 9), t24=("I", 11, "O", 8), t25=("O", 7, "I", 10), t26=("O", 6, "O", 5),
                       tAR=10, tAS=9, tAP=8, t29=7, t30=("O", 4, "O", 3), t32=6, t34=("O", 2, "O", 1), tAY=13,
                       t36=5, t38=("O", 15, "O", 14), groups=(13, 12, 11), ry=12)),
}


def _q4x(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema], spec: Q4Spec, name: str):
    """SSB Q4.2 / Q4.3: sum(lo_revenue - lo_supplycost) grouped by d_year and
    a supplier and a part attribute (ssbm-q42_continuous.cpp,
    ssbm-q43_continuous.cpp and their placement twins)."""
    res = ProgramResult()
    E = res.errors.extend
    strs = []
    for k in (spec.part[0], spec.supp[0]) + ((spec.cust[0],) if spec.cust else ()) + (spec.sgroup, spec.pgroup):
        if k not in strs:
            strs.append(k)

    def sel(sop, c, sp, A):
        k, o1, v1, o2, v2, cb = sp
        return sop(c[k], o1, v1 * A[k], o2, v2 * A[k], cb)

    if placement in ("normal", "early", "late"):
        if placement == "normal":
            c = _cols(plain, Q4X_COLS)
        elif placement == "early":  # check and decode every AN column first (ssbm-q42_early.cpp)
            enc = _cols(schema, Q4X_COLS)
            c = {}
            for k in ["CK", "DD", "DY", "LC", "LS", "LP", "LO", "LR", "LSC", "PP", "SS"] + strs:
                if enc[k].tail.type == STR:  # string columns are not AN-coded: kept as they are
                    c[k] = enc[k]
                    continue
                b, e1, e2 = ops.check_and_decode_an(enc[k])
                E([e1, e2])
                c[k] = b
        else:
            c = _cols(schema, Q4X_COLS)
        A = {k: (c[k].tail.A if placement == "late" else 1) for k in c}
        bat4 = ops.matchjoin(c["PP"].reverse(), sel(ops.select, c, spec.part, A).mirror_head())
        bat6 = ops.hashjoin(c["LP"], bat4).mirror_head()
        bat10 = ops.matchjoin(c["SS"].reverse(), sel(ops.select, c, spec.supp, A).mirror_head())
        bat20 = ops.hashjoin(ops.matchjoin(bat6, c["LS"]), bat10).mirror_head()
        if spec.cust:
            bat17 = ops.matchjoin(c["CK"].reverse(), sel(ops.select, c, spec.cust, A).mirror_head())
            bat20 = ops.hashjoin(ops.matchjoin(bat20, c["LC"]), bat17).mirror_head()
        bat21 = ops.select(c["DY"], EQ, 1997 * A["DY"], EQ, 1998 * A["DY"], OR)
        bat24 = ops.matchjoin(c["DD"].reverse(), bat21.mirror_head())
        bat28 = ops.hashjoin(ops.matchjoin(bat20, c["LO"]), bat24).mirror_head().clear_head()
        batAR = ops.fetchjoin(bat28, c["LR"])
        batAS = ops.fetchjoin(bat28, c["LSC"])
        batAP = ops.arithmetic(SUB, batAR.tail.type, batAR, batAS)
        bat30 = ops.hashjoin(ops.fetchjoin(bat28, c["LS"]), bat10)
        batAN = ops.fetchjoin(bat30.clear_head(), c[spec.sgroup])
        bat34 = ops.hashjoin(ops.fetchjoin(bat28, c["LO"]), bat24)
        batAY = ops.fetchjoin(bat34.clear_head(), c["DY"])
        bat38 = ops.hashjoin(ops.fetchjoin(bat28, c["LP"]), c["PP"].reverse())
        batAC = ops.fetchjoin(bat38.clear_head(), c[spec.pgroup])
        if placement == "late":  # check and decode (ssbm-q42_late.cpp)
            batAP, e1, e2 = ops.check_and_decode_an(batAP)
            batAY, e3, e4 = ops.check_and_decode_an(batAY)
            E([e1, e2, e3, e4])
        gy, fy = ops.groupby(batAY)
        gn, fn = ops.groupby2(batAN, gy, fy.count)
        gc, fc = ops.groupby2(batAC, gn, fn.count)
        res.profits = ops.aggregate_sum_grouped(batAP, gc, fc.count, BIGINT)
        if name == "q42":
            res.extra["s_group"] = ops.fetchjoin(fc, batAN)
            res.years = ops.fetchjoin(fc, batAY)
        else:
            res.years = ops.fetchjoin(fc, batAY)
            res.extra["s_group"] = ops.fetchjoin(fc, batAN)
        res.extra["p_group"] = ops.fetchjoin(fc, batAC)
        return res
    if placement not in ("continuous", "continuous_reenc"):
        raise ValueError(f"unknown placement {placement}")
    reenc = placement == "continuous_reenc"
    R = spec.reenc
    c = _cols(schema, Q4X_COLS)
    A = {k: c[k].tail.A for k in c}
    O = lambda i: _A(AS_RESOID, i, 64)
    last = len(AS_RESOID) - 1

    def mj(step, a, b):
        if not reenc:
            return ops.matchjoin_an(a, b)
        r = R[step]
        h, t = _ai(r[0], r[1]), _ai(r[2], r[3])
        return ops.matchjoin_an(a, b, reenc=True, ah1r=h[0], ah1invr=h[1], at2r=t[0], at2invr=t[1])

    def hj(l, r, h, t=None):
        kw = dict(reenc_head=True, ah1r=h[0], ah1invr=h[1])
        if t is not None:
            kw.update(reenc_tail=True, at2r=t[0], at2invr=t[1])
        return ops.hashjoin_an(l, r, **kw)

    def hjs(step, l, r, plain_call):
        if not reenc:
            return plain_call()
        x = R[step]
        return hj(l, r, _ai(x[0], x[1]), _ai(x[2], x[3]))

    def fj(step, a, b, kind="I"):
        if not reenc:
            return ops.fetchjoin_an(a, b)
        t = _ai(kind, R[step])
        return ops.fetchjoin_an(a, b, reenc=True, atr=t[0], atrinv=t[1])

    s1, e = sel(ops.select_an, c, spec.part, A)
    E([e])
    t4, e = mj("t4", c["PP"].reverse(), s1.mirror_head())
    E(e)
    t5, e = hjs("t5", c["LP"], t4, lambda: hj(c["LP"], t4, O(last), (t4.tail.A, t4.tail.Ainv)))
    E(e)
    bat6 = t5.mirror_head()
    s7, e = sel(ops.select_an, c, spec.supp, A)
    E([e])
    t10, e = mj("t10", c["SS"].reverse(), s7.mirror_head())
    E(e)
    t11, e = mj("t11", bat6, c["LS"])
    E(e)
    t12, e = hjs("t12", t11, t10, lambda: ops.hashjoin_an(t11, t10))
    E(e)
    bat20 = t12.mirror_head()
    if spec.cust:
        s14, e = sel(ops.select_an, c, spec.cust, A)
        E([e])
        t17, e = mj("t17", c["CK"].reverse(), s14.mirror_head())
        E(e)
        t18, e = mj("t18", bat20, c["LC"])
        E(e)
        t19, e = hjs("t19", t18, t17, lambda: ops.hashjoin_an(t18, t17))
        E(e)
        bat20 = t19.mirror_head()
    # (the reenc programs' selectAN overload takes an A that selectAN.tcc:51-70 ignores)
    s21, e = ops.select_an(c["DY"], EQ, 1997 * A["DY"], EQ, 1998 * A["DY"], OR)
    E([e])
    t24, e = mj("t24", c["DD"].reverse(), s21.mirror_head())
    E(e)
    t25, e = mj("t25", bat20, c["LO"])
    E(e)
    t26, e = hjs("t26", t25, t24, lambda: ops.hashjoin_an(t25, t24))
    E(e)
    bat28 = t26.mirror_head().clear_head()
    tAR, e = fj("tAR", bat28, c["LR"])
    E(e)
    tAS, e = fj("tAS", bat28, c["LSC"])
    E(e)
    ar = _A(AS_RESINT, R["tAP"] if reenc else len(AS_RESINT) - 1, 64)
    tAP, e = ops.arithmetic_an(SUB, RESINT, tAR, tAS, ar[0], ar[1])
    E(e)
    t29, e = fj("t29", bat28, c["LS"])
    E(e)
    t30, e = hjs("t30", t29, t10, lambda: hj(t29, t10, O(last)))
    E(e)
    tAN, e = ops.fetchjoin_an(t30.clear_head(), c[spec.sgroup])  # (a string column there: no re-encoding)
    E(e)
    t32, e = fj("t32", bat28, c["LO"])
    E(e)
    t34, e = hjs("t34", t32, t24, lambda: hj(t32, t24, O(last)))
    E(e)
    tAY, e = fj("tAY", t34.clear_head(), c["DY"], "S")
    E(e)
    t36, e = fj("t36", bat28, c["LP"])
    E(e)
    batPP = c["PP"].reverse()
    t38, e = hjs("t38", t36, batPP, lambda: hj(t36, batPP, (t36.head.A, t36.head.Ainv), O(last)))
    E(e)
    tAC, e = ops.fetchjoin_an(t38.clear_head(), c[spec.pgroup])
    E(e)
    g = [O(i) for i in R["groups"]] if reenc else [O(last)] * 3
    gy, fy, e = ops.groupby_an(tAY, g[0][0], g[0][1])
    E(e)
    gn, fn, e = ops.groupby2_an(tAN, gy, fy.count, g[1][0], g[1][1])
    E(e)
    gc, fc, e = ops.groupby2_an(tAC, gn, fn.count, g[2][0], g[2][1])
    E(e)
    rp, e = ops.aggregate_sum_grouped_an(tAP, gc, fc.count, RESBIGINT)
    E(e)
    res.profits = rp
    if name == "q42":
        rn, e = ops.fetchjoin_an(fc, tAN)
        E(e)
        ry, e = fj("ry", fc, tAY, "S")
        E(e)
    else:
        ry, e = fj("ry", fc, tAY, "S")
        E(e)
        rn, e = ops.fetchjoin_an(fc, tAN)
        E(e)
    rc, e = ops.fetchjoin_an(fc, tAC)
    E(e)
    res.years = ry
    res.extra["s_group"], res.extra["p_group"] = rn, rc
    return res


def q42(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema] = None) -> ProgramResult:
    """SSB Q4.2: by d_year, s_nation, p_category where c_region = s_region =
    'AMERICA', p_mfgr in ('MFGR#1', 'MFGR#2'), d_year in (1997, 1998)."""
    return _q4x(ops, schema, placement, plain, Q4X_SPECS["q42"], "q42")


def q43(ops, schema: StarSchema, placement: str, plain: Optional[StarSchema] = None) -> ProgramResult:
    """SSB Q4.3: by d_year, s_city, p_brand where s_nation = 'UNITED STATES',
    p_category = 'MFGR#14', d_year in (1997, 1998)."""
    return _q4x(ops, schema, placement, plain, Q4X_SPECS["q43"], "q43")


# ------------------------------------------------------------ DMR baseline
class ModularityError(RuntimeError):
    """The replicas' results differ (the reference's modularity_exception,
    include/util/ModularRedundant.hpp:32-35)."""


# The result the reference's DMR vote compares: Q1.x their single value; the
# grouped programs make a tuple of result BATs (ssbm-qNN_dmr_seq.cpp,
# `results[k] = std::make_tuple(...)`), and the tuple vote compares the size
# and the tail values of the tuple's FIRST BAT only -- its per-element helper
# reads element 0 at every step (ModularRedundant.hpp:226-243) -- so a
# difference in the other BATs goes through.
DMR_FIRST = {"q11": "total", "q12": "total", "q13": "total",
             "q21": "profits", "q22": "profits", "q23": "profits",             # (batRR, batRY, batRB)
             "q31": "nations", "q32": "nations", "q33": "nations", "q34": "nations",  # (batRC, batRS, batRD, batRR)
             "q41": "years", "q42": "years", "q43": "years"}                   # (batRY, ...)


def _bat_values(b):
    d = b.tail.data
    if hasattr(d, "cpu"):
        import numpy as np
        from .model import NP_DTYPE, WIDTH
        return np.frombuffer(d[: b.count * WIDTH[b.tail.type]].cpu().numpy().tobytes(), NP_DTYPE[WIDTH[b.tail.type]])
    return d[: b.count]


def _voted_equal(key, a, b) -> bool:
    """The vote's comparison of two replicas' results (ModularRedundant.hpp:
    114-150 for values, :222-243 for result tuples: size, then tail values)."""
    import numpy as np
    if key == "total":
        return a == b
    return a.count == b.count and np.array_equal(_bat_values(a), _bat_values(b))


def _run_replicas(prog, ops, plains, concurrent):
    opss = ops if isinstance(ops, (list, tuple)) else [ops] * len(plains)
    if len(opss) != len(plains):
        raise ValueError("one operator object per replica")
    if concurrent:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(len(plains)) as ex:  # (the operator calls release the GIL)
            return list(ex.map(lambda k: prog(opss[k], None, "normal", plains[k]), range(len(plains))))
    return [prog(opss[k], None, "normal", plains[k]) for k in range(len(plains))]


def tmr(prog, ops, plains: List[StarSchema], concurrent: bool = False) -> ProgramResult:
    """Triple modular redundancy: the program's normal placement on three
    replicas of the unencoded tables and the reference's majority vote for
    three values (ModularRedundant.hpp:155-200): replica 0's result when it
    equals replica 1's or replica 2's, else replica 1's when 1 and 2 agree,
    else ModularityError (whose message the reference keeps as "DMR: values do
    not match").  The results are compared as the DMR vote compares them (the
    first BAT of a grouped program's result tuple).  The reference defines this
    vote but ships no TMR program; this runs its DMR programs with a third
    replica."""
    if len(plains) != 3:
        raise ValueError("TMR takes three replicas")
    results = _run_replicas(prog, ops, plains, concurrent)
    key = DMR_FIRST[prog.__name__]
    v = [getattr(r, key) for r in results]
    if _voted_equal(key, v[0], v[1]) or _voted_equal(key, v[0], v[2]):
        return results[0]
    if _voted_equal(key, v[1], v[2]):
        return results[1]
    raise ModularityError("DMR: values do not match")


def dmr(prog, ops, plains: List[StarSchema], concurrent: bool = False) -> ProgramResult:
    """Dual modular redundancy, the reference's baseline for AN coding: the
    program's normal placement runs once on each replica of the unencoded
    tables (ssbm-q11_dmr_seq.cpp:80-131; `_mt`: the replicas in parallel,
    ssbm-q11_dmr_mt.cpp:85), then the results are voted on
    (ModularRedundant.hpp:114-150): equal -> replica 0's result, else
    ModularityError.  `ops` is one operator object, or one per replica (for
    the concurrent form: separate GPU contexts, each with its own stream)."""
    import numpy as np
    if len(plains) != 2:
        raise ValueError("DMR takes two replicas")
    results = _run_replicas(prog, ops, plains, concurrent)
    key = DMR_FIRST[prog.__name__]
    a, b = (getattr(r, key) for r in results)
    if key == "total":
        if a != b:
            raise ModularityError("DMR: values do not match")
    else:
        if a.count != b.count:
            raise ModularityError("DMR: size does not match")
        if not np.array_equal(_bat_values(a), _bat_values(b)):
            raise ModularityError("DMR: content does not match")
    return results[0]


# ----------------------------------------- the programs as fused star queries
def _dp(dim, attr, op1, v1, op2=CMP_NONE, v2=0, comb=AND) -> DimPred:
    return DimPred(dim, attr, op1, v1, op2, v2, comb)


_CITY_KI = (EQ, city_code("UNITED KI1"), EQ, city_code("UNITED KI5"), OR)
_US = NATION["UNITED STATES"]


def program_query(name: str, fact_rows: Optional[int] = None) -> StarQuery:
    """SSB program `name` (q11 ... q43) as one star query of the fused engine:
    the program's selections, groups and measure on the same integer
    attribute codes.  On clean data its answer equals the program's in every
    placement; under bit flips it detects as pipelines.starjoin_continuous
    composes the operators (fact predicates and foreign keys, then the
    measures, dropped row-consistently)."""
    if name in Q1_SPECS:
        sp = Q1_SPECS[name]
        q1, q2, q3, q4, q5 = sp.quantity
        return StarQuery([_dp("date", a, EQ, v) for a, v in sp.date], [], fact_rows,
                         [FactPred("quantity", q1, q2, q3, q4, q5),
                          FactPred("discount", GE, sp.discount[0], LE, sp.discount[1], AND)], "price_discount")
    if name in Q2_SPECS:
        region, (pk, p1, pv1, p2, pv2, pc) = Q2_SPECS[name]
        part_attr = {"PC": "category", "PB": "brand"}[pk]
        return StarQuery([_dp("supplier", "region", EQ, REGION[region]), _dp("part", part_attr, p1, pv1, p2, pv2, pc)],
                         [("date", "year"), ("part", "brand")], fact_rows, [], "revenue")
    if name in Q3_SPECS:
        sp = Q3_SPECS[name]
        attr = {"SR": "region", "CR": "region", "SN": "nation", "CN": "nation", "SCI": "city", "CCI": "city",
                "DY": "year", "DM": "yearmonth"}
        preds = [_dp("supplier", attr[sp.supp[0]], *sp.supp[1:]), _dp("customer", attr[sp.cust[0]], *sp.cust[1:]),
                 _dp("date", attr[sp.date[0]], *sp.date[1:])]
        return StarQuery(preds, [("date", "year"), ("customer", attr[sp.cgroup]), ("supplier", attr[sp.sgroup])],
                         fact_rows, [], "revenue")
    if name == "q41":
        return StarQuery([_dp("customer", "region", EQ, 1), _dp("supplier", "region", EQ, 1),
                          _dp("part", "mfgr", EQ, 1, EQ, 2, OR)], [("date", "year"), ("customer", "nation")],
                         fact_rows, [], "profit")
    if name in Q4X_SPECS:
        sp = Q4X_SPECS[name]
        attr = {"PM": "mfgr", "PC": "category", "PB": "brand", "SR": "region", "SN": "nation", "SCI": "city",
                "CR": "region"}
        preds = [_dp("part", attr[sp.part[0]], *sp.part[1:]), _dp("supplier", attr[sp.supp[0]], *sp.supp[1:]),
                 _dp("date", "year", EQ, 1997, EQ, 1998, OR)]
        if sp.cust:
            preds.append(_dp("customer", attr[sp.cust[0]], *sp.cust[1:]))
        return StarQuery(preds, [("date", "year"), ("supplier", attr[sp.sgroup]), ("part", attr[sp.pgroup])],
                         fact_rows, [], "profit")
    raise ValueError(f"unknown program {name}")


# the fields of each grouped program's result, in program_query's group order
PROGRAM_GROUP_FIELDS = {
    "q21": ("years", "brand"), "q22": ("years", "brand"), "q23": ("years", "brand"),
    "q31": ("years", "nations", "snations"), "q32": ("years", "nations", "snations"),
    "q33": ("years", "nations", "snations"), "q34": ("years", "nations", "snations"),
    "q41": ("years", "nations"), "q42": ("years", "s_group", "p_group"), "q43": ("years", "s_group", "p_group"),
}


# ------------------------------------------------ string attribute columns
class StringOps:
    """The operator interface over a schema whose string attributes are STR
    columns (`ssb.with_strings`): selectAN on such a column is the string
    selection (the thresholds, given as the attribute's integer codes, become
    its strings), fetchjoinAN from it the string fetch-join, and the binary
    groupbyAN over a fetched string BAT the string group-by; every other call
    goes to `ops`; select, fetchjoin and the binary groupby likewise for the
    unencoded placements.  With it Q2.x-Q4.x run on string columns in every
    placement as the reference's programs do
    (ssbm-q21_continuous.cpp:87,110,156,174; ssbm-q41_continuous.cpp:101,120,
    142,180).  String tails are not AN-coded, so these steps report no tail
    errors (their vectors are not present)."""

    def __init__(self, ops):
        self.ops = ops

    def __getattr__(self, name):
        return getattr(self.ops, name)

    def select_an(self, b: Bat, op1, th1, op2=CMP_NONE, th2=0, comb=AND, aoid=16089):
        if b.tail.type != STR:
            return self.ops.select_an(b, op1, th1, op2, th2, comb, aoid)
        t1 = b.tail.names(th1)
        t2 = b.tail.names(th2) if op2 != CMP_NONE else b""
        h = self.ops.select_str_an(b.tail.data, b.tail.width, b.head.seqbase, op1, t1, op2, t2, comb)
        if isinstance(h, Col):  # the GPU's form: a resoid column of u64 bytes
            n = h.data.numel() // 8 if h.data is not None else 0
        else:  # the oracle's form: the codes themselves
            n = len(h)
            h = Col(RESOID, h, 65117, ainv(65117, 64), (1 << 56) - 1, 0)
        return Bat(h, Col(STR, None, 1, 1, 0, 0, b.tail.width, b.tail.names), n), ErrVec(None, False)

    def fetchjoin_an(self, a: Bat, b: Bat, **kw):
        if b.tail.type != STR:
            return self.ops.fetchjoin_an(a, b, **kw)
        strs, errs = self.ops.fetchjoin_str_an(a, b.tail.data, b.tail.width)
        n = int(strs.shape[0])
        return Bat(Col(VOID, None, 1, 1, 0, 0), Col(STR, strs.reshape(-1), 1, 1, 0, 0, b.tail.width, b.tail.names),
                   n), errs

    def groupby2_an(self, b: Bat, grouping: Bat, ngroups: int, aoid=65117, aoidinv=0x3E36D3BC8D9BC5F5):
        if b.tail.type != STR:
            return self.ops.groupby2_an(b, grouping, ngroups, aoid, aoidinv)
        return self.ops.groupby2_str_an(b.tail.data, b.tail.width, grouping, ngroups, aoid, aoidinv,
                                        b.head.seqbase)

    # the unencoded twins (normal, early and late placements)
    def select(self, b: Bat, op1, th1, op2=CMP_NONE, th2=0, comb=AND):
        if b.tail.type != STR:
            return self.ops.select(b, op1, th1, op2, th2, comb)
        t1 = b.tail.names(th1)
        t2 = b.tail.names(th2) if op2 != CMP_NONE else b""
        h = self.ops.select_str(b.tail.data, b.tail.width, b.head.seqbase, op1, t1, op2, t2, comb)
        if isinstance(h, Col):  # the GPU's form: an oid_t column of u32 bytes
            n = h.data.numel() // 4 if h.data is not None else 0
        else:
            n = len(h)
            h = Col(OID, h, 1, 1, 0, 0)
        return Bat(h, Col(STR, None, 1, 1, 0, 0, b.tail.width, b.tail.names), n)

    def fetchjoin(self, a: Bat, b: Bat):
        if b.tail.type != STR:
            return self.ops.fetchjoin(a, b)
        strs = self.ops.fetchjoin_str(a, b.tail.data, b.tail.width)
        return Bat(Col(VOID, None, 1, 1, 0, 0), Col(STR, strs.reshape(-1), 1, 1, 0, 0, b.tail.width, b.tail.names),
                   int(strs.shape[0]))

    def groupby2(self, b: Bat, grouping: Bat, ngroups: int):
        if b.tail.type != STR:
            return self.ops.groupby2(b, grouping, ngroups)
        return self.ops.groupby2_str(b.tail.data, b.tail.width, grouping, ngroups, b.head.seqbase)
