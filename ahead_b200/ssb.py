"""Synthetic SSB-shaped star schema and star-join query descriptions.

The SSB dataset itself is not available here; seeded synthetic columns with
the schema's shapes stand in for it (lineorder fact table, date / customer /
part / supplier dimensions).  Every column is AN-coded the way the reference
loads it (lib/column_storage/Transaction.cpp:357-376): 8-bit values as
restiny (A = 233), 16-bit as resshort (A = 63877), 32-bit as resint
(A = 65117).

Columns
  date      : datekey (resint, yyyymmdd), year (resshort, 1992..1998),
              yearmonthnum and yearmonth (resint, yyyymm), weeknuminyear (restiny, 1..53)
  customer  : custkey (resint, 1..n), region (restiny, 0..4), nation (resshort, 8*region + 0..7),
              city (resshort, 10*nation + 0..9)
  part      : partkey (resint, 1..n), mfgr (restiny, 1..5), category (resshort, 0..39),
              brand (resshort, 40*category + 0..39)
  supplier  : suppkey (resint, 1..n), region (restiny, 0..4), nation (resshort),
              city (resshort, 10*nation + 0..9)

The reference stores region, nation, city, mfgr, category, brand and yearmonth
as strings; here they are integer dictionary codes, AN-coded like every other
column.  The ones a program fetches with fetchjoinAN are resshort: the
reference's fetchjoinAN check misreports valid 16-bit (restiny) codes.
  lineorder : orderdate, custkey, partkey, suppkey (resint foreign keys),
              quantity (restiny 1..50), discount (restiny 0..10),
              price (resint 90,000..11,000,000, the extended price),
              revenue (resint 80,000..11,000,000), supplycost (resint 1..100,000)
"""
from __future__ import annotations

import datetime
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from .model import (AND, CMP_NONE, EQ, GE, INT, LE, LT, NP_DTYPE, OR, RESINT, RESSHORT, RESTINY, SHORTINT, STR,
                    TINYINT, WIDTH, Bat, Col, an_meta, void_col)

DIMS = ("date", "customer", "part", "supplier")
FK = {"date": "orderdate", "customer": "custkey", "part": "partkey", "supplier": "suppkey"}
KEY = {"date": "datekey", "customer": "custkey", "part": "partkey", "supplier": "suppkey"}
ATTRS = {"date": ("year",), "customer": ("region", "nation"), "part": ("mfgr", "category"),
         "supplier": ("region", "nation")}
# the attributes a fused engine registers per dimension: the query family's
# (ATTRS, packed into the key records) first, then those the SSB programs
# filter or group on (packed when they fit, else joined in row mode)
ENGINE_ATTRS = {"date": ("year", "weeknuminyear", "yearmonthnum", "yearmonth"),
                "customer": ("region", "nation", "city"), "part": ("mfgr", "category", "brand"),
                "supplier": ("region", "nation", "city")}
# fact columns in the fused engine's error-vector order (the foreign keys by dimension, then the rest)
FACT_COLS = ["orderdate", "custkey", "partkey", "suppkey", "price", "discount", "quantity", "revenue", "supplycost"]
# measures of a star query: sum(price * discount), sum(revenue), sum(revenue - supplycost)
MEASURES = ("price_discount", "revenue", "profit")
TYPES = {"datekey": RESINT, "year": RESSHORT, "custkey": RESINT, "partkey": RESINT, "suppkey": RESINT,
         "region": RESTINY, "nation": RESSHORT, "mfgr": RESTINY, "category": RESSHORT, "orderdate": RESINT,
         "quantity": RESTINY, "discount": RESTINY, "price": RESINT, "revenue": RESINT, "supplycost": RESINT,
         "yearmonthnum": RESINT, "yearmonth": RESINT, "weeknuminyear": RESTINY, "city": RESSHORT, "brand": RESSHORT}
# value domain of each dimension attribute (for query generation and dense group indices)
DOMAIN = {("date", "year"): (1992, 1998), ("customer", "region"): (0, 4), ("customer", "nation"): (0, 39),
          ("part", "mfgr"): (1, 5), ("part", "category"): (0, 39), ("supplier", "region"): (0, 4),
          ("supplier", "nation"): (0, 39)}

# SSB cardinalities: SF1-shaped (6M facts) and SF100-shaped (600M facts)
SIZES = {
    "sf1": dict(fact=6_000_000, date=2556, customer=30_000, part=200_000, supplier=2_000),
    "sf100": dict(fact=600_000_000, date=2556, customer=3_000_000, part=1_400_000, supplier=200_000),
}


def date_keys(n: int = 2556) -> np.ndarray:
    d0 = datetime.date(1992, 1, 1)
    out = np.empty(n, dtype=np.uint64)
    for i in range(n):
        d = d0 + datetime.timedelta(days=i)
        out[i] = d.year * 10000 + d.month * 100 + d.day
    return out


def _enc(values: np.ndarray, t: int) -> np.ndarray:
    A = an_meta(t)["A"]
    m = (1 << (8 * WIDTH[t])) - 1
    return ((values.astype(np.uint64) * np.uint64(A)) & np.uint64(m)).astype(NP_DTYPE[WIDTH[t]])


def col_bat(name: str, codes) -> Bat:
    t = TYPES[name]
    m = an_meta(t)
    n = len(codes)
    return Bat(void_col(0), Col(t, codes, m["A"], m["Ainv"], m["unenc_max"], 0), n)


@dataclass
class StarSchema:
    """Host (numpy) or device (torch) BATs of one synthetic star schema."""
    tables: Dict[str, Dict[str, Bat]]
    sizes: Dict[str, int]

    def bat(self, table: str, column: str) -> Bat:
        return self.tables[table][column]


def generate(sizes: Dict[str, int], seed: int = 1) -> StarSchema:
    """Seeded schema in host memory (numpy); values -> AN codes."""
    rng = np.random.default_rng(seed)
    n = sizes
    t: Dict[str, Dict[str, Bat]] = {}
    dk = date_keys(n["date"])
    years = (dk // 10000).astype(np.uint64)
    t["date"] = {"datekey": col_bat("datekey", _enc(dk, RESINT)), "year": col_bat("year", _enc(years, RESSHORT))}
    for dim, key in (("customer", "custkey"), ("supplier", "suppkey")):
        k = np.arange(1, n[dim] + 1, dtype=np.uint64)
        reg = rng.integers(0, 5, n[dim], dtype=np.uint64)
        nat = reg * 8 + rng.integers(0, 8, n[dim], dtype=np.uint64)
        t[dim] = {key: col_bat(key, _enc(k, RESINT)), "region": col_bat("region", _enc(reg, RESTINY)),
                  "nation": col_bat("nation", _enc(nat, TYPES["nation"]))}
    k = np.arange(1, n["part"] + 1, dtype=np.uint64)
    t["part"] = {"partkey": col_bat("partkey", _enc(k, RESINT)),
                 "mfgr": col_bat("mfgr", _enc(rng.integers(1, 6, n["part"], dtype=np.uint64), RESTINY)),
                 "category": col_bat("category", _enc(rng.integers(0, 40, n["part"], dtype=np.uint64),
                                                      TYPES["category"]))}
    nf = n["fact"]
    f = {
        "orderdate": dk[rng.integers(0, n["date"], nf)],
        "custkey": rng.integers(1, n["customer"] + 1, nf, dtype=np.uint64),
        "partkey": rng.integers(1, n["part"] + 1, nf, dtype=np.uint64),
        "suppkey": rng.integers(1, n["supplier"] + 1, nf, dtype=np.uint64),
        "quantity": rng.integers(1, 51, nf, dtype=np.uint64),
        "discount": rng.integers(0, 11, nf, dtype=np.uint64),
        "price": rng.integers(90_000, 11_000_001, nf, dtype=np.uint64),
        "revenue": rng.integers(80_000, 11_000_001, nf, dtype=np.uint64),
        "supplycost": rng.integers(1, 100_001, nf, dtype=np.uint64),
    }
    t["lineorder"] = {c: col_bat(c, _enc(v, TYPES[c])) for c, v in f.items()}
    _more_attributes(t, n, seed)
    return StarSchema(t, dict(sizes))


def _more_attributes(t, n, seed: int):
    """The attributes only the wider SSB programs read, from a generator of
    their own (the columns above stay the same for a seed)."""
    rng = np.random.default_rng(seed + 7919)
    dec = lambda d, c: (t[d][c].tail.data.astype(np.uint64) * np.uint64(t[d][c].tail.Ainv)) \
        & np.uint64((1 << (8 * WIDTH[t[d][c].tail.type])) - 1)
    dk = date_keys(n["date"])
    ym = dk // 100
    doy = np.array([datetime.date(int(k // 10000), int(k // 100 % 100), int(k % 100)).timetuple().tm_yday
                    for k in dk], dtype=np.uint64)
    t["date"]["yearmonthnum"] = col_bat("yearmonthnum", _enc(ym, TYPES["yearmonthnum"]))
    t["date"]["yearmonth"] = col_bat("yearmonth", _enc(ym, TYPES["yearmonth"]))
    t["date"]["weeknuminyear"] = col_bat("weeknuminyear", _enc(1 + (doy - 1) // 7, TYPES["weeknuminyear"]))
    for dim in ("customer", "supplier"):
        city = dec(dim, "nation") * np.uint64(10) + rng.integers(0, 10, n[dim], dtype=np.uint64)
        t[dim]["city"] = col_bat("city", _enc(city, TYPES["city"]))
    brand = dec("part", "category") * np.uint64(40) + rng.integers(0, 40, n["part"], dtype=np.uint64)
    t["part"]["brand"] = col_bat("brand", _enc(brand, TYPES["brand"]))


FACT_RANGES = {"custkey": ("customer", 1), "partkey": ("part", 1), "suppkey": ("supplier", 1),
               "quantity": (1, 51), "discount": (0, 11), "price": (90_000, 11_000_001),
               "revenue": (80_000, 11_000_001), "supplycost": (1, 100_001)}


def generate_device(sizes: Dict[str, int], seed: int = 1, device: str = "cuda", flips: int = 0,
                    flip_seed: int = 7) -> StarSchema:
    """The same schema family built directly in device memory (fact tables of
    hundreds of millions of rows are generated on the GPU from a seeded torch
    generator; the small dimensions come from `generate`).  `flips` seeded
    single-bit flips are spread over the fact columns (see `flip_device`)."""
    import torch

    def to_dev(b: Bat) -> Bat:
        c = b.tail
        data = torch.from_numpy(np.ascontiguousarray(c.data).view(np.uint8).copy()).to(device)
        return Bat(b.head, Col(c.type, data, c.A, c.Ainv, c.unenc_max, c.seqbase), b.count)

    host = generate({**sizes, "fact": 0}, seed=seed)
    t = {d: {c: to_dev(b) for c, b in cols.items()} for d, cols in host.tables.items() if d != "lineorder"}
    nf = int(sizes["fact"])
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    dk = torch.from_numpy(date_keys(sizes["date"]).astype(np.int64)).to(device)

    def codes(v, name):
        ty = TYPES[name]
        w = WIDTH[ty]
        v.mul_(an_meta(ty)["A"])
        b = v.view(torch.uint8).view(-1, 8)
        return b if w == 8 else b[:, :w].contiguous()

    lo = {}
    for name in ("orderdate", "custkey", "partkey", "suppkey", "quantity", "discount", "price", "revenue",
                 "supplycost"):
        if name == "orderdate":
            v = dk[torch.randint(0, sizes["date"], (nf,), generator=g, device=device)]
        else:
            a, b = FACT_RANGES[name]
            hi = sizes[a] + 1 if isinstance(a, str) else b
            v = torch.randint(1 if isinstance(a, str) else a, hi, (nf,), generator=g, device=device, dtype=torch.int64)
        data = codes(v, name).reshape(-1)
        del v
        m = an_meta(TYPES[name])
        lo[name] = Bat(void_col(0), Col(TYPES[name], data, m["A"], m["Ainv"], m["unenc_max"], 0), nf)
    t["lineorder"] = lo
    s = StarSchema(t, dict(sizes))
    if flips:
        flip_device(s, flips, flip_seed)
    # the library launches on a stream of its own: the columns must be complete
    torch.cuda.synchronize()
    return s


def flip_device(schema: StarSchema, nflips: int, seed: int,
                columns=("orderdate", "custkey", "partkey", "suppkey", "quantity", "discount", "price")) -> Dict[str, np.ndarray]:
    """Flip one seeded bit in each of `nflips` seeded (column, row) places of a
    device fact table; returns the flipped rows per column."""
    import torch
    rng = np.random.default_rng(seed)
    n = schema.sizes["fact"]
    col = rng.integers(0, len(columns), nflips)
    out = {}
    for ci, name in enumerate(columns):
        rows = np.unique(rng.integers(0, n, int((col == ci).sum())))
        if not len(rows):
            continue
        b = schema.tables["lineorder"][name]
        w = WIDTH[b.tail.type]
        bits = rng.integers(0, 8 * w, len(rows))
        idx = torch.from_numpy((rows * w + bits // 8).astype(np.int64)).to(b.tail.data.device)
        mask = torch.from_numpy((1 << (bits % 8)).astype(np.uint8)).to(b.tail.data.device)
        b.tail.data[idx] ^= mask
        out[name] = rows
    return out


UNENC = {RESTINY: TINYINT, RESSHORT: SHORTINT, RESINT: INT}


def decoded(schema: StarSchema) -> StarSchema:
    """The unencoded tables of a host schema (what the reference's `normal`
    programs load): every code times A^-1, narrowed to the unencoded type."""
    t = {}
    for tab, cols in schema.tables.items():
        t[tab] = {}
        for c, b in cols.items():
            ty = b.tail.type
            if ty == STR:  # string columns are not AN-coded
                t[tab][c] = b
                continue
            w = WIDTH[ty]
            v = (b.tail.data.astype(np.uint64) * np.uint64(b.tail.Ainv)) & np.uint64((1 << (8 * w)) - 1 if w < 8 else
                                                                                     0xFFFFFFFFFFFFFFFF)
            u = UNENC[ty]
            t[tab][c] = Bat(void_col(0), Col(u, v.astype(NP_DTYPE[WIDTH[u]]), 1, 1, 0, WIDTH[u]), b.count)
    return StarSchema(t, dict(schema.sizes))


def decoded_device(schema: StarSchema, chunk: int = 1 << 25) -> StarSchema:
    """`decoded` for a device schema (byte tensors), in chunks of rows."""
    import torch
    tdt = {1: torch.uint8, 2: torch.int16, 4: torch.int32, 8: torch.int64}
    t = {}
    for tab, cols in schema.tables.items():
        t[tab] = {}
        for c, b in cols.items():
            ty = b.tail.type
            w, u = WIDTH[ty], UNENC[ty]
            wu = WIDTH[u]
            src = b.tail.data.view(tdt[w]) if w > 1 else b.tail.data
            out = torch.empty(b.count * wu, dtype=torch.uint8, device=b.tail.data.device)
            dst = out.view(tdt[wu]) if wu > 1 else out
            mask = (1 << (8 * w)) - 1 if w < 8 else -1  # (-1: all 64 bits, as a signed int64)
            ainv = b.tail.Ainv & ((1 << (8 * w)) - 1)
            ainv = ainv - (1 << 64) if ainv >= (1 << 63) else ainv
            for i in range(0, b.count, chunk):
                x = src[i:i + chunk].to(torch.int64) & mask
                v = (x * ainv) & mask  # wraps mod 2^64 first, then the mask keeps the code width
                if wu < 8:
                    v = torch.where(v >= (1 << (8 * wu - 1)), v - (1 << (8 * wu)), v) if wu > 1 else v
                dst[i:i + chunk] = v.to(tdt[wu])
            t[tab][c] = Bat(void_col(0), Col(u, out, 1, 1, 0, wu), b.count)
    torch.cuda.synchronize()  # complete before library calls on their own stream read it
    return StarSchema(t, dict(schema.sizes))


TYPE_HEADER = {RESTINY: "RESTINY", RESSHORT: "RESSHORT", RESINT: "RESINT"}


def write_tables(schema: StarSchema, directory: str, suffix: str = "AN", delim: str = "|") -> Dict[str, str]:
    """Write a host schema as `.tbl` text plus header files, the layout the
    reference's loader reads (`<table><suffix>.tbl`,
    `<table><suffix>_header.csv`; values decoded, AN types in the header).
    Returns table -> path prefix."""
    from .ingest import write_tbl
    paths = {}
    for tab, cols in schema.tables.items():
        names, types, values = [], [], []
        for c, b in cols.items():
            ty = b.tail.type
            w = WIDTH[ty]
            m = np.uint64((1 << (8 * w)) - 1)
            names.append(c)
            types.append(TYPE_HEADER[ty])
            values.append(((b.tail.data.astype(np.uint64) * np.uint64(b.tail.Ainv)) & m).astype(np.int64))
        path = f"{directory}/{tab}{suffix}"
        write_tbl(path, names, types, values, delim)
        paths[tab] = path
    return paths


def load_tables(ops, paths: Dict[str, str], **kw) -> Tuple[StarSchema, Dict[str, object]]:
    """Load the tables `write_tables` wrote into device memory through the
    table loader; returns the device schema and the loaded tables."""
    from .ingest import load
    t, loaded = {}, {}
    for tab, path in paths.items():
        lt = load(ops, path, table_name=tab, **kw)
        loaded[tab] = lt
        t[tab] = {c.name: c.bat() for c in lt.columns}
    sizes = {tab: loaded[tab].rows for tab in loaded}
    sizes["fact"] = sizes.pop("lineorder", 0)
    return StarSchema(t, sizes), loaded


def inject_flips(schema: StarSchema, table: str, column: str, nflips: int, seed: int) -> np.ndarray:
    """Flip one seeded bit in `nflips` seeded distinct rows of a host column."""
    rng = np.random.default_rng(seed)
    arr = schema.tables[table][column].tail.data
    rows = np.sort(rng.choice(len(arr), size=min(nflips, len(arr)), replace=False))
    bits = rng.integers(0, arr.dtype.itemsize * 8, size=len(rows))
    for r, b in zip(rows, bits):
        arr[r] ^= np.array(1, dtype=arr.dtype) << np.array(b, dtype=arr.dtype)
    return rows


# ---------------------------------------------------------------- queries
@dataclass
class DimPred:
    """A predicate on one dimension attribute, evaluated on its AN codes."""
    dim: str
    attr: str
    op1: int
    v1: int
    op2: int = CMP_NONE
    v2: int = 0
    comb: int = AND


@dataclass
class FactPred:
    """selectAN on a fact column ("quantity" or "discount"), on its AN codes."""
    col: str
    op1: int
    v1: int
    op2: int = CMP_NONE
    v2: int = 0
    comb: int = AND


@dataclass
class StarQuery:
    """select <group attrs>, sum(<measure>) from lineorder ⋈ dims
    where <fact predicates> and <dimension predicates> group by <group
    attrs>, over the first `fact_rows` rows of lineorder.  The measure is one
    of MEASURES (price * discount unless given); at most two dimension
    predicates per dimension, on different attributes (combined with AND)."""
    preds: List[DimPred]
    group: List[Tuple[str, str]]
    fact_rows: Optional[int] = None
    fpreds: List[FactPred] = field(default_factory=list)
    measure: str = "price_discount"

    def dims(self) -> List[str]:
        """Joined dimensions in join order (customer, supplier, part, date)."""
        used = {p.dim for p in self.preds} | {d for d, _ in self.group}
        return [d for d in ("customer", "supplier", "part", "date") if d in used]


def config2_query() -> StarQuery:
    """The single star join of the 6M / 600M configurations: c_region = 1,
    s_region = 1, p_mfgr in [1, 2] (joint selectivity ~1.6%), grouped by
    d_year and p_category (7 x 40 = 280 groups)."""
    return StarQuery(preds=[DimPred("customer", "region", EQ, 1), DimPred("supplier", "region", EQ, 1),
                            DimPred("part", "mfgr", GE, 1, LE, 2, AND)],
                     group=[("date", "year"), ("part", "category")])


def random_query(rng: np.random.Generator, fact_sizes=(1_000_000, 6_000_000, 60_000_000, 600_000_000),
                 max_fact: Optional[int] = None) -> StarQuery:
    """A seeded random star join: predicates on 1-4 dimensions with target
    selectivities 1e-4..0.1, group-by on 0-3 attributes, a fact prefix size."""
    ndims = int(rng.integers(1, 5))
    dims = list(rng.choice(list(DIMS), size=ndims, replace=False))
    target = float(np.exp(rng.uniform(np.log(1e-4), np.log(0.1))))
    per = target ** (1.0 / ndims)
    preds = []
    for d in dims:
        attr = ATTRS[d][int(rng.integers(0, len(ATTRS[d])))]
        lo, hi = DOMAIN[(d, attr)]
        span = hi - lo + 1
        width = max(1, int(round(per * span)))
        a = int(rng.integers(lo, hi - width + 2))
        if width == 1:
            preds.append(DimPred(d, attr, EQ, a))
        else:
            preds.append(DimPred(d, attr, GE, a, LE, a + width - 1, AND))
    ngroup = int(rng.integers(0, 4))
    cands = [(d, a) for d in DIMS for a in ATTRS[d]]
    group = []
    for i in rng.permutation(len(cands))[:ngroup]:
        group.append(cands[int(i)])
    sizes = [s for s in fact_sizes if max_fact is None or s <= max_fact] or [max_fact]
    return StarQuery(preds=preds, group=group, fact_rows=int(sizes[int(rng.integers(0, len(sizes)))]))


# ------------------------------------------------------- string attributes
# The reference loads region, nation, city, mfgr, category and brand as
# STRING:n columns (its lineorder / part / customer / supplier headers); here
# the generator keeps integer dictionary codes, and `with_strings` gives the
# same schema with those attributes as fixed-width string slots in the
# loader's layout (width n + 1, NUL padded), the strings in the order of the
# codes (so range predicates on brands select the same rows either way).
REGION_NAMES = ("AFRICA", "AMERICA", "ASIA", "EUROPE", "MIDDLE EAST")
STRING_WIDTH = {"region": 13, "nation": 16, "city": 11, "mfgr": 7, "category": 8, "brand": 10}


def nation_name(code: int) -> str:
    """Nation k of region k // 8; 12 and 28 are the programs' UNITED STATES and
    UNITED KINGDOM."""
    return {12: "UNITED STATES", 28: "UNITED KINGDOM"}.get(code, f"NATION {code:02d}")


def string_of(attr: str, code: int) -> str:
    if attr == "region":
        return REGION_NAMES[code]
    if attr == "nation":
        return nation_name(code)
    if attr == "city":  # the nation's name cut to 9 characters, then a digit (SSB's format)
        return nation_name(code // 10)[:9].ljust(9) + str(code % 10)
    if attr == "mfgr":
        return f"MFGR#{code}"
    if attr == "category":  # 5 (m - 1) + (c - 1)
        return f"MFGR#{code // 5 + 1}{code % 5 + 1}"
    if attr == "brand":  # 40 * category + bb - 1
        return string_of("category", code // 40) + f"{code % 40 + 1:02d}"
    raise ValueError(attr)


def with_strings(schema: StarSchema) -> StarSchema:
    """The host schema with the string attributes of customer, supplier and
    part as STR columns (the integer columns are replaced)."""
    t = {d: dict(cols) for d, cols in schema.tables.items()}
    for d, attrs in (("customer", ("region", "nation", "city")), ("supplier", ("region", "nation", "city")),
                     ("part", ("mfgr", "category", "brand"))):
        for a in attrs:
            b = t[d][a]
            w = STRING_WIDTH[a]
            dec = (np.asarray(b.tail.data).astype(np.uint64) * np.uint64(b.tail.Ainv)) & np.uint64(
                (1 << (8 * WIDTH[b.tail.type])) - 1)
            names = {}
            slots = np.zeros((b.count, w), np.uint8)
            for i, v in enumerate(dec.tolist()):
                if v not in names:
                    names[v] = string_of(a, int(v)).encode()
                s = names[v]
                slots[i, : len(s)] = np.frombuffer(s, np.uint8)
            fn = (lambda attr: (lambda code: string_of(attr, int(code)).encode()))(a)
            t[d][a] = Bat(b.head, Col(STR, slots.reshape(-1), 1, 1, 0, 0, w, fn), b.count)
    return StarSchema(t, dict(schema.sizes))
