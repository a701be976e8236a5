"""Seeded operator parity cases shared by the golden fixtures, the oracle
tests and the GPU parity tests.

A case is ``dict(op=<method name>, args=[Bat | int ...], kwargs={...})``; the
method names are those of the reference's operators (``selectAN`` ->
``select_an`` ...) and exist on both ``oracle.oracle.Oracle`` and
``ahead_b200.gpu.GpuOps``.  ``run_case`` normalises every result to a flat list
of host ``Bat`` / ``ErrVec`` / ``int`` items so outputs compare bit for bit.
"""
from __future__ import annotations

import json
from typing import Any, Dict, List

import numpy as np

from ahead_b200.model import (ADD, AND, DIV, EQ, GE, GT, HASH_LEFT, HASH_RIGHT, INT, LE, LT, MUL, NE, OID, OR,
                              RESBIGINT, RESINT, RESOID, RESSHORT, RESTINY, SHORTINT, SUB, TINYINT, VOID, WIDTH,
                              BIGINT, Bat, Col, ErrVec, ainv, void_col, NP_DTYPE)
from bats import encoded_col, flip_bits, oid_list, random_encoded

HI = {RESTINY: 256, RESSHORT: 65536, RESINT: 1 << 32, RESBIGINT: 1 << 40}


def _sel(oids, A=65117):
    o = oid_list(np.sort(np.asarray(oids, dtype=np.uint64)), A)
    return Bat(o.tail, o.tail, o.count)


def make_cases(seed: int = 7, scale: int = 1) -> List[Dict[str, Any]]:
    rng = np.random.default_rng(seed)
    cases: List[Dict[str, Any]] = []
    add = lambda op, *args, **kw: cases.append(dict(op=op, args=list(args), kwargs=kw))

    # ---------------------------------------------------------- selectAN
    for t in (RESTINY, RESSHORT, RESINT):
        for n in (0, 1, 31, 33, 1000 * scale, 5003 * scale):
            b, _, _ = random_encoded(t, n, 0, min(HI[t], 1 << 20), rng, nflips=min(n, 7),
                                     seqbase=int(rng.integers(0, 1000)))
            A = b.tail.A
            hi = min(HI[t], 1 << 20)
            for op1, op2, comb in ((LT, 0, AND), (GE, LE, AND), (EQ, NE, OR), (GT, LT, OR), (NE, 0, AND)):
                add("select_an", b, op1, int(rng.integers(0, hi)) * A, op2, int(rng.integers(0, hi)) * A, comb)
    # unaligned start (a view one element into a column)
    b, _, _ = random_encoded(RESSHORT, 4099, 0, 4000, rng, nflips=3)
    bu = Bat(b.head, Col(RESSHORT, b.tail.data[1:], b.tail.A, b.tail.Ainv, b.tail.unenc_max), b.count - 1)
    add("select_an", bu, GE, 1000 * b.tail.A, LT, 3000 * b.tail.A, AND)
    # ---------------------------------------------------------- select (unencoded, also on codes: late mode)
    for t, hi in ((TINYINT, 256), (SHORTINT, 65536), (INT, 1 << 32), (BIGINT, 1 << 50), (RESINT, 1 << 32)):
        n = 3001 * scale
        vals = rng.integers(0, hi, size=n, dtype=np.uint64).astype(NP_DTYPE[WIDTH[t]])
        bb = Bat(void_col(int(rng.integers(0, 50))), Col(t, vals), n)
        add("select", bb, LT, int(rng.integers(0, hi)))
        add("select", bb, GE, int(rng.integers(0, hi // 2)), LE, int(rng.integers(hi // 2, hi)), AND)
    # ---------------------------------------------------------- check / decode
    for t in (RESTINY, RESSHORT, RESINT, RESBIGINT, RESOID):
        for n in (0, 7, 2000 * scale):
            b, _, _ = random_encoded(t, n, 0, min(HI.get(t, 1 << 32), 1 << 30), rng, nflips=min(n, 9),
                                     A={RESOID: 65117, RESBIGINT: 65117}.get(t))
            add("check_an", b, b.tail.Ainv, b.tail.unenc_max)
            add("check_and_decode_an", b)
            if n:
                o = oid_list(np.arange(n), 65117)
                flip_bits(o.tail.data, 2, rng)
                gb = Bat(o.tail, b.tail, n)
                add("check_and_decode_an", gb)
                add("decode_an", gb)
                ob = Bat(Col(OID, np.arange(n, dtype=np.uint32) + 5), b.tail, n)
                add("check_and_decode_an", ob)
    # all-corrupt column
    b, _, _ = random_encoded(RESSHORT, 500, 0, 100, rng)
    b.tail.data[:] ^= np.uint32(1 << 31)
    add("check_and_decode_an", b)
    add("select_an", b, LT, 50 * b.tail.A)
    # ---------------------------------------------------------- encodeAN
    for t, hi in ((TINYINT, 256), (SHORTINT, 65536), (INT, 1 << 32)):
        vals = rng.integers(0, hi, size=777, dtype=np.uint64).astype(NP_DTYPE[WIDTH[t]])
        add("encode_an", Bat(void_col(3), Col(t, vals), 777), {TINYINT: 233, SHORTINT: 63877, INT: 65117}[t])
    # ---------------------------------------------------------- hashjoinAN
    for T in (RESTINY, RESSHORT, RESINT):
        for nl, nr in ((0, 5), (5, 0), (1, 1), (300 * scale, 60), (3000 * scale, 700)):
            hi = min(HI[T], 1 << 20)
            keys = rng.choice(hi, size=nr, replace=nr > hi).astype(np.uint64)
            if nr > 3:
                keys[2] = keys[1]  # a duplicate build key
            r = encoded_col(T, keys)
            flip_bits(r.tail.data, min(nr, 2), rng)
            rr = r.reverse()
            fk = (rng.choice(keys, size=nl) if nr else rng.integers(0, hi, size=nl)).astype(np.uint64)
            l = encoded_col(T, fk)
            flip_bits(l.tail.data, min(nl, 4), rng)
            for side in (HASH_RIGHT, HASH_LEFT):
                for rh, rt in ((0, 0), (1, 0), (1, 1)):
                    add("hashjoin_an", l, rr, reenc_head=rh, ah1r=32417, ah1invr=ainv(32417, 64), reenc_tail=rt,
                        at2r=7841, at2invr=ainv(7841, 64), side=side)
            if nl:
                sel = oid_list(np.sort(rng.choice(nl, size=min(nl, 40), replace=False)))
                lf = Bat(sel.tail, Col(T, l.tail.data[: sel.count].copy(), l.tail.A, l.tail.Ainv, l.tail.unenc_max),
                         sel.count)
                rres = Bat(r.tail, oid_list(np.arange(nr)).tail, nr)  # (key | resoid)
                add("hashjoin_an", lf, rres)
                add("hashjoin_an", lf, rres, reenc_head=1, ah1r=16089, ah1invr=ainv(16089, 64))
    # mixed key widths (resint probe, resshort build)
    keys = rng.choice(60000, size=400, replace=False).astype(np.uint64)
    r = encoded_col(RESSHORT, keys).reverse()
    l = encoded_col(RESINT, rng.choice(keys, size=2000).astype(np.uint64))
    flip_bits(l.tail.data, 6, rng)
    add("hashjoin_an", l, r)
    add("hashjoin_an", l, r, side=HASH_LEFT)
    # unencoded hash join
    for t, hi in ((INT, 1 << 20), (RESINT, 1 << 20)):
        keys = rng.choice(hi, size=500, replace=False).astype(np.uint64)
        keys[7] = keys[3]
        rb = Bat(Col(t, keys.astype(NP_DTYPE[WIDTH[t]])), void_col(11), 500)
        lb = Bat(void_col(0), Col(t, rng.choice(keys, size=4000).astype(NP_DTYPE[WIDTH[t]])), 4000)
        add("hashjoin", lb, rb)
        add("hashjoin", lb, rb, side=HASH_LEFT)
    # ---------------------------------------------------------- matchjoinAN / fetchjoinAN
    for T in (RESTINY, RESSHORT, RESINT, RESBIGINT):
        n = 3000 * scale
        col, _, _ = random_encoded(T, n, 0, 200, rng, nflips=6, A={RESBIGINT: 65117}.get(T))
        oids = np.sort(rng.choice(n, size=700, replace=False))
        ol = oid_list(oids)
        flip_bits(ol.tail.data, 2, rng)
        sel = Bat(ol.tail, ol.tail, ol.count)
        add("matchjoin_an", sel, col)
        add("matchjoin_an", sel, col, True, 32417, ainv(32417, 64), 7, ainv(7, 8 * WIDTH[T]))
        fl = Bat(void_col(), ol.tail, ol.count)
        add("fetchjoin_an", fl, col)
        add("fetchjoin_an", fl, col, True, 13, ainv(13, 8 * WIDTH[T]))
        o2 = oid_list(np.sort(rng.choice(n, size=900, replace=False)))
        s2 = Bat(o2.tail, o2.tail, o2.count)
        add("matchjoin_an", sel, s2)
        clean = oid_list(oids)
        add("matchjoin_an", Bat(clean.tail, clean.tail, clean.count), s2)
        bT = Bat(o2.tail, Col(T, col.tail.data[: o2.count].copy(), col.tail.A, col.tail.Ainv, col.tail.unenc_max),
                 o2.count)
        add("matchjoin_an", sel, bT)
        add("matchjoin_an", sel, bT, True, 32417, ainv(32417, 64), 7, ainv(7, 8 * WIDTH[T]))
        vv = Bat(ol.tail, void_col(3), ol.count)
        for sb in (0, 3, 10):
            add("matchjoin_an", vv, Bat(void_col(sb), col.tail, col.count))
        # (resint | void) x (resoid | resoid): key map of a dimension
        km = Bat(encoded_col(RESINT, np.arange(n) * 3 + 1).tail, void_col(0), n)
        add("matchjoin_an", km, s2)
    # unencoded matchjoin / fetchjoin
    n = 2000
    vals = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    colp = Bat(void_col(), Col(INT, vals), n)
    o = np.sort(rng.choice(n, size=300, replace=False)).astype(np.uint32)
    o2 = np.sort(rng.choice(n, size=500, replace=False)).astype(np.uint32)
    add("matchjoin", Bat(Col(OID, o), Col(OID, o), 300), colp)
    add("matchjoin", Bat(Col(OID, o), Col(OID, o), 300), Bat(Col(OID, o2), Col(OID, o2), 500))
    add("matchjoin", Bat(Col(OID, o), void_col(5), 300), Bat(void_col(0), Col(INT, vals), n))
    add("fetchjoin", Bat(void_col(), Col(OID, o), 300), colp)
    # ---------------------------------------------------------- groupby / aggregation / arithmetic
    for T in (RESTINY, RESSHORT, RESINT):
        n = 4000 * scale
        g1, _, _ = random_encoded(T, n, 0, 7, rng, nflips=3)
        g2, _, _ = random_encoded(T, n, 0, 40, rng, nflips=3)
        add("groupby_an", g1)
        add("groupby_an", Bat(oid_list(np.arange(n)).tail, g1.tail, n))
        cases.append(dict(op="groupby_chain", args=[g1, g2], kwargs={}))
        price, _, _ = random_encoded(RESINT, n, 90000, 11000000, rng, nflips=2)
        d, _, _ = random_encoded(T, n, 0, 11, rng, nflips=2)
        add("aggregate_mul_sum_an", price, d)
        for op in (ADD, SUB, MUL):
            for rt in (RESINT, RESBIGINT):
                add("arithmetic_an", op, rt, price, d, 65117, ainv(65117, 64))
        dnz, _, _ = random_encoded(T, n, 1, 11, rng)
        add("arithmetic_an", DIV, RESBIGINT, price, dnz, 65117, ainv(65117, 64))
    qa = Bat(void_col(), Col(INT, rng.integers(0, 1000, size=999, dtype=np.uint64).astype(np.uint32)), 999)
    qb = Bat(void_col(), Col(TINYINT, rng.integers(0, 11, size=999, dtype=np.uint64).astype(np.uint8)), 999)
    add("aggregate_mul_sum", qa, qb)
    # ---------------------------------------------------------- unencoded twins: groupby, sums, arithmetic
    # (values stay below each type's maximum: the reference's dictionary uses it as its empty key)
    gb_hi = {OID: 60, TINYINT: 200, SHORTINT: 900, INT: 5000, RESOID: 50, RESTINY: 40, RESSHORT: 70, RESINT: 90}
    for t, hi in gb_hi.items():
        for n in (0, 1, 1500 * scale):
            for oid_head in (False, True):
                vals = rng.integers(0, hi, size=n, dtype=np.uint64).astype(NP_DTYPE[WIDTH[t]])
                head = Col(OID, (rng.permutation(n) + 11).astype(np.uint32)) if oid_head else void_col(int(rng.integers(0, 9)))
                b = Bat(head, Col(t, vals), n)
                cases.append(dict(op="groupby_plain_chain", args=[b, int(rng.integers(0, 3))], kwargs={}))
    for t in (TINYINT, INT):  # binary keys that wrap in the larger type (u16 for tinyint)
        n = 800
        vals = rng.integers(0, 150, size=n, dtype=np.uint64).astype(NP_DTYPE[WIDTH[t]])
        grp = Bat(void_col(), Col(OID, rng.integers(0, 700, size=n, dtype=np.uint64).astype(np.uint32)), n)
        add("groupby2", Bat(void_col(), Col(t, vals), n), grp, 70000)
    for rt, t in ((TINYINT, TINYINT), (SHORTINT, TINYINT), (BIGINT, TINYINT), (INT, SHORTINT), (INT, INT),
                  (BIGINT, INT), (BIGINT, BIGINT)):
        n = 2000 * scale
        vals = rng.integers(0, 1 << min(8 * WIDTH[t], 62), size=n, dtype=np.uint64).astype(NP_DTYPE[WIDTH[t]])
        add("aggregate_sum", Bat(Col(OID, np.arange(n, dtype=np.uint32)), Col(t, vals), n), rt)
    for t in (INT, RESINT):
        n = 1700 * scale
        hi = 1 << (32 if t == INT else 48)
        x = Bat(void_col(3), Col(t, rng.integers(1, hi, size=n, dtype=np.uint64).astype(NP_DTYPE[WIDTH[t]]), 65117), n)
        y = Bat(void_col(5), Col(t, rng.integers(1, hi, size=n, dtype=np.uint64).astype(NP_DTYPE[WIDTH[t]])), n)
        for op in (ADD, SUB, MUL, DIV):
            add("arithmetic", op, t, x, y)
    return cases


def _norm(x) -> List[Any]:
    if isinstance(x, tuple):
        out = []
        for y in x:
            out.extend(_norm(y))
        return out
    if isinstance(x, list):
        out = []
        for y in x:
            out.extend(_norm(y))
        return out
    return [x]


def run_case(impl, case, to_dev=None, to_hst=None, err_hst=None) -> List[Any]:
    """Run one case on an oracle or on the GPU (with device conversion hooks)."""
    args = [to_dev(a) if (to_dev and isinstance(a, Bat)) else a for a in case["args"]]
    if case["op"] == "groupby_chain":
        # unary group-by, binary group-by on it, then the grouped sum
        g1, g2 = args
        gids, firsts, e1 = impl.groupby_an(g1)
        ng = firsts.count
        gids2, firsts2, e2 = impl.groupby2_an(g2, gids, ng)
        sums, e3 = impl.aggregate_sum_grouped_an(g1, gids2, firsts2.count)
        res = [gids, firsts, e1, gids2, firsts2, e2, sums, e3]
    elif case["op"] == "groupby_plain_chain":
        # unencoded: unary group-by, binary group-by on a second column, grouped int sums
        b, shift = args
        gids, firsts = impl.groupby(b)
        n = b.count
        hb = to_hst(b) if to_hst else b
        tail2 = ((np.asarray(hb.tail.data) >> shift) % 7).astype(np.uint32) if n else np.zeros(0, np.uint32)
        b2 = Bat(hb.head, Col(INT, tail2), n)
        b2 = to_dev(b2) if to_dev else b2
        gids2, firsts2 = impl.groupby2(b2, gids, firsts.count)
        sums = impl.aggregate_sum_grouped(b2, gids2, firsts2.count)
        res = [gids, firsts, gids2, firsts2, sums]
    else:
        res = getattr(impl, case["op"])(*args, **case["kwargs"])
    items = _norm(res)
    out = []
    for it in items:
        if isinstance(it, Bat) and to_hst:
            out.append(to_hst(it))
        elif isinstance(it, ErrVec) and err_hst:
            out.append(err_hst(it))
        else:
            out.append(it)
    return out


def assert_same(a: List[Any], b: List[Any], what: str = ""):
    assert len(a) == len(b), f"{what}: {len(a)} vs {len(b)} outputs"
    for i, (x, y) in enumerate(zip(a, b)):
        tag = f"{what} item {i}"
        if isinstance(x, Bat):
            assert isinstance(y, Bat), tag
            assert x.count == y.count, f"{tag}: count {x.count} vs {y.count}"
            for nm in ("head", "tail"):
                cx, cy = getattr(x, nm), getattr(y, nm)
                assert cx.type == cy.type, f"{tag} {nm}: type {cx.type} vs {cy.type}"
                assert (cx.A, cx.Ainv, cx.unenc_max, cx.seqbase) == (cy.A, cy.Ainv, cy.unenc_max, cy.seqbase), \
                    f"{tag} {nm}: meta {cx.meta()} vs {cy.meta()}"
                assert (cx.data is None) == (cy.data is None), f"{tag} {nm}: filled vs unfilled column"
                if cx.type != VOID and x.count and cx.data is not None:
                    dx = np.asarray(cx.data)[: x.count]
                    dy = np.asarray(cy.data)[: y.count]
                    if not np.array_equal(dx, dy):
                        bad = np.nonzero(dx != dy)[0]
                        raise AssertionError(f"{tag} {nm}: {len(bad)} rows differ, first at {bad[0]}: "
                                             f"{dx[bad[0]]} vs {dy[bad[0]]}")
        elif isinstance(x, ErrVec):
            assert x.present == y.present, f"{tag}: present {x.present} vs {y.present}"
            if x.present:
                vx = np.asarray(x.values if x.values is not None else [], dtype=np.uint64)
                vy = np.asarray(y.values if y.values is not None else [], dtype=np.uint64)
                assert np.array_equal(vx, vy), f"{tag}: errors {vx[:8]} vs {vy[:8]} (n {len(vx)} vs {len(vy)})"
        else:
            assert int(x) == int(y), f"{tag}: {x} vs {y}"


# ------------------------------------------------------------- serialisation
def _col_meta(c: Col) -> dict:
    return dict(type=c.type, A=c.A, Ainv=str(c.Ainv), unenc_max=str(c.unenc_max), seqbase=str(c.seqbase))


def save_cases(path_prefix: str, cases, outputs):
    arrays = {}
    manifest = []
    seen = {}  # identical input arrays are stored once

    def put_bat(b: Bat, key: str):
        d = dict(kind="bat", count=b.count, head=_col_meta(b.head), tail=_col_meta(b.tail))
        for nm in ("head", "tail"):
            c = getattr(b, nm)
            if c.type != VOID and c.data is not None:
                a = np.ascontiguousarray(np.asarray(c.data)[: b.count])
                h = (a.dtype.str, a.shape, hash(a.tobytes()))
                if h not in seen:
                    seen[h] = f"{key}_{nm}"
                    arrays[seen[h]] = a
                d[nm]["key"] = seen[h]
        return d

    def put(x, key):
        if isinstance(x, Bat):
            return put_bat(x, key)
        if isinstance(x, ErrVec):
            d = dict(kind="err", present=bool(x.present))
            if x.present:
                arrays[key] = np.asarray(x.values if x.values is not None else [], dtype=np.uint64)
                d["key"] = key
            return d
        return dict(kind="int", value=str(int(x)))

    for i, (c, o) in enumerate(zip(cases, outputs)):
        manifest.append(dict(op=c["op"], kwargs={k: str(v) for k, v in c["kwargs"].items()},
                             args=[put(a, f"c{i}_a{j}") for j, a in enumerate(c["args"])],
                             out=[put(x, f"c{i}_o{j}") for j, x in enumerate(o)]))
    np.savez_compressed(path_prefix + ".npz", **arrays)
    with open(path_prefix + ".json", "w") as f:
        json.dump(manifest, f)


def load_cases(path_prefix: str):
    arrays = np.load(path_prefix + ".npz")
    with open(path_prefix + ".json") as f:
        manifest = json.load(f)

    def col(d):
        data = arrays[d["key"]] if "key" in d else None
        return Col(d["type"], data, d["A"], int(d["Ainv"]), int(d["unenc_max"]), int(d["seqbase"]))

    def get(d):
        if d["kind"] == "bat":
            return Bat(col(d["head"]), col(d["tail"]), d["count"])
        if d["kind"] == "err":
            return ErrVec(arrays[d["key"]] if d["present"] else None, d["present"])
        return int(d["value"])

    cases, outs = [], []
    for m in manifest:
        kw = {k: int(v) for k, v in m["kwargs"].items()}
        cases.append(dict(op=m["op"], args=[get(a) for a in m["args"]], kwargs=kw))
        outs.append([get(x) for x in m["out"]])
    return cases, outs
