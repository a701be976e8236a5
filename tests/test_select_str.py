"""selectAN / select over string tails (selectAN_scalar.tcc:98-131, 185-222;
Normal/select_scalar.tcc:78-101, 137-165): a row is kept when
Op(strcmp(row, threshold), 0) holds; the AN form writes (seqbase + i) * 65117.

CPU: the C restatement against the reference's own templates (when they are
built here) and against Python's unsigned byte-string order, on rows with NUL
padding, empty and full-width strings and bytes >= 0x80.
GPU: the library against the restatement, on the same cases, on SSB-shaped
dimension columns of up to 3,000,000 rows, on a STRING column brought in by
the table loader, and on its argument errors.
"""
import os

import numpy as np
import pytest

from oracle.oracle import REF_LIB, Oracle

RESOID_A = 65117
LT, LE, EQ, NE, GE, GT = 1, 2, 3, 4, 5, 6
AND, OR = 0, 1
OPS = (LT, LE, EQ, NE, GE, GT)
ALPHABET = np.frombuffer(b"ABab\x7f\x80\xc3\xff 1", dtype=np.uint8)


def _rows(rng, n, width, full=0.1, empty=0.05):
    """n rows of `width` bytes: random strings from a small alphabet (so that
    equal prefixes are common), NUL padded; some fill the whole slot, some are
    empty."""
    out = np.zeros((n, width), dtype=np.uint8)
    lens = rng.integers(0, width + 1, n)
    lens[rng.random(n) < full] = width
    lens[rng.random(n) < empty] = 0
    for i in range(n):
        out[i, : lens[i]] = rng.choice(ALPHABET, lens[i])
    return out.reshape(-1)


def _thresholds(rng, rows, width, k):
    """Thresholds: existing rows (NUL-terminated), their prefixes and
    extensions, the empty string and random strings."""
    n = len(rows) // width
    out = [b""]
    for _ in range(k):
        r = bytes(rows[int(rng.integers(0, n)) * width:][:width]).split(b"\0")[0]
        c = int(rng.integers(0, 4))
        if c == 0:
            out.append(r)
        elif c == 1:
            out.append(r[: max(0, len(r) - 1)])
        elif c == 2:
            out.append(r + b"A")
        else:
            out.append(bytes(rng.choice(ALPHABET, int(rng.integers(1, width + 2)))))
    return out


def _py_select(rows, width, seqbase, op1, th1, op2=0, th2=b"", comb=AND):
    """Python's bytes order is the unsigned lexicographic order strcmp's sign follows."""
    def holds(op, a, b):
        c = (a > b) - (a < b)
        return {LT: c < 0, LE: c <= 0, EQ: c == 0, NE: c != 0, GE: c >= 0, GT: c > 0}[op]

    keep = []
    for i in range(len(rows) // width):
        s = bytes(rows[i * width:(i + 1) * width]).split(b"\0")[0]
        k = holds(op1, s, th1)
        if op2:
            b = holds(op2, s, th2)
            k = (k or b) if comb == OR else (k and b)
        if k:
            keep.append((seqbase + i) & 0xFFFFFFFF)
    return np.array(keep, dtype=np.uint64)


def _cases(seed, n, width, k=6):
    rng = np.random.default_rng(seed)
    rows = _rows(rng, n, width)
    ths = _thresholds(rng, rows, width, k)
    cases = []
    for op in OPS:
        for th in ths:
            cases.append((op, th, 0, b"", AND))
    for _ in range(24):
        a, b = ths[int(rng.integers(0, len(ths)))], ths[int(rng.integers(0, len(ths)))]
        cases.append((int(rng.choice(OPS)), a, int(rng.choice(OPS)), b, int(rng.integers(0, 2))))
    return rows, cases


@pytest.mark.parametrize("width", [1, 8, 26])
def test_restatement_against_python_order(width):
    port = Oracle("port")
    rows, cases = _cases(10 + width, 700, width)
    for seqbase in (0, 4_294_967_000):
        for op1, th1, op2, th2, comb in cases:
            want = _py_select(rows, width, seqbase, op1, th1, op2, th2, comb)
            got = port.select_str(rows, width, seqbase, op1, th1, op2, th2, comb)
            assert np.array_equal(got.astype(np.uint64), want), (op1, th1, op2, th2, comb)
            got_an = port.select_str_an(rows, width, seqbase, op1, th1, op2, th2, comb)
            assert np.array_equal(got_an, want * np.uint64(RESOID_A)), (op1, th1, op2, th2, comb)


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="the reference's operators are not built here")
@pytest.mark.parametrize("width", [1, 11, 26])
def test_restatement_against_reference(width):
    """The reference's own Selection(AN)1/2<..., v2_void_t, v2_str_t> templates."""
    port, ref = Oracle("port"), Oracle("reference")
    rows, cases = _cases(20 + width, 900, width)
    for op1, th1, op2, th2, comb in cases:
        for fn in ("select_str", "select_str_an"):
            a = getattr(port, fn)(rows, width, 77, op1, th1, op2, th2, comb)
            b = getattr(ref, fn)(rows, width, 77, op1, th1, op2, th2, comb)
            assert a.dtype == b.dtype and np.array_equal(a, b), (fn, op1, th1, op2, th2, comb)


def test_restatement_empty_input():
    port = Oracle("port")
    empty = np.zeros(0, np.uint8)
    assert len(port.select_str_an(empty, 8, 0, EQ, b"x")) == 0
    assert len(port.select_str(empty, 8, 0, NE, b"x", GE, b"", OR)) == 0


# ----------------------------------------------------------------------- GPU
def _dev(torch, rows):
    return torch.from_numpy(np.ascontiguousarray(rows)).to("cuda")


def _host(col, dtype):
    return col.data.cpu().numpy().view(dtype) if col.data.numel() else np.zeros(0, dtype)


@pytest.mark.gpu
@pytest.mark.parametrize("width", [1, 8, 26])
def test_gpu_select_str_matches_oracle(width):
    import torch

    from ahead_b200.gpu import GpuOps
    g = GpuOps(0)
    port = Oracle("port")
    rows, cases = _cases(30 + width, 5000, width)
    d = _dev(torch, rows)
    for seqbase in (0, 4_294_967_000):
        for op1, th1, op2, th2, comb in cases:
            want = port.select_str_an(rows, width, seqbase, op1, th1, op2, th2, comb)
            got = g.select_str_an(d, width, seqbase, op1, th1, op2, th2, comb)
            assert np.array_equal(_host(got, np.uint64), want), (op1, th1, op2, th2, comb)
            want_p = port.select_str(rows, width, seqbase, op1, th1, op2, th2, comb)
            got_p = g.select_str(d, width, seqbase, op1, th1, op2, th2, comb)
            assert np.array_equal(_host(got_p, np.uint32), want_p), (op1, th1, op2, th2, comb)
    g.close()


@pytest.mark.gpu
def test_gpu_select_str_dimension_sizes():
    """SSB-shaped region / nation / city / brand columns of 3,000,000 and
    1,400,000 rows (the SF100 customer and part cardinalities)."""
    import torch

    from ahead_b200.gpu import GpuOps
    g = GpuOps(0)
    port = Oracle("port")
    rng = np.random.default_rng(7)
    regions = [b"AFRICA", b"AMERICA", b"ASIA", b"EUROPE", b"MIDDLE EAST"]
    for n, width, vocab in ((3_000_000, 13, regions),
                            (1_400_000, 10, [b"MFGR#%d%d%02d" % (a, b, c) for a in range(1, 6) for b in range(1, 6)
                                             for c in range(1, 41)])):
        idx = rng.integers(0, len(vocab), n)
        table = np.zeros((len(vocab), width), np.uint8)
        for i, v in enumerate(vocab):
            table[i, : len(v)] = np.frombuffer(v, np.uint8)
        rows = table[idx].reshape(-1)
        d = _dev(torch, rows)
        for op1, th1, op2, th2, comb in ((EQ, vocab[2], 0, b"", AND), (GE, vocab[1], LE, vocab[-2], AND),
                                         (LT, vocab[1], GT, vocab[-2], OR), (NE, vocab[0], 0, b"", AND)):
            want = port.select_str_an(rows, width, 0, op1, th1, op2, th2, comb)
            got = g.select_str_an(d, width, 0, op1, th1, op2, th2, comb)
            assert len(want) > 0 and np.array_equal(_host(got, np.uint64), want), (n, op1, th1)
    g.close()


@pytest.mark.gpu
def test_gpu_select_str_on_loaded_column(tmp_path):
    """A STRING column brought into device memory by the table loader."""
    from ahead_b200 import ingest
    from ahead_b200.gpu import GpuOps
    # no empty field: strtok would merge it with the next delimiter (a short line)
    names = [b"alpha", b"beta", b"z", b"gamma", b"delta", b"\xc3\xa9t\xc3\xa9", b"alpha2", b"AB"]
    lines = [b"%d|%s|" % (i, names[i % len(names)]) for i in range(2000)]
    base = str(tmp_path / "t")
    with open(base + "_header.csv", "w") as f:
        f.write("k|s\nRESINT|STRING:7\n")
    with open(base + ".tbl", "wb") as f:
        f.write(b"\n".join(lines) + b"\n")
    g = GpuOps(0)
    t = ingest.load(g, base, "t", convert_table_files=False)
    col = t["s"]
    assert col.width == 8 and col.count == 2000
    rows = col.data.cpu().numpy()
    port = Oracle("port")
    for op1, th1, op2, th2, comb in ((EQ, b"beta", 0, b"", AND), (GT, b"alpha", LT, b"delta", AND),
                                     (LE, b"", GE, b"\xc3", OR)):
        want = port.select_str_an(rows, col.width, 0, op1, th1, op2, th2, comb)
        got = g.select_str_an(col.data, col.width, 0, op1, th1, op2, th2, comb)
        assert len(want) > 0 and np.array_equal(_host(got, np.uint64), want)
    del t, col
    g.close()


@pytest.mark.gpu
def test_gpu_select_str_arguments():
    import torch

    from ahead_b200.gpu import AheadError, GpuOps
    from ahead_b200.model import UNSUPPORTED
    g = GpuOps(0)
    d = torch.zeros(64, dtype=torch.uint8, device="cuda")
    assert _host(g.select_str_an(d, 8, 5, EQ, b""), np.uint64).tolist() == [(5 + i) * RESOID_A for i in range(8)]
    assert g.select_str(d[:0], 8, 0, EQ, b"").data.numel() == 0
    with pytest.raises(AheadError) as e:
        g.select_str_an(d, 8, 0, EQ, b"x" * 256)
    assert e.value.status == UNSUPPORTED
    with pytest.raises(AheadError):
        g.select_str_an(d, 8, 0, 9, b"x")
    g.close()


# ------------------------------------------------------- hashjoinAN (str tail)
def _join_cases(seed, scale=1):
    """(left, right, right slots, width, kwargs) for the string hash join: a
    void- and a resoid-headed left side, duplicate build keys, bit flips on
    both key columns, both hash sides, plain and re-encoded heads."""
    import sys
    sys.path.insert(0, os.path.dirname(__file__))
    from bats import encoded_col, flip_bits, oid_list

    from ahead_b200.model import HASH_LEFT, HASH_RIGHT, RESINT, RESSHORT, RESTINY, Bat, Col
    rng = np.random.default_rng(seed)
    port = Oracle("port")
    out = []
    for T, hi in ((RESTINY, 256), (RESSHORT, 65536), (RESINT, 1 << 20)):
        for nl, nr in ((0, 5), (5, 0), (1, 1), (400 * scale, 90), (3000 * scale, 700)):
            keys = rng.choice(hi, size=nr, replace=nr > hi).astype(np.uint64)
            if nr > 3:
                keys[2] = keys[1]  # a duplicate build key: two strings per match
            r = encoded_col(T, keys)
            flip_bits(r.tail.data, min(nr, 2), rng)
            rr = r.reverse()
            width = int(rng.choice([1, 7, 26]))
            strs = _rows(rng, nr, width)
            fk = (rng.choice(keys, size=nl) if nr else rng.integers(0, hi, size=nl)).astype(np.uint64)
            l = encoded_col(T, fk)
            flip_bits(l.tail.data, min(nl, 4), rng)
            lefts = [l]
            if nl:
                sel = oid_list(np.arange(nl) * 3 + 1)
                flip_bits(sel.tail.data, min(nl, 2), rng)
                lefts.append(Bat(sel.tail, l.tail, nl))
            for left in lefts:
                for side in (HASH_RIGHT, HASH_LEFT):
                    out.append((left, rr, strs, width, dict(side=side)))
                    out.append((left, rr, strs, width, dict(side=side, reenc_head=True, ah1r=32417,
                                                            ah1invr=port.ainv(32417, 64))))
    return out


def _same_join(a, b):
    ha, sa, ea = a
    hb, sb, eb = b
    assert ha.type == hb.type
    assert np.array_equal(np.asarray(ha.data), np.asarray(hb.data))
    assert np.array_equal(sa, sb)
    for x, y in zip(ea, eb):
        assert x.present == y.present
        if x.present:
            assert np.array_equal(np.asarray(x.values), np.asarray(y.values))


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="the reference's operators are not built here")
def test_hashjoin_str_restatement_against_reference():
    """The reference's own hashjoinANunencHashmap<..., v2_str_t, ...>, including
    the decoded left head it emits when the right side is hashed."""
    port, ref = Oracle("port"), Oracle("reference")
    n = 0
    for l, r, strs, width, kw in _join_cases(3):
        a = port.hashjoin_str_an(l, r, strs, width, **kw)
        b = ref.hashjoin_str_an(l, r, strs, width, **kw)
        _same_join(a, b)
        n += len(a[0].data)
    assert n > 0


def _errvec_host(e):
    from ahead_b200.model import ErrVec
    if not e.present:
        return e
    return ErrVec(e.values.cpu().numpy().view(np.uint64) if hasattr(e.values, "cpu") else e.values, True)


@pytest.mark.gpu
def test_gpu_hashjoin_str_matches_oracle():
    from ahead_b200.gpu import GpuOps
    from ahead_b200.model import Bat, Col
    import torch
    g = GpuOps(0)
    port = Oracle("port")

    def dev(b):
        def col(c):
            return c if c.data is None else Col(c.type, torch.from_numpy(np.ascontiguousarray(c.data).view(np.uint8))
                                                .to("cuda"), c.A, c.Ainv, c.unenc_max, c.seqbase)
        return Bat(col(b.head), col(b.tail), b.count)

    for l, r, strs, width, kw in _join_cases(5, scale=20):
        want = port.hashjoin_str_an(l, r, strs, width, **kw)
        h, s, e = g.hashjoin_str_an(dev(l), dev(r), torch.from_numpy(strs).to("cuda"), width, **kw)
        got_h = Col(h.type, h.data.cpu().numpy().view(want[0].data.dtype) if h.data.numel() else
                    np.zeros(0, want[0].data.dtype))
        _same_join((got_h, s.cpu().numpy(), [_errvec_host(x) for x in e]), want)
    g.close()


# ------------------------------------------------- fetchjoin and groupby2 over strings
def _fetch_group_cases(seed, n=3000, width=26, nstr=300):
    """String slots (a small dictionary, with full-width, empty and high-byte
    rows), a (void, resoid) OID list into them with flipped codes, and a
    (void, resoid) grouping of the fetched rows with flipped codes."""
    from bats import flip_bits, oid_list
    from ahead_b200.model import RESOID, Bat, Col, an_meta, void_col
    rng = np.random.default_rng(seed)
    dic = _rows(rng, nstr, width).reshape(nstr, width)
    oids = rng.integers(0, nstr, n)
    ol = oid_list(oids, 65117)
    flip_bits(ol.tail.data, 20, rng)
    m = an_meta(RESOID, 65117)
    ngroups = 7
    g = (rng.integers(0, ngroups, n).astype(np.uint64) * np.uint64(65117)).astype(np.uint64)
    flip_bits(g, 15, rng)
    grouping = Bat(void_col(0), Col(RESOID, g, 65117, m["Ainv"], m["unenc_max"], 0), n)
    return dic, width, ol, grouping, ngroups


def _fetch_group(o, dic, width, ol, grouping, ngroups):
    got, fe = o.fetchjoin_str_an(ol, dic, width)
    rows = got if len(got) == grouping.count else dic[np.arange(grouping.count) % len(dic)]
    gids, firsts, ge = o.groupby2_str_an(rows, width, grouping, ngroups, seqbase=5)
    return got, fe, gids, firsts, ge


def _same_fetch_group(a, b):
    assert np.array_equal(a[0], b[0])
    for x, y in zip(a[1] + a[4], b[1] + b[4]):
        assert x.present == y.present
        if x.present:
            assert np.array_equal(np.asarray(x.values), np.asarray(y.values))
    for x, y in ((a[2], b[2]), (a[3], b[3])):
        assert x.count == y.count and x.tail.A == y.tail.A
        assert np.array_equal(np.asarray(x.tail.data)[: x.count], np.asarray(y.tail.data)[: y.count])


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="the reference's operators are not built here")
@pytest.mark.parametrize("seed", [1, 2])
def test_fetchjoin_groupby2_str_restatement_against_reference(seed):
    """fetchjoinAN and the binary groupbyAN over string tails: the
    restatement against the reference's own templates (its Java-style string
    hash included), with corrupt OIDs and corrupt grouping codes."""
    port, ref = Oracle("port"), Oracle("reference")
    c = _fetch_group_cases(seed)
    _same_fetch_group(_fetch_group(port, *c), _fetch_group(ref, *c))


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [1, 2])
def test_gpu_fetchjoin_groupby2_str_match_oracle(seed):
    """The GPU's string fetchjoinAN and binary groupbyAN against the
    restatement, on the same cases."""
    import torch
    from ahead_b200.gpu import GpuOps, err_to_host, to_device, to_host
    g = GpuOps(0)
    port = Oracle("port")
    dic, width, ol, grouping, ngroups = _fetch_group_cases(seed, n=30000, nstr=3000)
    want = _fetch_group(port, dic, width, ol, grouping, ngroups)
    ddic = _dev(torch, dic.reshape(-1))
    got, fe = g.fetchjoin_str_an(to_device(ol), ddic, width)
    rows = want[0] if len(want[0]) == grouping.count else dic[np.arange(grouping.count) % len(dic)]
    gids, firsts, ge = g.groupby2_str_an(_dev(torch, rows.reshape(-1)), width, to_device(grouping), ngroups,
                                         seqbase=5)
    have = (got.cpu().numpy(), [err_to_host(e) for e in fe], to_host(gids), to_host(firsts),
            [err_to_host(e) for e in ge])
    _same_fetch_group(have, want)
    g.close()


def _plain_fetch_group(o, dic, width, ol, grouping, ngroups):
    """The unencoded twins on the same shapes: oid_t lists and groupings."""
    from ahead_b200.model import OID, Bat, Col, void_col
    oids = (np.asarray(ol.tail.data).astype(np.uint64) * np.uint64(ol.tail.Ainv)) & np.uint64(0xFFFFFFFF)
    oids = oids[oids < len(dic)].astype(np.uint32)  # (the reference reads past its vector otherwise)
    n = len(oids)
    a = Bat(void_col(0), Col(OID, oids), n)
    g = Bat(void_col(0), Col(OID, (np.arange(n) % ngroups).astype(np.uint32)), n)
    got = o.fetchjoin_str(a, dic, width)
    rows = got if len(got) == n else dic[np.arange(n) % len(dic)]
    gids, firsts = o.groupby2_str(rows, width, g, ngroups, seqbase=3)
    return got, gids, firsts


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="the reference's operators are not built here")
def test_plain_fetchjoin_groupby2_str_restatement_against_reference():
    port, ref = Oracle("port"), Oracle("reference")
    dic, width, ol, grouping, ngroups = _fetch_group_cases(3)
    a, b = _plain_fetch_group(port, dic, width, ol, grouping, ngroups), \
        _plain_fetch_group(ref, dic, width, ol, grouping, ngroups)
    assert np.array_equal(a[0], b[0])
    for x, y in zip(a[1:], b[1:]):
        assert x.count == y.count and np.array_equal(np.asarray(x.tail.data)[: x.count], np.asarray(y.tail.data)[: y.count])


@pytest.mark.gpu
def test_gpu_plain_fetchjoin_groupby2_str_match_oracle():
    import torch
    from ahead_b200.gpu import GpuOps, to_device, to_host
    g = GpuOps(0)
    dic, width, ol, grouping, ngroups = _fetch_group_cases(4, n=30000, nstr=3000)
    want = _plain_fetch_group(Oracle("port"), dic, width, ol, grouping, ngroups)

    class Dev:  # the GPU's wrappers on device copies of the same inputs
        def fetchjoin_str(self, a, strs, w):
            return g.fetchjoin_str(to_device(a), _dev(torch, np.asarray(strs).reshape(-1)), w).cpu().numpy()

        def groupby2_str(self, strs, w, grp, ng, seqbase=0):
            gi, fi = g.groupby2_str(_dev(torch, np.asarray(strs).reshape(-1)), w, to_device(grp), ng, seqbase)
            return to_host(gi), to_host(fi)

    have = _plain_fetch_group(Dev(), dic, width, ol, grouping, ngroups)
    assert np.array_equal(have[0], want[0])
    for x, y in zip(have[1:], want[1:]):
        assert x.count == y.count and np.array_equal(np.asarray(x.tail.data)[: x.count], np.asarray(y.tail.data)[: y.count])
    g.close()
