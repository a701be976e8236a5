"""The table loader (include/ahead_ingest.h): header files, `.tbl` parsing on
the device, `.ahead` column files and the min-BFW re-encode.

CPU: the header reader against the reference's own SSB header files
(tests/golden/ingest, extracted from the reference's headers.tgz), the A
tables against resilience.hpp, the restatement's field conversions against
hand-worked C-library results, the text formatter; the restatement against
the reference's own loader compiled from its sources (oracle/ref_loader.py)
on seeded texts, its .ahead files, min-BFW re-encodes and row limits, and
against the fixtures that loader wrote (tests/golden/ingest/refbin).
GPU: the loader on those fixtures; ahead_gpu_tbl_parse and ahead_gpu_reencode against the restatement
(oracle/tbl_oracle.c) on seeded texts spanning many tiles, every error
path, and whole-table loads (text, binary, min BFW, size limits, several
blocks) including the synthetic SSB schema loaded from `.tbl` files and
run through a star-join program.
"""
import os

import numpy as np
import pytest

from ahead_b200 import ingest
from ahead_b200.model import BAD_ARG, CAPACITY, SIZE_MISMATCH, UNSUPPORTED
from oracle import tbl_oracle as to

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = os.path.join(ROOT, "tests", "golden", "ingest")

# the AN headers of the reference (headers.tgz:database/headers/*AN_header.csv)
EXPECTED_AN = {
    "lineorderAN": [("orderkey", "RESINT"), ("linenumber", "RESTINY"), ("custkey", "RESINT"), ("partkey", "RESINT"),
                    ("suppkey", "RESINT"), ("orderdate", "RESINT"), ("orderpriority", "STRING:15"),
                    ("shippriority", "CHAR"), ("quantity", "RESTINY"), ("extendedprice", "RESINT"),
                    ("ordertotalprice", "RESINT"), ("discount", "RESTINY"), ("revenue", "RESINT"),
                    ("supplycost", "RESINT"), ("tax", "RESTINY"), ("commitdate", "RESINT"), ("shipmode", "STRING")],
    "partAN": [("partkey", "RESINT"), ("name", "STRING:22"), ("mfgr", "STRING:6"), ("category", "STRING:7"),
               ("brand", "STRING:9"), ("color", "STRING:11"), ("type", "STRING:25"), ("size", "RESTINY"),
               ("container", "STRING:10")],
}
TYPE_WIDTH = {"RESINT": (ingest.RESINT, 8), "RESTINY": (ingest.RESTINY, 2), "RESSHORT": (ingest.RESSHORT, 4),
              "CHAR": (ingest.CHAR, 1), "STRING": (ingest.STRING, 65), "INTEGER": (ingest.INT, 4),
              "TINYINT": (ingest.TINYINT, 1), "SHORTINT": (ingest.SHORTINT, 2)}


def _expected(t):
    if t.startswith("STRING:"):
        return ingest.STRING, int(t[7:]) + 1
    return TYPE_WIDTH[t]


# ------------------------------------------------------------------ CPU
@pytest.mark.parametrize("table", sorted(EXPECTED_AN))
def test_reference_headers(table):
    cols = ingest.read_header(os.path.join(HEADERS, table))
    assert [(n, t, w) for n, t, w in cols] == [(n, *_expected(t)) for n, t in EXPECTED_AN[table]]


def test_every_reference_header_reads():
    for f in sorted(os.listdir(HEADERS)):
        if not f.endswith("_header.csv"):
            continue
        cols = ingest.read_header(os.path.join(HEADERS, f[: -len("_header.csv")]))
        raw = open(os.path.join(HEADERS, f), "rb").read().split(b"\n")
        names = [x for x in raw[0].rstrip(b"\r").split(b"|") if x]
        assert [c[0].encode() for c in cols] == names, f
        if not f[: -len("_header.csv")].endswith("AN"):
            assert all(t < ingest.RESTINY for _, t, _ in cols), f


def test_header_prefix_and_errors(tmp_path):
    p = str(tmp_path / "t")
    with open(p + "_header.csv", "w") as f:
        f.write("a|b||c\r\nINT|STRING:3|LARGEINTEGER\n")
    assert ingest.read_header(p, prefix="x_") == [("x_a", ingest.INT, 4), ("x_b", ingest.STRING, 4),
                                                  ("x_c", ingest.LARGEINT, 8)]
    for bad in ("a|b\nINT|WHAT\n", "a|b\nINT\n", "a\n", "\nINT\n"):
        with open(p + "_header.csv", "w") as f:
            f.write(bad)
        with pytest.raises(ingest.AheadError) as e:
            ingest.read_header(p)
        assert e.value.status == BAD_ARG
    with open(p + "_header.csv", "w") as f:
        f.write("n" * 250 + "\nINT\n")
    with pytest.raises(ingest.AheadError):
        ingest.read_header(p, prefix="p" * 10)
    with pytest.raises(ingest.AheadError):
        ingest.read_header(str(tmp_path / "missing"))


def test_load_and_minbfw_tables():
    for t, a in to.LOAD_A.items():
        assert ingest.load_a(t) == a
    assert ingest.load_a(ingest.INT) == 0
    for t in (ingest.RESTINY, ingest.RESSHORT, ingest.RESINT):
        for bfw in range(0, 9):
            want = to.minbfw_a(t, bfw) if bfw else None
            assert ingest.minbfw_a(t, bfw) == (want or 0), (t, bfw)
    # the load A is the largest entry of each AsBFW table
    for t, tab in to.AS_BFW.items():
        assert tab[-1] == to.LOAD_A[t] or t == ingest.RESINT


def test_oracle_field_conversions():
    """Hand-worked results of the reference's conversions (glibc strtol /
    strtod semantics) through the restatement."""
    text = (b" 12abc|-5|+7|99999999999999999999|x|1.5e3|abcdefg|Zq|300\r\n"
            b"-99999999999999999999||\t-0|+0|  -128|-25|.25|ab|z|-1|extra\n")
    kinds = [to.KIND_INT, to.KIND_INT, to.KIND_INT, to.KIND_INT, to.KIND_RES, to.KIND_FIXED, to.KIND_STRING,
             to.KIND_CHAR, to.KIND_RES]
    widths = [1, 2, 4, 8, 2, 8, 4, 1, 2]
    As = [0, 0, 0, 0, 233, 0, 0, 0, 233]
    rc, lines, bad, cols = to.tbl_parse(text, kinds, widths, As)
    assert rc == 0 and lines == 2
    v = lambda i, dt: list(cols[i].view(dt))
    assert v(0, np.int8) == [12, 0]            # atoi: strtol saturates at LONG_MIN, (int) keeps the low word
    assert v(1, np.int16) == [-5, 0]
    assert v(2, np.int32) == [7, 0]
    assert v(3, np.int64) == [2 ** 63 - 1, -128]
    assert v(4, np.uint16) == [0, (-25 * 233) % 65536]
    assert v(5, np.float64) == [1500.0, 0.25]
    assert cols[6].tobytes() == b"abcdab\0\0"  # strncpy: no terminator when the field fills the width
    assert cols[7].tobytes() == b"Zz"
    assert v(8, np.uint16) == [(300 * 233) % 65536, (-233) % 65536]


def test_oracle_errors_and_limits():
    kinds, widths, As = [to.KIND_INT, to.KIND_INT], [4, 4], [0, 0]
    assert to.tbl_parse(b"1|2|3\n", kinds, widths, As, ignore_more_data=False)[:3] == (BAD_ARG, 1, 0)
    assert to.tbl_parse(b"1|2\n3\n", kinds, widths, As)[:3] == (SIZE_MISMATCH, 2, 1)
    long_ok = b"1|" + b"9" * 1020 + b"\n"
    assert to.tbl_parse(long_ok, kinds, widths, As)[0] == 0
    assert to.tbl_parse(b"1|" + b"9" * 1021 + b"\n", kinds, widths, As)[0] == BAD_ARG
    rc, lines, _, cols = to.tbl_parse(b"1|2\n3|4\n5|6\n", kinds, widths, As, max_lines=2)
    assert rc == 0 and lines == 3 and list(cols[1].view(np.int32)) == [2, 4]


def test_reencode_oracle_round_trip():
    rng = np.random.default_rng(5)
    for w, t in ((2, to.TBL_RESTINY), (4, to.TBL_RESSHORT), (8, to.TBL_RESINT)):
        a0 = to.LOAD_A[t]
        vals = rng.integers(0, 1 << (4 * w), 1000, dtype=np.uint64)
        m = (1 << (8 * w)) - 1
        codes = ((vals * np.uint64(a0)) & np.uint64(m)).astype({2: np.uint16, 4: np.uint32, 8: np.uint64}[w])
        for a1 in to.AS_BFW[t]:
            r = to.reencode(codes, w, a0, a1)
            assert np.array_equal(r.astype(np.uint64), (vals * np.uint64(a1)) & np.uint64(m))
            assert np.array_equal(to.reencode(r, w, a1, a0), codes)


def test_format_tbl_round_trip():
    rng = np.random.default_rng(9)
    n = 3000
    ints = rng.integers(-(2 ** 63), 2 ** 63 - 1, n, dtype=np.int64)
    small = rng.integers(-128, 128, n)
    strs = np.array([bytes(rng.integers(97, 123, int(k)).astype(np.uint8)) for k in rng.integers(1, 12, n)])
    text = ingest.format_tbl([ints, small, strs])
    assert text.count(b"\n") == n
    rc, lines, _, cols = to.tbl_parse(text, [to.KIND_INT, to.KIND_INT, to.KIND_STRING], [8, 1, 12], [0, 0, 0])
    assert rc == 0 and lines == n
    assert np.array_equal(cols[0].view(np.int64), ints)
    assert np.array_equal(cols[1].view(np.int8), small.astype(np.int8))
    assert list(cols[2].view("S12")) == list(strs)


# ------------------------------------------------------------------ seeded texts
ALPHA = np.frombuffer(b"ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789 #-.,/", dtype=np.uint8)


def _rand_int(rng, lo, hi):
    """Uniform in [lo, hi) for Python ints of any size."""
    return lo + int.from_bytes(rng.bytes(16), "little") % (hi - lo)


def _int_field(rng, w, res):
    k = rng.integers(0, 12)
    lim = 1 << (8 * w - 1)
    if k == 0:
        return str(_rand_int(rng, -lim, lim)) + "junk"
    if k == 1:
        return " \t" + str(_rand_int(rng, -lim, lim))
    if k == 2:
        return "+" + str(_rand_int(rng, 0, lim))
    if k == 3:
        return str(rng.choice(["99999999999999999999", "-99999999999999999999", "9223372036854775808",
                               "-9223372036854775808", "-", "abc", "+-3"]))
    if k == 4:
        return str(_rand_int(rng, -4 * lim, 4 * lim))  # outside the width: wraps (saturates at 64 bits)
    return str(_rand_int(rng, 0 if res else -lim, lim))


def _fixed_field(rng):
    """Decimals of at most 15 significant digits and small exponents: values
    strtod and the device's exact fast path both convert."""
    k = rng.integers(0, 6)
    m = int(rng.integers(0, 10 ** int(rng.integers(1, 13))))
    if k == 0:
        return f"{m}.{int(rng.integers(0, 1000)):03d}"
    if k == 1:
        return f"-{m}e{int(rng.integers(-10, 10))}"
    if k == 2:
        return f".{m}"
    if k == 3:
        return f"{m}."
    if k == 4:
        return f" +{m}E-{int(rng.integers(0, 10))}"
    return str(m)


def _string_field(rng, w):
    n = int(rng.integers(1, w + 6))
    return bytes(ALPHA[rng.integers(0, len(ALPHA), n)]).decode()


SPEC = [(to.KIND_INT, 1, 0), (to.KIND_INT, 2, 0), (to.KIND_INT, 4, 0), (to.KIND_INT, 8, 0), (to.KIND_RES, 2, 233),
        (to.KIND_RES, 4, 63877), (to.KIND_RES, 8, 65117), (to.KIND_STRING, 16, 0), (to.KIND_FIXED, 8, 0),
        (to.KIND_CHAR, 1, 0), (to.KIND_STRING, 3, 0)]


def _text(rng, nlines, spec=SPEC, delims="|", extra=0):
    lines = []
    for _ in range(nlines):
        fields = []
        for kind, w, _ in spec:
            if kind in (to.KIND_INT, to.KIND_RES):
                fields.append(_int_field(rng, w, kind == to.KIND_RES))
            elif kind == to.KIND_FIXED:
                fields.append(_fixed_field(rng))
            elif kind == to.KIND_CHAR:
                fields.append(_string_field(rng, 2).strip() or "c")
            else:
                fields.append(_string_field(rng, w).strip() or "s")
        fields += [str(i) for i in range(extra)]
        out = fields[0]
        for f in fields[1:]:
            d = delims[int(rng.integers(0, len(delims)))]
            out += d * int(rng.integers(1, 3)) + f  # doubled delimiters: empty fields vanish (strtok)
        if rng.random() < 0.5:
            out += delims[0]
        if rng.random() < 0.2:
            out = delims[-1] + out
        if rng.random() < 0.3:
            out += "\r"
        lines.append(out)
    return ("\n".join(lines) + "\n").encode()


def test_oracle_reads_seeded_text():
    rng = np.random.default_rng(1)
    text = _text(rng, 500)
    kinds, widths, As = zip(*SPEC)
    rc, lines, _, cols = to.tbl_parse(text, kinds, widths, As)
    assert rc == 0 and lines == 500 and all(len(c) == 500 * w for c, w in zip(cols, widths))


# ------------------------------------------------------------------ GPU
@pytest.fixture(scope="module")
def gpu():
    from ahead_b200.gpu import GpuOps
    g = GpuOps(0)
    yield g
    g.close()


def _dev_text(gpu, text: bytes):
    t = gpu.torch
    return t.frombuffer(bytearray(text), dtype=t.uint8).to("cuda")


def _gpu_parse(gpu, text, spec, cap=None, **kw):
    t = gpu.torch
    kinds, widths, As = zip(*spec)
    rows = text.count(b"\n")
    cap = rows if cap is None else cap
    outs = [t.zeros(max(cap, 1) * w, dtype=t.uint8, device="cuda") if k != to.KIND_SKIP else None
            for k, w, _ in spec]
    row0 = kw.pop("row0", 0)
    lines = ingest.tbl_parse(gpu, _dev_text(gpu, text), kinds, widths, As, outs, row0=row0, cap=cap, **kw)
    return lines, outs


@pytest.mark.gpu
@pytest.mark.parametrize("seed,nlines,delims", [(2, 30_000, "|"), (3, 7_000, "|;"), (4, 1, "|"), (5, 999, ",")])
def test_gpu_parse_matches_oracle(gpu, seed, nlines, delims):
    rng = np.random.default_rng(seed)
    text = _text(rng, nlines, delims=delims, extra=int(seed % 2))
    kinds, widths, As = zip(*SPEC)
    rc, lines, _, ref = to.tbl_parse(text, kinds, widths, As, delim=delims)
    assert rc == 0 and lines == nlines
    glines, outs = _gpu_parse(gpu, text, SPEC, delim=delims)
    assert glines == nlines
    for i, (o, r) in enumerate(zip(outs, ref)):
        assert np.array_equal(o.cpu().numpy(), r), f"column {i} kind {SPEC[i][0]}"


@pytest.mark.gpu
def test_gpu_parse_skip_rows_and_limits(gpu):
    rng = np.random.default_rng(7)
    text = _text(rng, 5000)
    spec = [s if i % 3 else (to.KIND_SKIP, s[1], 0) for i, s in enumerate(SPEC)]
    kinds, widths, As = zip(*spec)
    _, _, _, ref = to.tbl_parse(text, kinds, widths, As, max_lines=1234)
    lines, outs = _gpu_parse(gpu, text, spec, cap=1300, row0=66, max_lines=1234)
    assert lines == 5000
    for (k, w, _), o, r in zip(spec, outs, ref):
        if o is None:
            continue
        o = o.cpu().numpy()
        assert np.array_equal(o[66 * w:(66 + 1234) * w], r)
        assert not o[:66 * w].any() and not o[(66 + 1234) * w:].any()
    with pytest.raises(ingest.AheadError) as e:
        _gpu_parse(gpu, text, spec, cap=1299, row0=66, max_lines=1234)
    assert e.value.status == CAPACITY


@pytest.mark.gpu
def test_gpu_parse_errors(gpu):
    spec = [(to.KIND_INT, 4, 0), (to.KIND_STRING, 1100, 0)]
    ok = b"1|" + b"x" * 1020 + b"\n"
    lines, outs = _gpu_parse(gpu, b"5|a\n" * 3 + ok, spec)
    assert lines == 4 and outs[1].cpu().numpy()[3 * 1100: 3 * 1100 + 1020].tobytes() == b"x" * 1020
    cases = [
        (b"5|a\n" * 9 + b"1|" + b"x" * 1021 + b"\n" + b"5|a\n", BAD_ARG, 9, {}),
        (b"5|a\n" * 20_000 + b"1|2|3\n", BAD_ARG, 20_000, {"ignore_more_data": False}),
        (b"5|a\n5|a\n7\n5|a\n", SIZE_MISMATCH, 2, {}),
        (b"5|a\n|||\n", SIZE_MISMATCH, 1, {}),
        (b"5|a\n5|a", BAD_ARG, 0, {}),  # no trailing newline
    ]
    for text, status, line, kw in cases:
        with pytest.raises(ingest.AheadError) as e:
            _gpu_parse(gpu, text, spec, **kw)
        assert e.value.status == status, text[:20]
        if status != BAD_ARG or line:
            assert e.value.bad_line == line
    fspec = [(to.KIND_FIXED, 8, 0)]
    for bad in (b"1e300", b"inf", b"nan", b"0x10", b"12345678901234567891", b"1e-23"):
        with pytest.raises(ingest.AheadError) as e:
            _gpu_parse(gpu, b"1.5\n" + bad + b"\n", fspec)
        assert e.value.status == UNSUPPORTED and e.value.bad_line == 1, bad
    # exact cases the fast path keeps
    vals = [b"0", b"-0", b"1e22", b"9007199254740992", b"123456789012345.5e-1", b"1.50000000000000000000", b"7e-22"]
    _, outs = _gpu_parse(gpu, b"\n".join(vals) + b"\n", fspec)
    got = outs[0].cpu().numpy().view(np.float64)
    _, _, _, ref = to.tbl_parse(b"\n".join(vals) + b"\n", [to.KIND_FIXED], [8], [0])
    assert got.tobytes() == ref[0].tobytes()


@pytest.mark.gpu
def test_gpu_reencode_matches_oracle(gpu):
    from ahead_b200.model import RESINT, RESSHORT, RESTINY, Col
    t = gpu.torch
    rng = np.random.default_rng(11)
    for ty, tt, w in ((RESTINY, to.TBL_RESTINY, 2), (RESSHORT, to.TBL_RESSHORT, 4), (RESINT, to.TBL_RESINT, 8)):
        for n, off in ((1, 0), (37, 1), (100_003, 3), (3_000_001, 0)):
            dt = {2: np.uint16, 4: np.uint32, 8: np.uint64}[w]
            codes = rng.integers(0, np.iinfo(dt).max, n + off, dtype=dt, endpoint=True)
            buf = t.from_numpy(codes.view(np.uint8).copy()).to("cuda")
            a0 = to.LOAD_A[tt]
            col = Col(ty, buf[off * w:], a0, 0, 0, 0)
            for a1 in to.AS_BFW[tt][1:3]:
                col = ingest.reencode(gpu, col, n, a1)
                want = to.reencode(codes[off:], w, a0, a1)
                got = buf.cpu().numpy().view(dt)
                assert np.array_equal(got[off:], want) and np.array_equal(got[:off], codes[:off]), (w, n, off, a1)
                codes = got.copy()
                a0 = a1
                assert (a1 * col.Ainv) % (1 << (8 * w)) == 1


def _mixed_table(tmp_path, n, seed=3, name="mix"):
    rng = np.random.default_rng(seed)
    names = ["k", "t", "s", "i", "l", "rt", "rs", "ri", "str", "f", "c"]
    types = ["RESINT", "TINYINT", "SHORTINT", "INTEGER", "LARGEINT", "RESTINY", "RESSHORT", "RESINT", "STRING:9",
             "FIXED", "CHAR"]
    cols = [np.arange(1, n + 1), rng.integers(-128, 128, n), rng.integers(-2 ** 15, 2 ** 15, n),
            rng.integers(-2 ** 31, 2 ** 31, n), rng.integers(-2 ** 62, 2 ** 62, n), rng.integers(0, 256, n),
            rng.integers(0, 65536, n), rng.integers(0, 2 ** 32, n),
            np.array([bytes(ALPHA[rng.integers(0, 62, int(k))]) for k in rng.integers(1, 12, n)]),
            np.round(rng.uniform(-1e6, 1e6, n), 2), np.array([bytes([int(x)]) for x in rng.integers(65, 91, n)])]
    path = str(tmp_path / name)
    ingest.write_tbl(path, names, types, cols)
    return path, names, types, cols


def _oracle_table(path, names, types, size=None):
    hdr = ingest.read_header(path)
    text = open(path + ".tbl", "rb").read()
    kinds = [{ingest.STRING: to.KIND_STRING, ingest.FIXED: to.KIND_FIXED, ingest.CHAR: to.KIND_CHAR}.get(
        t, to.KIND_RES if t >= ingest.RESTINY else to.KIND_INT) for _, t, _ in hdr]
    As = [to.LOAD_A.get(t, 0) for _, t, _ in hdr]
    rc, lines, _, cols = to.tbl_parse(text, kinds, [w for _, _, w in hdr], As, max_lines=size)
    assert rc == 0
    return hdr, cols


@pytest.mark.gpu
@pytest.mark.parametrize("n,block_mb", [(20_000, 0), (150_000, 1)])
def test_gpu_table_load_text_then_binary(gpu, tmp_path, n, block_mb):
    path, names, types, _ = _mixed_table(tmp_path, n)
    hdr, ref = _oracle_table(path, names, types)
    t1 = ingest.load(gpu, path, "mix", block_mb=block_mb)
    assert t1.rows == n and t1.names() == names
    assert t1.stats["blocks"] >= (2 if block_mb else 1)
    for c, r in zip(t1.columns, ref):
        assert not c.from_file and c.count == n
        assert np.array_equal(c.data.cpu().numpy(), r), c.name
        assert open(f"{path}_{c.name}.ahead", "rb").read() == r.tobytes()
        if c.tbl_type >= ingest.RESTINY:
            assert c.A == to.LOAD_A[c.tbl_type] and (c.A * c.Ainv) % (1 << (8 * c.width)) == 1
    # second load: every column from its .ahead file, the text is not read
    os.rename(path + ".tbl", path + ".tbl.away")
    t2 = ingest.load(gpu, path, block_mb=block_mb)
    assert t2.rows == n and t2.stats["text_bytes"] == 0
    for c, r in zip(t2.columns, ref):
        assert c.from_file and np.array_equal(c.data.cpu().numpy(), r)
    # min BFW 2: AN columns re-encoded on read
    t3 = ingest.load(gpu, path, min_bfw=2, block_mb=block_mb)
    for c, r in zip(t3.columns, ref):
        if c.tbl_type >= ingest.RESTINY:
            a1 = to.minbfw_a(c.tbl_type, 2)
            assert c.A == a1 and (c.A * c.Ainv) % (1 << (8 * c.width)) == 1
            want = to.reencode(r.view({2: np.uint16, 4: np.uint32, 8: np.uint64}[c.width]), c.width,
                               to.LOAD_A[c.tbl_type], a1)
            assert np.array_equal(c.data.cpu().numpy(), want.view(np.uint8)), c.name
        else:
            assert np.array_equal(c.data.cpu().numpy(), r)
    assert t3.stats["reencoded"] == 4 * n
    # restiny has no A for a weight of 4: the reference throws there
    with pytest.raises(ingest.AheadError) as e:
        ingest.load(gpu, path, min_bfw=4)
    assert e.value.status == UNSUPPORTED
    os.rename(path + ".tbl.away", path + ".tbl")


@pytest.mark.gpu
def test_gpu_table_load_partial_binaries_and_sizes(gpu, tmp_path):
    n = 5000
    path, names, types, _ = _mixed_table(tmp_path, n, seed=4)
    _, ref = _oracle_table(path, names, types)
    ingest.load(gpu, path)  # writes the .ahead files
    ingest.remove_binaries(path, ["s", "str"])
    # two columns parsed from the text, the rest read back; nothing rewritten
    # for the read columns (convert: only the parsed ones are written)
    t = ingest.load(gpu, path)
    assert [c.from_file for c in t.columns] == [nm not in ("s", "str") for nm in names]
    for c, r in zip(t.columns, ref):
        assert np.array_equal(c.data.cpu().numpy(), r)
    # `size` limits only the text: a parsed column of 100 rows against read
    # columns of n rows is the reference's "column sizes don't match"
    ingest.remove_binaries(path, ["s"])
    with pytest.raises(ingest.AheadError) as e:
        ingest.load(gpu, path, size=100)
    assert e.value.status == SIZE_MISMATCH
    # without any binary file `size` keeps the first lines
    ingest.remove_binaries(path, names)
    t = ingest.load(gpu, path, size=100, convert_table_files=False)
    assert t.rows == 100 and not os.path.exists(f"{path}_k.ahead")
    _, ref100 = _oracle_table(path, names, types, size=100)
    for c, r in zip(t.columns, ref100):
        assert np.array_equal(c.data.cpu().numpy(), r)
    # a needed text that is missing
    os.remove(path + ".tbl")
    with pytest.raises(ingest.AheadError) as e:
        ingest.load(gpu, path)
    assert e.value.status == BAD_ARG


@pytest.mark.gpu
def test_gpu_table_load_last_line_and_empty(gpu, tmp_path):
    path = str(tmp_path / "e")
    with open(path + "_header.csv", "w") as f:
        f.write("a|b\nRESINT|STRING:4\n")
    open(path + ".tbl", "wb").close()
    t = ingest.load(gpu, path, convert_table_files=False)
    assert t.rows == 0 and all(c.count == 0 for c in t.columns)
    with open(path + ".tbl", "wb") as f:
        f.write(b"1|ab|\n2|cdefgh")  # no newline after the last line
    t = ingest.load(gpu, path, convert_table_files=False)
    assert t.rows == 2
    assert list(t["a"].host()) == [65117, 2 * 65117]
    assert list(t["b"].host()) == [b"ab", b"cdefg"]  # STRING:4 is 5 bytes wide
    with open(path + ".tbl", "wb") as f:
        f.write(b"1|ab\n2|" + b"c" * 2000 + b"\n")
    with pytest.raises(ingest.AheadError) as e:
        ingest.load(gpu, path, convert_table_files=False)
    assert e.value.status == BAD_ARG


@pytest.mark.gpu
def test_gpu_ssb_schema_from_tbl_files(gpu, tmp_path):
    """The synthetic SSB schema written as `.tbl` files, loaded by the table
    loader, is the generated schema bit for bit, and a star-join program
    over it returns the same result."""
    from ahead_b200.gpu import to_device, to_host
    from ahead_b200.ssb import generate, load_tables, write_tables
    from ahead_b200.ssb_programs import q21, q31
    sizes = dict(fact=40_000, date=2556, customer=300, part=2000, supplier=40)
    s = generate(sizes, seed=2)
    paths = write_tables(s, str(tmp_path))
    ds, loaded = load_tables(gpu, paths, block_mb=1)
    for tab, cols in s.tables.items():
        for c, b in cols.items():
            got = to_host(ds.tables[tab][c])
            assert got.count == b.count and got.tail.type == b.tail.type and got.tail.A == b.tail.A, (tab, c)
            assert np.array_equal(np.asarray(got.tail.data), np.asarray(b.tail.data)), (tab, c)
    dev = type(s)({t: {c: to_device(b) for c, b in cols.items()} for t, cols in s.tables.items()}, s.sizes)
    for prog in (q21, q31):
        a, b = prog(gpu, ds, "continuous"), prog(gpu, dev, "continuous")
        assert a.total == b.total
        for x, y in zip((a.years, a.nations, a.profits), (b.years, b.nations, b.profits)):
            if x is None:
                assert y is None
                continue
            hx, hy = to_host(x), to_host(y)
            assert np.array_equal(np.asarray(hx.tail.data), np.asarray(hy.tail.data))


@pytest.mark.gpu
def test_gpu_table_load_delimiter_and_prefix(gpu, tmp_path):
    """Another delimiter for header and text, and a column-name prefix, which
    also names the `.ahead` files (Transaction.cpp:184-201, 294)."""
    n = 3000
    rng = np.random.default_rng(21)
    path = str(tmp_path / "semi")
    names = ["a", "b", "c"]
    cols = [rng.integers(0, 2 ** 31, n), rng.integers(0, 256, n),
            np.array([bytes(ALPHA[rng.integers(0, 62, int(k))]) for k in rng.integers(1, 9, n)])]
    ingest.write_tbl(path, names, ["RESINT", "TINYINT", "STRING:6"], cols, delim=";")
    t = ingest.load(gpu, path, prefix="lo_", delim=";")
    assert t.names() == ["lo_a", "lo_b", "lo_c"] and t.rows == n
    text = open(path + ".tbl", "rb").read()
    _, _, _, ref = to.tbl_parse(text, [to.KIND_RES, to.KIND_INT, to.KIND_STRING], [8, 1, 7], [65117, 0, 0],
                                delim=";")
    for c, r in zip(t.columns, ref):
        assert np.array_equal(c.data.cpu().numpy(), r), c.name
        assert os.path.exists(f"{path}_{c.name}.ahead")
    # the same files read back under the prefix; without it they are not found
    t2 = ingest.load(gpu, path, prefix="lo_", delim=";")
    assert all(c.from_file for c in t2.columns)
    t3 = ingest.load(gpu, path, delim=";", convert_table_files=False)
    assert not any(c.from_file for c in t3.columns)


def test_ssb_tables_written_as_text_parse_back(tmp_path):
    """ssb.write_tables writes each table's decoded values under an AN header;
    the restatement of the reference's loader reads them back as the
    generator's AN codes (CPU)."""
    from ahead_b200.ssb import generate, write_tables
    s = generate(dict(fact=5_000, date=2556, customer=300, part=2000, supplier=40), seed=3)
    paths = write_tables(s, str(tmp_path))
    for tab, path in paths.items():
        hdr = ingest.read_header(path)
        assert [h[0] for h in hdr] == list(s.tables[tab])
        kinds = [to.KIND_RES] * len(hdr)
        rc, lines, _, cols = to.tbl_parse(open(path + ".tbl", "rb").read(), kinds, [w for _, _, w in hdr],
                                          [to.LOAD_A[t] for _, t, _ in hdr])
        assert rc == 0 and lines == next(iter(s.tables[tab].values())).count
        for (name, _, w), raw in zip(hdr, cols):
            want = np.ascontiguousarray(s.tables[tab][name].tail.data).view(np.uint8)
            assert np.array_equal(raw, want), (tab, name)


# ------------------------------------------------- the reference's own loader
# oracle/_ref/libahead_ref_load.so: TransactionManager::Transaction::load
# (lib/column_storage/Transaction.cpp:66-648) compiled from the reference
# sources, the checker that pins the restatement (CPU) and, through the
# fixtures it wrote (tests/golden/ingest/refbin), the GPU loader.
from oracle import ref_loader  # noqa: E402

REFLOAD = os.path.exists(ref_loader.REFLOAD_LIB)
SPEC_TYPES = ["TINYINT", "SHORTINT", "INTEGER", "LARGEINT", "RESTINY", "RESSHORT", "RESINT", "STRING:15", "FIXED",
              "CHAR", "STRING:2"]


def _write_text_table(tmp_path, name, text, types, delim):
    path = str(tmp_path / name)
    names = [f"c{i}" for i in range(len(types))]
    with open(path + "_header.csv", "w") as f:
        f.write(delim.join(names) + "\n" + delim.join(types) + "\n")
    with open(path + ".tbl", "wb") as f:
        f.write(text)
    return path, names


@pytest.mark.skipif(not REFLOAD, reason="the reference's loader is not built")
@pytest.mark.parametrize("seed,nlines,delims", [(11, 3000, "|"), (12, 2000, "|;"), (13, 500, ";")])
def test_restatement_matches_reference_loader_on_seeded_text(tmp_path, seed, nlines, delims):
    """The restatement's line loop equals the reference's loader, column by
    column and byte for byte, on seeded texts of every column type with
    strtol edge cases (junk suffixes, white space, signs, overflow,
    saturation), strtod decimals, strings longer than their slots, doubled
    and leading delimiters, multi-byte delimiter sets and '\\r' line ends."""
    rng = np.random.default_rng(seed)
    text = _text(rng, nlines, SPEC, delims)
    path, names = _write_text_table(tmp_path, "seeded", text, SPEC_TYPES, delims[0])
    hdr = ingest.read_header(path, delim=delims)
    assert [w for _, _, w in hdr] == [w for _, w, _ in SPEC]
    rows, got = ref_loader.load_table(str(tmp_path), "seeded", hdr, delim=delims)
    kinds, widths, As = zip(*SPEC)
    rc, lines, _, cols = to.tbl_parse(text, kinds, widths, As, delim=delims)
    assert rc == 0 and rows == lines == nlines
    for (name, _, _), col in zip(hdr, cols):
        assert np.array_equal(got[name], col), name


@pytest.mark.skipif(not REFLOAD, reason="the reference's loader is not built")
def test_restatement_matches_reference_loader_binary_minbfw_size(tmp_path):
    """The reference's loader on one table: parsed from the text (writing its
    .ahead files), read back from those files, read with minimum bit-flip
    weight 2 (the AN columns re-encoded to AsBFW[2]), and parsed again with a
    row limit.  Each equals the restatement's parse, its re-encode, or its
    first rows."""
    n = 2000
    path, names, types, _ = _mixed_table(tmp_path, n, name="mix")
    hdr, want = _oracle_table(path, names, types)
    d = str(tmp_path)
    rows, text_cols = ref_loader.load_table(d, "mix", hdr)
    assert rows == n
    assert all(os.path.exists(f"{path}_{c}.ahead") for c in names)
    rows2, file_cols = ref_loader.load_table(d, "mix", hdr)
    rows3, bfw_cols = ref_loader.load_table(d, "mix", hdr, min_bfw=2)
    assert rows2 == rows3 == n
    for (name, t, w), col in zip(hdr, want):
        assert np.array_equal(text_cols[name], col), name
        assert np.array_equal(file_cols[name], col), name
        if t >= to.TBL_RESTINY:
            vals = col.view({2: np.uint16, 4: np.uint32, 8: np.uint64}[w])
            exp = to.reencode(vals, w, to.LOAD_A[t], to.minbfw_a(t, 2)).view(np.uint8)
            assert np.array_equal(bfw_cols[name], exp), name
        else:
            assert np.array_equal(bfw_cols[name], col), name
    ingest.remove_binaries(path, names)
    rows4, part = ref_loader.load_table(d, "mix", hdr, size=700)
    assert rows4 == 700
    for (name, _, w), col in zip(hdr, want):
        assert np.array_equal(part[name], col[: 700 * w]), name


REFBIN = os.path.join(HEADERS, "refbin")


def _refbin_expected():
    z = np.load(os.path.join(REFBIN, "expected.npz"))
    return {k: z[k] for k in z.files}


def test_refbin_fixtures_match_restatement():
    """The reference loader's fixtures (tests/golden/ingest/make_refload.py:
    its parse of mixedAN.tbl, the .ahead files it wrote, and a second load
    of those with minimum bit-flip weight 2) against the restatement: the
    parse, the files' raw bytes, and the re-encode to AsBFW[2]."""
    exp = _refbin_expected()
    path = os.path.join(REFBIN, "mixedAN")
    hdr = ingest.read_header(path)
    kinds = [{ingest.STRING: to.KIND_STRING, ingest.FIXED: to.KIND_FIXED, ingest.CHAR: to.KIND_CHAR}.get(
        t, to.KIND_RES if t >= ingest.RESTINY else to.KIND_INT) for _, t, _ in hdr]
    As = [to.LOAD_A.get(t, 0) for _, t, _ in hdr]
    rc, lines, _, cols = to.tbl_parse(open(path + ".tbl", "rb").read(), kinds, [w for _, _, w in hdr], As)
    assert rc == 0 and lines == 300
    for (name, t, w), col in zip(hdr, cols):
        assert np.array_equal(exp[f"text_{name}"], col), name
        assert open(f"{path}_{name}.ahead", "rb").read() == col.tobytes(), name
        if t >= to.TBL_RESTINY:
            vals = col.view({2: np.uint16, 4: np.uint32, 8: np.uint64}[w])
            col = to.reencode(vals, w, to.LOAD_A[t], to.minbfw_a(t, 2)).view(np.uint8)
        assert np.array_equal(exp[f"bfw2_{name}"], col), name


@pytest.mark.gpu
def test_gpu_table_load_matches_reference_loader_fixtures(gpu, tmp_path):
    """The GPU loader on the reference loader's fixtures: the .ahead files the
    reference wrote read as they are and with minimum bit-flip weight 2, and
    the text parsed once those files are gone, each equal to the columns the
    reference itself loaded."""
    import shutil
    exp = _refbin_expected()
    d = tmp_path / "refbin"
    shutil.copytree(REFBIN, d)
    path = str(d / "mixedAN")
    t1 = ingest.load(gpu, path, "mixedAN")
    assert t1.rows == 300 and all(c.from_file for c in t1.columns)
    for c in t1.columns:
        assert np.array_equal(c.data.cpu().numpy(), exp[f"text_{c.name}"]), c.name
    t2 = ingest.load(gpu, path, "mixedAN", min_bfw=2)
    for c in t2.columns:
        assert np.array_equal(c.data.cpu().numpy(), exp[f"bfw2_{c.name}"]), c.name
    ingest.remove_binaries(path, t1.names())
    t3 = ingest.load(gpu, path, "mixedAN")
    assert not any(c.from_file for c in t3.columns)
    for c in t3.columns:
        assert np.array_equal(c.data.cpu().numpy(), exp[f"text_{c.name}"]), c.name
