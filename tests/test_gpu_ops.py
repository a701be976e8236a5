"""GPU parity tests: every operator of libahead_b200.so against the oracle.

- the golden fixtures (outputs of the reference's own scalar operators);
- fresh seeded cases, larger than the fixtures, against the C restatement;
- a size-independent property check at tens of millions of rows (selected
  count, ascending OIDs, error positions = the flipped rows).
All calls go through the C ABI (ahead_b200.gpu wraps include/ahead_gpu.h).
"""
import numpy as np
import pytest

from bats import flip_bits
from cases import assert_same, load_cases, make_cases, run_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from ahead_b200.gpu import GpuOps
    g = GpuOps(0)
    yield g
    g.close()


def _run_gpu(g, case):
    from ahead_b200.gpu import err_to_host, to_device, to_host
    return run_case(g, case, to_device, to_host, err_to_host)


def test_golden_fixtures(gpu):
    import os
    root = os.path.dirname(os.path.abspath(__file__))
    cases, outs = load_cases(os.path.join(root, "golden", "operators"))
    for i, (c, o) in enumerate(zip(cases, outs)):
        assert_same(_run_gpu(gpu, c), o, f"golden case {i} {c['op']}")


def test_fresh_cases_against_oracle(gpu):
    from oracle.oracle import Oracle
    port = Oracle("port")
    for i, c in enumerate(make_cases(seed=4242, scale=5)):
        assert_same(_run_gpu(gpu, c), run_case(port, c), f"case {i} {c['op']}")


def test_select_large_properties(gpu):
    import torch
    from ahead_b200.gpu import err_to_host, to_host
    from ahead_b200.model import AND, GE, LT, RESSHORT, Bat, Col, void_col
    n, A = 40_000_000, 233
    gen = torch.Generator(device="cuda").manual_seed(5)
    vals = torch.randint(0, 10000, (n,), device="cuda", generator=gen, dtype=torch.int64)
    codes = (vals * A).to(torch.int32)
    rng = np.random.default_rng(6)
    rows = np.sort(rng.choice(n, 50, replace=False))
    bits = rng.integers(0, 32, 50)
    r_t = torch.tensor(rows, device="cuda")
    codes[r_t] ^= torch.tensor([np.int32(np.uint32(1 << int(b)).view(np.int32)) for b in bits], device="cuda")
    b = Bat(void_col(7), Col(RESSHORT, codes.view(torch.uint8), A, pow(A, -1, 1 << 32), 0xFFFF), n)
    out, err = gpu.select_an(b, GE, 1000 * A, LT, 3000 * A, AND)
    c64 = codes.to(torch.int64) & 0xFFFFFFFF
    expect = int(((c64 >= 1000 * A) & (c64 < 3000 * A)).sum())
    assert out.count == expect
    oids = to_host(out).head.data // 65117 - 7
    assert np.all(np.diff(oids.astype(np.int64)) > 0)
    e = err_to_host(err).values
    assert list(e // 16089) == list(rows)  # every single-bit flip is detected, in row order


def _ordered_merge_case(rng, n1, n2, U, umax_key, umax_other, flips):
    """Two strictly increasing key sequences whose other columns (and, with a
    small unenc_max, whose keys) read as corrupt: the merge loop's ordered
    case with error positions."""
    from ahead_b200.model import RESINT, RESOID, Bat, Col, an_meta
    A = 65117
    m = an_meta(RESOID, A)
    k1 = np.sort(rng.choice(U, size=min(n1, U), replace=False)).astype(np.uint64)
    k2 = np.sort(rng.choice(U, size=min(n2, U), replace=False)).astype(np.uint64)
    h1 = rng.integers(0, 1 << 30, len(k1), dtype=np.uint64) * np.uint64(A)
    mi = an_meta(RESINT)
    t2 = (rng.integers(0, 1 << 31, len(k2), dtype=np.uint64) * np.uint64(mi["A"])).astype(np.uint64)
    for arr in (h1, t2):
        flip_bits(arr, min(flips, len(arr)), rng)
    key = lambda k: Col(RESOID, k * np.uint64(A), A, m["Ainv"], umax_key, 0)
    a = Bat(Col(RESOID, h1, A, m["Ainv"], umax_other, 0), key(k1), len(k1))
    b = Bat(key(k2), Col(RESINT, t2, mi["A"], mi["Ainv"], mi["unenc_max"], 0), len(k2))
    return a, b


def test_ordered_merge_with_corrupt_values(gpu):
    """matchjoinAN on ordered inputs whose values read as corrupt (as the
    re-encoded OID heads of hashjoinAN do, whose unenc_max is 0) runs the
    parallel merge; its output and all four error vectors equal the
    reference loop's."""
    from ahead_b200.gpu import err_to_host, to_device, to_host
    from oracle.oracle import Oracle
    port = Oracle("port")
    rng = np.random.default_rng(77)
    shapes = [(0, 5, 10), (5, 0, 10), (1, 1, 3), (3, 7, 10), (50, 40, 60), (300, 900, 1000), (900, 300, 1000),
              (2000, 2000, 100000), (4000, 50, 4100), (50, 4000, 4100), (20000, 30000, 40000)]
    for trial, (n1, n2, U) in enumerate(shapes * 3):
        umax_key = [0x00FFFFFFFFFFFFFF, 0, 5000][trial % 3]
        umax_other = [0, 0x00FFFFFFFFFFFFFF, 1 << 29][(trial // 3) % 3]
        a, b = _ordered_merge_case(rng, n1, n2, U, umax_key, umax_other, flips=trial % 4)
        exp, eerr = port.matchjoin_an(a, b)
        got, gerr = gpu.matchjoin_an(to_device(a), to_device(b))
        got = to_host(got)
        assert got.count == exp.count, trial
        assert np.array_equal(got.head.data, exp.head.data) and np.array_equal(got.tail.data, exp.tail.data), trial
        for k in range(4):
            ge, ee = err_to_host(gerr[k]), eerr[k]
            assert ge.present == ee.present, (trial, k)
            if ee.present:
                assert np.array_equal(np.asarray(ge.values), np.asarray(ee.values)), (trial, k)


def test_compaction_shapes_against_oracle(gpu):
    """selectAN and select (the compaction's row-offset form) and checkAN /
    checkAndDecodeAN (the rare-error passes, with the compaction past 4,096
    corrupt codes) on whole tiles only, one row past a tile, each code width,
    and columns with 4,096 and 5,000 corrupt codes."""
    from bats import random_encoded
    from ahead_b200.model import AND, GE, LE, LT, RESINT, RESSHORT, RESTINY, OR, GT, Bat, Col, void_col
    from oracle.oracle import Oracle
    port = Oracle("port")
    rng = np.random.default_rng(77)
    cases = []
    add = lambda op, *args: cases.append(dict(op=op, args=list(args), kwargs={}))
    for t, n, flips in ((RESSHORT, 3 * 4096, 40), (RESSHORT, 3 * 4096 + 1, 40), (RESTINY, 50_001, 300),
                        (RESINT, 50_003, 300), (RESSHORT, 20_000, 5000), (RESINT, 4096, 4096)):
        b, _, _ = random_encoded(t, n, 0, 200, rng, nflips=flips, seqbase=int(rng.integers(0, 99)))
        A = b.tail.A
        add("select_an", b, GE, 20 * A, LT, 150 * A, AND)
        add("select_an", b, LT, 3 * A, GT, 190 * A, OR)
        add("check_and_decode_an", b)
        add("check_an", b, b.tail.Ainv, b.tail.unenc_max)
        add("select", Bat(void_col(3), Col(RESINT, b.tail.data.astype(np.uint64)), n), LE, 100 * A)
    for i, c in enumerate(cases):
        assert_same(_run_gpu(gpu, c), run_case(port, c), f"case {i} {c['op']} n={c['args'][0].count}")


def test_check_and_decode_large_properties(gpu):
    """checkAndDecodeAN over 40M u32 codes with 50 single-bit flips: every
    clean row's decoded value in row order (compared on the device), the
    flipped rows in the error vector."""
    import torch
    from ahead_b200.gpu import err_to_host
    from ahead_b200.model import RESSHORT, Bat, Col, void_col
    n, A = 40_000_000, 233
    Ai = pow(A, -1, 1 << 32)
    gen = torch.Generator(device="cuda").manual_seed(9)
    vals = torch.randint(0, 60000, (n,), device="cuda", generator=gen, dtype=torch.int64)
    codes = (vals * A).to(torch.int32)
    rng = np.random.default_rng(10)
    rows = np.sort(rng.choice(n, 50, replace=False))
    bits = rng.integers(16, 32, 50)  # a flip in the high half always leaves the 16-bit range
    r_t = torch.tensor(rows, device="cuda")
    codes[r_t] ^= torch.tensor([np.int32(np.uint32(1 << int(b)).view(np.int32)) for b in bits], device="cuda")
    b = Bat(void_col(0), Col(RESSHORT, codes.view(torch.uint8), A, Ai, 0xFFFF), n)
    out, _, et = gpu.check_and_decode_an(b)
    assert out.count == n - 50
    keep = torch.ones(n, dtype=torch.bool, device="cuda")
    keep[r_t] = False
    got = out.tail.data.view(torch.int16)[: out.count].to(torch.int64) & 0xFFFF
    assert torch.equal(got, vals[keep])
    assert list(err_to_host(et).values // 16089) == list(rows)
