"""GPU parity tests: every operator of libahead_b200.so against the oracle.

- the golden fixtures (outputs of the reference's own scalar operators);
- fresh seeded cases, larger than the fixtures, against the C restatement;
- a size-independent property check at tens of millions of rows (selected
  count, ascending OIDs, error positions = the flipped rows).
All calls go through the C ABI (ahead_b200.gpu wraps include/ahead_gpu.h).
"""
import numpy as np
import pytest

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
