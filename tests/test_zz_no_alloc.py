"""The allocation-free checkAN entry point (ahead_gpu_check_an_noalloc), called
through the C ABI and compared with ahead_gpu_check_an on the same inputs: two
calls in a row on one input, then other inputs and sizes (empty, ragged, the
largest accepted), and the rejection of a column above the scratch limit.
This file is collected last, so it also runs after every other GPU test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_ROWS = 1 << 24


def _column(n, seed, nflips):
    """A device resshort column (u32 codes of v * 63877) with seeded flips."""
    import torch
    from ahead_b200.model import RESSHORT, Bat, Col, an_meta, void_col
    m = an_meta(RESSHORT)
    g = torch.Generator(device="cuda").manual_seed(seed)
    vals = torch.randint(0, 1 << 16, (n,), device="cuda", generator=g, dtype=torch.int64)
    codes = ((vals * m["A"]) & 0xFFFFFFFF).to(torch.int64)
    rng = np.random.default_rng(seed)
    if n and nflips:
        rows = torch.tensor(rng.choice(n, min(nflips, n), replace=False), device="cuda")
        bits = torch.tensor(rng.integers(0, 32, len(rows)), device="cuda")
        codes[rows] ^= torch.bitwise_left_shift(torch.ones_like(bits), bits)
    data = codes.to(torch.int32).view(torch.uint8) if n else torch.empty(0, dtype=torch.uint8, device="cuda")
    return Bat(void_col(0), Col(RESSHORT, data, m["A"], m["Ainv"], m["unenc_max"], 0), n)


def _noalloc(g, b, aoid=16089):
    """ahead_gpu_check_an_noalloc through ctypes; returns (status, error positions)."""
    import torch
    from ahead_b200.gpu import _in_bat
    from ahead_b200.model import CErrVec
    lib = g.lib
    lib.ahead_gpu_check_an_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                               ctypes.c_uint64, ctypes.c_void_p]
    cap = max(b.count, 1)
    buf = torch.empty(cap * 8, dtype=torch.uint8, device="cuda")
    ev = CErrVec()
    ev.data = buf.data_ptr()
    ev.capacity = cap
    cb = _in_bat(b)
    rc = lib.ahead_gpu_check_an_noalloc(g.ctx, ctypes.byref(cb), b.tail.Ainv, b.tail.unenc_max, aoid,
                                        ctypes.byref(ev))
    if rc != 0:
        return rc, None
    assert ev.present == 1
    return rc, buf[: ev.count * 8].cpu().numpy().view(np.uint64)


def _existing(g, b, aoid=16089):
    from ahead_b200.gpu import err_to_host
    e = err_to_host(g.check_an(b, b.tail.Ainv, b.tail.unenc_max, aoid))
    return np.asarray(e.values, dtype=np.uint64)


@pytest.fixture(scope="module")
def gpu():
    from ahead_b200.gpu import GpuOps
    g = GpuOps(0)
    yield g
    g.close()


def test_same_as_check_an_twice_in_a_row(gpu):
    b = _column(3_000_017, seed=1, nflips=500)
    want = _existing(gpu, b)
    assert len(want) > 400
    for _ in range(2):
        rc, got = _noalloc(gpu, b)
        assert rc == 0
        assert np.array_equal(got, want)


def test_other_inputs_and_sizes(gpu):
    for n, seed, flips in ((0, 2, 0), (1, 3, 1), (4097, 4, 30), (1_000_003, 5, 0), (MAX_ROWS, 6, 1000)):
        b = _column(n, seed, flips)
        rc, got = _noalloc(gpu, b, aoid=65117)
        assert rc == 0, n
        assert np.array_equal(got, _existing(gpu, b, aoid=65117)), n


def test_rejects_more_rows_than_the_scratch_holds(gpu):
    from ahead_b200.model import CAPACITY
    b = _column(MAX_ROWS + 1, seed=7, nflips=0)
    rc, _ = _noalloc(gpu, b)
    assert rc == CAPACITY
    assert b"16777216" in gpu.lib.ahead_ctx_last_error(gpu.ctx)


def test_allocates_nothing():
    """The defining property: on a fresh context, calls of the largest
    accepted size leave the context without scratch and the device's free
    memory unchanged (inputs and outputs are allocated before measuring)."""
    import torch
    from ahead_b200.gpu import GpuOps, _in_bat
    from ahead_b200.model import CErrVec
    g = GpuOps(0)
    lib = g.lib
    lib.ahead_ctx_scratch_bytes.argtypes = [ctypes.c_void_p]
    lib.ahead_ctx_scratch_bytes.restype = ctypes.c_uint64
    lib.ahead_gpu_check_an_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                               ctypes.c_uint64, ctypes.c_void_p]
    cr = ctypes.CDLL("libcudart.so.12")
    cr.cudaMemGetInfo.argtypes = [ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]

    def free_bytes():
        f, t = ctypes.c_size_t(), ctypes.c_size_t()
        assert cr.cudaMemGetInfo(ctypes.byref(f), ctypes.byref(t)) == 0
        return f.value

    b = _column(MAX_ROWS, seed=8, nflips=200)
    buf = torch.empty(MAX_ROWS * 8, dtype=torch.uint8, device="cuda")
    cb = _in_bat(b)
    torch.cuda.synchronize()
    assert lib.ahead_ctx_scratch_bytes(g.ctx) == 0
    before = free_bytes()
    counts = []
    for _ in range(3):
        ev = CErrVec()
        ev.data = buf.data_ptr()
        ev.capacity = MAX_ROWS
        assert lib.ahead_gpu_check_an_noalloc(g.ctx, ctypes.byref(cb), b.tail.Ainv, b.tail.unenc_max, 16089,
                                              ctypes.byref(ev)) == 0
        counts.append(ev.count)
    assert free_bytes() == before
    assert lib.ahead_ctx_scratch_bytes(g.ctx) == 0
    assert counts[0] == counts[1] == counts[2] > 0
    g.close()
