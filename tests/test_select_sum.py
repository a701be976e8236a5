"""The single-column select + sum path (a 6,000,000-row u16 column, values
uniform in [0, 10000), AN-coded with A = 233 into u32; select [1000, 3000)
on codes, fetch, checkAndDecode, AN-coded u64 sum; 10 seeded single-bit
flips): the restatement against the compiled reference on the CPU, and the
GPU operators against the restatement."""
import os

import numpy as np
import pytest

from ahead_b200.model import RESSHORT, host_bat
from ahead_b200.pipelines import select_sum_an
from oracle.oracle import REF_LIB, Oracle

N = 6_000_000


def _column(n=N, seed=1, nflips=10):
    rng = np.random.default_rng(seed)
    v = rng.integers(0, 10_000, n, dtype=np.uint64)
    codes = (v * np.uint64(233)).astype(np.uint32)
    frng = np.random.default_rng(seed + 1)
    rows = frng.choice(n, size=nflips, replace=False)
    bits = frng.integers(0, 32, nflips)
    for r, b in zip(rows, bits):
        codes[r] ^= np.uint32(1 << int(b))
    return host_bat(RESSHORT, codes, A=233), v, np.sort(rows)


def _outcome(r, to_host=None, err_host=None):
    h = (lambda b: to_host(b)) if to_host else (lambda b: b)
    e = (lambda x: err_host(x)) if err_host else (lambda x: x)
    oids = h(r.oids)
    errs = [e(r.select_errors)] + [e(x) for x in r.fetch_errors] + [e(x) for x in r.decode_errors]
    return (r.total, np.asarray(oids.head.data)[: oids.count].astype(np.uint64).tobytes(),
            tuple(None if not x.present else np.asarray(x.values, np.uint64).tobytes() for x in errs))


def test_select_sum_decodes_to_plain_sum():
    col, v, flipped = _column(200_000, seed=3)
    r = select_sum_an(Oracle("port"), col, 1000, 3000)
    clean = np.ones(len(v), bool)
    clean[flipped] = False
    want = int(v[clean & (v >= 1000) & (v < 3000)].sum())
    assert (r.total * pow(65117, -1, 1 << 64)) % (1 << 64) == want
    # every flip in the column is detected by the select (it checks every row)
    assert sorted(int(x) // 16089 for x in r.select_errors.values) == sorted(int(x) for x in flipped)


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference oracle not built")
def test_select_sum_restatement_matches_reference():
    col, _, _ = _column()
    assert _outcome(select_sum_an(Oracle("port"), col, 1000, 3000)) == \
        _outcome(select_sum_an(Oracle("reference"), col, 1000, 3000))


@pytest.mark.gpu
def test_gpu_select_sum_matches_oracle():
    from ahead_b200.gpu import GpuOps, err_to_host, to_device, to_host
    g = GpuOps(0)
    for seed in (1, 2):
        col, _, _ = _column(seed=seed)
        want = _outcome(select_sum_an(Oracle("port"), col, 1000, 3000))
        got = _outcome(select_sum_an(g, to_device(col), 1000, 3000), to_host, err_to_host)
        assert got == want
    g.close()
