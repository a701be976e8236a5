"""The C ABI from C++ host code: tests/cpp/select_sum.cpp composes selectAN,
matchjoinAN, checkAndDecodeAN and the sum the way the reference's programs
do, through include/ahead_gpu.h only.  CPU: it compiles against the headers
and links against the library.  GPU: its results (counts, the AN-coded sum
and every error vector) equal the oracle's composition on the same column."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "select_sum.cpp")
LIBDIR = os.path.join(ROOT, "ahead_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(out):
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(CUDA, "include"),
                    SRC, "-L" + LIBDIR, "-lahead_b200", "-L" + os.path.join(CUDA, "lib64"), "-lcudart",
                    "-Wl,-rpath," + LIBDIR, "-o", out], check=True)


def test_cpp_host_program_builds(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libahead_b200.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(LIBDIR, "csrc")], check=True)
    exe = str(tmp_path / "select_sum")
    _build(exe)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_cpp_host_program_matches_oracle(tmp_path):
    from ahead_b200.model import RESSHORT, host_bat
    from ahead_b200.pipelines import select_sum_an
    from oracle.oracle import Oracle
    rng = np.random.default_rng(3)
    n = 1_000_000
    v = rng.integers(0, 10_000, n, dtype=np.uint64)
    codes = (v * np.uint64(233)).astype(np.uint32)
    rows = rng.choice(n, size=10, replace=False)
    for r, bit in zip(rows, rng.integers(0, 32, 10)):
        codes[r] ^= np.uint32(1 << int(bit))
    path = str(tmp_path / "codes.u32")
    codes.tofile(path)
    exe = str(tmp_path / "select_sum")
    _build(exe)
    out = subprocess.run([exe, path, "233", "1000", "3000"], capture_output=True, text=True, check=True).stdout
    got = {}
    for line in out.strip().splitlines():
        k, *vals = line.split()
        got[k] = [int(x) for x in vals]
    exp = select_sum_an(Oracle("port"), host_bat(RESSHORT, codes, A=233), 1000, 3000)

    def ev(e):
        return [int(e.present)] + ([int(x) for x in e.values] if e.present and e.values is not None else [])
    assert got["selected"] == [exp.oids.count]
    assert got["total"] == [int(exp.total)]
    assert got["select_errors"] == ev(exp.select_errors) and len(got["select_errors"]) == 11
    for i, e in enumerate(exp.fetch_errors):
        assert got[f"fetch_errors{i}"] == ev(e), i
    for i, e in enumerate(exp.decode_errors):
        assert got[f"decode_errors{i}"] == ev(e), i
    assert got["launches"][0] > 0
