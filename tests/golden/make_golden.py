"""Regenerate the golden operator fixtures from the reference itself.

Runs every case of tests/cases.py through the reference's own scalar
operators (oracle/_ref/libahead_ref.so, compiled from the reference sources by
`make -C oracle ref`) and stores inputs and outputs in
tests/golden/operators.{npz,json}.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from cases import make_cases, run_case, save_cases  # noqa: E402
from oracle.oracle import Oracle, build_reference  # noqa: E402


def main():
    build_reference()
    ref = Oracle("reference")
    port = Oracle("port")
    cases = make_cases(seed=7, scale=1)
    # encodeAN's scalar definition does not compile in the reference
    # (encdecAN_scalar.tcc:59), so its expected outputs come from the restatement.
    outs = [run_case(port if c["op"] == "encode_an" else ref, c) for c in cases]
    save_cases(os.path.join(ROOT, "tests", "golden", "operators"), cases, outs)
    print(f"wrote {len(cases)} cases")


if __name__ == "__main__":
    main()
