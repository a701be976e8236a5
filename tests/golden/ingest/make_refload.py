"""Writes tests/golden/ingest/refbin: a small table loaded by the reference's
own loader (oracle/ref_loader.py over lib/column_storage/Transaction.cpp,
compiled here by ``make -C oracle refload``), so the GPU loader is checked
against it on the box where the reference is absent:

  mixedAN_header.csv, mixedAN.tbl   the input: 300 seeded rows of every column
                                    type, AN columns at their load A;
  mixedAN_<column>.ahead            the column files the reference wrote while
                                    it parsed the text (its binary format);
  expected.npz                      the reference's loaded columns as raw bytes:
                                    text_<column> from that parse, bfw2_<column>
                                    from a second load of the files with minimum
                                    bit-flip weight 2.

Run from the repository root:  python tests/golden/ingest/make_refload.py
"""
import os
import shutil
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
sys.path.insert(0, ROOT)

from ahead_b200 import ingest  # noqa: E402
from oracle import ref_loader  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "refbin")
TABLE = "mixedAN"
NAMES = ["key", "tiny", "short", "int", "large", "rtiny", "rshort", "rint", "name", "price", "flag"]
TYPES = ["RESINT", "TINYINT", "SHORTINT", "INTEGER", "LARGEINT", "RESTINY", "RESSHORT", "RESINT", "STRING:9",
         "FIXED", "CHAR"]


def main():
    if ref_loader.build_refload() is None:
        sys.exit("the reference's loader cannot be built here")
    rng = np.random.default_rng(2024)
    n = 300
    alpha = np.frombuffer(b"ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789", dtype=np.uint8)
    cols = [np.arange(1, n + 1), rng.integers(-128, 128, n), rng.integers(-2 ** 15, 2 ** 15, n),
            rng.integers(-2 ** 31, 2 ** 31, n), rng.integers(-2 ** 62, 2 ** 62, n), rng.integers(0, 256, n),
            rng.integers(0, 65536, n), rng.integers(0, 2 ** 32, n),
            np.array([bytes(alpha[rng.integers(0, len(alpha), int(k))]) for k in rng.integers(1, 13, n)]),
            np.round(rng.uniform(-1e5, 1e5, n), 2), np.array([bytes([int(x)]) for x in rng.integers(65, 91, n)])]
    if os.path.isdir(OUT):
        shutil.rmtree(OUT)
    os.makedirs(OUT)
    path = os.path.join(OUT, TABLE)
    ingest.write_tbl(path, NAMES, TYPES, cols)
    hdr = ingest.read_header(path)
    rows, text = ref_loader.load_table(OUT, TABLE, hdr)  # parses the text, writes the .ahead files
    rows2, bfw2 = ref_loader.load_table(OUT, TABLE, hdr, min_bfw=2)  # reads the files, re-encodes
    assert rows == rows2 == n
    np.savez_compressed(os.path.join(OUT, "expected.npz"),
                        **{f"text_{k}": v for k, v in text.items()}, **{f"bfw2_{k}": v for k, v in bfw2.items()})
    print("wrote", sorted(os.listdir(OUT)))


if __name__ == "__main__":
    main()
