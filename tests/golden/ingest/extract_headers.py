"""Extract the reference's SSB header files (headers.tgz:database/headers/*)
into this folder as loader fixtures.  Run where the reference tree exists:

    python tests/golden/ingest/extract_headers.py [/path/to/reference]

The files are the reference's own schema headers (names line, types line,
some with '\\r\\n' line ends); tests read them as committed here.
"""
import os
import sys
import tarfile

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    with tarfile.open(os.path.join(ref, "headers.tgz")) as tf:
        for m in tf.getmembers():
            name = os.path.basename(m.name)
            if not m.isfile() or not name.endswith("_header.csv"):
                continue
            data = tf.extractfile(m).read()
            with open(os.path.join(HERE, name), "wb") as f:
                f.write(data)
            print(name, len(data))


if __name__ == "__main__":
    main()
