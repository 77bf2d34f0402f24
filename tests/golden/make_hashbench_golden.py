"""Regenerates tests/golden/hashbench/ by running the reference's own hash benchmark.

efficient/ffbf's src/hashes/hashbench.cc, compiled for the scan's hash (oracle/Makefile target
`hashbench`, which needs a checkout of the reference named by FFBF_REFERENCE), is run as
`hashbench -l input.bin` on a seeded input built here, and its stdout is stored:

  input.bin.gz   the input: printable lines of random lengths, and the edges of hashbench's fgets loop --
                 lines of 4093, 4094 and 10000 bytes (fgets returns at most 4094 bytes per call), NUL bytes
                 at a line's start and middle (the loop stops there), bytes >= 0x80 (hashed raw), '\\r',
                 empty lines and a last line without '\\n'
  lines.out.gz   what `hashbench -l` printed
  meta.json      sizes and digests

Run from the repository root: python tests/golden/make_hashbench_golden.py
"""
import gzip
import hashlib
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "hashbench")


def build_input(seed=77):
    rng = np.random.default_rng(seed)
    parts = []
    for _ in range(500):
        n = int(rng.integers(0, 200))
        parts.append(rng.integers(0x20, 0x7F, n, dtype=np.uint8).tobytes() + b"\n")
    parts.insert(100, b"a" * 4093 + b"\n")
    parts.insert(200, b"b" * 4094 + b"\n")
    parts.insert(300, bytes(rng.integers(0x20, 0x7F, 10000, dtype=np.uint8)) + b"\n")
    parts.insert(400, b"\x00starts with NUL\n")
    parts.insert(500, b"middle\x00NUL then more\n")
    parts.insert(450, bytes(rng.integers(0, 256, 300, dtype=np.uint8)).replace(b"\n", b"x") + b"\n")
    parts.insert(470, b"carriage\r return\r\n")
    parts.insert(490, b"\n\n\n")
    parts.append(b"last line without newline")
    return b"".join(parts)


def main():
    ref = os.environ.get("FFBF_REFERENCE")
    if not ref:
        raise SystemExit("set FFBF_REFERENCE to a checkout of efficient/ffbf")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "hashbench", f"REF={ref}"], check=True)
    binary = os.path.join(ROOT, "oracle", "_ref", "hashbench")
    data = build_input()
    os.makedirs(OUT, exist_ok=True)
    path = os.path.join(OUT, "input.bin")
    with open(path, "wb") as f:
        f.write(data)
    out = subprocess.run([binary, "-l", path], capture_output=True, check=True).stdout
    os.unlink(path)
    with gzip.open(os.path.join(OUT, "input.bin.gz"), "wb") as f:
        f.write(data)
    with gzip.open(os.path.join(OUT, "lines.out.gz"), "wb") as f:
        f.write(out)
    meta = {"input_bytes": len(data), "input_sha256": hashlib.sha256(data).hexdigest(), "output_bytes": len(out),
            "output_sha256": hashlib.sha256(out).hexdigest(), "command": "hashbench -l input.bin",
            "hashfn": "hash_rot_sbox_pre_2<19>"}
    with open(os.path.join(OUT, "meta.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print(f"hashbench golden: {len(data)} input bytes, {len(out)} output bytes")


if __name__ == "__main__":
    sys.exit(main())
