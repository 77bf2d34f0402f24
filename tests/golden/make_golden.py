"""Regenerates the golden fixtures in tests/golden/<case>/ by running the reference's own ffbf binary.

For every case in tests/golden/cases.py: build its inputs, compile efficient/ffbf's src/rabin-karp/ffbf.cpp
for its geometry (oracle/Makefile; needs a checkout of the reference named by FFBF_REFERENCE),
run `ffbf pats out < text` in a scratch directory, and store what it wrote:

  meta.json      geometry, input digest, sizes, the reference's stderr timings
  stdout.gz      the candidate lines (processFile's stdout)
  pruned.gz      the pruned pattern file (filterPhrases' `out`)
  index.gz       the __index_out file (pattern line numbers)
  bloom.gz       the __bloom_filter_pats file (main filter, delta-coded set bits)
  ff.gz          the feed-forward bit array, delta-coded like bloom (the reference never saves it; the
                 oracle/ref_harness.cpp shim dumps it at exit)

Run from the repository root: python tests/golden/make_golden.py [case ...]
"""
import gzip
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import oracle  # noqa: E402
from cases import CASES, build_inputs, digest  # noqa: E402


def delta_encode(bits):
    bits = np.asarray(bits, dtype=np.uint64)
    d = np.diff(np.concatenate([[0], bits])).astype("<u4")
    return d.tobytes()


MAX_GZ = 128 * 1024


def write_gz(path, data):
    """Stores `data` gzipped, or, when that exceeds MAX_GZ, only its length and sha256 (<name>.sha256)."""
    import hashlib
    import io
    buf = io.BytesIO()
    with gzip.GzipFile(fileobj=buf, mode="wb", mtime=0, compresslevel=9) as g:
        g.write(data)
    base = path[:-3]
    for old in (path, base + ".sha256"):
        if os.path.exists(old):
            os.unlink(old)
    if buf.tell() > MAX_GZ:
        with open(base + ".sha256", "w") as f:
            f.write(f"{len(data)} {hashlib.sha256(data).hexdigest()}\n")
    else:
        with open(path, "wb") as f:
            f.write(buf.getvalue())


def make(name):
    prm, pats, text = build_inputs(name)
    binary = oracle.ref_binary(prm)
    if binary is None:
        raise SystemExit("reference sources not found; set FFBF_REFERENCE")
    r = oracle.run_reference(binary, pats, text=text.tobytes())
    nb = prm.nbits // 8
    ff = np.frombuffer(r["dump"], dtype=np.uint8)[nb:2 * nb]
    d = os.path.join(HERE, name)
    os.makedirs(d, exist_ok=True)
    write_gz(os.path.join(d, "stdout.gz"), r["stdout"])
    write_gz(os.path.join(d, "pruned.gz"), r["pruned"])
    write_gz(os.path.join(d, "index.gz"), r["index"])
    write_gz(os.path.join(d, "bloom.gz"), r["bloom"])
    write_gz(os.path.join(d, "ff.gz"), delta_encode(oracle.set_bits(ff)))
    meta = dict(case=name, params=dict(len=prm.len, k=prm.k, s=prm.s, cache_bits=prm.cache_bits,
                                       ext_bits=prm.ext_bits),
                input_sha256=digest(pats, text), pattern_bytes=len(pats), text_bytes=int(text.size),
                reference_times=r["times"], generated_by="tests/golden/make_golden.py",
                reference_binary=os.path.basename(binary))
    with open(os.path.join(d, "meta.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    n_ids = r["index"].count(b"\n")
    print(f"{name}: stdout {len(r['stdout'])} B, {n_ids} pruned ids, bloom {len(r['bloom'])} B")


if __name__ == "__main__":
    names = sys.argv[1:] or list(CASES)
    for n in names:
        make(n)
