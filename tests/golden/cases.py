"""Parity cases: how each golden case's inputs are made (seeded generator or explicit bytes) and with which
filter geometry. tests/golden/make_golden.py runs the reference binary on them and stores its outputs here;
the tests rebuild the inputs from this file, check their digest, and compare against the stored outputs.

Edge cases follow the reference's input handling (src/rabin-karp/ffbf.cpp): empty text, no trailing
newline, NUL bytes (C-string output), bytes >= 0x80 (hashed as 0), lines shorter than LEN, lines crossing
512 KiB read() chunks (carry buffer), empty and short pattern lines, a pattern file without a final newline,
duplicate patterns, and dense geometries that make false positives common.
"""
import hashlib

import numpy as np

from ffbf_b200 import datagen as dg
from ffbf_b200.lib import Params


def _gen(seed, kind, n_pat, lo, hi, text_bytes, nl_mean, n_plant):
    pats = dg.gen_patterns(seed, kind, n_pat, lo, hi)
    text = dg.gen_text(seed, kind, text_bytes, nl_mean)
    dg.plant(seed, pats, text, n_plant)
    return pats.tobytes(), text


def _edge_mixed():
    # printable patterns plus handcrafted oddities; text built from planted lines
    rng_pats, _ = _gen(11, dg.PRINTABLE, 300, 20, 40, 1, 80, 0)
    plist = rng_pats.split(b"\n")[:-1]
    extra = [b"", b"short", b"\x00" * 25 + b"nulpattern", b"\xc3\xa9" * 12 + b"highbytes", plist[3], plist[3],
             b"tab\tseparated\tpattern\there", b"trailing-cr-pattern-0123\r"]
    pats = b"\n".join(plist[:150] + extra + plist[150:]) + b"\n"
    lines = []
    for i, p in enumerate(plist[:60]):
        lines.append(b"prefix " + p + b" suffix")
    lines.append(b"x" * 19)  # shorter than LEN
    lines.append(b"")
    lines.append(b"emb\x00edded " + plist[5] + b" nul")  # NUL before the hit: C-string output cut
    lines.append(b"high \x80\x81\xfe\xff bytes " + plist[6])
    lines.append(b"\xc3\xa9" * 12 + b"highbytes here")
    lines.append(b"\x00" * 25 + b"nulpattern end")
    text = b"\n".join(lines) + b"\nlast line without newline " + plist[7]
    return pats, np.frombuffer(text, dtype=np.uint8).copy()


def _edge_chunks():
    # long lines straddling 512 KiB read() chunks: 2-chunk and 3-chunk lines, hits in every part,
    # and a final unterminated line that spans two chunks
    pats, _ = _gen(12, dg.PRINTABLE, 200, 20, 30, 1, 80, 0)
    plist = pats.split(b"\n")[:-1]
    body = dg.gen_text(13, dg.PRINTABLE, 2_600_000, 0).tobytes()
    C = 512 * 1024
    t = bytearray(body)
    for pos in [100, 2000, C - 40, C - 5, C + 10]:
        t[pos:pos + len(plist[pos % 50])] = plist[pos % 50]
    t[C - 1000] = 10                          # line 0 ends before chunk 1
    t[C + 500] = 10                           # line [C-999, C+500) crosses chunk 0/1
    t[C + 600:C + 600 + len(plist[1])] = plist[1]
    t[3 * C + 100] = 10                       # line [C+501, 3C+100) spans chunks 1, 2, 3
    t[2 * C + 7:2 * C + 7 + len(plist[2])] = plist[2]
    t[3 * C + 50:3 * C + 50 + len(plist[4])] = plist[4]
    t[4 * C + 10] = 10                        # ends a line in chunk 4
    t[4 * C + 300:4 * C + 300 + len(plist[9])] = plist[9]   # final line: (4C+10, end) spans chunks 4 and 5
    t[-100:-100 + len(plist[8])] = plist[8]
    return pats, np.frombuffer(bytes(t), dtype=np.uint8).copy()


def _edge_nul_chunk():
    # NUL bytes in the carried part and in the chunk part of a line crossing a chunk boundary
    pats, _ = _gen(14, dg.PRINTABLE, 100, 20, 24, 1, 80, 0)
    plist = pats.split(b"\n")[:-1]
    C = 512 * 1024
    t = bytearray(dg.gen_text(15, dg.PRINTABLE, C + 4096, 60).tobytes())
    t[C - 300] = 10
    t[C - 250] = 0
    t[C - 200:C - 200 + len(plist[0])] = plist[0]
    t[C + 30] = 0
    t[C + 100] = 10
    return pats, np.frombuffer(bytes(t), dtype=np.uint8).copy()


def _empty_text():
    pats, _ = _gen(16, dg.PRINTABLE, 50, 20, 30, 1, 80, 0)
    return pats, np.zeros(0, dtype=np.uint8)


def _pats_no_trailing_newline():
    pats, text = _gen(17, dg.PRINTABLE, 400, 20, 30, 300_000, 70, 60)
    return pats[:-1], text


CASES = {
    # name: (geometry, input builder)
    "plain_small": (Params(20, 5, 2, 1 << 24, 1 << 28),
                    lambda: _gen(7, dg.PRINTABLE, 2000, 20, 40, 3 << 20, 80, 100)),
    "scale_small": (Params(32, 5, 2, 1 << 23, 1 << 26),
                    lambda: _gen(8, dg.ZIPF_WORDS, 20000, 32, 64, 4 << 20, 100, 400)),
    "binary_small": (Params(16, 5, 2, 1 << 24, 1 << 28),
                     lambda: _gen(9, dg.BINARY, 20000, 16, 16, 2 << 20, 0, 300)),
    "dense_fp": (Params(20, 5, 2, 1 << 12, 1 << 14),
                 lambda: _gen(10, dg.PRINTABLE, 3000, 20, 40, 1 << 20, 80, 50)),
    "smem_cache": (Params(24, 5, 2, 1 << 20, 1 << 24),
                   lambda: _gen(18, dg.PRINTABLE, 20000, 24, 48, 2 << 20, 90, 200)),
    "k11_s0_len63": (Params(63, 11, 0, 1 << 16, 1 << 18),
                     lambda: _gen(19, dg.PRINTABLE, 800, 63, 90, 1 << 20, 300, 80)),
    "k3_s3_len1": (Params(1, 3, 3, 1 << 10, 1 << 12),
                   lambda: _gen(20, dg.PRINTABLE, 30, 1, 4, 200_000, 40, 10)),
    "len19_default": (Params(19, 5, 2, 1 << 24, 1 << 28),
                      lambda: _gen(21, dg.ZIPF_WORDS, 5000, 19, 40, 1 << 20, 60, 100)),
    "hit_flood": (Params(4, 2, 1, 1 << 10, 1 << 10),
                  lambda: _gen(22, dg.PRINTABLE, 2000, 4, 8, 300_000, 50, 10)),
    "edge_mixed": (Params(20, 5, 2, 1 << 24, 1 << 28), _edge_mixed),
    "edge_chunks": (Params(20, 5, 2, 1 << 20, 1 << 22), _edge_chunks),
    "edge_nul_chunk": (Params(20, 5, 2, 1 << 24, 1 << 28), _edge_nul_chunk),
    "empty_text": (Params(20, 5, 2, 1 << 24, 1 << 28), _empty_text),
    "pats_no_newline": (Params(20, 5, 2, 1 << 24, 1 << 28), _pats_no_trailing_newline),
}


def build_inputs(name):
    prm, fn = CASES[name]
    pats, text = fn()
    return prm, pats, np.ascontiguousarray(text, dtype=np.uint8)


def digest(pats, text):
    h = hashlib.sha256()
    h.update(len(pats).to_bytes(8, "little"))
    h.update(pats)
    h.update(np.ascontiguousarray(text, dtype=np.uint8).tobytes())
    return h.hexdigest()
