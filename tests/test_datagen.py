"""The seeded workload generator: deterministic, thread-count independent, with the stated shapes."""
import numpy as np

from ffbf_b200 import datagen as dg


def test_text_independent_of_thread_count():
    a = dg.gen_text(5, dg.ZIPF_WORDS, 5 << 20, 100, threads=1)
    b = dg.gen_text(5, dg.ZIPF_WORDS, 5 << 20, 100, threads=7)
    assert np.array_equal(a, b)


def test_shapes():
    t = dg.gen_text(1, dg.PRINTABLE, 4 << 20, 80)
    nl = np.count_nonzero(t == 10)
    assert abs(nl / t.size - 1 / 80) < 0.001
    body = t[t != 10]
    assert body.min() >= 0x20 and body.max() <= 0x7E
    z = dg.gen_text(1, dg.ZIPF_WORDS, 4 << 20, 100)
    counts = np.bincount(z, minlength=256)
    assert counts[ord("a")] > counts[ord("b")] > counts[ord("z")] > 0
    assert abs(counts[32] / z.size - (1 / 7) * 0.99) < 0.003
    p = dg.gen_patterns(3, dg.BINARY, 1000, 16, 16)
    assert p.size == 17 * 1000 and np.count_nonzero(p == 10) == 1000


def test_plant_copies_patterns():
    pats = dg.gen_patterns(2, dg.PRINTABLE, 100, 20, 40)
    t = dg.gen_text(2, dg.PRINTABLE, 1 << 20, 80)
    offs, ids = dg.plant(2, pats, t, 10)
    lines = pats.tobytes().split(b"\n")
    last = offs.size - 1
    assert bytes(t[offs[last]:offs[last] + len(lines[ids[last]])]) == lines[ids[last]]
