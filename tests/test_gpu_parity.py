"""Parity of the CUDA path (through the C ABI) with the reference binary's outputs and the oracle.

Each golden case runs: filter build on the device -> __bloom_filter_ image; scan -> stdout bytes, hit
offsets, line spans, feed-forward bit array; prune -> pruned file + __index_ file; verification -> exact
(offset, pattern id) pairs. All comparisons are bit-exact.
"""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from cases import CASES, build_inputs
from conftest import ROOT, Golden
from ffbf_b200 import FFBFError, Filter, Params

pytestmark = pytest.mark.gpu


def delta(bits):
    return np.diff(np.concatenate([[0], np.asarray(bits, dtype=np.uint64)])).astype("<u4").tobytes()


@pytest.fixture(scope="module", autouse=True)
def require_gpu():
    import torch
    assert torch.cuda.is_available(), "the gpu tests need a CUDA device"


def run_oracle(prm, pats, text):
    o = oracle.Oracle.from_params(prm)
    o.build(pats)
    s = o.scan(text)
    pr = o.prune(pats)
    off, pid = o.verify(pats, pr["ids"], text, s["hits"])
    return o, s, pr, off, pid


@pytest.mark.parametrize("name", list(CASES))
def test_parity_with_reference_and_oracle(name):
    g = Golden(name)
    prm, pats, text = build_inputs(name)
    o, s, pr, ooff, opid = run_oracle(prm, pats, text)
    with Filter(prm) as f:
        f.add_patterns(pats)
        assert g.matches("bloom", f.save_filter())
        r = f.process(text)
        np.testing.assert_array_equal(r.hit_offsets, s["hits"])
        np.testing.assert_array_equal(r.line_start, s["line_start"])
        np.testing.assert_array_equal(r.line_end, s["line_end"])
        assert g.matches("stdout", f.format_lines(text))
        main, ff = f.get_filters()
        assert np.array_equal(main, o.main)
        assert np.array_equal(ff, o.ff)
        assert g.matches("ff", delta(oracle.set_bits(ff)))
        ids = f.filter_phrases()
        np.testing.assert_array_equal(ids, pr["ids"])
        out, idx = f.format_pruned()
        assert g.matches("pruned", out) and g.matches("index", idx)
        off, pid = f.verify()
        np.testing.assert_array_equal(off, ooff)
        np.testing.assert_array_equal(pid, opid)


@pytest.mark.parametrize("name", ["plain_small", "scale_small", "edge_mixed"])
def test_loaded_filter_gives_same_results(name):
    """The CLI's cached-filter path: patterns set without building, main filter from the bloom file."""
    g = Golden(name)
    prm, pats, text = build_inputs(name)
    o, s, pr, _, _ = run_oracle(prm, pats, text)
    with Filter(prm) as f:
        f.set_patterns(pats)
        f.load_filter(o.save_filter())
        r = f.process(text)
        np.testing.assert_array_equal(r.hit_offsets, s["hits"])
        assert g.matches("stdout", f.format_lines(text))
        np.testing.assert_array_equal(f.filter_phrases(), pr["ids"])


def test_device_resident_text_matches_host_text():
    import torch
    prm, pats, text = build_inputs("scale_small")
    with Filter(prm) as f:
        f.add_patterns(pats)
        host = f.process(text)
        f.clear_ff()
        dt = torch.from_numpy(text).cuda()
        f.process_device(dt.data_ptr(), text.size)
        dev = f.collect()
        np.testing.assert_array_equal(host.hit_offsets, dev.hit_offsets)
        np.testing.assert_array_equal(host.line_start, dev.line_start)


def test_feed_forward_accumulates_over_scans():
    prm, pats, text = build_inputs("plain_small")
    o, s, pr, _, _ = run_oracle(prm, pats, text)
    cut = int(np.flatnonzero(text[: text.size // 2] == 10)[-1]) + 1
    with Filter(prm) as f:
        f.add_patterns(pats)
        a = f.process(text[:cut])
        b = f.process(text[cut:])
        hits = np.concatenate([a.hit_offsets, b.hit_offsets + cut])
        np.testing.assert_array_equal(hits, s["hits"])
        np.testing.assert_array_equal(f.get_filters()[1], o.ff)
        np.testing.assert_array_equal(f.filter_phrases(), pr["ids"])


def test_hit_buffer_regrows():
    prm, pats, text = build_inputs("hit_flood")
    o, s, _, _, _ = run_oracle(prm, pats, text)
    assert s["hits"].size > 65536, "case must overflow the initial hit buffer"
    with Filter(prm) as f:
        f.add_patterns(pats)
        np.testing.assert_array_equal(f.process(text).hit_offsets, s["hits"])


def test_test_line_matches_oracle():
    prm, pats, text = build_inputs("dense_fp")
    o = oracle.Oracle.from_params(prm)
    o.build(pats)
    lines = bytes(text[:200_000]).split(b"\n")[:400] + [pats.split(b"\n")[0], b"", b"x" * 19, b"a\nb" * 20]
    with Filter(prm) as f:
        f.add_patterns(pats)
        for ln in lines:
            assert f.test_line(ln) == o.test_line(ln), ln


def test_hbm_budget_is_enforced():
    prm, pats, text = build_inputs("plain_small")
    with Filter(prm) as f:
        f.add_patterns(pats)
        f.set_hbm_budget(1)
        with pytest.raises(FFBFError) as e:
            f.process(text)
        assert e.value.status == 2


def test_bad_filter_file_rejected():
    prm = Params(20, 5, 2, 1 << 12, 1 << 14)
    with Filter(prm) as f:
        bad = np.array([5, prm.nbits], dtype="<u4").tobytes()
        with pytest.raises(FFBFError) as e:
            f.load_filter(bad)
        assert e.value.status == 1
        assert not f.get_filters()[0].any()


def test_cli_matches_reference_files():
    g = Golden("plain_small")
    prm, pats, text = build_inputs("plain_small")
    cli = os.path.join(ROOT, "ffbf_b200", "_lib", "ffbf")
    with tempfile.TemporaryDirectory() as wd:
        open(os.path.join(wd, "pats"), "wb").write(pats)
        open(os.path.join(wd, "text"), "wb").write(text.tobytes())
        for run in range(2):  # the second run loads __bloom_filter_pats
            with open(os.path.join(wd, "text"), "rb") as fin:
                r = subprocess.run([cli, "--len", "20", "pats", "out"], stdin=fin, capture_output=True, cwd=wd)
            assert r.returncode == 0, r.stderr
            assert g.matches("stdout", r.stdout)
            assert g.matches("pruned", open(os.path.join(wd, "out"), "rb").read())
            assert g.matches("index", open(os.path.join(wd, "__index_out"), "rb").read())
            assert g.matches("bloom", open(os.path.join(wd, "__bloom_filter_pats"), "rb").read())
            assert (b"filter load time:" in r.stderr) == (run == 1)
            assert b"processFile time:" in r.stderr and b"filterPhrases time:" in r.stderr
        with open(os.path.join(wd, "text"), "rb") as fin:
            r = subprocess.run([cli, "--len", "20", "--exact", "pats", "out"], stdin=fin, capture_output=True, cwd=wd)
        assert r.returncode == 0
        # --exact prints the lines `grep -F -f pats` prints (all patterns here are >= LEN bytes)
        g = subprocess.run(["grep", "-F", "-a", "-f", "pats", "text"], capture_output=True, cwd=wd,
                           env=dict(os.environ, LC_ALL="C"))
        assert r.stdout == g.stdout and len(g.stdout) > 0


SCAN_VARIANTS = [
    {"FFBF_FORCE_GENERIC_SCAN": "1"},
    {"FFBF_SCAN_MODE": "0", "FFBF_SCAN_THREADS": "256"},
    {"FFBF_SCAN_MODE": "0", "FFBF_SCAN_THREADS": "384"},
    {"FFBF_SCAN_MODE": "0", "FFBF_SCAN_THREADS": "512"},
    {"FFBF_SCAN_MODE": "3"},
    {"FFBF_SCAN_MODE": "2", "FFBF_SCAN_THREADS": "192"},
    {"FFBF_SCAN_MODE": "2", "FFBF_SCAN_THREADS": "256"},
    {"FFBF_SCAN_MODE": "2", "FFBF_SCAN_THREADS": "384"},
    {"FFBF_SCAN_MODE": "1", "FFBF_SCAN_ORDER": "0"},
    {"FFBF_SCAN_MODE": "1", "FFBF_SCAN_ORDER": "0", "FFBF_SCAN_THREADS": "256"},
    {"FFBF_SCAN_MODE": "1", "FFBF_SCAN_ORDER": "0", "FFBF_SCAN_THREADS": "192"},
    {"FFBF_SCAN_MODE": "1", "FFBF_SCAN_ORDER": "1", "FFBF_SCAN_THREADS": "192"},
    {"FFBF_SCAN_MODE": "1", "FFBF_SCAN_ORDER": "2", "FFBF_SCAN_THREADS": "192"},
    {"FFBF_SCAN_MODE": "1", "FFBF_SCAN_ORDER": "1"},
    {"FFBF_SCAN_MODE": "1", "FFBF_SCAN_ORDER": "1", "FFBF_SCAN_THREADS": "256"},
    {"FFBF_SCAN_MODE": "1", "FFBF_SCAN_ORDER": "2"},
    {"FFBF_SCAN_MODE": "1", "FFBF_SCAN_ORDER": "2", "FFBF_SCAN_THREADS": "256"},
]
SCAN_ENV = ("FFBF_FORCE_GENERIC_SCAN", "FFBF_SCAN_MODE", "FFBF_SCAN_THREADS", "FFBF_SCAN_ORDER")


@pytest.mark.parametrize("name", ["plain_small", "scale_small", "smem_cache", "edge_chunks", "binary_small",
                                  "dense_fp", "len19_default"])
def test_scan_variants_agree_with_oracle(name, monkeypatch):
    """Every scan kernel variant (generic; tuned sparse at each CTA size, with candidates queued per byte,
    with per-stage barriers, or deferred to the end of each 32-byte block; tuned dense in every probe order)
    is bit-exact."""
    prm, pats, text = build_inputs(name)
    o, s, _, _, _ = run_oracle(prm, pats, text)
    for env in SCAN_VARIANTS:
        for k in SCAN_ENV:
            monkeypatch.delenv(k, raising=False)
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        with Filter(prm) as f:
            f.add_patterns(pats)
            r = f.process(text)
            np.testing.assert_array_equal(r.hit_offsets, s["hits"], err_msg=str(env))
            np.testing.assert_array_equal(r.line_start, s["line_start"], err_msg=str(env))
            np.testing.assert_array_equal(r.line_end, s["line_end"], err_msg=str(env))
            np.testing.assert_array_equal(f.get_filters()[1], o.ff, err_msg=str(env))
    monkeypatch.setenv("FFBF_SCAN_THREADS", "0")
    with Filter(prm):
        pass  # restores the default CTA size for later tests


@pytest.mark.parametrize("name", ["hit_flood", "edge_mixed", "binary_small", "scale_small", "empty_text"])
def test_device_and_host_result_order_agree(name, monkeypatch):
    """Scan results and verified matches are put in text order on the device (radix sorts and a line
    selection); FFBF_HOST_ORDER=1 orders the same records on the host, the path taken when the device has no
    room for the sort. Both give the oracle's hit windows, lines and (offset, pattern id) matches, including
    many hits per line (hit_flood) and one offset matched by several pattern ids (edge_mixed)."""
    prm, pats, text = build_inputs(name)
    o, s, pr, ooff, opid = run_oracle(prm, pats, text)
    for host in ("0", "1"):
        monkeypatch.setenv("FFBF_HOST_ORDER", host)
        with Filter(prm) as f:
            f.add_patterns(pats)
            r = f.process(text)
            np.testing.assert_array_equal(r.hit_offsets, s["hits"], err_msg=host)
            np.testing.assert_array_equal(r.line_start, s["line_start"], err_msg=host)
            np.testing.assert_array_equal(r.line_end, s["line_end"], err_msg=host)
            np.testing.assert_array_equal(f.filter_phrases(), pr["ids"], err_msg=host)
            off, pid = f.verify()
            np.testing.assert_array_equal(off, ooff, err_msg=host)
            np.testing.assert_array_equal(pid, opid, err_msg=host)
    monkeypatch.delenv("FFBF_HOST_ORDER", raising=False)


@pytest.mark.parametrize("L,k,s", [(20, 1, 1), (20, 2, 1), (20, 2, 2), (24, 3, 1), (24, 4, 3), (24, 4, 4),
                                   (32, 5, 1), (16, 6, 2), (19, 11, 0)])
def test_dense_probe_orders_over_geometries(L, k, s, monkeypatch):
    """The dense mode pipelines two probes: f0/f1 (order 0), f2/f3 (order 1, K >= 4), or f0/f1 behind a
    shared-memory prefilter of f0 (order 2). The shared-memory mode runs here too, at both CTA sizes, with
    S = 1 (one stage-1 probe) and S >= 2 (two). Each geometry's regions decide where those probes land (cache or
    external) and which queued windows still need which probes; K = 1 has no second index function and falls
    back to the shared-memory mode."""
    from cases import _gen
    from ffbf_b200 import datagen as dg
    prm = Params(L, k, s, 1 << 14, 1 << 16)  # small regions: dense fills, many false positives
    pats, text = _gen(40 + k * 3 + s, dg.PRINTABLE, 3000, L, L + 16, 2_000_000, 80, 300)
    o, so, _, _, _ = run_oracle(prm, pats, text)
    variants = [{}, {"FFBF_SCAN_MODE": "0", "FFBF_SCAN_THREADS": "384"}, {"FFBF_SCAN_MODE": "0", "FFBF_SCAN_THREADS": "512"},
                {"FFBF_SCAN_MODE": "3"},
                {"FFBF_SCAN_MODE": "2"}, {"FFBF_SCAN_MODE": "1", "FFBF_SCAN_ORDER": "0"},
                {"FFBF_SCAN_MODE": "1", "FFBF_SCAN_ORDER": "1"},
                {"FFBF_SCAN_MODE": "1", "FFBF_SCAN_ORDER": "1", "FFBF_SCAN_THREADS": "256"},
                {"FFBF_SCAN_MODE": "1", "FFBF_SCAN_ORDER": "1", "FFBF_SCAN_THREADS": "192"},
                {"FFBF_SCAN_MODE": "1", "FFBF_SCAN_ORDER": "2"}]
    for env in variants:
        for key in SCAN_ENV:
            monkeypatch.delenv(key, raising=False)
        for key, v in env.items():
            monkeypatch.setenv(key, v)
        with Filter(prm) as f:
            f.add_patterns(pats)
            r = f.process(text)
            np.testing.assert_array_equal(r.hit_offsets, so["hits"], err_msg=str(env))
            np.testing.assert_array_equal(r.line_start, so["line_start"], err_msg=str(env))
            np.testing.assert_array_equal(f.get_filters()[1], o.ff, err_msg=str(env))
            if k < 2:
                assert f.config()[1] != 1, "K = 1 must not run the dense mode"
            if s < 1:
                pass  # no cache-region probe: the generic scan runs and no probe plan is chosen
            elif env.get("FFBF_SCAN_ORDER") == "1" and k < 4:
                assert f.probe_order() == 0, "order 1 needs f2 and f3"
            elif "FFBF_SCAN_ORDER" in env:
                assert f.probe_order() == int(env["FFBF_SCAN_ORDER"])
    for key in SCAN_ENV:
        monkeypatch.delenv(key, raising=False)
    monkeypatch.setenv("FFBF_SCAN_THREADS", "0")
    with Filter(prm):
        pass  # restores the default CTA size for later tests


def test_line_resolution_over_many_tile_blocks():
    """Texts above 4096 tiles (64 MiB) resolve lines with the two-pass tile-newline scan: a 100 MiB text with
    50 KB lines and one 80 MiB line, so a whole block of tiles holds no '\\n' and the line's start and end
    come from other blocks. Lines, hits and feed-forward bits equal the oracle's."""
    from ffbf_b200 import datagen as dg

    prm = Params(20, 5, 2, 1 << 24, 1 << 28)
    pats = dg.gen_patterns(31, dg.PRINTABLE, 2000, 20, 40)
    text = dg.gen_text(32, dg.PRINTABLE, 100 << 20, 50000)
    seg = text[10 << 20:90 << 20]
    seg[seg == 10] = ord("x")
    dg.plant(33, pats, text, 3000)
    o = oracle.Oracle.from_params(prm)
    o.build(pats)
    s = o.scan(text)
    assert ((s["line_end"] - s["line_start"]) > (64 << 20)).any()
    with Filter(prm) as f:
        f.add_patterns(pats)
        r = f.process(text)
        np.testing.assert_array_equal(r.hit_offsets, s["hits"])
        np.testing.assert_array_equal(r.line_start, s["line_start"])
        np.testing.assert_array_equal(r.line_end, s["line_end"])
        np.testing.assert_array_equal(f.get_filters()[1], o.ff)


@pytest.mark.parametrize("mib", [300, 40])
def test_host_text_scan_with_overlapped_copy_equals_oracle(mib):
    """A host text of 32 MiB or more is copied in chunks (about an eighth of the text, 8-128 MiB) while the
    scan runs on the chunks that have landed; windows, lines and the feed-forward filter equal the oracle's,
    including windows across every MiB boundary (chunk boundaries fall on whole MiB here) and a long line
    across chunks."""
    from ffbf_b200 import datagen as dg

    prm = Params(20, 5, 2, 1 << 24, 1 << 28)
    pats = dg.gen_patterns(41, dg.PRINTABLE, 3000, 20, 40)
    text = dg.gen_text(42, dg.PRINTABLE, mib << 20, 2000)
    lo, hi = (mib << 20) // 3, (mib << 20) // 2
    seg = text[lo:hi]
    seg[seg == 10] = ord("y")
    dg.plant(43, pats, text, 4000)
    occ = np.frombuffer(pats[:25].tobytes(), dtype=np.uint8)
    for k in range(1, mib):  # occurrences straddling each MiB boundary
        text[(k << 20) - 10:(k << 20) - 10 + occ.size] = occ
    o = oracle.Oracle.from_params(prm)
    o.build(pats)
    s = o.scan(text)
    with Filter(prm) as f:
        f.add_patterns(pats)
        r = f.process(text)
        np.testing.assert_array_equal(r.hit_offsets, s["hits"])
        np.testing.assert_array_equal(r.line_start, s["line_start"])
        np.testing.assert_array_equal(r.line_end, s["line_end"])
        np.testing.assert_array_equal(f.get_filters()[1], o.ff)
    assert any((k << 20) - 10 in set(s["hits"].tolist()) for k in range(1, 4)), "a straddling window should hit"


def test_text_larger_than_the_device_budget_is_scanned_in_segments():
    """A host text that does not fit the context's HBM budget is scanned in line-aligned segments; hits,
    lines, the feed-forward filter, the prune and the verified matches equal the oracle's, and stdout
    formatting over the whole text is unchanged."""
    from ffbf_b200 import datagen as dg

    prm = Params(20, 5, 2, 1 << 20, 1 << 24)
    pats = dg.gen_patterns(51, dg.PRINTABLE, 3000, 20, 40)
    text = dg.gen_text(52, dg.PRINTABLE, 40 << 20, 200)
    dg.plant(53, pats, text, 3000)
    o, s, pr, ooff, opid = run_oracle(prm, pats, text)
    with Filter(prm) as f:
        f.add_patterns(pats)
        f.set_hbm_budget(32 << 20)  # about 24 MB left beside the filters: segments of about 18 MB
        r = f.process(text)
        np.testing.assert_array_equal(r.hit_offsets, s["hits"])
        np.testing.assert_array_equal(r.line_start, s["line_start"])
        np.testing.assert_array_equal(r.line_end, s["line_end"])
        assert f.format_lines(text) == s["out"]
        np.testing.assert_array_equal(f.get_filters()[1], o.ff)
        np.testing.assert_array_equal(f.filter_phrases(), pr["ids"])
        off, pid = f.verify()
        np.testing.assert_array_equal(off, ooff)
        np.testing.assert_array_equal(pid, opid)
        # a line longer than a segment cannot be split
        one_line = np.full(30 << 20, ord("a"), dtype=np.uint8)
        with pytest.raises(FFBFError) as e:
            f.process(one_line)
        assert e.value.status == 1


def test_cpp_mirror_program_matches_reference_files(tmp_path):
    """A C++ program driving ffbf::Filter like the reference's main prints the reference's stdout and writes its
    pruned and index files (golden plain_small); its server request finds the direct scan's hits."""
    from test_host_cpu import build_mirror_example

    exe = build_mirror_example(str(tmp_path))
    g = Golden("plain_small")
    prm, pats, text = build_inputs("plain_small")
    (tmp_path / "pats").write_bytes(pats)
    (tmp_path / "text").write_bytes(text.tobytes())
    for mode in ([], ["server"]):
        with open(tmp_path / "text", "rb") as fin:
            r = subprocess.run([exe, "20", "pats", "out"] + mode, stdin=fin, capture_output=True, cwd=tmp_path)
        assert r.returncode == 0, r.stderr
        assert g.matches("stdout", r.stdout)
        assert g.matches("pruned", (tmp_path / "out").read_bytes())
        assert g.matches("index", (tmp_path / "__index_out").read_bytes())
        direct = int(re.search(rb"direct scan: (\d+) hits", r.stderr).group(1))
        assert re.search(rb"scan config: (192|256|384|512) threads, mode [0-3], probe order [012]", r.stderr), r.stderr
        if mode:
            served = int(re.search(rb"status 0, (\d+) hits", r.stderr).group(1))
            assert served == direct > 0
