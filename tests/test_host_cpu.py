"""Host-side checks that need no GPU: the C ABI's exports, argument validation, and the output formatting
rules (ffbf_format_spans) against the oracle's literal restatement of processFile."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import ffbf_b200
import oracle
from cases import build_inputs
from conftest import ROOT, has_gpu


def header_functions():
    src = open(os.path.join(ROOT, "include", "ffbf.h")).read()
    return sorted(set(re.findall(r"\b(ffbf_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_function():
    lib = ffbf_b200.load_library()
    names = header_functions()
    assert len(names) >= 26
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/ffbf.h but not exported"
    assert set(ffbf_b200.EXPORTED) >= set(names)
    out = subprocess.run(["nm", "-D", "--defined-only", ffbf_b200.lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (ffbf_[a-z_0-9]+)$", out, re.M))
    assert set(names) <= exported


def test_status_strings_and_defaults():
    lib = ffbf_b200.load_library()
    assert lib.ffbf_status_string(0) == b"ok"
    assert lib.ffbf_status_string(5) == b"CUDA error"
    p = ffbf_b200.Params(1, 1, 1, 32, 32)
    assert lib.ffbf_params_default(ctypes.byref(p)) == 0
    assert p.as_tuple() == (19, 5, 2, 1 << 24, 1 << 28)


@pytest.mark.parametrize("bad", [
    (0, 5, 2, 1 << 24, 1 << 28), (64, 5, 2, 1 << 24, 1 << 28), (19, 0, 0, 1 << 24, 1 << 28),
    (19, 12, 2, 1 << 24, 1 << 28), (19, 5, 6, 1 << 24, 1 << 28), (19, 5, 2, 3 << 20, 1 << 28),
    (19, 5, 2, 16, 1 << 28), (19, 5, 2, 1 << 31, 1 << 31)])
def test_create_rejects_bad_geometry(bad):
    lib = ffbf_b200.load_library()
    h = ctypes.c_void_p()
    assert lib.ffbf_create(ctypes.byref(ffbf_b200.Params(*bad)), 0, ctypes.byref(h)) == 1
    assert not h.value


@pytest.mark.skipif(has_gpu(), reason="a GPU is present")
def test_create_without_gpu_fails_loudly():
    with pytest.raises(ffbf_b200.FFBFError) as e:
        ffbf_b200.Filter(ffbf_b200.Params())
    assert e.value.status == 5


@pytest.mark.parametrize("name", ["edge_chunks", "edge_nul_chunk", "edge_mixed", "plain_small", "binary_small"])
@pytest.mark.parametrize("chunk", [512 * 1024, 4096, 97])
def test_format_spans_matches_processfile_output(name, chunk):
    prm, pats, text = build_inputs(name)
    o = oracle.Oracle.from_params(prm)
    o.build(pats)
    s = o.scan(text, chunk=chunk)
    assert ffbf_b200.format_spans(text, s["line_start"], s["line_end"], chunk) == s["out"]


@pytest.mark.parametrize("chunk", [512 * 1024, 1000])
def test_format_spans_matches_filterphrases_output(chunk):
    prm, pats, text = build_inputs("dense_fp")
    o = oracle.Oracle.from_params(prm)
    o.build(pats)
    o.scan(text)
    pr = o.prune(pats, chunk=chunk)
    pa = np.frombuffer(pats, np.uint8)
    nl = np.flatnonzero(pa == 10)
    starts = np.concatenate([[0], nl + 1])[pr["ids"].astype(np.int64)]
    ends = np.concatenate([nl, [pa.size]])[pr["ids"].astype(np.int64)]
    assert ffbf_b200.format_spans(pats, starts, ends, chunk) == pr["out"]


def test_format_spans_rejects_bad_spans():
    with pytest.raises(ffbf_b200.FFBFError):
        ffbf_b200.format_spans(b"abc\ndef\n", [4, 0], [7, 3])
    with pytest.raises(ffbf_b200.FFBFError):
        ffbf_b200.format_spans(b"abc\n", [0], [9])


def test_cli_usage_error():
    cli = os.path.join(ROOT, "ffbf_b200", "_lib", "ffbf")
    r = subprocess.run([cli, "only_one_arg"], capture_output=True)
    assert r.returncode == 255
    assert b"Usage: ffbf phrases phrases.out < corpus > filtered_corpus" in r.stderr


def build_mirror_example(out_dir):
    """Compiles tests/cpp/mirror_example.cpp against include/ffbf.hpp and links it to libffbf.so."""
    exe = os.path.join(out_dir, "mirror_example")
    lib = os.path.join(ROOT, "ffbf_b200", "_lib")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", f"-I{os.path.join(ROOT, 'include')}",
                    os.path.join(ROOT, "tests", "cpp", "mirror_example.cpp"), "-o", exe, f"-L{lib}", "-lffbf",
                    f"-Wl,-rpath,{lib}"], check=True, capture_output=True)
    return exe


def test_cpp_mirror_header_compiles_and_links(tmp_path):
    """include/ffbf.hpp (Filter, Batch, Server) compiles warning-free in a program written like the reference's
    main and links against the library; without a device the program reports FilterError, not a crash."""
    exe = build_mirror_example(str(tmp_path))
    if has_gpu():
        return
    (tmp_path / "pats").write_bytes(b"abcdefghijklmnopqrstuvwxyz\n")
    r = subprocess.run([exe, "20", "pats", "out"], input=b"text\n", capture_output=True, cwd=tmp_path)
    assert r.returncode == 1 and b"FilterError" in r.stderr


def test_scan_sizing_rules_on_the_host(tmp_path):
    """tests/cpp/row_model.cu, linked against libffbf.so, checks the tuned scan's rows per stream (waves of
    items over the CTA slots, alone and in a batch), CTA sizes per configuration and the result sorts' key
    widths; all host code, so it runs without a device."""
    import shutil
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    exe = str(tmp_path / "row_model")
    lib = os.path.join(ROOT, "ffbf_b200", "_lib")
    subprocess.run([nvcc, "-std=c++17", "-O2", f"-I{os.path.join(ROOT, 'include')}",
                    f"-I{os.path.join(ROOT, 'ffbf_b200', 'csrc')}", os.path.join(ROOT, "tests", "cpp", "row_model.cu"),
                    "-o", exe, f"-L{lib}", "-lffbf", f"-Xlinker=-rpath,{lib}", "-lcuda"], check=True,
                   capture_output=True)
    r = subprocess.run([exe], capture_output=True)
    assert r.returncode == 0, r.stdout.decode() + r.stderr.decode()


def _bench():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_bench_reads_the_committed_profiles():
    """bench.py's roofline traffic and probe bound come from the ncu summaries in profiles/."""
    b = _bench()
    assert 1.0 < b.profiled_traffic_ratio("scale") < 1.2
    assert 1.0 < b.profiled_traffic_ratio("plain") < 1.2
    pb = b.probe_bound("scale", 319.0, 1965.0, 148)
    assert pb["probes_per_text_byte"] == pytest.approx(0.766, abs=0.01)
    assert pb["achieved"] == pytest.approx(pb["probes_per_text_byte"] * 319e9 / (148 * 1965e6))
    assert b.probe_bound("plain", 500.0, 1965.0, 148) is None  # no probe row for the sparse workload
    assert b.probe_bound("scale", 319.0, None, 148) is None     # no clock sample, no figure


def test_bench_pattern_override_names_its_own_workload(monkeypatch):
    """--patterns makes another workload: its line names it and no committed profile applies to it."""
    import sys
    b = _bench()
    monkeypatch.setattr(sys, "argv", ["bench.py", "--patterns", "200000", "--text-bytes", str(1 << 20)])
    wl = b.workload(b.parse())
    assert wl.name == "scale_200k" and wl.n_patterns == 200000 and wl.text_bytes == 1 << 20
    assert b.profiled_traffic_ratio(wl.name) is None
    assert b.describe(wl)["workload"].startswith("scale_200k: 200000 patterns")


def test_reference_arm_runs_the_whole_text_without_repository_libraries(tmp_path):
    """bench.py --impl reference needs no GPU: the reference binary scans the whole workload text in
    line-aligned shards, and the arm's own process maps none of this repository's shared libraries (a child
    process writes the inputs)."""
    import json
    import sys

    from ffbf_b200 import datagen
    if oracle.ref_binary(datagen.plain().params) is None:
        pytest.skip("reference binary for the plain geometry not built (oracle/_ref)")
    probe = tmp_path / "arm.py"
    probe.write_text(
        "import json, sys\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'plain', '--steps', '1', '--warmup', '0']\n"
        "import bench\n"
        "bench.main_reference(bench.parse())\n"
        "maps = open('/proc/self/maps').read().split('\\n')\n"
        f"mine = sorted({{m.split()[-1] for m in maps if {ROOT!r} in m and m.endswith('.so')}})\n"
        "print(json.dumps({'repo_libraries': mine}))\n")
    out = subprocess.run([sys.executable, str(probe)], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(x) for x in out.stdout.strip().splitlines()]
    arm, maps = lines[-2], lines[-1]
    assert arm["impl"] == "reference" and arm["value"] > 0
    assert arm["config"]["text_bytes"] == 64 << 20
    assert "whole" in arm["cpu_baseline"]["sample"]
    assert maps["repo_libraries"] == []
