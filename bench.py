"""Benchmark: FFBF scan throughput on one B200 (or N independent replicas).

Default workload ("scale"): 1,000,000 Zipf-word patterns of 32-64 bytes, LEN 32, filter geometry K 5, S 2,
2^23 cache bits + 2^26 external bits (9 MiB, L2-resident); a 4 GiB text of the same letters with '\\n' every
geometric(mean 100) bytes and 20,000 planted occurrences; all from one seed (synthetic data, see
ffbf_b200/datagen.py).

One step = one pass of the scan over the whole text: zero the feed-forward filter, then run the scan kernel
(hash every window, probe the main filter, set feed-forward bits for hits, record hit windows and per-tile
newline summaries). `value` is text GB/s with the text resident in HBM, timed with CUDA events on the
library's stream; the 4 GiB input is larger than L2, so no flush is needed between steps. `e2e` is the same
metric through the public C ABI from pinned host memory: ffbf_scan (H2D copy, scan, hit/line collection)
+ ffbf_prune + ffbf_verify, with every result copied back to the host.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--workload scale|plain|binary]

With --impl reference the same workload is scanned by efficient/ffbf's own x86 binary (oracle/_ref, built
from the reference sources) on all host cores: one process per core, each on its own line-aligned shard of
the text, filter loaded from a __bloom_filter_ cache; throughput = shard bytes / the slowest process's
`processFile time` (the reference's own timer).
"""
import argparse
import collections
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "scan GB/s & %HBM roofline at 1M patterns"
UNIT = "GB/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["scale", "plain", "binary", "batched", "served"], default="scale")
    ap.add_argument("--batch-jobs", type=int, default=512, help="jobs of the batched workload")
    ap.add_argument("--batch-max-text", type=int, default=256 << 20, help="largest job text of the batched workload")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched leg of the default run")
    ap.add_argument("--no-served", action="store_true", help="skip the served leg of the default run")
    ap.add_argument("--served-requests", type=int, default=4000, help="requests of the served workload")
    ap.add_argument("--served-rate", type=float, default=2000.0, help="Poisson arrival rate (requests/s)")
    ap.add_argument("--text-bytes", type=int, default=0, help="override the workload's text size")
    ap.add_argument("--patterns", type=int, default=0,
                    help="override the workload's pattern count (the line then names it, e.g. scale_200k)")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--e2e-steps", type=int, default=0, help="steps of the end-to-end leg (default: min(steps, 5))")
    ap.add_argument("--cpu-sample", type=int, default=1 << 30, help="bytes of text for the CPU baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def workload(args):
    from ffbf_b200 import datagen as dg
    fn = {"scale": dg.scale, "plain": dg.plain, "binary": dg.binary}[args.workload]
    kw = {}
    if args.text_bytes:
        kw["text_bytes"] = args.text_bytes
    if args.patterns:
        kw["n_patterns"] = args.patterns
    wl = fn(**kw)
    if args.patterns:
        # another pattern count is another workload: no committed profile describes it
        wl.name = f"{wl.name}_{args.patterns // 1000}k"
    return wl


def describe(wl):
    p = wl.params
    return {"workload": f"{wl.name}: {wl.n_patterns} patterns ({wl.len_lo}-{wl.len_hi} B), LEN {p.len}, "
                        f"{wl.text_bytes / 2**30:.3g} GiB text, {wl.n_plant} planted",
            "geometry": {"len": p.len, "k": p.k, "s": p.s, "cache_bits": p.cache_bits, "ext_bits": p.ext_bits},
            "text_bytes": wl.text_bytes, "n_patterns": wl.n_patterns}


# ---- clocks -------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.path = tempfile.mktemp(prefix="ffbf_clocks_", suffix=".csv")
        self.proc = None
        self.gpu_id = gpu_id

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.out = open(self.path, "w")
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"]
        if self.gpu_id is not None:
            cmd += ["-i", str(self.gpu_id)]
        self.proc = subprocess.Popen(cmd, stdout=self.out, stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        sm, mx, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm), "power_w_max": max(power) if power else None}


def gpu_id_for(dev):
    import torch
    try:
        p = torch.cuda.get_device_properties(dev)
        return f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
    except Exception:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        return vis.split(",")[dev] if vis else dev


def profiled_value(workload_name, row):
    """A per-text-byte figure of the scan kernel (table row `row`) from the committed ncu summary for this
    workload: traffic_bytes_per_text_byte (DRAM bytes) or l2_probes_per_text_byte (L2 requests)."""
    paths = [os.path.join(ROOT, "profiles", f"k_scan_fast_{m}_{workload_name}_256MiB.md") for m in ("dense", "sparse")]
    path = next((q for q in paths if os.path.exists(q)), None)
    if path is None:
        return None
    for line in open(path):
        if line.startswith(f"| {row} |"):
            return float(line.split("|")[2])
    return None


def profiled_traffic_ratio(workload_name):
    return profiled_value(workload_name, "traffic_bytes_per_text_byte")


PROBE_CEILING = 1.0  # random 4-byte L2 probes per clock per SM, measured on this pool's B200s


def probe_bound(workload_name, gbs, sm_mhz, n_sms):
    """The dense scan's real limit: random L2 probes of the filter, issued through the L1TEX unit."""
    per_byte = profiled_value(workload_name, "l2_probes_per_text_byte")
    if per_byte is None or not sm_mhz:
        return None
    achieved = per_byte * gbs * 1e9 / (n_sms * sm_mhz * 1e6)
    return {"unit": "L2 probes/clk/SM", "achieved": achieved, "ceiling": PROBE_CEILING, "frac": achieved / PROBE_CEILING,
            "probes_per_text_byte": per_byte, "sms": n_sms, "sm_mhz": sm_mhz,
            "source": "probes per byte from the ncu summary in profiles/; ceiling from a random-probe microbenchmark"}


L2_FLUSH_BYTES = 256 << 20  # about twice the 126 MB L2


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---- the reference on the host cores ----------------------------------------------------------------
def line_shards(text, n_shards, shard_bytes):
    """Line-aligned [a, b) slices: shard i starts after the first '\\n' at or past i*shard_bytes."""
    out = []
    for i in range(n_shards):
        a = i * shard_bytes
        b = (i + 1) * shard_bytes
        if b > text.size:
            break
        if a > 0:
            nl = np.flatnonzero(text[a:a + 65536] == 10)
            a = a + int(nl[0]) + 1 if nl.size else a
        nl = np.flatnonzero(text[b:b + 65536] == 10)
        b = b + int(nl[0]) + 1 if nl.size else b
        out.append((a, min(b, text.size)))
    return out


def reference_binary(prm):
    import oracle
    return oracle.ref_binary(prm, build=os.path.exists(oracle.DEFAULT_REF_SRC))


def prepare_reference_dirs(binary, pats, text, shards):
    """One scratch dir per shard holding pats, the shard text and a __bloom_filter_pats cache built by the
    reference itself (one run over an empty text)."""
    base = tempfile.mkdtemp(prefix="ffbf_refbench_", dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    seed_dir = os.path.join(base, "seed")
    os.makedirs(seed_dir)
    with open(os.path.join(seed_dir, "pats"), "wb") as f:
        f.write(pats.tobytes())
    open(os.path.join(seed_dir, "empty"), "wb").close()
    with open(os.path.join(seed_dir, "empty"), "rb") as fin:
        subprocess.run([binary, "pats", "out"], stdin=fin, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                       cwd=seed_dir, check=True)
    dirs = []
    for i, (a, b) in enumerate(shards):
        d = os.path.join(base, f"s{i}")
        os.makedirs(d)
        os.link(os.path.join(seed_dir, "pats"), os.path.join(d, "pats"))
        shutil.copyfile(os.path.join(seed_dir, "__bloom_filter_pats"), os.path.join(d, "__bloom_filter_pats"))
        text[a:b].tofile(os.path.join(d, "text"))
        dirs.append((d, b - a))
    return base, dirs


def run_reference_step(binary, dirs):
    procs = []
    for d, _ in dirs:
        fin = open(os.path.join(d, "text"), "rb")
        p = subprocess.Popen([binary, "pats", "out"], stdin=fin, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE,
                             cwd=d)
        procs.append((p, fin))
    times = []
    for p, fin in procs:
        _, err = p.communicate()
        fin.close()
        if p.returncode != 0:
            raise RuntimeError(f"reference exited {p.returncode}: {err.decode(errors='replace')}")
        t = [float(x.split(b":")[1]) for x in err.splitlines() if x.startswith(b"processFile time:")]
        times.append(t[0])
    return max(times)


def cpu_baseline_single(wl, pats, text, sample_bytes):
    """The reference binary on one core over a bounded, line-aligned prefix of the workload text."""
    binary = reference_binary(wl.params)
    if binary is None:
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "unavailable: reference binary for this geometry was not built"}
    shards = line_shards(text, 1, min(sample_bytes, text.size - 65536))
    base, dirs = prepare_reference_dirs(binary, pats, text, shards)
    try:
        t = run_reference_step(binary, dirs)
    finally:
        shutil.rmtree(base, ignore_errors=True)
    nbytes = dirs[0][1]
    return {"value": nbytes / t / 1e9, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"{nbytes / 2**20:.0f} MiB line-aligned prefix of the workload text, 1 process, filter "
                      f"loaded from its __bloom_filter_ cache; processFile time {t:.3f} s"}


def main_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wl = workload(args)
    binary = reference_binary(wl.params)
    cfg = describe(wl)
    if binary is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference binary for this geometry not built"}))
        return 0
    pats = wl.patterns(args.seed)
    text = wl.text(args.seed, pats)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    nproc = max(1, min(cores, 64))
    shard = min(32 << 20, (text.size - 65536) // nproc)
    shards = line_shards(text, nproc, shard)
    base, dirs = prepare_reference_dirs(binary, pats, text, shards)
    try:
        total = sum(n for _, n in dirs)
        for _ in range(args.warmup):
            run_reference_step(binary, dirs)
        ts = [run_reference_step(binary, dirs) for _ in range(args.steps)]
    finally:
        shutil.rmtree(base, ignore_errors=True)
    t = statistics.mean(ts)
    value = total / t / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": len(dirs), "kind": "reference",
                             "sample": f"{len(dirs)} processes x {shard / 2**20:.0f} MiB line-aligned shards "
                                       f"({total / 2**30:.2f} GiB per step), filter from __bloom_filter_ cache"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---- batched form: 512 uneven jobs in one graph launch vs plain per-job launches ------------------------
def ff_digest(f):
    """A 64-bit digest of a filter's feed-forward bit array (copied to the host)."""
    import ctypes
    ff = np.zeros(f.filter_bytes, dtype=np.uint8)
    f._check(f._lib.ffbf_get_filters(f._h, None, ff.ctypes.data_as(ctypes.c_void_p)))
    w = ff.view(np.uint64)
    idx = np.arange(w.size, dtype=np.uint64)
    return int(np.bitwise_xor.reduce(w * (idx * np.uint64(0x9E3779B97F4A7C15) | np.uint64(1)))) ^ int(w.sum())


def run_batched(args, local):
    """Scans every job of the batched workload in three forms and checks that they agree bit for bit.

    Forms: `batched` = ffbf_batch_launch (one graph: counters reset, one persistent tuned launch per
    (LEN, configuration) group with a work queue over all its jobs' items, one generic launch for every
    job's ragged tail); `plain_serial` = ffbf_scan_device per job, each waited for before the next (one
    job per launch, as a caller of the plain API runs them); `plain_streams` = ffbf_scan_device for all jobs
    back to back, each on its own context stream, then one wait (the plain API's best case).
    Texts are device resident in all forms; all are timed by the host clock between device-idle points,
    the batched form also by CUDA events on the batch's stream.
    """
    from concurrent.futures import ThreadPoolExecutor

    import torch

    import ffbf_b200
    from ffbf_b200 import Batch, Filter
    from ffbf_b200 import datagen as dg

    dev = torch.device("cuda", local)
    jobs = dg.batched(n_jobs=args.batch_jobs, text_hi=args.batch_max_text, seed=args.seed)
    t_gen = time.perf_counter()
    with ThreadPoolExecutor(min(32, os.cpu_count() or 1)) as ex:
        pats = list(ex.map(lambda w: w.patterns(w.seed), jobs))
    offs, total = [], 0
    for w in jobs:
        offs.append(total)
        total += (w.text_bytes + 255) // 256 * 256
    host = torch.empty(total, dtype=torch.uint8, pin_memory=True)
    hv = host.numpy()
    for w, pb, o in zip(jobs, pats, offs):
        w.text(w.seed, pb, out=hv[o:o + w.text_bytes])
    d_all = torch.empty(total, dtype=torch.uint8, device=dev)
    d_all.copy_(host)
    filters = []
    for w, pb in zip(jobs, pats):
        f = Filter(w.params, device=local)
        f.add_patterns(pb)
        filters.append(f)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t_gen
    base = d_all.data_ptr()
    nbytes = sum(w.text_bytes for w in jobs)

    def plain_serial():
        for f, w, o in zip(filters, jobs, offs):
            f.process_device(base + o, w.text_bytes)
            torch.cuda.ExternalStream(f.stream, device=dev).synchronize()

    def plain_streams():
        for f, w, o in zip(filters, jobs, offs):
            f.process_device(base + o, w.text_bytes)
        for f in filters:
            torch.cuda.ExternalStream(f.stream, device=dev).synchronize()

    b = Batch(local)
    for f, w, o in zip(filters, jobs, offs):
        b.add(f, base + o, w.text_bytes)
    # the autotuner picks each class of jobs' configuration; plain and batched forms both use it
    t0 = time.perf_counter()
    n_classes = b.autotune(16 << 20)
    tune_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    b.prepare()
    prepare_s = time.perf_counter() - t0

    def batched():
        b.launch()
        b.wait()

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        launches0 = ffbf_b200.kernel_launches()
        ts = []
        for _ in range(args.steps):
            t = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t)
        return statistics.median(ts), (ffbf_b200.kernel_launches() - launches0) // max(args.steps, 1)

    def results():
        out = []
        for f in filters:
            r = f.collect()
            out.append((r.hit_offsets.copy(), r.line_start.copy(), r.line_end.copy(), ff_digest(f)))
        return out

    # every form starts from cleared feed-forward filters, so each form's results stand alone
    for f in filters:
        f.clear_ff()
    t_plain, l_plain = timed(plain_serial)
    ref = results()
    for f in filters:
        f.clear_ff()
    t_streams, l_streams = timed(plain_streams)
    got_streams = results()
    for f in filters:
        f.clear_ff()
    t_batch, l_batch = timed(batched)
    bst = torch.cuda.ExternalStream(b.stream, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dev_ms = []
    for _ in range(args.steps):
        e0.record(bst)
        b.launch()
        e1.record(bst)
        b.wait()
        dev_ms.append(e0.elapsed_time(e1))
    got_batch = results()

    def same(x, y):
        return all(np.array_equal(a[0], c[0]) and np.array_equal(a[1], c[1]) and np.array_equal(a[2], c[2])
                   and a[3] == c[3] for a, c in zip(x, y))

    out = {
        "workload": f"batched: {len(jobs)} jobs, {sum(w.n_patterns for w in jobs)} patterns (per job 1k-256k "
                    f"log-uniform, 24-48 B, LEN 24), {nbytes / 2**30:.2f} GiB text (per job 256 KiB-"
                    f"{args.batch_max_text >> 20} MiB log-uniform), 0.01% of windows planted",
        "text_bytes": nbytes, "jobs": len(jobs), "hit_windows": sum(int(r[0].size) for r in ref),
        "batched_gbs": nbytes / t_batch / 1e9,
        "batched_device_gbs": nbytes / (statistics.median(dev_ms) * 1e-3) / 1e9,
        "plain_serial_gbs": nbytes / t_plain / 1e9, "plain_streams_gbs": nbytes / t_streams / 1e9,
        "batched_over_plain_serial": t_plain / t_batch, "batched_over_plain_streams": t_streams / t_batch,
        "launches_per_step": {"batched": int(l_batch), "plain_serial": int(l_plain), "plain_streams": int(l_streams)},
        "ms_per_step": {"batched": t_batch * 1e3, "batched_device": statistics.median(dev_ms),
                        "plain_serial": t_plain * 1e3, "plain_streams": t_streams * 1e3},
        "bit_exact": {"plain_streams_vs_plain": same(got_streams, ref), "batched_vs_plain": same(got_batch, ref)},
        "setup_s": {"generate_and_build": gen_s, "autotune": tune_s, "batch_prepare": prepare_s},
        "autotune_classes": n_classes,
        "configs": dict(collections.Counter(
            (f"dense-{f.config()[0]}-order{f.probe_order()}" if f.config()[1] else f"sparse-{f.config()[0]}")
            for f in filters)),
        "timing": "host clock between device-idle points, median of steps; batched_device = CUDA events",
    }
    b.close()
    for f in filters:
        f.close()
    del d_all
    torch.cuda.empty_cache()
    return out


# ---- served form: resident sets, Poisson arrivals, continuous batching vs serial plain calls ------------
def served_trace(n, rate, seed, n_sets, pool_bytes):
    """(arrival s, set, offset, length) per request: Poisson arrivals, sets uniform, sizes log-normal
    (median 1 MiB, sigma 1.5, capped at 512 MiB), 256-byte aligned offsets into the text pool."""
    rng = np.random.default_rng(seed ^ 0x5E4BED)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
    sets = rng.integers(0, n_sets, n)
    sizes = np.minimum(np.exp(np.log(1 << 20) + 1.5 * rng.standard_normal(n)), 512 << 20).astype(np.int64)
    sizes = np.maximum(sizes, 1)
    offs = (rng.integers(0, pool_bytes - sizes + 1) // 256 * 256).astype(np.int64)
    return [(float(a), int(si), int(o), int(z)) for a, si, o, z in zip(arrivals, sets, offs, sizes)]


def wait_until(start, t):
    """Sleeps, then spins, until t seconds after start (sleeping releases the GIL for other threads)."""
    while True:
        dt = t - (time.perf_counter() - start)
        if dt <= 0:
            return
        if dt > 5e-4:
            time.sleep(dt - 3e-4)


def pct(xs, q):
    return float(np.percentile(np.asarray(xs), q)) if len(xs) else None


def run_served(args, local):
    """The served workload through ffbf_server_* and through serial plain ffbf_scan calls.

    8 resident sets of 100k-1M printable patterns (32-64 B, LEN 32, the scale workload's geometry); one
    1 GiB pinned pool of printable text ('\\n' after geometric(mean 100) bytes) with occurrences of every
    set planted, from which each request takes a slice. Runs: `served` at the Poisson rate (latency =
    server's done - submit time), `served_saturated` with every request submitted at once (capacity),
    `plain_serial` = one ffbf_scan call per request in arrival order, paced by the same arrival times
    (latency includes waiting for the previous call), and its unpaced capacity. All from host memory:
    every request's bytes cross PCIe in every run.
    """
    import threading

    import torch

    from ffbf_b200 import Filter, Server
    from ffbf_b200 import datagen as dg

    n_sets, pool_bytes = 8, 1 << 30
    rng = np.random.default_rng(args.seed ^ 0x5E7)
    counts = rng.integers(100_000, 1_000_001, n_sets)
    prm = dg.scale().params
    t0 = time.perf_counter()
    pats = [dg.gen_patterns(args.seed + 100 + i, dg.PRINTABLE, int(c), 32, 64) for i, c in enumerate(counts)]
    host = torch.empty(pool_bytes, dtype=torch.uint8, pin_memory=True)
    pool = host.numpy()
    dg.gen_text(args.seed + 99, dg.PRINTABLE, pool_bytes, 100, out=pool)
    for i, pb in enumerate(pats):
        dg.plant(args.seed + 200 + i, pb, pool, 2000)
    filters = []
    for pb in pats:
        f = Filter(prm, device=local)
        f.add_patterns(pb)
        filters.append(f)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    trace = served_trace(args.served_requests, args.served_rate, args.seed, n_sets, pool_bytes)
    total = sum(z for _, _, _, z in trace)

    # serial plain calls: paced by the arrival times, then back to back
    def plain(paced):
        for f in filters:
            f.clear_ff()
        lat, res = [], []
        start = time.perf_counter()
        for a, si, o, z in trace:
            if paced:
                wait_until(start, a)
            r = filters[si].process(pool[o:o + z])
            done = time.perf_counter() - start
            lat.append(done - (a if paced else 0.0))
            res.append((r.hit_offsets.copy(), r.line_start.copy()))
        return lat, res, time.perf_counter() - start, [ff_digest(f) for f in filters]

    # warm-up: each set's context scans the trace's largest text once, so no timed call grows a buffer
    big = max(trace, key=lambda x: x[3])
    for f in filters:
        f.process(pool[big[2]:big[2] + big[3]])
    _, _, plain_cap_span, _ = plain(False)
    plain_lat, plain_res, plain_span, plain_ff = plain(True)

    def served(paced):
        for f in filters:
            f.clear_ff()
        torch.cuda.synchronize()
        srv = Server(local, arena_bytes=16 << 30, slots=64)
        sids = [srv.add_set(f) for f in filters]
        ids = [None] * len(trace)

        def submitter():
            start = time.perf_counter()
            for i, (a, si, o, z) in enumerate(trace):
                if paced:
                    wait_until(start, a)
                ids[i] = srv.submit(sids[si], pool[o:o + z])

        th = threading.Thread(target=submitter)
        th.start()
        got = {}
        while len(got) < len(trace):
            for r in srv.poll(max_results=512, wait_us=2000):
                got[r.request_id] = r
        th.join()
        st = srv.stats()
        srv.close()
        out = [got[i] for i in ids]
        span = max(r.t_done for r in out) - min(r.t_submit for r in out)
        return out, span, st, [ff_digest(f) for f in filters]

    srv_res, srv_span, srv_stats, srv_ff = served(True)
    _, sat_span, sat_stats, _ = served(False)
    lat = [r.latency for r in srv_res]
    worst = max(range(len(srv_res)), key=lambda i: srv_res[i].latency)
    w = srv_res[worst]
    breakdown = {
        "admit_wait_p99_ms": pct([r.t_admit - r.t_submit for r in srv_res], 99) * 1e3,
        "copy_and_queue_p99_ms": pct([r.t_launch - r.t_admit for r in srv_res], 99) * 1e3,
        "scan_and_collect_p99_ms": pct([r.t_done - r.t_launch for r in srv_res], 99) * 1e3,
        "worst": {"ms": w.latency * 1e3, "bytes": w.text_len, "submitted_at_s": w.t_submit,
                  "admit_wait_ms": (w.t_admit - w.t_submit) * 1e3, "copy_and_queue_ms": (w.t_launch - w.t_admit) * 1e3,
                  "scan_and_collect_ms": (w.t_done - w.t_launch) * 1e3},
    }
    exact = all(r.status == 0 and np.array_equal(r.hit_offsets, p[0]) and np.array_equal(r.line_start, p[1])
                for r, p in zip(srv_res, plain_res)) and srv_ff == plain_ff
    out = {
        "workload": f"served: {n_sets} resident sets of {int(counts.min())}-{int(counts.max())} printable "
                    f"patterns (32-64 B, LEN 32, K 5, S 2, 2^23+2^26 bits); {len(trace)} requests, Poisson "
                    f"{args.served_rate:g}/s, sizes log-normal (median 1 MiB, sigma 1.5, cap 512 MiB), "
                    f"{total / 2**30:.2f} GiB in all, slices of a 1 GiB pinned host pool",
        "requests": len(trace), "text_bytes": total, "offered_gbs": total / trace[-1][0] / 1e9,
        "served": {"p50_ms": pct(lat, 50) * 1e3, "p99_ms": pct(lat, 99) * 1e3, "gbs": total / srv_span / 1e9,
                   "batches": srv_stats["batches"], "max_batch": srv_stats["max_batch"],
                   "mean_batch": len(trace) / max(srv_stats["batches"], 1), "latency_parts": breakdown},
        "served_saturated": {"gbs": total / sat_span / 1e9, "batches": sat_stats["batches"],
                             "max_batch": sat_stats["max_batch"]},
        "plain_serial": {"p50_ms": pct(plain_lat, 50) * 1e3, "p99_ms": pct(plain_lat, 99) * 1e3,
                         "gbs": total / plain_span / 1e9, "capacity_gbs": total / plain_cap_span / 1e9},
        "served_over_plain_capacity": plain_cap_span / sat_span,
        "bit_exact_vs_plain": bool(exact),
        "setup_s": setup_s,
        "timing": "host steady clock; served latency = done - submit inside the server; plain latency = done - "
                  "arrival; every run copies each request's text from pinned host memory",
    }
    for f in filters:
        f.close()
    del host
    torch.cuda.empty_cache()
    return out


# ---- our arm --------------------------------------------------------------------------------------------
def main_ours(args):
    import torch

    import ffbf_b200
    from ffbf_b200 import Filter
    from ffbf_b200.replicas import Replicas

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    rep = Replicas.from_env("nccl", device=dev)  # N GPUs: N independent replicas, no data-path collective
    world, rank = rep.world, rep.rank
    barrier, max_over_ranks = rep.barrier, rep.max

    if args.workload == "batched":
        return main_batched(args, rep)
    if args.workload == "served":
        return main_served(args, rep)

    wl = workload(args)
    seed = rep.seed(args.seed)
    pats = wl.patterns(seed)
    host = torch.empty(wl.text_bytes, dtype=torch.uint8, pin_memory=True)
    text = host.numpy()
    wl.text(seed, pats, out=text)
    n = wl.text_bytes

    f = Filter(wl.params, device=local)
    f.add_patterns(pats)
    d_text = torch.empty(n + 64, dtype=torch.uint8, device=dev)
    d_text[:n].copy_(host, non_blocking=False)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(f.stream, device=dev)

    def step():
        f.clear_ff()
        f.process_device(d_text.data_ptr(), n)

    # a text that L2 could hold is evicted before every timed step by writing a buffer twice L2's size
    # (outside the step's events); larger texts stream through L2 on their own
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev) if n < L2_FLUSH_BYTES else None

    def evict_l2(i):
        if flush is not None:
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)

    sampler = ClockSampler(gpu_id_for(local))
    sampler.start()
    for _ in range(args.warmup):
        step()
        f.collect()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches0 = ffbf_b200.kernel_launches()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps)]
    for i in range(args.steps):
        evict_l2(i)
        ev[2 * i].record(stream)
        step()
        ev[2 * i + 1].record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    barrier()
    launches = ffbf_b200.kernel_launches() - launches0
    per_step = [ev[2 * i].elapsed_time(ev[2 * i + 1]) for i in range(args.steps)]
    # with evictions between steps only the steps themselves count
    total_ms = sum(per_step) if flush is not None else ev[0].elapsed_time(ev[-1])
    total_ms = max_over_ranks(total_ms)
    del flush
    res = f.collect()

    # end-to-end through the public API from pinned host memory: per-step host times, the median reported
    # (the host's PCIe and memory are shared with other jobs on this machine, so single steps vary)
    e2e_steps = args.e2e_steps or max(5, min(args.steps, 10))
    barrier()
    d2h = 0
    e2e_times = []
    for _ in range(e2e_steps):
        t0 = time.perf_counter()
        f.clear_ff()
        r = f.process(text)
        ids = f.filter_phrases()
        off, pid = f.verify()
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
        d2h += r.hit_offsets.size * 32 + ids.size * 8 + off.size * 12
    e2e_s = max_over_ranks(statistics.median(e2e_times))
    # the bare host-to-device copy of the same pinned text, for context: e2e cannot beat it
    d_probe = torch.empty(n, dtype=torch.uint8, device=dev)
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    copy_ms = []
    for _ in range(2):
        c0.record()
        d_probe.copy_(host[:n], non_blocking=True)
        c1.record()
        c1.synchronize()
        copy_ms.append(c0.elapsed_time(c1))
    del d_probe
    h2d_gbs = n / (min(copy_ms) * 1e-3) / 1e9
    clocks = sampler.stop()

    value = world * n * args.steps / (total_ms * 1e-3) / 1e9
    kernel_ms = statistics.mean(per_step)
    peak, peak_kind = measured_peaks()
    achieved = n / (kernel_ms * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": dict(describe(wl), parallelism=f"replicas x{world}" if world > 1 else "single GPU",
                       l2="inputs larger than L2 (text > 126 MB), no flush" if n >= L2_FLUSH_BYTES else
                       f"text smaller than L2: a {L2_FLUSH_BYTES >> 20} MiB buffer is written between timed steps "
                       "(outside the step's events)"),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "traffic": (lambda r: None if r is None else r * n)(profiled_traffic_ratio(wl.name)),
                     "traffic_source": "ncu dram bytes of a 256 MiB capture scaled to this text (profiles/)",
                     "algorithmic_bytes_per_launch": n,
                     "probe_bound": probe_bound(wl.name, achieved, clocks.get("sm_mhz"),
                                                torch.cuda.get_device_properties(dev).multi_processor_count)},
        "e2e": {"value": world * n / e2e_s / 1e9, "unit": UNIT, "h2d_bytes_per_step": n,
                "d2h_bytes_per_step": d2h // max(e2e_steps, 1),
                "api": "ffbf_scan + ffbf_prune + ffbf_verify from pinned host memory",
                "steps": e2e_steps, "step_s": {"median": statistics.median(e2e_times), "min": min(e2e_times),
                                               "max": max(e2e_times)},
                "bare_h2d_copy_gbs": h2d_gbs},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "results": {"hits": int(res.hit_offsets.size), "lines": int(res.line_start.size),
                    "pruned_patterns": int(ids.size), "exact_matches": int(off.size)},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline_single(wl, pats, text, args.cpu_sample)
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                                    "sample": f"failed: {e}"}
    f.close()
    del d_text, host
    torch.cuda.empty_cache()
    rep.close()
    if world == 1 and args.workload == "scale":
        # the batched and served forms on their own workloads, each in a fresh process on the same GPU
        for leg, skip in (("batched", args.no_batched), ("served", args.no_served)):
            if not skip:
                line[leg] = run_leg(leg, args)
    if rank == 0:
        print(json.dumps(line))
    return 0


def run_leg(workload, args):
    """Runs `bench.py --workload <workload>` in a child process and returns its line's summary object."""
    cmd = [sys.executable, os.path.abspath(__file__), "--workload", workload, "--steps", str(args.steps),
           "--warmup", str(args.warmup), "--seed", str(args.seed)]
    p = subprocess.run(cmd, capture_output=True, text=True, env=dict(os.environ, WORLD_SIZE="1", RANK="0"))
    if p.returncode != 0:
        return {"error": f"exit {p.returncode}: {p.stderr.strip().splitlines()[-1] if p.stderr.strip() else ''}"}
    d = json.loads(p.stdout.strip().splitlines()[-1])
    return dict(d[workload], clocks=d.get("clocks"))


def main_batched(args, rep):
    """Headline line for the batched workload: value = device-timed GB/s of one batch launch."""
    world, rank, local = rep.world, rep.rank, rep.local
    sampler = ClockSampler(gpu_id_for(local))
    sampler.start()
    rep.barrier()
    r = run_batched(args, local)
    clocks = sampler.stop()
    ms = rep.max(r["ms_per_step"]["batched_device"])
    value = world * r["text_bytes"] / (ms * 1e-3) / 1e9
    achieved = r["text_bytes"] / (ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    line = {"metric": "batched vs plain GB/s", "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": r["workload"], "l2": "inputs larger than L2 (19 GiB of text), no flush",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": f"{peak_kind} hbm_gbs", "traffic": None,
                         "algorithmic_bytes_per_launch": r["text_bytes"]},
            "gpu_launches": r["launches_per_step"]["batched"] * args.steps, "clocks": clocks, "batched": r}
    rep.close()
    if rank == 0:
        print(json.dumps(line))
    return 0


def main_served(args, rep):
    """Headline line for the served workload: value = GB/s at the Poisson rate, with p50/p99 latency."""
    world, rank, local = rep.world, rep.rank, rep.local
    sampler = ClockSampler(gpu_id_for(local))
    sampler.start()
    rep.barrier()
    r = run_served(args, local)
    clocks = sampler.stop()
    line = {"metric": "served GB/s and p50/p99 latency", "value": world * r["served"]["gbs"], "unit": UNIT,
            "n_gpus": world, "steps": 1, "warmup": 0, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": r["workload"], "l2": "request texts stream from host memory",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "e2e": {"value": world * r["served"]["gbs"], "unit": UNIT, "h2d_bytes_per_step": r["text_bytes"],
                    "d2h_bytes_per_step": None},
            "clocks": clocks, "served": r}
    rep.close()
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    a = parse()
    sys.exit(main_reference(a) if a.impl == "reference" else main_ours(a))
