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
from the reference sources) on all host cores: the whole text, cut into one line-aligned shard per core, one
process per shard, filter loaded from a __bloom_filter_ cache; throughput = text bytes / the slowest
process's `processFile time` (the reference's own timer). A child process writes the inputs, so the arm's
own process loads none of this repository's native libraries.
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
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="bytes of text for the CPU baseline (default: 1 GiB; the whole 64 MiB plain text; 512 MiB "
                         "of the binary text; 2 GiB of the batched jobs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain leg of the default run")
    ap.add_argument("--no-binary", action="store_true", help="skip the binary leg of the default run")
    ap.add_argument("--write-reference-inputs", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--ref-shards", type=int, default=1, help=argparse.SUPPRESS)
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
def reference_binary(prm):
    import oracle
    return oracle.ref_binary(prm)


def host_cores():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def cpu_baseline_single(wl, pats, text, sample_bytes):
    """The reference binary on one core over a bounded, line-aligned prefix of the workload text, its filter
    loaded from a __bloom_filter_ cache it built itself; timed by its own processFile timer."""
    from oracle.shards import ReferenceShards, line_shards
    binary = reference_binary(wl.params)
    if binary is None:
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "unavailable: reference binary for this geometry was not built"}
    cut = line_shards(text, max(1, -(-text.size // max(1, sample_bytes))))[0][1]
    with ReferenceShards(binary, pats, text, [(0, cut)]) as ref:
        ref.prepare()
        t = ref.run(procs=1)[0]
    return {"value": cut / t / 1e9, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"{cut / 2**20:.0f} MiB line-aligned prefix of the workload text, 1 process, filter loaded "
                      f"from its __bloom_filter_ cache; processFile time {t:.3f} s"}


def write_reference_inputs(args):
    """Child process of the reference arm: writes the workload's pattern file and its text, cut into
    line-aligned shards covering all of it, under args.write_reference_inputs (the arm's own process loads
    none of this repository's native libraries)."""
    from oracle.shards import ReferenceShards, line_shards
    wl = workload(args)
    pats = wl.patterns(args.seed)
    text = wl.text(args.seed, pats)
    shards = line_shards(text, args.ref_shards)
    ReferenceShards(None, pats, text, shards, base=args.write_reference_inputs).write_shards(
        write_threads=min(16, host_cores()))
    return 0


def main_reference(args):
    """efficient/ffbf's own x86 processFile (oracle/_ref) over the whole workload text on all host cores:
    one process per core, each on a line-aligned shard, all shards together covering the text; one step =
    every shard scanned once; step time = the slowest process's `processFile time` (the reference's own
    timer). The inputs are written by a child process."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle.shards import ReferenceShards, scratch_base
    wl = workload(args)
    binary = reference_binary(wl.params)
    cfg = describe(wl)
    if binary is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference binary for this geometry not built"}))
        return 0
    nproc = max(1, min(host_cores(), 64))
    base = scratch_base(wl.text_bytes)
    try:
        cmd = [sys.executable, os.path.abspath(__file__), "--workload", args.workload, "--seed", str(args.seed),
               "--write-reference-inputs", base, "--ref-shards", str(nproc)]
        if args.text_bytes:
            cmd += ["--text-bytes", str(args.text_bytes)]
        if args.patterns:
            cmd += ["--patterns", str(args.patterns)]
        subprocess.run(cmd, check=True, env=dict(os.environ, WORLD_SIZE="1", RANK="0"))
        ref = ReferenceShards(binary, base=base).build_cache()
        total = sum(ref.shard_bytes())
        for _ in range(args.warmup):
            ref.run(procs=nproc)
        ts = [max(ref.run(procs=nproc)) for _ in range(args.steps)]
    finally:
        shutil.rmtree(base, ignore_errors=True)
    t = statistics.mean(ts)
    value = total / t / 1e9
    n = len(ref.dirs)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": n, "kind": "reference",
                             "sample": f"the whole {total / 2**30:.2f} GiB text in {n} line-aligned shards, one "
                                       f"process each on {n} host cores; filter from a __bloom_filter_ cache"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---- batched form: 512 uneven jobs in one graph launch vs plain per-job launches ------------------------
def cpu_baseline_jobs(jobs, pats, texts, sample_bytes, seed):
    """The reference binary over a seeded random sample of the batched jobs, one process per job and as
    many at a time as there are host cores (each job's filter loaded from the __bloom_filter_ cache its
    process built beforehand); aggregate = sampled text bytes / wall time of the pool."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle.shards import ReferenceShards, run_many
    order = np.random.default_rng(seed ^ 0xC0BE).permutation(len(jobs))
    pick, total = [], 0
    for j in order:
        if total >= sample_bytes:
            break
        pick.append(int(j))
        total += jobs[j].text_bytes
    binaries = {j: reference_binary(jobs[j].params) for j in pick}
    if any(b is None for b in binaries.values()):
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "unavailable: a reference binary of the batched geometry menu was not built"}
    cores = host_cores()
    refs = [ReferenceShards(binaries[j], pats[j], texts[j], [(0, jobs[j].text_bytes)]) for j in pick]
    try:
        with ThreadPoolExecutor(cores) as ex:
            list(ex.map(lambda r: r.prepare(write_threads=1), refs))
        wall = run_many(refs, cores)
    finally:
        for r in refs:
            r.close()
    return {"value": total / wall / 1e9, "unit": UNIT, "cores": min(cores, len(pick)), "kind": "reference",
            "sample": f"{len(pick)} of the {len(jobs)} jobs picked at random ({total / 2**30:.2f} GiB, "
                      f"{len({jobs[j].params.cache_bits for j in pick})} of the menu's geometries), one reference "
                      f"process per job, {cores} at a time; wall time of the pool (process start, filter load "
                      f"from its cache, processFile, filterPhrases)"}


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

    # Zero-gap schedule of lone jobs: every job scanned at the rate its configuration reaches alone on the GPU
    # (measured on the largest job of each (configuration, geometry) class), back to back with no launch or
    # host gaps. plain_serial / it is the share of per-call host and launch overhead in the plain form;
    # batched / it below 1 means packing jobs together beats even gap-free lone launches.
    def cls(f):
        t, m = f.config()
        return (t, m, f.probe_order() if m == 1 else -1, f.params.cache_bits)
    rates = {}
    for key in {cls(f) for f in filters}:
        j = max((i for i, f in enumerate(filters) if cls(f) == key), key=lambda i: jobs[i].text_bytes)
        f, w, o = filters[j], jobs[j], offs[j]
        fst = torch.cuda.ExternalStream(f.stream, device=dev)
        ms = []
        for _ in range(5):
            e0.record(fst)
            f.process_device(base + o, w.text_bytes)
            e1.record(fst)
            fst.synchronize()
            ms.append(e0.elapsed_time(e1))
        rates[key] = (w.text_bytes / (statistics.median(ms[1:]) * 1e-3), w.text_bytes)
    ideal_s = sum(w.text_bytes / rates[cls(f)][0] for f, w in zip(filters, jobs))
    ideal = {"ms": ideal_s * 1e3, "gbs": nbytes / ideal_s / 1e9,
             "batched_over_it": t_batch / ideal_s, "plain_serial_over_it": t_plain / ideal_s,
             "classes": [{"threads": k[0], "mode": k[1], "order": k[2], "cache_bits": k[3],
                          "jobs": sum(cls(f) == k for f in filters),
                          "bytes": sum(w.text_bytes for f, w in zip(filters, jobs) if cls(f) == k),
                          "gbs_alone": r / 1e9, "measured_on_bytes": n} for k, (r, n) in sorted(rates.items())],
             "how": "sum over jobs of bytes / (its class's rate on the class's largest job, alone on the GPU)"}

    cpu = None
    if not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_jobs(jobs, pats, [hv[o:o + w.text_bytes] for w, o in zip(jobs, offs)],
                                    args.cpu_sample or (2 << 30), args.seed)
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {e}"}

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
            (f"dense-{f.config()[0]}-order{f.probe_order()}" if f.config()[1] == 1 else
             f"sparse-deferred-{f.config()[0]}" if f.config()[1] == 2 else
             f"sparse-staged-{f.config()[0]}" if f.config()[1] == 3 else f"sparse-{f.config()[0]}")
            for f in filters)),
        "timing": "host clock between device-idle points, median of steps; batched_device = CUDA events",
        "lone_jobs_without_gaps": ideal,
        "cpu_baseline": cpu,
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


def cpu_baseline_requests(prm, pats, pool, trace, results, seed, n_sample=256):
    """The reference binary on a seeded random sample of the served requests (one process per request, as
    many at a time as there are host cores, each set's filter from a __bloom_filter_ cache built beforehand),
    and a spot check: each sampled request's lines as the server returned them, printed by processFile's
    rules, equal what the reference printed for that request's text."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle.shards import ReferenceShards, run_many

    from ffbf_b200 import format_spans
    binary = reference_binary(prm)
    if binary is None:
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "unavailable: reference binary for the served geometry was not built"}
    pick = np.random.default_rng(seed ^ 0x5A3F).choice(len(trace), size=min(n_sample, len(trace)), replace=False)
    by_set = collections.defaultdict(list)
    for i in sorted(int(x) for x in pick):
        by_set[trace[i][1]].append(i)
    refs = {si: ReferenceShards(binary, pats[si], pool, [(trace[i][2], trace[i][2] + trace[i][3]) for i in ids])
            for si, ids in by_set.items()}
    cores = host_cores()
    try:
        with ThreadPoolExecutor(cores) as ex:
            list(ex.map(lambda r: r.prepare(write_threads=4), refs.values()))
        wall = run_many(list(refs.values()), cores)
        mismatches = 0
        for si, ids in by_set.items():
            for k, i in enumerate(ids):
                _, _, o, z = trace[i]
                r = results[i]
                mine = format_spans(pool[o:o + z], r.line_start, r.line_end)
                mismatches += mine != refs[si].stdout(k)
    finally:
        for r in refs.values():
            r.close()
    nbytes = sum(trace[int(i)][3] for i in pick)
    return {"value": nbytes / wall / 1e9, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{len(pick)} of the {len(trace)} requests picked at random ({nbytes / 2**20:.0f} MiB), one "
                      f"reference process per request, {cores} at a time; wall time of the pool",
            "spot_check": {"requests": int(len(pick)), "stdout_equal": int(len(pick) - mismatches),
                           "against": "the reference binary's stdout for each sampled request's text"}}


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
    cpu = None
    if not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_requests(prm, pats, pool, trace, srv_res, args.seed)
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {e}"}
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
        "cpu_baseline": cpu,
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
            sample = args.cpu_sample or {"binary": 512 << 20}.get(wl.name, 1 << 30)
            line["cpu_baseline"] = cpu_baseline_single(wl, pats, text, sample)
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                                    "sample": f"failed: {e}"}
    f.close()
    del d_text, host
    torch.cuda.empty_cache()
    rep.close()
    if world == 1 and args.workload == "scale":
        # the other workloads (plain, binary) and the batched and served forms, each in a fresh process on the
        # same GPU
        for leg, skip in (("plain", args.no_plain), ("binary", args.no_binary), ("batched", args.no_batched),
                          ("served", args.no_served)):
            if not skip:
                line[leg] = run_leg(leg, args)
    if rank == 0:
        print(json.dumps(line))
    return 0


LEG_KEYS = ("metric", "value", "unit", "ms_per_step", "config", "roofline", "e2e", "cpu_baseline", "gpu_launches",
            "clocks", "results")


def run_leg(workload, args):
    """Runs `bench.py --workload <workload>` in a child process and returns its line's summary object: the
    batched/served object, or the headline keys of a plain/binary line."""
    cmd = [sys.executable, os.path.abspath(__file__), "--workload", workload, "--steps", str(args.steps),
           "--warmup", str(args.warmup), "--seed", str(args.seed)]
    if args.no_cpu_baseline:
        cmd.append("--no-cpu-baseline")
    p = subprocess.run(cmd, capture_output=True, text=True, env=dict(os.environ, WORLD_SIZE="1", RANK="0"))
    if p.returncode != 0:
        return {"error": f"exit {p.returncode}: {p.stderr.strip().splitlines()[-1] if p.stderr.strip() else ''}"}
    d = json.loads(p.stdout.strip().splitlines()[-1])
    if workload in d:
        return dict(d[workload], clocks=d.get("clocks"))
    return {k: d[k] for k in LEG_KEYS if k in d}


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
    if a.write_reference_inputs:
        sys.exit(write_reference_inputs(a))
    sys.exit(main_reference(a) if a.impl == "reference" else main_ours(a))
