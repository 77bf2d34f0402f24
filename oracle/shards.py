"""TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.

efficient/ffbf's own binary (oracle/_ref) and the C restatement (oracle/ffbf_oracle.c) run over line-aligned
shards of one text, in parallel on the host cores, so that texts of many GiB can be checked in minutes.

Why shards give the whole text's answer:
  * processFile (src/rabin-karp/ffbf.cpp:310-392) resets its hash at every '\\n', so a window never spans a
    line break; a shard that starts just after a '\\n' and ends just after one holds every window of its
    lines. The hit windows, flagged lines and feed-forward bits of the whole text are therefore the union
    of the shards' (offsets moved by the shard's start), and the feed-forward array is the OR of theirs.
  * filterPhrases (:394-485) reads only the feed-forward array and the pattern file, so one more reference
    run over an empty text, whose feed-forward half starts as that OR (FFBF_REF_FF_IN in ref_harness.cpp),
    prints the pruned file and index the single run would.
  * stdout is the one output that depends on the cut: lines are printed as C strings per 512 KiB read()
    chunk (:344-354, :372-382), so a line with a NUL prints differently where a chunk boundary falls inside
    it. Each shard's stdout is therefore compared with the flagged lines of that shard formatted on that
    shard's own chunk grid.

Shard processes load the filter from a `__bloom_filter_` cache that one reference run builds first.
"""
import os
import shutil
import subprocess
import tempfile
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np


def host_cores():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def line_shards(text, n_shards):
    """[a, b) pieces covering all of `text`: cut points near i * size / n moved to just after the next '\\n'
    (a piece with no '\\n' after its nominal end runs to the end of the text). Empty pieces are dropped."""
    size = int(text.size)
    cuts = [0]
    for i in range(1, n_shards):
        c = max(i * size // n_shards, cuts[-1])
        step = 1 << 16
        while c < size:
            nl = np.flatnonzero(text[c:c + step] == 10)
            if nl.size:
                c += int(nl[0]) + 1
                break
            c += step
            step *= 2
        cuts.append(min(c, size))
    cuts.append(size)
    return [(a, b) for a, b in zip(cuts[:-1], cuts[1:]) if b > a]


def scratch_base(need_bytes=0):
    """A scratch directory in /dev/shm when it has room for `need_bytes` (plus a quarter), else in TMPDIR."""
    shm = "/dev/shm"
    use_shm = os.path.isdir(shm) and shutil.disk_usage(shm).free > need_bytes * 1.25 + (64 << 20)
    return tempfile.mkdtemp(prefix="ffbf_shards_", dir=shm if use_shm else None)


def _run(binary, cwd, stdin_path, env_extra=None):
    env = dict(os.environ)
    env.pop("FFBF_REF_DUMP", None)
    env.pop("FFBF_REF_FF_IN", None)
    env.update(env_extra or {})
    with open(stdin_path, "rb") as fin, open(os.path.join(cwd, "stdout"), "wb") as fout:
        p = subprocess.run([binary, "pats", "out"], stdin=fin, stdout=fout, stderr=subprocess.PIPE, cwd=cwd, env=env)
    err = p.stderr.decode(errors="replace")
    if p.returncode != 0:
        raise RuntimeError(f"reference exited {p.returncode} in {cwd}: {err}")
    t = [float(x.split(":")[1]) for x in err.splitlines() if x.startswith("processFile time:")]
    return t[0] if t else None


class ReferenceShards:
    """The reference binary for one geometry over line-aligned shards of one text.

    Made from the inputs (`patterns`, `text`, `shards`): the constructor writes the pattern file, and
    write_shards() one directory per shard with its text. Attached to a directory another process wrote
    that way (`patterns` None, `base` given): nothing is written. build_cache() then builds the
    `__bloom_filter_` cache (one reference run over an empty text, which also dumps the main bit array) and
    links it into every shard directory; run() scans every shard, at most `procs` processes at a time.
    """

    def __init__(self, binary, patterns=None, text=None, shards=None, base=None):
        self.binary = binary
        self.text = text
        self.shards = shards
        self.own_base = base is None
        self.base = base or scratch_base(int(text.size))
        self.seed = os.path.join(self.base, "seed")
        self.empty = os.path.join(self.seed, "empty")
        if patterns is not None:
            os.makedirs(self.seed, exist_ok=True)
            with open(os.path.join(self.seed, "pats"), "wb") as f:
                f.write(np.asarray(patterns, dtype=np.uint8).tobytes())
            open(self.empty, "wb").close()
            self.dirs = [os.path.join(self.base, f"s{i}") for i in range(len(shards))]
        else:
            n = 0
            while os.path.isdir(os.path.join(self.base, f"s{n}")):
                n += 1
            self.dirs = [os.path.join(self.base, f"s{i}") for i in range(n)]

    def write_shards(self, write_threads=8):
        def one(i):
            a, b = self.shards[i]
            d = self.dirs[i]
            os.makedirs(d, exist_ok=True)
            self.text[a:b].tofile(os.path.join(d, "text"))

        with ThreadPoolExecutor(max(1, write_threads)) as ex:
            list(ex.map(one, range(len(self.shards))))
        return self

    def shard_bytes(self):
        return [os.path.getsize(os.path.join(d, "text")) for d in self.dirs]

    def build_cache(self):
        dump = os.path.join(self.seed, "dump.bin")
        _run(self.binary, self.seed, self.empty, {"FFBF_REF_DUMP": dump})
        raw = np.fromfile(dump, dtype=np.uint8)
        self.nbytes = raw.size // 2
        self.main = raw[:self.nbytes].copy()
        os.unlink(dump)
        with open(os.path.join(self.seed, "__bloom_filter_pats"), "rb") as f:
            self.bloom = f.read()
        for d in self.dirs:
            for fn in ("pats", "__bloom_filter_pats"):
                if not os.path.exists(os.path.join(d, fn)):
                    os.link(os.path.join(self.seed, fn), os.path.join(d, fn))
        return self

    def prepare(self, write_threads=8):
        self.write_shards(write_threads)
        return self.build_cache()

    def run(self, procs=None, dump_ff=False):
        """Scans every shard. Returns [processFile seconds] per shard; with dump_ff also keeps each shard's
        feed-forward array (read back by ff_or())."""
        procs = procs or host_cores()

        def one(d):
            env = {"FFBF_REF_DUMP": os.path.join(d, "dump.bin")} if dump_ff else {}
            return _run(self.binary, d, os.path.join(d, "text"), env)

        with ThreadPoolExecutor(max(1, procs)) as ex:
            return list(ex.map(one, self.dirs))

    def stdout(self, i):
        with open(os.path.join(self.dirs[i], "stdout"), "rb") as f:
            return f.read()

    def ff_or(self):
        """OR of the shards' feed-forward arrays (reference byte layout)."""
        acc = np.zeros(self.nbytes, dtype=np.uint8)
        for d in self.dirs:
            raw = np.fromfile(os.path.join(d, "dump.bin"), dtype=np.uint8)
            np.bitwise_or(acc, raw[self.nbytes:], out=acc)
        return acc

    def prune_with_ff(self, ff):
        """filterPhrases over the given feed-forward array: (pruned file, __index_ file) bytes."""
        d = os.path.join(self.base, "prune")
        os.makedirs(d, exist_ok=True)
        for fn in ("pats", "__bloom_filter_pats"):
            if not os.path.exists(os.path.join(d, fn)):
                os.link(os.path.join(self.seed, fn), os.path.join(d, fn))
        ff_path = os.path.join(d, "ff_in.bin")
        np.ascontiguousarray(ff, dtype=np.uint8).tofile(ff_path)
        _run(self.binary, d, self.empty, {"FFBF_REF_FF_IN": ff_path})
        with open(os.path.join(d, "out"), "rb") as f:
            pruned = f.read()
        with open(os.path.join(d, "__index_out"), "rb") as f:
            index = f.read()
        return pruned, index

    def close(self):
        if self.own_base:
            shutil.rmtree(self.base, ignore_errors=True)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def run_many(refs, procs=None):
    """Scans every shard of several ReferenceShards (their caches built) in one pool of `procs` processes at a
    time. Returns the pool's wall time in seconds."""
    jobs = [(r.binary, d) for r in refs for d in r.dirs]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max(1, procs or host_cores())) as ex:
        list(ex.map(lambda bd: _run(bd[0], bd[1], os.path.join(bd[1], "text")), jobs))
    return time.perf_counter() - t0


def oracle_scan_shards(prm, main, text, shards, threads=None):
    """The C restatement's processFile over each shard in its own thread (the library releases the GIL).

    Returns (hit offsets, line starts, line ends) of the whole text, ascending, and the OR of the shards'
    feed-forward arrays."""
    from . import Oracle

    def one(ab):
        a, b = ab
        o = Oracle.from_params(prm)
        o.main[:] = main
        s = o.scan(text[a:b])
        return s["hits"] + np.uint64(a), s["line_start"] + np.uint64(a), s["line_end"] + np.uint64(a), o.ff

    with ThreadPoolExecutor(max(1, threads or host_cores())) as ex:
        parts = list(ex.map(one, shards))
    ff = parts[0][3].copy()
    for p in parts[1:]:
        np.bitwise_or(ff, p[3], out=ff)
    cat = lambda i: np.concatenate([p[i] for p in parts]) if parts else np.zeros(0, np.uint64)  # noqa: E731
    return cat(0), cat(1), cat(2), ff
