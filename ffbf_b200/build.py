"""Builds the native parts of ffbf_b200 in-tree.

Outputs (all under ffbf_b200/_lib/, git-ignored, shipped beside the sources):
  libffbf.so          the C-ABI library (include/ffbf.h): host C++ plus the sm_100a kernels
  ffbf                the drop-in CLI (same argv and files as efficient/ffbf's `ffbf`)
  libffbf_datagen.so  the seeded synthetic-data generator used by tests and bench.py

Every CUDA source is compiled for sm_100a only: -gencode arch=compute_100a,code=sm_100a.
Run: python -m ffbf_b200.build [--force]
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
OBJ = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
                  f"-I{os.path.join(ROOT, 'include')}"]

CUDA_SOURCES = ["ffbf_kernels.cu", "ffbf_scan_fast.cu", "ffbf_capi.cu", "ffbf_batch.cu", "ffbf_serve.cu", "ffbf_static.cu", "ffbf_hashbench.cu", "ffbf_order.cu"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    return hs


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed: " + " ".join(cmd) + "\n" + r.stdout)
    return r.stdout


def build(force=False, verbose=False):
    os.makedirs(OUT, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    hdrs = _headers()
    objs = []
    jobs = []
    for src in CUDA_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            jobs.append([NVCC] + NVFLAGS + ["-c", s, "-o", o])
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    lib = os.path.join(OUT, "libffbf.so")
    if force or _newer(lib, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart=static", "-Xcompiler", "-pthread", "-o", lib + ".tmp"] + objs)
        os.replace(lib + ".tmp", lib)
    cli_src = os.path.join(CSRC, "ffbf_cli.cpp")
    cli = os.path.join(OUT, "ffbf")
    if os.path.exists(cli_src) and (force or _newer(cli, [cli_src, lib] + hdrs)):
        _run(["g++", "-std=c++17", "-O2", "-Wall", f"-I{os.path.join(ROOT, 'include')}", cli_src, "-o", cli + ".tmp",
              f"-L{OUT}", "-lffbf", "-Wl,-rpath,$ORIGIN"])
        os.replace(cli + ".tmp", cli)
    hb_src = os.path.join(CSRC, "hashbench_cli.cpp")
    hb = os.path.join(OUT, "hashbench")
    if os.path.exists(hb_src) and (force or _newer(hb, [hb_src, lib] + hdrs)):
        _run(["g++", "-std=c++17", "-O2", "-Wall", f"-I{os.path.join(ROOT, 'include')}", hb_src, "-o", hb + ".tmp",
              f"-L{OUT}", "-lffbf", "-Wl,-rpath,$ORIGIN"])
        os.replace(hb + ".tmp", hb)
    gen_src = os.path.join(CSRC, "datagen.c")
    gen = os.path.join(OUT, "libffbf_datagen.so")
    if force or _newer(gen, [gen_src]):
        _run(["gcc", "-std=c11", "-O2", "-fPIC", "-shared", "-pthread", gen_src, "-o", gen + ".tmp"])
        os.replace(gen + ".tmp", gen)
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print("built", OUT)
