#!/usr/bin/env python3
"""Build the B200 engine in-tree: lib/libcuckoo_b200.so (C ABI of include/cuckoo_b200.h) and
bin/cuckoo_fast_b200 (the CLI).  Every kernel is compiled for sm_100a only.

    python cuckoo-failure_b200/build.py [--force] [-j N]

Translation units compile in parallel; a unit is rebuilt when any source under csrc/ or the
public header is newer than its object.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "lib", "libcuckoo_b200.so")
CLI = os.path.join(PKG, "bin", "cuckoo_fast_b200")
PROBE = os.path.join(PKG, "lib", "libcuckoo_b200_probe.so")
PROBE_SRC = os.path.join(PKG, "probe", "imad_peak.cu")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v"]
# Per-unit assembler options.  The L = 2^14 kernel runs 1024 threads, so it has 64 registers per
# thread; at the default level ptxas schedules its transform passes far past that budget (frames
# above 800 bytes), while -O1 keeps the 50-bit kernel to a 152-byte frame and the 62-bit one to
# 320 bytes (the cluster kernel with 1024 threads of 8 entries: 56 bytes).  The L = 2^10 kernel is compiled for 16 CTAs per SM (MinBlocks in kernel_lg.cuh), also
# 128 registers: -O1 keeps it to a 208-byte frame where the default level spills 1.4 KB.  The other
# kernels have up to 255 registers and spill at neither level.
UNIT_FLAGS = {"k_lg14.cu": ["-Xptxas", "-O1"], "k_lg10.cu": ["-Xptxas", "-O1"], "k_lg15_c4e8.cu": ["-Xptxas", "-O1"],
              "k_lg14_tune.cu": ["-Xptxas", "-O1"], "k_lg10_tune.cu": ["-Xptxas", "-O1"]}


def newest_dep():
    deps = glob.glob(os.path.join(CSRC, "*")) + [os.path.join(ROOT, "include", "cuckoo_b200.h"), __file__]
    return max(os.path.getmtime(p) for p in deps)


def compile_unit(src, force, dep_time):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= dep_time:
        return obj, ""
    cmd = [NVCC] + NVFLAGS + UNIT_FLAGS.get(os.path.basename(src), []) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force=False, jobs=None, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    dep_time = newest_dep()
    units = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    jobs = jobs or max(1, min(len(units), os.cpu_count() or 4))
    with cf.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: compile_unit(s, force, dep_time), units))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            for line in log.splitlines():
                if "registers" in line or "spill" in line or "Compiling" in line:
                    print(line)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        subprocess.run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs, check=True)
    if force or not os.path.exists(CLI) or os.path.getmtime(CLI) < max(os.path.getmtime(LIB), dep_time):
        subprocess.run(["g++", "-O2", "-std=c++17", os.path.join(CSRC, "cuckoo_fast_main.cpp"), "-o", CLI,
                        "-L" + os.path.dirname(LIB), "-lcuckoo_b200", "-Wl,-rpath,$ORIGIN/../lib"], check=True)
    if force or not os.path.exists(PROBE) or os.path.getmtime(PROBE) < os.path.getmtime(PROBE_SRC):
        subprocess.run([NVCC] + ARCH + ["-O3", "-Xcompiler", "-fPIC", "-shared", PROBE_SRC, "-o", PROBE], check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.j, a.v))
    sys.exit(0)
