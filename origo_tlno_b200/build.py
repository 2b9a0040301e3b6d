"""Builds the in-tree native library origo_tlno_b200/_lib/libtlno_gpu.so.

CUDA code is compiled for sm_100a only (`-gencode arch=compute_100a,
code=sm_100a`); host C++ with g++.  Objects go to origo_tlno_b200/_build/
(git-ignored); the .so is written in-tree so it travels with the source.
Usage: python -m origo_tlno_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libtlno_gpu.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["kernels.cu", "noalloc.cu"]
def _fast_count():
    """Number of compile-time ERI classes (TLNO_FAST_COUNT in csrc/fast_classes.hpp)."""
    import re
    text = open(os.path.join(CSRC, "fast_classes.hpp")).read()
    return int(re.search(r"#define TLNO_FAST_COUNT (\d+)", text).group(1))


FAST_COUNT = _fast_count()
CPP_SOURCES = ["tables.cpp", "basis.cpp", "plan.cpp", "capi.cpp", "incremental.cpp"]


def _deps(src, seen=None):
    """The source file plus every local header it includes (recursively)."""
    import re
    seen = set() if seen is None else seen
    if src in seen or not os.path.exists(src):
        return seen
    seen.add(src)
    with open(src) as f:
        for m in re.finditer(r'^\s*#\s*include\s+"([^"]+)"', f.read(), re.M):
            _deps(os.path.normpath(os.path.join(os.path.dirname(src), m.group(1))), seen)
    return seen


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, list(_deps(s))):
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "--expt-relaxed-constexpr", "-c", s, "-o", o]
            if ptxas_verbose:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    inst = os.path.join(CSRC, "eri_fast_inst.cu")
    for fid in range(FAST_COUNT):
        o = os.path.join(BUILD, f"eri_fast_{fid}.o")
        objs.append(o)
        if force or _stale(o, list(_deps(inst))):
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "--expt-relaxed-constexpr", f"-DTLNO_FAST_ID={fid}", "-c", inst, "-o", o]
            if ptxas_verbose:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, list(_deps(s))):
            jobs.append(["g++", "-O2", "-std=c++17", "-fPIC", "-pthread", "-I" + os.path.join(CUDA_HOME, "include"),
                         "-c", s, "-o", o])
    out = ""
    with ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        for r in ex.map(lambda c: _run(c, verbose), jobs):
            out += r
    if force or jobs or not os.path.exists(LIB):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lpthread"], verbose)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v register/spill report")
    a = ap.parse_args(argv)
    out = build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas)
    if a.ptxas:
        print(out)
    print(LIB)


if __name__ == "__main__":
    sys.exit(main())
