"""Builds libctc.so (C++ host code + sm_100a CUDA kernels) and the `tc` CLI
in-tree, with nvcc and g++ directly.

    python -m cutc_b200.build [--force]

Objects go to cutc_b200/_build/; outputs are cutc_b200/libctc.so and
cutc_b200/tc.  Rebuilds only what changed (by modification time).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libctc.so")
CLI = os.path.join(PKG, "tc")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
# the system g++ (it carries libgomp for the parallel host passes)
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-march=x86-64-v3", "-Wall",
            "-Wno-unused-function", f"-I{INCLUDE}", f"-I{CSRC}", f"-I{CUDA_HOME}/include"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           f"-I{INCLUDE}", f"-I{CSRC}", "-Xptxas", "-warn-spills"]

HOST_SOURCES = ["host.cpp"]
CUDA_SOURCES = ["engine.cu", "noalloc.cu", "fo.cu", "ciss_gpu.cu", "stage_gpu.cu"]
HEADERS = ["ctc_internal.h", "kernels.cuh", "als_tc.cuh", "ptx.cuh", "runtime.cuh", "fo.cuh", "stage_gpu.h"]


def _newer(src_list, out):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in src_list)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "ctc.h")]
    jobs = []
    objs = []
    for s in HOST_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if force or _newer([src, *hdrs], obj):
            jobs.append([CXX, *CXXFLAGS, "-c", "-o", obj, src])
    for s in CUDA_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if force or _newer([src, *hdrs], obj):
            jobs.append([NVCC, *NVFLAGS, "-c", "-o", obj, src])
    logs = []
    with ThreadPoolExecutor(max_workers=max(1, len(jobs))) as ex:
        for out in ex.map(_run, jobs):
            logs.append(out)
    if force or jobs or _newer(objs, LIB):
        _run([CXX, "-shared", "-o", LIB, *objs, f"-L{CUDA_HOME}/lib64", "-lcudart", "-fopenmp",
              "-Wl,-rpath," + f"{CUDA_HOME}/lib64"])
    cli_src = os.path.join(CSRC, "tc_main.cpp")
    if os.path.exists(cli_src) and (force or _newer([cli_src, LIB, os.path.join(INCLUDE, "ctc.h")], CLI)):
        _run([CXX, "-O2", "-std=c++17", f"-I{INCLUDE}", "-o", CLI, cli_src, f"-L{PKG}", "-lctc",
              "-Wl,-rpath,$ORIGIN"])
    text = "".join(logs)
    if verbose:
        sys.stdout.write(text)
    return text


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True) or "up to date")
