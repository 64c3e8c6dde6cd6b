"""Builds the CUDA library ``librbmpp.so`` in-tree for sm_100a (B200)."""
from __future__ import annotations

import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "librbmpp.so")
SOURCES = ["capi.cu", "sampler.cu", "sampler_stream.cu", "estimator.cu", "correlation.cu", "linalg.cu", "sr_solve.cu", "gemm_bf16x3.cu", "skew.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-O2", "--expt-relaxed-constexpr"]


def _stale() -> bool:
    if not os.path.exists(LIB) or not os.path.exists(DRIVER) or not os.path.exists(POST):
        return True
    t = min(os.path.getmtime(LIB), os.path.getmtime(DRIVER), os.path.getmtime(POST))
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "rbmpp.h"),
                                                                DRIVER_SRC, POST_SRC]
    objdir = os.path.join(HERE, "_build")
    # a source edited while an earlier build ran leaves its object older than the source
    for s in SOURCES:
        o = os.path.join(objdir, s.replace(".cu", ".o"))
        if os.path.exists(o) and os.path.getmtime(o) < os.path.getmtime(os.path.join(CSRC, s)):
            return True
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def _headers_mtime() -> float:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(HERE, "..", "include", "rbmpp.h"))
    return max(os.path.getmtime(h) for h in hs if os.path.exists(h))


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs, cmds = [], []
    th = _headers_mtime()
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        sp = os.path.join(CSRC, src)
        # recompile a source whose object is older than it or than any shared header
        if force or extra or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(sp), th):
            cmds.append([NVCC, *FLAGS, *(extra or []), "-c", sp, "-o", obj])
        objs.append(obj)
    # one nvcc per source, run side by side (each is single-threaded)
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd), flush=True)
        list(ex.map(subprocess.check_call, cmds))
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs, "-lcuda"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    build_driver(verbose)
    return LIB


DRIVER_SRC = os.path.join(HERE, "driver", "rbmpp_driver.cpp")
DRIVER = os.path.join(HERE, "rbmpp_driver")
POST_SRC = os.path.join(HERE, "driver", "rbmpp_post_process.cpp")
POST = os.path.join(HERE, "rbmpp_post_process")


def build_driver(verbose: bool = False) -> str:
    """The C++ main.f90 host program, linked against librbmpp.so (found next to it at run time)."""
    cmd = ["g++", "-O2", "-std=c++17", "-Wall", DRIVER_SRC, "-o", DRIVER, "-L" + HERE, "-lrbmpp",
           "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    build_post_process(verbose)
    return DRIVER


def build_post_process(verbose: bool = False) -> str:
    """The host-only C++ correlation post-processing program (no GPU, no library)."""
    cmd = ["g++", "-O2", "-std=c++17", "-Wall", POST_SRC, "-o", POST]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return POST


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
