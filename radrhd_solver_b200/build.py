"""Builds radrhd_solver_b200/librrhd.so for sm_100a with nvcc.

Usage: python -m radrhd_solver_b200.build [--force] [-j N]

The FP64 translation units are compiled with --fmad=false so that each
floating-point operation is rounded once, as in the reference's CPU code; the
tensor-core and learned-guess units keep FMA contraction.  Objects go to
radrhd_solver_b200/_build/, the shared library next to this file.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "librrhd.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"),
          "-I", CSRC, "--expt-relaxed-constexpr"]

# source -> extra flags
SOURCES = {
    "mesh.cpp": [],
    "partition.cpp": [],
    "hydro.cu": ["--fmad=false"],
    "radiation_fp64.cu": ["--fmad=false"],
    "scatter_tc.cu": [],
    "scatter_lowrank.cu": [],
    "synth.cu": [],
    "c2p_mlp.cu": ["--fmad=false"],
    "sweep.cu": ["--fmad=false"],
    "compton.cu": [],
    "raytrace.cu": ["--fmad=false"],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src: str, flags: list[str]) -> str:
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "rrhd.h"))
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps if os.path.exists(d)):
        return obj
    cmd = [nvcc()] + ARCH + COMMON + flags + ["-c", path, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [nvcc()] + COMMON + flags + ["-x", "c++", "-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int = 8, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda kv: _compile(*kv), SOURCES.items()))
    if os.path.exists(LIB) and not force and all(os.path.getmtime(LIB) >= os.path.getmtime(o) for o in objs):
        return LIB
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcuda"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    a = ap.parse_args()
    try:
        build(a.force, a.j, verbose=True)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
