"""Builds libchy_pot3.so in-tree for sm_100a (B200).

    python -m chymera_uo_b200.build [--force] [--verbose]

Objects go to chymera_uo_b200/_build/, the library to
chymera_uo_b200/libchy_pot3.so, the ITYPE=71 driver to
chymera_uo_b200/chy_itype71.  Transform and boundary kernels are compiled
with --fmad=false (their products and sums must round like the reference's);
host code with -ffp-contract=off for the same reason.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libchy_pot3.so")
CLI = os.path.join(HERE, "chy_itype71")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
                      "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
                      "-I" + INC, "-I" + CSRC]
NOFMA = {"k_fft.cu", "k_bdy.cu", "k_source.cu", "k_blktri.cu"}
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
             "-I" + INC, "-I" + CSRC]


def nvcc() -> str:
    for cand in (os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc"),
                 shutil.which("nvcc") or ""):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INC, "*.h"))


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd[:3]) + " ... " + cmd[-1])
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = _headers()
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp"))):
        name = os.path.basename(src)
        obj = os.path.join(BUILD, name + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [src] + hdrs + [__file__]):
            continue
        if name.endswith(".cu"):
            cmd = [nvcc()] + NVCC_COMMON + (["--fmad=false"] if name in NOFMA else []) + \
                ["-c", src, "-o", obj]
        else:
            cmd = ["g++"] + CXX_FLAGS + ["-c", src, "-o", obj]
        _run(cmd, verbose)
    if force or _stale(LIB, objs):
        _run([nvcc()] + ARCH + ["-shared", "-o", LIB] + objs, verbose)
    # the ITYPE=71 driver, linked against the library next to it
    cli_src = os.path.join(CSRC, "cli", "itype71.cpp")
    if force or _stale(CLI, [cli_src, LIB] + hdrs):
        _run(["g++"] + CXX_FLAGS + [cli_src, "-o", CLI, "-L" + HERE, "-lchy_pot3", "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
