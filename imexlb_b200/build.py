"""Build the native library and the case drivers in-tree for sm_100a.

    python -m imexlb_b200.build [--verbose] [--ptxas]

Outputs (git-ignored, they travel with the working tree):
    imexlb_b200/libimexlb.so       the C ABI of include/imexlb.h
    imexlb_b200/bin/imexlb_{tgv,cavity,sphere}   drivers mirroring the
                                   reference's three main() programs

nvcc cross-compiles here without a GPU.  Host code is built with
-ffp-contract=off so the FP64 case set-up rounds every operation as written.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libimexlb.so")
BIN = os.path.join(HERE, "bin")

SOURCES = ["kernels.cu", "lattice.cu", "ghost_plan.cpp", "noalloc.cu", "engine.cu"]
APPS = ["tgv", "cavity", "sphere"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
          "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps() -> list[str]:
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".cpp", ".h"))]
    out.append(os.path.join(ROOT, "include", "imexlb.h"))
    return out


def build(verbose: bool = False, ptxas: bool = False, force: bool = False) -> str:
    deps = _deps()
    cc = nvcc()
    if force or _stale(LIB, deps):
        cmd = [cc, *COMMON, *ARCH, "-shared", "-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES]
        if ptxas:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    os.makedirs(BIN, exist_ok=True)
    for app in APPS:
        src = os.path.join(CSRC, "apps", f"{app}_main.cpp")
        exe = os.path.join(BIN, f"imexlb_{app}")
        if not os.path.exists(src):
            continue
        if force or _stale(exe, [src, LIB, os.path.join(CSRC, "apps", "driver.h")]):
            cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")
            cmd = [cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-o", exe, src,
                   "-L", HERE, "-limexlb", "-Wl,-rpath,$ORIGIN/.."]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, ptxas="--ptxas" in sys.argv, force=True)
    print(LIB)
