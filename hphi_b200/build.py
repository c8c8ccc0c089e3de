"""Build recipe for the CUDA engine (libhphi_b200.so and the HPhi_b200 executable).

Compiles every source in hphi_b200/csrc with nvcc for sm_100a into the package
directory, so the shared library travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libhphi_b200.so")
EXE = os.path.join(HERE, "HPhi_b200")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall", "-Wno-deprecated-gpu-targets",
              "--expt-relaxed-constexpr"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith((".cu", ".cpp")) and f != "main.cpp")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh"))]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "hphi_b200.h"))
    nvcc = _nvcc()
    if force or _stale(LIB, deps):
        objdir = os.path.join(HERE, "_build")
        os.makedirs(objdir, exist_ok=True)
        objs = []
        for src in sources():
            obj = os.path.join(objdir, os.path.basename(src) + ".o")
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-c", src, "-o", obj]
            if src.endswith(".cpp"):
                cmd = [nvcc, *NVCC_FLAGS, "-x", "c++", "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
            objs.append(obj)
        tmp = LIB + ".tmp"
        subprocess.run([nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], check=True)
        os.replace(tmp, LIB)
    main = os.path.join(CSRC, "main.cpp")
    if force or _stale(EXE, [main, LIB]):
        subprocess.run([nvcc, "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets", "-o", EXE, main, "-L" + HERE, "-lhphi_b200",
                        "-Xlinker", "-rpath=$ORIGIN"], check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
