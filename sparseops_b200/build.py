"""Build the in-tree native libraries.

    python -m sparseops_b200.build          # both libraries
    python -m sparseops_b200.build --check  # also print ptxas register/spill lines

libsparseops_b200.so  every csrc/*.cu and csrc/*.cpp except synth.cpp, compiled
                      by nvcc for sm_100a only (-gencode arch=compute_100a,
                      code=sm_100a), linked against the CUDA runtime.
libsparseops_synth.so csrc/synth.cpp, host C++ (seeded workload generators).

Objects go to _build/ (git-ignored); the .so files land in the package
directory so they travel with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(ROOT, "_build", "obj")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-ccbin", HOST_CXX, "-I" + os.path.join(ROOT, "include")] + ARCH
LIB = os.path.join(PKG, "libsparseops_b200.so")
SYNTH = os.path.join(PKG, "libsparseops_synth.so")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers() -> list[str]:
    return (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(ROOT, "include", "*.h")))


def _compile(src: str, verbose_ptxas: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if not _stale(obj, [src] + _headers()) and not verbose_ptxas:
        return obj
    cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
    if verbose_ptxas and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas:
        sys.stderr.write(r.stderr)
    return obj


def build_lib(verbose_ptxas: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) +
                  [s for s in glob.glob(os.path.join(CSRC, "*.cpp")) if not s.endswith("synth.cpp")])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    if _stale(LIB, objs):
        cmd = [NVCC, "-shared", "-o", LIB] + ARCH + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def build_synth() -> str:
    src = os.path.join(CSRC, "synth.cpp")
    if _stale(SYNTH, [src]):
        subprocess.run([HOST_CXX, "-O3", "-std=c++17", "-shared", "-fPIC", "-pthread", "-o", SYNTH, src], check=True)
    return SYNTH


def build(verbose_ptxas: bool = False) -> None:
    if not os.path.exists(NVCC) and shutil.which("nvcc") is None:
        raise RuntimeError("nvcc not found: set CUDA_HOME")
    build_synth()
    build_lib(verbose_ptxas)


if __name__ == "__main__":
    build(verbose_ptxas="--check" in sys.argv)
    print(LIB)
