"""Builds libphoton_cuda.so in place (sm_100a only).

The host scene builder is compiled with g++ and the kernels with nvcc; both without FMA
contraction so the traversal and hit-record arithmetic round exactly like the reference CPU
path.  Re-running is cheap: objects are rebuilt only when a source or header changed.
"""
from __future__ import annotations

import os
import pathlib
import shutil
import subprocess

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
OBJ = HERE / "_build"
LIB = HERE / "libphoton_cuda.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libphoton_cuda.so")
    return cand


def _deps() -> list[pathlib.Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "photon_cuda.h"]


def _stale(target: pathlib.Path, sources: list[pathlib.Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"build step failed ({res.returncode}):\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")


def build(verbose: bool = False) -> pathlib.Path:
    OBJ.mkdir(exist_ok=True)
    deps = _deps()
    inc = [f"-I{INCLUDE}", f"-I{CSRC}"]
    objs = []
    host_src = CSRC / "pe_host.cpp"
    host_obj = OBJ / "pe_host.o"
    if _stale(host_obj, [host_src] + deps):
        _run(["g++", *CXX_FLAGS, *inc, "-c", str(host_src), "-o", str(host_obj)], verbose)
    objs.append(host_obj)
    nvcc = _nvcc()
    for cu in sorted(CSRC.glob("*.cu")):
        o = OBJ / (cu.stem + ".o")
        if _stale(o, [cu] + deps):
            _run([nvcc, *ARCH, *NVCC_FLAGS, *inc, "-c", str(cu), "-o", str(o)], verbose)
        objs.append(o)
    if _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart_static", "-lrt", "-ldl", "-lpthread"],
             verbose)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
