"""Build the in-tree CUDA library neo_fft_b200/libneofft_b200.so for sm_100a.

Run as ``python -m neo_fft_b200.build`` (or via __graft_entry__.build()). Host
table builders are compiled with g++ (-fno-fast-math -ffp-contract=off) and the
kernels with nvcc (--fmad=false; every float operation of the pipeline is written
with explicit round-to-nearest intrinsics).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libneofft_b200.so"

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
CXX = shutil.which("g++") or "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = [f"-I{ROOT / 'include'}", f"-I{CSRC}"]
CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-fno-fast-math", "-ffp-contract=off"]
NVCCFLAGS = ["-std=c++17", "-O3", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-fno-fast-math,-ffp-contract=off",
             "-Xptxas", "-warn-spills"] + ARCH

HOST_SOURCES = ["plan_build.cpp"]
# (source, object stem, extra defines): the tile kernel is compiled once per block shape.
SPATIAL_SHAPES = [(8, 8), (16, 16), (32, 32), (12, 12), (48, 48), (0, 0)]
CUDA_UNITS = [("nf_api.cu", "nf_api", []), ("nf_noalloc.cu", "nf_noalloc", []), ("nf_server.cu", "nf_server", [])] + \
    [("spatial_inst.cu", f"spatial_{h}x{w}", [f"-DNF_BH={h}", f"-DNF_BW={w}"]) for h, w in SPATIAL_SHAPES] + \
    [("volume_inst.cu", f"volume_{h}x{w}", [f"-DNF_BH={h}", f"-DNF_BW={w}"]) for h, w in SPATIAL_SHAPES] + \
    [("temporal_inst.cu", f"temporal_{h}x{w}", [f"-DNF_BH={h}", f"-DNF_BW={w}"]) for h, w in SPATIAL_SHAPES] + \
    [("adjoint_inst.cu", f"adjoint_{h}x{w}", [f"-DNF_BH={h}", f"-DNF_BW={w}"]) for h, w in [(16, 16), (0, 0)]]


def _run(cmd: list[str]) -> None:
    print(" ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.cuh")) + [CSRC / "launch.hpp"]
    if src.name in ("nf_api.cu", "nf_noalloc.cu", "plan_build.cpp"):  # kernel units do not see the C ABI
        deps += list(CSRC.glob("*.hpp")) + list((ROOT / "include").glob("*.h"))
    return any(d.stat().st_mtime > obj.stat().st_mtime for d in deps)


def build(force: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    objs = []
    procs = []
    for name in HOST_SOURCES:
        src, obj = CSRC / name, BUILD / (name + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            cmd = [CXX, *CXXFLAGS, *INCLUDES, "-c", src, "-o", obj]
            print(" ".join(map(str, cmd)), flush=True)
            procs.append(subprocess.Popen([str(c) for c in cmd]))
    for name, stem, defs in CUDA_UNITS:
        src, obj = CSRC / name, BUILD / (stem + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            cmd = [NVCC, *NVCCFLAGS, *defs, *INCLUDES, "-c", src, "-o", obj]
            print(" ".join(map(str, cmd)), flush=True)
            procs.append(subprocess.Popen([str(c) for c in cmd]))
    for p in procs:
        if p.wait() != 0:
            raise RuntimeError("compilation failed")
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        _run([NVCC, "-shared", *ARCH, "-cudart", "static", "-o", LIB, *objs, "-lpthread"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
