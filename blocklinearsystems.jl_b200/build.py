"""Build libblsgpu.so (sm_100a kernels + C ABI) and libblsscene.so (scene generator) in-tree.

    python blocklinearsystems.jl_b200/build.py [--force] [--ptxas-verbose]

The shared objects land next to this file, so they travel with the source tree; objects go to _build/.
CUDA code is compiled for sm_100a only (-gencode arch=compute_100a,code=sm_100a), with the CUDA runtime linked
statically. Host C++ is compiled with the system g++ (the image's /opt/gcc toolchain lacks the OpenMP runtime spec).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
INCLUDE = HERE.parent / "include"

GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-fopenmp",
              "-ccbin", "g++"] + GENCODE
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-Wno-unknown-pragmas"]

GPU_SOURCES = ["schur.cu", "noalloc.cu", "qr.cu", "pcg.cu", "gnn.cu", "conditioning.cu", "dense.cu", "capi.cpp", "host_layout.cpp"]
SCENE_SOURCES = ["scene.cpp"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libblsgpu")


def _cuda_include() -> str:
    return str(Path(_nvcc()).resolve().parent.parent / "include")


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.hpp")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0 or (verbose and (r.stdout or r.stderr)):
        sys.stdout.write(r.stdout)
        sys.stderr.write(r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}")


def _compile(src: Path, force: bool, verbose: bool, ptxas_verbose: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if force or _stale(obj, [src] + _headers()):
        if src.suffix == ".cu":
            cmd = [_nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_verbose else []) + ["-c", str(src), "-o", str(obj)]
        else:
            cmd = ["g++"] + CXX_FLAGS + ["-I", _cuda_include(), "-c", str(src), "-o", str(obj)]
        _run(cmd, verbose or ptxas_verbose)
    return obj


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> dict[str, Path]:
    BUILD.mkdir(exist_ok=True)
    gpu_objs = [_compile(CSRC / s, force, verbose, ptxas_verbose) for s in GPU_SOURCES]
    lib = HERE / "libblsgpu.so"
    if force or _stale(lib, gpu_objs):
        _run([_nvcc(), "-shared", "-o", str(lib)] + GENCODE + gpu_objs_str(gpu_objs) +
             ["-Xcompiler", "-fopenmp", "-lgomp"], verbose)
    scene_objs = [_compile(CSRC / s, force, verbose, False) for s in SCENE_SOURCES]
    scene = HERE / "libblsscene.so"
    if force or _stale(scene, scene_objs):
        _run(["g++", "-shared", "-fopenmp", "-o", str(scene)] + gpu_objs_str(scene_objs), verbose)
    return {"libblsgpu": lib, "libblsscene": scene}


def gpu_objs_str(objs: list[Path]) -> list[str]:
    return [str(o) for o in objs]


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    out = build(a.force, a.verbose, a.ptxas_verbose)
    for k, v in out.items():
        print(k, v)
