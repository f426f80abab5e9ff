"""Builds the in-tree shared library math_b200/libntrace.so (C ABI: include/ntrace.h).

The CUDA kernels are compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``) with
``-fmad=false`` so that every fused multiply-add is an explicit one, and the host code with
``-ffp-contract=off`` so that its float arithmetic follows the reference's operation order (the tree
built here is the tree the reference's Mesh<N,float> builds).  The CUDA runtime is linked statically,
so the library only needs the driver at run time.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
INCLUDE = ROOT / "include"
LIB = HERE / "libntrace.so"
BUILD_DIR = ROOT / "_build" / "ntrace"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    nvcc = Path(cuda_home) / "bin" / "nvcc"
    if nvcc.exists():
        return str(nvcc)
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build ntrace")
    return found


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("command failed: " + " ".join(cmd))


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compiles libntrace.so if any source is newer than it; returns its path."""
    nvcc = _nvcc()
    headers = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.hpp")) + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "ntrace.h"]
    cu = CSRC / "kernels.cu"
    cpp = CSRC / "scene.cpp"
    BUILD_DIR.mkdir(parents=True, exist_ok=True)
    cu_obj = BUILD_DIR / "kernels.o"
    cpp_obj = BUILD_DIR / "scene.o"
    # NTRACE_DEFINES: extra -D options for the kernels (build-time tuning, e.g. -DNT_WALK_MIN_BLOCKS=3)
    common = ["-std=c++17", "-I", str(INCLUDE), "-I", str(CSRC)] + os.environ.get("NTRACE_DEFINES", "").split()
    if force or _stale(cu_obj, [cu] + headers):
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off", *common,
               "-c", str(cu), "-o", str(cu_obj)]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    if force or _stale(cpp_obj, [cpp] + headers):
        cmd = [nvcc, "-x", "c++", "-Wno-deprecated-gpu-targets", "-O2", "-Xcompiler", "-fPIC,-ffp-contract=off,-pthread", *common, "-c", str(cpp),
               "-o", str(cpp_obj)]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    noalloc = CSRC / "noalloc.cu"
    noalloc_obj = BUILD_DIR / "noalloc.o"
    if force or _stale(noalloc_obj, [noalloc] + headers):
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-Xcompiler", "-fPIC", *common, "-c", str(noalloc), "-o",
               str(noalloc_obj)]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    probes = CSRC / "probes.cu"
    probes_obj = BUILD_DIR / "probes.o"
    if force or _stale(probes_obj, [probes, INCLUDE / "ntrace.h"]):
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-Xcompiler", "-fPIC", *common, "-c", str(probes), "-o", str(probes_obj)]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    denoise = CSRC / "denoise.cu"
    denoise_obj = BUILD_DIR / "denoise.o"
    if force or _stale(denoise_obj, [denoise] + headers + [INCLUDE / "ntrace_denoise.h"]):
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-Xcompiler", "-fPIC", *common, "-c", str(denoise), "-o",
               str(denoise_obj)]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    tree = CSRC / "treebuild.cu"
    tree_obj = BUILD_DIR / "treebuild.o"
    if force or _stale(tree_obj, [tree] + headers):
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-fmad=false", "--expt-relaxed-constexpr", "-Xcompiler",
               "-fPIC,-ffp-contract=off", *common, "-c", str(tree), "-o", str(tree_obj)]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    hull = CSRC / "hull.cpp"
    hull_obj = BUILD_DIR / "hull.o"
    if force or _stale(hull_obj, [hull, INCLUDE / "ntrace.h"]):
        cmd = [nvcc, "-x", "c++", "-Wno-deprecated-gpu-targets", "-O2", "-Xcompiler", "-fPIC", *common, "-c", str(hull),
               "-o", str(hull_obj)]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    objload = CSRC / "objload.cpp"
    objload_obj = BUILD_DIR / "objload.o"
    if force or _stale(objload_obj, [objload, INCLUDE / "ntrace.h"]):
        cmd = [nvcc, "-x", "c++", "-Wno-deprecated-gpu-targets", "-O2", "-Xcompiler", "-fPIC", *common, "-c", str(objload),
               "-o", str(objload_obj)]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    if force or _stale(LIB, [cu_obj, cpp_obj, noalloc_obj, probes_obj, denoise_obj, objload_obj, tree_obj, hull_obj]):
        cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), str(cu_obj), str(cpp_obj),
               str(noalloc_obj), str(probes_obj), str(denoise_obj), str(objload_obj), str(tree_obj), str(hull_obj),
               "-Xlinker",
               "--no-undefined", "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
