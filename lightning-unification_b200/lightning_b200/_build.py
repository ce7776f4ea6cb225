"""Build recipe for the native parts of lightning_b200 (run in-tree).

* ``libb200sv.so``  — the CUDA kernels and the C ABI (include/b200sv.h), compiled
  by nvcc for sm_100a only.
* ``lightning_qubit_ops*.so`` — the pybind11 module with the lightning.qubit
  Python surface, compiled by g++ against the C++ host API and linked to
  libb200sv.so through an $ORIGIN rpath.

Both land next to this file so they travel with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sysconfig
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent                       # lightning-unification_b200/
REPO = ROOT.parent
CSRC = ROOT / "csrc"
INCLUDE = REPO / "include"
BUILD = ROOT / "_build"

CU_SOURCES = ["sv_gates.cu", "sv_reduce.cu", "sv_sample.cu", "sv_sparse.cu", "sv_fused.cu", "sv_mcmc.cu",
              "sv_capi.cu", "sv_batch.cu", "sv_noalloc.cu", "sv_tensor.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xcompiler", "-Wall"]

LIB = PKG / "libb200sv.so"
EXT_SUFFIX = sysconfig.get_config_var("EXT_SUFFIX")
MODULE = PKG / f"lightning_qubit_ops{EXT_SUFFIX}"


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libb200sv")


def _cuda_home() -> Path:
    return Path(_nvcc()).resolve().parent.parent


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, verbose: bool):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}):\n{' '.join(map(str, cmd))}\n{r.stdout}\n{r.stderr}")
    return r


def build_capi(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + [INCLUDE / "b200sv.h"]
    nvcc = _nvcc()
    objs = []
    jobs = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if force or _stale(o, [s, *headers]):
            jobs.append([nvcc, *ARCH, *NVCC_FLAGS, f"-I{INCLUDE}", "-c", s, "-o", o])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            list(ex.map(lambda c: _run(c, verbose), jobs))
    if force or jobs or _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"], verbose)
    return LIB


def build_bindings(verbose: bool = False, force: bool = False) -> Path:
    import pybind11

    src = CSRC / "bindings" / "lightning_qubit_ops.cpp"
    host_headers = list((CSRC / "host").glob("*.hpp")) + [INCLUDE / "b200sv.h"]
    if not (force or _stale(MODULE, [src, LIB, *host_headers])):
        return MODULE
    cuda = _cuda_home()
    cmd = ["g++", "-O2", "-std=c++20", "-shared", "-fPIC", "-fvisibility=hidden",
           f"-I{INCLUDE}", f"-I{CSRC / 'host'}", f"-I{pybind11.get_include()}",
           f"-I{sysconfig.get_paths()['include']}", f"-I{cuda / 'include'}",
           src, "-o", MODULE, f"-L{PKG}", "-lb200sv", "-Wl,-rpath,$ORIGIN"]
    _run(cmd, verbose)
    return MODULE


def build_all(verbose: bool = False, force: bool = False) -> None:
    build_capi(verbose, force)
    build_bindings(verbose, force)


if __name__ == "__main__":
    import sys
    build_all(verbose=True, force="--force" in sys.argv)
