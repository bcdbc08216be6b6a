"""Builds the native library in-tree: threert_b200/libthreert_b200.so (the C ABI of include/threert_cuda.h and
include/threert_prep.h) from csrc/, for sm_100a only.

`python -m threert_b200.build` or `threert_b200.build.build()`. Rebuilds when a source is newer than the library.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libthreert_b200.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: the pass's arithmetic rounds as the CPU restatement's does (no fused multiply-adds it did not write).
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wextra"]


def _sources():
    cu = sorted(CSRC.glob("*.cu"))
    cpp = sorted(CSRC.glob("*.cpp"))
    headers = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))
    return cu, cpp, headers


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build failed: {' '.join(str(c) for c in cmd[:3])} ...")
    out = (r.stdout + r.stderr).strip()
    if out and verbose:
        print(out)
    return out


def build(verbose: bool = False, force: bool = False) -> Path:
    cu, cpp, headers = _sources()
    if not force and not _stale(LIB, cu + cpp + headers + [Path(__file__)]):
        return LIB
    BUILD.mkdir(exist_ok=True)
    jobs = [([NVCC, *NVCC_FLAGS, "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", BUILD / (src.stem + ".o")],
             BUILD / (src.stem + ".o")) for src in cu]
    jobs += [(["g++", *CXX_FLAGS, "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", BUILD / (src.stem + ".o")],
              BUILD / (src.stem + ".o")) for src in cpp]
    # The translation units compile independently: one compiler process each, side by side.
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        list(pool.map(lambda j: _run(j[0], verbose), jobs))
    objs = [obj for _, obj in jobs]
    tmp = LIB.with_suffix(".so.tmp")
    _run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], verbose)
    os.replace(tmp, LIB)
    return LIB


def ptxas_report() -> str:
    """Registers, spills and shared memory per kernel (nvcc -Xptxas -v) of the CUDA sources."""
    cu, _, _ = _sources()
    BUILD.mkdir(exist_ok=True)
    out = []
    for src in cu:
        r = subprocess.run([NVCC, *NVCC_FLAGS, "-Xptxas", "-v", "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src),
                            "-o", str(BUILD / (src.stem + ".v.o"))], capture_output=True, text=True)
        out.append(r.stdout + r.stderr)
    return "\n".join(out)


if __name__ == "__main__":
    if "--ptxas" in sys.argv:
        print(ptxas_report())
    else:
        print(build(verbose=True, force="--force" in sys.argv))
