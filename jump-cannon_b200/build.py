"""Build recipe for libjc_layout.so (the product library).

Compiles every CUDA/C++ source under csrc/ for sm_100a only and links one
shared library next to this file, so it travels with the repository
snapshot. Run directly (`python jump-cannon_b200/build.py`) or through
`__graft_entry__.build()`.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libjc_layout.so"
# The bounds-check build (-DJC_BOUNDS_CHECK): device index checks that record
# JC_ERR_BOUNDS instead of reading or writing out of range; same sources.
BUILD_BC = HERE / "_build_bc"
LIB_BC = HERE / "libjc_layout_bc.so"

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
# The image's CXX variable points at a compiler without OpenMP; use the
# system g++ as nvcc's host compiler.
HOST_CXX = shutil.which("g++", path="/usr/bin:/bin") or "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off",
          "-ccbin", HOST_CXX, "--expt-relaxed-constexpr"]


def _sources():
    return sorted(p for p in CSRC.iterdir() if p.suffix in (".cu", ".cpp"))


def _deps():
    return sorted(p for p in CSRC.iterdir() if p.suffix in (".cu", ".cpp", ".h", ".cuh")) + [
        HERE.parent / "include" / "jc_layout.h"]


def needs_build(lib: Path = LIB) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _deps())


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False, bounds_check: bool = False) -> Path:
    lib_path, build_dir = (LIB_BC, BUILD_BC) if bounds_check else (LIB, BUILD)
    extra = ["-DJC_BOUNDS_CHECK"] if bounds_check else []
    if not force and not needs_build(lib_path):
        return lib_path
    build_dir.mkdir(exist_ok=True)
    jobs = []
    for src in _sources():
        obj = build_dir / (src.stem + ".o")
        cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", str(src), "-o", str(obj)]
        if src.suffix == ".cpp":
            cmd = [NVCC, *COMMON, *extra, "-x", "cu", "-c", str(src), "-o", str(obj), *ARCH]
        if ptxas_info and src.suffix == ".cu":
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        jobs.append((src, obj, cmd))
    # one nvcc per source, side by side (the large sources dominate)
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda j: subprocess.run(j[2], capture_output=True, text=True), jobs))
    objs = []
    for (src, obj, _), r in zip(jobs, results):
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src.name}")
        if ptxas_info or verbose:
            sys.stderr.write(r.stderr)
        objs.append(str(obj))
    tmp = lib_path.with_suffix(".so.tmp")
    cmd = [NVCC, *ARCH, "-shared", "-o", str(tmp), *objs, "-ccbin", HOST_CXX, "-Xcompiler", "-fopenmp",
           "-lcudart", "-lgomp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, lib_path)
    return lib_path


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv, ptxas_info="--ptxas" in sys.argv,
                bounds_check="--bounds-check" in sys.argv))
