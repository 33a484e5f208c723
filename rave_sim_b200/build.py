"""Build the rsw engine into ``rave_sim_b200/librsw.so`` (sm_100a).

    python -m rave_sim_b200.build [--verbose] [--force]

The library is built in-tree so that it travels with the source tree; the
build is incremental on source modification times.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "librsw.so"
BUILD = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
]

SOURCES = ["rsw_row_f64.cu", "rsw_row_f32.cu", "rsw_col.cu", "rsw_col_det.cu", "rsw_row_f64_batch.cu",
           "rsw_row_f32_batch.cu", "rsw_col_batch.cu", "rsw_kernels.cu", "rsw_noalloc.cu", "rsw_host.cpp"]
HEADERS = ["rsw_block_fft.cuh", "rsw_internal.h", "rsw_passes.cuh", "rsw_stages.h", "rsw_col_dispatch.h",
           "rsw_row_dispatch.h"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_verbose: bool = False) -> Path:
    from concurrent.futures import ThreadPoolExecutor

    BUILD.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [INCLUDE / "rsw.h"]
    objs, jobs = [], []
    for src in SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if force or _stale(o, [s, *headers]):
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(s), "-o", str(o)]
            if ptxas_verbose and s.suffix == ".cu":
                cmd.insert(1, "-Xptxas=-v")
            jobs.append((src, cmd))

    def run(job):
        src, cmd = job
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, cmd, r

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(run, jobs))
    for src, cmd, r in results:
        if verbose:
            print(" ".join(cmd), flush=True)
        if r.returncode != 0 or (verbose and r.stderr):
            sys.stderr.write(r.stdout + r.stderr)
    for src, cmd, r in results:
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}")
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print register/spill usage")
    a = ap.parse_args()
    print(build(verbose=a.verbose, force=a.force, ptxas_verbose=a.ptxas))
