"""Build the fast-wave GPU baseline into baseline/_ref/libfastwave_harness.so.

    python -m baseline.fastwave.build

Compiles the reference's unmodified fast-wave/fwcuda/kernels.cu and
fast-wave/src/fft.cpp for sm_100a from the reference checkout, where they
lie (nothing is copied), plus harness.cu, and links them with cuFFT. The
output directory is git-ignored and travels with the tree to the GPU host,
which has no reference checkout: there the prebuilt library is used and this
recipe does nothing.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
OUT = ROOT / "baseline" / "_ref"
LIB = OUT / "libfastwave_harness.so"
REF = Path(os.environ.get("RAVE_SIM_REFERENCE", "/root/reference")) / "fast-wave"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def build(verbose: bool = False) -> Path | None:
    """Compile the baseline; returns the library path, or None when the
    reference checkout is absent (the prebuilt library, if any, stays)."""
    kernels, fft = REF / "fwcuda" / "kernels.cu", REF / "src" / "fft.cpp"
    if not (kernels.exists() and fft.exists()):
        return LIB if LIB.exists() else None
    OUT.mkdir(parents=True, exist_ok=True)
    inc = ["-I", str(REF / "fwcuda"), "-I", str(REF / "src"), "-I", str(ROOT / "include")]
    units = [(kernels, OUT / "fw_kernels.o"), (fft, OUT / "fw_fft.o"), (HERE / "harness.cu", OUT / "fw_harness.o")]
    srcs = [s for s, _ in units]
    if LIB.exists() and all(LIB.stat().st_mtime > s.stat().st_mtime for s in srcs):
        return LIB
    for src, obj in units:
        cmd = [nvcc(), *ARCH, *FLAGS, *inc, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src.name}")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *(str(o) for _, o in units), "-lcufft"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
