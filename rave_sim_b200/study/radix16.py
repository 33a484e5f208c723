"""Radix-16 stage study: the engine's register butterflies against the
tensor cores (mma.sync TF32, single and split-operand) for one radix-16 DFT
stage of complex64 data plus its shared-memory exchange (radix16_study.cu).
Not part of the propagation path: the measurement behind keeping the FFT
stages on the FMA pipes.

    python -m rave_sim_b200.study.radix16 [--n 16777216] [--reps 64] [--once]

Prints one JSON line: per kind the time per stage and sample (median of 5
launches of `reps` stages over n samples), the tensor-core FLOP rate it
implies, and the rel-L2 error of one stage against an FP64 DFT. ``--once``
launches each kind once (for profiler captures).
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PKG = HERE.parent
SRC = HERE / "radix16_study.cu"
LIB = HERE / "libradix16_study.so"
KINDS = {0: "fma-pipe network (FFMA2 + lifting)", 1: "mma.sync TF32", 2: "mma.sync 3xTF32 (split operands)"}
MMA_FLOP_PER_SAMPLE = {1: 8 * 2048 / 128, 2: 24 * 2048 / 128}  # per stage


def build(force: bool = False) -> Path:
    from ..build import ARCH, NVCC_FLAGS, CSRC, nvcc

    deps = [SRC, CSRC / "rsw_block_fft.cuh", CSRC / "rsw_stages.h"]
    if force or not LIB.exists() or any(d.stat().st_mtime > LIB.stat().st_mtime for d in deps):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(CSRC), "-shared", "-o", str(LIB), str(SRC), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stderr)
            raise RuntimeError("nvcc failed on radix16_study.cu")
    return LIB


def dft_matrix() -> np.ndarray:
    """32 x 32 real form of the 16-point DFT scaled by 1/4: [Re y; Im y] =
    [[C, S], [-S, C]] [Re x; Im x] with C, S = cos, sin(2 pi j k / 16) / 4."""
    jk = np.outer(np.arange(16), np.arange(16))
    c = np.cos(2 * np.pi * jk / 16) / 4
    s = np.sin(2 * np.pi * jk / 16) / 4
    return np.block([[c, s], [-s, c]]).astype(np.float32)


def _brev4(k: int) -> int:
    return int(f"{k:04b}"[::-1], 2)


def main(argv=None) -> int:
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1 << 24)
    ap.add_argument("--reps", type=int, default=64)
    ap.add_argument("--once", action="store_true")
    a = ap.parse_args(argv)
    lib = C.CDLL(str(build()))
    lib.rsw_study_radix16.restype = C.c_int
    lib.rsw_study_radix16.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int,
                                      C.POINTER(C.c_float)]
    dev = "cuda"
    F = torch.from_numpy(dft_matrix()).to(dev)

    def launch(kind, x, y, reps):
        ms = C.c_float()
        st = lib.rsw_study_radix16(kind, F.data_ptr(), x.data_ptr(), y.data_ptr(), x.numel(), reps, C.byref(ms))
        if st != 0:
            raise RuntimeError(f"kind {kind}: error {st}")
        return ms.value

    rng = np.random.default_rng(1)
    if a.once:
        x = torch.randn(a.n, dtype=torch.complex64, device=dev)
        y = torch.empty_like(x)
        for k in KINDS:
            launch(k, x, y, a.reps)
        return 0

    # error of one stage against the FP64 DFT
    ns = 1 << 16
    xs = (rng.standard_normal(ns) + 1j * rng.standard_normal(ns)).astype(np.complex64)
    ref = np.fft.fft(xs.reshape(-1, 16).astype(np.complex128), axis=1)
    err = {}
    xd = torch.from_numpy(xs).to(dev)
    for k in KINDS:
        yd = torch.empty_like(xd)
        launch(k, xd, yd, 1)
        got = yd.cpu().numpy().reshape(-1, 16).astype(np.complex128)
        if k == 0:
            got = got[:, [_brev4(j) for j in range(16)]]
        else:
            got = got * 4
        err[k] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))

    x = torch.randn(a.n, dtype=torch.complex64, device=dev)
    y = torch.empty_like(x)
    out = {"n": a.n, "reps": a.reps, "kinds": {}}
    for k, name in KINDS.items():
        launch(k, x, y, a.reps)  # warm-up
        t = float(np.median([launch(k, x, y, a.reps) for _ in range(5)]))
        per = t * 1e6 / (a.reps * a.n)  # ns per sample and stage
        rec = {"what": name, "ms": t, "ns_per_sample_stage": per, "us_per_stage_at_n": per * a.n * 1e-3,
               "rel_l2_one_stage": err[k]}
        if k in MMA_FLOP_PER_SAMPLE:
            rec["tensor_tflops"] = MMA_FLOP_PER_SAMPLE[k] / per * 1e-3
        out["kinds"][str(k)] = rec
    out["device"] = torch.cuda.get_device_name(0)
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
