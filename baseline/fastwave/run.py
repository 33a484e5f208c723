"""Time the reference's GPU path (fast-wave's kernels and cuFFT, driven by
harness.cu over fast-wave's schedule) on one of the engine's workloads.

    python -m baseline.fastwave.run --workload talbot_lau --dtype c16 --logn 24 \
        --energies 32 --repeats 1 --warmup 1 [--detector out.npy]

Prints one JSON line: throughput in propagated complex samples * split steps
per second (CUDA events around each whole repeat), the device time per
repeat and per split step, and the split steps of one repeat. The workload
is the same seeded construction as bench.py's (plane wave, the Talbot-Lau
gratings, the cracked-cylinder phantom), passed to the harness in the
engine's own descriptors. Runs in its own process: the reference's error
handling exits the process.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

LIB = ROOT / "baseline" / "_ref" / "libfastwave_harness.so"


def workload(name: str, dtype: str, logn: int, energies: int):
    """(case, grids, energies, weights, deltabeta table function) as bench.py
    builds them for one rank."""
    from rave_sim_b200 import workloads

    e, w = workloads.config2_energies(energies)
    if name == "talbot_lau":
        return workloads.talbot_lau(n=1 << logn, dtype=dtype), None, e, w, workloads.db_table
    if name == "thick_sample":
        case, grids = workloads.thick_sample(n=1 << logn, dtype=dtype)
        return case, grids, e, w, workloads.db_table_sample
    raise ValueError(f"workload {name!r} has no GPU baseline")


def run(name: str, dtype: str, logn: int, energies: int, repeats: int = 1, warmup: int = 1):
    from rave_sim_b200 import _lib as L
    from rave_sim_b200.engine import deltabeta_vector, dtype_code, sim_descriptor

    if not LIB.exists():
        raise FileNotFoundError(f"{LIB.relative_to(ROOT)} is not built (python -m baseline.fastwave.build)")
    lib = C.CDLL(str(LIB))
    lib.fwh_run.restype = C.c_int
    lib.fwh_run.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int, C.c_void_p,
                            C.c_void_p, C.c_void_p, C.c_char_p, C.c_int]
    lib.fwh_detector_pixels.restype = C.c_int
    lib.fwh_detector_pixels.argtypes = [C.c_void_p]

    case, grids, es, ws, db_fn = workload(name, dtype, logn, energies)
    code = dtype_code(dtype)
    desc, _arr, keep, slots = sim_descriptor(case, grids, code, case["cutoff_angles"])
    runs = (L.SourceRun * len(es))()
    for r, e, w in zip(runs, es, ws):
        db = deltabeta_vector(slots, db_fn(float(e)))
        keep.append(db)
        r.energy_ev = float(e)
        r.deltabeta = db.view(np.float64).ctypes.data_as(L._DP)
        r.n_deltabeta = db.size
        r.weight = float(w)
        r.wavelength_m = 0.0
    nps = max(len(el["x_positions"]) for el in case["elements"])
    npix = lib.fwh_detector_pixels(C.byref(desc))
    det = np.zeros((nps, npix), dtype=np.float64)
    total = warmup + repeats
    ms = np.zeros(total, dtype=np.float64)
    steps = C.c_int64()
    err = C.create_string_buffer(256)
    st = lib.fwh_run(C.byref(desc), runs, len(es), float(case["source"]["z"]), nps, total,
                     det.ctypes.data, ms.ctypes.data, C.byref(steps), err, 256)
    if st != 0:
        raise RuntimeError(err.value.decode())
    n = int(case["sim_params"]["N"])
    t = float(np.mean(ms[warmup:])) if repeats > 0 else float(ms[-1])
    out = {"value": n * steps.value / (t * 1e-3), "unit": "samples*steps/s", "ms_per_repeat": t,
           "ms_per_split_step": t / max(steps.value, 1), "split_steps": steps.value, "n": n,
           "energies": len(es), "phase_steps": nps, "dtype": dtype, "workload": name,
           "path": "fast-wave fwcuda/kernels.cu + src/fft.cpp (cuFFT), unmodified, sm_100a; "
                   "run_simulation_inner schedule (src/simulation.cpp:375-549)"}
    return out, det


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="talbot_lau")
    ap.add_argument("--dtype", default="c16")
    ap.add_argument("--logn", type=int, default=24)
    ap.add_argument("--energies", type=int, default=32)
    ap.add_argument("--repeats", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--detector", default=None, help="save the weighted detector sum (.npy)")
    a = ap.parse_args()
    out, det = run(a.workload, a.dtype, a.logn, a.energies, a.repeats, a.warmup)
    if a.detector:
        np.save(a.detector, det)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
