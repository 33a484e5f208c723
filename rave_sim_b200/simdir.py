"""Simulation-directory drop-in: run one source of a rave-sim simulation
directory on the engine and write its ``detected.npy``.

The directory layout is the reference's (big-wave/Readme.md, written by
``multisim.setup_simulation``, big-wave/multisim.py:282-521):

    <sim_dir>/config.yaml        sim_params, elements, dtype, save_final_u_vectors, ...
    <sim_dir>/computed.yaml      cutoff_angles (len(elements)+1), ...
    <sim_dir>/<grid>.npy         int8 sample grids named by the elements' grid_path
    <sim_dir>/NNNNNNNN/subconfig.yaml   energy, source, deltabeta_table

``run_single_simulation`` mirrors ``multisim.run_single_simulation``
(big-wave/multisim.py:50-150): it writes ``NNNNNNNN/detected.npy`` (float64,
shape (nr_phase_steps, nr_pixels)) and, with ``save_final_u_vectors``, the
field at the detector of each phase step as ``NNNNNNNN/u_{step:04}.npy``
(big-wave/wavesim.py:58-82). The command line mirrors fast-wave's
``fastwave <sim_dir> -s <idx>`` (fast-wave/main.cpp:18-57):

    python -m rave_sim_b200.simdir <sim_dir> -s <source_idx> [--dtype c8|c16] [--history_dz DZ]
        [--save_keypoints_path DIR]

``-s`` also takes several indices (``0-31``, ``0,4,9-12``): ``run_simulations``
runs the point sources at one z as one lockstep batch and writes each one's
detected.npy.

With ``--history_dz`` the history of the source is written as
``history.npy`` (n_pix, entries), ``history_z.npy`` and ``history_x.npy``
(big-wave/multisim.py:132-141). The field stays in GPU memory for the whole
source, so ``use_disk_vector`` is accepted and ignored. With
``--save_keypoints_path`` the field before and after each element of the first
pass is written as ``keypoint_{element:02}_{0|1}.npy`` (big-wave/wavesim.py:35-55).
"""

from __future__ import annotations

import argparse
import sys
from pathlib import Path
from typing import Optional

import numpy as np
import yaml


def sub_dir(sim_dir: Path, source_idx: int) -> Path:
    """``util.get_sub_dir`` (big-wave/util.py:92-97)."""
    return Path(sim_dir) / f"{source_idx:08}"


def detector_x_vector(detector_size: float, pixel_size_x: float) -> np.ndarray:
    """``util.detector_x_vector`` (big-wave/util.py:78-82)."""
    n = detector_size // pixel_size_x
    return (np.arange(n) - n // 2) * pixel_size_x


def _load(path: Path):
    with open(path) as f:
        return yaml.safe_load(f)


def _dtype(config) -> str:
    """``config.parse_dtype`` (big-wave/config.py:171-188): default c16."""
    val = config.get("dtype", "c16")
    if val not in ("c8", "c16"):
        raise ValueError(f"Unknown dtype: {val}. Has to be either c8 or c16")
    return val


def load_source(sim_dir, source_idx: int) -> dict:
    """Everything one source needs, in the case schema used by the engine:
    the config keys plus ``cutoff_angles``, ``energy``, ``db``, ``source``
    and the sample grids (``grids``: element index -> int8 array)."""
    sim_dir = Path(sim_dir)
    config = _load(sim_dir / "config.yaml")
    computed = _load(sim_dir / "computed.yaml")
    sub = _load(sub_dir(sim_dir, source_idx) / "subconfig.yaml")
    els = []
    grids = {}
    for i, el in enumerate(config["elements"]):
        t = el["type"]
        if t == "save_and_exit":
            raise ValueError("save_and_exit elements are resolved by the setup; run the reduced config")
        if t == "sample":
            g = np.load(sim_dir / el["grid_path"])
            if g.dtype != np.int8:
                raise AssertionError("sample grids must be int8")
            grids[i] = g
        if t not in ("grating", "dba_grating", "sample"):
            raise ValueError(f"Unknown optical element type: {t}.")
        els.append(dict(el))
    angles = [float(a) for a in computed["cutoff_angles"]]
    if len(angles) != len(els) + 1:
        raise AssertionError("computed.yaml must hold len(elements) + 1 cutoff angles")
    src = sub["source"]
    if src["type"] == "point":
        source = {"type": "point", "x": float(src["x"]), "z": float(src["z"])}
    elif src["type"] == "vector":
        source = {"type": "vector", "z": float(src["z"]), "path": str(src["input_path"])}
    else:
        raise ValueError(f'Unknown source type: {src["type"]}.')
    return {
        "sim_params": dict(config["sim_params"]),
        "elements": els,
        "dtype": _dtype(config),
        "save_final_u_vectors": bool(config.get("save_final_u_vectors", False)),
        "cutoff_angles": angles,
        "energy": float(sub["energy"]),
        "db": [[list(m), list(v)] for m, v in sub["deltabeta_table"]],
        "source": source,
        "grids": grids,
    }


def run_single_simulation(sim_dir, source_idx: int, scratch_dir=None, save_keypoints_path=None,
                          history_dz: Optional[float] = None, dtype: Optional[str] = None) -> np.ndarray:
    """Run source ``source_idx`` of ``sim_dir`` and write its detected.npy
    (big-wave/multisim.py:50-150, same argument order). With
    ``save_keypoints_path`` the field before and after each element of the
    first pass is saved there as keypoint_{element:02}_{0|1}.npy
    (big-wave/wavesim.py:35-55). ``dtype`` overrides the config's. Returns the
    detector array."""
    from .engine import Simulation

    sim_dir = Path(sim_dir)
    c = load_source(sim_dir, source_idx)
    dt = dtype or c["dtype"]
    field = None
    if c["source"]["type"] == "vector":
        field = np.load(c["source"]["path"])
        want = np.complex128 if dt == "c16" else np.complex64
        if field.dtype != want:
            field = field.astype(want)  # the reference converts with a warning (config.py:155-160)
    sim = Simulation(c, grids=c["grids"], dtype=dt, cutoff_angles=c["cutoff_angles"])
    try:
        sim.set_history(history_dz)
        if save_keypoints_path is not None:
            sim.set_keypoints(True)
        if c["save_final_u_vectors"]:
            sim.set_final_fields(True)
        sim.reset()
        sim.run_source(energy=c["energy"], db_table=c["db"], source=c["source"], field=field)
        det = sim.detected()
        if save_keypoints_path is not None:
            kp_dir = Path(save_keypoints_path)
            for k, t in enumerate(sim.keypoints()):
                np.save(kp_dir / f"keypoint_{k // 2:02}_{k % 2}.npy", t.cpu().numpy())
        out_dir = sub_dir(sim_dir, source_idx)
        if history_dz:
            h, z = sim.history()
            sp = c["sim_params"]
            np.save(out_dir / "history.npy", h)
            np.save(out_dir / "history_z.npy", z)
            np.save(out_dir / "history_x.npy",
                    detector_x_vector(sp["detector_size"], sp["detector_pixel_size_x"]))
        np.save(out_dir / "detected.npy", det)
        if c["save_final_u_vectors"]:
            for step, u in enumerate(sim.final_fields()):
                np.save(out_dir / f"u_{step:04}.npy", u.cpu().numpy())
        return det
    finally:
        sim.close()


def run_simulations(sim_dir, source_indices, dtype: Optional[str] = None) -> dict:
    """Run several sources of ``sim_dir`` and write each one's detected.npy,
    as ``run_single_simulation`` per index would (fast-wave's loop over
    ``-s k``, fast-wave/Readme.md:22-26). The sources share the directory's
    setup, so the point sources at one z run as one lockstep batch (their x
    positions may differ): one launch per pass for all of them, each
    source's detector kept apart. Vector sources (their own input files) and
    configs that save final fields run one by one. Returns {index: detector
    array}."""
    from .engine import Simulation

    sim_dir = Path(sim_dir)
    cases = {int(k): load_source(sim_dir, int(k)) for k in source_indices}
    out = {}
    groups: dict = {}
    for k, c in cases.items():
        src = c["source"]
        if src["type"] == "point" and not c["save_final_u_vectors"]:
            groups.setdefault(src["z"], []).append(k)
        else:
            out[k] = run_single_simulation(sim_dir, k, dtype=dtype)
    for ks in groups.values():
        c = cases[ks[0]]
        dt = dtype or c["dtype"]
        sim = Simulation(c, grids=c["grids"], dtype=dt, cutoff_angles=c["cutoff_angles"])
        try:
            sim.reset()
            each = sim.run_sources([{"energy": cases[k]["energy"], "db_table": cases[k]["db"]} for k in ks],
                                   sources=[cases[k]["source"] for k in ks], each=True).cpu().numpy()
        finally:
            sim.close()
        for k, det in zip(ks, each):
            np.save(sub_dir(sim_dir, k) / "detected.npy", det)
            out[k] = det
    return out


def parse_indices(spec: str) -> list:
    """Source indices of ``-s``: ``7``, ``0-31`` or ``0,4,9-12``."""
    ks = []
    for part in spec.split(","):
        part = part.strip()
        if "-" in part:
            a, b = part.split("-", 1)
            a, b = int(a), int(b)
            if b < a:
                raise ValueError(f"empty range {part!r}")
            ks.extend(range(a, b + 1))
        else:
            ks.append(int(part))
    if not ks or min(ks) < 0:
        raise ValueError(f"bad source indices {spec!r}")
    return ks


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m rave_sim_b200.simdir",
                                 description="Run sources of a rave-sim simulation directory on the GPU engine.")
    ap.add_argument("sim_dir")
    ap.add_argument("-s", "--source_idx", required=True,
                    help="source index, or several: 0-31, 0,4,9-12 (point sources at one z run together)")
    ap.add_argument("--dtype", choices=["c8", "c16"], default=None, help="override the config's dtype")
    ap.add_argument("--history_dz", type=float, default=None)
    ap.add_argument("--save_keypoints_path", default=None,
                    help="directory for keypoint_{element:02}_{0|1}.npy (the field before / after each element)")
    a = ap.parse_args(argv)
    try:
        ks = parse_indices(a.source_idx)
        if len(ks) > 1 and (a.history_dz or a.save_keypoints_path):
            raise ValueError("--history_dz and --save_keypoints_path take a single source index")
        if len(ks) == 1:
            run_single_simulation(a.sim_dir, ks[0], save_keypoints_path=a.save_keypoints_path,
                                  history_dz=a.history_dz, dtype=a.dtype)
        else:
            run_simulations(a.sim_dir, ks, dtype=a.dtype)
    except Exception as e:  # mirror fastwave: message and non-zero exit, no traceback
        print(f"error: {e}", file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
