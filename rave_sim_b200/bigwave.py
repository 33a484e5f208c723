"""Drop-in replacements with rave-sim big-wave's signatures.

These accept big-wave's ``NumpyVector`` (any object with a ``.vec`` numpy
array) and ``SimParams`` (any object with the same attributes), copy to the
GPU, run the CUDA engine and copy back, so big-wave's own driver code and
tests can run on the engine unchanged:

    propagate(u, U, dx, wl, dz, chunk_size, cutoff_frequency, skip_fft=False)
        big-wave/propagation.py:100-138
    square_and_downsample(u, sim_params, current_z) -> np.ndarray
        big-wave/propagation.py:279-320
    run_simulation(params, source, elements, cutoff_angles, u, U,
                   deltabeta_table, sub_dir, vectors_dir, save_final_u_vectors,
                   history=None, save_keypoints_path=None) -> list[np.ndarray]
        big-wave/wavesim.py:84-298, with history and keypoints (the field
        before and after each element, saved as keypoint_{el:02}_{0|1}.npy)

Errors are raised as ``ValueError`` / ``AssertionError`` like the reference's.
"""

from __future__ import annotations

from pathlib import Path
from typing import Optional

import numpy as np

from .engine import Plan, Simulation

_plans: dict = {}


def _plan(n: int, dtype) -> Plan:
    key = (n, np.dtype(dtype).str)
    if key not in _plans:
        _plans[key] = Plan(n, "c16" if np.dtype(dtype) == np.complex128 else "c8")
    return _plans[key]


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def propagate(u, U, dx, wl, dz, chunk_size, cutoff_frequency, skip_fft=False):
    """big-wave ``propagate``: ``u`` is updated in place and ``U`` receives
    the spectrum of the new ``u`` (or must hold FFT(u) when ``skip_fft``)."""
    vec = u.vec
    if vec.dtype not in (np.complex128, np.complex64):
        raise ValueError("u must be complex64 or complex128")
    p = _plan(len(vec), vec.dtype)
    ud = _dev(vec)
    Ud = _dev(U.vec.astype(vec.dtype)) if skip_fft else _dev(np.empty_like(vec))
    p.propagate(ud, Ud, dx=float(dx), wl=float(wl), dz=float(dz), cutoff_freq=float(cutoff_frequency),
                skip_fft=bool(skip_fft))
    u.vec = ud.cpu().numpy()
    U.vec = Ud.cpu().numpy()


def square_and_downsample(u, sim_params, current_z) -> np.ndarray:
    """big-wave ``square_and_downsample``: detector intensity (float64)."""
    vec = u.vec
    p = _plan(len(vec), vec.dtype)
    out = p.square_and_downsample(_dev(vec), dx=float(sim_params.dx),
                                  detector_size=float(sim_params.detector_size),
                                  pixel_size_x=float(sim_params.detector_pixel_size_x),
                                  pixel_size_y=float(sim_params.detector_pixel_size_y), z=float(current_z))
    return out.cpu().numpy()


def _material(m):
    if m is None:
        return None
    return [m.mat, float(m.density)]


def _element_dict(el) -> dict:
    """big-wave OpticalElement dataclass -> config.yaml element dict."""
    name = type(el).__name__
    d = {"z_start": float(el.z_start), "x_positions": [float(x) for x in np.asarray(el.x_positions).ravel()]}
    if name == "Grating":
        d.update(type="grating", pitch=float(el.pitch), dc=[float(el.dc[0]), float(el.dc[1])],
                 thickness=float(el.thickness), nr_steps=int(el.nr_steps),
                 substrate_thickness=float(el.substrate_thickness), mat_a=_material(el.mat_a),
                 mat_b=_material(el.mat_b), mat_substrate=_material(el.mat_substrate))
    elif name == "DBAGrating":
        d.update(type="dba_grating", pitch0=float(el.pitch0), pitch1=float(el.pitch1),
                 dc0=[float(el.dc0[0]), float(el.dc0[1])], dc1=[float(el.dc1[0]), float(el.dc1[1])],
                 thickness=float(el.thickness), nr_steps=int(el.nr_steps),
                 substrate_thickness=float(el.substrate_thickness), mat_a=_material(el.mat_a),
                 mat_b=_material(el.mat_b), mat_substrate=_material(el.mat_substrate))
    elif name == "Sample":
        d.update(type="sample", pixel_size_x=float(el.pixel_size_x), pixel_size_z=float(el.pixel_size_z),
                 materials=[_material(m) for m in el.materials])
    else:
        raise ValueError(f"unsupported optical element {name}")
    return d


def run_simulation(params, source, elements, cutoff_angles, u, U, deltabeta_table, sub_dir, vectors_dir,
                   save_final_u_vectors, history=None, save_keypoints_path=None):
    """big-wave ``wavesim.run_simulation`` for one source on the fused engine.
    Returns the list of detector arrays (one per phase step); with
    ``save_final_u_vectors`` the final field of the last phase step is left
    in ``u``. ``history`` is big-wave's ``(History, dz)`` pair
    (big-wave/wavesim.py:95, :129-131): the engine records the history and its
    entries are pushed into the History object in order."""
    n = len(u)
    dtype = u.vec.dtype
    config = {
        "sim_params": {"N": n, "dx": params.dx, "z_detector": params.z_detector,
                       "detector_size": params.detector_size,
                       "detector_pixel_size_x": params.detector_pixel_size_x,
                       "detector_pixel_size_y": params.detector_pixel_size_y, "chunk_size": params.chunk_size},
        "elements": [_element_dict(e) for e in elements],
        "cutoff_angles": list(cutoff_angles),
    }
    grids = {i: np.asarray(e.grid) for i, e in enumerate(elements) if type(e).__name__ == "Sample"}
    table = [[[m.mat, float(m.density)], [float(np.real(v)), float(np.imag(v))]] for m, v in deltabeta_table]
    sim = Simulation(config, grids=grids, dtype="c16" if dtype == np.complex128 else "c8")
    try:
        sname = type(source).__name__
        if sname == "PointSource":
            src = {"type": "point", "x": float(source.x), "z": float(source.z)}
            field = None
        elif sname == "VectorSource":
            src = {"type": "vector", "z": float(source.z)}
            field = np.asarray(source.input.vec)
        else:
            raise ValueError(f"unsupported source {sname}")
        sim.reset()
        if history is not None:
            sim.set_history(float(history[1]))
        if save_keypoints_path is not None:
            sim.set_keypoints(True)
        sim.run_source(energy=1.0, wavelength=float(params.wl), db_table=table, source=src, field=field)
        det = sim.detected()
        if save_keypoints_path is not None:
            # save_keypoint (big-wave/wavesim.py:35-55)
            kp_dir = Path(save_keypoints_path)
            for k, t in enumerate(sim.keypoints()):
                np.save(kp_dir / f"keypoint_{k // 2:02}_{k % 2}.npy", t.cpu().numpy())
        if history is not None:
            images, zs = sim.history()
            for e in range(images.shape[1]):
                history[0].push(images[:, e].copy(), float(zs[e]))
        if save_final_u_vectors:
            u.vec = sim.final_field().cpu().numpy()
        return [det[i] for i in range(det.shape[0])]
    finally:
        sim.close()
