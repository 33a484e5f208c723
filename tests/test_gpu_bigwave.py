"""The big-wave-signature shim (rave_sim_b200.bigwave) on minimal stand-ins
of big-wave's data classes (same field names as big-wave/optical_element.py,
source.py, vector.py, propagation.py), checked against the reference goldens
and the oracle."""

from dataclasses import dataclass
from typing import Optional

import numpy as np
import pytest

from conftest import load_case, rel_l2
from oracle import bigwave_np as bw

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from rave_sim_b200 import bigwave  # noqa: E402


@dataclass
class SimParams:
    N: int
    dx: float
    z_detector: float
    detector_size: float
    detector_pixel_size_x: float
    detector_pixel_size_y: float
    wl: float
    chunk_size: int


@dataclass
class Material:
    mat: str
    density: float


@dataclass
class Grating:
    pitch: float
    dc: tuple
    z_start: float
    thickness: float
    nr_steps: int
    x_positions: np.ndarray
    substrate_thickness: float
    mat_a: Optional[Material]
    mat_b: Optional[Material]
    mat_substrate: Optional[Material]


@dataclass
class PointSource:
    x: float
    z: float


class NumpyVector:
    def __init__(self, vec):
        self.vec = vec

    def __len__(self):
        return len(self.vec)


def _mat(m):
    return None if m is None else Material(m[0], m[1])


class History:
    """big-wave/history.py:10-40: entries and z pushed in order."""

    def __init__(self):
        self.entries, self.zs = [], []

    def push(self, downscaled, z):
        self.entries.append(downscaled)
        self.zs.append(z)

    def get_history(self):
        return np.stack(self.entries, axis=-1) if self.entries else np.empty((0, 0))


def _shim_inputs(case):
    sp = case["sim_params"]
    params = SimParams(N=sp["N"], dx=sp["dx"], z_detector=sp["z_detector"], detector_size=sp["detector_size"],
                       detector_pixel_size_x=sp["detector_pixel_size_x"],
                       detector_pixel_size_y=sp["detector_pixel_size_y"],
                       wl=bw.wavelength_from_energy(case["energy"]), chunk_size=sp["chunk_size"])
    els = [Grating(pitch=e["pitch"], dc=tuple(e["dc"]), z_start=e["z_start"], thickness=e["thickness"],
                   nr_steps=e["nr_steps"], x_positions=np.array(e["x_positions"]),
                   substrate_thickness=e["substrate_thickness"], mat_a=_mat(e["mat_a"]), mat_b=_mat(e["mat_b"]),
                   mat_substrate=_mat(e["mat_substrate"])) for e in case["elements"]]
    table = [(Material(m[0], m[1]), complex(v[0], v[1])) for m, v in case["db"]]
    src = PointSource(x=case["source"]["x"], z=case["source"]["z"])
    u = NumpyVector(np.zeros(sp["N"], np.complex128))
    U = NumpyVector(np.zeros(sp["N"], np.complex128))
    return params, src, els, table, u, U


def test_run_simulation_shim_matches_golden():
    case, grids, d = load_case("tl3g_point_phase")
    params, src, els, table, u, U = _shim_inputs(case)
    out = bigwave.run_simulation(params, src, els, case["cutoff_angles"], u, U, table, ".", ".", False)
    assert len(out) == d["detected"].shape[0]
    assert rel_l2(np.array(out), d["detected"]) < 1e-10


def test_run_simulation_shim_history():
    # wavesim.run_simulation(..., history=(History(), dz)) as multisim.py:114-137 calls it
    case, grids, d = load_case("hist_point_tl")
    params, src, els, table, u, U = _shim_inputs(case)
    hist = History()
    out = bigwave.run_simulation(params, src, els, case["cutoff_angles"], u, U, table, ".", ".", False,
                                 history=(hist, case["history_dz"]))
    assert rel_l2(np.array(out), d["detected"]) < 1e-10
    assert np.array_equal(np.array(hist.zs), d["history_z"])
    assert rel_l2(hist.get_history(), d["history"]) < 1e-10


def test_propagate_and_detect_shims():
    n = 1 << 15
    rng = np.random.default_rng(3)
    vec = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    sim = bw.Sim(N=n, dx=1e-9, z_detector=0.3, detector_size=20e-6, psx=0.5e-6, psy=1e-6, wl=2.7e-11,
                 chunk_size=n)
    u, U = NumpyVector(vec.copy()), NumpyVector(np.zeros(n, np.complex128))
    bigwave.propagate(u, U, 1e-9, 2.7e-11, 0.05, n, np.sin(2e-3) / 2.7e-11)
    u_ref, U_ref = bw.propagate(vec, None, sim, 0.05, np.sin(2e-3) / 2.7e-11)
    assert rel_l2(u.vec, u_ref) < 1e-10 and rel_l2(U.vec, U_ref) < 1e-10
    params = SimParams(N=n, dx=1e-9, z_detector=0.3, detector_size=20e-6, detector_pixel_size_x=0.5e-6,
                       detector_pixel_size_y=1e-6, wl=2.7e-11, chunk_size=n)
    det = bigwave.square_and_downsample(u, params, 0.3)
    assert rel_l2(det, bw.square_and_downsample(u.vec, sim, 0.3)) < 1e-13


def test_run_simulation_shim_keypoints(tmp_path):
    # save_keypoints_path (big-wave/wavesim.py:35-55): keypoint_{el:02}_{0|1}.npy
    case, grids, d = load_case("stepping_n6")
    params, src, els, table, u, U = _shim_inputs(case)
    out = bigwave.run_simulation(params, src, els, case["cutoff_angles"], u, U, table, ".", ".", False,
                                 save_keypoints_path=tmp_path)
    assert rel_l2(np.array(out), d["detected"]) < 1e-10
    kps = np.stack([np.load(tmp_path / f"keypoint_{i:02}_{k}.npy") for i in range(len(els)) for k in (0, 1)])
    assert kps.dtype == np.complex128
    assert rel_l2(kps[:, ::int(d["keypoints_stride"])], d["keypoints_sub"]) < 1e-10
