"""Keypoints (big-wave/wavesim.py:35-55, :186, :196): the field right before
and right after each element of the first phase-step pass, on the device,
against the reference's own keypoint files (tests/golden/case_*.npz: every
s-th sample, full-vector sums and norms) and the oracle's full fields. Covers
a plane wave held implicitly, fields in the passes' intermediate order and
in natural order, a point source, a phase-stepped sample, history recorded in
the same run, and a Bluestein length (N = 6, N = 3^8). The sim-dir runner
writes them as big-wave's test_keypoints expects (big-wave/test.py:575-590:
two per element, complex128, length N)."""

import numpy as np
import pytest

from conftest import load_case, rel_l2
from oracle import bigwave_np as bw

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import rave_sim_b200 as rsw  # noqa: E402
from rave_sim_b200 import simdir  # noqa: E402

NAMES = ["sample_stepped", "hist_sample", "stepping_n6", "odd_point_sample"]


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("dtype,tol", [("c16", 1e-10), ("c8", 1e-5)])
def test_keypoints_match_reference(name, dtype, tol):
    case, grids, d = load_case(name)
    kps = []
    out = rsw.run_case(case, grids, dtype=dtype, history_dz=case.get("history_dz"), keypoints=kps)
    det = out[0] if isinstance(out, tuple) else out
    kps = np.stack(kps).astype(np.complex128)
    n = case["sim_params"]["N"]
    assert kps.shape == (2 * len(case["elements"]), n)
    assert rel_l2(kps[:, ::int(d["keypoints_stride"])], d["keypoints_sub"]) < tol
    norm2 = (np.abs(kps) ** 2).sum(axis=1)
    assert rel_l2(norm2, d["keypoints_norm2"]) < tol
    assert np.all(np.abs(kps.sum(axis=1) - d["keypoints_sum"]) <= tol * np.sqrt(n * d["keypoints_norm2"]))
    assert rel_l2(det, d["detected"]) < tol
    if isinstance(out, tuple):
        assert rel_l2(out[1], d["history"]) < tol
    if dtype == "c16":
        ref = []
        bw.run_simulation(case, grids, keypoints=ref)
        assert rel_l2(kps, np.stack(ref)) < 1e-10


def test_keypoints_off_and_reused():
    case, grids, d = load_case("sample_stepped")
    sim = rsw.Simulation(case, grids, dtype="c16", cutoff_angles=case["cutoff_angles"])
    try:
        with pytest.raises(ValueError):
            sim.keypoints()
        sim.set_keypoints(True)
        for _ in range(2):  # the buffers are rewritten by every run
            sim.reset()
            sim.run_source(energy=case["energy"], db_table=case["db"], source=case["source"])
            k = np.stack([t.cpu().numpy() for t in sim.keypoints()])
            assert rel_l2(k[:, ::int(d["keypoints_stride"])], d["keypoints_sub"]) < 1e-10
        sim.set_keypoints(False)
        sim.reset()
        sim.run_source(energy=case["energy"], db_table=case["db"], source=case["source"])
        assert rel_l2(sim.detected(), d["detected"]) < 1e-10
    finally:
        sim.close()


def test_simdir_keypoints(tmp_path):
    import yaml

    case, grids, d = load_case("sample_stepped")
    cfg = {"sim_params": case["sim_params"], "use_disk_vector": False, "save_final_u_vectors": False,
           "dtype": "c16", "elements": case["elements"]}
    for i, g in grids.items():
        np.save(tmp_path / case["elements"][i]["grid_path"], g)
    (tmp_path / "config.yaml").write_text(yaml.safe_dump(cfg))
    (tmp_path / "computed.yaml").write_text(yaml.safe_dump({"cutoff_angles": case["cutoff_angles"]}))
    sub = tmp_path / "00000000"
    sub.mkdir()
    (sub / "subconfig.yaml").write_text(yaml.safe_dump({
        "source": {"type": "point", "x": case["source"]["x"], "z": case["source"]["z"]},
        "energy": case["energy"], "deltabeta_table": case["db"]}))
    kp = tmp_path / "keypoints"
    kp.mkdir()
    det = simdir.run_single_simulation(tmp_path, 0, tmp_path, kp)
    assert rel_l2(det, d["detected"]) < 1e-10
    files = sorted(p.name for p in kp.iterdir())
    assert files == [f"keypoint_{i:02}_{k}.npy" for i in range(len(case["elements"])) for k in (0, 1)]
    kps = np.stack([np.load(kp / f) for f in files])
    assert kps.dtype == np.complex128 and kps.shape[1] == case["sim_params"]["N"]
    assert rel_l2(kps[:, ::int(d["keypoints_stride"])], d["keypoints_sub"]) < 1e-10


# ---------------------------------------------------------------- final fields
# big-wave's save_u (wavesim.py:58-82) with save_final_u_vectors writes the
# field at the detector after every phase step (u_0000.npy, u_0001.npy, ...).
@pytest.mark.parametrize("name", ["sample_stepped", "tl3g_point_phase"])
@pytest.mark.parametrize("dtype,tol", [("c16", 1e-13), ("c8", 1e-6)])
def test_final_field_of_every_phase_step(name, dtype, tol):
    case, grids, d = load_case(name)
    sim = rsw.Simulation(case, grids=grids, dtype=dtype, cutoff_angles=case["cutoff_angles"])
    try:
        sim.set_final_fields(True)
        sim.reset()
        sim.run_source(energy=case["energy"], db_table=case["db"], source=case["source"])
        det = sim.detected()
        fields = [f.cpu().numpy().astype(np.complex128) for f in sim.final_fields()]
        last = sim.final_field().cpu().numpy().astype(np.complex128)
    finally:
        sim.close()
    assert len(fields) == det.shape[0] > 1
    ref = bw.make_sim(case)
    for p, u in enumerate(fields):
        # each field bins to its own phase step's detector row
        assert rel_l2(bw.square_and_downsample(u, ref, ref.z_detector), det[p]) < tol, p
    assert rel_l2(fields[0], fields[1]) > 1e-6  # the stepped element moved
    assert np.array_equal(fields[-1], last)


def test_simdir_writes_the_final_field_of_every_phase_step(tmp_path):
    case, grids, d = load_case("tl3g_point_phase")
    import yaml

    cfg = {"sim_params": case["sim_params"], "use_disk_vector": False, "save_final_u_vectors": True,
           "dtype": "c16", "elements": case["elements"]}
    (tmp_path / "config.yaml").write_text(yaml.safe_dump(cfg))
    (tmp_path / "computed.yaml").write_text(yaml.safe_dump({"cutoff_angles": case["cutoff_angles"]}))
    sub = tmp_path / "00000000"
    sub.mkdir()
    (sub / "subconfig.yaml").write_text(yaml.safe_dump({
        "source": case["source"], "energy": case["energy"], "deltabeta_table": case["db"]}))
    det = simdir.run_single_simulation(tmp_path, 0)
    ref = bw.make_sim(case)
    for p in range(det.shape[0]):
        u = np.load(sub / f"u_{p:04}.npy")
        assert u.dtype == np.complex128 and u.shape == (ref.N,)
        assert rel_l2(bw.square_and_downsample(u, ref, ref.z_detector), det[p]) < 1e-13
    assert not (sub / f"u_{det.shape[0]:04}.npy").exists()
