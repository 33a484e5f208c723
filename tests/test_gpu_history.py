"""History recording (big-wave/history.py:43-135) on the device against the
reference's own History of the same runs (tests/golden/case_hist_*.npz):
analytic point-source entries, gaps sampled from their start, grating
sub-steps, sample rows; first phase-step pass only."""

import numpy as np
import pytest

from conftest import load_case, rel_l2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import rave_sim_b200 as rsw  # noqa: E402

NAMES = ["hist_point_tl", "hist_sample"]


# stepping_n6: big-wave's test_stepping setup at N = 6 (a Bluestein plan)
@pytest.mark.parametrize("name", NAMES + ["stepping_n6"])
@pytest.mark.parametrize("dtype,tol", [("c16", 1e-10), ("c8", 1e-5)])
def test_history_matches_reference(name, dtype, tol):
    case, grids, d = load_case(name)
    det, h, z = rsw.run_case(case, grids, dtype=dtype, history_dz=case["history_dz"])
    assert np.array_equal(z, d["history_z"])
    assert h.shape == d["history"].shape
    assert rel_l2(h, d["history"]) < tol
    assert rel_l2(det, d["detected"]) < tol


@pytest.mark.parametrize("name", NAMES)
def test_history_three_level(name, monkeypatch):
    case, grids, d = load_case(name)
    logn = int(np.log2(case["sim_params"]["N"]))
    monkeypatch.setenv("RSW_SPLIT3", f"4,{logn - 11},7")
    det, h, z = rsw.run_case(case, grids, dtype="c16", history_dz=case["history_dz"])
    assert rel_l2(h, d["history"]) < 1e-10


def test_history_off_and_repeated_runs():
    case, grids, d = load_case("hist_point_tl")
    sim = rsw.Simulation(case, grids, dtype="c16", cutoff_angles=case["cutoff_angles"])
    try:
        sim.set_history(case["history_dz"])
        for _ in range(2):  # each run restarts the history
            sim.reset()
            sim.run_source(energy=case["energy"], db_table=case["db"], source=case["source"])
            h, z = sim.history()
            assert np.array_equal(z, d["history_z"])
        sim.set_history(None)
        sim.reset()
        sim.run_source(energy=case["energy"], db_table=case["db"], source=case["source"])
        h, z = sim.history()
        assert h.shape[1] == 0 and len(z) == 0
        assert rel_l2(sim.detected(), d["detected"]) < 1e-10
    finally:
        sim.close()
