"""Lockstep batches of sources (rsw_sim_run_batch) against the same sources
run one after the other (rsw_sim_run), through the C ABI.

Each instance of a batch runs the same arithmetic as its own run; only the
order of the atomic per-pixel sums of the fused detection differs. Tolerance
(detector intensity, rel-L2): 1e-12 for both dtypes, far below the 1e-10
(complex128) and 1e-5 (complex64) budgets against the oracle that single runs
are held to.

Cases: the three-grating interferometer (gratings, phase stepping) in both
dtypes, with each instance checked alone through one-hot weights and the
complex64 batch checked to launch one kernel per pass for all instances; a
batch run in chunks (RSW_BATCH_CHUNK, as when the buffers do not fit); a sample
(int8 grid, per-energy material tables) with a cutoff angle that is active
for some energies only; a point source; a forced three-level plan; batches
that grow the sim's batch buffers; the configurations that run one source
after the other (history, exact propagator).
"""

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import rave_sim_b200 as rsw  # noqa: E402
from rave_sim_b200 import workloads  # noqa: E402
from rave_sim_b200.engine import Simulation  # noqa: E402

TOL = 1e-12
ENERGIES = [24000.0, 33000.0, 46000.0, 58000.0, 69000.0]


def _sequential(sim, runs, source):
    sim.reset()
    for r in runs:
        sim.run_source(energy=r["energy"], db_table=r["db_table"], source=source, weight=r["weight"])
    return sim.detected()


def _batched(sim, runs, source):
    sim.reset()
    sim.run_sources(runs, source=source)
    return sim.detected()


def _talbot_lau(dtype):
    return workloads.talbot_lau(n=1 << 16, dx=2e-9, dtype=dtype, nr_steps=3, phase_steps=4,
                                detector_size=100e-6, pixel_size=1e-6)


@pytest.mark.parametrize("dtype", ["c16", "c8"])
def test_interferometer_batch_equals_runs(dtype):
    case = _talbot_lau(dtype)
    w = workloads.kramers_weights(np.array(ENERGIES), 70000.0)
    runs = [{"energy": e, "db_table": workloads.db_table(e), "weight": float(wi)} for e, wi in zip(ENERGIES, w)]
    sim = Simulation(case, dtype=dtype)
    try:
        lib = rsw.load_library()
        l0 = lib.rsw_launch_count()
        seq = _sequential(sim, runs, case["source"])
        l1 = lib.rsw_launch_count()
        bat = _batched(sim, runs, case["source"])
        l2 = lib.rsw_launch_count()
        assert seq.shape == (4, 100)
        assert rel_l2(bat, seq) < TOL
        # one launch per pass for all instances (complex64 column kernels
        # keep their occupancy when batched; complex128 shapes that would not
        # run the sources one after the other)
        if dtype == "c8":
            assert (l2 - l1) * 3 < (l1 - l0)
        # every instance alone: one-hot weights against its own run
        for b, e in enumerate(ENERGIES):
            one = [dict(r, weight=1.0 if i == b else 0.0) for i, r in enumerate(runs)]
            got = _batched(sim, one, case["source"])
            ref = _sequential(sim, [dict(runs[b], weight=1.0)], case["source"])
            assert rel_l2(got, ref) < TOL, f"instance {b} ({e} eV)"
    finally:
        sim.close()


@pytest.mark.parametrize("dtype", ["c16", "c8"])
def test_sample_batch_with_partial_cutoff(dtype):
    case, grids = workloads.thick_sample(
        n=1 << 16, dx=100e-9, dtype=dtype, nr_steps=3, phase_steps=2, rows=40, cols=120,
        psz=0.25e-6, psx=0.1e-6, diameter=10e-6, axis_range=(0.2e-6, 1.0e-6), seed=7,
        detector_size=6e-6, pixel_size=0.5e-6)
    # a cutoff angle between the energies' sin(a) = wl / (2 dx) limits: the
    # cut is active for the low energies and absent for the high ones
    lim = [workloads.wavelength_from_energy(e) / (2 * 100e-9) for e in (30000.0, 60000.0)]
    ang = float(np.arcsin(0.5 * (lim[0] + lim[1])))
    angles = [ang] * (len(case["elements"]) + 1)
    energies = [30000.0, 40000.0, 52000.0, 60000.0]
    runs = [{"energy": e, "db_table": workloads.db_table_sample(e), "weight": 1.0 + 0.25 * i}
            for i, e in enumerate(energies)]
    sim = Simulation(case, grids=grids, dtype=dtype, cutoff_angles=angles)
    try:
        seq = _sequential(sim, runs, case["source"])
        bat = _batched(sim, runs, case["source"])
        assert np.abs(seq).max() > 0
        assert rel_l2(bat, seq) < TOL
    finally:
        sim.close()


def _point_case():
    n = 1 << 16
    return {
        "sim_params": {"N": n, "dx": 1e-9, "z_detector": 0.2, "detector_size": 40e-6,
                       "detector_pixel_size_x": 1e-6, "detector_pixel_size_y": 1.0, "chunk_size": n},
        "elements": [
            {"type": "grating", "pitch": 4.2e-6, "dc": [0.5, 0.5], "z_start": 0.05, "thickness": 40e-6,
             "nr_steps": 2, "x_positions": [0.0], "substrate_thickness": 20e-6,
             "mat_a": ["Au", 19.32], "mat_b": None, "mat_substrate": ["Si", 2.34]},
            {"type": "grating", "pitch": 4.2e-6, "dc": [0.5, 0.5], "z_start": 0.15, "thickness": 30e-6,
             "nr_steps": 2, "x_positions": [0.0, 1.05e-6, 2.1e-6], "substrate_thickness": 0.0,
             "mat_a": ["Si", 2.34], "mat_b": None, "mat_substrate": None},
        ],
        "source": {"type": "point", "x": 0.1e-6, "z": 0.0},
        "cutoff_angles": [1e-4, 1e-4, 2e-4],
    }


@pytest.mark.parametrize("dtype", ["c16", "c8"])
def test_point_source_batch(dtype):
    case = _point_case()
    db = [[["Si", 2.34], [2.2888e-7, 2.5847e-10]], [["Au", 19.32], [1.4981e-6, 3.6174e-8]]]
    runs = [{"energy": e, "db_table": db, "weight": 1.0 / (i + 1)} for i, e in enumerate([40000.0, 46000.0, 55000.0])]
    sim = Simulation(case, dtype=dtype)
    try:
        seq = _sequential(sim, runs, case["source"])
        bat = _batched(sim, runs, case["source"])
        assert rel_l2(bat, seq) < TOL
    finally:
        sim.close()


def test_three_level_batch(monkeypatch):
    monkeypatch.setenv("RSW_SPLIT3", "4,4,8")
    case = _talbot_lau("c16")
    runs = [{"energy": e, "db_table": workloads.db_table(e), "weight": 1.0} for e in ENERGIES[:3]]
    plan = rsw.Plan(1 << 16, "c16")
    assert plan.info()["log_rows"] == 4  # the forced split's column level
    plan.close()
    sim = Simulation(case, dtype="c16")
    try:
        seq = _sequential(sim, runs, case["source"])
        bat = _batched(sim, runs, case["source"])
        assert rel_l2(bat, seq) < TOL
    finally:
        sim.close()


def test_batch_buffers_grow_and_restart():
    case = _talbot_lau("c8")
    runs = [{"energy": e, "db_table": workloads.db_table(e), "weight": 1.0} for e in ENERGIES]
    sim = Simulation(case, dtype="c8")
    try:
        small = _batched(sim, runs[:2], case["source"])
        full = _batched(sim, runs, case["source"])
        again = _batched(sim, runs[:2], case["source"])
        assert rel_l2(full, _sequential(sim, runs, case["source"])) < TOL
        assert rel_l2(again, small) < TOL
    finally:
        sim.close()


def test_unbatchable_configurations_run_one_by_one():
    case = _talbot_lau("c16")
    runs = [{"energy": e, "db_table": workloads.db_table(e), "weight": 1.0} for e in ENERGIES[:2]]
    sim = Simulation(case, dtype="c16", propagator="exact")
    try:
        assert rel_l2(_batched(sim, runs, case["source"]), _sequential(sim, runs, case["source"])) < TOL
    finally:
        sim.close()
    sim = Simulation(case, dtype="c16")
    try:
        sim.set_history(0.2)
        assert rel_l2(_batched(sim, runs, case["source"]), _sequential(sim, runs, case["source"])) < TOL
    finally:
        sim.close()


def test_batch_in_chunks(monkeypatch):
    monkeypatch.setenv("RSW_BATCH_CHUNK", "2")
    case = _talbot_lau("c8")
    runs = [{"energy": e, "db_table": workloads.db_table(e), "weight": 1.0 + i} for i, e in enumerate(ENERGIES)]
    sim = Simulation(case, dtype="c8")
    try:
        lib = rsw.load_library()
        l0 = lib.rsw_launch_count()
        seq = _sequential(sim, runs, case["source"])
        l1 = lib.rsw_launch_count()
        bat = _batched(sim, runs, case["source"])
        l2 = lib.rsw_launch_count()
        assert rel_l2(bat, seq) < TOL
        # chunks of 2, 2 and 1 sources: three runs' worth of pass launches
        assert (l2 - l1) * 5 < (l1 - l0) * 4
    finally:
        sim.close()


@pytest.mark.parametrize("dtype", ["c16", "c8"])
def test_point_sources_at_several_x_in_one_batch(dtype):
    # one source description per run: point sources at one z, different x
    # (an extended source spot), against the same sources one by one
    case = _point_case()
    db = [[["Si", 2.34], [2.2888e-7, 2.5847e-10]], [["Au", 19.32], [1.4981e-6, 3.6174e-8]]]
    xs = [0.1e-6, -0.3e-6, 0.45e-6, 0.0]
    runs = [{"energy": 46000.0 + 1000.0 * i, "db_table": db, "weight": 1.0} for i in range(len(xs))]
    srcs = [{"type": "point", "x": x, "z": 0.0} for x in xs]
    sim = Simulation(case, dtype=dtype)
    try:
        lib = rsw.load_library()
        l0 = lib.rsw_launch_count()
        each = sim.run_sources(runs, sources=srcs, each=True).cpu().numpy()
        l1 = lib.rsw_launch_count()
        for r, s_, e in zip(runs, srcs, each):
            sim.reset()
            sim.run_source(energy=r["energy"], db_table=r["db_table"], source=s_)
            assert rel_l2(e, sim.detected()) < TOL
        if dtype == "c8":  # one batch, not four runs
            l2 = lib.rsw_launch_count()
            assert (l1 - l0) * 2 < (l2 - l1)
        # sources at different z cannot share a batch: they run one by one
        mixed = [dict(srcs[0]), dict(srcs[1], z=-0.01)]
        each = sim.run_sources(runs[:2], sources=mixed, each=True).cpu().numpy()
        for r, s_, e in zip(runs[:2], mixed, each):
            sim.reset()
            sim.run_source(energy=r["energy"], db_table=r["db_table"], source=s_)
            assert rel_l2(e, sim.detected()) < TOL
    finally:
        sim.close()


def test_vector_sources_with_their_own_fields():
    case = _talbot_lau("c16")
    n = case["sim_params"]["N"]
    rng = np.random.default_rng(5)
    fields = [np.exp(1j * rng.uniform(-0.1, 0.1, n)) for _ in range(3)]
    runs = [{"energy": e, "db_table": workloads.db_table(e), "weight": 1.0} for e in ENERGIES[:3]]
    srcs = [{"type": "vector", "z": 0.0, "u": f} for f in fields]
    sim = Simulation(case, dtype="c16")
    try:
        each = sim.run_sources(runs, sources=srcs, each=True).cpu().numpy()
        for r, f, e in zip(runs, fields, each):
            sim.reset()
            sim.run_source(energy=r["energy"], db_table=r["db_table"], source={"type": "vector", "z": 0.0}, field=f)
            assert rel_l2(e, sim.detected()) < TOL
    finally:
        sim.close()
