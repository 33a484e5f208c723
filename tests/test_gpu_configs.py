"""Parity on the shapes of the benchmark configurations (configs 2-5), through
the C ABI.

Tolerances (detector intensity, rel-L2):
  complex128 against the CPU oracle (the FP64 restatement of big-wave):
      <= 1e-10;
  complex64 against complex128 on the same inputs: <= 1e-5 (the mixed
      precision tolerance of the complex64 path; the complex128 run is the
      oracle of full-size cases, itself pinned to the CPU oracle).

Cases:
  * config 4 (thick sample) scaled to 2^18 samples: the interferometer with a
    200-slice cracked cylinder, 2 phase steps, complex128 vs the CPU oracle
    and complex64 vs both;
  * config 4 at its full size (2^26 samples, 200 slices, 1 energy, 2 phase
    steps): complex64 vs complex128 (three-level complex128 plan);
  * config 2 at its full N = 2^24 (1 energy, 2 phase steps, 2 grating
    sub-steps): complex128 vs the CPU oracle;
  * config 3 (energies on fields of different lengths) and config 5 (fields
    above the two-level limit, forced three-level splits) at reduced sizes:
    complex64 vs complex128;
  * complex64 rows of 2^13 in two-level plans (N = 2^20 split 2^7 x 2^13, the
    two-CTA-per-SM row kernel): FFT vs numpy and propagate vs the oracle.
"""

import os

import numpy as np
import pytest

from conftest import rel_l2
from oracle import bigwave_np as bw

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import rave_sim_b200 as rsw  # noqa: E402
from rave_sim_b200 import workloads  # noqa: E402

TOL_C16 = 1e-10
TOL_C8 = 1e-5


def _oracle(case, grids=None):
    import scipy.fft as spfft

    with spfft.set_workers(os.cpu_count() or 1):
        return bw.run_simulation(case, grids=grids)


def _small_thick_sample():
    """Config 4 scaled down: 2^18 samples of 100 nm (26 um), a 20 um cracked
    aluminium cylinder of 200 x 200 pixels of 0.1 um, 0.5 um detector pixels."""
    case, grids = workloads.thick_sample(
        n=1 << 18, dx=100e-9, dtype="c16", nr_steps=10, phase_steps=2, rows=200, cols=200,
        psz=0.1e-6, psx=0.1e-6, diameter=20e-6, axis_range=(0.2e-6, 1.5e-6), seed=4,
        detector_size=20e-6, pixel_size=0.5e-6)
    return case, grids


def test_config4_scaled_against_oracle():
    case, grids = _small_thick_sample()
    ref = _oracle(case, grids)
    c16 = rsw.run_case(case, grids=grids, dtype="c16")
    c8 = rsw.run_case(case, grids=grids, dtype="c8")
    assert ref.shape == c16.shape == (2, 40)
    assert rel_l2(c16, ref) < TOL_C16
    assert rel_l2(c8, c16) < TOL_C8
    assert rel_l2(c8, ref) < TOL_C8


def test_config4_full_size_mixed_vs_fp64():
    case, grids = workloads.thick_sample(n=1 << 26, dtype="c16", phase_steps=2)
    e = 40000.0
    case = dict(case, energy=e, db=workloads.db_table_sample(e))
    c16 = rsw.run_case(case, grids=grids, dtype="c16")
    torch.cuda.empty_cache()
    c8 = rsw.run_case(case, grids=grids, dtype="c8")
    assert np.all(np.isfinite(c8)) and c16.max() > 0
    assert rel_l2(c8, c16) < TOL_C8


def test_config2_full_n_against_oracle():
    case = workloads.talbot_lau(n=1 << 24, dtype="c16", nr_steps=2, phase_steps=2)
    e = 52000.0
    case = dict(case, energy=e, db=workloads.db_table(e))
    ref = _oracle(case)
    got = rsw.run_case(case, dtype="c16")
    assert got.shape == (2, 2048)
    assert rel_l2(got, ref) < TOL_C16


def test_config3_scaled_mixed_vs_fp64():
    groups = workloads.batched_energies(count=6, log_min=16, log_max=18, window=float(1 << 18) * 4e-9,
                                        nr_steps=4, phase_steps=4)
    assert [int(g[0]["sim_params"]["N"]) for g in groups] == [1 << 16, 1 << 17, 1 << 18]
    tot = {"c8": 0.0, "c16": 0.0}
    for case, energies, weights in groups:
        for dt in ("c8", "c16"):
            sim = rsw.Simulation(case, dtype=dt)
            try:
                sim.reset()
                for e, w in zip(energies, weights):
                    sim.run_source(energy=float(e), db_table=workloads.db_table(float(e)),
                                   source=case["source"], weight=float(w))
                tot[dt] = tot[dt] + sim.detected()
            finally:
                sim.close()
    assert rel_l2(tot["c8"], tot["c16"]) < TOL_C8


@pytest.mark.parametrize("dt,split", [("c8", "4,4,14"), ("c16", "4,5,13")])
def test_config5_three_level_mixed_vs_fp64(monkeypatch, dt, split):
    """Config 5's plans are three-level; forced here at 2^22 samples. The
    three-level result matches the two-level one of the same dtype, and the
    complex64 one matches the complex128 two-level one."""
    case = workloads.large_field(dtype=dt, n=1 << 22, nr_steps=4, phase_steps=2)
    e = 46000.0
    case = dict(case, energy=e, db=workloads.db_table(e))
    two = rsw.run_case(case, dtype=dt)
    ref16 = two if dt == "c16" else rsw.run_case(case, dtype="c16")
    monkeypatch.setenv("RSW_SPLIT3", split)
    three = rsw.run_case(case, dtype=dt)
    assert rel_l2(three, two) < (1e-12 if dt == "c16" else 2e-6)
    assert rel_l2(three, ref16) < (1e-12 if dt == "c16" else TOL_C8)


def test_c8_two_level_rows_of_2_13(monkeypatch):
    monkeypatch.setenv("RSW_SPLIT", "7")
    n = 1 << 20
    p = rsw.Plan(n, "c8")
    assert p.info()["log_cols"] == 13
    rng = np.random.default_rng(13)
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    xd = torch.from_numpy(x).cuda()
    X = p.fft(xd, torch.empty_like(xd))
    ref = np.fft.fft(x.astype(np.complex128))
    assert rel_l2(X.cpu().numpy(), ref) < 2e-6
    assert rel_l2(p.ifft(X).cpu().numpy(), x) < 2e-6
    dx, wl = 2e-9, 2.6953e-11
    sim = bw.Sim(N=n, dx=dx, z_detector=1, detector_size=1e-6, psx=1e-7, psy=1, wl=wl, chunk_size=n)
    u = x.astype(np.complex128)
    cut = np.sin(3e-3) / wl
    u_ref, _ = bw.propagate(u, np.fft.fft(u), sim, 0.0818, cut)
    ud = torch.from_numpy(x.copy()).cuda()
    p.propagate(ud, None, dx=dx, wl=wl, dz=0.0818, cutoff_freq=cut)
    assert rel_l2(ud.cpu().numpy(), u_ref) < TOL_C8
