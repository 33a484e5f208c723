"""Three-level plans (N = N1 x Nb x Nr, four passes per split step).

Plans switch to three levels above the two-level limit: 2^24 samples for
complex128 and 2^26 for complex64. Here the split is forced on small
fields with RSW_SPLIT3 = "l1,lb,lr", so that the oracle, numpy and the
golden fixtures can check it. The last tests create plans above the limit
without an override.
"""

import numpy as np
import pytest

from conftest import case_names, load_case, load_snapshot_case, rel_l2
from oracle import bigwave_np as bw

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import rave_sim_b200 as rsw  # noqa: E402
from rave_sim_b200 import workloads  # noqa: E402
from rave_sim_b200.autotune import plan_tuning  # noqa: E402

DEV = "cuda"
TOL_FFT = {"c16": 1e-12, "c8": 2e-6}


@pytest.fixture
def split3(monkeypatch):
    def set_split(l1, lb, lr):
        monkeypatch.setenv("RSW_SPLIT3", f"{l1},{lb},{lr}")
    return set_split


def cplx(n, seed, dt):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return a.astype(np.complex128 if dt == "c16" else np.complex64)


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def split_for(logn):
    return 4, logn - 11, 7


@pytest.mark.parametrize("dt", ["c16", "c8"])
@pytest.mark.parametrize("split", [(4, 4, 7), (5, 4, 8), (4, 6, 10), (6, 6, 8), (7, 5, 9)])
def test_fft_matches_numpy(dt, split, split3):
    split3(*split)
    n = 1 << sum(split)
    p = rsw.Plan(n, dt)
    info = p.info()
    assert info["log_rows"] == split[0] and info["log_cols"] == split[1] + split[2]
    x = cplx(n, sum(split), dt)
    X = p.fft(to_dev(x), torch.empty(n, dtype=p.dtype, device=DEV))
    ref = np.fft.fft(x.astype(np.complex128))
    assert rel_l2(X.cpu().numpy(), ref) < TOL_FFT[dt]
    y = p.ifft(X.clone())
    assert rel_l2(y.cpu().numpy(), x) < TOL_FFT[dt]


@pytest.mark.parametrize("dt", ["c16", "c8"])
@pytest.mark.parametrize("split,skip", [((4, 5, 7), False), ((4, 5, 7), True), ((6, 6, 8), False)])
def test_propagate_matches_oracle(dt, split, skip, split3):
    split3(*split)
    n = 1 << sum(split)
    dx, wl = 2e-9, 2.6953e-11
    sim = bw.Sim(N=n, dx=dx, z_detector=1, detector_size=1e-6, psx=1e-7, psy=1, wl=wl, chunk_size=n)
    u = cplx(n, 5, "c16")
    cut = np.sin(3e-3) / wl
    U0 = np.fft.fft(u)
    u_ref, U_ref = bw.propagate(u, U0, sim, 0.0818, cut, skip_fft=skip)
    p = rsw.Plan(n, dt)
    ud = to_dev(u.astype(np.complex128 if dt == "c16" else np.complex64))
    Ud = to_dev(U0.astype(np.complex128 if dt == "c16" else np.complex64)) if skip else \
        torch.empty(n, dtype=p.dtype, device=DEV)
    p.propagate(ud, Ud, dx=dx, wl=wl, dz=0.0818, cutoff_freq=cut, skip_fft=skip)
    tol = 1e-10 if dt == "c16" else 1e-5
    assert rel_l2(ud.cpu().numpy(), u_ref) < tol
    assert rel_l2(Ud.cpu().numpy(), U_ref) < tol
    if dt == "c16":
        u_ex, _ = bw.propagate(u, U0, sim, 0.0818, cut, skip_fft=skip, exact_phase=True)
        assert rel_l2(ud.cpu().numpy(), u_ex) < 1e-13


@pytest.mark.parametrize("name", case_names())
def test_golden_cases(name, split3):
    case, grids, d = load_case(name)
    logn = int(np.log2(case["sim_params"]["N"]))
    if logn < 15:
        pytest.skip("three-level plans need N >= 2^15")
    split3(*split_for(logn))
    det = rsw.run_case(case, grids, dtype="c16")
    assert rel_l2(det, d["detected"]) < 1e-10
    det8 = rsw.run_case(case, grids, dtype="c8")
    assert rel_l2(det8, d["detected"]) < 1e-5


def test_snapshot_golden(split3):
    # big-wave/test.py:853-960 at N = 2^19, split 2^6 x 2^6 x 2^7
    split3(6, 6, 7)
    case, d = load_snapshot_case()
    det = rsw.run_case(case, dtype="c16")
    assert np.allclose(det[0], d["known_data"], rtol=0, atol=1e-14)


def test_three_level_matches_two_level_talbot_lau(split3):
    case = workloads.talbot_lau(n=1 << 20, dx=8e-9, dtype="c16", nr_steps=3, phase_steps=2)
    e = 30000.0
    two = rsw.run_case(dict(case, energy=e, db=workloads.db_table(e)), dtype="c16")
    split3(6, 6, 8)
    three = rsw.run_case(dict(case, energy=e, db=workloads.db_table(e)), dtype="c16")
    assert rel_l2(three, two) < 1e-12


# 2^25 c16: two levels with columns of 2^12 (two-column tiles); 2^26 c16 and
# 2^27 c8: three levels
@pytest.mark.parametrize("dt,logn,levels", [("c16", 25, 2), ("c16", 26, 3), ("c8", 27, 3)])
def test_plans_above_the_two_level_limit(dt, logn, levels):
    n = 1 << logn
    p = rsw.Plan(n, dt)
    info = p.info()
    assert info["log_rows"] + info["log_cols"] == logn
    assert plan_tuning(p)["levels"] == levels
    x = to_dev(cplx(n, 11, dt))
    X = p.fft(x, torch.empty_like(x))
    ref = torch.fft.fft(x.to(torch.complex128))
    err = float(torch.linalg.vector_norm(X.to(torch.complex128) - ref) / torch.linalg.vector_norm(ref))
    assert err < TOL_FFT[dt]
    y = p.ifft(X)
    err = float(torch.linalg.vector_norm((y - x).to(torch.complex128)) / torch.linalg.vector_norm(x.to(torch.complex128)))
    assert err < TOL_FFT[dt]
