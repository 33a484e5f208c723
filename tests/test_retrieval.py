"""Phase-stepping signal retrieval (the crack-simulation notebook's
signal_retrieval_least_squares, notebooks/Crack_simulation.ipynb cell 4): the
numpy restatement in oracle/retrieval_np.py and the device implementation,
both against the notebook function itself (tests/golden/retrieval.npz, made
by tests/golden/make_retrieval_golden.py, which runs the notebook cell)."""

import numpy as np
import pytest

from conftest import GOLDEN, load_case
from oracle import retrieval_np as ro


def golden_cases():
    """(data [steps][pixels], period, dabs, dphase, dvis, mean chi2) of the
    notebook function's runs."""
    d = np.load(GOLDEN / "retrieval.npz")
    return [(d[f"data_{i}"], float(d[f"period_{i}"]), d[f"dabs_{i}"], d[f"dphase_{i}"], d[f"dvis_{i}"],
             float(d[f"chi2_{i}"])) for i in range(int(d["n_cases"]))]


def check_against_golden(got, ref, chi2=True):
    data, period, dabs, dphase, dvis, c2 = ref
    np.testing.assert_allclose(got[0], dabs, rtol=1e-12)
    np.testing.assert_allclose(got[1], dphase, atol=1e-12)
    np.testing.assert_allclose(got[2], dvis, rtol=1e-11)
    if chi2:
        assert got[3] == pytest.approx(c2, rel=1e-9, abs=1e-24)


def test_oracle_matches_notebook_function():
    for ref in golden_cases():
        got = ro.signal_retrieval_least_squares(ref[0], period=ref[1], axis=0)
        check_against_golden(got, ref)


def curves(n_pix, nsteps, period, seed):
    rng = np.random.default_rng(seed)
    a, b = rng.normal(size=(2, n_pix))
    c = rng.uniform(2.0, 5.0, n_pix)
    phi = np.linspace(0, 2 * np.pi * nsteps / period, nsteps, endpoint=False)
    data = a[:, None] * np.sin(phi) + b[:, None] * np.cos(phi) + c[:, None]
    return data, a, b, c


# ------------------------------------------------------------------ oracle
@pytest.mark.parametrize("nsteps,period", [(4, 4), (5, 5), (8, 8), (7, 9.5)])
def test_oracle_recovers_exact_curves(nsteps, period):
    data, a, b, c = curves(50, nsteps, period, nsteps)
    dabs, dphase, dvis, chi2, _ = ro.signal_retrieval_least_squares(data, period=period)
    np.testing.assert_allclose(dabs, nsteps * c, rtol=1e-12)
    np.testing.assert_allclose(dphase, -np.arctan2(a, b), atol=1e-12)
    np.testing.assert_allclose(dvis, np.sqrt(a * a + b * b) / c, rtol=1e-11)
    assert chi2 < 1e-20


def test_oracle_axis_matches_last_axis():
    data, *_ = curves(30, 6, 6, 1)
    r0 = ro.signal_retrieval_least_squares(data.T, axis=0)
    r1 = ro.signal_retrieval_least_squares(data)
    for x, y in zip(r0[:3], r1[:3]):
        np.testing.assert_allclose(x, y, rtol=1e-14)


# ---------------------------------------------------------------- device
gpu = pytest.mark.gpu


def _need_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


@gpu
@pytest.mark.parametrize("nsteps,period", [(3, 3), (4, 4), (8, 8), (5, 7.25), (64, 64)])
def test_device_matches_oracle(nsteps, period):
    _need_cuda()
    from rave_sim_b200 import signal_retrieval_least_squares

    rng = np.random.default_rng(nsteps)
    data, *_ = curves(1000, nsteps, period, nsteps)
    data += rng.normal(scale=0.05, size=data.shape)  # residuals
    got = signal_retrieval_least_squares(data, period=period)
    ref = ro.signal_retrieval_least_squares(data, period=period)
    np.testing.assert_allclose(got[0], ref[0], rtol=1e-12)
    np.testing.assert_allclose(got[1], ref[1], atol=1e-12)
    np.testing.assert_allclose(got[2], ref[2], rtol=1e-11)
    if nsteps > 3:
        assert got[3] == pytest.approx(ref[3], rel=1e-9)


@gpu
def test_device_on_detector_output_and_axes():
    torch = _need_cuda()
    import rave_sim_b200 as rsw

    case, grids, d = load_case("tl3g_point_phase")
    det = rsw.run_case(case, grids, dtype="c16")  # (phase steps, pixels)
    ref = ro.signal_retrieval_least_squares(det, axis=0)
    got = rsw.signal_retrieval_least_squares(det, axis=0)
    np.testing.assert_allclose(got[0], ref[0], rtol=1e-12)
    np.testing.assert_allclose(got[2], ref[2], rtol=1e-10)
    dev = rsw.signal_retrieval_least_squares(torch.from_numpy(det).cuda(), axis=0)
    assert dev[0].is_cuda
    np.testing.assert_allclose(dev[0].cpu().numpy(), ref[0], rtol=1e-12)
    t, dphi, df = rsw.dark_field(det, det)
    np.testing.assert_allclose(t, 1.0, rtol=1e-14)
    np.testing.assert_allclose(dphi, 0.0, atol=1e-14)
    np.testing.assert_allclose(df, 1.0, rtol=1e-14)


@gpu
def test_device_rejects_bad_step_counts():
    _need_cuda()
    from rave_sim_b200 import RswError, signal_retrieval_least_squares

    with pytest.raises(RswError):
        signal_retrieval_least_squares(np.ones((10, 2)), axis=-1)
    with pytest.raises(RswError):
        signal_retrieval_least_squares(np.ones((10, 65)), axis=-1)


@gpu
def test_device_matches_notebook_function():
    _need_cuda()
    from rave_sim_b200 import signal_retrieval_least_squares

    for ref in golden_cases():
        got = signal_retrieval_least_squares(ref[0], period=ref[1], axis=0)
        check_against_golden(got, ref, chi2=ref[0].shape[0] > 3)
