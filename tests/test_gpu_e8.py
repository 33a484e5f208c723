"""Kernels with 8 samples per thread (radix-8 stages, 1024-thread CTAs),
selected with RSW_ROW_E=8 / RSW_COL_E=8, against numpy and the oracle."""

import numpy as np
import pytest

from conftest import rel_l2
from oracle import bigwave_np as bw

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import rave_sim_b200 as rsw  # noqa: E402

TOL = {"c16": 1e-12, "c8": 2e-6}


def cplx(n, seed, dt):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return a.astype(np.complex128 if dt == "c16" else np.complex64)


@pytest.fixture
def e8(monkeypatch):
    def set_e(row, col, split=None):
        monkeypatch.setenv("RSW_ROW_E", str(row))
        monkeypatch.setenv("RSW_COL_E", str(col))
        if split is not None:
            monkeypatch.setenv("RSW_SPLIT", str(split))
    return set_e


@pytest.mark.parametrize("dt", ["c16", "c8"])
@pytest.mark.parametrize("row,col", [(8, 8), (8, 16), (16, 8)])
def test_fft_matches_numpy(dt, row, col, e8):
    e8(row, col, 11)
    n = 1 << 22
    p = rsw.Plan(n, dt)
    x = cplx(n, row + col, dt)
    xd = torch.from_numpy(x).cuda()
    X = p.fft(xd, torch.empty_like(xd))
    ref = np.fft.fft(x.astype(np.complex128))
    assert rel_l2(X.cpu().numpy(), ref) < TOL[dt]
    assert rel_l2(p.ifft(X).cpu().numpy(), x) < TOL[dt]


@pytest.mark.parametrize("dt", ["c16", "c8"])
def test_propagate_matches_oracle(dt, e8):
    e8(8, 8, 11)
    n = 1 << 22
    dx, wl = 2e-9, 2.6953e-11
    sim = bw.Sim(N=n, dx=dx, z_detector=1, detector_size=1e-6, psx=1e-7, psy=1, wl=wl, chunk_size=n)
    u = cplx(n, 9, "c16")
    cut = np.sin(3e-3) / wl
    U0 = np.fft.fft(u)
    u_ref, _ = bw.propagate(u, U0, sim, 0.0818, cut)
    p = rsw.Plan(n, dt)
    ud = torch.from_numpy(u.astype(np.complex128 if dt == "c16" else np.complex64)).cuda()
    p.propagate(ud, None, dx=dx, wl=wl, dz=0.0818, cutoff_freq=cut)
    assert rel_l2(ud.cpu().numpy(), u_ref) < (1e-10 if dt == "c16" else 1e-5)


def test_simulation_matches_default_kernels(e8):
    from rave_sim_b200 import workloads

    case = workloads.talbot_lau(n=1 << 22, dx=8e-9, dtype="c8", nr_steps=3, phase_steps=2)
    e = 30000.0
    c = dict(case, energy=e, db=workloads.db_table(e))
    ref = rsw.run_case(c, dtype="c16")
    e8(8, 8)
    got = rsw.run_case(c, dtype="c8")
    assert rel_l2(got, ref) < 1e-5
