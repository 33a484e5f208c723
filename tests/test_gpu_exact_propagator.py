"""The opt-in exact angular-spectrum propagator (RSW_PROP_EXACT; no
counterpart in the reference, whose transfer function is the Fresnel one)
against its CPU restatement (oracle.bigwave_np.transfer_function_angular):
complex128 rel-L2 <= 1e-10, complex64 <= 1e-5, through the C ABI."""

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

TOL = {"c16": 1e-10, "c8": 1e-5}


def _field(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


@pytest.mark.parametrize("dt", ["c16", "c8"])
@pytest.mark.parametrize("logn,split3", [(12, None), (16, None), (20, None), (20, "c3")])
def test_exact_propagate_matches_oracle(monkeypatch, dt, logn, split3):
    if split3:
        monkeypatch.setenv("RSW_SPLIT3", "4,4,12" if dt == "c16" else "4,4,12")
    n = 1 << logn
    dx, wl, dz = 2e-9, 2.6953e-11, 0.0818
    sim = bw.Sim(N=n, dx=dx, z_detector=1, detector_size=1e-6, psx=1e-7, psy=1, wl=wl, chunk_size=n,
                 propagator="exact")
    u = _field(n, logn)
    cut = np.sin(2e-3) / wl
    u_ref, _ = bw.propagate(u, np.fft.fft(u), sim, dz, cut)
    p = rsw.Plan(n, dt)
    p.set_propagator("exact")
    ud = torch.from_numpy(u.astype(np.complex128 if dt == "c16" else np.complex64)).cuda()
    p.propagate(ud, None, dx=dx, wl=wl, dz=dz, cutoff_freq=cut)
    assert rel_l2(ud.cpu().numpy(), u_ref) < TOL[dt]
    # it is a different kernel from the Fresnel one at these frequencies
    fres, _ = bw.propagate(u, np.fft.fft(u), bw.Sim(**{**sim.__dict__, "propagator": "fresnel"}), dz, cut)
    assert rel_l2(fres, u_ref) > 1e-6


def test_exact_zeroes_evanescent_components():
    # wavelength above twice the sampling: part of the spectrum is evanescent
    n, dx, wl, dz = 1 << 12, 2e-7, 1e-6, 3e-6
    sim = bw.Sim(N=n, dx=dx, z_detector=1, detector_size=1e-6, psx=1e-7, psy=1, wl=wl, chunk_size=n,
                 propagator="exact")
    u = _field(n, 5)
    u_ref, U_ref = bw.propagate(u, np.fft.fft(u), sim, dz, 1.0 / dx)
    assert np.count_nonzero(U_ref == 0) > n // 4
    p = rsw.Plan(n, "c16")
    p.set_propagator("exact")
    ud = torch.from_numpy(u).cuda()
    Ud = torch.empty_like(ud)
    p.propagate(ud, Ud, dx=dx, wl=wl, dz=dz, cutoff_freq=1.0 / dx)
    assert rel_l2(ud.cpu().numpy(), u_ref) < 1e-12
    assert rel_l2(Ud.cpu().numpy(), U_ref) < 1e-12


@pytest.mark.parametrize("dt", ["c16", "c8"])
def test_exact_simulation_config1(dt):
    case = dict(workloads.single_grating(n=1 << 20, dtype=dt), propagator="exact")
    ref = bw.run_simulation(case)
    got = rsw.run_case(case, dtype=dt)
    assert rel_l2(got, ref) < TOL[dt]
    fres = rsw.run_case(dict(case, propagator="fresnel"), dtype="c16")
    assert rel_l2(fres, ref) > 1e-6  # the two kernels give different detector images


def test_unknown_propagator_rejected():
    p = rsw.Plan(1 << 10, "c16")
    with pytest.raises(ValueError):
        p.set_propagator("paraxial")
