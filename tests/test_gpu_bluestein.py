"""Lengths that are not a power of two, and powers of two below 16 (Bluestein
plans), against numpy and the oracle through the C ABI: the FFT both ways and
in place, propagate with the reference's Fresnel kernel and with the exact
kernel (with and without a given spectrum, with a cutoff), the point source
and the detector binning at odd and even N, and the schedule a Bluestein plan
reports. Big-wave runs any N (numpy's FFT; fast-wave's cufftPlan1d takes any
int N); the simulations of the non-power-of-two golden cases run in
test_gpu_parity.py and test_gpu_history.py.

Tolerances: c16 rel-L2 <= 1e-12 (FFT, propagate); c8 <= 5e-6 (three FP32
transforms of length M >= 2N - 1 per FFT, chirps applied in FP64).
"""

import numpy as np
import pytest

from conftest import rel_l2
from oracle import bigwave_np as bw

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import rave_sim_b200 as rsw  # noqa: E402
from rave_sim_b200.autotune import plan_tuning  # noqa: E402

DEV = "cuda"
TOL = {"c16": 1e-12, "c8": 5e-6}
LENGTHS = [1, 2, 3, 5, 6, 8, 12, 15, 100, 1000, 3000, 6561, 12000, 99991, 3 << 18, 1000003]


def cplx(n, seed, dt):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return a.astype(np.complex128 if dt == "c16" else np.complex64)


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


@pytest.mark.parametrize("dt", ["c16", "c8"])
@pytest.mark.parametrize("n", LENGTHS)
def test_fft_matches_numpy(dt, n):
    p = rsw.Plan(n, dt)
    x = cplx(n, n, dt)
    ref = np.fft.fft(x.astype(np.complex128))
    X = p.fft(to_dev(x), torch.empty(n, dtype=p.dtype, device=DEV))
    assert rel_l2(X.cpu().numpy(), ref) < TOL[dt]
    y = p.ifft(X.clone())
    assert rel_l2(y.cpu().numpy(), x) < TOL[dt]
    xd = to_dev(x)
    p.fft(xd)  # in place
    assert rel_l2(xd.cpu().numpy(), ref) < TOL[dt]
    # fast-wave's fft test (fwtest.cu:89-109): ones -> N * delta -> ones
    o = torch.ones(n, dtype=p.dtype, device=DEV)
    p.fft(o)
    d = np.zeros(n)
    d[0] = n
    assert rel_l2(o.cpu().numpy(), d) < TOL[dt]
    p.ifft(o)
    assert rel_l2(o.cpu().numpy(), np.ones(n)) < TOL[dt]


def test_large_odd_length():
    n = 3 ** 15  # 14348907: M = 2^25
    x = cplx(n, 3, "c8")
    ref = np.fft.fft(x.astype(np.complex128))
    for dt in ("c16", "c8"):
        p = rsw.Plan(n, dt)
        X = p.fft(to_dev(x.astype(np.complex128 if dt == "c16" else np.complex64)))
        assert rel_l2(X.cpu().numpy(), ref) < TOL[dt]


@pytest.mark.parametrize("dt", ["c16", "c8"])
@pytest.mark.parametrize("n", [6, 6561, 12000, 3 << 16])
@pytest.mark.parametrize("skip", [False, True])
@pytest.mark.parametrize("prop", ["fresnel", "exact"])
def test_propagate_matches_oracle(dt, n, skip, prop):
    dx, wl, dz = 2e-9, 2.6953e-11, 0.0818
    sim = bw.Sim(N=n, dx=dx, z_detector=1, detector_size=1e-6, psx=1e-7, psy=1, wl=wl, chunk_size=n)
    sim.propagator = prop
    u = cplx(n, n + 1, "c16")
    cut = np.sin(3e-3) / wl
    U0 = np.fft.fft(u)
    u_ref, U_ref = bw.propagate(u, U0, sim, dz, cut, skip_fft=skip)
    p = rsw.Plan(n, dt)
    p.set_propagator(prop)
    cd = np.complex128 if dt == "c16" else np.complex64
    ud = to_dev(u.astype(cd))
    Ud = to_dev(U0.astype(cd)) if skip else torch.empty(n, dtype=p.dtype, device=DEV)
    p.propagate(ud, Ud, dx=dx, wl=wl, dz=dz, cutoff_freq=cut, skip_fft=skip)
    assert rel_l2(ud.cpu().numpy(), u_ref) < TOL[dt]
    assert rel_l2(Ud.cpu().numpy(), U_ref) < TOL[dt]
    # without a spectrum buffer
    ud = to_dev(u.astype(cd))
    p.propagate(ud, None, dx=dx, wl=wl, dz=dz, cutoff_freq=cut)
    u_ns, _ = bw.propagate(u, None, sim, dz, cut)
    assert rel_l2(ud.cpu().numpy(), u_ns) < TOL[dt]


@pytest.mark.parametrize("n", [6, 7, 6561, 12000])
def test_point_source_and_binning(n):
    dx, wl = 3.1e-10, 2.67e-11
    sim = bw.Sim(N=n, dx=dx, z_detector=1, detector_size=1e-6, psx=1e-7, psy=1, wl=wl, chunk_size=n)
    ref = bw.point_source_field(sim, 0.1, 0.44e-9 * n, np.complex128)
    p = rsw.Plan(n, "c16")
    got = p.point_source(torch.empty(n, dtype=torch.complex128, device=DEV), dx=dx, wl=wl, z=0.1,
                         x_source=0.44e-9 * n).cpu().numpy()
    assert rel_l2(got, ref) < 1e-13
    u = cplx(n, 2 * n, "c16")
    for det, psx in [(n * dx * 0.8, dx * 2.5), (n * dx * 1.5, dx * 3), (7.5 * dx, dx)]:
        s2 = bw.Sim(N=n, dx=dx, z_detector=1.3, detector_size=det, psx=psx, psy=2.0, wl=wl, chunk_size=n)
        r = bw.square_and_downsample(u, s2, 1.3)
        g = p.square_and_downsample(to_dev(u), dx=dx, detector_size=det, pixel_size_x=psx, pixel_size_y=2.0,
                                    z=1.3).cpu().numpy()
        assert g.shape == r.shape
        assert rel_l2(g, r) < 1e-13


def test_bluestein_plan_reports_its_power_of_two_schedule():
    p = rsw.Plan(12000, "c8")
    info = p.info()
    assert info["n"] == 12000 and info["log_rows"] == 0 and info["log_cols"] == 0
    t = plan_tuning(p)
    inner = plan_tuning(rsw.Plan(1 << 15, "c8"))  # M = 2^15 >= 2 * 12000 - 1
    assert t == inner
