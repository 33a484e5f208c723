"""GPU parity of the CUDA engine against the CPU oracle and the reference's
golden vectors. Every call goes through the C ABI (librsw.so via ctypes).

Tolerances:
  c16 (FP64) detector output: rel-L2 <= 1e-10 vs the reference's FP64 output;
  c16 FFT: rel-L2 <= 1e-12; c16 propagate on white-spectrum random fields:
      rel-L2 <= 1e-10 vs the reference's rounded phase and <= 1e-13 vs the
      exactly evaluated phase (the engine evaluates c*fx^2 without the
      reference's intermediate roundings on two-level plans);
  c8  (FP32 fields, FP64 phases and sums) detector output: rel-L2 <= 1e-5
      vs the FP64 reference, FFT rel-L2 <= 2e-6.
"""

import json

import numpy as np
import pytest

from conftest import case_names, load_case, load_snapshot_case, rel_l2
from oracle import bigwave_np as bw

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import rave_sim_b200 as rsw  # noqa: E402

DEV = "cuda"
TOL_FFT = {"c16": 1e-12, "c8": 2e-6}


def cplx(n, seed, dt):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return a.astype(np.complex128 if dt == "c16" else np.complex64)


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


@pytest.mark.parametrize("dt", ["c16", "c8"])
@pytest.mark.parametrize("logn", [4, 5, 7, 9, 12, 13, 14, 15, 17, 20])
def test_fft_matches_numpy(dt, logn):
    n = 1 << logn
    p = rsw.Plan(n, dt)
    x = cplx(n, logn, dt)
    X = p.fft(to_dev(x), torch.empty(n, dtype=p.dtype, device=DEV))
    ref = np.fft.fft(x.astype(np.complex128))
    assert rel_l2(X.cpu().numpy(), ref) < TOL_FFT[dt]
    # fast-wave fft test (fwtest.cu:89-109): ones -> N * delta, inverse -> ones
    y = p.ifft(X.clone())
    assert rel_l2(y.cpu().numpy(), x) < TOL_FFT[dt]
    # in place
    xd = to_dev(x)
    p.fft(xd)
    assert rel_l2(xd.cpu().numpy(), ref) < TOL_FFT[dt]


def test_fft_golden_fastwave():
    # fast-wave/test/fwtest.cu:111-127 (np.fft.fft of an 8-vector), zero-padded
    # to the minimum plan length by running it as a 16-periodic sequence
    x = np.array([0, 0, 1, 2 + 1j, 3 + 2j, 2, 1, 0], dtype=np.complex128)
    expected = np.array([9 + 3j, -5.12132034 - 2.70710678j, 2j, 0.53553391 - 1.29289322j,
                         1 + 1j, -0.87867966 - 1.29289322j, 2 + 2j, -6.53553391 - 2.70710678j])
    p = rsw.Plan(16, "c16")
    X = p.fft(to_dev(np.tile(x, 2))).cpu().numpy()
    # a period-8 sequence repeated twice has its spectrum on the even bins, doubled
    np.testing.assert_allclose(X[0::2] / 2, expected, atol=1e-7)
    np.testing.assert_allclose(X[1::2], 0, atol=1e-12)


@pytest.mark.parametrize("dt", ["c16", "c8"])
@pytest.mark.parametrize("logn,skip", [(10, False), (16, False), (16, True), (20, False)])
def test_propagate_matches_oracle(dt, logn, skip):
    n = 1 << logn
    dx, wl = 2e-9, 2.6953e-11
    sim = bw.Sim(N=n, dx=dx, z_detector=1, detector_size=1e-6, psx=1e-7, psy=1, wl=wl, chunk_size=n)
    u = cplx(n, 3, "c16")
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
        u_ex, U_ex = bw.propagate(u, U0, sim, 0.0818, cut, skip_fft=skip, exact_phase=True)
        exact = p.info()["log_rows"] > 0  # two-level plans use the exact phase
        assert rel_l2(ud.cpu().numpy(), u_ex if exact else u_ref) < 1e-13
    if not skip:
        ud2 = to_dev(u.astype(np.complex128 if dt == "c16" else np.complex64))
        p.propagate(ud2, None, dx=dx, wl=wl, dz=0.0818, cutoff_freq=cut)
        assert rel_l2(ud2.cpu().numpy(), u_ref) < tol


@pytest.mark.parametrize("chunk", [0, 4096, 3001])
def test_grating_and_dba_masks(chunk):
    """Mask decisions are bit-exact: with u = 1 the product equals the chosen
    factor exactly; with a random u it agrees to rounding (FMA in the complex
    product)."""
    n = 1 << 14
    dx = 1e-9
    sim = bw.Sim(N=n, dx=dx, z_detector=1, detector_size=1e-6, psx=1e-7, psy=1, wl=1e-11,
                 chunk_size=chunk if chunk else n)
    p = rsw.Plan(n, "c16")
    ones = np.ones(n, np.complex128)
    u = cplx(n, 5, "c16")
    fa, fb = 0.3 + 0.8j, -0.5 + 0.1j
    for pitch, dc, xpos in [(4.2e-6, 0.5, 0.0), (1.3e-6, 0.37, 0.211e-6), (2e-9 * 7, 0.45, -3.3e-9)]:
        def g(s, c):
            return bw.grating_mask_chunk(dx, s, c, pitch, dc, xpos)

        def d(s, c):
            return bw.dba_mask_chunk(dx, s, c, pitch, 3.1 * pitch, dc, 0.6, xpos)

        kw = dict(dx=dx, chunk_size=chunk, x_position=xpos, factor_a=fa, factor_b=fb)
        for v in (ones, u):
            exact = v is ones
            ref = bw._apply_binary(v, sim, g, fa, fb)
            got = p.apply_grating(to_dev(v), pitch=pitch, dc=dc, **kw).cpu().numpy()
            assert np.array_equal(got, ref) if exact else rel_l2(got, ref) < 1e-15
            ref = bw._apply_binary(v, sim, d, fa, fb)
            got = p.apply_dba_grating(to_dev(v), pitch0=pitch, pitch1=3.1 * pitch, dc0=dc, dc1=0.6,
                                      **kw).cpu().numpy()
            assert np.array_equal(got, ref) if exact else rel_l2(got, ref) < 1e-15


def test_sample_row():
    n = 1 << 13
    dx = 1e-9
    wl = 3e-11
    rng = np.random.default_rng(1)
    mats = np.array([0, 1e-6 + 2e-9j, 3e-7 + 1e-10j, 2e-6 + 5e-8j])
    grid = rng.integers(0, 4, size=53)
    row_db = mats[grid]
    psx, psz, xpos = 0.11e-6, 5e-6, 0.123e-6
    row_x = bw.sample_row_coordinates(len(grid), psx, xpos)
    x = (np.arange(n) - n / 2) * dx
    ref = cplx(n, 2, "c16") * bw.material_factor(np.interp(x, row_x, row_db, left=0.0, right=0.0), psz, wl)
    p = rsw.Plan(n, "c16")
    got = p.apply_sample_row(to_dev(cplx(n, 2, "c16")), dx=dx, wl=wl, dz=psz, pixel_size_x=psx,
                             x_position=xpos, row_db=row_db).cpu().numpy()
    assert rel_l2(got, ref) < 1e-14


@pytest.mark.parametrize("dt", ["c16", "c8"])
def test_square_and_downsample(dt):
    n = 1 << 12
    u = cplx(n, 9, dt)
    p = rsw.Plan(n, dt)
    for dx, det, psx, psy, z in [(0.5, 300.0, 1.0, 1.0, 1.0), (2e-9, 7e-6, 1e-7, 1e-6, 0.3),
                                 (3.1e-10, 1e-6, 3.1e-10 * 7.5, 1.0, 1.77)]:
        sim = bw.Sim(N=n, dx=dx, z_detector=z, detector_size=det, psx=psx, psy=psy, wl=1, chunk_size=n)
        ref = bw.square_and_downsample(u.astype(np.complex128), sim, z)
        got = p.square_and_downsample(to_dev(u), dx=dx, detector_size=det, pixel_size_x=psx,
                                      pixel_size_y=psy, z=z).cpu().numpy()
        assert got.shape == ref.shape
        assert rel_l2(got, ref) < (1e-13 if dt == "c16" else 1e-6)


def test_point_source():
    n = 1 << 14
    dx, wl = 3.1e-10, 2.67e-11
    sim = bw.Sim(N=n, dx=dx, z_detector=1, detector_size=1e-6, psx=1e-7, psy=1, wl=wl, chunk_size=n)
    ref = bw.point_source_field(sim, 0.1, 0.44e-6, np.complex128)
    p = rsw.Plan(n, "c16")
    got = p.point_source(torch.empty(n, dtype=torch.complex128, device=DEV), dx=dx, wl=wl, z=0.1,
                         x_source=0.44e-6).cpu().numpy()
    assert rel_l2(got, ref) < 1e-13


@pytest.mark.parametrize("name", case_names())
def test_golden_case_c16(name):
    case, grids, d = load_case(name)
    det = rsw.run_case(case, grids, dtype="c16")
    assert det.shape == d["detected"].shape
    assert rel_l2(det, d["detected"]) < 1e-10


@pytest.mark.parametrize("name", case_names())
def test_golden_case_c8(name):
    case, grids, d = load_case(name)
    det = rsw.run_case(case, grids, dtype="c8")
    assert rel_l2(det, d["detected"]) < 1e-5


def test_golden_final_fields():
    for name in case_names():
        case, grids, d = load_case(name)
        if "u_final" not in d or len(case["elements"][0]["x_positions"]) > 1:
            continue
        sim = rsw.Simulation(case, grids, dtype="c16", cutoff_angles=case["cutoff_angles"])
        sim.run_source(energy=case["energy"], db_table=case["db"], source=case["source"])
        u = sim.final_field().cpu().numpy()
        assert rel_l2(u, d["u_final"]) < 1e-10, name


def test_snapshot_golden():
    # big-wave/test.py:853-960: 3-grating Talbot-Lau, point source, N = 2^19
    case, d = load_snapshot_case()
    det = rsw.run_case(case, dtype="c16")
    assert np.allclose(det[0], d["known_data"], rtol=0, atol=1e-14)
    assert rel_l2(det, d["detected"]) < 1e-10


def test_config1_full_size():
    """Config 1 at its full size: plane wave, one pi-phase Si grating at 46 keV,
    N = 2^20 complex128, dx = 2 nm, gap p^2/(8 wl), 1 um pixels."""
    wl = bw.wavelength_from_energy(46000.0)
    p = 4.2e-6
    h = wl / (2 * 2.27e-7)
    d = p * p / (8 * wl)
    n = 1 << 20
    case = {
        "sim_params": {"N": n, "dx": 2e-9, "z_detector": 0.1 + h + d, "detector_size": 2.048e-3,
                       "detector_pixel_size_x": 1e-6, "detector_pixel_size_y": 1.0, "chunk_size": n},
        "elements": [{"type": "grating", "pitch": p, "dc": [0.5, 0.5], "z_start": 0.1, "thickness": h,
                      "nr_steps": 10, "x_positions": [0.0], "substrate_thickness": 0.0,
                      "mat_a": ["Si", 2.34], "mat_b": None, "mat_substrate": None}],
        "source": {"type": "plane", "z": 0.1}, "energy": 46000.0,
        "db": [[["Si", 2.34], [2.27e-7, 1e-10]]], "cutoff_angles": [np.pi / 2] * 2,
    }
    ref = bw.run_simulation(case)
    got = rsw.run_case(case, dtype="c16")
    assert rel_l2(got, ref) < 1e-10
    got8 = rsw.run_case(case, dtype="c8")
    assert rel_l2(got8, ref) < 1e-5


def test_errors_are_raised():
    with pytest.raises(rsw.RswError):
        rsw.Plan(0, "c16")
    with pytest.raises(rsw.RswError):
        rsw.Plan((1 << 31) + 1, "c16")  # Bluestein lengths end at 2^31
    with pytest.raises(ValueError):
        rsw.Plan(1 << 10, "c16").set_propagator("angular")
    p = rsw.Plan(1 << 10, "c16")
    with pytest.raises(ValueError):
        p.fft(torch.zeros(10, dtype=torch.complex128, device=DEV))
