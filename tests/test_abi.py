"""C-ABI checks that need no GPU: the library loads, exports every entry point
declared in include/rsw.h with matching struct layouts, validates arguments
before touching the device, and its host-side detector geometry reproduces
np.histogram binning (big-wave/propagation.py:279-320)."""

import ctypes as C
import re

import numpy as np
import pytest

from conftest import ROOT
from oracle import bigwave_np as bw
from rave_sim_b200 import _lib as L


def header_functions():
    txt = (ROOT / "include" / "rsw.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(rsw_[a-z0-9_]+)\s*\(", txt)))


def test_every_header_symbol_exported_and_bound():
    lib = L.load()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
        assert n in L.SIGNATURES, f"{n} has no ctypes signature"
    assert lib.rsw_abi_version() == 1


def test_struct_layouts():
    lib = L.load()
    for i, st in enumerate((L.Element, L.SimDesc, L.Source, L.SourceRun)):
        assert lib.rsw_struct_size(i) == C.sizeof(st)


def test_invalid_sizes_rejected_without_device():
    lib = L.load()
    h = C.c_void_p()
    # any length from 1 to 2^31 is planned (Bluestein's algorithm where it is
    # not a power of two >= 16); these are refused before any device call
    for n, code in [(0, L.RSW_ERR_UNSUPPORTED), (-6, L.RSW_ERR_UNSUPPORTED),
                    ((1 << 31) + 1, L.RSW_ERR_UNSUPPORTED), (3 << 31, L.RSW_ERR_UNSUPPORTED),
                    (1 << 40, L.RSW_ERR_UNSUPPORTED)]:
        st = lib.rsw_plan_create(C.byref(h), n, L.RSW_C128)
        assert st == code, (n, st)
        assert lib.rsw_last_error()
    assert lib.rsw_plan_create(C.byref(h), 1 << 10, 7) == L.RSW_ERR_INVALID
    assert lib.rsw_plan_create(None, 1 << 10, 0) == L.RSW_ERR_INVALID


def geometry(n, dx, det, psx, z):
    lib = L.load()
    npx = C.c_int64()
    L.check(lib.rsw_detector_geometry(n, dx, det, psx, z, C.byref(npx), None, None, None))
    b = np.zeros(npx.value + 1, np.int64)
    cs = np.zeros(max(npx.value, 1))
    rv = np.zeros(max(npx.value, 1))
    L.check(lib.rsw_detector_geometry(n, dx, det, psx, z, C.byref(npx),
                                      b.ctypes.data_as(C.POINTER(C.c_int64)),
                                      cs.ctypes.data_as(L._DP), rv.ctypes.data_as(L._DP)))
    return b, cs[:npx.value], rv[:npx.value]


def detect_host(u, n, dx, det, psx, psy, z):
    b, cs, rv = geometry(n, dx, det, psx, z)
    w = u.real * u.real + u.imag * u.imag
    raw = np.array([w[b[j]:b[j + 1]].sum() for j in range(len(b) - 1)])
    return raw * cs * dx * psy / rv


def test_detector_golden():
    # big-wave/test.py:209-225
    out = detect_host(np.arange(8, dtype=np.complex128), 8, 0.5, 3.0, 1.0, 1.0, 1.0)
    assert list(out) == [1.25, 12.5, 15.249999999999998]


@pytest.mark.parametrize("seed", range(40))
def test_detector_geometry_matches_histogram(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.choice([64, 100, 1024, 4096, 1 << 14]))
    dx = float(rng.choice([0.2, 0.5, 3.1e-10, 2e-9, 1e-9 / 3]))
    psx = dx * float(rng.choice([1.0, 2.5, 7.3, 16.0, 100.0, 513.7]))
    det = psx * float(rng.integers(1, max(2, int(n * dx / psx)))) * float(rng.choice([1.0, 1.0000001, 0.99999]))
    if int(det // psx) > n or int(det // psx) < 1:
        pytest.skip("degenerate")
    z = float(rng.choice([1.0, 0.3, 1.77]))
    u = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    sim = bw.Sim(N=n, dx=dx, z_detector=z, detector_size=det, psx=psx, psy=0.7, wl=1.0,
                 chunk_size=int(rng.choice([n, 7, 1000])))
    ref = bw.square_and_downsample(u, sim, z)
    got = detect_host(u, n, dx, det, psx, 0.7, z)
    assert got.shape == ref.shape
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=0)


def test_wavelength_bit_exact():
    lib = L.load()
    from rave_sim_b200.engine import wavelength_from_energy
    for e in np.linspace(1000.0, 150000.0, 997).tolist() + [46000.0, 46417.02200470257, 20000.0, 70000.0]:
        assert lib.rsw_energy_to_wavelength(e) == bw.wavelength_from_energy(e)
        assert wavelength_from_energy(e) == bw.wavelength_from_energy(e)
