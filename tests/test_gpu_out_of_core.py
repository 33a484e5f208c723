"""Out-of-core FFT through the GPU (rsw_fft_host: big-fourier's four-step,
big-fourier/src/bfft.rs:27-100, with the transform passes on the device)
against numpy, and the bfpy-compatible file functions
(big-fourier/src/lib.rs:65-126) on .npy files."""

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import rave_sim_b200 as rsw  # noqa: E402
from rave_sim_b200 import bigfourier as bf  # noqa: E402

TOL = {"c16": 1e-12, "c8": 2e-6}
NP = {"c16": np.complex128, "c8": np.complex64}


def cplx(n, seed, dt):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(NP[dt])


def min_device_bytes(n, dt):
    """six slabs of one row transform: the smallest working set, many slabs"""
    logn = n.bit_length() - 1
    return 6 * (1 << (logn - logn // 2)) * np.dtype(NP[dt]).itemsize


@pytest.mark.parametrize("dt", ["c16", "c8"])
@pytest.mark.parametrize("logn", [8, 9, 13, 16, 20])
@pytest.mark.parametrize("tight", [True, False])
def test_matches_numpy(dt, logn, tight):
    n = 1 << logn
    x = cplx(n, logn, dt)
    db = min_device_bytes(n, dt) if tight else 1 << 30
    x128 = x.astype(np.complex128)
    X = bf.fft_host(x, device_bytes=db)
    assert X.dtype == x.dtype
    assert rel_l2(X, np.fft.fft(x128)) < TOL[dt]
    assert rel_l2(bf.fft_host(x, inverse=True, device_bytes=db), np.fft.ifft(x128)) < TOL[dt]
    assert rel_l2(bf.fft_host(X, inverse=True, device_bytes=db), x) < TOL[dt]


@pytest.mark.parametrize("dt", ["c16", "c8"])
@pytest.mark.parametrize("logn", [22, 23])
def test_batched_two_level_plans(dt, logn, monkeypatch):
    # transforms of 2^11 / 2^12 forced to two levels (columns of 2^4): the
    # batched column, row and reorder passes of every slab
    monkeypatch.setenv("RSW_SPLIT", "4")
    n = 1 << logn
    x = cplx(n, 3, dt)
    X = bf.fft_host(x, device_bytes=min_device_bytes(n, dt) * 4)
    assert rel_l2(X, np.fft.fft(x.astype(np.complex128))) < TOL[dt]
    assert rel_l2(bf.fft_host(X, inverse=True, device_bytes=1 << 28), x) < TOL[dt]


def test_aliasing_rules():
    n = 1 << 14
    x = cplx(n, 7, "c16")
    ref = np.fft.fft(x)
    y = x.copy()
    scratch = np.empty_like(x)
    bf.fft_host(y, out=y, scratch=scratch, device_bytes=min_device_bytes(n, "c16"))
    assert rel_l2(y, ref) < 1e-12
    out = np.empty_like(x)
    bf.fft_host(x, out=out, scratch=out)
    assert rel_l2(out, ref) < 1e-12
    with pytest.raises(rsw.RswError):
        bf.fft_host(x, out=x)  # no scratch: intermediate results would overwrite the input


def test_rejects_bad_sizes():
    with pytest.raises(rsw.RswError):
        bf.fft_host(cplx(128, 0, "c16"))
    with pytest.raises(rsw.RswError):
        bf.fft_host(cplx(1 << 12, 0, "c16"), device_bytes=1000)
    with pytest.raises(ValueError):
        bf.fft_host(cplx(1 << 12, 0, "c16").reshape(64, 64))


@pytest.mark.parametrize("dt", ["c16", "c8"])
def test_npy_files(tmp_path, dt):
    # big-wave/vector.py:134-146: fft(self.file -> destination.file, scratch)
    n = 1 << 18
    x = cplx(n, 11, dt)
    src, dst, scr = tmp_path / "u.npy", tmp_path / "U.npy", tmp_path / "scratch.npy"
    np.save(src, x)
    getattr(bf, f"fft_{dt}")(src, dst, scr, device_bytes=1 << 22)
    X = np.load(dst)
    assert X.dtype == NP[dt] and rel_l2(X, np.fft.fft(x.astype(np.complex128))) < TOL[dt]
    assert np.array_equal(np.load(src), x)
    getattr(bf, f"ifft_{dt}")(dst, dst, scr, device_bytes=1 << 22)  # in place, through the scratch file
    assert rel_l2(np.load(dst), x) < TOL[dt]
    with pytest.raises(ValueError):
        getattr(bf, f"fft_{'c8' if dt == 'c16' else 'c16'}")(src, dst, scr)
