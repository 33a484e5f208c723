"""Pin the CPU oracle against the reference's golden vectors (CPU only).

The fixtures were produced by running the unmodified big-wave FP64 path
(tests/golden/make_golden.py); TestSnapshot's 25 values are the reference's
own stored golden (big-wave/test.py:861-890, atol 1e-14 at :960)."""

import numpy as np
import pytest

from conftest import GOLDEN, case_names, load_case, load_snapshot_case, rel_l2
from oracle import bigwave_np as bw


def test_snapshot_golden():
    case, d = load_snapshot_case()
    det = bw.run_simulation(case)
    # the reference test's own criterion
    assert np.allclose(det[0], d["known_data"], rtol=0, atol=1e-14)
    # full-precision output of the reference run
    assert rel_l2(det, d["detected"]) < 1e-13


@pytest.mark.parametrize("name", case_names())
def test_case_golden(name):
    case, grids, d = load_case(name)
    det, fields = bw.run_simulation(case, grids, return_fields=True)
    assert det.shape == d["detected"].shape
    assert rel_l2(det, d["detected"]) < 1e-13
    if "u_final" in d:
        assert rel_l2(fields[0], d["u_final"]) < 1e-13


def test_square_and_downsample_golden():
    # big-wave/test.py:209-225
    u = np.arange(8, dtype=np.complex128)
    sim = bw.Sim(N=8, dx=0.5, z_detector=1.0, detector_size=3.0, psx=1.0, psy=1.0,
                 wl=1.0, chunk_size=3)
    out = bw.square_and_downsample(u, sim, 1.0)
    assert list(out) == [1.25, 12.5, 15.249999999999998]
    units = np.load(GOLDEN / "units.npz")
    assert np.array_equal(out, units["sqd_out"])


def test_grating_masks_golden():
    units = np.load(GOLDEN / "units.npz")
    off = 0
    for prm, n in zip(units["mask_params"], units["mask_lengths"]):
        pitch, dx, dc0, dc1, xpos, start, count, zf = prm
        dc = (1 - zf) * dc0 + zf * dc1
        m = bw.grating_mask_chunk(dx, int(start), int(count), pitch, dc, xpos)
        assert np.array_equal(m.astype(np.uint8), units["mask_concat"][off:off + n])
        off += n


def test_frequency_cutoff_golden():
    units = np.load(GOLDEN / "units.npz")
    for (dx, n, freq), cnt, first in zip(units["cut_params"], units["cut_zero_counts"],
                                         units["cut_zero_first"]):
        rng = bw.cutoff_zero_range(int(n), freq, dx)
        if rng is None:
            assert cnt == 0
        else:
            s, e = rng
            assert max(0, min(e, n) - s) == cnt
            if cnt:
                assert s == first


def test_fft2_golden():
    # fast-wave/test/fwtest.cu:111-127
    units = np.load(GOLDEN / "units.npz")
    expected = np.array([9 + 3j, -5.12132034 - 2.70710678j, 2j, 0.53553391 - 1.29289322j,
                         1 + 1j, -0.87867966 - 1.29289322j, 2 + 2j, -6.53553391 - 2.70710678j])
    assert np.allclose(units["fft2_out"], expected, atol=1e-7)


def test_energy_conversion():
    # big-wave/test.py:201-207
    assert abs(bw.wavelength_from_energy(46000) - 26.95e-12) < 0.01e-12


@pytest.mark.parametrize("name", ["hist_point_tl", "hist_sample", "stepping_n6"])
def test_oracle_history_matches_reference(name):
    """History recording (big-wave/history.py) against the reference's own
    History of the same run."""
    case, grids, d = load_case(name)
    det, h, z = bw.run_simulation(case, grids, history_dz=case["history_dz"])
    assert np.array_equal(z, d["history_z"])
    assert h.shape == d["history"].shape
    assert rel_l2(h, d["history"]) < 1e-13
    assert rel_l2(det, d["detected"]) < 1e-13


def test_angular_kernel_reduces_to_fresnel_at_small_frequencies():
    # sqrt(1/wl^2 - f^2) = 1/wl - wl f^2 / 2 - wl^3 f^4 / 8 - ...: the exact
    # kernel's phase exceeds the Fresnel one by 2 pi dz wl^3 f^4 / 8 to leading order
    n, dx, wl, dz = 1 << 12, 2e-9, 2.6953e-11, 0.0818
    ha = bw.transfer_function_angular(n, dx, wl, dz)
    hf = bw.transfer_function(n, dx, wl, dz)
    fx = np.fft.fftfreq(n, dx)
    d = np.angle(ha * np.conj(hf))
    small = np.abs(fx) < 0.05 / dx
    pred = 2 * np.pi * dz * wl ** 3 * fx ** 4 / 8
    np.testing.assert_allclose(d[small], pred[small], rtol=1e-3, atol=1e-9)
    assert np.all(np.abs(np.abs(ha) - 1) < 1e-14)


@pytest.mark.parametrize("name", ["sample_stepped", "hist_sample", "stepping_n6", "odd_point_sample"])
def test_oracle_keypoints_match_reference(name):
    """Keypoints (big-wave/wavesim.py:35-55): the field before and after each
    element of the first pass, against the reference's own keypoint files
    (every s-th sample and full-vector sums)."""
    case, grids, d = load_case(name)
    kps = []
    bw.run_simulation(case, grids, keypoints=kps)
    kps = np.stack(kps)
    s = int(d["keypoints_stride"])
    assert kps.shape[0] == d["keypoints_sub"].shape[0] == 2 * len(case["elements"])
    assert rel_l2(kps[:, ::s], d["keypoints_sub"]) < 1e-13
    assert rel_l2(kps.sum(axis=1), d["keypoints_sum"]) < 1e-12
    assert rel_l2((np.abs(kps) ** 2).sum(axis=1), d["keypoints_norm2"]) < 1e-13
