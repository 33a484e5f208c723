"""The schedule autotuner (rsw_autotune, rave_sim_b200.autotune): every
candidate it times is a correct FFT (checked against numpy, which runs every
kernel variant the tuner can pick), the best is the fastest timed, and a
registered tuning is what later plans use."""

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import rave_sim_b200 as rsw  # noqa: E402
from rave_sim_b200 import _lib as L  # noqa: E402
from rave_sim_b200 import autotune  # noqa: E402

TOL = {"c16": 1e-12, "c8": 2e-6}


@pytest.mark.parametrize("dt,logn", [("c16", 20), ("c8", 20), ("c8", 14)])
def test_candidates_are_correct_and_best_is_fastest(dt, logn, monkeypatch):
    for v in ("RSW_SPLIT", "RSW_SPLIT3", "RSW_ROW_E", "RSW_COL_E"):
        monkeypatch.delenv(v, raising=False)
    n = 1 << logn
    res = autotune.tune(n, dt, reps=2, save=False)
    try:
        tried = res["tried"]
        assert len(tried) >= 3
        assert res["ms_per_split_step"] == pytest.approx(min(ms for _, ms in tried))
        rng = np.random.default_rng(logn)
        x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(
            np.complex128 if dt == "c16" else np.complex64)
        ref = np.fft.fft(x.astype(np.complex128))
        for t, _ in tried:
            p = rsw.Plan(n, dt, tuning=t)
            assert autotune.plan_tuning(p) == t
            X = p.fft(torch.from_numpy(x).cuda(), torch.empty(n, dtype=p.dtype, device="cuda"))
            assert rel_l2(X.cpu().numpy(), ref) < TOL[dt], t
            p.close()
        # registered: later plans of this length use the best tuning
        assert autotune.plan_tuning(rsw.Plan(n, dt)) == res["best"]
    finally:
        autotune.register(n, dt, None)
    assert autotune.plan_tuning(rsw.Plan(n, dt)) != {} and True


def test_unavailable_tuning_rejected():
    with pytest.raises(L.RswError):
        rsw.Plan(1 << 20, "c16", tuning={"levels": 2, "log_rows": 3})
    with pytest.raises(L.RswError):
        rsw.Plan(1 << 20, "c16", tuning={"levels": 2, "log_rows": 10, "row_e": 8})  # rows of 2^10: no E=8
    with pytest.raises(L.RswError):
        rsw.Plan(1 << 26, "c16", tuning={"levels": 1})


@pytest.mark.parametrize("dt", ["c16", "c8"])
def test_batched_autotune(dt, monkeypatch):
    # rsw_autotune_batch times every candidate over several fields in one
    # launch per pass: the same candidates, each time the split step of all
    # fields (longer than one field's), and the best of them registered
    for v in ("RSW_SPLIT", "RSW_SPLIT3", "RSW_ROW_E", "RSW_COL_E"):
        monkeypatch.delenv(v, raising=False)
    n = 1 << 18
    try:
        one = autotune.tune(n, dt, reps=2, save=False, register_result=False)
        four = autotune.tune(n, dt, reps=2, save=False, fields=4)
        assert sorted(map(str, (t for t, _ in four["tried"]))) == sorted(map(str, (t for t, _ in one["tried"])))
        assert four["ms_per_split_step"] == pytest.approx(min(ms for _, ms in four["tried"]))
        assert four["ms_per_split_step"] > one["ms_per_split_step"]
        assert autotune.plan_tuning(rsw.Plan(n, dt)) == four["best"]
    finally:
        autotune.register(n, dt, None)
    with pytest.raises(L.RswError):
        autotune.tune(n, dt, reps=1, save=False, register_result=False, fields=0)
