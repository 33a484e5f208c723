"""Autotuning of the FFT schedule: the level split and the samples per thread
of each kernel, chosen by timing on the device (the choice cuFFT makes inside
cufftPlan1d, fast-wave/src/fft.cpp:8, made here by measurement).

``tune(n, dtype)`` times every available tuning of a length on one
steady-state split step (``rsw_autotune``, or ``rsw_autotune_batch`` over
several fields at once), registers the fastest for the
plans and simulations created afterwards in this process
(``rsw_set_tuning``) and records it in a JSON cache, keyed by device name,
length and dtype. ``load_cache()`` registers the cached tunings of the
current device. The cache file is ``$RSW_TUNING_CACHE`` or
``~/.cache/rave_sim_b200/tuning.json``.
"""

from __future__ import annotations

import ctypes as C
import json
import os
from pathlib import Path
from typing import Optional

from . import _lib as L
from .engine import _stream_ptr, dtype_code

FIELDS = ("levels", "log_rows", "log_mid", "row_e", "col_e", "mid_e")


def cache_path() -> Path:
    p = os.environ.get("RSW_TUNING_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "rave_sim_b200" / "tuning.json"


def _device_name() -> str:
    import torch

    return torch.cuda.get_device_name(torch.cuda.current_device())


def _to_dict(t: L.Tuning) -> dict:
    return {f: int(getattr(t, f)) for f in FIELDS}


def _from_dict(d: dict) -> L.Tuning:
    return L.Tuning(*(int(d.get(f, 0)) for f in FIELDS))


def register(n: int, dtype, tuning: Optional[dict]) -> None:
    """Use ``tuning`` (a dict of FIELDS; None removes it) for the plans of
    length n and this dtype created from now on in this process."""
    lib = L.load()
    t = _from_dict(tuning) if tuning is not None else None
    L.check(lib.rsw_set_tuning(int(n), dtype_code(dtype), C.byref(t) if t is not None else None))


def plan_tuning(plan) -> dict:
    """The effective choices of an engine Plan."""
    t = L.Tuning()
    L.check(L.load().rsw_plan_tuning(plan._h, C.byref(t)))
    return _to_dict(t)


def tune(n: int, dtype="c8", reps: int = 5, register_result: bool = True, save: bool = True,
         fields: int = 1) -> dict:
    """Time every available tuning of (n, dtype); returns {"best": tuning,
    "ms_per_split_step": t, "tried": [(tuning, ms), ...]} and registers /
    caches the best one. ``fields`` > 1 times each split step over that many
    fields of n samples in one launch per pass, as a lockstep batch of
    sources runs (``rsw_autotune_batch``); the times are then per split step
    of all fields."""
    lib = L.load()
    code = dtype_code(dtype)
    best, best_ms, count = L.Tuning(), C.c_double(), C.c_int()
    cap = 256
    tried = (L.Tuning * cap)()
    tried_ms = (C.c_double * cap)()
    L.check(lib.rsw_autotune_batch(int(n), code, int(fields), int(reps), C.byref(best), C.byref(best_ms), tried,
                                   tried_ms, cap, C.byref(count), _stream_ptr()))
    out = {"best": _to_dict(best), "ms_per_split_step": best_ms.value,
           "tried": [(_to_dict(tried[i]), tried_ms[i]) for i in range(min(count.value, cap))]}
    if register_result:
        register(n, dtype, out["best"])
    if save and fields == 1:  # the cache holds single-field tunings
        _save_entry(n, code, out["best"], best_ms.value)
    return out


def _save_entry(n: int, code: int, best: dict, ms: float) -> None:
    path = cache_path()
    try:
        data = json.loads(path.read_text()) if path.exists() else {}
    except (OSError, ValueError):
        data = {}
    key = f"{_device_name()}|{int(n)}|{'c16' if code == L.RSW_C128 else 'c8'}"
    data[key] = {"tuning": best, "ms_per_split_step": ms}
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_suffix(".tmp")
    tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
    tmp.replace(path)


def load_cache() -> int:
    """Register every cached tuning of the current device; returns how many."""
    path = cache_path()
    if not path.exists():
        return 0
    try:
        data = json.loads(path.read_text())
    except (OSError, ValueError):
        return 0
    dev = _device_name()
    k = 0
    for key, entry in data.items():
        name, n, dt = key.rsplit("|", 2)
        if name == dev:
            register(int(n), dt, entry["tuning"])
            k += 1
    return k
