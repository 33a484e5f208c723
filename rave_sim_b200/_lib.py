"""ctypes binding of the rsw C ABI (include/rsw.h).

The shared library ``librsw.so`` is built in-tree by ``rave_sim_b200.build``.
Loading fails loudly when it is missing: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "librsw.so"

RSW_OK, RSW_ERR_INVALID, RSW_ERR_UNSUPPORTED, RSW_ERR_CUDA, RSW_ERR_NOMEM, RSW_ERR_TIMEOUT = range(6)
RSW_C128, RSW_C64 = 0, 1
RSW_EL_GRATING, RSW_EL_DBA_GRATING, RSW_EL_SAMPLE = 0, 1, 2
RSW_SRC_PLANE, RSW_SRC_POINT, RSW_SRC_VECTOR = 0, 1, 2
RSW_PROP_FRESNEL, RSW_PROP_EXACT = 0, 1

STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "UNSUPPORTED", 3: "CUDA", 4: "NOMEM", 5: "TIMEOUT"}


class RswError(RuntimeError):
    """An rsw call returned a non-OK status."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"rsw {STATUS_NAMES.get(status, status)}: {message}")


class Element(C.Structure):
    _fields_ = [
        ("type", C.c_int),
        ("z_start", C.c_double),
        ("thickness", C.c_double),
        ("substrate_thickness", C.c_double),
        ("nr_steps", C.c_int),
        ("pitch", C.c_double),
        ("pitch1", C.c_double),
        ("dc", C.c_double * 2),
        ("dc1", C.c_double * 2),
        ("n_x_positions", C.c_int),
        ("x_positions", C.POINTER(C.c_double)),
        ("pixel_size_x", C.c_double),
        ("pixel_size_z", C.c_double),
        ("grid_z", C.c_int64),
        ("grid_x", C.c_int64),
        ("grid", C.POINTER(C.c_int8)),
        ("n_materials", C.c_int),
    ]


class SimDesc(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("dtype", C.c_int),
        ("dx", C.c_double),
        ("z_detector", C.c_double),
        ("detector_size", C.c_double),
        ("pixel_size_x", C.c_double),
        ("pixel_size_y", C.c_double),
        ("chunk_size", C.c_int64),
        ("n_elements", C.c_int),
        ("elements", C.POINTER(Element)),
        ("cutoff_angles", C.POINTER(C.c_double)),
    ]


class Source(C.Structure):
    _fields_ = [
        ("type", C.c_int),
        ("x", C.c_double),
        ("z", C.c_double),
        ("h_field", C.c_void_p),
        ("d_field", C.c_void_p),
    ]


class SourceRun(C.Structure):
    _fields_ = [
        ("energy_ev", C.c_double),
        ("deltabeta", C.POINTER(C.c_double)),
        ("n_deltabeta", C.c_int64),
        ("weight", C.c_double),
        ("wavelength_m", C.c_double),
    ]


class Tuning(C.Structure):
    _fields_ = [
        ("levels", C.c_int),
        ("log_rows", C.c_int),
        ("log_mid", C.c_int),
        ("row_e", C.c_int),
        ("col_e", C.c_int),
        ("mid_e", C.c_int),
    ]


_P = C.c_void_p
_D = C.c_double
_I64 = C.c_int64
_DP = C.POINTER(C.c_double)

# name -> (restype, argtypes); every symbol of include/rsw.h
SIGNATURES = {
    "rsw_last_error": (C.c_char_p, []),
    "rsw_abi_version": (C.c_int, []),
    "rsw_launch_count": (C.c_uint64, []),
    "rsw_struct_size": (C.c_size_t, [C.c_int]),
    "rsw_energy_to_wavelength": (C.c_double, [C.c_double]),
    "rsw_plan_create": (C.c_int, [C.POINTER(_P), _I64, C.c_int]),
    "rsw_plan_create_tuned": (C.c_int, [C.POINTER(_P), _I64, C.c_int, C.POINTER(Tuning)]),
    "rsw_plan_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "rsw_set_tuning": (C.c_int, [_I64, C.c_int, C.POINTER(Tuning)]),
    "rsw_autotune": (C.c_int, [_I64, C.c_int, C.c_int, C.POINTER(Tuning), _DP, C.POINTER(Tuning), _DP,
                               C.c_int, C.POINTER(C.c_int), _P]),
    "rsw_autotune_batch": (C.c_int, [_I64, C.c_int, _I64, C.c_int, C.POINTER(Tuning), _DP, C.POINTER(Tuning), _DP,
                               C.c_int, C.POINTER(C.c_int), _P]),
    "rsw_plan_destroy": (C.c_int, [_P]),
    "rsw_plan_info": (C.c_int, [_P, C.POINTER(_I64), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                C.POINTER(C.c_int), C.POINTER(_I64)]),
    "rsw_fft_forward": (C.c_int, [_P, _P, _P, _P]),
    "rsw_fft_inverse": (C.c_int, [_P, _P, _P, _P]),
    "rsw_fft_forward_noalloc": (C.c_int, [_P, _P, _I64, C.c_int, _P]),
    "rsw_fft_host": (C.c_int, [_P, _P, _P, _I64, C.c_int, C.c_int, _I64, _P]),
    "rsw_propagate": (C.c_int, [_P, _P, _P, _D, _D, _D, _D, C.c_int, _P]),
    "rsw_apply_grating_factors": (C.c_int, [_P, _P, _D, _I64, _D, _D, _D, _DP, _DP, _P]),
    "rsw_apply_dba_grating_factors": (C.c_int, [_P, _P, _D, _I64, _D, _D, _D, _D, _D, _DP, _DP, _P]),
    "rsw_apply_sample_row": (C.c_int, [_P, _P, _D, _D, _D, _D, _D, _I64, _DP, _P]),
    "rsw_scale": (C.c_int, [_P, _P, _DP, _P]),
    "rsw_point_source": (C.c_int, [_P, _P, _D, _D, _D, _D, _P]),
    "rsw_square_and_downsample": (C.c_int, [_P, _P, _D, _D, _D, _D, _D, _DP, C.POINTER(_I64), _P]),
    "rsw_detector_geometry": (C.c_int, [_I64, _D, _D, _D, _D, C.POINTER(_I64), C.POINTER(_I64), _DP, _DP]),
    "rsw_signal_retrieval": (C.c_int, [_P, _I64, C.c_int, _D, _P, _P, _P, _P, _P]),
    "rsw_sim_set_history": (C.c_int, [_P, _D]),
    "rsw_sim_set_propagator": (C.c_int, [_P, C.c_int]),
    "rsw_plan_set_propagator": (C.c_int, [_P, C.c_int]),
    "rsw_sim_history": (C.c_int, [_P, _DP, _DP, C.POINTER(_I64), _P]),
    "rsw_sim_set_keypoints": (C.c_int, [_P, C.POINTER(C.c_void_p), _I64]),
    "rsw_sim_set_final_fields": (C.c_int, [_P, C.POINTER(C.c_void_p), _I64]),
    "rsw_sim_create": (C.c_int, [C.POINTER(_P), C.POINTER(SimDesc)]),
    "rsw_sim_destroy": (C.c_int, [_P]),
    "rsw_sim_shape": (C.c_int, [_P, C.POINTER(_I64), C.POINTER(_I64), C.POINTER(_I64)]),
    "rsw_sim_run": (C.c_int, [_P, C.POINTER(Source), C.POINTER(SourceRun), _P]),
    "rsw_sim_run_batch": (C.c_int, [_P, C.POINTER(Source), _I64, C.POINTER(SourceRun), _I64, _DP, _P]),
    "rsw_sim_reset": (C.c_int, [_P, _P]),
    "rsw_sim_read": (C.c_int, [_P, _DP, _P]),
    "rsw_sim_read_device": (C.c_int, [_P, _DP, _P]),
    "rsw_sim_accumulator": (C.c_int, [_P, C.POINTER(_DP)]),
    "rsw_sim_final_field": (C.c_int, [_P, _P, _P]),
    "rsw_sim_set_timing": (C.c_int, [_P, C.c_int]),
    "rsw_sim_timing": (C.c_int, [_P, C.c_int, _DP, C.POINTER(_I64)]),
}

_lib = None


def load(path: os.PathLike | None = None) -> C.CDLL:
    """Load librsw.so (once) and declare every entry point's signature."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"{p} not found: build the CUDA library with `python -m rave_sim_b200.build`"
        )
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    for i, st in enumerate((Element, SimDesc, Source, SourceRun, Tuning)):
        if lib.rsw_struct_size(i) != C.sizeof(st):
            raise ImportError(f"ABI mismatch for {st.__name__}: C {lib.rsw_struct_size(i)} "
                              f"vs ctypes {C.sizeof(st)}")
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != RSW_OK:
        msg = load().rsw_last_error().decode(errors="replace")
        raise RswError(status, msg)
