"""Python API of the rsw engine (torch CUDA tensors in and out, no host copies).

``Plan``        length-N FFT plan with the reference's per-call operations
                (fast-wave FFT<S>, propagate, transmission kernels, detection).
``Simulation``  a whole rave-sim setup (the reference's config.yaml schema)
                run per source on the fused two-pass engine, detector output
                accumulated in FP64 on the device.

All calls are asynchronous on torch's current CUDA stream.
"""

from __future__ import annotations

import ctypes as C
import math
from typing import Iterable, Optional, Sequence

import numpy as np

from . import _lib as L

# evaluated as the reference writes them (big-wave/propagation.py:26-28):
# 1.602176634 * 10 ** (-19) differs from the literal 1.602176634e-19 by one ulp
H_PLANCK = 6.62607004 * 10 ** (-34)
C_0 = 299792458
EV_TO_JOULE = 1.602176634 * 10 ** (-19)


def wavelength_from_energy(energy_ev: float) -> float:
    """Photon wavelength in metres (big-wave/propagation.py:69-71)."""
    return H_PLANCK * C_0 / (energy_ev * EV_TO_JOULE)


def _torch():
    import torch

    return torch


def _stream_ptr(stream=None) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def dtype_code(dtype) -> int:
    """'c16'/complex128 -> RSW_C128, 'c8'/complex64 -> RSW_C64."""
    if isinstance(dtype, str):
        d = dtype.lower()
        if d in ("c16", "complex128"):
            return L.RSW_C128
        if d in ("c8", "complex64"):
            return L.RSW_C64
        raise ValueError(f"unknown dtype {dtype!r}: use c8 or c16")
    torch = _torch()
    if dtype in (torch.complex128, np.complex128):
        return L.RSW_C128
    if dtype in (torch.complex64, np.complex64):
        return L.RSW_C64
    raise ValueError(f"unsupported dtype {dtype}")


def torch_dtype(code: int):
    torch = _torch()
    return torch.complex128 if code == L.RSW_C128 else torch.complex64


def _dptr(t) -> int:
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return int(t.data_ptr())


PROPAGATORS = {"fresnel": L.RSW_PROP_FRESNEL, "exact": L.RSW_PROP_EXACT}


def propagator_code(name) -> int:
    """'fresnel' (the reference's transfer function, the default) or 'exact'
    (the angular-spectrum kernel, opt-in)."""
    if name is None:
        return L.RSW_PROP_FRESNEL
    try:
        return PROPAGATORS[str(name).lower()]
    except KeyError:
        raise ValueError(f"unknown propagator {name!r}: use 'fresnel' or 'exact'") from None


def _pair(c: complex):
    arr = (C.c_double * 2)(float(np.real(c)), float(np.imag(c)))
    return arr


class Plan:
    """FFT plan of length ``n`` for c16 or c8 fields (any n >= 1: powers of two
    >= 16 run the pass kernels, other lengths Bluestein's algorithm over them)."""

    def __init__(self, n: int, dtype="c16", tuning: Optional[dict] = None):
        """``tuning``: explicit schedule choices (rave_sim_b200.autotune.FIELDS;
        default: the registered or built-in choice)."""
        self._lib = L.load()
        self.n = int(n)
        self.code = dtype_code(dtype)
        h = C.c_void_p()
        if tuning is None:
            L.check(self._lib.rsw_plan_create(C.byref(h), self.n, self.code))
        else:
            t = L.Tuning(*(int(tuning.get(f, 0)) for f in ("levels", "log_rows", "log_mid", "row_e", "col_e",
                                                             "mid_e")))
            L.check(self._lib.rsw_plan_create_tuned(C.byref(h), self.n, self.code, C.byref(t)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.rsw_plan_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def dtype(self):
        return torch_dtype(self.code)

    def info(self) -> dict:
        n, d, r, c, s = C.c_int64(), C.c_int(), C.c_int(), C.c_int(), C.c_int64()
        L.check(self._lib.rsw_plan_info(self._h, C.byref(n), C.byref(d), C.byref(r), C.byref(c), C.byref(s)))
        return {"n": n.value, "dtype": d.value, "log_rows": r.value, "log_cols": c.value,
                "scratch_bytes": s.value}

    def _check_field(self, t):
        if t.dtype != self.dtype or t.numel() != self.n:
            raise ValueError(f"expected {self.n} values of {self.dtype}, got {t.numel()} of {t.dtype}")
        return _dptr(t)

    def fft(self, x, out=None):
        """Unnormalised forward FFT (fast-wave FFT<S>::forward)."""
        out = x if out is None else out
        L.check(self._lib.rsw_fft_forward(self._h, self._check_field(x), self._check_field(out), _stream_ptr()))
        return out

    def ifft(self, x, out=None):
        """Inverse FFT scaled by 1/N (fast-wave FFT<S>::inverse)."""
        out = x if out is None else out
        L.check(self._lib.rsw_fft_inverse(self._h, self._check_field(x), self._check_field(out), _stream_ptr()))
        return out

    def set_propagator(self, name: str):
        """Transfer function of ``propagate``: 'fresnel' (the reference's,
        default) or 'exact' (angular spectrum)."""
        L.check(self._lib.rsw_plan_set_propagator(self._h, propagator_code(name)))

    def propagate(self, u, U=None, *, dx, wl, dz, cutoff_freq, skip_fft=False):
        """big-wave ``propagate`` (propagation.py:100-138); ``u`` updated in
        place, ``U`` (if given) receives FFT(u_new)."""
        Up = self._check_field(U) if U is not None else None
        L.check(self._lib.rsw_propagate(self._h, self._check_field(u), Up, dx, wl, dz, cutoff_freq,
                                        int(bool(skip_fft)), _stream_ptr()))
        return u

    def apply_grating(self, u, *, dx, chunk_size, pitch, dc, x_position, factor_a, factor_b):
        L.check(self._lib.rsw_apply_grating_factors(
            self._h, self._check_field(u), dx, int(chunk_size), pitch, dc, x_position,
            _pair(factor_a), _pair(factor_b), _stream_ptr()))
        return u

    def apply_dba_grating(self, u, *, dx, chunk_size, pitch0, pitch1, dc0, dc1, x_position,
                          factor_a, factor_b):
        L.check(self._lib.rsw_apply_dba_grating_factors(
            self._h, self._check_field(u), dx, int(chunk_size), pitch0, pitch1, dc0, dc1, x_position,
            _pair(factor_a), _pair(factor_b), _stream_ptr()))
        return u

    def apply_sample_row(self, u, *, dx, wl, dz, pixel_size_x, x_position, row_db):
        row = np.ascontiguousarray(np.asarray(row_db, dtype=np.complex128))
        L.check(self._lib.rsw_apply_sample_row(
            self._h, self._check_field(u), dx, wl, dz, pixel_size_x, x_position, len(row),
            row.view(np.float64).ctypes.data_as(L._DP), _stream_ptr()))
        return u

    def scale(self, u, factor):
        L.check(self._lib.rsw_scale(self._h, self._check_field(u), _pair(factor), _stream_ptr()))
        return u

    def point_source(self, u, *, dx, wl, z, x_source):
        L.check(self._lib.rsw_point_source(self._h, self._check_field(u), dx, wl, z, x_source,
                                           _stream_ptr()))
        return u

    def detector_pixels(self, *, dx, detector_size, pixel_size_x, z) -> int:
        n = C.c_int64()
        L.check(self._lib.rsw_square_and_downsample(self._h, None, dx, detector_size, pixel_size_x, 1.0,
                                                    z, None, C.byref(n), _stream_ptr()))
        return n.value

    def square_and_downsample(self, u, *, dx, detector_size, pixel_size_x, pixel_size_y, z):
        """big-wave ``square_and_downsample`` (propagation.py:279-320) -> float64 tensor."""
        torch = _torch()
        npix = self.detector_pixels(dx=dx, detector_size=detector_size, pixel_size_x=pixel_size_x, z=z)
        out = torch.empty(max(npix, 0), dtype=torch.float64, device=u.device)
        if npix > 0:
            L.check(self._lib.rsw_square_and_downsample(
                self._h, self._check_field(u), dx, detector_size, pixel_size_x, pixel_size_y, z,
                C.cast(out.data_ptr(), L._DP), None, _stream_ptr()))
        return out


# ------------------------------------------------------------------ setups
def lookup_deltabeta(db_table, material) -> complex:
    """Nearest-density entry of the deltabeta table for ``[name, density]``
    (big-wave/optical_element.py:42-63): same name, density within 1e-5."""
    if material is None:
        return 0j
    name, density = material[0], float(material[1])
    cands = sorted((abs(float(m[1]) - density), complex(v[0], v[1]))
                   for m, v in db_table if m[0] == name)
    if not cands or not cands[0][0] < 1e-5:
        raise ValueError(f"material {material} not found in the deltabeta table")
    return cands[0][1]


def deltabeta_vector(material_slots, db_table) -> np.ndarray:
    """The per-run deltabeta vector (rsw_source_run.deltabeta): the materials
    of every element in descriptor order, looked up in a subconfig deltabeta
    table."""
    vals = []
    for slots in material_slots:
        vals.extend(lookup_deltabeta(db_table, m) for m in slots)
    return np.ascontiguousarray(np.asarray(vals, dtype=np.complex128).reshape(-1))


def sim_descriptor(config: dict, grids: Optional[dict], code: int, angles: Sequence[float]):
    """The C descriptors (rsw_sim_desc and its rsw_element array) of a
    setup in the reference's config.yaml schema. Returns (desc, elements,
    keep, material_slots): ``keep`` holds the arrays the descriptors point to
    (keep it alive while they are used), ``material_slots`` the materials of
    each element in the order of the per-run deltabeta vector."""
    grids = grids or {}
    sp = config["sim_params"]
    n = int(sp["N"])
    dx = float(sp["dx"])
    els = config["elements"]
    if len(angles) != len(els) + 1:
        raise ValueError("cutoff_angles must have len(elements) + 1 entries")
    keep = []
    arr = (L.Element * max(len(els), 1))()
    material_slots = []  # per element: list of materials in deltabeta order
    for i, el in enumerate(els):
        e = arr[i]
        xp = np.ascontiguousarray(np.asarray(el["x_positions"], dtype=np.float64).reshape(-1))
        keep.append(xp)
        e.n_x_positions = len(xp)
        e.x_positions = xp.ctypes.data_as(L._DP)
        e.z_start = float(el["z_start"])
        t = el["type"]
        if t in ("grating", "dba_grating"):
            e.type = L.RSW_EL_GRATING if t == "grating" else L.RSW_EL_DBA_GRATING
            e.thickness = float(el["thickness"])
            e.substrate_thickness = float(el["substrate_thickness"])
            e.nr_steps = int(el["nr_steps"])
            if t == "grating":
                e.pitch = float(el["pitch"])
                e.dc[0], e.dc[1] = (float(v) for v in el["dc"])
            else:
                e.pitch = float(el["pitch0"])
                e.pitch1 = float(el["pitch1"])
                e.dc[0], e.dc[1] = (float(v) for v in el["dc0"])
                e.dc1[0], e.dc1[1] = (float(v) for v in el["dc1"])
            material_slots.append([el.get("mat_a"), el.get("mat_b"), el.get("mat_substrate")])
        elif t == "sample":
            g = np.ascontiguousarray(np.asarray(grids[i]))
            if g.dtype != np.int8 or g.ndim != 2:
                raise ValueError("sample grids must be 2-D int8 arrays")
            keep.append(g)
            e.type = L.RSW_EL_SAMPLE
            e.pixel_size_x = float(el["pixel_size_x"])
            e.pixel_size_z = float(el["pixel_size_z"])
            e.grid_z, e.grid_x = g.shape
            e.grid = g.ctypes.data_as(C.POINTER(C.c_int8))
            e.n_materials = len(el["materials"])
            material_slots.append(list(el["materials"]))
        else:
            raise ValueError(f"unknown element type {t!r}")
    ang = np.ascontiguousarray(np.asarray(angles, dtype=np.float64))
    keep.append(ang)
    d = L.SimDesc()
    d.n = n
    d.dtype = code
    d.dx = dx
    d.z_detector = float(sp["z_detector"])
    d.detector_size = float(sp["detector_size"])
    d.pixel_size_x = float(sp["detector_pixel_size_x"])
    d.pixel_size_y = float(sp["detector_pixel_size_y"])
    d.chunk_size = int(sp.get("chunk_size", n))
    d.n_elements = len(els)
    d.elements = arr
    d.cutoff_angles = ang.ctypes.data_as(L._DP)
    return d, arr, keep, material_slots


class Simulation:
    """A rave-sim setup on the fused engine.

    ``config``: the reference's config.yaml content (``sim_params``,
    ``elements``, optional ``dtype``) plus ``cutoff_angles`` (computed.yaml);
    ``grids``: element index -> int8 sample grid for ``sample`` elements.
    """

    def __init__(self, config: dict, grids: Optional[dict] = None, dtype=None,
                 cutoff_angles: Optional[Sequence[float]] = None, propagator: Optional[str] = None):
        self._lib = L.load()
        sp = config["sim_params"]
        self.config = config
        self.code = dtype_code(dtype if dtype is not None else config.get("dtype", "c16"))
        self.n = int(sp["N"])
        self.dx = float(sp["dx"])
        angles = list(cutoff_angles if cutoff_angles is not None else config["cutoff_angles"])
        d, arr, self._keep, self.material_slots = sim_descriptor(config, grids, self.code, angles)
        self._elements = arr
        h = C.c_void_p()
        L.check(self._lib.rsw_sim_create(C.byref(h), C.byref(d)))
        self._h = h
        nps, npix, _ = C.c_int64(), C.c_int64(), C.c_int64()
        L.check(self._lib.rsw_sim_shape(self._h, C.byref(nps), C.byref(npix), C.byref(_)))
        self.nr_phase_steps = nps.value
        self.n_pix = npix.value
        prop = propagator if propagator is not None else config.get("propagator")
        if prop is not None:
            L.check(self._lib.rsw_sim_set_propagator(self._h, propagator_code(prop)))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.rsw_sim_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def split_steps(self) -> int:
        a, b, s = C.c_int64(), C.c_int64(), C.c_int64()
        L.check(self._lib.rsw_sim_shape(self._h, C.byref(a), C.byref(b), C.byref(s)))
        return s.value

    def deltabeta_vector(self, db_table) -> np.ndarray:
        return deltabeta_vector(self.material_slots, db_table)

    def reset(self):
        L.check(self._lib.rsw_sim_reset(self._h, _stream_ptr()))

    def run_source(self, *, energy: float, db_table, source: dict, weight: float = 1.0,
                   field=None, wavelength: Optional[float] = None):
        """Run one source (big-wave wavesim.run_simulation) and add
        ``weight * detected`` to the device accumulator.

        ``source``: {type: plane, z} | {type: point, x, z} | {type: vector, z}
        with ``field`` a host numpy array or CUDA tensor of N samples."""
        keep = []
        src = self._source(source, field, keep)
        run = self._run(energy, db_table, weight, wavelength, keep)
        L.check(self._lib.rsw_sim_run(self._h, C.byref(src), C.byref(run), _stream_ptr()))

    def run_sources(self, runs: Sequence[dict], *, source: Optional[dict] = None, field=None, each: bool = False,
                    sources: Optional[Sequence[dict]] = None):
        """Run several sources in lockstep (rsw_sim_run_batch): ``runs``
        holds one dict per source with ``energy``, ``db_table`` and optional
        ``weight`` (1.0) and ``wavelength``; ``source`` (with ``field`` for a
        vector source) is shared by all of them, or ``sources`` gives one
        source dict per run (with ``u``: its own vector field). The detector
        values are added in list order, as run_source calls in that order
        would add them. With ``each`` it returns every source's own detector
        values, unweighted, as a CUDA tensor (sources, nr_phase_steps, n_pix)."""
        keep = []
        if sources is not None:
            if len(sources) != len(runs):
                raise ValueError("sources needs one entry per run")
            srcs = (L.Source * max(len(sources), 1))()
            for i, sd in enumerate(sources):
                srcs[i] = self._source(sd, sd.get("u"), keep)
            n_src = len(sources)
        else:
            srcs = (L.Source * 1)(self._source(source, field, keep))
            n_src = 1
        arr = (L.SourceRun * max(len(runs), 1))()
        for i, r in enumerate(runs):
            arr[i] = self._run(r["energy"], r["db_table"], r.get("weight", 1.0), r.get("wavelength"), keep)
        out = None
        if each:
            torch = _torch()
            out = torch.empty((len(runs), self.nr_phase_steps, self.n_pix), dtype=torch.float64, device="cuda")
        L.check(self._lib.rsw_sim_run_batch(self._h, srcs, n_src, arr, len(runs),
                                            C.cast(_dptr(out), L._DP) if each else None, _stream_ptr()))
        return out

    def _run(self, energy, db_table, weight, wavelength, keep):
        db = self.deltabeta_vector(db_table)
        keep.append(db)
        run = L.SourceRun()
        run.energy_ev = float(energy)
        run.deltabeta = db.view(np.float64).ctypes.data_as(L._DP) if db.size else None
        run.n_deltabeta = db.size
        run.weight = float(weight)
        run.wavelength_m = float(wavelength) if wavelength is not None else 0.0
        return run

    def _source(self, source: dict, field, keep):
        src = L.Source()
        t = source["type"]
        src.z = float(source.get("z", 0.0))
        if t == "plane":
            src.type = L.RSW_SRC_PLANE
        elif t == "point":
            src.type = L.RSW_SRC_POINT
            src.x = float(source["x"])
        elif t == "vector":
            src.type = L.RSW_SRC_VECTOR
            if field is None:
                field = source.get("u")
            if field is None:
                raise ValueError("vector source without a field")
            if hasattr(field, "is_cuda") and field.is_cuda:
                if field.dtype != torch_dtype(self.code) or field.numel() != self.n:
                    raise ValueError("vector source field has the wrong dtype or length")
                src.d_field = _dptr(field)
            else:
                npd = np.complex128 if self.code == L.RSW_C128 else np.complex64
                f = np.ascontiguousarray(np.asarray(field, dtype=npd).reshape(-1))
                if f.size != self.n:
                    raise ValueError("vector source field has the wrong length")
                keep.append(f)
                src.h_field = f.ctypes.data
        else:
            raise ValueError(f"unknown source type {t!r}")
        return src

    def detected(self) -> np.ndarray:
        """The FP64 accumulator as (nr_phase_steps, n_pix); synchronises."""
        out = np.zeros((self.nr_phase_steps, self.n_pix), dtype=np.float64)
        L.check(self._lib.rsw_sim_read(self._h, out.ctypes.data_as(L._DP), _stream_ptr()))
        return out

    def detected_device(self, out=None):
        """The FP64 accumulator copied into a CUDA tensor (asynchronous)."""
        torch = _torch()
        if out is None:
            out = torch.empty((self.nr_phase_steps, self.n_pix), dtype=torch.float64, device="cuda")
        L.check(self._lib.rsw_sim_read_device(self._h, C.cast(_dptr(out), L._DP), _stream_ptr()))
        return out

    def accumulator(self):
        """Device pointer of the FP64 accumulator."""
        p = L._DP()
        L.check(self._lib.rsw_sim_accumulator(self._h, C.byref(p)))
        return C.cast(p, C.c_void_p).value

    def final_field(self):
        torch = _torch()
        out = torch.empty(self.n, dtype=torch_dtype(self.code), device="cuda")
        L.check(self._lib.rsw_sim_final_field(self._h, _dptr(out), _stream_ptr()))
        return out

    def set_timing(self, enable: bool):
        L.check(self._lib.rsw_sim_set_timing(self._h, int(bool(enable))))

    def set_history(self, history_dz: Optional[float]):
        """Record the history of the following runs every ``history_dz``
        metres (big-wave --history_dz); None or 0 disables."""
        L.check(self._lib.rsw_sim_set_history(self._h, float(history_dz or 0.0)))

    def history(self):
        """History of the last run: (images (n_pix, entries), z of each
        entry) as big-wave's History.get_history() / get_z()."""
        n = C.c_int64()
        L.check(self._lib.rsw_sim_history(self._h, None, None, C.byref(n), _stream_ptr()))
        h = np.zeros((self.n_pix, n.value), dtype=np.float64)
        z = np.zeros(n.value, dtype=np.float64)
        L.check(self._lib.rsw_sim_history(self._h, h.ctypes.data_as(L._DP), z.ctypes.data_as(L._DP),
                                          C.byref(n), _stream_ptr()))
        return h, z

    def set_keypoints(self, enable: bool):
        """Keep the field right before and right after each element of the
        first pass of the following runs (big-wave's save_keypoints_path,
        wavesim.py:35-55) in device buffers; ``keypoints()`` returns them."""
        if not enable:
            L.check(self._lib.rsw_sim_set_keypoints(self._h, None, 0))
            self._kp = None
            return
        torch = _torch()
        k = 2 * len(self.config["elements"])
        bufs = [torch.empty(self.n, dtype=torch_dtype(self.code), device="cuda") for _ in range(k)]
        ptrs = (C.c_void_p * max(k, 1))(*[_dptr(b) for b in bufs])
        L.check(self._lib.rsw_sim_set_keypoints(self._h, ptrs, k))
        self._kp = bufs

    def keypoints(self):
        """Keypoints of the last run, in big-wave's order (element 0 before,
        element 0 after, element 1 before, ...): CUDA tensors of N samples."""
        if getattr(self, "_kp", None) is None:
            raise ValueError("keypoints are off (set_keypoints(True) before the run)")
        return list(self._kp)

    def set_final_fields(self, enable: bool):
        """Keep the field at the detector of every phase step of the
        following runs (big-wave's save_u with save_final_u_vectors,
        wavesim.py:58-82) in device buffers; ``final_fields()`` returns them."""
        if not enable:
            L.check(self._lib.rsw_sim_set_final_fields(self._h, None, 0))
            self._ff = None
            return
        torch = _torch()
        k = self.nr_phase_steps
        bufs = [torch.empty(self.n, dtype=torch_dtype(self.code), device="cuda") for _ in range(k)]
        ptrs = (C.c_void_p * k)(*[_dptr(b) for b in bufs])
        L.check(self._lib.rsw_sim_set_final_fields(self._h, ptrs, k))
        self._ff = bufs

    def final_fields(self):
        """Final field of each phase step of the last run (u_0000, u_0001, ...
        of big-wave): CUDA tensors of N samples."""
        if getattr(self, "_ff", None) is None:
            raise ValueError("final fields are off (set_final_fields(True) before the run)")
        return list(self._ff)

    def timing(self, kind: int):
        ms, n = C.c_double(), C.c_int64()
        L.check(self._lib.rsw_sim_timing(self._h, int(kind), C.byref(ms), C.byref(n)))
        return ms.value, n.value


def run_case(case: dict, grids: Optional[dict] = None, dtype=None, history_dz: Optional[float] = None,
             keypoints: Optional[list] = None):
    """Run one source described by a case dict (the oracle's schema: the
    reference config + ``source``, ``energy``, ``db``, ``cutoff_angles``) and
    return its detector array (nr_phase_steps, n_pix); with ``history_dz``,
    (detector, history (n_pix, entries), z of each entry). A ``keypoints``
    list receives the keypoint fields as numpy arrays."""
    sim = Simulation(case, grids=grids, dtype=dtype if dtype is not None else case.get("dtype", "c16"),
                     cutoff_angles=case["cutoff_angles"])
    try:
        sim.set_history(history_dz)
        if keypoints is not None:
            sim.set_keypoints(True)
        sim.reset()
        sim.run_source(energy=case["energy"], db_table=case["db"], source=case["source"],
                       field=case["source"].get("u"))
        det = sim.detected()
        if keypoints is not None:
            keypoints.extend(t.cpu().numpy() for t in sim.keypoints())
        if history_dz:
            h, z = sim.history()
            return det, h, z
        return det
    finally:
        sim.close()
