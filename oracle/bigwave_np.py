"""CPU oracle: a numpy/scipy restatement of rave-sim big-wave's FP64 split-step
propagation path.

TEST INFRASTRUCTURE ONLY. Nothing in the product imports this module; it is
used by ``tests/``, by ``__graft_entry__.smoke()`` as the checker, and by
``bench.py`` as the timed CPU baseline. It is pinned against golden outputs of
the unmodified reference (``tests/golden/*.npz``, produced by
``tests/golden/make_golden.py``), including the reference's own TestSnapshot
vector (``big-wave/test.py:853-960``).

Every function cites the reference lines it restates. The discrete decisions
(grating mask coordinates, frequency-cutoff index range, histogram bin
membership, interpolation brackets) follow the reference's numpy expressions
operation by operation, because one misplaced sample changes a detector pixel
by ~dx/pixel.

The description of one simulation (a "case") is a dict in the schema of the
reference's ``config.yaml`` + ``subconfig.yaml`` + ``computed.yaml``:

    sim_params: {N, dx, z_detector, detector_size, detector_pixel_size_x,
                 detector_pixel_size_y, chunk_size}
    elements:   [ {type: grating|dba_grating|sample, ...reference keys...} ]
    source:     {type: point, x, z} | {type: plane, z} | {type: vector, z, u}
    energy:     eV
    db:         [[[name, density], [delta, beta]], ...]   (deltabeta_table)
    cutoff_angles: [len(elements)+1 angles]
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.fft as spfft

# big-wave/propagation.py:26-28
H_PLANCK = 6.62607004 * 10 ** (-34)
C_0 = 299792458
EV_TO_JOULE = 1.602176634 * 10 ** (-19)


def wavelength_from_energy(energy_ev: float) -> float:
    """``convert_energy_wavelength`` (big-wave/propagation.py:69-71)."""
    return H_PLANCK * C_0 / (energy_ev * EV_TO_JOULE)


@dataclass
class Sim:
    N: int
    dx: float
    z_detector: float
    detector_size: float
    psx: float
    psy: float
    wl: float
    chunk_size: int
    propagator: str = "fresnel"  # or "exact": the opt-in angular-spectrum kernel


# --------------------------------------------------------------------------
# free-space step
# --------------------------------------------------------------------------
def signed_fft_index(n: int) -> np.ndarray:
    """Integer numerators of ``np.fft.fftfreq(n)`` in storage order
    (``fftfreq_chunk``, big-wave/propagation.py:154-175)."""
    k = np.arange(n)
    return np.where(k < (n - 1) // 2 + 1, k, k - n)


def cutoff_zero_range(n: int, freq: float, dx: float):
    """Index range [start, end) zeroed by ``apply_frequency_cutoff``
    (big-wave/propagation.py:74-97), or None when nothing is removed."""
    start = math.ceil(n * (freq * dx))
    if start > n / 2:
        return None
    return start, n - start + 1


def transfer_function(n: int, dx: float, wl: float, dz: float) -> np.ndarray:
    """Fresnel transfer function of ``propagate`` (big-wave/propagation.py:124-128):
    ``exp(-i 2 pi dz / wl) * exp(i pi wl dz fx^2)`` with ``fx = (k * (1/n)) / dx``."""
    fx = (signed_fft_index(n) * (1.0 / n)) / dx
    return np.exp(-1j * 2 * np.pi / wl * dz) * np.exp(1j * np.pi * wl * dz * (fx**2))


def transfer_function_exact(n: int, dx: float, wl: float, dz: float) -> np.ndarray:
    """The transfer function with the phase c * fx^2 evaluated without
    intermediate rounding (long double, reduced mod 2 pi) for the reference's
    c = fl(fl(pi wl) dz). Differs from ``transfer_function`` by the reference's
    own rounding of fx and fx^2 (a few ulp of phases up to ~1e7 rad)."""
    ks = signed_fft_index(n).astype(np.longdouble)
    c = np.longdouble(float((np.pi * wl) * dz))
    th = c * (ks / (np.longdouble(n) * np.longdouble(dx))) ** 2
    two_pi = np.longdouble("6.283185307179586476925286766559005768")
    th = (th - np.round(th / two_pi) * two_pi).astype(np.float64)
    return np.exp(-1j * 2 * np.pi / wl * dz) * np.exp(1j * th)


def transfer_function_angular(n: int, dx: float, wl: float, dz: float) -> np.ndarray:
    """The exact angular-spectrum kernel of the engine's opt-in propagator
    (no counterpart in the reference, whose kernel is the Fresnel one):
    exp(-i 2 pi dz sqrt(1/wl^2 - fx^2)) as the same constant
    exp(-i 2 pi dz / wl) times exp(i phi), phi = 2 pi dz fx^2 /
    (1/wl + sqrt(1/wl^2 - fx^2)) (no cancellation), fx as in
    ``transfer_function``; evanescent components (fx^2 >= 1/wl^2) are zero.
    The FP64 operations are those of the engine, in the same order."""
    fx = (signed_fft_index(n) * (1.0 / n)) / dx
    f2 = fx * fx
    inv_wl = 1.0 / wl
    d = inv_wl * inv_wl - f2
    prop = d > 0
    phi = np.where(prop, ((2.0 * np.pi) * dz) * f2 / (inv_wl + np.sqrt(np.where(prop, d, 1.0))), 0.0)
    return np.where(prop, np.exp(-1j * 2 * np.pi / wl * dz) * np.exp(1j * phi), 0.0)


def propagate(u, U, sim: Sim, dz: float, cutoff_freq: float, skip_fft=False, exact_phase=False):
    """``propagate`` (big-wave/propagation.py:100-138). Returns (u_new, U_new)
    with ``U_new`` the spectrum of ``u_new`` as in the reference. With
    ``sim.propagator == "exact"`` the transfer function is the engine's
    opt-in angular-spectrum kernel instead of the reference's."""
    if not skip_fft:
        U = spfft.fft(u)
    # ``chunk *= H``: computed in complex128, stored in the field's dtype
    if sim.propagator == "exact":
        tf = transfer_function_angular
    else:
        tf = transfer_function_exact if exact_phase else transfer_function
    U = (U * tf(len(u), sim.dx, sim.wl, dz)).astype(U.dtype, copy=False)
    rng = cutoff_zero_range(len(u), cutoff_freq, sim.dx)
    if rng is not None:
        U[rng[0]:rng[1]] = 0
    return spfft.ifft(U), U


# --------------------------------------------------------------------------
# transmission functions
# --------------------------------------------------------------------------
def material_factor(deltabeta, thickness: float, wl: float):
    """``material_factor`` (big-wave/optical_element.py:36-39)."""
    return np.exp(2j * np.pi * thickness / wl * deltabeta)


def _chunk_linspace(dx: float, start: int, count: int, x_pos: float) -> np.ndarray:
    """x coordinates of one chunk as built in ``generate_grating_chunk``
    (big-wave/optical_element.py:352-354)."""
    x_start = start * dx + x_pos
    x_stop = x_start + count * dx
    return np.linspace(x_start, x_stop, count, endpoint=False)


def grating_mask_chunk(dx, start, count, pitch, dc, x_pos) -> np.ndarray:
    """``generate_grating_chunk`` (big-wave/optical_element.py:341-357) for an
    already interpolated duty cycle ``dc``."""
    x = _chunk_linspace(dx, start, count, x_pos)
    return np.mod(x / pitch + dc / 2, 1) < dc


def dba_mask_chunk(dx, start, count, pitch0, pitch1, dc0, dc1, x_pos) -> np.ndarray:
    """``generate_dba_grating_chunk`` (big-wave/optical_element.py:359-377)."""
    x = _chunk_linspace(dx, start, count, x_pos)
    return (np.mod(x / pitch0 + dc0 / 2, 1) < dc0) * (np.mod(x / pitch1, 1) < dc1)


def interpolated_dc(dc_pair, i: int, nr_steps: int) -> float:
    """Duty cycle of sub-step ``i`` (big-wave/optical_element.py:350 and the
    ``z_fraction = i / nr_steps`` of ``Grating.apply`` :157)."""
    zf = i / nr_steps
    return (1 - zf) * dc_pair[0] + zf * dc_pair[1]


def _chunks(N, chunk_size):
    for idx in range(0, N, chunk_size):
        yield idx, min(chunk_size, N - idx)


def _apply_binary(u, sim, mask_fn, fa, fb):
    """Multiply ``u`` by ``mask ? fa : fb`` chunk by chunk, in ``u``'s dtype
    (``np.place`` into a ``u.dtype`` factor vector, big-wave/optical_element.py:165-172)."""
    fa = np.asarray(fa).astype(u.dtype)
    fb = np.asarray(fb).astype(u.dtype)
    out = u.copy()
    for idx, cnt in _chunks(sim.N, sim.chunk_size):
        m = mask_fn(idx - sim.N // 2, cnt)
        out[idx:idx + cnt] = u[idx:idx + cnt] * np.where(m, fa, fb)
    return out


def _lookup_db(db_table, mat):
    """``extract_from_deltabeta_table`` (big-wave/optical_element.py:42-63)."""
    if mat is None:
        return np.complex128(0.0)
    cands = sorted(
        (abs(m[1] - mat[1]), complex(v[0], v[1])) for m, v in db_table if m[0] == mat[0]
    )
    assert cands and cands[0][0] < 1e-5, f"material {mat} not in deltabeta table"
    return np.complex128(cands[0][1])


def apply_grating(u, U, sim, el, db_table, cutoff, step_idx, dba=False, hist=None):
    """``Grating.apply`` / ``DBAGrating.apply`` (big-wave/optical_element.py:134-206,
    :247-319): ``nr_steps`` x [binary mask multiply, propagate(thickness/nr_steps)],
    then the substrate as a scalar factor and one more propagate. ``hist``
    (a list) receives the detector image after every sub-step (:181-186)."""
    z_step = el["thickness"] / el["nr_steps"]
    fa = material_factor(_lookup_db(db_table, el.get("mat_a")), z_step, sim.wl)
    fb = material_factor(_lookup_db(db_table, el.get("mat_b")), z_step, sim.wl)
    x_pos = el["x_positions"][step_idx]
    for i in range(el["nr_steps"]):
        if dba:
            dc0 = interpolated_dc(el["dc0"], i, el["nr_steps"])
            dc1 = interpolated_dc(el["dc1"], i, el["nr_steps"])
            fn = lambda s, c: dba_mask_chunk(sim.dx, s, c, el["pitch0"], el["pitch1"],
                                             dc0, dc1, x_pos)
        else:
            dc = interpolated_dc(el["dc"], i, el["nr_steps"])
            fn = lambda s, c: grating_mask_chunk(sim.dx, s, c, el["pitch"], dc, x_pos)
        u = _apply_binary(u, sim, fn, fa, fb)
        u, U = propagate(u, U, sim, z_step, cutoff)
        if hist is not None:
            z = el["z_start"] + (i + 1) * z_step
            hist.append((square_and_downsample(u, sim, z), z))
    t_sub = el["substrate_thickness"]
    if t_sub > 0:
        fs = material_factor(_lookup_db(db_table, el.get("mat_substrate")), t_sub, sim.wl)
        u = (u * fs).astype(u.dtype)
        u, U = propagate(u, U, sim, t_sub, cutoff)
    return u, U


def sample_row_coordinates(rowlen, psx, x_pos):
    """``row_x`` of ``Sample.apply`` (big-wave/optical_element.py:442-446)."""
    return np.arange(rowlen) * psx + x_pos - rowlen * psx * 0.5


def apply_sample(u, U, sim, el, grid, db_table, cutoff, step_idx, hist=None):
    """``Sample.apply`` (big-wave/optical_element.py:432-476): per z-row,
    linear interpolation (``np.interp`` with zero outside) of the row's delta+i*beta
    at the field's x, ``exp(i 2 pi dz/wl * db)``, then propagate(pixel_size_z).
    ``hist`` receives the detector image before every row (:447-452)."""
    db_list = np.zeros(len(el["materials"]) + 1, dtype=np.complex128)
    for i, m in enumerate(el["materials"]):
        db_list[i + 1] = _lookup_db(db_table, m)
    psx, psz = el["pixel_size_x"], el["pixel_size_z"]
    row_x = sample_row_coordinates(grid.shape[1], psx, el["x_positions"][step_idx])
    for r in range(grid.shape[0]):
        if hist is not None:
            z = el["z_start"] + r * psz
            hist.append((square_and_downsample(u, sim, z), z))
        row_db = db_list[grid[r, :]]
        out = u.copy()
        for idx, cnt in _chunks(sim.N, sim.chunk_size):
            start = idx - sim.N / 2
            x = np.arange(start, start + cnt) * sim.dx
            db = np.interp(x, xp=row_x, fp=row_db, left=0.0, right=0.0)
            out[idx:idx + cnt] = u[idx:idx + cnt] * material_factor(db, psz, sim.wl)
        u = out.astype(u.dtype)
        u, U = propagate(u, U, sim, psz, cutoff)
    return u, U


# --------------------------------------------------------------------------
# sources and detection
# --------------------------------------------------------------------------
def point_source_field(sim: Sim, z: float, x_source: float, dtype) -> np.ndarray:
    """``propagate_analytically`` (big-wave/propagation.py:141-151)."""
    x = (np.arange(sim.N, dtype=np.float64) - sim.N / 2) * sim.dx - x_source
    r = np.sqrt(x**2 + z**2)
    return (np.exp(r * (-2j * np.pi / sim.wl)) / np.sqrt(r)).astype(dtype)


def detector_x(detector_size: float, psx: float) -> np.ndarray:
    """``detector_x_vector`` (big-wave/util.py:78-82)."""
    n = detector_size // psx
    return (np.arange(n) - n // 2) * psx


def square_and_downsample(u, sim: Sim, z: float) -> np.ndarray:
    """``square_and_downsample`` (big-wave/propagation.py:279-320): |u|^2
    binned by ``np.histogram`` over ``n+1`` uniform bins of
    ``[-(n/2) psx, (n/2+1) psx]`` (last bin dropped), then the cos/r scaling."""
    outsize = int(sim.detector_size // sim.psx)
    rng = (-(outsize / 2) * sim.psx, (outsize / 2 + 1) * sim.psx)
    out = np.zeros(outsize, dtype=np.float64)
    for idx, cnt in _chunks(sim.N, sim.chunk_size):
        chunk = u[idx:idx + cnt]
        pos = (idx + np.arange(cnt) - sim.N / 2) * sim.dx
        w = chunk.real * chunk.real + chunk.imag * chunk.imag
        out += np.histogram(pos, bins=outsize + 1, range=rng, weights=w)[0][:-1]
    x = detector_x(sim.detector_size, sim.psx)
    ang = np.arctan(x / z)
    return out * np.cos(ang) * sim.dx * sim.psy / np.sqrt(x**2 + z**2)


def element_thickness(el) -> float:
    if el["type"] == "sample":
        return el["pixel_size_z"] * np.asarray(el["_grid"]).shape[0]
    return el["thickness"] + el["substrate_thickness"]


# --------------------------------------------------------------------------
# per-source schedule
# --------------------------------------------------------------------------
def make_sim(case) -> Sim:
    sp = case["sim_params"]
    return Sim(N=int(sp["N"]), dx=float(sp["dx"]), z_detector=float(sp["z_detector"]),
               detector_size=float(sp["detector_size"]),
               psx=float(sp["detector_pixel_size_x"]),
               psy=float(sp["detector_pixel_size_y"]),
               wl=wavelength_from_energy(float(case["energy"])),
               chunk_size=int(sp["chunk_size"]),
               propagator=str(case.get("propagator", "fresnel")))


def history_zs(dz, hdz):
    """z offsets visited by ``propagate_with_history`` (big-wave/history.py:90-97)."""
    zs = np.arange(0, dz, hdz)
    if dz - zs[-1] < hdz / 2.0 and len(zs) > 1:
        zs[-1] = dz
    else:
        zs = np.append(zs, [dz])
    return zs


def propagate_with_history(u, U, sim, dz, cutoff, current_z, skip_fft, hist, hdz):
    """``propagate_with_history`` (big-wave/history.py:67-135): every history
    point is reached from the spectrum at the start of the gap."""
    if dz == 0:
        return u, U
    if hist is None:
        return propagate(u, U, sim, dz, cutoff, skip_fft=skip_fft)
    zs = history_zs(dz, hdz)
    if not skip_fft:
        U = spfft.fft(u)
    U_start = U.copy()
    for i in range(1, len(zs)):
        u, U = propagate(u, U_start.copy(), sim, zs[i] - zs[0], cutoff, skip_fft=True)
        z = zs[i] + current_z
        hist.append((square_and_downsample(u, sim, z), z))
    return u, U


def analytic_history(hist, zs, x_source, sim, cutoff):
    """``generate_analytic_history`` (big-wave/history.py:43-64): the point
    source's intensity on the detector grid at each z, zero outside the cutoff
    cone."""
    gradient = cutoff * sim.wl
    n = sim.detector_size // sim.psx
    x = (np.arange(n) - n // 2) * sim.psx - x_source
    for z in zs:
        angle = np.arctan(x / z)
        r2 = x ** 2 + z ** 2
        inten = sim.psx * sim.psy * np.cos(angle) / r2
        inten[np.abs(x) > gradient * z] = 0
        hist.append((inten, z))


def run_simulation(case, grids=None, dtype=np.complex128, return_fields=False, history_dz=None, keypoints=None):
    """``run_simulation`` (big-wave/wavesim.py:84-298) for one source: source
    initialisation, element loop with gap propagation, final gap reusing the
    spectrum (``skip_fft``), detection, then the remaining phase steps
    restarted from the snapshot taken before the first stepped element.

    ``grids`` maps element index -> int8 grid for sample elements.
    Returns the detector array ``(nr_phase_steps, n_pix)`` (and the final
    fields of every phase step when ``return_fields``). With ``history_dz``
    the first pass records the history (big-wave/wavesim.py:153-219) and the
    result is ``(detector, history (n_pix, entries), z of each entry)``.
    A ``keypoints`` list receives copies of the field right before and right
    after each element of the first pass (big-wave/wavesim.py:35-55, :186,
    :196), in element order."""
    hist = [] if history_dz else None
    grids = grids or {}
    sim = make_sim(case)
    elements = [dict(e) for e in case["elements"]]
    for i, e in enumerate(elements):
        if e["type"] == "sample":
            e["_grid"] = grids[i]
    db_table = case["db"]
    cut = [np.sin(a) / sim.wl for a in case["cutoff_angles"]]
    z_tol = 1e-8

    def apply(el, u, U, cutoff, step, h=None):
        if el["type"] == "grating":
            return apply_grating(u, U, sim, el, db_table, cutoff, step, hist=h)
        if el["type"] == "dba_grating":
            return apply_grating(u, U, sim, el, db_table, cutoff, step, dba=True, hist=h)
        if el["type"] == "sample":
            return apply_sample(u, U, sim, el, el["_grid"], db_table, cutoff, step, hist=h)
        raise ValueError(el["type"])

    # source.propagate_to (big-wave/source.py:46-101)
    cutoff = cut[0]
    z = elements[0]["z_start"] if elements else sim.z_detector
    src = case["source"]
    U = None
    if src["type"] == "point":
        u = point_source_field(sim, z - src["z"], src["x"], dtype)
        Us = spfft.fft(u)
        rng = cutoff_zero_range(sim.N, cutoff, sim.dx)
        if rng is not None:
            Us[rng[0]:rng[1]] = 0
        u = spfft.ifft(Us)
        if hist is not None:
            analytic_history(hist, np.arange(0, z, history_dz)[1:], src["x"], sim, cutoff)
    else:
        u0 = np.ones(sim.N, dtype) if src["type"] == "plane" else np.asarray(src["u"], dtype)
        dz = z - src["z"]
        if dz == 0:
            u = u0.copy()
        else:
            u, U = propagate_with_history(u0, spfft.fft(u0), sim, dz, cutoff, src["z"], True, hist, history_dz)

    snapshot = None
    for i, el in enumerate(elements):
        if z < el["z_start"]:
            u, U = propagate_with_history(u, U, sim, el["z_start"] - z, cutoff, z, False, hist, history_dz)
        z = el["z_start"]
        if len(el["x_positions"]) > 1 and snapshot is None:
            snapshot = (z, i, u.copy(), len(el["x_positions"]))
        cutoff = cut[i + 1]
        if keypoints is not None:
            keypoints.append(u.copy())
        u, U = apply(el, u, U, cutoff, 0, hist)
        if keypoints is not None:
            keypoints.append(u.copy())
        z = el["z_start"] + element_thickness(el)
    if z < sim.z_detector - z_tol:
        u, U = propagate_with_history(u, U, sim, sim.z_detector - z, cutoff, z, len(elements) > 0, hist,
                                      history_dz)
    outs = [square_and_downsample(u, sim, sim.z_detector)]
    fields = [u]

    if snapshot is not None:
        z0, i0, u0, nsteps = snapshot
        for step in range(1, nsteps):
            z, u, cutoff = z0, u0.copy(), cut[i0]
            for i in range(i0, len(elements)):
                el = elements[i]
                if z < el["z_start"]:
                    u, U = propagate(u, U, sim, el["z_start"] - z, cutoff)
                z = el["z_start"]
                cutoff = cut[i + 1]
                u, U = apply(el, u, U, cutoff, step if len(el["x_positions"]) > 1 else 0)
                z = el["z_start"] + element_thickness(el)
            if z < sim.z_detector - z_tol:
                u, U = propagate(u, U, sim, sim.z_detector - z, cutoff)
            outs.append(square_and_downsample(u, sim, sim.z_detector))
            fields.append(u)
    det = np.array(outs)
    if hist is not None:
        h = np.stack([e for e, _ in hist], axis=-1) if hist else np.empty((0, 0))
        return det, h, np.array([z for _, z in hist], dtype=np.float64)
    return (det, fields) if return_fields else det


def count_split_steps(case, grids=None) -> int:
    """Number of ``propagate`` calls of ``run_simulation``'s schedule (the
    throughput numerator: one split step = one FFT/transfer/iFFT round)."""
    elements = case["elements"]
    n_el = len(elements)
    z_tol = 1e-8

    def el_steps(i):
        el = elements[i]
        if el["type"] == "sample":
            return np.asarray(grids[i]).shape[0]
        return el["nr_steps"] + (1 if el["substrate_thickness"] > 0 else 0)

    def thick(i):
        el = elements[i]
        if el["type"] == "sample":
            return el["pixel_size_z"] * np.asarray(grids[i]).shape[0]
        return el["thickness"] + el["substrate_thickness"]

    src = case["source"]
    z = elements[0]["z_start"] if elements else case["sim_params"]["z_detector"]
    steps = 1 if (src["type"] == "point" or z - src["z"] != 0) else 0
    snap = None
    for i in range(n_el):
        if z < elements[i]["z_start"]:
            steps += 1
        z = elements[i]["z_start"]
        if len(elements[i]["x_positions"]) > 1 and snap is None:
            snap = (z, i, len(elements[i]["x_positions"]))
        steps += el_steps(i)
        z = elements[i]["z_start"] + thick(i)
    zd = case["sim_params"]["z_detector"]
    if z < zd - z_tol:
        steps += 1
    if snap is not None:
        z0, i0, n = snap
        per = 0
        z = z0
        for i in range(i0, n_el):
            if z < elements[i]["z_start"]:
                per += 1
            z = elements[i]["z_start"]
            per += el_steps(i)
            z = elements[i]["z_start"] + thick(i)
        if z < zd - z_tol:
            per += 1
        steps += per * (n - 1)
    return steps


def case_from_simdir_yaml(config: dict, computed: dict, subconfig: dict) -> dict:
    """Build a case from the three YAML documents of a reference simulation
    directory (``config.yaml``, ``computed.yaml``, ``NNNNNNNN/subconfig.yaml``;
    read by ``multisim.run_single_simulation``, big-wave/multisim.py:70-112).
    Sample grids are not loaded here."""
    sp = config["sim_params"]
    src = subconfig["source"]
    if src["type"] == "point":
        source = {"type": "point", "x": float(src["x"]), "z": float(src["z"])}
    else:
        source = {"type": "vector", "z": float(src["z"]), "path": src["input_path"]}
    return {
        "sim_params": {k: sp[k] for k in ("N", "dx", "z_detector", "detector_size",
                                          "detector_pixel_size_x",
                                          "detector_pixel_size_y", "chunk_size")},
        "elements": [dict(e) for e in config["elements"]],
        "source": source,
        "energy": float(subconfig["energy"]),
        "db": [[list(m), list(v)] for m, v in subconfig["deltabeta_table"]],
        "cutoff_angles": [float(a) for a in computed["cutoff_angles"]],
        "dtype": config.get("dtype", "c16"),
    }
