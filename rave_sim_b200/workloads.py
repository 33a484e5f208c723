"""Synthetic Talbot-Lau workloads in the reference's configuration schema.

Seeded, deterministic stand-ins for the benchmark setups of the hot path
(there is no public dataset for it): ``single_grating`` (one pi-phase
grating), ``talbot_lau`` (three-grating interferometer, 32 energies x 8
phase steps), ``batched_energies`` (the interferometer over 128 energies with
per-energy field lengths 2^20..2^25), ``thick_sample`` (a 200-slice cracked
aluminium cylinder between G1 and G2) and ``large_field`` (2^30/2^31-sample
fields). Each builder returns a ``case`` dict:
the reference's config.yaml keys (``sim_params``, ``elements``, ``dtype``)
plus ``cutoff_angles`` (computed.yaml) and per-source entries (``energy``,
``db`` = subconfig deltabeta table, ``source``).

Material values: delta and beta at 46 keV scaled as delta ~ E^-2 and
beta ~ E^-4; source spectrum: Kramers bremsstrahlung (E_max - E)/E filtered by
3 mm of aluminium (attenuation table generated from the reference's material
lookup, tests/golden/al_attenuation.npz).
"""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np

from .engine import wavelength_from_energy

PITCH = 4.2e-6
E_REF = 46000.0
AU_46 = (1.44e-6, 8e-9)
SI_46 = (2.27e-7, 1e-10)
AU = ["Au", 19.32]
SI = ["Si", 2.34]
_AL_TABLE = Path(__file__).resolve().parents[1] / "tests" / "golden" / "al_attenuation.npz"


def deltabeta_at(db46, energy):
    d, b = db46
    r = E_REF / energy
    return [d * r * r, b * r ** 4]


def db_table(energy):
    return [[AU, deltabeta_at(AU_46, energy)], [SI, deltabeta_at(SI_46, energy)]]


def al_mu_per_cm(energy):
    d = np.load(_AL_TABLE)
    return float(np.exp(np.interp(np.log(energy), np.log(d["energy_ev"]), np.log(d["mu_per_cm"]))))


def kramers_weights(energies, e_max=70000.0, al_cm=0.3):
    w = np.array([max(e_max - e, 0.0) / e * math.exp(-al_mu_per_cm(e) * al_cm) for e in energies])
    return w / w.sum()


def _grating(z, thickness, mat, x_positions, nr_steps):
    return {"type": "grating", "pitch": PITCH, "dc": [0.5, 0.5], "z_start": z, "thickness": thickness,
            "nr_steps": nr_steps, "x_positions": list(x_positions), "substrate_thickness": 0.0,
            "mat_a": mat, "mat_b": None, "mat_substrate": None}


def talbot_lau(n=1 << 24, dx=2e-9, dtype="c16", nr_steps=10, phase_steps=8, detector_size=2.048e-3,
               pixel_size=1e-6):
    """Three-grating Talbot-Lau interferometer (benchmark config 2 shape):
    G0 Au absorption grating at z = 0 (h = 100 um), G1 pi-phase Si grating at
    0.8 m (59.37 um, pi at 46 keV), G2 Au analyser at 0.882 m (h = 100 um)
    stepped over ``phase_steps`` positions of p/phase_steps, detector at the
    G2 exit, plane-wave illumination at z = 0, no frequency cutoff."""
    h_g1 = wavelength_from_energy(E_REF) / (2 * SI_46[0])
    z1, z2 = 0.8, 0.882
    els = [
        _grating(0.0, 100e-6, AU, [0.0], nr_steps),
        _grating(z1, h_g1, SI, [0.0], nr_steps),
        _grating(z2, 100e-6, AU, [k * PITCH / phase_steps for k in range(phase_steps)], nr_steps),
    ]
    return {
        "sim_params": {"N": int(n), "dx": float(dx), "z_detector": z2 + 100e-6, "detector_size": detector_size,
                       "detector_pixel_size_x": pixel_size, "detector_pixel_size_y": 1.0, "chunk_size": int(n)},
        "elements": els,
        "dtype": dtype,
        "cutoff_angles": [math.pi / 2] * (len(els) + 1),
        "source": {"type": "plane", "z": 0.0},
        "energy": E_REF,
        "db": db_table(E_REF),
    }


def config2_energies(count=32, e_min=20000.0, e_max=70000.0):
    """Energies and normalised spectrum weights of the config-2 batch."""
    e = np.linspace(e_min, e_max, count)
    return e, kramers_weights(e, e_max)


def single_grating(n=1 << 20, dx=2e-9, dtype="c16", nr_steps=10):
    """Benchmark config 1: plane wave through one pi-phase Si grating at
    46 keV, then the first fractional Talbot distance p^2/(8 wl), 1 um pixels."""
    wl = wavelength_from_energy(E_REF)
    h = wl / (2 * SI_46[0])
    d = PITCH * PITCH / (8 * wl)
    z0 = 0.1
    return {
        "sim_params": {"N": int(n), "dx": dx, "z_detector": z0 + h + d, "detector_size": 2.048e-3,
                       "detector_pixel_size_x": 1e-6, "detector_pixel_size_y": 1.0, "chunk_size": int(n)},
        "elements": [_grating(z0, h, SI, [0.0], nr_steps)],
        "dtype": dtype,
        "cutoff_angles": [math.pi / 2] * 2,
        "source": {"type": "plane", "z": z0},
        "energy": E_REF,
        "db": [[SI, list(SI_46)]],
    }


# ---------------------------------------------------------------- batched
def batched_energies(count=128, e_min=20000.0, e_max=70000.0, log_min=20, log_max=25, window=None,
                     dtype="c8", nr_steps=10, phase_steps=8):
    """Benchmark config 3: the interferometer over ``count`` energies, energy
    j (ascending) on a field of N_j = 2^(log_min + floor((log_max - log_min + 1) j / count))
    samples over a fixed window (default 2^log_max * 1 nm), dx_j = window / N_j.
    Returns a list of groups ``(case, energies, weights)``, one per field
    length; ``case["energy"]``/``case["db"]`` are per-energy (see ``db_table``)."""
    levels = log_max - log_min + 1
    win = window if window is not None else float(1 << log_max) * 1e-9
    e = np.linspace(e_min, e_max, count)
    w = kramers_weights(e, e_max)
    groups = []
    for lg in range(log_min, log_max + 1):
        idx = [j for j in range(count) if log_min + (levels * j) // count == lg]
        if not idx:
            continue
        n = 1 << lg
        case = talbot_lau(n=n, dx=win / n, dtype=dtype, nr_steps=nr_steps, phase_steps=phase_steps)
        groups.append((case, e[idx], w[idx]))
    return groups


# ------------------------------------------------------------ thick sample
AL = ["Al", 2.70]
# delta of aluminium at 46 keV from silicon's by the electron-density ratio
# (rho Z / A: Al 2.70 * 13 / 26.982, Si 2.34 * 14 / 28.086)
AL_DELTA_46 = SI_46[0] * (2.70 * 13 / 26.982) / (2.34 * 14 / 28.086)


def al_deltabeta(energy):
    """delta ~ E^-2 from the 46 keV value; beta = mu wl / (4 pi) from the
    tabulated attenuation."""
    wl = wavelength_from_energy(energy)
    r = E_REF / energy
    return [AL_DELTA_46 * r * r, al_mu_per_cm(energy) * 100.0 * wl / (4 * math.pi)]


def db_table_sample(energy):
    return db_table(energy) + [[AL, al_deltabeta(energy)]]


def cracked_cylinder(rows=200, cols=4000, psz=10e-6, psx=0.5e-6, diameter=2e-3, cracks=50,
                     axis_range=(1e-6, 20e-6), seed=4):
    """int8 grid [rows, cols] of a z-x section through an aluminium cylinder
    (material 1) with ``cracks`` elliptical air cracks (material 0). Crack
    centres are uniform inside the disk, semi-axes uniform in ``axis_range``,
    orientation uniform in [0, pi); each cell is classified by its centre."""
    rng = np.random.default_rng(seed)
    rad = diameter / 2
    zc = (np.arange(rows) + 0.5) * psz - rows * psz / 2
    xc = (np.arange(cols) + 0.5) * psx - cols * psx / 2
    Z, X = np.meshgrid(zc, xc, indexing="ij")
    grid = (Z * Z + X * X <= rad * rad).astype(np.int8)
    for _ in range(cracks):
        while True:
            cz, cx = rng.uniform(-rad, rad, 2)
            if cz * cz + cx * cx <= rad * rad:
                break
        a, b = rng.uniform(axis_range[0], axis_range[1], 2)
        th = rng.uniform(0.0, math.pi)
        dz, dx = Z - cz, X - cx
        u = dz * math.cos(th) + dx * math.sin(th)
        v = -dz * math.sin(th) + dx * math.cos(th)
        grid[(u / a) ** 2 + (v / b) ** 2 <= 1.0] = 0
    return grid


def thick_sample(n=1 << 26, dx=50e-9, dtype="c8", nr_steps=10, phase_steps=8, rows=200, cols=4000,
                 psz=10e-6, psx=0.5e-6, gap=1e-3, seed=4, diameter=2e-3, axis_range=(1e-6, 20e-6),
                 detector_size=2.048e-3, pixel_size=1e-6):
    """Benchmark config 4: the interferometer with a ``sample`` element (the
    cracked cylinder of ``cracked_cylinder``) starting ``gap`` after the G1
    exit. Returns (case, grids) with the grid under element index 2; the
    deltabeta table of an energy is ``db_table_sample``. The phantom and
    detector arguments scale the setup down for parity tests."""
    case = talbot_lau(n=n, dx=dx, dtype=dtype, nr_steps=nr_steps, phase_steps=phase_steps,
                      detector_size=detector_size, pixel_size=pixel_size)
    g1 = case["elements"][1]
    z0 = g1["z_start"] + g1["thickness"] + gap
    grid = cracked_cylinder(rows, cols, psz, psx, diameter=diameter, axis_range=axis_range, seed=seed)
    sample = {"type": "sample", "z_start": z0, "pixel_size_x": psx, "pixel_size_z": psz,
              "grid_path": "cracked_cylinder.npy", "materials": [AL], "x_positions": [0.0]}
    case["elements"].insert(2, sample)
    case["cutoff_angles"] = [math.pi / 2] * (len(case["elements"]) + 1)
    case["db"] = db_table_sample(E_REF)
    return case, {2: grid}


# ------------------------------------------------------------- large field
def large_field(dtype="c8", n=None, dx=5e-9, nr_steps=10, phase_steps=8, pixel_size=75e-6,
                detector_size=9.6e-3):
    """Benchmark config 5: the interferometer on one large field, 2^31
    complex64 or 2^30 complex128 samples at 5 nm, 75 um detector pixels."""
    if n is None:
        n = 1 << (31 if dtype == "c8" else 30)
    return talbot_lau(n=n, dx=dx, dtype=dtype, nr_steps=nr_steps, phase_steps=phase_steps,
                      detector_size=detector_size, pixel_size=pixel_size)
