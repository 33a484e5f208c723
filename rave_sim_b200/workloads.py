"""Synthetic Talbot-Lau workloads in the reference's configuration schema.

Seeded, deterministic stand-ins for the benchmark setups of the hot path
(there is no public dataset for it). Each builder returns a ``case`` dict:
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
