"""Simulation-geometry helpers of big-wave's propagation module, host side.

``grid_density_check`` (big-wave/propagation.py:31-45), ``max_dx`` (:48-66)
and ``compute_cutoff_angles`` (:178-276) with the reference's signatures,
results and exceptions, so a setup written for big-wave (its
``setup_simulation`` computes the cutoff angles of computed.yaml with
``compute_cutoff_angles``) can be prepared without the reference. The
arithmetic follows the reference's operations in the same order, so the
results are the same floats (checked against the reference's own outputs in
tests/test_geometry.py).
"""

from __future__ import annotations

import math
from typing import Sequence, Tuple

import numpy as np

from .engine import wavelength_from_energy


def grid_density_check(dz: float, x_source: float, N: int, dx: float, wl: float) -> None:
    """Raise ValueError when neighbouring samples of the analytically
    propagated point-source field (distance dz, source at x_source) differ in
    path length by more than half a wavelength (the Nyquist condition)."""
    def path(i):
        return np.sqrt(((N / 2 - i) * dx + np.abs(x_source)) ** 2 + dz ** 2)

    if not np.abs(path(0) - path(1)) <= wl / 2:
        raise ValueError("Nyquist not satisfied, dx too large: max_dx(dz, x_source, N, wl) gives the largest "
                         "dx that passes")


def max_dx(dz: float, x_source: float, N: int, wl: float) -> float:
    """The largest dx that passes grid_density_check, to 1 %: bisection of
    [0, 0.1] until the interval's relative width is at most 1 %, returning its
    lower end (the reference's search, so the same value)."""
    lo, hi = 0.0, 0.1
    while (hi - lo) / hi > 0.01:
        mid = (hi + lo) / 2
        try:
            grid_density_check(dz, x_source, N, mid, wl)
        except ValueError:
            hi = mid
        else:
            lo = mid
    return lo


def compute_cutoff_angles(detector_size: float, dx: float, energy_range: Tuple[float, float], z_source: float,
                          z_distances: Sequence[float], element_heights: Sequence[float], z_detector: float,
                          max_x: float) -> Tuple[list, list]:
    """Frequency cutoff angles per free-space section (source to the first
    element, between elements, to the detector) that keep every ray from
    source positions |x| <= max_x reaching the detector, and the largest |x|
    reached at each element start and at the detector.

    The ray slope of a section is what reaches the detector edge from the
    current extent, bounded by the largest angle the grid resolves at the
    lowest energy (arcsin(2 wl_max / dx)); the extent grows by slope * length.
    When the detector sits right after the last element, the last section
    keeps the previous slope. Raises ValueError when the grid is too coarse
    for the highest energy to cover the detector, AssertionError on
    inconsistent arguments, as the reference does."""
    if len(z_distances) != len(element_heights):
        raise AssertionError("z_distances and element_heights differ in length")
    if not energy_range[0] <= energy_range[1]:
        raise AssertionError("energy_range must be (min, max)")
    wl_long = wavelength_from_energy(energy_range[0])
    wl_short = wavelength_from_energy(energy_range[1])

    edge_angle = np.arctan((detector_size / 2 + max_x) / z_detector)
    if 2 / (np.sin(edge_angle) / wl_short) < dx:
        need = 2 / (np.sin(edge_angle) / wl_short)
        raise ValueError(f"Grid sampled too coarsely: the highest energy's waves do not cover the detector; the "
                         f"edge angle {edge_angle * 180.0 / math.pi} degrees needs dx <= {need}")

    # the steepest slope the grid holds at the lowest energy (no bound when
    # even 90 degrees is resolved)
    slope_cap = float(np.inf)
    if wl_long * 2 / dx < 1:
        slope_cap = np.tan(np.arcsin(wl_long * 2 / dx))

    extent = max_x
    z = z_source
    slopes: list = []
    extents: list = []
    for z_next in list(z_distances) + [z_detector]:
        if z == z_detector:
            raise ValueError("an element starts at the detector's z coordinate")
        slopes.append(min((detector_size / 2 + extent) / (z_detector - z), slope_cap))
        extent += slopes[-1] * (z_next - z)
        extents.append(float(extent))
        z = z_next
    if not extent >= detector_size / 2:
        raise AssertionError("the rays do not cover the detector")

    if len(z_distances) > 0 and np.abs(z_detector - (z_distances[-1] + element_heights[-1])) < 1e-8:
        slopes[-1] = slopes[-2]
        extents[-1] = extents[-2] + slopes[-1] * element_heights[-1]
    return [float(np.arctan(s)) for s in slopes], extents
