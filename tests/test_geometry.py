"""big-wave's geometry helpers (grid_density_check, max_dx,
compute_cutoff_angles; big-wave/propagation.py:31-66, :178-276) restated in
rave_sim_b200.geometry, against the reference's own outputs on the same
arguments (tests/golden/geometry.json, made by
tests/golden/make_geometry_golden.py): the same floats, the same
exceptions."""

import json
import math

import numpy as np
import pytest

from conftest import GOLDEN
from rave_sim_b200 import geometry as g

GEO = json.loads((GOLDEN / "geometry.json").read_text())


@pytest.mark.parametrize("case", GEO["compute_cutoff_angles"], ids=lambda c: str(c["args"][:2]))
def test_compute_cutoff_angles_matches_reference(case):
    a = case["args"]
    args = (a[0], a[1], tuple(a[2]), *a[3:])
    if "raises" in case:
        with pytest.raises(ValueError):
            g.compute_cutoff_angles(*args)
        return
    angles, xs = g.compute_cutoff_angles(*args)
    assert angles == case["angles"]  # bit-identical floats
    assert xs == case["max_x"]


def test_slope_bound_case_is_exercised():
    # one golden case has the lowest energy's slope bound active
    c = GEO["compute_cutoff_angles"][3]
    dx, wl = c["args"][1], g.wavelength_from_energy(c["args"][2][0])
    bound = math.atan(math.tan(math.asin(2 * wl / dx)))
    assert any(abs(x - bound) < 1e-15 for x in c["angles"])


@pytest.mark.parametrize("case", GEO["max_dx"], ids=lambda c: str(c["args"][:2]))
def test_max_dx_matches_reference(case):
    assert g.max_dx(*case["args"]) == case["result"]
    # the returned dx passes the density check
    dz, xs, n, wl = case["args"]
    g.grid_density_check(dz, xs, n, case["result"], wl)


@pytest.mark.parametrize("case", GEO["grid_density_check"], ids=lambda c: str(c["args"][3]))
def test_grid_density_check_matches_reference(case):
    if case["ok"]:
        g.grid_density_check(*case["args"])
    else:
        with pytest.raises(ValueError):
            g.grid_density_check(*case["args"])


def test_cutoff_argument_checks():
    with pytest.raises(AssertionError):
        g.compute_cutoff_angles(1e-3, 1e-9, (2e4, 3e4), 0.0, [0.1], [], 0.5, 0.0)
    with pytest.raises(AssertionError):
        g.compute_cutoff_angles(1e-3, 1e-9, (3e4, 2e4), 0.0, [], [], 0.5, 0.0)
    with pytest.raises(ValueError):
        g.compute_cutoff_angles(1e-3, 1e-9, (2e4, 3e4), 0.0, [0.5], [1e-4], 0.5, 0.0)
    assert np.isfinite(g.compute_cutoff_angles(1e-3, 1e-9, (2e4, 3e4), 0.0, [], [], 0.5, 0.0)[0][0])
