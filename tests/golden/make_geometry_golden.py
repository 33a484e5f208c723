"""Generate tests/golden/geometry.json by running the reference's own
big-wave geometry helpers (big-wave/propagation.py: grid_density_check
:31-45, max_dx :48-66, compute_cutoff_angles :178-276) on a set of cases,
through the import stand-ins of make_golden.py.

Usage:  python tests/golden/make_geometry_golden.py [/path/to/reference]
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from make_golden import _install_stubs  # noqa: E402

# compute_cutoff_angles(detector_size, dx, energy_range, z_source, z_distances,
#                       element_heights, z_detector, max_x)
CUTOFF_CASES = [
    # Talbot-Lau, source at the first grating, detector at the G2 exit
    [2.048e-3, 2e-9, [20000.0, 70000.0], 0.0, [0.0, 0.8, 0.882], [100e-6, 59.37e-6, 100e-6], 0.8821, 0.0],
    # point source 0.1 m before G0, gap to the detector
    [2.048e-3, 1e-9, [30000.0, 60000.0], -0.1, [0.0, 0.5], [50e-6, 40e-6], 1.2, 5e-6],
    # no elements
    [1e-3, 5e-9, [46000.0, 46000.0], 0.0, [], [], 0.3, 1e-6],
    # coarse grid: the lowest energy's slope bound is active
    [1.5e-4, 2e-7, [10000.0, 80000.0], 0.0, [0.49], [1e-4], 0.5, 0.0],
    # the highest energy does not cover the detector: ValueError
    [5e-2, 1e-6, [50000.0, 90000.0], 0.0, [0.01], [1e-4], 0.02, 1e-3],
]
# max_dx(dz, x_source, N, wl)
MAXDX_CASES = [[0.1, 0.0, 1 << 20, 2.695e-11], [0.5, 1e-5, 1 << 24, 6.2e-11], [1.0, 2e-4, 1 << 16, 1e-10],
               [0.02, 0.0, 1 << 22, 2.7e-11]]
# grid_density_check(dz, x_source, N, dx, wl)
DENSITY_CASES = [[0.1, 0.0, 1 << 20, 1e-9, 2.695e-11], [0.1, 0.0, 1 << 20, 1e-6, 2.695e-11],
                 [0.05, 1e-5, 1 << 18, 2e-9, 5e-11], [0.5, 0.0, 1 << 16, 5e-8, 2.7e-11]]


def main(ref: Path) -> None:
    _install_stubs(ref)
    import config  # noqa: F401  (first: breaks the propagation<->config import cycle)
    import propagation as p

    out = {"compute_cutoff_angles": [], "max_dx": [], "grid_density_check": []}
    for args in CUTOFF_CASES:
        try:
            angles, xs = p.compute_cutoff_angles(*args[:2], tuple(args[2]), *args[3:])
            out["compute_cutoff_angles"].append({"args": args, "angles": angles, "max_x": xs})
        except ValueError:
            out["compute_cutoff_angles"].append({"args": args, "raises": "ValueError"})
    for args in MAXDX_CASES:
        out["max_dx"].append({"args": args, "result": p.max_dx(*args)})
    for args in DENSITY_CASES:
        try:
            p.grid_density_check(*args)
            out["grid_density_check"].append({"args": args, "ok": True})
        except ValueError:
            out["grid_density_check"].append({"args": args, "ok": False})
    (HERE / "geometry.json").write_text(json.dumps(out, indent=1))
    print("wrote", HERE / "geometry.json")


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference"))
