"""rave_sim_b200: B200-native split-step wavefront propagation (rave-sim hot path).

The CUDA engine lives in ``librsw.so`` (built in-tree from ``csrc/`` by
``python -m rave_sim_b200.build``) behind the C ABI of ``include/rsw.h``.
"""

from ._lib import RswError, load as load_library  # noqa: F401
from .engine import Plan, Simulation, run_case, wavelength_from_energy  # noqa: F401
from .retrieval import dark_field, signal_retrieval_least_squares  # noqa: F401

__all__ = ["Plan", "Simulation", "run_case", "wavelength_from_energy", "RswError", "load_library",
           "signal_retrieval_least_squares", "dark_field"]
from .geometry import compute_cutoff_angles, grid_density_check, max_dx  # noqa: E402,F401
