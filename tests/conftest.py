import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_case(name):
    """Golden case: (case dict, grids by element index, npz arrays)."""
    d = np.load(GOLDEN / f"case_{name}.npz")
    case = json.loads(str(d["case_json"]))
    grids = {i: d["grid"] for i, e in enumerate(case["elements"]) if e["type"] == "sample"}
    return case, grids, d


def case_names():
    return sorted(p.stem[len("case_"):] for p in GOLDEN.glob("case_*.npz"))


def load_snapshot_case():
    import yaml
    from oracle import bigwave_np as bw

    d = np.load(GOLDEN / "snapshot.npz")
    case = bw.case_from_simdir_yaml(
        yaml.safe_load(str(d["config_yaml"])),
        yaml.safe_load(str(d["computed_yaml"])),
        yaml.safe_load(str(d["subconfig_yaml"])),
    )
    return case, d


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
