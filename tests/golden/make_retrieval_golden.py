"""Generate tests/golden/retrieval.npz by running the reference's own
phase-stepping signal retrieval: ``signal_retrieval_least_squares`` as
defined in cell 4 of the reference's notebooks/Crack_simulation.ipynb.

The cell's source is read from the notebook JSON and executed unchanged in a
namespace holding numpy (``np``) and ``scipy.stats`` (``stats``), the names
the cell's definitions use; only signal_retrieval_least_squares is called.
Inputs are seeded phase-stepping curves (sinusoid plus offset and noise,
several step counts and fringe periods) in the [steps][pixels] layout of a
detector output, retrieved with axis=0 as the notebook does. The outputs are
committed so the tests can pin the oracle restatement and the device
implementation without the reference present.

Usage:  python tests/golden/make_retrieval_golden.py [/path/to/reference]
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import scipy.stats as stats

HERE = Path(__file__).resolve().parent

# (step count, fringe period in steps, pixels, noise)
CASES = [(8, 8.0, 96, 0.05), (5, 5.0, 64, 0.02), (7, 9.5, 80, 0.1), (4, 4.0, 48, 0.0), (16, 16.0, 40, 0.3)]


def notebook_function(ref: Path):
    nb = json.loads((ref / "notebooks" / "Crack_simulation.ipynb").read_text())
    src = "".join(nb["cells"][4]["source"])
    ns = {"np": np, "stats": stats}
    exec(compile(src, "Crack_simulation.ipynb:cell4", "exec"), ns)
    return ns["signal_retrieval_least_squares"]


def main(ref: Path) -> None:
    retrieve = notebook_function(ref)
    out = {}
    for i, (k, period, n_pix, noise) in enumerate(CASES):
        rng = np.random.default_rng(100 + i)
        a, b = rng.normal(size=(2, n_pix))
        c = rng.uniform(2.0, 5.0, n_pix)
        phi = np.linspace(0, 2 * np.pi * k / period, k, endpoint=False)
        data = (a[None, :] * np.sin(phi)[:, None] + b[None, :] * np.cos(phi)[:, None] + c[None, :]
                + noise * rng.normal(size=(k, n_pix)))
        dabs, dphase, dvis, chi2 = retrieve(data, period=period, axis=0)
        out[f"data_{i}"] = data
        out[f"period_{i}"] = np.float64(period)
        out[f"dabs_{i}"] = dabs
        out[f"dphase_{i}"] = dphase
        out[f"dvis_{i}"] = dvis
        out[f"chi2_{i}"] = np.float64(chi2)
    out["n_cases"] = np.int64(len(CASES))
    np.savez_compressed(HERE / "retrieval.npz", **out)
    print("wrote", HERE / "retrieval.npz")


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference"))
