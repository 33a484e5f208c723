"""Test oracle (CPU, numpy): phase-stepping signal retrieval.

Restates ``signal_retrieval_least_squares`` of the reference's crack-simulation
notebook (notebooks/Crack_simulation.ipynb, cell 4): the least-squares fit of
I_k = a sin(phi_k) + b cos(phi_k) + c over the phase steps with
phi = np.linspace(0, 2 pi nsteps / period, nsteps, endpoint=False), solved by
np.linalg.lstsq on the design matrix [sin, cos, 1]; returns
(nsteps * c, -atan2(a, b), sqrt(a^2 + b^2) / c, nanmean of the residuals).

Test infrastructure only: used by the tests as the checker of the device
implementation, never by the library.
"""

from __future__ import annotations

import numpy as np


def signal_retrieval_least_squares(data, period=None, axis=-1):
    data = np.asarray(data, dtype=np.float64)
    if axis != -1:
        data = np.moveaxis(data, axis, -1)
    nsteps = data.shape[-1]
    if period is None:
        period = nsteps
    phi = np.linspace(0, 2 * np.pi * nsteps / period, nsteps, endpoint=False)
    m = np.c_[np.sin(phi), np.cos(phi), np.ones(nsteps)]
    res, chi2, _rank, _sv = np.linalg.lstsq(m, data.reshape((-1, nsteps)).T, rcond=-1)
    res = res.T.reshape((*data.shape[:-1], -1))
    dabs = res[..., 2]
    dphase = -np.arctan2(res[..., 0], res[..., 1])
    dvis = np.sqrt(res[..., 0] ** 2 + res[..., 1] ** 2) / dabs
    dabs = dabs * nsteps
    return dabs, dphase, dvis, np.nanmean(chi2), chi2
