"""Phase-stepping signal retrieval on the GPU.

``signal_retrieval_least_squares`` has the signature and results of the
function of the same name in the reference's crack-simulation notebook
(notebooks/Crack_simulation.ipynb, cell 4): per pixel, the least-squares fit
of the phase-stepping curve I_k = a sin(phi_k) + b cos(phi_k) + c with
phi = np.linspace(0, 2 pi nsteps / period, nsteps, endpoint=False), returned as
(transmission nsteps * c, phase -atan2(a, b), visibility sqrt(a^2 + b^2) / c,
mean squared residual). The fit runs in the engine (rsw_signal_retrieval) on
FP64 data; numpy input is copied to the device and results back, CUDA
tensors stay on the device.

``dark_field`` combines a sample and a reference (flat) scan into the usual
transmission, differential phase and dark-field (visibility ratio) maps.
"""

from __future__ import annotations

import numpy as np

from . import _lib as L
from .engine import _stream_ptr, _torch


def _retrieve(data2d, period):
    """data2d: CUDA float64 tensor [nsteps, n_pix] (contiguous)."""
    torch = _torch()
    nsteps, n_pix = data2d.shape
    out = torch.empty((4, n_pix), dtype=torch.float64, device=data2d.device)
    lib = L.load()
    ptr = [int(out[i].data_ptr()) for i in range(4)]
    L.check(lib.rsw_signal_retrieval(int(data2d.data_ptr()), n_pix, nsteps, float(period), *ptr, _stream_ptr()))
    return out


def signal_retrieval_least_squares(data, period=None, axis=-1):
    """Drop-in for the notebook function: ``data`` with the phase steps on
    ``axis``; returns (dabs, dphase, dvis, mean chi2). numpy in -> numpy out,
    CUDA tensor in -> CUDA tensors out (mean chi2 as a float)."""
    torch = _torch()
    on_device = hasattr(data, "is_cuda") and data.is_cuda
    t = data if on_device else torch.from_numpy(np.ascontiguousarray(np.asarray(data, dtype=np.float64)))
    t = t.to(dtype=torch.float64)
    t = torch.movedim(t, axis, 0)
    nsteps = t.shape[0]
    lead = t.shape[1:]
    t2 = t.reshape(nsteps, -1).contiguous()
    if not on_device:
        t2 = t2.cuda()
    if period is None:
        period = nsteps
    out = _retrieve(t2, period)
    dabs, dphase, dvis, chi2 = (out[i].reshape(lead) for i in range(4))
    mchi2 = float(torch.nanmean(chi2)) if nsteps > 3 else float("nan")
    if on_device:
        return dabs, dphase, dvis, mchi2
    return dabs.cpu().numpy(), dphase.cpu().numpy(), dvis.cpu().numpy(), mchi2


def dark_field(sample, reference, period=None, axis=0):
    """Transmission, differential phase (wrapped to (-pi, pi]) and dark field
    (visibility ratio) of a sample scan against a reference scan, both with
    the phase steps on ``axis`` (detector arrays: axis 0)."""
    ts, ps, vs, _ = signal_retrieval_least_squares(sample, period, axis)
    tr, pr, vr, _ = signal_retrieval_least_squares(reference, period, axis)
    dphi = np.angle(np.exp(1j * (np.asarray(ps) - np.asarray(pr)))) if not hasattr(ps, "is_cuda") else None
    if dphi is None:
        torch = _torch()
        d = ps - pr
        dphi = torch.atan2(torch.sin(d), torch.cos(d))
    return ts / tr, dphi, vs / vr
