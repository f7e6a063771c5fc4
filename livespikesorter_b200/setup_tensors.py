"""One-time setup of the tensors the sorter consumes (host side, run once per
template set / probe).

These are the Kilosort4 4.0.13 setup steps whose outputs LiveSpikeSorter loads
from its input directory (writers: ``src/Python/run_online_spikes.py:483-578``):

* ``prepare_matching`` -> ``ctc``          (``kilosort/template_matching.py:110-121``)
* ``prepare_extract``  -> ``iCC, iU, Ucc``  (``kilosort/template_matching.py:20-26``)
* ``get_highpass_filter`` -> ``hp_filter`` (``kilosort/preprocessing.py:121-136``)
* ``whitening_local``  -> ``Wrot``          (``kilosort/preprocessing.py:8-35``)
* ``inv_kernel`` / ``get_drift_matrix``    (``kilosort/datashift.py:213-219``,
  ``kilosort/preprocessing.py:44-69``, nblocks == 1)
* ``template_waveforms`` -> ``preclustered_template_waveforms``
  (``src/Python/run_online_spikes.py:539``)

They run in torch on the CPU with the same operations as Kilosort so that the
tensors match what Kilosort would export; the per-batch hot path never calls
them.
"""
from __future__ import annotations

import numpy as np
import torch
from torch.nn.functional import conv1d


def prepare_matching(wPCA: torch.Tensor, U: torch.Tensor) -> torch.Tensor:
    """Template cross-correlations ``ctc[i, j, l]``, ``[T, T, 2*nt+1]`` float32."""
    nt = wPCA.shape[1]
    W = wPCA.contiguous()
    WtW = torch.flip(conv1d(W.reshape(-1, 1, nt), W.reshape(-1, 1, nt), padding=nt), [2])
    UtU = torch.einsum('ikl, jml -> ijkm', U, U)
    return torch.einsum('ijkm, kml -> ijl', UtU, WtW)


def prepare_extract(xc: np.ndarray, yc: np.ndarray, U: torch.Tensor, nC: int):
    """Nearest-channel tables: ``iCC [nC, C]``, ``iU [T]``, ``Ucc [nC, T, K]``."""
    ds = (xc - xc[:, np.newaxis]) ** 2 + (yc - yc[:, np.newaxis]) ** 2
    iCC = torch.from_numpy(np.argsort(ds, 0)[:nC])
    iU = torch.argmax((U ** 2).sum(1), -1)
    Ucc = U[torch.arange(U.shape[0]), :, iCC[:, iU]]
    return iCC, iU, Ucc


def get_highpass_filter(fs: float = 30000, cutoff: float = 300) -> torch.Tensor:
    """Zero-phase impulse response (30122 taps) of a 3rd-order Butterworth highpass."""
    from scipy.signal import butter, filtfilt
    n = 30122
    b, a = butter(3, cutoff, fs=fs, btype='high')
    x = np.zeros(n)
    x[n // 2] = 1
    return torch.from_numpy(filtfilt(b, a, x).copy()).float()


def whitening_local(CC: torch.Tensor, xc, yc, nrange: int = 32) -> torch.Tensor:
    """Local ZCA whitening: each channel whitened against its ``nrange`` nearest."""
    n = CC.shape[0]
    Wrot = torch.zeros((n, n), dtype=CC.dtype)
    for j in range(n):
        ds = (xc[j] - xc) ** 2 + (yc[j] - yc) ** 2
        ix = np.argsort(ds)[:nrange]
        E, D, _ = torch.linalg.svd(CC[np.ix_(ix, ix)])
        wrot = (E / (D + 1e-6) ** .5) @ E.T
        Wrot[j, ix] = wrot[0]
    return Wrot


def inv_kernel(xc, yc, sig_interp: float = 20) -> torch.Tensor:
    """Inverse of the regularised radial kernel between channel sites (``iKxx``)."""
    xp = np.vstack((xc, yc)).T
    ds = ((xp[:, np.newaxis] - xp) ** 2).sum(-1)
    Kxx = torch.from_numpy(np.exp(-ds / (2 * sig_interp ** 2)))
    return torch.linalg.inv(Kxx + 0.01 * torch.eye(Kxx.shape[0], dtype=Kxx.dtype))


def get_drift_matrix(xc, yc, dshift: float, iKxx: torch.Tensor, sig_interp: float = 20) -> torch.Tensor:
    """Drift interpolation matrix ``M [C, C]`` for a vertical shift ``dshift`` (microns)."""
    xp = np.vstack((xc, yc)).T
    yp = xp.copy()
    yp[:, 1] -= dshift
    xp_t = torch.from_numpy(xp)
    yp_t = torch.from_numpy(yp)
    ds = ((yp_t.unsqueeze(1) - xp_t) ** 2).sum(-1)
    Kyx = torch.exp(-ds / (2 * sig_interp ** 2))
    return Kyx @ iKxx.to(Kyx.dtype)


def template_waveforms(U: torch.Tensor, wPCA: torch.Tensor) -> torch.Tensor:
    """Full waveforms ``[T, nt, C]`` of the templates (``einsum('ijk,jl->kil')`` permuted)."""
    return torch.einsum('ijk,jl->kil', U, wPCA).permute(1, 2, 0).contiguous()
