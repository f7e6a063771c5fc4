"""CPU oracle for the per-batch spike-sorting hot path (TEST INFRASTRUCTURE ONLY).

This module restates, in torch on the CPU, the Kilosort4 4.0.13 functions that
LiveSpikeSorter's sorter mirrors, as vendored in the reference under
``src/Python/run_online_spikes/Lib/site-packages/kilosort/``:

* ``padded_batch``       <- ``io.py:584-637``        (BinaryRWFile.padded_batch_to_torch)
* ``filter_batch``       <- ``io.py:757-790``        (BinaryFiltered.filter)
* ``fft_highpass``       <- ``preprocessing.py:138-154``
* ``get_highpass_filter``, ``whitening_local``, ``get_drift_matrix`` / ``inv_kernel``,
  ``prepare_matching``, ``prepare_extract`` <- ``preprocessing.py:8-35,44-69,121-136``,
  ``datashift.py:215-219``, ``template_matching.py:20-26,110-121``: these one-time
  setup steps are the product's own host code (``livespikesorter_b200/setup_tensors.py``),
  re-exported here and pinned against the reference like the rest
* ``run_matching``       <- ``template_matching.py:128-202``
* ``extract_batch``      <- ``template_matching.py:46-73`` (xfeat and time conversion)
* ``spike_positions``    <- ``postprocessing.py:33-46``  (compute_spike_positions)
* ``remove_duplicates``  <- ``postprocessing.py:10-31``
* ``closest_cluster``    <- LiveSpikeSorter ``OnlineSpikesV2.cu:1028-1043`` (closestCluster)
* ``postprocess``        <- the order of ``io.py:233-246`` (positions, then
                            duplicates per cluster on time-sorted spikes) with
                            ``saveSpikes``' cluster relabelling (``OnlineSpikesV2.cu:1131-1164``)

It is the checker, never the thing measured or shipped: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import it.
The product path never routes through this file.

Parity pin: ``tests/test_oracle_pin.py`` imports the vendored reference itself
(when the reference tree is present) and checks that every function here returns
bit-identical tensors on seeded inputs; ``tests/golden/`` holds fixtures that the
reference produced (``tests/golden/make_golden.py``), including the reference's
own known-answer case ``src/Python/conv1d_test.py:14-43``, so the pin also holds
where the reference tree is absent.

``dtype=torch.float64`` turns ``run_matching`` into the FP64 score oracle (the
reference hard-codes float32 amplitudes at ``template_matching.py:151``; the
FP64 mode keeps every intermediate in float64).
"""
from __future__ import annotations

import numpy as np
import torch
from torch.nn.functional import conv1d, max_pool1d
from torch.fft import fft, ifft, fftshift

from livespikesorter_b200 import setup_tensors as _setup
from livespikesorter_b200.setup_tensors import (get_drift_matrix, get_highpass_filter,  # noqa: F401
                                                inv_kernel, prepare_extract, whitening_local)


# --------------------------------------------------------------------------
# ingest: io.py:584-637 and io.py:757-790
# --------------------------------------------------------------------------
def padded_batch(raw: np.ndarray, ibatch: int, NT: int, nt: int,
                 imin: int = 0, imax: int | None = None) -> torch.Tensor:
    """``BinaryRWFile.padded_batch_to_torch`` (io.py:584-637) on an int16 array.

    ``raw`` is the file's ``[n_samples, n_chan_bin]`` int16 matrix.  Returns
    float32 ``[n_chan_bin, NT + 2*nt]`` with the reference's edge handling:
    batch 0 replicates its first sample into the leading ``nt`` columns, the
    last batch replicates its last sample to the end, and a short single batch
    leaves zeros at the tail.
    """
    if imax is None:
        imax = raw.shape[0]
    n_samples = imax - imin
    n_batches = int(np.ceil(n_samples / NT))
    C = raw.shape[1]
    if ibatch == 0:
        bstart = imin
        bend = imin + NT + nt
    else:
        bstart = imin + ibatch * NT - nt
        bend = min(imax, bstart + NT + 2 * nt)
    data = raw[bstart:bend].T
    nsamp = data.shape[-1]
    X = torch.zeros((C, NT + 2 * nt), dtype=torch.float32)
    if ibatch == 0:
        X[:, nt:nt + nsamp] = torch.from_numpy(np.ascontiguousarray(data)).float()
        X[:, :nt] = X[:, nt:nt + 1]
    elif ibatch == n_batches - 1:
        X[:, :nsamp] = torch.from_numpy(np.ascontiguousarray(data)).float()
        X[:, nsamp:] = X[:, nsamp - 1:nsamp]
    else:
        X[:] = torch.from_numpy(np.ascontiguousarray(data)).float()
    return X


def fft_highpass(hp_filter: torch.Tensor, NT: int) -> torch.Tensor:
    """preprocessing.py:138-154: pad or crop the impulse response to NT, FFT it."""
    ft = hp_filter.shape[0]
    if ft < NT:
        pad = (NT - ft) // 2
        fhp = fft(torch.cat((torch.zeros(pad, dtype=hp_filter.dtype), hp_filter,
                             torch.zeros(pad + (NT - pad * 2 - ft), dtype=hp_filter.dtype))))
    elif ft > NT:
        crop = (ft - NT) // 2
        fhp = fft(hp_filter[crop:crop + NT])
    else:
        fhp = fft(hp_filter)
    return fhp


def filter_batch(X: torch.Tensor, chan_map=None, invert_sign=False, do_CAR=True,
                 hp_filter: torch.Tensor | None = None,
                 whiten_mat: torch.Tensor | None = None,
                 drift_M: torch.Tensor | None = None) -> torch.Tensor:
    """``BinaryFiltered.filter`` (io.py:757-790) without the artifact branch."""
    if chan_map is not None:
        X = X[torch.as_tensor(chan_map, dtype=torch.int64)]
    if invert_sign:
        X = X * -1
    X = X - X.mean(1).unsqueeze(1)
    if do_CAR:
        X = X - torch.median(X, 0)[0]
    if hp_filter is not None:
        fwav = fft_highpass(hp_filter, NT=X.shape[1])
        X = torch.real(ifft(fft(X) * torch.conj(fwav)))
        X = fftshift(X, dim=-1)
    if whiten_mat is not None:
        if drift_M is not None:
            X = (drift_M @ whiten_mat) @ X
        else:
            X = whiten_mat @ X
    return X


# --------------------------------------------------------------------------
# one-time setup: preprocessing.py, datashift.py, template_matching.py
#
# The product's host-side setup (livespikesorter_b200/setup_tensors.py) holds
# the one copy of these Kilosort steps; the oracle uses it, and
# tests/test_oracle_pin.py pins it bit for bit against the reference itself.
# --------------------------------------------------------------------------

def prepare_matching(wPCA: torch.Tensor, U: torch.Tensor, nt: int) -> torch.Tensor:
    """template_matching.py:110-121: ctc[i, j, l] template cross-correlations."""
    assert wPCA.shape[1] == nt
    return _setup.prepare_matching(wPCA, U)


# --------------------------------------------------------------------------
# matching pursuit: template_matching.py:128-202
# --------------------------------------------------------------------------
def run_matching(X: torch.Tensor, U: torch.Tensor, ctc: torch.Tensor, wPCA: torch.Tensor,
                 Th: float, nt: int, dtype=torch.float32, B: torch.Tensor | None = None,
                 nm: torch.Tensor | None = None, max_rounds: int = 100,
                 capacity: int = 100000, return_rounds=False, return_field=False):
    """``run_matching`` restated (template_matching.py:128-202).

    ``B`` optionally injects the score field (so the rounds can be checked in
    isolation from the score GEMM's rounding); ``nm`` likewise injects the
    template energies.  Returns ``(st int64 [n,2], amps [n,1], Xres [C,N])``,
    with ``return_rounds`` also the round index of every spike, and with
    ``return_field`` the score field left after the last round.
    """
    X = X.to(dtype)
    U = U.to(dtype)
    ctc = ctc.to(dtype)
    W = wPCA.to(dtype).contiguous()
    if nm is None:
        nm = (U ** 2).sum(-1).sum(-1)
    else:
        nm = nm.to(dtype)
    if B is None:
        B = conv1d(X.unsqueeze(1), W.unsqueeze(1), padding=nt // 2)
        B = torch.einsum('ijk, kjl -> il', U, B)
    else:
        B = B.to(dtype).clone()
    trange = torch.arange(-nt, nt + 1)
    tiwave = torch.arange(-(nt // 2), nt // 2 + 1)
    st = torch.zeros((capacity, 2), dtype=torch.int64)
    amps = torch.zeros((capacity, 1), dtype=dtype)
    rounds = torch.zeros(capacity, dtype=torch.int64)
    k = 0
    Xres = X.clone()
    for t in range(max_rounds):
        Cf = torch.relu(B) ** 2 / nm.unsqueeze(-1)
        Cf[:, :nt] = 0
        Cf[:, -nt:] = 0
        Cfmax, imax = torch.max(Cf, 0)
        Cmax = max_pool1d(Cfmax.unsqueeze(0).unsqueeze(0), (2 * nt + 1), stride=1, padding=(nt))
        cnd1 = Cmax[0, 0] > Th ** 2
        cnd2 = torch.abs(Cmax[0, 0] - Cfmax) < 1e-9
        xs = torch.nonzero(cnd1 * cnd2)
        if len(xs) == 0:
            break
        iX = xs[:, :1]
        iY = imax[iX]
        nsp = len(iX)
        st[k:k + nsp, 0] = iX[:, 0]
        st[k:k + nsp, 1] = iY[:, 0]
        amps[k:k + nsp] = B[iY, iX] / nm[iY]
        rounds[k:k + nsp] = t
        amp = amps[k:k + nsp]
        k += nsp
        n = 2
        for j in range(n):
            Xres[:, iX[j::n] + tiwave] -= amp[j::n] * torch.einsum('ijk, jl -> kil', U[iY[j::n, 0]], W)
            B[:, iX[j::n] + trange] -= amp[j::n] * ctc[:, iY[j::n, 0], :]
    out = (st[:k], amps[:k], Xres) + ((rounds[:k],) if return_rounds else ()) + ((B,) if return_field else ())
    return out


def score_field(X: torch.Tensor, U: torch.Tensor, wPCA: torch.Tensor, nt: int,
                dtype=torch.float32) -> torch.Tensor:
    """The score GEMM of template_matching.py:145-146: ``B[t, s]``."""
    W = wPCA.to(dtype)
    B0 = conv1d(X.to(dtype).unsqueeze(1), W.unsqueeze(1), padding=nt // 2)
    return torch.einsum('ijk, kjl -> il', U.to(dtype), B0)


def extract_batch(st: torch.Tensor, amps: torch.Tensor, Xres: torch.Tensor,
                  iCC: torch.Tensor, iU: torch.Tensor, Ucc: torch.Tensor,
                  wPCA: torch.Tensor, nt: int, nt0min: int, ibatch: int, NT: int):
    """template_matching.py:46-73 for one batch: PC features and time conversion.

    Returns ``(st3 float64 [n,3] (time, template, amplitude), tF [n, nC, K])``.
    """
    tiwave = torch.arange(-(nt // 2), nt // 2 + 1)
    xfeat = Xres[iCC[:, iU[st[:, 1:2]]], st[:, :1] + tiwave] @ wPCA.T.to(Xres.dtype)
    xfeat += amps * Ucc[:, st[:, 1]].to(Xres.dtype)
    if ibatch == 0:
        neg = (st[:, 0] - nt - nt // 2 + nt0min) < 0
        st = st[~neg, :]
        xfeat = xfeat[:, ~neg, :]
        amps = amps[~neg, :]
    stt = st.double()
    out = np.zeros((len(st), 3), 'float64')
    out[:, 0] = ((stt[:, 0] - nt) + ibatch * NT).numpy() - nt // 2 + nt0min
    out[:, 1] = stt[:, 1].numpy()
    out[:, 2] = amps[:, 0].double().numpy()
    return out, xfeat.transpose(0, 1).contiguous()


# --------------------------------------------------------------------------
# diagnostics
# --------------------------------------------------------------------------
def margin_report(B: torch.Tensor, nm: torch.Tensor, Th: float, nt: int) -> dict:
    """Round-1 decision margins of a score field (FP64): how close each column's
    best template is to the threshold, to the runner-up template, and to the
    largest other value in its pooling window.  Used to judge whether a spike
    that differs between two FP32 evaluations sat on a near-tie."""
    B = B.double()
    Cf = torch.relu(B) ** 2 / nm.double().unsqueeze(-1)
    Cf[:, :nt] = 0
    Cf[:, -nt:] = 0
    top2 = torch.topk(Cf, 2, dim=0).values
    best, second = top2[0], top2[1]
    return {'best': best, 'runner_up_gap': best - second, 'threshold_gap': best - Th ** 2}


def spike_positions(st: np.ndarray, tF: torch.Tensor, iCC: torch.Tensor, iU: torch.Tensor, xc, yc):
    """x, y of each spike from its PC-feature energy on the nearest channels
    (postprocessing.py:33-46)."""
    tmass = (tF ** 2).sum(-1)
    tmass = tmass / tmass.sum(1, keepdim=True)
    xc = torch.as_tensor(np.asarray(xc)).to(tmass.dtype)
    yc = torch.as_tensor(np.asarray(yc)).to(tmass.dtype)
    chs = iCC[:, iU[torch.as_tensor(st[:, 1]).long()]]
    xs = (xc[chs.T] * tmass).sum(1).numpy()
    ys = (yc[chs.T] * tmass).sum(1).numpy()
    return xs, ys


def remove_duplicates(spike_times: np.ndarray, spike_clusters: np.ndarray, dt: int, t0=None):
    """Same-cluster spikes within dt samples of the last kept one are dropped
    (postprocessing.py:10-31). ``t0`` optionally carries the last kept time
    per cluster in (and is updated): the reference processes the whole
    recording at once, a stream carries it from batch to batch."""
    keep = np.zeros(spike_times.size, bool)
    last = {} if t0 is None else t0
    for i in range(spike_times.size):
        t, c = int(spike_times[i]), int(spike_clusters[i])
        prev = last.get(c, t - dt)
        if t >= prev + dt:
            last[c] = t
            keep[i] = True
    return spike_times[keep], spike_clusters[keep], keep


def closest_cluster(xs: np.ndarray, ys: np.ndarray, centroids: np.ndarray) -> np.ndarray:
    """Nearest centroid (float32 distances, first index on ties), as
    OnlineSpikesV2::closestCluster (OnlineSpikesV2.cu:1028-1043)."""
    out = np.empty(len(xs), np.int64)
    cx = centroids[:, 0].astype(np.float32)
    cy = centroids[:, 1].astype(np.float32)
    for i in range(len(xs)):
        dx = np.float32(xs[i]) - cx
        dy = np.float32(ys[i]) - cy
        d = np.sqrt(dx * dx + dy * dy, dtype=np.float32)
        out[i] = int(np.argmin(d))
    return out


def postprocess(times: np.ndarray, templates: np.ndarray, tF: torch.Tensor, iCC, iU, xc, yc,
                centroids: np.ndarray | None, dt: int, t0=None):
    """One batch's records in matching order -> (order, x, y, cluster) of the
    kept spikes in time order (ties in matching order)."""
    st = np.stack([times, templates], 1)
    xs, ys = spike_positions(st, tF, iCC, iU, xc, yc)
    clu = closest_cluster(xs, ys, centroids) if centroids is not None and len(centroids) else templates.copy()
    order = np.argsort(times, kind='stable')
    _, _, keep = remove_duplicates(times[order], clu[order], dt, t0)
    o = order[keep]
    return o, xs[o], ys[o], clu[o]
