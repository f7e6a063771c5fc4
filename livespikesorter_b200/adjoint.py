"""Differentiable reconstruction for template refinement.

``Reconstruction`` is a ``torch.autograd.Function`` over the hand-written
kernels of ``csrc/adjoint.cu`` (``lss_recon_forward`` / ``lss_recon_backward``):

    R[c, s] = sum_i amp_i sum_k U[y_i, k, c] wPCA[k, s - x_i + nt/2]

which is the waveform Kilosort subtracts for each accepted spike
(template_matching.py:195-198). With the assignments (x, y, amp) held fixed,
``refine`` adjusts U (and optionally the temporal basis) by gradient on the
residual energy 0.5 * ||X - R||^2 summed over recent batches. The backward
pass recomputes the temporal-basis convolution of the incoming gradient per
spike; nothing from the forward pass is stored. Both directions run in the
tensors' dtype (float32, or float64 for the finite-difference checks).
"""
from __future__ import annotations

import torch

from . import _lib
from ._lib import check

_DT = {torch.float32: 0, torch.float64: 1}


def _stream(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


class Reconstruction(torch.autograd.Function):
    """``R = Reconstruction.apply(U, wPCA, amp, x, y, N)``; gradients for U,
    wPCA and amp."""

    @staticmethod
    def forward(ctx, U, wPCA, amp, x, y, N: int):
        lib = _lib.load()
        if U.dtype not in _DT or wPCA.dtype != U.dtype or amp.dtype != U.dtype:
            raise TypeError('U, wPCA and amp must share float32 or float64')
        if not (U.is_cuda and wPCA.is_cuda and amp.is_cuda and x.is_cuda and y.is_cuda):
            raise ValueError('all tensors must be on the GPU (there is no CPU path)')
        U, wPCA, amp = U.contiguous(), wPCA.contiguous(), amp.contiguous().view(-1)
        x, y = x.to(torch.int32).contiguous().view(-1), y.to(torch.int32).contiguous().view(-1)
        T, K, C = U.shape
        nt = wPCA.shape[1]
        ox = torch.argsort(x, stable=True)
        xs, ys, as_ = x[ox].contiguous(), y[ox].contiguous(), amp[ox].contiguous()
        R = torch.empty((C, N), device=U.device, dtype=U.dtype)
        check(lib.lss_recon_forward(_DT[U.dtype], U.data_ptr(), wPCA.data_ptr(), T, K, C, nt, xs.data_ptr(),
                                    ys.data_ptr(), as_.data_ptr(), x.numel(), R.data_ptr(), N, _stream(U)))
        ctx.save_for_backward(U, wPCA, amp, x, y)
        ctx.N = N
        return R

    @staticmethod
    def backward(ctx, dR):
        lib = _lib.load()
        U, wPCA, amp, x, y = ctx.saved_tensors
        T, K, C = U.shape
        nt = wPCA.shape[1]
        dR = dR.to(U.dtype).contiguous()
        order = torch.argsort(y, stable=True).to(torch.int32)
        counts = torch.bincount(y.long(), minlength=T)
        start = torch.zeros(T + 1, device=U.device, dtype=torch.int64)
        start[1:] = torch.cumsum(counts, 0)
        start = start.to(torch.int32)
        dU = torch.empty_like(U)
        dW = torch.empty_like(wPCA)
        damp = torch.empty_like(amp) if ctx.needs_input_grad[2] else None
        work = torch.empty((T, K, nt), device=U.device, dtype=U.dtype)
        check(lib.lss_recon_backward(_DT[U.dtype], U.data_ptr(), wPCA.data_ptr(), T, K, C, nt, x.data_ptr(),
                                     amp.data_ptr(), order.data_ptr(), start.data_ptr(), dR.data_ptr(), ctx.N,
                                     dU.data_ptr(), dW.data_ptr(), None if damp is None else damp.data_ptr(),
                                     work.data_ptr(), _stream(U)))
        return dU, dW, damp, None, None, None


def reconstruct(U, wPCA, x, y, amp, N: int) -> torch.Tensor:
    return Reconstruction.apply(U, wPCA, amp, x, y, N)


def residual_energy(X, U, wPCA, x, y, amp) -> torch.Tensor:
    """0.5 * ||X - R||^2 for one batch X [C, N]."""
    R = Reconstruction.apply(U, wPCA, amp, x, y, X.shape[1])
    return 0.5 * (X - R).square().sum()


def reference_reconstruction(U, wPCA, x, y, amp, N: int) -> torch.Tensor:
    """The same reconstruction written with Kilosort's own tensor ops
    (template_matching.py:195-198: einsum('ijk,jl->kil', U[iY], W) scattered
    at x + tiwave), differentiable by torch autograd; the check for the
    hand-written adjoint."""
    nt = wPCA.shape[1]
    tiwave = torch.arange(-(nt // 2), nt // 2 + 1, device=U.device)
    waves = torch.einsum('ijk,jl->kil', U[y.long()], wPCA)            # [C, n, nt]
    cols = (x.long()[:, None] + tiwave[None, :]).reshape(-1)             # [n * nt]
    vals = (amp.reshape(-1, 1, 1) * waves.permute(1, 0, 2)).permute(1, 0, 2).reshape(U.shape[2], -1)
    R = torch.zeros((U.shape[2], N), device=U.device, dtype=U.dtype)
    return R.index_add(1, cols, vals)


def refine(batches, U0, wPCA0, *, steps: int = 50, lr: float = 1e-2, refine_basis: bool = False,
           method: str = 'jacobi', callback=None):
    """Gradient refinement of the templates on the residual energy of
    ``batches`` (a list of ``(X [C, N], x, y, amp)`` with fixed assignments).

    method 'jacobi': U_t -= lr * dL/dU_t / sum_{i: y_i = t} amp_i^2, the
    Gauss-Newton step for non-overlapping spikes when the temporal basis has
    orthonormal rows (Kilosort's does: right singular vectors), so lr ~ 1
    converges in a few steps and channels without signal are not pushed by
    noise; the basis, when refined, takes plain gradient steps of lr * 1e-3
    scaled the same way. method 'adam': torch.optim.Adam on the same loss.
    Returns ``(U, wPCA, losses)``."""
    U = U0.detach().clone().requires_grad_(True)
    W = wPCA0.detach().clone().requires_grad_(refine_basis)
    if method == 'adam':
        opt = torch.optim.Adam([U, W] if refine_basis else [U], lr=lr)
    elif method == 'jacobi':
        T = U.shape[0]
        H = torch.zeros(T, device=U.device, dtype=U.dtype)
        for _, _, y, a in batches:
            H.index_add_(0, y.long(), a.to(U.dtype).square())
        Hinv = torch.where(H > 0, 1.0 / H.clamp_min(1e-30), torch.zeros_like(H))[:, None, None]
        Htot = float(H.sum()) if float(H.sum()) > 0 else 1.0
    else:
        raise ValueError(f'unknown method {method!r}')
    losses = []
    for it in range(steps):
        U.grad = None
        W.grad = None
        loss = sum(residual_energy(X, U, W, x, y, a) for X, x, y, a in batches)
        loss.backward()
        if method == 'adam':
            opt.step()
        else:
            with torch.no_grad():
                U -= lr * U.grad * Hinv
                if refine_basis:
                    W -= 1e-3 * lr * W.grad / Htot
        losses.append(float(loss.detach()))
        if callback is not None:
            callback(it, U, W, losses[-1])
    return U.detach(), W.detach(), losses
