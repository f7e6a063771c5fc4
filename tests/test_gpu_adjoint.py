"""Hand-written adjoint of the reconstruction (csrc/adjoint.cu) behind
``adjoint.Reconstruction``.

* FP64, 8 channels x 4 templates: the forward equals Kilosort's own
  reconstruction ops (einsum + scatter, template_matching.py:195-198) to
  rounding, and the gradients equal torch autograd through those ops.
* FP64 central finite differences of the residual energy along random
  directions in U, wPCA and the amplitudes match the adjoint.
* FP32 at 384 channels / 400 templates agrees with the FP64 kernels.
* Refinement with fixed assignments moves perturbed templates back toward the
  templates that generated the data.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _case(C=8, T=4, K=3, nt=21, N=400, n=30, seed=0, dtype=torch.float64):
    g = torch.Generator().manual_seed(seed)
    U = torch.randn(T, K, C, generator=g, dtype=dtype)
    W = torch.randn(K, nt, generator=g, dtype=dtype)
    h = nt // 2
    x = torch.randint(h, N - h, (n,), generator=g, dtype=torch.int32)
    y = torch.randint(0, T, (n,), generator=g, dtype=torch.int32)
    a = torch.rand(n, generator=g, dtype=dtype) + 0.5
    X = torch.randn(C, N, generator=g, dtype=dtype)
    return [t.cuda() for t in (U, W, x, y, a, X)] + [N]


def test_forward_and_gradients_equal_torch_autograd_fp64():
    from livespikesorter_b200.adjoint import Reconstruction, reference_reconstruction
    U, W, x, y, a, X, N = _case()
    R = Reconstruction.apply(U, W, a, x, y, N)
    R_ref = reference_reconstruction(U, W, x, y, a, N)
    assert torch.allclose(R, R_ref, rtol=1e-13, atol=1e-12)

    def grads(fn):
        Uq, Wq, aq = (t.detach().clone().requires_grad_(True) for t in (U, W, a))
        loss = 0.5 * (X - fn(Uq, Wq, aq)).square().sum()
        loss.backward()
        return Uq.grad, Wq.grad, aq.grad

    g1 = grads(lambda Uq, Wq, aq: Reconstruction.apply(Uq, Wq, aq, x, y, N))
    g2 = grads(lambda Uq, Wq, aq: reference_reconstruction(Uq, Wq, x, y, aq, N))
    for p, q in zip(g1, g2):
        assert torch.allclose(p, q, rtol=1e-11, atol=1e-10), (p - q).abs().max()


def test_adjoint_matches_finite_differences_fp64():
    from livespikesorter_b200.adjoint import residual_energy
    U, W, x, y, a, X, N = _case(seed=3)
    Uq, Wq, aq = (t.detach().clone().requires_grad_(True) for t in (U, W, a))
    residual_energy(X, Uq, Wq, x, y, aq).backward()
    g = torch.Generator().manual_seed(9)
    for _ in range(4):
        dU = torch.randn(U.shape, generator=g, dtype=torch.float64).cuda()
        dW = torch.randn(W.shape, generator=g, dtype=torch.float64).cuda()
        da = torch.randn(a.shape, generator=g, dtype=torch.float64).cuda()
        eps = 1e-6
        with torch.no_grad():
            lp = residual_energy(X, U + eps * dU, W + eps * dW, x, y, a + eps * da)
            lm = residual_energy(X, U - eps * dU, W - eps * dW, x, y, a - eps * da)
        fd = float((lp - lm) / (2 * eps))
        an = float((Uq.grad * dU).sum() + (Wq.grad * dW).sum() + (aq.grad * da).sum())
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)


def test_fp32_agrees_with_fp64_at_full_size():
    from livespikesorter_b200.adjoint import residual_energy
    U, W, x, y, a, X, N = _case(C=384, T=400, K=6, nt=61, N=6000, n=1500, seed=5)
    grads = {}
    for dt in (torch.float64, torch.float32):
        Uq, Wq, aq = (t.detach().to(dt).clone().requires_grad_(True) for t in (U, W, a))
        residual_energy(X.to(dt), Uq, Wq, x, y, aq).backward()
        grads[dt] = (Uq.grad.double(), Wq.grad.double(), aq.grad.double())
    for p, q in zip(grads[torch.float32], grads[torch.float64]):
        assert (p - q).norm() <= 1e-4 * q.norm()


def test_refinement_recovers_templates():
    from livespikesorter_b200.adjoint import reference_reconstruction, refine
    g = torch.Generator().manual_seed(11)
    C, T, K, nt, N = 16, 6, 3, 31, 3000
    U_true = torch.randn(T, K, C, generator=g, dtype=torch.float64)
    W = torch.linalg.qr(torch.randn(nt, K, generator=g, dtype=torch.float64))[0].T.contiguous()
    batches = []
    noise_energy = 0.0
    for b in range(4):
        n = 120
        x = torch.randint(nt, N - nt, (n,), generator=g, dtype=torch.int32)
        y = torch.randint(0, T, (n,), generator=g, dtype=torch.int32)
        a = torch.rand(n, generator=g, dtype=torch.float64) + 0.5
        noise = 0.01 * torch.randn(C, N, generator=g, dtype=torch.float64)
        noise_energy += 0.5 * float(noise.square().sum())
        X = reference_reconstruction(U_true, W, x, y, a, N) + noise
        batches.append(tuple(t.float().cuda() if t.is_floating_point() else t.cuda() for t in (X, x, y, a)))
    scale = 1.0 + 0.1 * (2 * torch.rand(T, 1, 1, generator=g, dtype=torch.float64) - 1)
    U0 = (U_true * scale + 0.05 * torch.randn(T, K, C, generator=g, dtype=torch.float64)).float().cuda()
    e0 = float((U0.double().cpu() - U_true).norm() / U_true.norm())
    U1, _, losses = refine(batches, U0, W.float().cuda(), steps=150, lr=2e-2, method='adam')
    U2, _, losses2 = refine(batches, U0, W.float().cuda(), steps=8, lr=0.8, method='jacobi')
    e2 = float((U2.double().cpu() - U_true).norm() / U_true.norm())
    assert e2 < 0.2 * e0 and losses2[-1] < 1.05 * noise_energy, (e0, e2, losses2[-1], noise_energy)
    e1 = float((U1.double().cpu() - U_true).norm() / U_true.norm())
    # the residual energy falls to the noise floor and the templates move
    # most of the way back to the generating ones
    assert losses[-1] < 1.05 * noise_energy < 0.2 * losses[0], (losses[0], losses[-1], noise_energy)
    assert e1 < 0.2 * e0, (e0, e1)
