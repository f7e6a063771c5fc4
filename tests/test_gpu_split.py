"""Short batches split the score GEMM's templates over CTAs (one work item
per sample tile and 128 templates) and combine the fused column maxima with
64-bit atomic keys. The rounds started from those maxima must equal the rounds
that recompute the maxima from the same score field (bit-identical spikes and
amplitudes), for short (split) and long (unsplit) batches and a template count
that leaves a ragged last pass.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('NT', [700, 12000])
def test_fused_maxima_equal_recomputed_maxima(NT):
    import ks4_oracle as ko
    from livespikesorter_b200.sorter import Sorter
    g = np.random.default_rng(4)
    T, K, C, nt = 300, 3, 48, 31
    U = g.standard_normal((T, K, C)).astype(np.float32)
    wPCA = np.linalg.qr(g.standard_normal((nt, K)))[0].T.astype(np.float32)
    wav = np.einsum('tkc,km->tcm', U, wPCA)
    X = 0.3 * g.standard_normal((C, NT + 2 * nt)).astype(np.float32)
    for s0 in range(50, NT, 53):
        X[:, s0 - nt // 2:s0 + nt // 2 + 1] += 2.0 * wav[g.integers(0, T)]
    ctc = ko.prepare_matching(torch.from_numpy(wPCA), torch.from_numpy(U), nt).numpy()
    s = Sorter(U=U, wPCA=wPCA, ctc=ctc, Wrot=np.eye(C, dtype=np.float32), NT=NT, Th=6.0)
    Xd = torch.from_numpy(X).cuda()
    st1, a1, _ = s.match(Xd, return_xres=False)
    B = s.scores(Xd)
    st2, a2 = s.match_scores(B)
    assert len(st1) > 10
    assert torch.equal(st1, st2) and torch.equal(a1, a2)
