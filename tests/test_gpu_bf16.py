"""The BF16 tensor-core score path (tcgen05 GEMM, FP32 accumulation in tensor
memory) through the C ABI.

With small-integer inputs every bf16 product and every FP32 partial sum is
exact, so the tensor-core scores must equal the FP32 path bit for bit; the
shapes exercise several sample tiles, double-buffered accumulators (T <= 256),
two TMA boxes per stage (T = 300) and two template passes (T = 600). On real
data the BF16 scores are compared with the FP32 scores against the bf16
rounding bound.
"""
import numpy as np
import pytest
import torch

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _int_case(T, C=64, K=3, nt=5, NT=1000, seed=0):
    g = np.random.default_rng(seed)
    U = g.integers(-3, 4, (T, K, C)).astype(np.float32)
    U[:, 0, 0] += 1 + (np.abs(U).sum((1, 2)) == 0)  # no zero-energy template
    wPCA = g.integers(-1, 2, (K, nt)).astype(np.float32)
    X = g.integers(-2, 3, (C, NT + 2 * nt)).astype(np.float32)
    return U, wPCA, X, NT


@pytest.mark.parametrize('T', [40, 300, 600])
def test_bf16_scores_exact_on_integer_data(T):
    from livespikesorter_b200.sorter import Sorter
    U, wPCA, X, NT = _int_case(T)
    kw = dict(U=U, wPCA=wPCA, ctc=np.zeros((T, T, 2 * wPCA.shape[1] + 1), np.float32),
              Wrot=np.eye(U.shape[2], dtype=np.float32), NT=NT, Th=4.0)
    s32 = Sorter(**kw)
    s16 = Sorter(precision='bf16', **kw)
    Xd = torch.from_numpy(X).cuda()
    B32 = s32.scores(Xd)
    B16 = s16.scores(Xd)
    assert torch.equal(B32, B16)
    ref = torch.einsum('ijk,kjl->il', torch.from_numpy(U).double(),
                       torch.nn.functional.conv1d(torch.from_numpy(X).double().unsqueeze(1),
                                                  torch.from_numpy(wPCA).double().unsqueeze(1),
                                                  padding=wPCA.shape[1] // 2))
    assert torch.equal(B16.cpu().double(), ref)


def test_bf16_known_answer_case():
    from livespikesorter_b200.sorter import Sorter
    g = np.load(GOLDEN / 'conv1d_known_answer.npz')
    M = int(g['M'])
    s = Sorter(U=g['Wall3'].astype(np.float32), wPCA=g['wPCA'].astype(np.float32),
               ctc=np.zeros((2, 2, 2 * M + 1), np.float32), Wrot=np.eye(2, dtype=np.float32),
               NT=g['batch'].shape[1] - 2 * M, Th=1.0, precision='bf16')
    B = s.scores(torch.from_numpy(g['batch'].astype(np.float32)).cuda()).cpu().double()
    # the batch holds values (e.g. 321 * 9) that bf16 cannot represent: compare
    # against the bf16 rounding bound 2^-7 * sum |U| |B0|
    ref = torch.from_numpy(g['C']).double()
    U = torch.from_numpy(g['Wall3']).double()
    B0 = torch.from_numpy(g['B']).double()
    bound = 2.0 ** -7 * torch.einsum('ijk,kjl->il', U.abs(), B0.abs())
    assert torch.all((B - ref).abs() <= bound)


def test_bf16_rounds_equal_fp32_rounds_on_exact_scores():
    """Integer scores are exact in both paths, so the fused column maxima of the
    GEMM epilogue must lead the rounds to the identical spikes."""
    import ks4_oracle as ko
    from livespikesorter_b200.sorter import Sorter
    T = 24
    U, wPCA, X, NT = _int_case(T, nt=5, NT=2000, seed=3)
    # plant spikes: exact template waveforms at known times
    wav = torch.einsum('tkc,km->tcm', torch.from_numpy(U), torch.from_numpy(wPCA)).numpy()
    g = np.random.default_rng(1)
    for s0 in range(40, NT, 97):
        X[:, s0 - 2:s0 + 3] += 3 * wav[g.integers(0, T)]
    ctc = ko.prepare_matching(torch.from_numpy(wPCA), torch.from_numpy(U), 5).numpy()
    kw = dict(U=U, wPCA=wPCA, ctc=ctc, Wrot=np.eye(U.shape[2], dtype=np.float32), NT=NT, Th=20.0)
    st32, a32, _ = Sorter(**kw).match(torch.from_numpy(X).cuda())
    st16, a16, _ = Sorter(precision='bf16', **kw).match(torch.from_numpy(X).cuda())
    assert len(st32) > 10
    assert torch.equal(st32, st16) and torch.equal(a32, a16)


def test_bf16_scores_within_rounding_bound_on_real_data():
    from livespikesorter_b200.sorter import Sorter
    g = np.load(GOLDEN / 'ks4_extract_c32_t12.npz')
    C, T, NT, nt = [int(v) for v in g['params'][:4]]
    kw = dict(U=g['U'], wPCA=g['wPCA'], ctc=g['ctc'], Wrot=g['Wrot'], NT=NT, Th=float(g['Th']))
    X = torch.from_numpy(g['X_1']).cuda()
    B32 = Sorter(**kw).scores(X).double()
    B16 = Sorter(precision='bf16', **kw).scores(X).double()
    # |dB| <= 2^-8 * ||U_t|| * ||B0[:, s]||  (both operands rounded to bf16)
    U = torch.from_numpy(g['U']).double()
    B0 = torch.nn.functional.conv1d(X.cpu().double().unsqueeze(1), torch.from_numpy(g['wPCA']).double().unsqueeze(1),
                                    padding=nt // 2)
    bound = 2.0 ** -7 * U.reshape(T, -1).norm(dim=1)[:, None] * B0.permute(1, 0, 2).reshape(-1, B0.shape[-1]).norm(dim=0)[None]
    err = (B16 - B32).abs().cpu()
    assert torch.all(err <= bound + 1e-6)
    assert err.max() > 0  # the path really rounds to bf16
