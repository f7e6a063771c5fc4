"""FP32 re-check of the BF16 score path.

The BF16 path splits both GEMM operands into bf16 parts (hi = bf16(x),
lo = bf16(x - hi)) and accumulates three bf16 MMAs in FP32; its scores are
within about 2^-11 ||U_t|| ||P_s|| of the FP32 path's (the tests check the
looser 2^-7). From that
bound the BF16 GEMM gives each column an interval for the FP32 path's best Cf
and an upper bound for every other template; columns whose first-round
decisions the intervals leave open (threshold, best template, or the max-pool
peak test against a column of the +-nt window) are projected with the FP32
path's arithmetic and re-scored by its 3xTF32 GEMM. So re-scored columns are
bit-identical to the FP32 path, the first round's peaks and templates are the
FP32 path's, and the sorted spikes agree with the FP32 path on all but a small
fraction (later rounds run on the BF16 field).
"""
import numpy as np
import pytest
import torch

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _fixture():
    g = np.load(GOLDEN / 'ks4_extract_c32_t12.npz')
    C, T, NT, nt, nt0min, nC, K, nb = [int(v) for v in g['params']]
    kw = dict(U=g['U'], wPCA=g['wPCA'], ctc=g['ctc'], Wrot=g['Wrot'], hp_filter=g['hp_filter'], iCC=g['iCC'],
              iU=g['iU'], Ucc=g['Ucc'], NT=NT, nt0min=nt0min, Th=float(g['Th']))
    return g, kw


def test_rechecked_columns_equal_fp32_scores():
    from livespikesorter_b200.sorter import Sorter
    g, kw = _fixture()
    X = torch.from_numpy(g['X_1']).cuda()
    s32 = Sorter(**kw)
    s16 = Sorter(precision='bf16', **kw)
    B32 = s32.scores(X)
    B16 = s16.scores(X)
    st = s16.stats()
    assert st['recheck_columns'] <= st['recheck_rescored']
    same = (B16 == B32).all(dim=0)
    # every re-scored column is bit-identical to the FP32 path (a column the
    # BF16 GEMM got exactly right by chance only adds to the count)
    assert int(same.sum()) >= st['recheck_rescored']
    # the first round's peaks (time, template) are the FP32 path's
    nt = int(g['params'][3])
    nm = (torch.from_numpy(g['U']) ** 2).sum(-1).sum(-1).cuda()
    assert _first_round(B16, nm, kw['Th'], nt) == _first_round(B32, nm, kw['Th'], nt)


def _first_round(B, nm, Th, nt):
    """Kilosort's first-round peak set (template_matching.py:159-181)."""
    Cf = torch.relu(B.float()) ** 2 / nm.float()[:, None]
    Cf[:, :nt] = 0
    Cf[:, -nt:] = 0
    Cfmax, imax = torch.max(Cf, 0)
    Cmax = torch.nn.functional.max_pool1d(Cfmax[None, None], 2 * nt + 1, stride=1, padding=nt)[0, 0]
    x = torch.nonzero((Cmax > Th ** 2) & ((Cmax - Cfmax).abs() < 1e-9))[:, 0]
    return list(zip(x.tolist(), imax[x].tolist()))


def test_bf16_recheck_sort_batch_agrees_with_fp32():
    from livespikesorter_b200.sorter import Sorter
    g, kw = _fixture()
    NT, nt, nb = kw['NT'], int(g['params'][3]), int(g['params'][7])
    s32 = Sorter(**kw)
    s16 = Sorter(precision='bf16', **kw)
    for ib in range(nb):
        rows = g['raw'][0:NT + nt] if ib == 0 else g['raw'][ib * NT - nt: ib * NT + NT + nt]
        r32 = s32.sort_batch(rows, ib, nb)
        r16 = s16.sort_batch(rows, ib, nb)
        a = set(zip(r32['time'].tolist(), r32['template'].tolist()))
        b = set(zip(r16['time'].tolist(), r16['template'].tolist()))
        assert len(a) > 0
        assert len(a & b) >= 0.99 * max(len(a), len(b)), (ib, len(a), len(b), len(a & b))


def test_bf16_recheck_agreement_on_synthetic_recording():
    from livespikesorter_b200 import synth
    from livespikesorter_b200.sorter import Sorter
    setup, rec = synth.config(1, duration_s=4.0, seed=17, T=400)
    s32 = Sorter.from_setup(setup)
    s16 = Sorter.from_setup(setup, precision='bf16')
    NT, nt = setup.NT, setup.nt
    ib = 1
    rows = np.ascontiguousarray(rec.raw[ib * NT - nt: ib * NT + NT + nt])
    M = setup.drift_matrix(rec.dshift[ib])
    s32.set_drift(M)
    s16.set_drift(M)
    r32 = s32.sort_batch(rows, ib, rec.n_batches)
    r16 = s16.sort_batch(rows, ib, rec.n_batches)
    st = s16.stats()
    a = set(zip(r32['time'].tolist(), r32['template'].tolist()))
    b = set(zip(r16['time'].tolist(), r16['template'].tolist()))
    assert len(a) > 1000
    assert st['recheck_columns'] > 0
    assert len(a & b) >= 0.99 * max(len(a), len(b)), (len(a), len(b), len(a & b), st)


def test_bf16_recheck_at_800_templates_with_near_duplicates():
    """384 channels, 800 templates of which 10 % are near-duplicate pairs
    (centres 10 um apart: runner-up decisions sit close to the best), drift
    on: the BF16 + FP32 re-check path keeps >= 0.99 spike agreement with the
    FP32 path, and its score field stays within the bf16 rounding bound of the
    FP32 path's (|dB| <= 2^-7 ||U_t|| ||P_s||, re-scored columns exact)."""
    from livespikesorter_b200 import synth
    from livespikesorter_b200.sorter import Sorter
    setup, rec = synth.config(2, duration_s=4.0, seed=19, T=800)
    s32 = Sorter.from_setup(setup)
    s16 = Sorter.from_setup(setup, precision='bf16')
    NT, nt = setup.NT, setup.nt
    ib = 1
    rows = np.ascontiguousarray(rec.raw[ib * NT - nt: ib * NT + NT + nt])
    M = setup.drift_matrix(rec.dshift[ib])
    s32.set_drift(M)
    s16.set_drift(M)
    r32 = s32.sort_batch(rows, ib, rec.n_batches)
    r16 = s16.sort_batch(rows, ib, rec.n_batches)
    st = s16.stats()
    a = set(zip(r32['time'].tolist(), r32['template'].tolist()))
    b = set(zip(r16['time'].tolist(), r16['template'].tolist()))
    assert len(a) > 10000
    assert st['recheck_columns'] > 0
    assert len(a & b) >= 0.99 * max(len(a), len(b)), (len(a), len(b), len(a & b), st)
    # score fields of one filtered batch
    X = s32.filter(rows, ib, rec.n_batches)
    B32 = s32.scores(X).double()
    B16 = s16.scores(X).double()
    U = setup.U.double().cuda()
    P = torch.nn.functional.conv1d(X.double().unsqueeze(1), setup.wPCA.double().cuda().unsqueeze(1), padding=nt // 2)
    bound = 2.0 ** -7 * U.reshape(U.shape[0], -1).norm(dim=1)[:, None] * P.permute(1, 0, 2).reshape(-1, P.shape[-1]).norm(dim=0)[None]
    err = (B16 - B32).abs()
    assert bool((err <= bound + 1e-6).all())
    st = s16.stats()
    assert int(((B16 == B32).all(dim=0)).sum()) >= st['recheck_rescored']
    # the re-check is column-granular and selective: a small part of the batch
    assert 0 < st['recheck_rescored'] < 0.2 * B16.shape[1], st
    nm = (setup.U.double() ** 2).sum(-1).sum(-1).cuda()
    assert _first_round(B16, nm, setup.Th, nt) == _first_round(B32, nm, setup.Th, nt)
