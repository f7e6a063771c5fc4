"""Pin the CPU oracle to the reference: its known-answer case, the golden
fixtures the reference produced, and (where the reference tree is present)
live calls into the vendored Kilosort4 functions on seeded inputs."""
import contextlib
import io

import numpy as np
import pytest
import torch

import ks4_oracle as ko
from conftest import GOLDEN


def _npz(name):
    return np.load(GOLDEN / name)


def test_known_answer_conv1d_case():
    """src/Python/conv1d_test.py:14-43: conv -> score -> Cf -> Cfmax -> Cmax."""
    g = _npz('conv1d_known_answer.npz')
    batch = torch.from_numpy(g['batch']).double()
    wPCA = torch.from_numpy(g['wPCA']).double()
    U = torch.from_numpy(g['Wall3']).double()
    M = int(g['M'])
    B = ko.score_field(batch, U, wPCA, nt=M, dtype=torch.float64)
    assert np.array_equal(B.numpy(), g['C'].astype(np.float64))
    nm = torch.from_numpy(g['nm']).double()
    Cf = torch.relu(B) ** 2 / nm.unsqueeze(-1)
    Cf[:, :M] = 0
    Cf[:, -M:] = 0
    Cfmax, imax = torch.max(Cf, 0)
    Cmax = torch.nn.functional.max_pool1d(Cfmax[None, None], 2 * M + 1, stride=1, padding=M)[0, 0]
    np.testing.assert_allclose(Cf.numpy(), g['Cf'], rtol=1e-6)
    np.testing.assert_allclose(Cfmax.numpy(), g['Cfmax'], rtol=1e-6)
    assert np.array_equal(imax.numpy(), g['imax'])
    np.testing.assert_allclose(Cmax.numpy(), g['Cmax'], rtol=1e-6)
    ctc_p = torch.from_numpy(g['ctc_permuted'])
    assert np.array_equal(ctc_p[torch.from_numpy(g['spike_templates'])].numpy(), g['ctc_sub'])


@pytest.mark.parametrize('name', ['ks4_extract_c32_t12.npz', 'ks4_extract_c16_t8_drift.npz'])
def test_oracle_reproduces_reference_fixture(name):
    g = _npz(name)
    C, T, NT, nt, nt0min, nC, K, _ = [int(v) for v in g['params']]
    raw = g['raw']
    n_batches = int(np.ceil(raw.shape[0] / NT))
    U = torch.from_numpy(g['U'])
    wPCA = torch.from_numpy(g['wPCA'])
    ctc = torch.from_numpy(g['ctc'])
    assert torch.equal(ko.prepare_matching(wPCA, U, nt), ctc)
    iCC, iU, Ucc = ko.prepare_extract(g['xc'], g['yc'], U, nC)
    assert np.array_equal(iCC.numpy(), g['iCC']) and np.array_equal(iU.numpy(), g['iU'])
    assert np.array_equal(Ucc.numpy(), g['Ucc'])
    st_all, tF_all = [], []
    for ib in range(n_batches):
        X = ko.padded_batch(raw, ib, NT, nt)
        M = torch.from_numpy(g['drift_M'][ib]) if 'drift_M' in g.files else None
        X = ko.filter_batch(X, chan_map=np.arange(C), hp_filter=torch.from_numpy(g['hp_filter']),
                            whiten_mat=torch.from_numpy(g['Wrot']), drift_M=M)
        assert np.array_equal(X.numpy(), g[f'X_{ib}']), f'filter, batch {ib}'
        st, amps, Xres = ko.run_matching(X, U, ctc, wPCA, float(g['Th']), nt)
        assert np.array_equal(st.numpy(), g[f'st_{ib}'])
        assert np.array_equal(amps.numpy(), g[f'amps_{ib}'])
        if ib == 0:
            assert np.array_equal(Xres.numpy(), g['Xres_0'])
        s3, tF = ko.extract_batch(st, amps, Xres, iCC, iU, Ucc, wPCA, nt, nt0min, ib, NT)
        st_all.append(s3)
        tF_all.append(tF)
    st_all = np.concatenate(st_all)
    tF_all = torch.cat(tF_all)
    isort = np.argsort(st_all[:, 0])
    assert np.array_equal(st_all[isort], g['extract_st'])
    np.testing.assert_array_equal(tF_all[isort].numpy(), g['extract_tF'])


def _rand_case(seed, C=12, T=6, K=3, nt=21, N=900):
    g = torch.Generator().manual_seed(seed)
    wPCA = torch.linalg.qr(torch.randn(nt, K, generator=g))[0].T.contiguous()
    U = torch.randn(T, K, C, generator=g) * 3
    X = torch.randn(C, N, generator=g)
    # plant template waveforms so that there are spikes
    wav = torch.einsum('tkc,km->tcm', U, wPCA)
    for i in range(25):
        t = int(torch.randint(0, T, (1,), generator=g))
        s = int(torch.randint(nt, N - nt, (1,), generator=g))
        X[:, s - nt // 2:s + nt // 2 + 1] += wav[t] * (1 + torch.rand(1, generator=g))
    return X, U, wPCA, nt


@pytest.mark.parametrize('seed', [0, 1, 2])
def test_oracle_matches_live_reference(reference_ks, seed):
    X, U, wPCA, nt = _rand_case(seed)
    ops = {'Th_learned': 6.0, 'nt': nt, 'wPCA': wPCA}
    with contextlib.redirect_stdout(io.StringIO()):
        ctc_ref = reference_ks.tm.prepare_matching(ops, U)
        st_r, amps_r, xres_r = reference_ks.tm.run_matching(ops, X, U, ctc_ref, device=torch.device('cpu'))
    ctc = ko.prepare_matching(wPCA, U, nt)
    assert torch.equal(ctc, ctc_ref)
    st, amps, xres = ko.run_matching(X, U, ctc, wPCA, 6.0, nt)
    assert len(st_r) > 10
    assert torch.equal(st, st_r) and torch.equal(amps, amps_r) and torch.equal(xres, xres_r)


def test_setup_functions_match_reference(reference_ks):
    from livespikesorter_b200 import setup_tensors as stp
    X, U, wPCA, nt = _rand_case(5)
    xc = np.arange(12, dtype=np.float32) % 2 * 16
    yc = np.arange(12, dtype=np.float32) // 2 * 20
    ops = {'xc': xc, 'yc': yc, 'wPCA': wPCA, 'nt': nt}
    ctc_ref = reference_ks.tm.prepare_matching(ops, U)
    assert torch.equal(stp.prepare_matching(wPCA, U), ctc_ref)
    r = reference_ks.tm.prepare_extract(ops, U, 4, device=torch.device('cpu'))
    m = stp.prepare_extract(xc, yc, U, 4)
    for a, b in zip(r, m):
        assert torch.equal(a, b)
    assert torch.equal(reference_ks.pp.get_highpass_filter(30000, 300, device=torch.device('cpu')),
                       stp.get_highpass_filter(30000, 300))


def test_fp64_oracle_agrees_with_fp32_on_clear_margins():
    X, U, wPCA, nt = _rand_case(3)
    ctc = ko.prepare_matching(wPCA, U, nt)
    st32, a32, _ = ko.run_matching(X, U, ctc, wPCA, 6.0, nt)
    st64, a64, _ = ko.run_matching(X, U, ko.prepare_matching(wPCA.double(), U.double(), nt), wPCA, 6.0, nt,
                                   dtype=torch.float64)
    assert torch.equal(st32, st64)
    np.testing.assert_allclose(a32.numpy(), a64.numpy(), rtol=1e-5)


def test_postprocess_oracle_reproduces_reference_fixture():
    """Positions and duplicate removal restated in the oracle equal the
    reference's compute_spike_positions / remove_duplicates output
    (tests/golden/post_c32_t12.npz, made by make_golden.post_case)."""
    g = np.load(GOLDEN / 'ks4_extract_c32_t12.npz')
    p = np.load(GOLDEN / 'post_c32_t12.npz')
    st = np.stack([g['extract_st'][:, 0], g['extract_st'][:, 1]], 1).astype(np.int64)
    xs, ys = ko.spike_positions(st, torch.from_numpy(g['extract_tF']), torch.from_numpy(g['iCC']),
                                torch.from_numpy(g['iU']), g['xc'], g['yc'])
    assert np.array_equal(xs, p['xs']) and np.array_equal(ys, p['ys'])
    dt = int(p['dt'])
    _, _, keep = ko.remove_duplicates(st[:, 0], st[:, 1], dt)
    assert np.array_equal(keep, p['keep_t'])
    clu = ko.closest_cluster(xs, ys, p['centroids'])
    assert np.array_equal(clu, p['clu'])
    _, _, keep = ko.remove_duplicates(st[:, 0], clu, dt)
    assert np.array_equal(keep, p['keep_c'])
    # carrying the last kept time across a split gives the same answer
    t0 = {}
    k1 = ko.remove_duplicates(st[:30, 0], clu[:30], dt, t0)[2]
    k2 = ko.remove_duplicates(st[30:, 0], clu[30:], dt, t0)[2]
    assert np.array_equal(np.concatenate([k1, k2]), p['keep_c'])


def test_postprocess_oracle_matches_live_reference(reference_ks):
    from kilosort.postprocessing import compute_spike_positions, remove_duplicates
    g = np.random.default_rng(5)
    n, nC, K, C, T = 400, 6, 4, 24, 9
    tF = torch.from_numpy(g.standard_normal((n, nC, K)).astype(np.float32))
    st = np.stack([np.sort(g.integers(0, 30000, n)), g.integers(0, T, n)], 1).astype(np.int64)
    iCC = torch.from_numpy(g.integers(0, C, (nC, C)))
    iU = torch.from_numpy(g.integers(0, C, T))
    xc, yc = g.uniform(0, 50, C).astype(np.float32), g.uniform(0, 700, C).astype(np.float32)
    ops = dict(xc=xc, yc=yc, iCC=iCC, iU=iU)
    xs, ys = compute_spike_positions(st, tF, ops)
    xo, yo = ko.spike_positions(st, tF, iCC, iU, xc, yc)
    assert np.array_equal(xs, xo) and np.array_equal(ys, yo)
    for dt in (7, 90):
        a = remove_duplicates(st[:, 0], st[:, 1].astype(np.int32), np.int32(dt))
        b = ko.remove_duplicates(st[:, 0], st[:, 1], dt)
        assert np.array_equal(a[2], b[2])
