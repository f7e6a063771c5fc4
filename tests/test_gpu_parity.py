"""Parity of the CUDA path (through the C ABI) with the oracle and with the
reference's golden fixtures.

Tolerances:
* matching-pursuit rounds on a given score field: bit-identical spikes and
  amplitudes (the update arithmetic is single-rounded FP32 like the reference);
* end to end from a filtered batch or from int16: identical (time, template)
  spike set, amplitudes within 1e-4 relative (the score GEMM sums in a
  different order than torch's CPU kernels);
* filtered batch: max |dX| <= 2e-5 * max|X| (FP32 transform rounding);
* PC features: max |dF| <= 1e-3 * max|F|.
"""
import numpy as np
import pytest
import torch

import ks4_oracle as ko
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

AMP_RTOL = 1e-4


def _fixture(name):
    g = np.load(GOLDEN / name)
    C, T, NT, nt, nt0min, nC, K, _ = [int(v) for v in g['params']]
    return g, dict(C=C, T=T, NT=NT, nt=nt, nt0min=nt0min, nC=nC, K=K)


def _sorter(g, p, **kw):
    from livespikesorter_b200.sorter import Sorter
    return Sorter(U=g['U'], wPCA=g['wPCA'], ctc=g['ctc'], Wrot=g['Wrot'], hp_filter=g['hp_filter'],
                  iCC=g['iCC'], iU=g['iU'], Ucc=g['Ucc'], NT=p['NT'], nt0min=p['nt0min'], Th=float(g['Th']), **kw)


def _assert_same_spikes(st_a, amp_a, st_b, amp_b):
    """Same (time, template) sequence in run_matching order (round-major,
    time-minor; Kilosort may pick the same pair again in a later round), and
    amplitudes within AMP_RTOL."""
    ka = np.asarray(st_a)[:, :2].astype(np.int64)
    kb = np.asarray(st_b)[:, :2].astype(np.int64)
    assert ka.shape == kb.shape, (ka.shape, kb.shape)
    bad = np.nonzero((ka != kb).any(1))[0]
    assert len(bad) == 0, (bad[:5], ka[bad[:5]], kb[bad[:5]])
    a = np.ravel(amp_a).astype(np.float64)
    b = np.ravel(amp_b).astype(np.float64)
    assert np.all(np.abs(a - b) <= AMP_RTOL * np.maximum(np.abs(b), 1e-6)), np.max(np.abs(a - b) / np.abs(b))


def test_known_answer_case_scores():
    """The reference's conv1d_test.py integer case through lss_scores: exact."""
    from livespikesorter_b200.sorter import Sorter
    g = np.load(GOLDEN / 'conv1d_known_answer.npz')
    M = int(g['M'])
    U = g['Wall3'].astype(np.float32)
    s = Sorter(U=U, wPCA=g['wPCA'].astype(np.float32), ctc=np.zeros((2, 2, 2 * M + 1), np.float32),
               Wrot=np.eye(2, dtype=np.float32), NT=g['batch'].shape[1] - 2 * M, Th=1.0)
    B = s.scores(torch.from_numpy(g['batch'].astype(np.float32)).cuda())
    assert np.array_equal(B.cpu().numpy(), g['C'].astype(np.float32))


@pytest.mark.parametrize('name', ['ks4_extract_c32_t12.npz', 'ks4_extract_c16_t8_drift.npz'])
def test_rounds_bit_exact_on_given_scores(name):
    g, p = _fixture(name)
    U = torch.from_numpy(g['U'])
    wPCA = torch.from_numpy(g['wPCA'])
    nm = (U ** 2).sum(-1).sum(-1)
    s = _sorter(g, p, nm=nm)
    for ib in range(int(g['params'][-1])):
        X = torch.from_numpy(g[f'X_{ib}'])
        B = ko.score_field(X, U, wPCA, p['nt'])
        st_o, amps_o, _ = ko.run_matching(X, U, torch.from_numpy(g['ctc']), wPCA, float(g['Th']), p['nt'],
                                          B=B, nm=nm)
        st, amps = s.match_scores(B.cuda())
        assert len(st_o) > 0
        assert torch.equal(st.cpu(), st_o), ib
        assert torch.equal(amps.cpu(), amps_o), ib


@pytest.mark.parametrize('name', ['ks4_extract_c32_t12.npz', 'ks4_extract_c16_t8_drift.npz'])
def test_match_matches_reference_run_matching(name):
    g, p = _fixture(name)
    s = _sorter(g, p)
    for ib in range(int(g['params'][-1])):
        X = torch.from_numpy(g[f'X_{ib}']).cuda()
        st, amps, xres = s.match(X)
        _assert_same_spikes(st.cpu(), amps.cpu(), g[f'st_{ib}'], g[f'amps_{ib}'])
        if ib == 0:
            ref = g['Xres_0']
            assert np.abs(xres.cpu().numpy() - ref).max() <= 1e-4 * np.abs(ref).max()


@pytest.mark.parametrize('name', ['ks4_extract_c32_t12.npz', 'ks4_extract_c16_t8_drift.npz'])
def test_filter_matches_reference(name):
    g, p = _fixture(name)
    s = _sorter(g, p)
    raw = g['raw']
    nb = int(np.ceil(raw.shape[0] / p['NT']))
    for ib in range(nb):
        if 'drift_M' in g.files:
            s.set_drift(g['drift_M'][ib])
        rows = _rows(raw, ib, nb, p['NT'], p['nt'])
        X = s.filter(rows, ib, nb).cpu().numpy()
        ref = g[f'X_{ib}']
        err = np.abs(X - ref).max() / np.abs(ref).max()
        assert err <= 2e-5, (ib, err)


def _rows(raw, ib, nb, NT, nt):
    """The rows padded_batch_to_torch reads for batch ib (kilosort/io.py:589-599)."""
    if ib == 0:
        return raw[0:NT + nt]
    b0 = ib * NT - nt
    return raw[b0:min(raw.shape[0], b0 + NT + 2 * nt)]


@pytest.mark.parametrize('on_device', [False, True])
def test_sort_batch_matches_reference_extract(on_device):
    g, p = _fixture('ks4_extract_c16_t8_drift.npz')
    s = _sorter(g, p)
    raw = g['raw']
    nb = int(np.ceil(raw.shape[0] / p['NT']))
    times, tmpl, amp, pc = [], [], [], []
    for ib in range(nb):
        s.set_drift(g['drift_M'][ib])
        rows = _rows(raw, ib, nb, p['NT'], p['nt'])
        r = s.sort_batch(torch.from_numpy(rows).cuda() if on_device else rows, ib, nb, on_device=on_device)
        times.append(r['time'].cpu().numpy())
        tmpl.append(r['template'].cpu().numpy())
        amp.append(r['amplitude'].cpu().numpy())
        pc.append(r['pc'].cpu().numpy())
    times, tmpl, amp, pc = map(np.concatenate, (times, tmpl, amp, pc))
    ref = g['extract_st']
    ref_tf = g['extract_tF']
    ia = np.lexsort((amp, tmpl, times))
    ib_ = np.lexsort((ref[:, 2], ref[:, 1], ref[:, 0]))
    _assert_same_spikes(np.stack([times, tmpl], 1)[ia], amp[ia], ref[ib_, :2], ref[ib_, 2])
    assert np.abs(pc[ia] - ref_tf[ib_]).max() <= 1e-3 * np.abs(ref_tf).max()


def test_run_matching_drop_in():
    from livespikesorter_b200 import sorter
    g, p = _fixture('ks4_extract_c32_t12.npz')
    ops = {'Th_learned': float(g['Th']), 'nt': p['nt'], 'wPCA': torch.from_numpy(g['wPCA']), 'nt0min': p['nt0min']}
    X = torch.from_numpy(g['X_1'])
    st, amps, xres = sorter.run_matching(ops, X, torch.from_numpy(g['U']), torch.from_numpy(g['ctc']))
    assert st.dtype == torch.int64 and st.shape[1] == 2 and amps.shape[1] == 1 and xres.shape == X.shape
    _assert_same_spikes(st.cpu(), amps.cpu(), g['st_1'], g['amps_1'])


def test_create_from_dir_honours_fortran_order(tmp_path):
    """drift_matrix.npy holds M.T written in Fortran order (run_online_spikes.py:532)."""
    from livespikesorter_b200.sorter import Sorter
    g, p = _fixture('ks4_extract_c16_t8_drift.npz')
    M = g['drift_M'][1]
    for k, v in dict(Wall3=g['U'], wPCA=g['wPCA'], ctc=g['ctc'], whitening_mat=g['Wrot'],
                     hp_filter=g['hp_filter'], iCC=g['iCC'], iU=g['iU'], Ucc=g['Ucc'],
                     channel_map=np.arange(p['C'], dtype=np.int32)).items():
        np.save(tmp_path / f'{k}.npy', v)
    np.save(tmp_path / 'drift_matrix.npy', np.array(M).T)
    assert np.load(tmp_path / 'drift_matrix.npy').flags.f_contiguous
    (tmp_path / 'misc.txt').write_text(f"nt0min:{p['nt0min']}\nnumNearestChans:{p['nC']}\n"
                                       f"Th_learned:{float(g['Th'])}\nduplicate_spike_bins:7\n")
    a = Sorter.from_dir(tmp_path, NT=p['NT'])
    b = _sorter(g, p)
    b.set_drift(M)
    rows = _rows(g['raw'], 1, 2, p['NT'], p['nt'])
    assert torch.equal(a.filter(rows, 1, 2), b.filter(rows, 1, 2))


def test_zero_input_gives_no_spikes():
    g, p = _fixture('ks4_extract_c32_t12.npz')
    s = _sorter(g, p)
    r = s.sort_batch(np.zeros((p['NT'] + 2 * p['nt'], p['C']), np.int16), 1, 3)
    assert len(r['time']) == 0 and s.stats()['rounds'] == 0


def test_errors_are_status_codes():
    from livespikesorter_b200._lib import LssError, LSS_ERR_CAPACITY, LSS_ERR_SHAPE, LSS_ERR_ARG
    g, p = _fixture('ks4_extract_c32_t12.npz')
    s = _sorter(g, p, max_spikes=3)
    with pytest.raises(LssError) as e:
        s.match(torch.from_numpy(g['X_1']).cuda())
    assert e.value.code == LSS_ERR_CAPACITY
    s2 = _sorter(g, p)
    with pytest.raises(LssError) as e:
        s2.sort_batch(g['raw'][:100], 1, 3)
    assert e.value.code == LSS_ERR_SHAPE
    with pytest.raises(LssError) as e:
        s2.sort_batch(g['raw'][:100], 3, 3)
    assert e.value.code == LSS_ERR_ARG
    # record capacity: the call reports the required size
    rows = _rows(g['raw'], 1, 3, p['NT'], p['nt'])
    with pytest.raises(LssError) as e:
        s2.sort_batch(rows, 1, 3, capacity=2)
    assert e.value.code == LSS_ERR_CAPACITY
    # the handle stays usable after errors
    r = s2.sort_batch(rows, 1, 3)
    assert len(r['time']) == len(g['st_1'])


def _oracle_sort(setup, rec, ib, nb):
    NT, nt = setup.NT, setup.nt
    X = ko.padded_batch(rec.raw, ib, NT, nt)
    X = ko.filter_batch(X, hp_filter=setup.hp_filter, whiten_mat=setup.Wrot)
    st, amps, Xres = ko.run_matching(X, setup.U, setup.ctc, setup.wPCA, setup.Th, nt)
    s3, tF = ko.extract_batch(st, amps, Xres, setup.iCC, setup.iU, setup.Ucc, setup.wPCA, nt, setup.nt0min, ib, NT)
    return s3, tF.numpy()


def test_synthetic_config0_end_to_end():
    """64 channels, 32 templates, 60000 samples of int16: identical spike set."""
    from livespikesorter_b200 import synth
    from livespikesorter_b200.sorter import Sorter
    setup, rec = synth.config(0, seed=3)
    s = Sorter.from_setup(setup)
    ref, ref_tf = _oracle_sort(setup, rec, 0, 1)
    r = s.sort_batch(rec.raw, 0, 1)
    assert len(ref) > 300
    got = np.stack([r['time'].numpy(), r['template'].numpy()], 1)
    _assert_same_spikes(got, r['amplitude'].numpy(), ref[:, :2], ref[:, 2])
    assert np.abs(r['pc'].numpy() - ref_tf).max() <= 1e-3 * np.abs(ref_tf).max()
