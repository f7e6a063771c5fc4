"""PC features on both kernel paths: the warp-per-spike kernel (nC = 10,
K = 6) and the CTA-per-spike kernel (other nC / K), against the oracle's
extract (template_matching.py:46-73) on the same batch: identical records,
features within 1e-3 of their largest magnitude."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('nC', [10, 8])
def test_features_match_oracle_extract(nC):
    import ks4_oracle as ko
    from livespikesorter_b200 import synth
    from livespikesorter_b200.sorter import Sorter, setup_kwargs
    probe = synth.probe_two_column(64)
    setup, units = synth.make_setup_and_units(probe, 24, seed=13, NT=6000, nC=nC)
    rec = synth.render(setup, units, 1.0, seed=113)
    NT, nt, ib, nb = setup.NT, setup.nt, 2, rec.n_batches
    s = Sorter.from_setup(setup)
    r = s.sort_batch(np.ascontiguousarray(rec.raw[ib * NT - nt: ib * NT + NT + nt]), ib, nb)
    X = ko.padded_batch(rec.raw, ib, NT, nt)
    X = ko.filter_batch(X, hp_filter=setup.hp_filter, whiten_mat=setup.Wrot)
    st, amps, Xres = ko.run_matching(X, setup.U, setup.ctc, setup.wPCA, setup.Th, nt)
    st3, tF = ko.extract_batch(st, amps, Xres, setup.iCC, setup.iU, setup.Ucc, setup.wPCA, nt, setup.nt0min, ib, NT)
    assert len(st3) > 20
    got = sorted(zip(r['time'].tolist(), r['template'].tolist()))
    want = sorted(zip(st3[:, 0].astype(np.int64).tolist(), st3[:, 1].astype(np.int64).tolist()))
    assert got == want
    o1 = np.lexsort((r['template'].numpy(), r['time'].numpy()))
    o2 = np.lexsort((st3[:, 1], st3[:, 0]))
    pc = r['pc'].numpy()[o1]
    ref = tF.numpy()[o2]
    assert pc.shape == ref.shape == (len(st3), nC, setup.K)
    assert np.abs(pc - ref).max() <= 1e-3 * np.abs(ref).max()
