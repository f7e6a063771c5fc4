"""Regenerate the golden fixtures in this directory from the reference itself.

Run where the reference tree is present (its root in ``LSS_REFERENCE_ROOT``,
default ``/root/reference``):

    python tests/golden/make_golden.py

It writes
* ``conv1d_known_answer.npz`` - the reference's hand-made integer case,
  obtained by executing the computation part of ``src/Python/conv1d_test.py``
  (lines 1-31; the file-writing tail is not run);
* ``ks4_extract_<name>.npz`` - small seeded recordings pushed through the
  vendored Kilosort4 ``BinaryFiltered`` filter chain and ``extract`` (which
  calls ``run_matching``), storing the inputs and every stage output.

The fixtures are what the oracle and the CUDA path are pinned against on
machines where the reference tree is absent.
"""
from __future__ import annotations

import contextlib
import io
import os
import sys
import tempfile
import types
from pathlib import Path

import numpy as np
import torch

REF = Path(os.environ.get('LSS_REFERENCE_ROOT', '/root/reference'))
KS_SITE = REF / 'src/Python/run_online_spikes/Lib/site-packages'
HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))


def import_reference():
    sys.path.insert(0, str(KS_SITE))
    sys.modules.setdefault('faiss', types.ModuleType('faiss'))
    import warnings
    warnings.filterwarnings('ignore')
    from kilosort import template_matching, io as ksio, preprocessing
    return template_matching, ksio, preprocessing


def known_answer():
    src = (REF / 'src/Python/conv1d_test.py').read_text().splitlines()
    cut = next(i for i, l in enumerate(src) if l.startswith('write_tensor(test_dir'))
    ns: dict = {}
    exec(compile('\n'.join(src[:cut]), 'conv1d_test.py', 'exec'), ns)
    out = {k: ns[k].numpy() for k in ('batch', 'wPCA', 'nm', 'B', 'Wall3', 'C', 'Cf', 'Cfmax',
                                      'imax', 'ctc_permuted', 'spike_templates', 'ctc_sub')}
    out['Cmax'] = ns['Cmax'][0][0].numpy()
    out['M'] = np.array(ns['M'])
    np.savez_compressed(HERE / 'conv1d_known_answer.npz', **out)


def ks4_extract_case(name: str, C: int, T: int, NT: int, n_batches: int, seed: int,
                     drift: bool, tail: int = 0):
    tm, ksio, pp = import_reference()
    from livespikesorter_b200 import synth
    probe = synth.probe_staggered(C) if C % 4 == 0 else synth.probe_two_column(C)
    setup, units = synth.make_setup_and_units(probe, T, seed, NT=NT, n_cov_samples=20000)
    dur = (n_batches * NT - tail) / setup.fs
    rec = synth.render(setup, units, dur, seed + 100, drift_um_per_min=(300.0 if drift else 0.0))
    raw = rec.raw
    xc = probe.xc.astype(np.float32)
    yc = probe.yc.astype(np.float32)
    ops = dict(nt=setup.nt, nt0min=setup.nt0min, Th_learned=setup.Th, fs=setup.fs, batch_size=NT,
               Nchan=C, wPCA=setup.wPCA, xc=xc, yc=yc, yblk=np.array([0.0]), nblocks=1,
               probe=dict(xc=xc, yc=yc), iKxx=setup.iKxx.float(),
               settings=dict(nearest_chans=setup.nC, n_pcs=setup.K, sig_interp=20.0))
    dshift = rec.dshift.astype(np.float32) if drift else None
    bfile = ksio.BinaryFiltered('unused.bin', C, setup.fs, NT, setup.nt, setup.nt0min,
                                chan_map=np.arange(C), hp_filter=setup.hp_filter,
                                whiten_mat=setup.Wrot, dshift=dshift, device=torch.device('cpu'),
                                file_object=raw)
    out = dict(raw=raw, xc=xc, yc=yc, wPCA=setup.wPCA.numpy(), U=setup.U.numpy(),
               Wrot=setup.Wrot.numpy(), hp_filter=setup.hp_filter.numpy(),
               iKxx=setup.iKxx.float().numpy(), dshift=(rec.dshift.astype(np.float32) if drift else np.zeros(0)),
               params=np.array([C, T, NT, setup.nt, setup.nt0min, setup.nC, setup.K, n_batches]),
               Th=np.array(setup.Th))
    sink = io.StringIO()
    with contextlib.redirect_stdout(sink):
        ctc = tm.prepare_matching(ops, setup.U)
        iCC, iU, Ucc = tm.prepare_extract(ops, setup.U, setup.nC, device=torch.device('cpu'))
        out.update(ctc=ctc.numpy(), iCC=iCC.numpy(), iU=iU.numpy(), Ucc=Ucc.numpy())
        if drift:
            out['drift_M'] = np.stack([pp.get_drift_matrix(ops, dshift[i], device=torch.device('cpu')).numpy()
                                       for i in range(bfile.n_batches)])
        for ib in range(bfile.n_batches):
            X = bfile.padded_batch_to_torch(ib, ops)
            stt, amps, Xres = tm.run_matching(ops, X, setup.U, ctc, device=torch.device('cpu'))
            out[f'X_{ib}'] = X.numpy()
            out[f'st_{ib}'] = stt.numpy()
            out[f'amps_{ib}'] = amps.numpy()
            if ib == 0:
                out['Xres_0'] = Xres.numpy()
        with tempfile.TemporaryDirectory() as td:
            st_all, tF, _ = tm.extract(ops, Path(td), bfile, setup.U, device=torch.device('cpu'))
    out['extract_st'] = st_all
    out['extract_tF'] = tF.numpy()
    np.savez_compressed(HERE / f'ks4_extract_{name}.npz', **out)
    print(name, 'batches', bfile.n_batches, 'spikes', len(st_all))


def post_case():
    """Reference postprocessing (postprocessing.py:10-46) on the c32_t12
    extract output: spike positions, and duplicate removal per template and
    per nearest-centroid cluster."""
    import_reference()
    from kilosort.postprocessing import compute_spike_positions, remove_duplicates
    sys.path.insert(0, str(HERE.parents[1] / 'oracle'))
    import ks4_oracle as ko
    g = np.load(HERE / 'ks4_extract_c32_t12.npz')
    st = g['extract_st']
    sti = np.stack([st[:, 0], st[:, 1]], 1).astype(np.int64)
    tF = torch.from_numpy(g['extract_tF'])
    ops = dict(xc=g['xc'], yc=g['yc'], iCC=torch.from_numpy(g['iCC']), iU=torch.from_numpy(g['iU']))
    xs, ys = compute_spike_positions(sti, tF, ops)
    # dt: Kilosort's default (7 samples at 30 kHz) removes nothing in this
    # sparse case, so a wide window (600 samples) exercises the removal
    dt = 600
    t = sti[:, 0].astype(np.int64)
    _, _, keep_t = remove_duplicates(t, sti[:, 1].astype(np.int32), np.int32(dt))
    # centroids: four well separated points over the probe; clusters by the
    # reference's nearest-centroid rule (restated: its code is C++)
    rng = np.random.default_rng(3)
    cen = np.stack([rng.uniform(g['xc'].min(), g['xc'].max(), 4), np.linspace(g['yc'].min(), g['yc'].max(), 4)], 1)
    cen = cen.astype(np.float32)
    clu = ko.closest_cluster(xs, ys, cen)
    _, _, keep_c = remove_duplicates(t, clu.astype(np.int32), np.int32(dt))
    np.savez_compressed(HERE / 'post_c32_t12.npz', xs=xs, ys=ys, dt=dt, keep_t=keep_t, centroids=cen, clu=clu,
                        keep_c=keep_c)
    print('post', len(t), 'kept (templates)', int(keep_t.sum()), 'kept (centroids)', int(keep_c.sum()))


if __name__ == '__main__':
    torch.set_num_threads(8)
    known_answer()
    # three batches: first (leading replicate), middle, last (tail replicate),
    # highpass cropped (N < 30122), no drift
    ks4_extract_case('c32_t12', C=32, T=12, NT=4000, n_batches=3, seed=11, drift=False, tail=1500)
    # two batches with drift correction and the padded-highpass branch (N > 30122)
    ks4_extract_case('c16_t8_drift', C=16, T=8, NT=31000, n_batches=2, seed=12, drift=True, tail=7000)
    post_case()
