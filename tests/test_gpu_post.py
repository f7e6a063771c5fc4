"""Post-processing on the GPU (csrc/post.cu): positions, nearest-centroid
clusters, per-cluster duplicate removal carried across batches, time order.

Checked against the reference's own compute_spike_positions and
remove_duplicates output on the c32_t12 recording
(tests/golden/post_c32_t12.npz), through lss_sort_batch over its three
batches, and for a serving stream by the invariants the stage guarantees.
"""
import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _sorter():
    from livespikesorter_b200.sorter import Sorter
    g = np.load(GOLDEN / 'ks4_extract_c32_t12.npz')
    C, T, NT, nt, nt0min, nC, K, nb = [int(v) for v in g['params']]
    s = Sorter(U=g['U'], wPCA=g['wPCA'], ctc=g['ctc'], Wrot=g['Wrot'], hp_filter=g['hp_filter'], iCC=g['iCC'],
               iU=g['iU'], Ucc=g['Ucc'], NT=NT, nt0min=nt0min, Th=float(g['Th']))
    return g, s, NT, nt, nb


def _run(g, s, NT, nt, nb):
    recs = []
    for ib in range(nb):
        rows = g['raw'][0:NT + nt] if ib == 0 else g['raw'][ib * NT - nt: ib * NT + NT + nt]
        r = s.sort_batch(rows, ib, nb)
        t = r['time'].numpy()
        assert np.all(np.diff(t) >= 0)                      # time order within the batch
        recs.append({k: v.numpy() for k, v in r.items() if v is not None})
    return {k: np.concatenate([r[k] for r in recs]) for k in recs[0]}


def _by_time(time, *cols):
    o = np.lexsort((cols[0], time))
    return (time[o],) + tuple(c[o] for c in cols)


@pytest.mark.parametrize('centroids', [False, True])
def test_sort_batch_postprocessing_matches_reference(centroids):
    g, s, NT, nt, nb = _sorter()
    p = np.load(GOLDEN / 'post_c32_t12.npz')
    dt = int(p['dt'])
    s.set_postprocess(xc=g['xc'], yc=g['yc'], centroids=p['centroids'] if centroids else None, dt=dt)
    got = _run(g, s, NT, nt, nb)
    st = g['extract_st']
    keep = p['keep_c'] if centroids else p['keep_t']
    clu = p['clu'] if centroids else st[:, 1].astype(np.int64)
    want_t, want_y, want_c, want_x, want_yy = _by_time(st[keep, 0].astype(np.int64), st[keep, 1].astype(np.int64),
                                                       clu[keep], p['xs'][keep], p['ys'][keep])
    got_t, got_y, got_c, got_x, got_yy = _by_time(got['time'], got['template'].astype(np.int64),
                                                  got['cluster'].astype(np.int64), got['x'], got['y'])
    assert np.array_equal(got_t, want_t) and np.array_equal(got_y, want_y)
    assert np.array_equal(got_c, want_c)
    # positions: the PC features agree with the reference to 1e-3 of their scale
    assert np.allclose(got_x, want_x, atol=0.5) and np.allclose(got_yy, want_yy, atol=0.5)
    # a first batch resets the carried state: a second pass gives the same records
    again = _run(g, s, NT, nt, nb)
    for k in got:
        assert np.array_equal(got[k], again[k])


def test_stream_postprocessing_invariants():
    from livespikesorter_b200 import synth
    from livespikesorter_b200.serve import ProbeServer, Stream, run_streams
    from livespikesorter_b200.sorter import setup_kwargs
    setup, rec = synth.config(0, duration_s=1.0, seed=4, T=32)
    kw = setup_kwargs(setup) | dict(NT=600)
    xc, yc = setup.probe.xc, setup.probe.yc
    cen = np.stack([np.full(6, xc.mean()), np.linspace(yc.min(), yc.max(), 6)], 1)
    dt = 30
    srv = ProbeServer(memory_budget=4 << 30)
    st = Stream('p', kw, rec.raw, 600, depth=3, capacity=4096, post=dict(xc=xc, yc=yc, centroids=cen, dt=dt))
    run_streams(srv, [st], realtime=False)
    batches = [st.results[b] for b in sorted(st.results)]
    t = np.concatenate([r['time'] for r in batches])
    c = np.concatenate([r['cluster'] for r in batches])
    y = np.concatenate([r['y'] for r in batches])
    assert len(t) > 50
    assert np.all(np.diff(t) >= 0) and np.all(t >= 0)
    assert c.min() >= 0 and c.max() < len(cen)
    for k in range(len(cen)):
        tk = t[c == k]
        assert np.all(np.diff(tk) >= dt)                      # no duplicates, across batch borders too
    # every spike's cluster is its nearest centroid (x is on the probe's axis here)
    xs = np.concatenate([r['x'] for r in batches])
    d = np.hypot(xs[:, None] - cen[None, :, 0], y[:, None] - cen[None, :, 1])
    assert np.all(d[np.arange(len(c)), c] <= d.min(1) + 1e-3)
