"""Streaming serving loop (lss_server_* through ``serve.ProbeServer``).

* A stream's batches equal ``lss_sort_batch`` on the same windows (rows
  [b*NT - 2nt, (b+1)*NT), the stream's first window replicating row 0), with
  record times shifted by the stream convention: bit-identical records.
* Continuous batching: probes with different template counts, block sizes
  and precisions run together; one that does not fit the memory budget waits
  and is admitted when another is released; every probe's records are the
  same alone and in the mix (bit-identical: the per-probe work is
  deterministic and the probes share no device memory).
* A real-time run reports arrival-to-emit latency for every batch, and its
  split into host, queueing, device and callback time.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _probe(T, block, seed, duration_s=1.0, **extra):
    from livespikesorter_b200 import synth
    from livespikesorter_b200.sorter import setup_kwargs
    setup, rec = synth.config(0, duration_s=duration_s, seed=seed, T=T)
    return setup, rec, setup_kwargs(setup) | dict(NT=block) | extra


def _equal(a, b):
    assert np.array_equal(a['time'], b['time'])
    assert np.array_equal(a['template'], b['template'])
    assert np.array_equal(a['amplitude'], b['amplitude'])
    if a['pc'] is not None or b['pc'] is not None:
        assert np.array_equal(a['pc'], b['pc'])


def test_stream_batches_equal_sort_batch_windows():
    from livespikesorter_b200.serve import ProbeServer
    from livespikesorter_b200.sorter import Sorter
    setup, rec, kw = _probe(32, 600, seed=3)
    nt, NT = setup.nt, 600
    srv = ProbeServer(memory_budget=4 << 30)
    pid = srv.admit(depth=3, capacity=4096, **kw)
    nb = 6
    for k in range(nb):
        srv.push(pid, rec.raw[k * NT:(k + 1) * NT])
    got = {}
    for _ in range(nb):
        b, r = srv.poll(pid, wait=True)
        got[b] = r
    assert sorted(got) == list(range(nb))
    assert srv.poll(pid) is None
    lat = srv.latency(pid)
    assert lat['batches'] == nb
    srv.release(pid)
    s = Sorter(**kw)
    total = 0
    for b in range(nb):
        if b == 0:
            rows = np.concatenate([np.repeat(rec.raw[:1], 2 * nt, 0), rec.raw[:NT]])
            r = s.sort_batch(rows, 1, 3)
            shift = NT + nt
        else:
            rows = rec.raw[b * NT - 2 * nt:(b + 1) * NT]
            r = s.sort_batch(rows, b, b + 2)
            shift = nt
        t = r['time'].numpy() - shift
        keep = t >= 0
        want = dict(time=t[keep], template=r['template'].numpy()[keep], amplitude=r['amplitude'].numpy()[keep],
                    pc=r['pc'].numpy()[keep])
        _equal(got[b], want)
        total += keep.sum()
    assert total > 20


def test_continuous_batching_same_alone_and_in_the_mix():
    from livespikesorter_b200.serve import ProbeServer, Stream, run_streams
    probes = [('A', *_probe(32, 600, seed=5)), ('B', *_probe(16, 300, seed=6)),
              ('C', *_probe(24, 1500, seed=7, precision='bf16'))]
    alone, bytes_ = {}, {}
    for name, setup, rec, kw in probes:
        srv = ProbeServer(memory_budget=8 << 30)
        st = Stream(name, kw, rec.raw, kw['NT'], depth=3, capacity=4096)
        run_streams(srv, [st], realtime=False)
        assert len(st.results) == rec.raw.shape[0] // kw['NT']
        alone[name] = st.results
        pid = srv.admit(depth=3, capacity=4096, **kw)
        bytes_[name] = srv.memory()[0]
        srv.release(pid)
        srv.close()
    # room for A and B together, not for all three: C waits for a release
    budget = bytes_['A'] + bytes_['B'] + bytes_['C'] // 2
    srv = ProbeServer(memory_budget=budget)
    streams = [Stream(name, kw, rec.raw, kw['NT'], depth=3, capacity=4096) for name, _, rec, kw in probes]
    out = run_streams(srv, streams, realtime=False)
    by = {st.name: st for st in out['streams']}
    assert by['C'].waited and not by['A'].waited and not by['B'].waited
    for name in alone:
        assert sorted(by[name].results) == sorted(alone[name])
        for b in alone[name]:
            _equal(by[name].results[b], alone[name][b])
    assert srv.memory()[0] == 0


def test_realtime_latency_is_reported():
    from livespikesorter_b200.serve import ProbeServer, Stream, run_streams
    _, rec1, kw1 = _probe(32, 300, seed=8)
    _, rec2, kw2 = _probe(16, 600, seed=9)
    srv = ProbeServer(memory_budget=8 << 30)
    streams = [Stream('p300', kw1, rec1.raw, 300, n_blocks=40), Stream('p600', kw2, rec2.raw, 600, n_blocks=20)]
    out = run_streams(srv, streams, realtime=True, seed=1)
    for st in out['streams']:
        assert st.latency['batches'] == st.n_blocks
        assert 0 < st.latency['p50_ms'] <= st.latency['p99_ms'] < 1000
        # the four parts of each batch's latency add up to it
        parts, lat = np.array(st.latency['parts_ms']), np.array(st.latency['samples_ms'])
        assert parts.shape == (st.n_blocks, 4)
        assert np.allclose(parts.sum(1), lat, rtol=0, atol=1e-6)
        assert np.all(parts[:, 0] >= 0) and np.all(parts[:, 2] > 0)
        # device times mapped to the host clock (offset re-anchored on every
        # batch's own launch / completion bracket): no part is negative
        assert np.all(parts >= 0), parts[(parts < 0).any(1)][:3]
    assert out['wall_s'] >= 0.35


def test_server_rejects_bad_calls():
    from livespikesorter_b200._lib import LssError
    from livespikesorter_b200.serve import ProbeServer
    _, rec, kw = _probe(16, 300, seed=2)
    srv = ProbeServer(memory_budget=1 << 20)
    assert srv.admit(**kw) is None           # does not fit 1 MiB
    srv2 = ProbeServer(memory_budget=4 << 30, max_probes=1)
    pid = srv2.admit(**kw)
    assert pid == 0
    assert srv2.admit(**kw) is None          # no slot
    from livespikesorter_b200._lib import check
    with pytest.raises(LssError):
        check(srv2._lib.lss_server_push(srv2._s, 5, None, 1, 0))   # no such probe
    srv2.release(pid)
    assert srv2.admit(**kw) == 0             # the slot is free again


def test_stream_batches_match_the_oracle_at_384ch():
    """One 384-channel, 400-template probe streamed in 1500-sample blocks:
    every stream batch against the oracle (filter + run_matching + PC
    features) on the same window. Identical (time, template) sequence,
    amplitudes within 1e-4 relative, PC features within 1e-3 of their
    largest magnitude."""
    import torch
    import ks4_oracle as ko
    from livespikesorter_b200 import synth
    from livespikesorter_b200.serve import ProbeServer
    from livespikesorter_b200.sorter import setup_kwargs
    (setup, rec), = synth.streaming_probes(seed=13, duration_s=0.3, Ts=(400,))
    NT, nt = 1500, setup.nt
    kw = setup_kwargs(setup) | dict(NT=NT)
    srv = ProbeServer(memory_budget=16 << 30)
    pid = srv.admit(depth=3, capacity=16384, **kw)
    nb = 5
    for k in range(nb):
        srv.push(pid, rec.raw[k * NT:(k + 1) * NT])
    got = {}
    for _ in range(nb):
        b, r = srv.poll(pid, wait=True)
        got[b] = r
    srv.release(pid)
    srv.close()
    total = 0
    for b in range(nb):
        # the stream's window of batch b: rows [b*NT - 2nt, (b+1)*NT), row 0 replicated before the stream start
        rows = (np.concatenate([np.repeat(rec.raw[:1], 2 * nt, 0), rec.raw[:NT]]) if b == 0
                else rec.raw[b * NT - 2 * nt:(b + 1) * NT])
        X = ko.filter_batch(torch.from_numpy(rows.T.astype(np.float32).copy()), hp_filter=setup.hp_filter,
                            whiten_mat=setup.Wrot)
        st, amps, Xres = ko.run_matching(X, setup.U, setup.ctc, setup.wPCA, setup.Th, nt)
        _, tf = ko.extract_batch(st, amps, Xres, setup.iCC, setup.iU, setup.Ucc, setup.wPCA, nt, setup.nt0min, 1, NT)
        # stream sample time of the window's column x
        t = st[:, 0].numpy() - 2 * nt + b * NT - nt // 2 + setup.nt0min
        keep = t >= 0
        r = got[b]
        assert np.array_equal(r['time'], t[keep]), b
        assert np.array_equal(r['template'], st[:, 1].numpy()[keep]), b
        a = amps[:, 0].numpy().astype(np.float64)[keep]
        assert np.all(np.abs(r['amplitude'] - a) <= 1e-4 * np.maximum(np.abs(a), 1e-6)), b
        ref_pc = tf.numpy()[keep]
        assert np.abs(r['pc'] - ref_pc).max() <= 1e-3 * np.abs(ref_pc).max(), b
        total += int(keep.sum())
    assert total > 100
