"""Pipelined submission (lss_sort_batch_async + lss_sync): batches enqueued
back to back, with a drift change before each, give the records of the
synchronous lss_sort_batch, bit for bit."""
import numpy as np
import pytest
import torch

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def test_async_batches_equal_sync_batches():
    from livespikesorter_b200.sorter import Sorter
    g = np.load(GOLDEN / 'ks4_extract_c16_t8_drift.npz')
    C, T, NT, nt, nt0min, nC, K, nb = [int(v) for v in g['params']]
    kw = dict(U=g['U'], wPCA=g['wPCA'], ctc=g['ctc'], Wrot=g['Wrot'], hp_filter=g['hp_filter'], iCC=g['iCC'],
              iU=g['iU'], Ucc=g['Ucc'], NT=NT, nt0min=nt0min, Th=float(g['Th']))
    raw = g['raw']
    nbt = int(np.ceil(raw.shape[0] / NT))
    rows = [raw[0:NT + nt] if ib == 0 else raw[ib * NT - nt:min(raw.shape[0], ib * NT + NT + nt)] for ib in range(nbt)]
    sync = Sorter(**kw)
    want = []
    for ib in range(nbt):
        sync.set_drift(g['drift_M'][ib])
        want.append(sync.sort_batch(torch.from_numpy(rows[ib]).cuda(), ib, nbt, on_device=True))
    asy = Sorter(**kw)
    got = []
    for rep in range(2):  # twice in a row, nothing waited for in between
        for ib in range(nbt):
            asy.set_drift(g['drift_M'][ib])
            got.append(asy.sort_batch_async(torch.from_numpy(rows[ib]).cuda(), ib, nbt))
    asy.sync()
    for k, r in enumerate(got):
        w = want[k % nbt]
        n = int(r['count'].item())
        assert n == len(w['time']) and n > 0
        for key in ('time', 'template', 'amplitude', 'pc'):
            assert torch.equal(r[key][:n], w[key]), key


def test_async_batches_from_host_rows_into_pinned_records():
    """Host rows upload on the handle's upload stream into two alternating
    device buffers under the previous batch's work; records land in pinned
    host memory. Same records as the synchronous call."""
    from livespikesorter_b200.sorter import Sorter
    g = np.load(GOLDEN / 'ks4_extract_c16_t8_drift.npz')
    C, T, NT, nt, nt0min, nC, K, nb = [int(v) for v in g['params']]
    kw = dict(U=g['U'], wPCA=g['wPCA'], ctc=g['ctc'], Wrot=g['Wrot'], hp_filter=g['hp_filter'], iCC=g['iCC'],
              iU=g['iU'], Ucc=g['Ucc'], NT=NT, nt0min=nt0min, Th=float(g['Th']))
    raw = g['raw']
    nbt = int(np.ceil(raw.shape[0] / NT))
    rows = [torch.from_numpy(np.ascontiguousarray(raw[0:NT + nt] if ib == 0 else
                                                  raw[ib * NT - nt:min(raw.shape[0], ib * NT + NT + nt)])).pin_memory()
            for ib in range(nbt)]
    sync = Sorter(**kw)
    want = []
    for ib in range(nbt):
        sync.set_drift(g['drift_M'][ib])
        want.append(sync.sort_batch(rows[ib].numpy(), ib, nbt))
    asy = Sorter(**kw)
    got = []
    for rep in range(3):  # more batches than upload buffers, nothing waited for in between
        for ib in range(nbt):
            asy.set_drift(g['drift_M'][ib])
            got.append(asy.sort_batch_async(rows[ib], ib, nbt, out=asy.records(4096, pinned=True)))
    asy.sync()
    for k, r in enumerate(got):
        w = want[k % nbt]
        n = int(r['count'].item())
        assert not r['time'].is_cuda
        assert n == len(w['time']) and n > 0
        for key in ('time', 'template', 'amplitude', 'pc'):
            assert torch.equal(r[key][:n], w[key]), key
