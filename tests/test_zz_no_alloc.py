"""The allocation-free rounds entry point (lss_mp_rounds_noalloc).

It exists for callers that cannot allocate device memory while they run (for
instance a plugin inside an acquisition program that owns the GPU's memory, or
a real-time loop that must not pay for cudaMalloc). This file is named so that
pytest collects it last. It checks the entry point through the C ABI against
the handle-based entry point (lss_match_scores) on two calls in a row, since
the calls share one fixed scratch array whose contents persist between them.
"""
import ctypes

import numpy as np
import pytest
import torch

import ks4_oracle as ko
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

AMP_RTOL = 1e-4


def _call(lib, B, T, nt, th, nm_d, ctcP_d, cap=100000, max_rounds=100):
    x = torch.full((cap,), -1, dtype=torch.int32, device='cuda')
    y = torch.full((cap,), -1, dtype=torch.int32, device='cuda')
    a = torch.zeros(cap, dtype=torch.float32, device='cuda')
    n, r = ctypes.c_int32(-1), ctypes.c_int32(-1)
    rc = lib.lss_mp_rounds_noalloc(B.data_ptr(), B.shape[1], T, B.shape[1], nt, th, nm_d.data_ptr(),
                                   ctcP_d.data_ptr(), max_rounds, cap, x.data_ptr(), y.data_ptr(), a.data_ptr(),
                                   ctypes.byref(n), ctypes.byref(r), torch.cuda.current_stream().cuda_stream)
    return rc, x[:max(n.value, 0)], y[:max(n.value, 0)], a[:max(n.value, 0)], r.value


def test_no_alloc_rounds_match_the_handle_entry_point():
    from livespikesorter_b200 import _lib
    from livespikesorter_b200.sorter import Sorter
    lib = _lib.load()
    g = np.load(GOLDEN / 'ks4_extract_c32_t12.npz')
    C, T, NT, nt, nt0min, nC, K, nb = [int(v) for v in g['params']]
    th = float(g['Th'])
    U = torch.from_numpy(g['U'])
    wPCA = torch.from_numpy(g['wPCA'])
    ctc = torch.from_numpy(g['ctc'])
    nm = (U ** 2).sum(-1).sum(-1)
    s = Sorter(U=U, wPCA=wPCA, ctc=ctc, Wrot=np.eye(C, dtype=np.float32), NT=NT, Th=th, nm=nm)
    nm_d = nm.cuda()
    ctcP_d = ctc.permute(1, 0, 2).contiguous().cuda()
    # two calls in a row on different batches: nothing from the first call may
    # leak into the second through the shared scratch
    for ib in (1, 2):
        B = ko.score_field(torch.from_numpy(g[f'X_{ib}']), U, wPCA, nt).cuda()
        st_ref, amps_ref = s.match_scores(B)
        rc, x, y, a, rounds = _call(lib, B.clone(), T, nt, th, nm_d, ctcP_d)
        assert rc == 0, lib.lss_last_error(None)
        assert len(x) == len(st_ref) > 0
        assert torch.equal(x.long().cpu(), st_ref[:, 0].cpu())
        assert torch.equal(y.long().cpu(), st_ref[:, 1].cpu())
        ref = amps_ref[:, 0].cpu().double()
        assert torch.all((a.cpu().double() - ref).abs() <= AMP_RTOL * ref.abs().clamp_min(1e-6))
        assert rounds == s.stats()['rounds']


def test_no_alloc_rejects_oversized_batches():
    from livespikesorter_b200 import _lib
    from livespikesorter_b200._lib import LSS_ERR_ARG
    lib = _lib.load()
    dummy = torch.zeros(4, device='cuda')
    n, r = ctypes.c_int32(), ctypes.c_int32()
    p = dummy.data_ptr()
    rc = lib.lss_mp_rounds_noalloc(p, 70000, 2, 70000, 61, 8.0, p, p, 100, 10, p, p, p,
                                   ctypes.byref(n), ctypes.byref(r), None)
    assert rc == LSS_ERR_ARG
    assert b'LSS_NOALLOC_MAX_SAMPLES' in lib.lss_last_error(None)


def test_no_alloc_refuses_pageable_host_arrays():
    """A pageable host array passed as the score field is refused with
    LSS_ERR_ARG before anything is launched (it would fault in the kernel)."""
    from livespikesorter_b200 import _lib
    from livespikesorter_b200._lib import LSS_ERR_ARG
    lib = _lib.load()
    T, nt, N = 2, 61, 1000
    host_B = np.zeros((T, N), np.float32)
    dev = torch.zeros(T * T * (2 * nt + 1) + N, device='cuda')
    outs = [torch.zeros(16, dtype=torch.int32, device='cuda') for _ in range(2)] + [torch.zeros(16, device='cuda')]
    n, r = ctypes.c_int32(-7), ctypes.c_int32(-7)
    rc = lib.lss_mp_rounds_noalloc(host_B.ctypes.data, N, T, N, nt, 8.0, dev.data_ptr(), dev.data_ptr(), 100, 16,
                                   *(o.data_ptr() for o in outs), ctypes.byref(n), ctypes.byref(r), None)
    torch.cuda.synchronize()
    assert rc == LSS_ERR_ARG
    assert b'current device' in lib.lss_last_error(None)
    assert n.value == -7 and r.value == -7
