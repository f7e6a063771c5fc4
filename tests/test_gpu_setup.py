"""One-time set-up on the GPU in FP64 (csrc/setup.cu).

* lss_set_templates: a handle whose templates and basis are swapped in sorts
  like a handle created with them: bit-identical scores, and bit-identical
  rounds on a given score field when the created handle's ctc is the FP64
  prepare_matching (oracle) rounded to FP32.
* lss_set_drift_model / lss_set_drift_shift: drift matrices built on the GPU
  give the filtered batch of the oracle's get_drift_matrix.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _setups():
    from livespikesorter_b200 import synth
    a, _ = synth.config(0, duration_s=0.5, seed=21, T=24)
    b, rec = synth.config(0, duration_s=1.0, seed=22, T=24)
    return a, b, rec


def test_swapped_templates_sort_like_created_ones():
    import ks4_oracle as ko
    from livespikesorter_b200.sorter import Sorter, setup_kwargs
    a, b, rec = _setups()
    kwb = setup_kwargs(b) | dict(NT=6000)
    ctc64 = ko.prepare_matching(b.wPCA.double(), b.U.double(), b.nt).float()
    created = Sorter(**(kwb | dict(ctc=ctc64)))
    # the same probe, whitening and filters, created with a's templates
    swapped = Sorter(**(kwb | dict(U=a.U, wPCA=a.wPCA, ctc=a.ctc, iU=a.iU, Ucc=a.Ucc)))
    swapped.set_templates(b.U, b.wPCA)
    rows = rec.raw[6000 - b.nt: 12000 + b.nt]
    X = created.filter(rows, 1, 3)
    assert torch.equal(X, swapped.filter(rows, 1, 3))
    B1, B2 = created.scores(X), swapped.scores(X)
    assert torch.equal(B1, B2)
    st1, a1 = created.match_scores(B1)
    st2, a2 = swapped.match_scores(B1)
    assert len(st1) > 10 and torch.equal(st1, st2) and torch.equal(a1, a2)
    # end to end, PC features included (iU / Ucc rebuilt on the GPU)
    r1, r2 = created.sort_batch(rows, 1, 3), swapped.sort_batch(rows, 1, 3)
    for k in ('time', 'template', 'amplitude', 'pc'):
        assert torch.equal(r1[k], r2[k]), k


def test_gpu_ctc_close_to_reference_fp32():
    from livespikesorter_b200.sorter import Sorter, setup_kwargs
    a, b, rec = _setups()
    # the reference's FP32 ctc (setup.ctc) and the FP64 one differ by rounding:
    # the rounds agree on the spike set
    kwb = setup_kwargs(b) | dict(NT=6000)
    s_ref = Sorter(**kwb)
    s_gpu = Sorter(**(kwb | dict(U=a.U, wPCA=a.wPCA, ctc=a.ctc, iU=a.iU, Ucc=a.Ucc)))
    s_gpu.set_templates(b.U, b.wPCA)
    rows = rec.raw[6000 - b.nt: 12000 + b.nt]
    B = s_ref.scores(s_ref.filter(rows, 1, 3))
    st1, a1 = s_ref.match_scores(B)
    st2, a2 = s_gpu.match_scores(B)
    assert torch.equal(st1, st2)
    assert torch.allclose(a1, a2, rtol=1e-4)


@pytest.mark.parametrize('dshift', [0.0, 7.5, -12.0])
def test_drift_shift_on_gpu_matches_oracle_matrix(dshift):
    import ks4_oracle as ko
    from livespikesorter_b200.sorter import Sorter, setup_kwargs
    _, b, rec = _setups()
    xc, yc = b.probe.xc, b.probe.yc
    M = ko.get_drift_matrix(xc, yc, dshift, ko.inv_kernel(xc, yc, 20), 20).float()
    s1 = Sorter(**(setup_kwargs(b) | dict(NT=6000)))
    s2 = Sorter(**(setup_kwargs(b) | dict(NT=6000)))
    s1.set_drift(M)
    s2.set_drift_model(xc, yc, 20.0)
    s2.set_drift_shift(dshift)
    rows = rec.raw[6000 - b.nt: 12000 + b.nt]
    X1, X2 = s1.filter(rows, 1, 3), s2.filter(rows, 1, 3)
    assert (X1 - X2).abs().max() <= 1e-4 * X1.abs().max()
