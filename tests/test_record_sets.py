"""Caller-provided record sets for asynchronous batches are checked before
their pointers reach the kernels (a wrong dtype or a short array would be
written past its end). Host logic, no GPU."""
import pytest
import torch

from livespikesorter_b200.sorter import check_record_set


def _set(cap=16, nC=10, K=6, **over):
    o = dict(time=torch.empty(cap, dtype=torch.int64), template=torch.empty(cap, dtype=torch.int32),
             amplitude=torch.empty(cap, dtype=torch.float32), pc=torch.empty((cap, nC, K), dtype=torch.float32),
             count=torch.zeros(1, dtype=torch.int64))
    o.update(over)
    return o


@pytest.mark.parametrize('over, msg', [
    (dict(time=torch.empty(16, dtype=torch.int32)), 'time'),
    (dict(template=torch.empty(16, dtype=torch.int64)), 'template'),
    (dict(amplitude=torch.empty(16, dtype=torch.float64)), 'amplitude'),
    (dict(template=torch.empty(8, dtype=torch.int32)), 'one capacity'),
    (dict(pc=torch.empty((8, 10, 6), dtype=torch.float32)), 'pc'),
    (dict(pc=torch.empty((16, 6, 10), dtype=torch.float32)), 'pc'),
    (dict(count=torch.zeros(0, dtype=torch.int64)), 'count'),
    (dict(time=torch.empty(32, dtype=torch.int64)[::2]), 'time'),
])
def test_malformed_record_sets_are_refused(over, msg):
    with pytest.raises(ValueError, match=msg):
        check_record_set(_set(**over), 10, 6)


def test_pageable_host_record_sets_are_refused():
    # well-formed, but ordinary host memory: the kernels cannot write it
    with pytest.raises(ValueError, match='pinned'):
        check_record_set(_set(), 10, 6)
    with pytest.raises(ValueError, match='pinned'):
        check_record_set(_set(pc=None), 10, 6)


@pytest.mark.gpu
def test_record_sets_on_another_gpu_are_refused():
    # a record set on cuda:0 handed to a sorter said to run on cuda:1: the
    # kernels would write another GPU's memory without peer access
    o = _set(**{k: v.cuda() for k, v in _set().items()})
    check_record_set(o, 10, 6, 'cuda:0')
    with pytest.raises(ValueError, match='sorter runs on cuda:1'):
        check_record_set(o, 10, 6, 'cuda:1')
