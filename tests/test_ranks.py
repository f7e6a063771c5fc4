"""The multi-GPU path is replicas (one sorter per rank, no data-path
collective); its one collective is the step time taken as the maximum over
ranks. Checked with two gloo ranks on the CPU."""
import importlib.util
import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location('bench', ROOT / 'bench.py')
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        b = _bench()
        mine = 10.0 + 7.5 * rank              # this rank's timed region, ms
        q.put((rank, b.max_over_ranks(mine, dist, 'cpu'), b.max_over_ranks(mine, None, 'cpu')))
    finally:
        dist.destroy_process_group()


def test_step_time_is_the_slowest_rank():
    with socket.socket() as sk:
        sk.bind(('127.0.0.1', 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, 17.5, 10.0), (1, 17.5, 17.5)]
