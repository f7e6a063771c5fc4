"""Host logic of the streaming loop (serve.run_streams) against a fake server:
admissions and releases on the worker thread, refusal and retry after a
release, start_together, and the bookkeeping of pushes and results. No GPU.
"""
import threading

import numpy as np

from livespikesorter_b200.serve import Stream, run_streams


class FakeServer:
    """Admits while the summed probe sizes fit the budget; a pushed block is
    finished at once. Records which thread made each call."""

    def __init__(self, budget, sizes):
        self.budget, self.sizes, self.used = budget, sizes, 0
        self.probes, self.next_id, self.log = {}, 0, []
        self.lock = threading.Lock()

    def admit(self, *, depth, capacity, drift, post, name):
        with self.lock:
            self.log.append(('admit', name, threading.current_thread().name))
            if self.used + self.sizes[name] > self.budget:
                return None
            pid = self.next_id
            self.next_id += 1
            self.used += self.sizes[name]
            self.probes[pid] = dict(name=name, pushed=0, polled=0)
            return pid

    def push(self, pid, rows, arrival_ns):
        self.log.append(('push', self.probes[pid]['name'], threading.current_thread().name))
        self.probes[pid]['pushed'] += 1

    def poll(self, pid, wait=False):
        p = self.probes[pid]
        if p['polled'] == p['pushed']:
            return None
        b = p['polled']
        p['polled'] += 1
        return b, dict(time=np.arange(3) + 100 * b)

    def latency(self, pid, samples=False):
        n = self.probes[pid]['polled']
        return dict(p50_ms=1.0, p99_ms=1.0, batches=n, samples_ms=[1.0] * n, parts_ms=[[0.25] * 4] * n)

    def release(self, pid):
        with self.lock:
            p = self.probes.pop(pid)
            self.used -= self.sizes[p['name']]
            self.log.append(('release', p['name'], threading.current_thread().name))


def _stream(name, n_blocks, start_s=0.0, block=30):
    raw = np.zeros((n_blocks * block, 4), np.int16)
    return Stream(name, dict(name=name), raw, block, start_s=start_s)


def test_admissions_and_releases_run_off_the_serving_thread():
    srv = FakeServer(100, dict(A=40, B=40, C=40))
    streams = [_stream('A', 5), _stream('B', 3), _stream('C', 4)]
    out = run_streams(srv, streams, realtime=False)
    by = {st.name: st for st in out['streams']}
    # C did not fit beside A and B; it joined after the first release
    assert by['C'].waited and not by['A'].waited and not by['B'].waited
    for name, n in (('A', 5), ('B', 3), ('C', 4)):
        assert sorted(by[name].results) == list(range(n))
        assert by[name].latency['batches'] == n
    main = threading.current_thread().name
    assert all(t != main for kind, _, t in srv.log if kind in ('admit', 'release'))
    assert all(t == main for kind, _, t in srv.log if kind == 'push')
    first_release = next(i for i, e in enumerate(srv.log) if e[0] == 'release')
    c_admits = [i for i, e in enumerate(srv.log) if e[:2] == ('admit', 'C')]
    assert len(c_admits) == 2 and c_admits[0] < first_release < c_admits[1]
    assert srv.used == 0 and out['rec_s'] == 12 * 30 / 30000


def test_start_together_holds_the_first_streams_until_all_are_admitted():
    srv = FakeServer(100, dict(A=30, B=30, C=30))
    streams = [_stream('A', 4), _stream('B', 4), _stream('C', 4)]
    run_streams(srv, streams, realtime=False, start_together=True)
    last_admit = max(i for i, e in enumerate(srv.log) if e[0] == 'admit')
    first_push = min(i for i, e in enumerate(srv.log) if e[0] == 'push')
    assert last_admit < first_push
    assert len({st.started_ns for st in streams}) == 1


def test_start_together_does_not_wait_for_a_refused_stream():
    srv = FakeServer(70, dict(A=30, B=30, C=30))
    streams = [_stream('A', 3), _stream('B', 3), _stream('C', 3)]
    out = run_streams(srv, streams, realtime=False, start_together=True)
    by = {st.name: st for st in out['streams']}
    assert by['C'].waited and sorted(by['C'].results) == [0, 1, 2]
    assert sorted(by['A'].results) == [0, 1, 2] and sorted(by['B'].results) == [0, 1, 2]


def test_realtime_pushes_wait_for_arrival():
    srv = FakeServer(100, dict(A=10))
    st = _stream('A', 6, block=300)  # 10 ms blocks
    out = run_streams(srv, [st], realtime=True, jitter_frac=0.0)
    assert sorted(st.results) == list(range(6))
    assert len(st.push_late_ms) == 6 and min(st.push_late_ms) >= 0
    assert out['wall_s'] >= 0.06
