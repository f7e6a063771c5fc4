"""Streaming serving loop: several probe streams on one GPU.

``ProbeServer`` wraps ``lss_server_*`` (include/lss.h): each admitted probe
has its own templates, batch length (its block size), CUDA stream, device ring
of raw rows and a CUDA graph that sorts one block end to end; probes' batches
overlap on the device. Admission is by device memory and probe slots: a probe
that does not fit waits until another is released.

``run_streams`` drives probes the way an acquisition system would: each
stream's blocks arrive at real-time instants (block / fs apart, plus seeded
jitter), are pushed as they arrive and their results are polled as they
finish; streams that are not admitted yet wait in a queue and join when a
release frees room (continuous batching). Latency is measured per batch from
the block's scheduled arrival instant to the poll that sees the batch's
completion event.

The reference has no such loop as an API: each probe runs its own
``OnlineSpikesV2`` on a host thread (main.cpp:77-85) whose ``runSpikeSorting``
(OnlineSpikesV2.cu:632-820) sorts the latest window with synchronous copies.
"""
from __future__ import annotations

import ctypes
import gc
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import LSS_ERR_BUSY, LssRecords, check
from .sorter import _f32, _ptr, build_config, post_config

FS = 30000


class ProbeServer:
    """Owns one device; admits, feeds, polls and releases probe streams."""

    def __init__(self, device: int = 0, memory_budget: int = 16 << 30, max_probes: int = 8):
        self._lib = _lib.load()
        self.device = device
        s = ctypes.c_void_p()
        check(self._lib.lss_server_create(device, int(memory_budget), max_probes, ctypes.byref(s)))
        self._s = s
        self._out = {}

    def close(self):
        if getattr(self, '_s', None):
            self._lib.lss_server_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def admit(self, *, depth: int = 4, capacity: int = 8192, drift=None, post: dict | None = None,
              **sorter_kwargs) -> int | None:
        """Admits a probe (``Sorter`` constructor arguments, NT = block size;
        ``post``: ``sorter.post_config`` arguments for positions, clusters and
        duplicate removal). Returns its id, or None when memory or slots are
        not free now."""
        cfg, tens, keep = build_config(device=self.device, **sorter_kwargs)
        M = None if drift is None else _f32(drift)
        pcfg, pkeep = post_config(**post) if post is not None else (None, None)
        pid = ctypes.c_int32(-1)
        rc = self._lib.lss_server_admit(self._s, cfg, tens, _ptr(M), pcfg, depth, capacity, ctypes.byref(pid))
        del keep, pkeep
        if rc == LSS_ERR_BUSY:
            return None
        check(rc)
        K, nC = cfg.n_pcs, cfg.n_nearest
        self._out[pid.value] = dict(
            time=np.empty(capacity, np.int64), tmpl=np.empty(capacity, np.int32),
            amp=np.empty(capacity, np.float32), pc=np.empty((capacity, max(nC, 1), K), np.float32),
            x=np.empty(capacity, np.float32), y=np.empty(capacity, np.float32), clu=np.empty(capacity, np.int32),
            nC=nC, K=K, cap=capacity, Cbin=cfg.n_chan_bin, post=post is not None)
        return pid.value

    def push(self, probe: int, rows: np.ndarray, arrival_ns: int = 0):
        """Appends raw int16 rows ``[n, n_chan_bin]``; arrival_ns on the
        CLOCK_MONOTONIC clock of ``time.perf_counter_ns`` (0 = now)."""
        rows = np.ascontiguousarray(rows, dtype=np.int16)
        if rows.ndim != 2 or rows.shape[1] != self._out[probe]['Cbin']:
            raise ValueError('rows must be int16 [n, n_chan_bin]')
        check(self._lib.lss_server_push(self._s, probe, rows.ctypes.data, rows.shape[0], int(arrival_ns)))

    def poll(self, probe: int, wait: bool = False):
        """``(batch, records)`` of the oldest finished batch, or None."""
        o = self._out[probe]
        rec = LssRecords(time=o['time'].ctypes.data, template_id=o['tmpl'].ctypes.data,
                         amplitude=o['amp'].ctypes.data, pc=o['pc'].ctypes.data if o['nC'] > 0 else None,
                         capacity=o['cap'], count=0, on_device=0,
                         x_pos=o['x'].ctypes.data if o['post'] else None,
                         y_pos=o['y'].ctypes.data if o['post'] else None,
                         cluster=o['clu'].ctypes.data if o['post'] else None)
        b = ctypes.c_int64(-1)
        check(self._lib.lss_server_poll(self._s, probe, rec, ctypes.byref(b), int(wait)))
        if b.value < 0:
            return None
        n = rec.count
        out = dict(time=o['time'][:n].copy(), template=o['tmpl'][:n].copy(), amplitude=o['amp'][:n].copy(),
                   pc=o['pc'][:n].copy() if o['nC'] > 0 else None)
        if o['post']:
            out.update(x=o['x'][:n].copy(), y=o['y'][:n].copy(), cluster=o['clu'][:n].copy())
        return b.value, out

    def release(self, probe: int):
        check(self._lib.lss_server_release(self._s, probe))
        self._out.pop(probe, None)

    def set_drift(self, probe: int, M):
        Mt = _f32(M)
        check(self._lib.lss_server_set_drift(self._s, probe, Mt.data_ptr()))

    def latency(self, probe: int, samples: bool = False) -> dict:
        p50, p99, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        check(self._lib.lss_server_latency(self._s, probe, ctypes.byref(p50), ctypes.byref(p99), ctypes.byref(n)))
        out = dict(p50_ms=p50.value, p99_ms=p99.value, batches=n.value)
        if samples:
            buf = np.zeros(max(n.value, 1), np.float64)
            m = ctypes.c_int64()
            check(self._lib.lss_server_latencies(self._s, probe, buf.ctypes.data, len(buf), ctypes.byref(m)))
            out['samples_ms'] = buf[:m.value].tolist()
            parts = np.zeros((max(n.value, 1), 4), np.float64)
            check(self._lib.lss_server_latency_parts(self._s, probe, parts.ctypes.data, len(parts), ctypes.byref(m)))
            # per batch: arrival -> launch, launch -> device start, device span, device end -> completion seen
            out['parts_ms'] = parts[:m.value].tolist()
        return out

    def memory(self) -> tuple[int, int]:
        u, b = ctypes.c_int64(), ctypes.c_int64()
        check(self._lib.lss_server_memory(self._s, ctypes.byref(u), ctypes.byref(b)))
        return u.value, b.value


@dataclass
class Stream:
    """One probe's input: sorter arguments (NT = block), raw rows, timing."""
    name: str
    sorter_kwargs: dict
    raw: np.ndarray                 # int16 [n_rows, n_chan_bin]
    block: int                      # samples per block (= NT of the probe)
    start_s: float = 0.0            # when the probe asks to join
    n_blocks: int | None = None     # blocks to stream (default: all whole blocks)
    drift: object = None
    depth: int = 4
    capacity: int = 8192
    post: dict | None = None        # sorter.post_config arguments
    # filled by run_streams
    results: dict = field(default_factory=dict)
    latency: dict = field(default_factory=dict)
    admitted_s: float | None = None
    waited: bool = False
    push_late_ms: list = field(default_factory=list)  # realtime: push instant - arrival instant
    started_ns: int | None = None                      # when its blocks began to flow


def arrival_schedule(n_blocks: int, block: int, jitter_frac: float, rng: np.random.Generator) -> np.ndarray:
    """Seconds after the stream's start at which each block has fully arrived:
    the block's nominal end (k + 1) * block / fs plus a seeded delay of up to
    jitter_frac of the block period (kept in order)."""
    period = block / FS
    t = (np.arange(n_blocks) + 1) * period + rng.uniform(0.0, jitter_frac * period, n_blocks)
    return np.maximum.accumulate(t)


def run_streams(server, streams: list[Stream], *, realtime: bool = True, jitter_frac: float = 0.2, seed: int = 0,
                start_together: bool = False, clock=time.perf_counter_ns, sleep=time.sleep) -> dict:
    """Feeds every stream to ``server`` and collects its results.

    realtime: blocks are pushed at their arrival instants (latency is then
    arrival -> emit); otherwise every block is available at once and the loop
    measures the server's capacity (recording-seconds sorted per second).
    Streams whose admission is refused wait and retry after each release.
    start_together: the streams that ask to join at 0 s start streaming once
    all of them are admitted (a rig whose probes are set up before the
    acquisition starts); otherwise each starts as soon as it is admitted,
    while the others' admissions are still running.

    Admissions and releases run on one worker thread, in submission order:
    building a probe (allocations, graph capture) or tearing one down
    (frees, which wait for the device) takes tens to hundreds of ms, and on
    the serving thread that would hold back the pushes of every other stream.
    """
    rng = np.random.default_rng(seed)
    gc_was = gc.isenabled()
    gc.collect()
    gc.disable()  # a collector pause would show up as arrival-to-emit latency
    admin = ThreadPoolExecutor(max_workers=1, thread_name_prefix='lss-admin')
    try:
        return _run_streams(server, streams, realtime, jitter_frac, rng, clock, sleep, admin, start_together)
    finally:
        admin.shutdown(wait=True)
        if gc_was:
            gc.enable()


def _start(parked, active, start_ns, now):
    for pid, (st, sched) in parked.items():
        active[pid] = [st, sched, 0, start_ns]
        st.started_ns = now
    parked.clear()


def _run_streams(server, streams, realtime, jitter_frac, rng, clock, sleep, admin, start_together):
    t0 = clock()
    held = [st for st in streams if st.start_s <= 0] if start_together else []
    parked = {}        # probe id -> stream, admitted and waiting for the others in `held`
    order = {id(st): i for i, st in enumerate(sorted(streams, key=lambda s: s.start_s))}
    waiting = sorted(streams, key=lambda s: order[id(s)])
    active = {}        # probe id -> [stream, schedule, next block index, stream start ns]
    admitting = {}     # future -> (stream, releases completed when it was submitted)
    releasing = []     # futures
    done = []
    samples = 0
    releases = 0       # a refused stream retries only after a release
    refused_at = {}
    while waiting or active or admitting or releasing or parked:
        progressed = False
        # finished admissions and releases
        for f in [f for f in releasing if f.done()]:
            releasing.remove(f)
            f.result()
            releases += 1
            progressed = True
        for f in [f for f in admitting if f.done()]:
            st, rel0 = admitting.pop(f)
            pid = f.result()
            progressed = True
            is_held = any(h is st for h in held)
            if pid is None:
                st.waited = True
                refused_at[id(st)] = rel0
                waiting = sorted(waiting + [st], key=lambda s: order[id(s)])  # keeps its place
                if is_held:  # not all of them fit: the admitted ones start now
                    held = []
                    _start(parked, active, clock() if realtime else t0, clock())
                continue
            nb = st.n_blocks if st.n_blocks is not None else st.raw.shape[0] // st.block
            sched = arrival_schedule(nb, st.block, jitter_frac, rng) if realtime else np.zeros(nb)
            st.admitted_s = (clock() - t0) * 1e-9
            if is_held:
                parked[pid] = (st, sched)
                if len(parked) == len(held):
                    held = []
                    _start(parked, active, clock() if realtime else t0, clock())
                continue
            # a stream's clock starts once its probe is built
            st.started_ns = clock()
            active[pid] = [st, sched, 0, st.started_ns if realtime else t0]
        # admission requests (in request order)
        now = clock()
        still = []
        for st in waiting:
            if (now - t0) * 1e-9 < st.start_s or refused_at.get(id(st)) == releases:
                still.append(st)
                continue
            f = admin.submit(server.admit, depth=st.depth, capacity=st.capacity, drift=st.drift, post=st.post,
                             **st.sorter_kwargs)
            admitting[f] = (st, releases)
        waiting = still
        # pushes of blocks that have arrived
        next_due = None
        for pid, a in active.items():
            st, sched, k, start_ns = a
            while k < len(sched):
                due = start_ns + int(sched[k] * 1e9)
                if realtime:
                    now = clock()
                    if now < due:
                        next_due = due if next_due is None else min(next_due, due)
                        break
                    st.push_late_ms.append((now - due) * 1e-6)
                rows = st.raw[k * st.block:(k + 1) * st.block]
                server.push(pid, rows, due if realtime else 0)
                k += 1
                progressed = True
                if not realtime:
                    break  # interleave the streams' blocks
            a[2] = k
        # results
        for pid, a in list(active.items()):
            st, sched, k, _ = a
            while True:
                r = server.poll(pid, wait=False)
                if r is None:
                    break
                st.results[r[0]] = r[1]
                samples += st.block
                progressed = True
            if k == len(sched) and len(st.results) == len(sched):
                st.latency = server.latency(pid, samples=True)
                del active[pid]
                releasing.append(admin.submit(server.release, pid))
                done.append(st)
                progressed = True
        if not progressed:
            if realtime and next_due is not None:
                gap = (next_due - clock()) * 1e-9
                if gap > 3e-4:
                    # short naps: results are seen by polling, so the nap bounds their delay
                    sleep(min(gap - 2e-4, 2e-4))
            else:
                sleep(2e-5)
    end = clock()
    wall = (end - t0) * 1e-9
    first = min((st.started_ns for st in done if st.started_ns is not None), default=end)
    span = (end - first) * 1e-9
    # rec_s_per_s counts the admissions' time too; rec_s_per_s_streaming starts
    # at the first stream's start
    return dict(wall_s=wall, rec_s=samples / FS, rec_s_per_s=samples / FS / wall if wall > 0 else 0.0,
                rec_s_per_s_streaming=samples / FS / span if span > 0 else 0.0, streams=done)
