"""Benchmark of the per-batch sorting hot path on B200.

Workload (one step = one padded 60000-sample batch through the whole path:
int16 ingest, highpass, whitening + drift, score GEMM, matching pursuit, PC
features, records): 384-channel staggered probe, 800 templates of which 10 %
are near-duplicate pairs (footprint centres 10 um apart), NT = 60000, linear
drift of 5 um/min, BF16 score GEMM with FP32 re-check of near decisions.
Synthetic, seeded recording (no public dataset exists for this path). Metric:
recording-seconds sorted per second. The same line carries the FP32 path's
rate on the same batches, the BF16 path's spike agreement with it, the BF16
score error against an FP64 score field, and the FP32 path on the
400-template workload without near-duplicates.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
    python bench.py --templates 400 --precision fp32      # 400 templates, FP32 path
    python bench.py --workload serving [--duration S]

The serving workload runs four independent 384-channel probes (200, 400,
600 and 800 templates) fed as real-time 30 kHz streams in blocks of 3000,
1500, 600 and 300 samples (100 ms down to 10 ms) with seeded arrival jitter
through the streaming loop, and reports per-probe p50/p99 arrival-to-emit
latency and the loop's capacity (all blocks available at once).

N > 1 runs one independent replica per GPU (the path has no exchange step);
value = total recording-seconds of all ranks / max over ranks of device time.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FS = 30000.0
METRIC = 'rec-sec sorted/sec & p99 latency, 384ch; BF16 vs FP32 at >=0.99 spike agreement'
N_BATCH_POOL = 6   # distinct device-resident batches the steps rotate over (276 MB int16 > L2)
E2E_RING = 4       # pinned host record sets of the pipelined end-to-end steps


def parse():
    p = argparse.ArgumentParser()
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=20)
    p.add_argument('--warmup', type=int, default=3)
    p.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    p.add_argument('--templates', type=int, default=800,
                   help='800: templates with 10%% near-duplicate pairs; other counts: no duplicates')
    p.add_argument('--precision', default='bf16', choices=['fp32', 'bf16'])
    p.add_argument('--no-extras', action='store_true', help='skip the FP32 / 400-template / FP64 extras')
    p.add_argument('--no-cpu-baseline', action='store_true')
    p.add_argument('--workload', default='batch', choices=['batch', 'serving', 'refine'])
    p.add_argument('--refine-steps', type=int, default=10)
    p.add_argument('--duration', type=float, default=3.0, help='serving: seconds of recording per probe')
    return p.parse_args()


def workload(T, rank):
    """800 templates: 10 % near-duplicate pairs (the headline workload); any
    other count: the same generator without duplicates. Both drift 5 um/min."""
    from livespikesorter_b200 import synth
    cfg = 2 if T == 800 else 1
    setup, rec = synth.config(cfg, duration_s=(N_BATCH_POOL + 2) * 2.0, seed=17 + rank, T=T)
    return setup, rec


def batch_rows(rec, setup, ib):
    NT, nt = setup.NT, setup.nt
    b0 = ib * NT - nt
    return np.ascontiguousarray(rec.raw[b0:b0 + NT + 2 * nt])


def workload_desc(T, precision):
    dup = ' (10% near-duplicate pairs, centres 10 um apart)' if T == 800 else ''
    path = 'BF16 score GEMM + FP32 re-check' if precision == 'bf16' else 'FP32 (3xTF32 tensor-core) score GEMM'
    return {'workload': f'384-ch staggered probe, {T} templates{dup}, NT=60000 int16 batches (+-61 context), '
                        f'drift 5 um/min, highpass+whitening+drift, score GEMM, matching pursuit, PC features; '
                        f'{path}',
            'channels': 384, 'templates': T, 'batch_samples': 60000, 'nt': 61, 'n_pcs': 6,
            'nearest_chans': 10, 'precision': precision,
            'l2': f'steps rotate over {N_BATCH_POOL} device-resident batches (276 MB int16) and each step '
                  'streams >1 GB of intermediates, both larger than the 126 MB L2'}


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index, period_ms=200):
        self.index = index
        self.period_ms = period_ms
        self.proc = None
        self.path = Path(tempfile.gettempdir()) / f'lss_clocks_{os.getpid()}.csv'

    def __enter__(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
            q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
                 'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
                 'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')
            self.f = open(self.path, 'w')
            self.proc = subprocess.Popen(['nvidia-smi', f'--id={self.index}', f'--query-gpu={q}',
                                          '--format=csv,noheader,nounits', '-lms', str(self.period_ms)],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            # the sampler's start-up (NVML initialisation) must not fall into
            # the timed region: wait for its first sample
            t0 = time.time()
            while time.time() - t0 < 5.0 and self.proc.poll() is None:
                self.f.flush()
                if self.path.exists() and self.path.stat().st_size > 0:
                    break
                time.sleep(0.02)
            time.sleep(0.2)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        if not self.proc or not self.path.exists():
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unsampled']}
        rows = [l.split(',') for l in self.path.read_text().strip().splitlines() if l.count(',') >= 8]
        if not rows:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unsampled']}
        sm = [float(r[1]) for r in rows]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if 'Active' in v and 'Not' not in v})
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': float(rows[0][2]), 'reasons': reasons,
                'samples': len(rows)}


def algorithmic_work(setup, spikes_per_batch, T):
    """Per-batch algorithmic FLOPs and bytes (the per-unit formulas of the
    design notes, times one batch)."""
    C, K, nt = setup.C, setup.K, setup.nt
    N = setup.NT + 2 * nt
    L2 = 2 * nt + 1
    gemm_flops = 2.0 * T * C * K * N
    mp_bytes = 4.0 * T * N + spikes_per_batch * 12.0 * T * L2
    return gemm_flops, mp_bytes


def run_b200(args):
    from livespikesorter_b200.sorter import Sorter
    rank = int(os.environ.get('RANK', 0))
    world = int(os.environ.get('WORLD_SIZE', 1))
    local = int(os.environ.get('LOCAL_RANK', 0))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=300))
    T = args.templates
    setup, rec = workload(T, rank)
    s = Sorter.from_setup(setup, device=local, precision=args.precision)
    s.set_profiling(True)
    ids = list(range(1, N_BATCH_POOL + 1))
    rows_h = [torch.from_numpy(batch_rows(rec, setup, ib)).pin_memory() for ib in ids]
    rows_d = [r.cuda(local) for r in rows_h]
    drifts = [setup.drift_matrix(rec.dshift[ib]) for ib in ids]
    nb = rec.n_batches
    stream = torch.cuda.current_stream(local)

    def step(i, host):
        j = i % len(ids)
        s.set_drift(drifts[j])
        return s.sort_batch(rows_h[j] if host else rows_d[j], ids[j], nb, on_device=not host)

    def step_async(i, out):
        j = i % len(ids)
        s.set_drift(drifts[j])
        return s.sort_batch_async(rows_d[j], ids[j], nb, out=out)

    ring = [s.records(32768, pinned=True) for _ in range(E2E_RING)]

    def timed_e2e(K, W):
        """End to end from pinned host memory through the pipelined calls: each
        step sets the drift matrix and submits a batch of host rows
        (lss_sort_batch_async uploads them under the previous batch's work) whose
        records land in one of E2E_RING pinned host record sets; before a set is
        reused, the host waits for its batch and reads its records."""
        seen = []

        def consume(r):
            n = int(r['count'][0])
            if n > r['time'].shape[0]:
                raise RuntimeError('record ring capacity exceeded')
            seen.append((n, int(r['time'][:n].sum()), float(r['amplitude'][:n].sum())))

        for i in range(W):
            step_host_async(i, ring[i % E2E_RING])
        s.sync()
        gc.collect()
        gc.disable()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(K + 1)]
        ev[0].record(stream)
        for i in range(K):
            if i >= E2E_RING:
                ev[i - E2E_RING + 1].synchronize()
                consume(ring[i % E2E_RING])
            step_host_async(i, ring[i % E2E_RING])
            ev[i + 1].record(stream)
        s.sync()
        for i in range(max(0, K - E2E_RING), K):
            consume(ring[i % E2E_RING])
        ev[K].synchronize()
        gc.enable()
        per = np.array([ev[i].elapsed_time(ev[i + 1]) for i in range(K)])
        tot = float(ev[0].elapsed_time(ev[K]))
        tot = max_over_ranks(tot, dist, f'cuda:{local}')
        return tot, per, seen

    def step_host_async(i, out):
        j = i % len(ids)
        s.set_drift(drifts[j])
        return s.sort_batch_async(rows_h[j], ids[j], nb, out=out)

    def profiled(K):
        """Per-stage device times, spikes and rounds of K synchronous batches
        (untimed: the stage events serialise the host and the device)."""
        s.set_profiling(True)
        stages, spikes, rounds = [], [], []
        for i in range(K):
            r = step(i, False)
            stages.append(s.stage_times())
            spikes.append(len(r['time']))
            rounds.append(s.stats()['rounds'])
        s.set_profiling(False)
        return stages, spikes, rounds

    def timed(K, W, host):
        """Device-resident steps are submitted back to back (lss_sort_batch_async,
        one host wait at the end); host-buffer steps go through lss_sort_batch
        with its host copies and wait."""
        # device record sets of every timed step, allocated before the timed
        # region (the results stay valid until the final sync)
        outs = [] if host else [s.records() for _ in range(max(K, W))]
        for i in range(W):
            if host:
                step(i, host)
            else:
                step_async(i, outs[i])
        if not host:
            s.sync()
        gc.collect()
        gc.disable()  # no collector pauses inside the timed region
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(K + 1)]
        launches0 = s.stats()['launches']
        ev[0].record(stream)
        for i in range(K):
            if host:
                step(i, host)
            else:
                step_async(i, outs[i])
            ev[i + 1].record(stream)
        if not host:
            s.sync()
        torch.cuda.synchronize()
        gc.enable()
        del outs
        per = np.array([ev[i].elapsed_time(ev[i + 1]) for i in range(K)])
        tot = float(ev[0].elapsed_time(ev[K]))
        tot = max_over_ranks(tot, dist, f'cuda:{local}')
        return tot, per, s.stats()['launches'] - launches0

    K, W = args.steps, max(3, args.warmup)
    s.set_profiling(False)
    with Clocks(local) as clk:
        tot, per, launches = timed(K, W, host=False)
    clocks = clk.summary()
    tot_h, per_h, seen = timed_e2e(K, W)
    tot_s, per_s, _ = timed(K, W, host=True)
    stages, spikes, rounds = profiled(min(K, 2 * len(ids)))
    phases = s.stats()['mp_phases_ms']
    rec_s = setup.NT / FS
    value = world * K * rec_s / (tot / 1e3)
    e2e = world * K * rec_s / (tot_h / 1e3)
    e2e_sync = world * K * rec_s / (tot_s / 1e3)
    # the pipelined steps read back as many records per batch as the synchronous calls
    by_batch = {i % len(ids): n for i, n in enumerate(spikes)}
    if any(n != by_batch[i % len(ids)] for i, (n, _, _) in enumerate(seen)):
        raise RuntimeError('pipelined end-to-end steps returned other spike counts than the synchronous calls')
    # roofline of the dominant kernel, from the device-resident timed steps
    mean_st = {k: float(np.mean([st[k] for st in stages])) for k in stages[0]}
    kern = {k: v for k, v in mean_st.items() if k not in ('total_ms', 'h2d_ms', 'records_ms')}
    top = max(kern, key=kern.get)
    gemm_flops, mp_bytes = algorithmic_work(setup, float(np.mean(spikes)), T)
    peaks = json.loads((ROOT / 'MEASURED_PEAKS.json').read_text()) if (ROOT / 'MEASURED_PEAKS.json').exists() else {}
    hbm = peaks.get('hbm_gbs', 6650.0)
    tfl = peaks.get('bf16_tflops', 1590.0)
    src = 'measured' if peaks else 'fallback'
    if top == 'mp_ms':
        ach = mp_bytes / (mean_st['mp_ms'] / 1e3) / 1e9
        # the rounds kernel this handle runs (block-skipping from 600 templates)
        kname, prof = (('k_mp_blocks (matching pursuit, block-skipping)', f'k_mp_blocks_384ch_{T}t.md')
                       if s.round_kernel() else ('k_mp (matching pursuit)', f'k_mp_384ch_{T}t.md'))
        roof = {'kernel': kname, 'bound': 'hbm', 'achieved': ach, 'peak': hbm, 'unit': 'GB/s',
                'frac': ach / hbm, 'traffic': profile_traffic(prof),
                'traffic_source': 'ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of this workload '
                                  f'(profiles/{prof})',
                'algorithmic_bytes': mp_bytes, 'peak_source': src,
                'note': 'achieved counts the algorithmic bytes of every row update; the block-skipping kernel '
                        'proves most of them no-ops and moves only `traffic`'}
    else:
        ach = gemm_flops / (mean_st['score_ms'] / 1e3) / 1e12
        roof = {'kernel': 'k_score_tc (tcgen05 3xTF32 score GEMM)' if args.precision == 'fp32'
                else 'k_score_tc (tcgen05 BF16 score GEMM)',
                'bound': 'tensor', 'achieved': ach, 'peak': tfl, 'unit': 'TFLOP/s', 'frac': ach / tfl,
                'traffic': None, 'peak_source': src, 'top_stage': top}
    h2d = int(rows_h[0].numel() * 2 + setup.C * setup.C * 4)
    d2h = int(np.mean(spikes) * (8 + 4 + 4 + setup.nC * setup.K * 4) + 16)
    out = {
        'metric': METRIC, 'value': value, 'unit': 'rec-s/s', 'n_gpus': world, 'steps': K, 'warmup': W,
        'ms_per_step': tot / K, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f32' if args.precision == 'fp32' else 'bf16+f32', 'data': 'synthetic',
        'config': workload_desc(T, args.precision) | {'parallelism': f'replicas x{world}'},
        'e2e': {'value': e2e, 'unit': 'rec-s/s', 'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h,
                'api': f'lss_set_drift + lss_sort_batch_async per step, rows from pinned host memory, records into '
                       f'a ring of {E2E_RING} pinned host record sets read back before reuse, lss_sync at the end',
                'step_ms_p50': float(np.percentile(per_h, 50)), 'step_ms_p99': float(np.percentile(per_h, 99))},
        'e2e_sync': {'value': e2e_sync, 'unit': 'rec-s/s', 'api': 'lss_set_drift + lss_sort_batch per step (host '
                     'rows in, host records out, returns when the batch is done)',
                     'latency_ms_p50': float(np.percentile(per_s, 50)),
                     'latency_ms_p99': float(np.percentile(per_s, 99))},
        'latency_ms_p50': float(np.percentile(per, 50)), 'latency_ms_p99': float(np.percentile(per, 99)),
        'roofline': roof, 'roofline_path': path_roofline(setup, float(np.mean(spikes)), T, value / world, hbm, tfl, src),
        'gpu_launches': int(launches), 'clocks': clocks,
        'stage_ms': mean_st, 'mp_phases_ms': phases,
        'spikes_per_batch': float(np.mean(spikes)), 'rounds_per_batch': float(np.mean(rounds)),
        'step_ms': [round(float(v), 3) for v in per],
    }
    if not args.no_extras:
        # the FP32 path on the same batches, and the BF16 path's agreement with it
        s32 = s if args.precision == 'fp32' else Sorter.from_setup(setup, device=local)
        if s32 is not s:
            t32, st32 = device_resident_rate(s32, rows_d, drifts, ids, nb, K, W, stream, dist, local)
            out['fp32_path'] = {'value': world * K * rec_s / (t32 / 1e3), 'unit': 'rec-s/s',
                                'ms_per_step': t32 / K, 'stage_ms': st32,
                                'api': 'lss_set_drift + lss_sort_batch_async, device-resident rows, same batches'}
        # the two rounds kernels on the same batches (identical results): every
        # row updated, or provably unchanged template-row blocks skipped
        kernels = {}
        default_skip = s32.round_kernel()
        for skip in (False, True):
            s32.set_round_kernel(skip)
            tk, stk = device_resident_rate(s32, rows_d, drifts, ids, nb, K, W, stream, dist, local)
            st_k = s32.stats()
            kernels['skip_blocks' if skip else 'full'] = {
                'rec_s_per_s': world * K * rec_s / (tk / 1e3), 'mp_ms': stk['mp_ms'], 'phases_ms': stk['mp_phases_ms'],
                'update_items': st_k['mp_items'], 'update_items_changed': st_k['mp_items_updated']}
        s32.set_round_kernel(default_skip)
        out['round_kernels_fp32'] = kernels
        if args.precision == 'bf16':
            out['bf16'] = bf16_report(s, s32, rows_d, drifts, ids, nb)
            out['bf16']['score_err_fp64'] = fp64_score_error(s, s32, setup, rows_d[0], drifts[0], ids[0], nb)
        if T != 400:
            # the 400-template workload without near-duplicates, FP32 path
            setup4, rec4 = workload(400, rank)
            s4 = Sorter.from_setup(setup4, device=local)
            rows4 = [torch.from_numpy(batch_rows(rec4, setup4, ib)).cuda(local) for ib in ids]
            dr4 = [setup4.drift_matrix(rec4.dshift[ib]) for ib in ids]
            t4, st4 = device_resident_rate(s4, rows4, dr4, ids, rec4.n_batches, K, W, stream, dist, local)
            out['t400_fp32'] = {'value': world * K * rec_s / (t4 / 1e3), 'unit': 'rec-s/s', 'ms_per_step': t4 / K,
                                'stage_ms': st4, 'config': workload_desc(400, 'fp32')}
            del s4, rows4
        # the streaming loop: 4 probes, 3 s of real-time arrival each
        sv = serving_report(local, rank, 3.0, 3)
        out['serving'] = {k: sv[k] for k in ('metric', 'value', 'unit', 'latency_ms', 'realtime_rec_s_per_s',
                                             'capacity_rec_s_per_s', 'clocks', 'config')}
    if rank == 0 and not args.no_cpu_baseline:
        out['cpu_baseline'] = cpu_baseline(setup, rec)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


def device_resident_rate(s, rows_d, drifts, ids, nb, K, W, stream, dist, local):
    """rec-s/s of K batches submitted back to back from device-resident rows
    (lss_set_drift + lss_sort_batch_async, one host wait at the end), after W
    warm-up batches; also the mean per-stage device times of two profiled
    synchronous batches."""
    outs = [s.records() for _ in range(max(K, W))]
    for i in range(W):
        j = i % len(ids)
        s.set_drift(drifts[j])
        s.sort_batch_async(rows_d[j], ids[j], nb, out=outs[i])
    s.sync()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(K):
        j = i % len(ids)
        s.set_drift(drifts[j])
        s.sort_batch_async(rows_d[j], ids[j], nb, out=outs[i])
    e1.record(stream)
    s.sync()
    torch.cuda.synchronize()
    tot = max_over_ranks(float(e0.elapsed_time(e1)), dist, f'cuda:{local}')
    s.set_profiling(True)
    st, ph = [], []
    for i in range(2):
        s.set_drift(drifts[i % len(ids)])
        s.sort_batch(rows_d[i % len(ids)], ids[i % len(ids)], nb, on_device=True)
        st.append(s.stage_times())
        ph.append(s.stats()['mp_phases_ms'])
    s.set_profiling(False)
    stages = {k: float(np.mean([x[k] for x in st])) for k in st[0]}
    stages['mp_phases_ms'] = {k: float(np.mean([x[k] for x in ph])) for k in ph[0]}
    return tot, stages


def fp64_score_error(s16, s32, setup, rows_d, drift, ib, nb):
    """Max and RMS error of the BF16+re-check and the FP32 score fields against
    an FP64 score field of the same filtered batch (torch float64 conv1d with
    the temporal basis, then the template contraction: template_matching.py:
    145-146), over all T x N scores."""
    s32.set_drift(drift)
    s16.set_drift(drift)
    X = s32.filter(rows_d, ib, nb)
    B16 = s16.scores(X).double()
    B32 = s32.scores(X).double()
    nt = setup.nt
    W = setup.wPCA.double().to(X.device)
    B0 = torch.nn.functional.conv1d(X.double().unsqueeze(1), W.unsqueeze(1), padding=nt // 2)
    B64 = torch.einsum('ijk,kjl->il', setup.U.double().to(X.device), B0)
    scale = float(B64.abs().max())
    rms64 = float(B64.square().mean().sqrt())
    out = {}
    for name, B in (('bf16_recheck', B16), ('fp32', B32)):
        d = B - B64
        out[name] = {'max_abs': float(d.abs().max()), 'rms': float(d.square().mean().sqrt()),
                     'max_rel_to_max_score': float(d.abs().max()) / scale,
                     'rms_rel_to_rms_score': float(d.square().mean().sqrt()) / rms64}
    out['fp64_max_abs_score'] = scale
    out['fp64_rms_score'] = rms64
    out['scores'] = int(B64.numel())
    out['batch'] = int(ib)
    return out


def max_over_ranks(x: float, dist, device) -> float:
    """The largest of every rank's x (x itself without a process group): a
    multi-GPU step time is the slowest rank's."""
    if not dist:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def path_roofline(setup, spikes_per_batch, T, rec_s_per_s, hbm_gbs, tensor_tflops, src):
    """The whole path against both bounds: algorithmic FLOPs and bytes per
    recording-second (whitening/drift C^2, temporal basis C*K*nt, score GEMM
    T*K*C per sample, plus 2*T*(2nt+1) FLOPs and 12*T*(2nt+1) bytes per
    accepted spike; int16 in and the score field written and read once),
    times the measured rate."""
    C, K, nt = setup.C, setup.K, setup.nt
    L2 = 2 * nt + 1
    S = spikes_per_batch / (setup.NT / FS)  # accepted spikes per recording-second
    flops = 2.0 * FS * (C * C + C * K * nt + T * K * C) + S * 2.0 * T * L2
    nbytes = 2.0 * C * FS + 8.0 * T * FS + S * 12.0 * T * L2
    f_t = flops * rec_s_per_s / 1e12 / tensor_tflops
    f_h = nbytes * rec_s_per_s / 1e9 / hbm_gbs
    return {'flops_per_rec_s': flops, 'bytes_per_rec_s': nbytes,
            'tflops': flops * rec_s_per_s / 1e12, 'gbs': nbytes * rec_s_per_s / 1e9,
            'frac_tensor': f_t, 'frac_hbm': f_h, 'bound': 'hbm' if f_h >= f_t else 'tensor',
            'frac': max(f_t, f_h), 'peaks': f'{src}: HBM {hbm_gbs} GB/s, dense bf16 {tensor_tflops} TFLOP/s'}


def profile_traffic(name):
    """DRAM bytes per launch recorded in a committed ncu summary (None if absent)."""
    f = ROOT / 'profiles' / name
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith('dram_bytes_per_launch:'):
            return int(line.split(':')[1])
    return None


def bf16_report(s16, s32, rows_d, drifts, ids, nb):
    """Untimed: the BF16 path's re-check statistics and its spike agreement
    with the FP32 path over the batch pool ((time, template) pairs)."""
    near = rescored = flips = common = n32 = n16 = 0
    for j, ib in enumerate(ids):
        s16.set_drift(drifts[j])
        s32.set_drift(drifts[j])
        r16 = s16.sort_batch(rows_d[j], ib, nb, on_device=True)
        st = s16.stats()
        near += st['recheck_columns']
        rescored += st['recheck_rescored']
        flips += st['recheck_flips']
        r32 = s32.sort_batch(rows_d[j], ib, nb, on_device=True)
        a = set(zip(r32['time'].tolist(), r32['template'].tolist()))
        b = set(zip(r16['time'].tolist(), r16['template'].tolist()))
        common += len(a & b)
        n32 += len(a)
        n16 += len(b)
    nbat = len(ids)
    return {'agreement_vs_fp32': common / max(n32, n16, 1), 'spikes_fp32': n32, 'spikes_bf16': n16,
            'common': common, 'recheck_near_columns_per_batch': near / nbat,
            'recheck_rescored_columns_per_batch': rescored / nbat, 'recheck_flips_per_batch': flips / nbat}


def oracle_batch(setup, rec, ib, ns=None):
    """The oracle's filter + run_matching + PC features on one batch."""
    sys.path.insert(0, str(ROOT / 'oracle'))
    import ks4_oracle as ko
    X = ko.padded_batch(rec.raw, ib, setup.NT, setup.nt)
    if ns is not None:
        X = X[:, :ns + 2 * setup.nt]
    X = ko.filter_batch(X, hp_filter=setup.hp_filter, whiten_mat=setup.Wrot,
                        drift_M=setup.drift_matrix(rec.dshift[ib]))
    st, amps, Xres = ko.run_matching(X, setup.U, setup.ctc, setup.wPCA, setup.Th, setup.nt)
    ko.extract_batch(st, amps, Xres, setup.iCC, setup.iU, setup.Ucc, setup.wPCA, setup.nt, setup.nt0min, ib,
                     setup.NT)
    return len(st)


def cpu_model():
    """The host CPU's model name (Linux /proc/cpuinfo), or the platform string."""
    try:
        for line in open('/proc/cpuinfo'):
            if line.startswith('model name'):
                return line.split(':', 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or platform.machine()


def cpu_baseline(setup, rec, n_batches=5, budget_s=60.0):
    """The oracle on the host cores: one warm-up batch, then n_batches full
    batches (fewer if budget_s runs out, at least one); rate = batch length in
    seconds / median seconds per batch."""
    cores = os.cpu_count() or 1
    torch.set_num_threads(cores)
    oracle_batch(setup, rec, 1)  # warm-up
    times = []
    t_start = time.perf_counter()
    for nb in range(n_batches):
        t = time.perf_counter()
        oracle_batch(setup, rec, 1 + nb % N_BATCH_POOL)
        times.append(time.perf_counter() - t)
        if time.perf_counter() - t_start > budget_s:
            break
    med = float(np.median(times))
    return {'value': setup.NT / FS / med, 'unit': 'rec-s/s', 'cores': cores, 'kind': 'port',
            'seconds_per_batch_median': med, 'cpu': cpu_model(),
            'sample': f'median of {len(times)} full 60000-sample batches of the same workload (after one warm-up '
                      f'batch) through the CPU oracle (torch {torch.__version__}, {cores} threads): filter + '
                      f'run_matching + PC features'}


def run_reference(args):
    """The reference's CPU implementation of the path (Kilosort4's torch
    template matching, restated in the oracle because the reference is Python
    and cannot travel), on the host cores, same workload and metric."""
    rank = int(os.environ.get('RANK', 0))
    if rank != 0:
        return
    T = args.templates
    setup, rec = workload(T, 0)
    cores = os.cpu_count() or 1
    torch.set_num_threads(cores)
    t0 = time.perf_counter()
    oracle_batch(setup, rec, 1, ns=6000)
    # size each step so that warmup + steps stay within ~3 minutes
    t_small = time.perf_counter() - t0
    est_full = t_small * 10
    budget = 180.0 / max(1, args.steps + args.warmup)
    ns = int(min(setup.NT, max(3000, setup.NT * budget / max(est_full, 1e-3))) // 1000 * 1000)
    for i in range(args.warmup):
        oracle_batch(setup, rec, 1 + i % N_BATCH_POOL, ns=ns)
    times = []
    for i in range(args.steps):
        t = time.perf_counter()
        oracle_batch(setup, rec, 1 + i % N_BATCH_POOL, ns=ns)
        times.append(time.perf_counter() - t)
    tot = float(np.sum(times))
    value = args.steps * ns / FS / tot
    cpu = {'value': value, 'unit': 'rec-s/s', 'cores': cores, 'kind': 'port', 'cpu': cpu_model(),
           'sample': f'each step: one {ns}-sample slice (+-61 context) of a 60000-sample batch through the '
                     f'oracle filter + run_matching + PC features, torch CPU, {cores} threads'}
    out = {'metric': METRIC, 'value': value, 'unit': 'rec-s/s', 'n_gpus': args.gpus, 'steps': args.steps,
           'warmup': args.warmup, 'ms_per_step': tot / args.steps * 1e3, 'higher_is_better': True,
           'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic', 'impl': 'reference',
           'config': workload_desc(T, 'fp32') | {'parallelism': 'cpu', 'samples_per_step': ns,
                                                  'batch_samples_of_workload': setup.NT},
           'cpu_baseline': cpu, 'e2e': {'value': value, 'unit': 'rec-s/s', 'h2d_bytes_per_step': 0,
                                        'd2h_bytes_per_step': 0},
           'latency_ms_p50': float(np.percentile(times, 50) * 1e3),
           'latency_ms_p99': float(np.percentile(times, 99) * 1e3)}
    print(json.dumps(out))


def run_serving(args):
    """Four probes through the streaming loop: real-time latency, then capacity."""
    rank = int(os.environ.get('RANK', 0))
    local = int(os.environ.get('LOCAL_RANK', 0))
    torch.cuda.set_device(local)
    out = serving_report(local, rank, args.duration, args.warmup)
    if rank == 0:
        print(json.dumps(out))


def serving_report(local, rank, duration, warmup):
    """Four 384-channel probes (200/400/600/800 templates, 3000/1500/600/300-
    sample blocks) through the streaming loop: a real-time run with seeded
    arrival jitter for latency, then a run with all blocks available at once
    for capacity."""
    from livespikesorter_b200 import synth
    from livespikesorter_b200.serve import ProbeServer, Stream, run_streams
    from livespikesorter_b200.sorter import setup_kwargs
    blocks = (3000, 1500, 600, 300)
    probes = synth.streaming_probes(seed=23 + rank, duration_s=duration)

    def streams(n_blocks=None):
        out = []
        for (setup, rec), blk in zip(probes, blocks):
            kw = setup_kwargs(setup) | dict(NT=blk)
            out.append(Stream(f'T{setup.T}_b{blk}', kw, rec.raw, blk, depth=4, capacity=16384,
                              n_blocks=None if n_blocks is None else min(n_blocks, rec.raw.shape[0] // blk)))
        return out

    srv = ProbeServer(device=local, memory_budget=40 << 30, max_probes=8)
    run_streams(srv, streams(n_blocks=max(3, warmup)), realtime=False)            # warm-up
    # an NVML clock query stalls the submitting thread for tens of ms, which the
    # real-time run would count as latency: clocks are sampled during the
    # capacity run that follows, on the same streams and kernels
    rt = run_streams(srv, streams(), realtime=True, jitter_frac=0.2, seed=5 + rank, start_together=True)
    with Clocks(local, period_ms=200) as clk:
        cap = run_streams(srv, streams(), realtime=False, start_together=True)
    clocks = clk.summary()
    lat = {st.name: {k: v for k, v in st.latency.items() if k not in ('samples_ms', 'parts_ms')} for st in rt['streams']}
    # medians and 99th percentiles of the latency's parts: arrival -> launch, launch -> device start,
    # device span, device end -> completion seen (ms)
    for st in rt['streams']:
        P = np.array(st.latency['parts_ms'])
        lat[st.name]['parts_p50_ms'] = np.round(np.median(P, 0), 3).tolist()
        lat[st.name]['parts_p99_ms'] = np.round(np.percentile(P, 99, 0), 3).tolist()
    # the three slowest batches of each stream: [latency, batch, [arrival->launch, launch->device start,
    # device span, device end->completion seen]] (ms)
    worst = {st.name: [[round(v, 2), i, [round(x, 2) for x in st.latency['parts_ms'][i]]]
                       for v, i in sorted((v, i) for i, v in enumerate(st.latency['samples_ms']))[-3:]]
             for st in rt['streams']}
    spikes = {st.name: int(sum(len(r['time']) for r in st.results.values())) for st in rt['streams']}
    # how late the serving loop pushed each block after its arrival instant (host-side share of the latency)
    push_late = {st.name: round(max(st.push_late_ms, default=0.0), 3) for st in rt['streams']}
    out = {
        'metric': 'p99 arrival-to-emit latency, 4 concurrent 384ch probes, 10-100 ms blocks',
        'value': max(v['p99_ms'] for v in lat.values()), 'unit': 'ms', 'higher_is_better': False,
        'n_gpus': 1, 'steps': int(sum(v['batches'] for v in lat.values())), 'warmup': max(3, warmup),
        'dtype': 'f32', 'data': 'synthetic',
        'config': {'workload': 'serving: 4 probes x 384 ch, T = 200/400/600/800, blocks 3000/1500/600/300 samples, '
                               f'{duration:g} s each, real-time arrival with 20% seeded jitter, '
                               'streaming starts once the four probes are admitted',
                   'parallelism': 'one GPU, probes overlap on separate streams'},
        'latency_ms': lat, 'worst_latencies_ms': worst, 'push_late_max_ms': push_late, 'spikes': spikes,
        'realtime_rec_s_per_s': rt['rec_s_per_s'],
        'capacity_rec_s_per_s': cap['rec_s_per_s_streaming'], 'capacity_wall_s': cap['wall_s'],
        'clocks': clocks,
    }
    srv.close()
    return out


def run_refine(args):
    """Template refinement with fixed assignments: 384 ch, 400 templates, 16
    batches rendered from templates whose footprints are shifted 10 um and
    scaled +-10% from the sorter's. Sort every batch with the sorter's
    templates, then take Gauss-Newton (Jacobi-preconditioned) steps on the
    residual energy of all 16 batches through the hand-written adjoint; report
    steps/s and the template error against the rendering templates before and
    after."""
    from livespikesorter_b200 import synth
    from livespikesorter_b200.adjoint import refine
    from livespikesorter_b200.sorter import Sorter
    local = int(os.environ.get('LOCAL_RANK', 0))
    torch.cuda.set_device(local)
    setup, rec = synth.config(4, duration_s=32.0, seed=29)
    U_true = rec.meta['U_true'].double()
    s = Sorter.from_setup(setup, device=local)
    nb = rec.n_batches
    batches = []
    for ib in range(nb):
        NT, nt = setup.NT, setup.nt
        rows = rec.raw[0:NT + nt] if ib == 0 else rec.raw[ib * NT - nt: min(rec.raw.shape[0], ib * NT + NT + nt)]
        X = s.filter(np.ascontiguousarray(rows), ib, nb)
        st, amps, _ = s.match(X, return_xres=False)
        batches.append((X, st[:, 0].to(torch.int32), st[:, 1].to(torch.int32), amps[:, 0].contiguous()))
    spikes = sum(len(b[1]) for b in batches)
    U0 = setup.U.cuda()
    W = setup.wPCA.cuda()

    def errors(U):
        Ud = U.double().cpu()
        rel = float((Ud - U_true).norm() / U_true.norm())
        # per-template best scale (amplitude and template norm trade off)
        sc = (Ud * U_true).sum((1, 2)) / Ud.square().sum((1, 2)).clamp_min(1e-30)
        shape = float((Ud * sc[:, None, None] - U_true).norm() / U_true.norm())
        return rel, shape

    e0 = errors(U0)
    lr = 0.8
    refine(batches, U0, W, steps=2, lr=lr)                 # warm-up
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    U1, _, losses = refine(batches, U0, W, steps=args.refine_steps, lr=lr)
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    e1 = errors(U1)
    # the same refinement with the rendering's own assignments (spike times,
    # units, amplitudes relative to the 80 uV templates): what the adjoint
    # recovers when the assignments are right
    gt = []
    for ib, (X, _, _, _) in enumerate(batches):
        NT, nt = setup.NT, setup.nt
        x = rec.spike_times - ib * NT + nt + nt // 2 - setup.nt0min
        keep = (x >= nt) & (x < X.shape[1] - nt)
        gt.append((X, torch.from_numpy(x[keep].astype(np.int32)).cuda(),
                   torch.from_numpy(rec.spike_units[keep].astype(np.int32)).cuda(),
                   torch.from_numpy((rec.spike_amps_uv[keep] / 80.0).astype(np.float32)).cuda()))
    U2, _, losses2 = refine(gt, U0, W, steps=args.refine_steps, lr=lr)
    e2 = errors(U2)
    out = {
        'metric': 'template refinement: residual-energy gradient steps per second (16 batches, fixed assignments)',
        'value': args.refine_steps / (ms / 1e3), 'unit': 'steps/s', 'higher_is_better': True, 'n_gpus': 1,
        'steps': args.refine_steps, 'warmup': 2, 'dtype': 'f32', 'data': 'synthetic',
        'config': {'workload': 'refine: 384 ch, 400 templates, 16 x 60000-sample batches rendered with footprints '
                               'shifted 10 um and scaled +-10%; Gauss-Newton (Jacobi) steps on U, wPCA fixed',
                   'spikes': spikes},
        'ms_per_step': ms / args.refine_steps,
        'loss_first': losses[0], 'loss_last': losses[-1],
        'template_rel_err_before': e0[0], 'template_rel_err_after': e1[0],
        'template_shape_err_before': e0[1], 'template_shape_err_after': e1[1],
        'with_true_assignments': {'loss_first': losses2[0], 'loss_last': losses2[-1],
                                  'template_rel_err_after': e2[0], 'template_shape_err_after': e2[1],
                                  'spikes': int(sum(len(b[1]) for b in gt))},
    }
    print(json.dumps(out))


if __name__ == '__main__':
    a = parse()
    if a.impl == 'reference':
        run_reference(a)
    elif a.workload == 'serving':
        run_serving(a)
    elif a.workload == 'refine':
        run_refine(a)
    else:
        run_b200(a)
