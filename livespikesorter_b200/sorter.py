"""Torch-facing host API over the C ABI.

``Sorter`` owns one ``lss_handle`` (one probe stream). ``run_matching`` keeps
the signature and return types of ``kilosort/template_matching.py:128-202`` so
it can stand in for it.

All compute happens in ``liblss_b200.so`` on the GPU; tensors only carry
device memory and the current CUDA stream across the boundary.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._lib import LssConfig, LssPostConfig, LssRecords, LssStageTimes, LssStats, LssTensors, STAGES, check


def _f32(x) -> torch.Tensor:
    if isinstance(x, np.ndarray):
        x = torch.from_numpy(x)
    return x.detach().to('cpu', torch.float32).contiguous()


def _i64(x) -> torch.Tensor:
    if isinstance(x, np.ndarray):
        x = torch.from_numpy(x)
    return x.detach().to('cpu', torch.int64).contiguous()


def _ptr(t):
    return None if t is None else t.data_ptr()


def _stream(device) -> int | None:
    return torch.cuda.current_stream(device).cuda_stream


def build_config(*, U, wPCA, ctc, Wrot, hp_filter=None, drift=None, iCC=None, iU=None, Ucc=None, chan_map=None,
                 nm=None, NT: int = 60000, nt0min: int = 20, Th: float = 8.0, n_chan_bin: int | None = None,
                 max_rounds: int = 100, max_spikes: int = 100000, do_CAR: bool = True, invert_sign: bool = False,
                 precision: str = 'fp32', device: int = 0):
    """``(lss_config, lss_tensors, keep)`` for ``lss_create``; ``keep`` holds the
    host tensors the pointers refer to and must outlive the call."""
    U = _f32(U)
    T, K, C = U.shape
    wPCA = _f32(wPCA)
    nt = wPCA.shape[1]
    k = dict(U=U, wPCA=wPCA, ctc=_f32(ctc), Wrot=_f32(Wrot),
             hp=None if hp_filter is None else _f32(hp_filter),
             drift=None if drift is None else _f32(drift),
             iCC=None if iCC is None else _i64(iCC), iU=None if iU is None else _i64(iU),
             Ucc=None if Ucc is None else _f32(Ucc),
             cmap=None if chan_map is None else torch.as_tensor(np.asarray(chan_map), dtype=torch.int32).contiguous(),
             nm=None if nm is None else _f32(nm))
    nC = 0 if k['iCC'] is None else k['iCC'].shape[0]
    cfg = LssConfig(n_chan=C, n_chan_bin=n_chan_bin or C, n_templates=T, n_pcs=K, nt=nt, n_nearest=nC,
                    batch_size=NT, nt0min=nt0min, th_learned=float(Th), max_rounds=max_rounds,
                    max_spikes=max_spikes, do_car=int(do_CAR), invert_sign=int(invert_sign),
                    precision={'fp32': 0, 'bf16': 1}[precision], device=device,
                    hp_len=0 if k['hp'] is None else k['hp'].numel())
    tens = LssTensors(wall3=_ptr(k['U']), wpca=_ptr(k['wPCA']), ctc=_ptr(k['ctc']), whitening=_ptr(k['Wrot']),
                      drift=_ptr(k['drift']), hp_filter=_ptr(k['hp']), iCC=_ptr(k['iCC']), iU=_ptr(k['iU']),
                      Ucc=_ptr(k['Ucc']), chan_map=_ptr(k['cmap']), nm=_ptr(k['nm']))
    return cfg, tens, k


def post_config(xc=None, yc=None, centroids=None, dt: int = 7):
    """``(lss_post_config, keep)`` for positions (channel coordinates xc, yc),
    nearest-centroid clusters (``centroids`` [n, 2]) and duplicate removal
    within ``dt`` samples; ``keep`` holds the arrays the pointers refer to."""
    k = dict(xc=None if xc is None else np.ascontiguousarray(xc, np.float32),
             yc=None if yc is None else np.ascontiguousarray(yc, np.float32),
             cen=None if centroids is None else np.ascontiguousarray(centroids, np.float32).reshape(-1, 2))
    cfg = LssPostConfig(xc=None if k['xc'] is None else k['xc'].ctypes.data,
                        yc=None if k['yc'] is None else k['yc'].ctypes.data,
                        centroids_xy=None if k['cen'] is None else k['cen'].ctypes.data,
                        n_clusters=0 if k['cen'] is None else k['cen'].shape[0], dt_samples=int(dt))
    return cfg, k


def check_record_set(o: dict, nC: int, K: int, device=None) -> None:
    """Raises ValueError unless ``o`` is a record set the kernels can write:
    contiguous tensors of one capacity with the record dtypes (time int64,
    template int32, amplitude f32, pc f32 [cap, nC, K] or None, count int64),
    each on the sorter's GPU (``device``, when given) or in pinned host memory.
    A wrong dtype or a short array would let the kernels write past its end;
    another GPU's tensor would be written without peer access."""
    want = dict(time=torch.int64, template=torch.int32, amplitude=torch.float32, count=torch.int64)
    for k, dt in want.items():
        t = o.get(k)
        if not isinstance(t, torch.Tensor) or t.dtype != dt or not t.is_contiguous():
            raise ValueError(f'record set: {k} must be a contiguous {dt} tensor')
    cap = o['time'].shape[0]
    if o['time'].dim() != 1 or o['template'].shape != (cap,) or o['amplitude'].shape != (cap,):
        raise ValueError('record set: time, template and amplitude must be 1-D of one capacity')
    if o['count'].numel() < 1:
        raise ValueError('record set: count needs one element')
    pc = o.get('pc')
    if pc is not None:
        if (not isinstance(pc, torch.Tensor) or pc.dtype != torch.float32 or not pc.is_contiguous()
                or tuple(pc.shape) != (cap, max(nC, 1), K)):
            raise ValueError(f'record set: pc must be a contiguous float32 [{cap}, {max(nC, 1)}, {K}] tensor')
    for k in ('time', 'template', 'amplitude', 'pc', 'count'):
        t = o.get(k)
        if t is not None and not (t.is_cuda or t.is_pinned()):
            raise ValueError(f'record set: {k} must be on the GPU or in pinned host memory')
        if t is not None and t.is_cuda and device is not None and t.device != torch.device(device):
            raise ValueError(f'record set: {k} is on {t.device}, the sorter runs on {torch.device(device)}')


def setup_kwargs(setup) -> dict:
    """Constructor arguments of a ``synth.SortSetup``."""
    return dict(U=setup.U, wPCA=setup.wPCA, ctc=setup.ctc, Wrot=setup.Wrot, hp_filter=setup.hp_filter,
                iCC=setup.iCC, iU=setup.iU, Ucc=setup.Ucc, NT=setup.NT, nt0min=setup.nt0min, Th=setup.Th)


class Sorter:
    """One sorter handle: templates, ctc, whitening, filters and all device
    workspaces live on ``device`` for the handle's lifetime."""

    def __init__(self, *, device: int = 0, **kw):
        self._lib = _lib.load()
        cfg, tens, keep = build_config(device=device, **kw)
        h = __import__('ctypes').c_void_p()
        check(self._lib.lss_create(cfg, tens, h))
        del keep
        self._h = h
        self._init_dims(device)

    @classmethod
    def from_dir(cls, path: str, **overrides) -> 'Sorter':
        """Build from an LSS input directory (the files
        ``src/Python/run_online_spikes.py:548-576`` writes)."""
        import ctypes
        self = cls.__new__(cls)
        self._lib = _lib.load()
        ov = LssConfig(n_chan_bin=overrides.get('n_chan_bin', 0), batch_size=overrides.get('NT', 0),
                       nt0min=overrides.get('nt0min', 0), th_learned=float(overrides.get('Th', 0.0)),
                       max_rounds=overrides.get('max_rounds', 0), max_spikes=overrides.get('max_spikes', 0),
                       do_car=int(overrides.get('do_CAR', True)), invert_sign=int(overrides.get('invert_sign', False)),
                       precision={'fp32': 0, 'bf16': 1}[overrides.get('precision', 'fp32')],
                       device=overrides.get('device', 0))
        h = ctypes.c_void_p()
        check(self._lib.lss_create_from_dir(str(path).encode(), ov, h))
        self._h = h
        self._init_dims(ov.device)
        return self

    @classmethod
    def from_setup(cls, setup, **kw) -> 'Sorter':
        """Build from a ``synth.SortSetup``."""
        return cls(**(setup_kwargs(setup) | kw))

    def _init_dims(self, device):
        cfg = LssConfig()
        check(self._lib.lss_get_config(self._h, cfg), self._h)
        self.cfg = cfg
        self.device = torch.device('cuda', device)
        self.C, self.T, self.K, self.nt = cfg.n_chan, cfg.n_templates, cfg.n_pcs, cfg.nt
        self.nC, self.NT = cfg.n_nearest, cfg.batch_size
        self.N = self.NT + 2 * self.nt

    def close(self):
        if getattr(self, '_h', None):
            self._lib.lss_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        check(rc, self._h)

    # ------------------------------------------------------------- stages
    def set_drift(self, M):
        """Drift interpolation matrix for the following batches (None = identity)."""
        Mt = None if M is None else _f32(M)
        self._check(self._lib.lss_set_drift(self._h, _ptr(Mt)))

    def filter(self, raw, ibatch: int, n_batches: int) -> torch.Tensor:
        """Padded, filtered, whitened batch ``[C, NT + 2nt]`` (kilosort/io.py:584-637, 757-790)."""
        raw_t, on_dev = self._raw(raw)
        X = torch.empty((self.C, self.N), device=self.device, dtype=torch.float32)
        self._check(self._lib.lss_filter(self._h, raw_t.data_ptr(), raw_t.shape[0], ibatch, n_batches, on_dev,
                                         X.data_ptr(), _stream(self.device)))
        return X

    def _raw(self, raw):
        if isinstance(raw, np.ndarray):
            raw = torch.from_numpy(np.ascontiguousarray(raw))
        if raw.dtype != torch.int16 or raw.dim() != 2:
            raise ValueError('raw must be an int16 [n_rows, n_chan_bin] array')
        raw = raw.contiguous()
        if raw.shape[1] != self.cfg.n_chan_bin:
            raise ValueError(f'raw has {raw.shape[1]} channels, expected {self.cfg.n_chan_bin}')
        return raw, int(raw.is_cuda)

    def scores(self, X: torch.Tensor) -> torch.Tensor:
        X = X.to(self.device, torch.float32).contiguous()
        B = torch.empty((self.T, X.shape[1]), device=self.device, dtype=torch.float32)
        self._check(self._lib.lss_scores(self._h, X.data_ptr(), X.shape[1], B.data_ptr(), _stream(self.device)))
        return B

    def match(self, X: torch.Tensor, return_xres: bool = True, capacity: int | None = None):
        """``run_matching`` on a filtered batch: ``(st int64 [n,2], amps f32 [n,1], Xres [C,N])``."""
        import ctypes
        X = X.to(self.device, torch.float32).contiguous()
        N = X.shape[1]
        cap = capacity or self.cfg.max_spikes
        st = torch.empty((cap, 2), device=self.device, dtype=torch.int64)
        amps = torch.empty((cap, 1), device=self.device, dtype=torch.float32)
        xres = torch.empty_like(X) if return_xres else None
        n = ctypes.c_int64(0)
        self._check(self._lib.lss_match(self._h, X.data_ptr(), N, st.data_ptr(), amps.data_ptr(),
                                        _ptr(xres), cap, ctypes.byref(n), _stream(self.device)))
        return st[:n.value], amps[:n.value], xres

    def match_scores(self, B: torch.Tensor, capacity: int | None = None):
        """The rounds alone on a given score field ``B [T, N]``: ``(st, amps)``."""
        import ctypes
        B = B.to(self.device, torch.float32).contiguous()
        cap = capacity or self.cfg.max_spikes
        st = torch.empty((cap, 2), device=self.device, dtype=torch.int64)
        amps = torch.empty((cap, 1), device=self.device, dtype=torch.float32)
        n = ctypes.c_int64(0)
        self._check(self._lib.lss_match_scores(self._h, B.data_ptr(), B.shape[1], st.data_ptr(), amps.data_ptr(),
                                               cap, ctypes.byref(n), _stream(self.device)))
        return st[:n.value], amps[:n.value]

    def sort_batch(self, raw, ibatch: int, n_batches: int, with_pc: bool = True, on_device: bool = False,
                   capacity: int | None = None) -> dict:
        """One batch end to end: records ``time, template, amplitude, pc [n, nC, K]``."""
        raw_t, raw_dev = self._raw(raw)
        cap = capacity or self.cfg.max_spikes
        dev = self.device if on_device else 'cpu'
        pin = (not on_device)
        time = torch.empty(cap, dtype=torch.int64, device=dev, pin_memory=pin)
        tmpl = torch.empty(cap, dtype=torch.int32, device=dev, pin_memory=pin)
        amp = torch.empty(cap, dtype=torch.float32, device=dev, pin_memory=pin)
        pc = torch.empty((cap, self.nC, self.K), dtype=torch.float32, device=dev, pin_memory=pin) \
            if (with_pc and self.nC > 0) else None
        post = getattr(self, '_post', False)
        xs = torch.empty(cap, dtype=torch.float32, device=dev, pin_memory=pin) if post else None
        ys = torch.empty(cap, dtype=torch.float32, device=dev, pin_memory=pin) if post else None
        clu = torch.empty(cap, dtype=torch.int32, device=dev, pin_memory=pin) if post else None
        rec = LssRecords(time=time.data_ptr(), template_id=tmpl.data_ptr(), amplitude=amp.data_ptr(),
                         pc=_ptr(pc), capacity=cap, count=0, on_device=int(on_device), x_pos=_ptr(xs),
                         y_pos=_ptr(ys), cluster=_ptr(clu))
        self._check(self._lib.lss_sort_batch(self._h, raw_t.data_ptr(), raw_t.shape[0], ibatch, n_batches,
                                             raw_dev, rec, _stream(self.device)))
        n = rec.count
        out = dict(time=time[:n], template=tmpl[:n], amplitude=amp[:n], pc=None if pc is None else pc[:n])
        if post:
            out.update(x=xs[:n], y=ys[:n], cluster=clu[:n])
        return out

    def records(self, capacity: int | None = None, pinned: bool = False) -> dict:
        """Record tensors for ``sort_batch_async``: device tensors, or pinned
        host tensors that the batch's kernels write across the bus."""
        cap = capacity or self.cfg.max_spikes
        kw = dict(pin_memory=True) if pinned else dict(device=self.device)
        return dict(time=torch.empty(cap, dtype=torch.int64, **kw), template=torch.empty(cap, dtype=torch.int32, **kw),
                    amplitude=torch.empty(cap, dtype=torch.float32, **kw),
                    pc=torch.empty((cap, self.nC, self.K), dtype=torch.float32, **kw) if self.nC > 0 else None,
                    count=torch.zeros(1, dtype=torch.int64, **kw))

    def sort_batch_async(self, raw, ibatch: int, n_batches: int, capacity: int | None = None,
                         out: dict | None = None) -> dict:
        """``sort_batch`` with no host wait: returns the record tensors and
        ``count`` (new device tensors, or ``out`` from ``records()``); call
        ``sync()`` before reading them (it raises the first error the batches
        met). Host rows (pinned) upload under the previous batch's work and
        must stay unchanged until then."""
        raw_t, raw_dev = self._raw(raw)
        o = out if out is not None else self.records(capacity)
        if out is not None:
            check_record_set(o, self.nC, self.K, self.device)
        cap = o['time'].shape[0]
        rec = LssRecords(time=o['time'].data_ptr(), template_id=o['template'].data_ptr(),
                         amplitude=o['amplitude'].data_ptr(), pc=_ptr(o['pc']), capacity=cap, count=0, on_device=1,
                         x_pos=None, y_pos=None, cluster=None)
        self._check(self._lib.lss_sort_batch_async(self._h, raw_t.data_ptr(), raw_t.shape[0], ibatch, n_batches,
                                                   raw_dev, rec, o['count'].data_ptr(), _stream(self.device)))
        return o

    def sync(self):
        self._check(self._lib.lss_sync(self._h, _stream(self.device)))

    def stats(self) -> dict:
        s = LssStats()
        self._check(self._lib.lss_get_stats(self._h, s))
        return dict(rounds=s.rounds, spikes=s.spikes, recheck_columns=s.recheck_columns,
                    recheck_flips=s.recheck_flips, recheck_rescored=s.recheck_rescored, launches=s.launches,
                    mp_items=s.mp_items, mp_items_updated=s.mp_items_updated,
                    mp_phases_ms={k[3:-3]: getattr(s, k) * 1e-6 for k in ('mp_peak_ns', 'mp_peak_wait_ns',
                                                                             'mp_update_ns', 'mp_update_wait_ns',
                                                                             'mp_peak_max_ns', 'mp_update_max_ns')})

    def set_templates(self, U, wPCA=None):
        """Swap in new templates (same shapes) and optionally a new temporal
        basis; ctc, nm, iU, Ucc and the GEMM operands are rebuilt on the GPU."""
        Ut = _f32(U)
        Wt = None if wPCA is None else _f32(wPCA)
        if tuple(Ut.shape) != (self.T, self.K, self.C):
            raise ValueError(f'U must be [{self.T}, {self.K}, {self.C}]')
        self._check(self._lib.lss_set_templates(self._h, Ut.data_ptr(), _ptr(Wt)))

    def set_drift_model(self, xc, yc, sig_interp: float = 20.0):
        """Channel positions for drift matrices computed on the GPU."""
        x = np.ascontiguousarray(xc, np.float32)
        y = np.ascontiguousarray(yc, np.float32)
        self._check(self._lib.lss_set_drift_model(self._h, x.ctypes.data, y.ctypes.data, float(sig_interp)))

    def set_drift_shift(self, dshift: float):
        """Drift correction for a vertical shift (um), matrix built on the GPU."""
        self._check(self._lib.lss_set_drift_shift(self._h, float(dshift)))

    def set_postprocess(self, xc=None, yc=None, centroids=None, dt: int = 7, enable: bool = True):
        """Positions, nearest-centroid clusters, duplicate removal within dt
        samples and time order for the records of later batches
        (``lss_set_postprocess``); ``enable=False`` switches it off."""
        if not enable:
            self._check(self._lib.lss_set_postprocess(self._h, None))
            self._post = False
            return
        cfg, keep = post_config(xc, yc, centroids, dt)
        self._check(self._lib.lss_set_postprocess(self._h, cfg))
        del keep
        self._post = True

    def reset_postprocess(self):
        """Forget the last kept time per cluster (a new stream)."""
        self._check(self._lib.lss_reset_postprocess(self._h))

    def set_round_kernel(self, skip_blocks: bool):
        """Rounds kernel: skip provably unchanged template-row blocks (True) or
        update every row (False); the results are identical. The default is
        True from 600 templates up."""
        self._check(self._lib.lss_set_round_kernel(self._h, int(bool(skip_blocks))))

    def round_kernel(self) -> bool:
        """True when the rounds skip provably unchanged template-row blocks."""
        import ctypes
        v = ctypes.c_int32(0)
        self._check(self._lib.lss_get_round_kernel(self._h, ctypes.byref(v)))
        return bool(v.value)

    def set_profiling(self, on: bool = True):
        self._check(self._lib.lss_set_profiling(self._h, int(on)))

    def stage_times(self) -> dict:
        t = LssStageTimes()
        self._check(self._lib.lss_get_stage_times(self._h, t))
        return {n: getattr(t, n) for n in STAGES}


# ---------------------------------------------------------------- KS4 API
_cache: dict = {}


def _sorter_for(ops, U, ctc, N, device) -> Sorter:
    dev = device.index if device.index is not None else torch.cuda.current_device()
    key = (U.data_ptr(), tuple(U.shape), ctc.data_ptr(), ops['wPCA'].data_ptr(), float(ops['Th_learned']),
           int(ops['nt']), N, dev)
    s = _cache.get(key)
    if s is None:
        _cache.clear()
        nt = int(ops['nt'])
        C = U.shape[2]
        s = Sorter(U=U, wPCA=ops['wPCA'], ctc=ctc, Wrot=torch.eye(C), NT=N - 2 * nt, Th=float(ops['Th_learned']),
                   nt0min=int(ops.get('nt0min', 20)), device=dev)
        _cache[key] = s
    return s


def run_matching(ops, X, U, ctc, device=torch.device('cuda')):
    """Drop-in for ``kilosort.template_matching.run_matching`` (template_matching.py:128-202)."""
    device = torch.device(device)
    s = _sorter_for(ops, U, ctc, X.shape[1], device)
    st, amps, Xres = s.match(X.to(s.device))
    return st, amps, Xres
