"""Seeded synthetic recordings and sorter setups for benchmarking and tests.

No public dataset ships with the reference, and Kilosort's own
``kilosort/simulation.py`` needs external waveform files, so this module builds
recordings from a stated generative model:

* probe: a 2-column layout (16 um horizontal, 20 um vertical pitch) or a
  Neuropixels-like 4-column staggered layout at 20 um pitch;
* units: a biphasic waveform (negative Gaussian trough of 0.3 ms FWHM at
  sample ``nt0min``, positive lobe of 1/3 the amplitude 0.5 ms later) with 5 %
  seeded noise; a Gaussian spatial footprint (sigma 30 um) centred at a
  uniform random probe position;
* spike trains: Poisson at rates uniform in 2-20 Hz with a 1.5 ms refractory
  period; amplitudes lognormal (median 80 uV, sigma 0.3);
* background: 10 uV RMS Gaussian noise with a 1/f component, quantised at
  0.195 uV/bit into int16;
* optional linear drift of the footprints (um/min), corrected per batch by the
  drift interpolation matrix.

The sorter setup is derived the way Kilosort derives it: the highpass impulse
response, ``Wrot`` from the filtered noise covariance (local ZCA), a 6-PC
temporal basis from the SVD of the filtered waveforms, ``U`` as the whitened
templates projected on that basis, then ``ctc`` and the nearest-channel tables.

All randomness comes from numpy generators and rendering is float64 on the CPU,
so a given seed yields the same int16 recording on every machine.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from . import setup_tensors as st

UV_PER_BIT = 0.195


@dataclass
class Probe:
    xc: np.ndarray
    yc: np.ndarray

    @property
    def C(self) -> int:
        return len(self.xc)


def probe_two_column(C: int = 64, dx: float = 16.0, dy: float = 20.0) -> Probe:
    i = np.arange(C)
    return Probe((i % 2) * dx, (i // 2) * dy)


def probe_staggered(C: int = 384, pitch: float = 20.0) -> Probe:
    """Four columns, two sites per row, alternate rows offset (Neuropixels 1.0 style)."""
    i = np.arange(C)
    xs = np.array([43.0, 11.0, 59.0, 27.0])
    return Probe(xs[i % 4], (i // 2) * pitch)


@dataclass
class SortSetup:
    """Everything the sorter loads for one probe (the LSS input directory)."""
    probe: Probe
    fs: float
    NT: int
    nt: int
    nt0min: int
    Th: float
    nC: int
    wPCA: torch.Tensor      # [K, nt] f32
    U: torch.Tensor         # [T, K, C] f32 (Wall3)
    ctc: torch.Tensor       # [T, T, 2nt+1] f32
    Wrot: torch.Tensor      # [C, C] f32
    hp_filter: torch.Tensor  # [30122] f32
    iKxx: torch.Tensor      # [C, C] f64
    iCC: torch.Tensor       # [nC, C] i64
    iU: torch.Tensor        # [T] i64
    Ucc: torch.Tensor       # [nC, T, K] f32

    @property
    def C(self):
        return self.probe.C

    @property
    def T(self):
        return self.U.shape[0]

    @property
    def K(self):
        return self.U.shape[1]

    def drift_matrix(self, dshift: float) -> torch.Tensor:
        return st.get_drift_matrix(self.probe.xc, self.probe.yc, dshift, self.iKxx).float()


@dataclass
class Recording:
    raw: np.ndarray                 # [n_samples, C] int16
    spike_times: np.ndarray         # trough sample of every ground-truth spike
    spike_units: np.ndarray
    spike_amps_uv: np.ndarray
    dshift: np.ndarray              # per-batch drift estimate (um) for the sorter
    setup: SortSetup
    meta: dict = field(default_factory=dict)

    @property
    def n_batches(self) -> int:
        return int(np.ceil(self.raw.shape[0] / self.setup.NT))


def _waveforms(rng, T, nt, nt0min, fs):
    m = np.arange(nt)[None, :].astype(np.float64)
    sig = 0.3e-3 * fs / 2.355
    lobe = nt0min + 0.5e-3 * fs
    w = -np.exp(-(m - nt0min) ** 2 / (2 * sig ** 2)) + np.exp(-(m - lobe) ** 2 / (2 * (2 * sig) ** 2)) / 3.0
    w = np.repeat(w, T, 0)
    w = w + 0.05 * rng.standard_normal(w.shape)
    return w / np.abs(w[:, nt0min:nt0min + 1])


def _footprints(xc, yc, cx, cy, sigma=30.0):
    d2 = (xc[None, :] - cx[:, None]) ** 2 + (yc[None, :] - cy[:, None]) ** 2
    return np.exp(-d2 / (2 * sigma ** 2))


def _hp_apply(x: np.ndarray, h: np.ndarray) -> np.ndarray:
    """Zero-phase filtering of short rows with the impulse response (same length)."""
    L = len(h)
    c = L // 2
    out = np.empty_like(x)
    for i in range(x.shape[0]):
        out[i] = np.convolve(x[i], h, mode='full')[c:c + x.shape[1]]
    return out


def _noise(rng, n, C, rms_white=9.0, rms_pink=4.4):
    white = rng.standard_normal((C, n)) * rms_white
    f = np.fft.rfftfreq(n)
    f[0] = f[1]
    spec = (rng.standard_normal((C, len(f))) + 1j * rng.standard_normal((C, len(f)))) / np.sqrt(f)
    pink = np.fft.irfft(spec, n)
    pink *= rms_pink / (pink.std() + 1e-12)
    return (white + pink).T  # [n, C] uV


def make_setup_and_units(probe: Probe, T: int, seed: int, nt: int = 61, nt0min: int = 20,
                         fs: float = 30000, NT: int = 60000, Th: float = 8.0, nC: int = 10,
                         K: int = 6, dup_frac: float = 0.0, n_cov_samples: int = 60000):
    """Build unit parameters and the sorter setup derived from them."""
    rng = np.random.default_rng(seed)
    C = probe.C
    cx = rng.uniform(probe.xc.min(), probe.xc.max(), T)
    cy = rng.uniform(probe.yc.min(), probe.yc.max(), T)
    n_dup = int(round(dup_frac * T / 2))
    for p in range(n_dup):  # second member of a pair sits 10 um from the first
        a, b = 2 * p, 2 * p + 1
        ang = rng.uniform(0, 2 * np.pi)
        cx[b] = cx[a] + 10.0 * np.cos(ang)
        cy[b] = cy[a] + 10.0 * np.sin(ang)
    waves = _waveforms(rng, T, nt, nt0min, fs)
    if n_dup:
        waves[1:2 * n_dup:2] = waves[0:2 * n_dup:2] + 0.05 * rng.standard_normal((n_dup, nt))
    rates = rng.uniform(2.0, 20.0, T)

    hp = st.get_highpass_filter(fs, 300)
    h64 = hp.double().numpy()
    # noise covariance after the reference filter chain -> local ZCA whitening
    noise = _noise(np.random.default_rng(seed + 7), n_cov_samples, C)
    Xn = torch.from_numpy(np.round(noise / UV_PER_BIT).T.copy()).float()
    Xn = Xn - Xn.mean(1, keepdim=True)
    Xn = Xn - torch.median(Xn, 0)[0]
    fwav = _fft_hp(hp, Xn.shape[1])
    Xn = torch.fft.fftshift(torch.real(torch.fft.ifft(torch.fft.fft(Xn) * torch.conj(fwav))), dim=-1)
    Xn = Xn[:, nt:-nt]
    CC = (Xn @ Xn.T) / Xn.shape[1]
    Wrot = st.whitening_local(CC, probe.xc, probe.yc, nrange=min(32, C)).float()

    # temporal basis from the filtered waveforms
    wf = _hp_apply(waves, h64)
    _, _, Vt = np.linalg.svd(wf, full_matrices=False)
    wPCA = Vt[:K].copy()
    for k in range(K):
        if wPCA[k, np.argmax(np.abs(wPCA[k]))] > 0:
            wPCA[k] *= -1
    wPCA = torch.from_numpy(wPCA).float()

    # whitened templates at the median amplitude, projected on the basis
    fp = _footprints(probe.xc, probe.yc, cx, cy)                     # [T, C]
    U = _project_templates(fp, wf, Wrot, wPCA)

    ctc = st.prepare_matching(wPCA, U)
    iCC, iU, Ucc = st.prepare_extract(probe.xc, probe.yc, U, nC)
    iKxx = st.inv_kernel(probe.xc, probe.yc, 20.0)
    setup = SortSetup(probe, fs, NT, nt, nt0min, Th, nC, wPCA, U, ctc.contiguous(), Wrot.contiguous(),
                      hp, iKxx, iCC.contiguous(), iU.contiguous(), Ucc.contiguous())
    units = dict(cx=cx, cy=cy, waves=waves, rates=rates, fp=fp)
    return setup, units


def _project_templates(fp: np.ndarray, wf: np.ndarray, Wrot: torch.Tensor, wPCA: torch.Tensor) -> torch.Tensor:
    """U [T, K, C]: footprints x filtered waveforms at the median amplitude,
    whitened and projected on the temporal basis."""
    amp_bits = 80.0 / UV_PER_BIT
    tmpl = amp_bits * fp[:, :, None] * wf[:, None, :]                # [T, C, nt]
    tw = np.einsum('ij,tjm->tim', Wrot.double().numpy(), tmpl)      # whitened
    return torch.from_numpy(np.einsum('tcm,km->tkc', tw, wPCA.double().numpy())).float().contiguous()


def true_templates(setup: SortSetup, units: dict, fp_shift_um: float = 0.0,
                   fp_scale: np.ndarray | None = None) -> torch.Tensor:
    """Templates of the units as rendered with shifted / scaled footprints
    (the ground truth template refinement should recover)."""
    probe = setup.probe
    wf = _hp_apply(units['waves'], setup.hp_filter.double().numpy())
    scale = np.ones(len(units['cx'])) if fp_scale is None else fp_scale
    fp = _footprints(probe.xc, probe.yc, units['cx'], units['cy'] + fp_shift_um) * scale[:, None]
    return _project_templates(fp, wf, setup.Wrot, setup.wPCA)


def _fft_hp(hp: torch.Tensor, n: int) -> torch.Tensor:
    ft = hp.shape[0]
    if ft < n:
        pad = (n - ft) // 2
        return torch.fft.fft(torch.cat((torch.zeros(pad), hp, torch.zeros(pad + (n - pad * 2 - ft)))))
    if ft > n:
        crop = (ft - n) // 2
        return torch.fft.fft(hp[crop:crop + n])
    return torch.fft.fft(hp)


def render(setup: SortSetup, units: dict, duration_s: float, seed: int,
           drift_um_per_min: float = 0.0, chunk: int = 60000,
           fp_shift_um: float = 0.0, fp_scale: np.ndarray | None = None) -> Recording:
    """Render an int16 recording ``[n_samples, C]`` for the given units."""
    rng = np.random.default_rng(seed)
    fs, nt, nt0min = setup.fs, setup.nt, setup.nt0min
    probe = setup.probe
    C = probe.C
    n = int(round(duration_s * fs))
    T = len(units['rates'])
    refr = int(round(1.5e-3 * fs))
    times, uid = [], []
    for u in range(T):
        mean_isi = fs / units['rates'][u]
        k = int(duration_s * units['rates'][u] * 1.5) + 16
        isi = refr + rng.exponential(mean_isi - refr, k)
        t = np.cumsum(isi).astype(np.int64)
        t = t[(t >= nt) & (t < n - nt)]
        times.append(t)
        uid.append(np.full(len(t), u))
    times = np.concatenate(times)
    uid = np.concatenate(uid)
    order = np.argsort(times, kind='stable')
    times, uid = times[order], uid[order]
    amps = 80.0 * np.exp(0.3 * rng.standard_normal(len(times)))

    raw = np.zeros((n, C), np.int16)
    waves = units['waves']
    cx, cy = units['cx'].copy(), units['cy'] + fp_shift_um
    scale = np.ones(T) if fp_scale is None else fp_scale
    m = np.arange(nt)
    nrng = np.random.default_rng(seed + 1)
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        L = c1 - c0
        drift = drift_um_per_min * ((c0 + c1) / 2 / fs) / 60.0
        fp = _footprints(probe.xc, probe.yc, cx, cy + drift) * scale[:, None]  # [T, C]
        S = np.zeros((L + 2 * nt, T))
        sel = (times > c0 + nt0min - nt) & (times < c1 + nt0min)
        ts, us, a = times[sel], uid[sel], amps[sel]
        rows = (ts - nt0min - c0 + nt)[:, None] + m[None, :]
        np.add.at(S, (rows.ravel(), np.repeat(us, nt)), (a[:, None] * waves[us]).ravel())
        sig = torch.from_numpy(S[nt:nt + L]) @ torch.from_numpy(fp)         # float64 [L, C]
        x = sig.numpy() + _noise(nrng, L, C)
        raw[c0:c1] = np.clip(np.round(x / UV_PER_BIT), -32768, 32767).astype(np.int16)
    NT = setup.NT
    nb = int(np.ceil(n / NT))
    tb = (np.arange(nb) * NT + NT / 2) / fs
    dshift = -drift_um_per_min * tb / 60.0
    return Recording(raw, times, uid, amps, dshift, setup,
                     meta=dict(duration_s=duration_s, drift_um_per_min=drift_um_per_min, seed=seed))


# ------------------------------------------------------------------ configs
def config(index: int, duration_s: float | None = None, seed: int = 0,
           T: int | None = None, C: int | None = None):
    """The five benchmark configurations (``index`` 0-4); ``duration_s``, ``T``
    and ``C`` shrink them for tests.  Returns ``(setup, recording)``."""
    if index == 0:
        probe = probe_two_column(C or 64)
        setup, units = make_setup_and_units(probe, T or 32, seed)
        return setup, render(setup, units, duration_s or 2.0, seed + 100)
    if index in (1, 4):
        probe = probe_staggered(C or 384)
        setup, units = make_setup_and_units(probe, T or 400, seed)
        if index == 1:
            return setup, render(setup, units, duration_s or 60.0, seed + 100, drift_um_per_min=5.0)
        rng = np.random.default_rng(seed + 5)
        sc = rng.uniform(0.9, 1.1, setup.T)
        rec = render(setup, units, duration_s or 32.0, seed + 100, fp_shift_um=10.0, fp_scale=sc)
        rec.meta['U_true'] = true_templates(setup, units, 10.0, sc)
        return setup, rec
    if index == 2:
        probe = probe_staggered(C or 384)
        setup, units = make_setup_and_units(probe, T or 800, seed, dup_frac=0.1)
        return setup, render(setup, units, duration_s or 600.0, seed + 100, drift_um_per_min=5.0)
    raise ValueError(f'config {index}: use streaming_probes() for the multi-probe config')


def streaming_probes(seed: int = 0, duration_s: float = 2.0, Ts=(200, 400, 600, 800), C: int = 384):
    """Four independent probes (config 3) with their own template counts."""
    out = []
    for i, T in enumerate(Ts):
        probe = probe_staggered(C)
        setup, units = make_setup_and_units(probe, T, seed + 31 * i)
        out.append((setup, render(setup, units, duration_s, seed + 31 * i + 100)))
    return out
