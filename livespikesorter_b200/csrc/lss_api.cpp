// C ABI of the sorter (include/lss.h): construction, device memory, and the
// per-batch orchestration of the kernels.
//
// Mirrors OnlineSpikesV2 (src/SpikeSorter/OnlineSpikesV2.cu): the constructor
// path (initializeSorter / allocateMemory / initializeStaticMemory,
// :321-352, :380-422, :470-608) becomes lss_create, which allocates every
// device buffer once; runSpikeSorting's per-batch body (:738-792) becomes
// lss_filter + lss_match / lss_sort_batch. Kilosort semantics are followed
// where LiveSpikeSorter departs from them (round cap 100, strict threshold,
// exact-equality peak test, division by nm, [C, N] residual indexing).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "lss.h"
#include "lss_handle.h"
#include "lss_kernels.cuh"
#include "npy.h"

using namespace lss;

namespace {

thread_local std::string g_create_err;

}  // namespace

// Error text for entry points that have no handle (read back through
// lss_last_error(NULL)).
void lss::set_thread_error(const char* msg) { g_create_err = msg; }


// Circular-correlation taps of the highpass for a batch of N samples: the
// impulse response is zero-padded or centre-cropped to N exactly as
// fft_highpass does (kilosort/preprocessing.py:138-154), fftshift moves its
// centre to lag 0, and the lags beyond L are dropped, L being the smallest
// half-width whose discarded tail holds at most 2^-30 of the L1 mass.
static int make_taps(const std::vector<float>& h, int64_t N, std::vector<float>& taps, std::string& err) {
    const int64_t ft = (int64_t)h.size();
    std::vector<double> g(N, 0.0);
    if (ft < N) {
        const int64_t pad = (N - ft) / 2;
        for (int64_t m = 0; m < ft; ++m) g[pad + m] = h[m];
    } else if (ft > N) {
        const int64_t crop = (ft - N) / 2;
        for (int64_t m = 0; m < N; ++m) g[m] = h[crop + m];
    } else {
        for (int64_t m = 0; m < N; ++m) g[m] = h[m];
    }
    const int64_t c = N / 2;
    const int64_t dlo = -c, dhi = N - 1 - c;
    auto hc = [&](int64_t d) -> double { return (d < dlo || d > dhi) ? 0.0 : g[d + c]; };
    double total = 0.0;
    for (int64_t m = 0; m < N; ++m) total += std::fabs(g[m]);
    const double tol = std::ldexp(total, -30);
    int64_t Lmax = std::max(-dlo, dhi);
    // tail mass beyond L, scanning inwards from the outermost lags
    double tail = 0.0;
    int64_t L = Lmax;
    while (L > 0) {
        const double add = std::fabs(hc(L)) + std::fabs(hc(-L));
        if (tail + add > tol) break;
        tail += add;
        --L;
    }
    const int64_t LCAP = 4096;
    if (L > LCAP) {
        err = "highpass impulse response does not decay within 4096 taps of its centre";
        return -1;
    }
    taps.assign(2 * L + 1, 0.f);
    for (int64_t d = -L; d <= L; ++d) {
        // with an even N the lag +N/2 aliases -N/2; keep a single copy
        if ((N % 2 == 0) && d == N / 2 && L >= N / 2) continue;
        taps[d + L] = (float)hc(d);
    }
    return (int)L;
}

// Whitening with drift: Mw = M @ Wrot on the device (FP32, like the
// reference's (M @ self.whiten_mat), kilosort/io.py:786), or Wrot when M is NULL.
// In-place forward DFT (radix-2, double precision), exp(-2 pi i k n / n).
static void fft_double(std::vector<std::complex<double>>& a) {
    const size_t n = a.size();
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        const double ang = -2.0 * M_PI / (double)len;
        for (size_t i = 0; i < n; i += len)
            for (size_t k = 0; k < len / 2; ++k) {
                const std::complex<double> w(std::cos(ang * k), std::sin(ang * k));
                const std::complex<double> u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
    }
}

int lss::rebuild_uw(lss_handle* h) {
    const int C = h->C;
    // templates with the whitening folded in, for lss_sort_batch
    const bool bf16 = h->cfg.precision == LSS_PREC_BF16_RECHECK;
    // one product, stored as the tf32 split (FP32 path, BF16 re-check) and, on
    // the BF16 path, as the bf16 split too
    CK(launch_build_uw(h->U.p, h->Mw.p, h->T, h->K, C, h->CKpad, bf16 ? h->Uw16.p : nullptr,
                       bf16 ? h->Uw16lo.p : nullptr, h->Uw_hi.p, h->Uw_lo.p, 0));
    h->stats.launches += 1;
    if (bf16) {
        // template norms of the BF16 error bound, for the folded operand and (once
        // per template set: it does not depend on the drift) the plain one
        CK(launch_row_norms(h->Uw_hi.p, h->Uw_lo.p, h->T, h->CKpad, h->un_w.p, 0));
        h->stats.launches += 1;
        if (h->un_p_stale) {
            CK(launch_row_norms(h->Up_hi.p, h->Up_lo.p, h->T, h->CKpad, h->un_p.p, 0));
            h->un_p_stale = false;
            h->stats.launches += 1;
        }
    }
    // callers may sort on streams that do not wait for the legacy default
    // stream: the batch entry points wait for this event on their stream
    if (!h->mix_ev) CK(cudaEventCreateWithFlags(&h->mix_ev, cudaEventDisableTiming));
    CK(cudaEventRecord(h->mix_ev, 0));
    return LSS_OK;
}

// Template rows of the block-skipping rounds, ordered along the probe: by the
// centre of mass, over the channel index, of each template's energy
// sum_k U[t, k, c]^2 (channels follow the probe's geometry in the channel map,
// so templates adjacent in this order sit close together and their
// cross-correlations with distant spikes vanish together). Any order gives the
// same spikes; this one lets whole blocks be skipped. Then the |ctc| maxima per
// (spike template, row).
int lss::rebuild_mp_blocks(lss_handle* h) {
    const int T = h->T, K = h->K, C = h->C, nb = h->mp_nb;
    std::vector<float> u((size_t)T * K * C);
    CK(cudaMemcpy(u.data(), h->U.p, u.size() * sizeof(float), cudaMemcpyDeviceToHost));
    std::vector<double> com(T, 0.0);
    for (int t = 0; t < T; ++t) {
        double w = 0.0, wc = 0.0;
        for (int k = 0; k < K; ++k)
            for (int c = 0; c < C; ++c) {
                const double v = u[((size_t)t * K + k) * C + c];
                w += v * v;
                wc += v * v * c;
            }
        com[t] = w > 0.0 ? wc / w : 0.0;
    }
    std::vector<int32_t> perm((size_t)nb * MPB_ROWS, -1);
    for (int t = 0; t < T; ++t) perm[t] = t;
    std::stable_sort(perm.begin(), perm.begin() + T, [&](int32_t i, int32_t j) { return com[i] < com[j]; });
    std::vector<int32_t> rowof(T);
    for (int r = 0; r < T; ++r) rowof[perm[r]] = r;
    CK(cudaMemcpy(h->mp_perm.p, perm.data(), perm.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->mp_rowof.p, rowof.data(), T * sizeof(int32_t), cudaMemcpyHostToDevice));
    // the rounds read each spike template's ctc rows in the score rows' order
    CK(launch_permute_ctc(h->ctcP.p, h->mp_perm.p, T, 2 * h->nt + 1, h->mp_ctcq.p, 0));
    CK(launch_ctc_row_max(h->mp_ctcq.p, T, 2 * h->nt + 1, h->mp_cmaxr.p, 0));
    CK(cudaDeviceSynchronize());
    h->stats.launches += 1;
    return LSS_OK;
}

int lss::mix_device_drift(lss_handle* h) {
    const int C = h->C;
    CK(launch_sgemm(h->Mdrift.p, C, h->Wrot.p, C, h->Mw.p, C, C, C, C, 0));
    h->stats.launches += 1;
    return rebuild_uw(h);
}

// Drift / whitening change, all on the legacy default stream without a host
// wait: it first waits for the last batch enqueued on any stream (batch_ev),
// the matrix goes through a pinned staging buffer, and the batch entry points
// wait for mix_ev.
static int set_mixing(lss_handle* h, const float* M) {
    const int C = h->C;
    if (h->batch_ev) CK(cudaStreamWaitEvent(0, h->batch_ev, 0));
    if (!M) {
        CK(cudaMemcpyAsync(h->Mw.p, h->Wrot.p, (size_t)C * C * sizeof(float), cudaMemcpyDeviceToDevice, 0));
        return rebuild_uw(h);
    }
    const size_t cc = (size_t)C * C;
    if (!h->m_pin) {
        CK(cudaHostAlloc(reinterpret_cast<void**>(&h->m_pin), lss_handle::M_PIN_SLOTS * cc * sizeof(float),
                         cudaHostAllocDefault));
        for (cudaEvent_t& e : h->m_pin_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    const int k = h->m_pin_next;
    h->m_pin_next = (k + 1) % lss_handle::M_PIN_SLOTS;
    CK(cudaEventSynchronize(h->m_pin_ev[k]));  // the slot's previous upload has left it
    float* slot = h->m_pin + k * cc;
    std::memcpy(slot, M, cc * sizeof(float));
    CK(cudaMemcpyAsync(h->Mdrift.p, slot, cc * sizeof(float), cudaMemcpyHostToDevice, 0));
    CK(cudaEventRecord(h->m_pin_ev[k], 0));
    return mix_device_drift(h);
}

static int validate(const lss_config* c, std::string& err) {
    if (!c) { err = "null config"; return LSS_ERR_ARG; }
    if (c->n_chan <= 0 || c->n_templates <= 0 || c->n_pcs <= 0 || c->nt <= 0 || c->batch_size <= 0) {
        err = "n_chan, n_templates, n_pcs, nt and batch_size must be positive";
        return LSS_ERR_ARG;
    }
    if (c->n_pcs > 8) { err = "n_pcs > 8 is not supported"; return LSS_ERR_ARG; }
    if (c->nt % 2 == 0) { err = "nt must be odd (conv1d with padding nt//2 keeps N columns only then)"; return LSS_ERR_ARG; }
    if (c->nt > 255) { err = "nt > 255 is not supported"; return LSS_ERR_ARG; }
    if (c->n_chan_bin < c->n_chan) { err = "n_chan_bin < n_chan"; return LSS_ERR_ARG; }
    if (c->n_nearest < 0 || c->n_nearest > c->n_chan) { err = "n_nearest out of range"; return LSS_ERR_ARG; }
    if (c->n_nearest * c->n_pcs > 256) { err = "n_nearest * n_pcs > 256"; return LSS_ERR_ARG; }
    if (c->max_rounds <= 0 || c->max_rounds > 1000) { err = "max_rounds must be in 1..1000"; return LSS_ERR_ARG; }
    if (c->max_spikes <= 0) { err = "max_spikes must be positive"; return LSS_ERR_ARG; }
    if (c->precision != LSS_PREC_FP32 && c->precision != LSS_PREC_BF16_RECHECK) {
        err = "unknown precision";
        return LSS_ERR_ARG;
    }
    if (c->n_chan > 1024) { err = "n_chan > 1024 is not supported"; return LSS_ERR_ARG; }
    if (!(c->th_learned > 0.f) || !std::isfinite(c->th_learned)) {
        err = "th_learned must be positive and finite";
        return LSS_ERR_ARG;
    }
    if (c->batch_size > (1 << 26)) { err = "batch_size too large"; return LSS_ERR_ARG; }
    return LSS_OK;
}

// A pointer the kernels running on `device` may dereference: memory of that
// device, managed memory, or pinned host memory (mapped under unified
// addressing). Pageable host memory and another GPU's memory (no peer access
// is enabled) are refused; a null pointer passes (optional arrays).
bool lss::device_accessible(const void* p, int device) {
    if (!p) return true;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeUnregistered) return false;
    if (a.type == cudaMemoryTypeDevice && a.device != device) return false;
    return true;
}

extern "C" {

int lss_create(const lss_config* cfg, const lss_tensors* t, lss_handle** out) {
    if (!out) { g_create_err = "null output pointer"; return LSS_ERR_ARG; }
    *out = nullptr;
    int rc = validate(cfg, g_create_err);
    if (rc) return rc;
    if (!t || !t->wall3 || !t->wpca || !t->ctc || !t->whitening) {
        g_create_err = "wall3, wpca, ctc and whitening are required";
        return LSS_ERR_ARG;
    }
    if (cfg->n_nearest > 0 && (!t->iCC || !t->iU || !t->Ucc)) {
        g_create_err = "iCC, iU and Ucc are required when n_nearest > 0";
        return LSS_ERR_ARG;
    }
    if (cfg->hp_len > 0 && !t->hp_filter) { g_create_err = "hp_len > 0 but hp_filter is NULL"; return LSS_ERR_ARG; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        g_create_err = "no CUDA device available";
        return LSS_ERR_CUDA;
    }
    if (cfg->device < 0 || cfg->device >= ndev) { g_create_err = "device ordinal out of range"; return LSS_ERR_ARG; }
    cudaError_t ce = cudaSetDevice(cfg->device);
    if (ce != cudaSuccess) { g_create_err = cudaGetErrorString(ce); return LSS_ERR_CUDA; }

    std::unique_ptr<lss_handle> hp(new lss_handle());
    lss_handle* h = hp.get();
    h->cfg = *cfg;
    h->C = cfg->n_chan; h->Cbin = cfg->n_chan_bin; h->T = cfg->n_templates; h->K = cfg->n_pcs;
    h->nt = cfg->nt; h->nC = cfg->n_nearest; h->NT = cfg->batch_size;
    h->N = h->NT + 2 * h->nt;
    h->ld = round_up(h->N, 4);
    const int C = h->C, T = h->T, K = h->K, nt = h->nt, nC = h->nC;
    const int64_t ld = h->ld, L2 = 2 * nt + 1;

    if (t->chan_map) {
        for (int c = 0; c < C; ++c)
            if (t->chan_map[c] < 0 || t->chan_map[c] >= h->Cbin) {
                g_create_err = "chan_map entry out of range";
                return LSS_ERR_ARG;
            }
    }
    // template energies nm[t] = sum over (k, c) of U^2 (template_matching.py:141),
    // the exact sum of the FP32 squares rounded once to FP32
    std::vector<float> nmv(T);
    for (int i = 0; i < T; ++i) {
        if (t->nm) { nmv[i] = t->nm[i]; }
        else {
            double acc = 0.0;
            for (int64_t e = 0; e < (int64_t)K * C; ++e) {
                const float u = t->wall3[(int64_t)i * K * C + e];
                acc += (double)(u * u);
            }
            nmv[i] = (float)acc;
        }
        if (!(nmv[i] > 0.f) || !std::isfinite(nmv[i])) {
            g_create_err = "template " + std::to_string(i) + " has zero or non-finite energy";
            return LSS_ERR_ARG;
        }
    }
    if (t->iU) {
        for (int i = 0; i < T; ++i)
            if (t->iU[i] < 0 || t->iU[i] >= C) { g_create_err = "iU entry out of range"; return LSS_ERR_ARG; }
    }
    if (t->iCC && nC > 0) {
        for (int64_t e = 0; e < (int64_t)nC * C; ++e)
            if (t->iCC[e] < 0 || t->iCC[e] >= C) { g_create_err = "iCC entry out of range"; return LSS_ERR_ARG; }
    }
    // U_p[t, c*K + k] = U[t, k, c]; ctcP[j, i, l] = ctc[i, j, l];
    // wave[t, c, m] = sum_k U[t, k, c] * wPCA[k, m] (run_online_spikes.py:539)
    std::vector<float> up((size_t)T * C * K);
    for (int i = 0; i < T; ++i)
        for (int k = 0; k < K; ++k)
            for (int c = 0; c < C; ++c)
                up[((size_t)i * C + c) * K + k] = t->wall3[((size_t)i * K + k) * C + c];
    std::vector<float> wave((size_t)T * C * nt);
    for (int i = 0; i < T; ++i)
        for (int c = 0; c < C; ++c)
            for (int m = 0; m < nt; ++m) {
                double acc = 0.0;
                for (int k = 0; k < K; ++k)
                    acc += (double)t->wall3[((size_t)i * K + k) * C + c] * (double)t->wpca[(size_t)k * nt + m];
                wave[((size_t)i * C + c) * nt + m] = (float)acc;
            }
    if (cfg->hp_len > 0) {
        h->h_hp.assign(t->hp_filter, t->hp_filter + cfg->hp_len);
    }
    std::vector<float> taps;
    if (!h->h_hp.empty()) {
        h->hpL = make_taps(h->h_hp, h->N, taps, g_create_err);
        if (h->hpL < 0) return LSS_ERR_ARG;
    }

    // one CTA per >= 32 columns (a serving loop lowers it further so that
    // its probes' rounds kernels fit on the device together)
    h->mp_grid = std::min<int>(std::min(mp_blocks_max_grid(cfg->device), mp_max_grid(cfg->device)),
                               (int)std::max<int64_t>(1, (h->N + 31) / 32));
    cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, cfg->device);
    h->CKpad = (C * K + 63) / 64 * 64;
    const int64_t cap = cfg->max_spikes;
#define ALLOC(buf, cnt)                                                                    \
    do {                                                                                   \
        cudaError_t e_ = h->buf.alloc(cnt);                                                \
        h->dev_bytes += std::max<size_t>(h->buf.n, 1) * sizeof(*h->buf.p);                 \
        if (e_ != cudaSuccess) {                                                           \
            g_create_err = std::string("cudaMalloc " #buf ": ") + cudaGetErrorString(e_);  \
            return LSS_ERR_CUDA;                                                           \
        }                                                                                  \
    } while (0)
    ALLOC(raw, (size_t)h->N * h->Cbin);
    ALLOC(chan_map, C);
    ALLOC(sums, C);
    ALLOC(taps, std::max<size_t>(taps.size(), 1));
    ALLOC(Mw, (size_t)C * C);
    ALLOC(Wrot, (size_t)C * C);
    ALLOC(Mdrift, (size_t)C * C);
    ALLOC(X1, (size_t)C * ld);
    ALLOC(Xh, (size_t)C * ld);
    ALLOC(X, (size_t)C * ld);
    const bool bf16 = cfg->precision == LSS_PREC_BF16_RECHECK;
    const TcPlan plan = tc_plan(T, bf16 ? TC_BF16X3 : TC_TF32X3);
    if (plan.stages < 2) {
        g_create_err = "too many templates for the tensor-core score GEMM's shared memory";
        return LSS_ERR_ARG;
    }
    if (bf16) {
        if (tc_plan(T, TC_TF32X3).stages < 2) {
            g_create_err = "too many templates for the FP32 re-check GEMM's shared memory";
            return LSS_ERR_ARG;
        }
        ALLOC(B0T, (size_t)h->N * h->CKpad);
        ALLOC(B0T16lo, (size_t)h->N * h->CKpad);
        ALLOC(Up16, (size_t)plan.Tpad * h->CKpad);
        ALLOC(Up16lo, (size_t)plan.Tpad * h->CKpad);
        ALLOC(Uw16, (size_t)plan.Tpad * h->CKpad);
        ALLOC(Uw16lo, (size_t)plan.Tpad * h->CKpad);
        // FP32 re-check of open decisions: projection rows of the listed columns, bookkeeping
        const size_t rc_rows = (size_t)(h->N + 127) / 128 * 128;
        ALLOC(Pc_hi, rc_rows * h->CKpad);
        ALLOC(Pc_lo, rc_rows * h->CKpad);
        ALLOC(cf2, ld);
        ALLOC(cf_lo, ld);
        ALLOC(cf_hi, ld);
        ALLOC(pn2, ld);
        ALLOC(un_w, T);
        ALLOC(un_p, T);
        ALLOC(pre_cf, ld);
        ALLOC(pre_im, ld);
        ALLOC(rc_cols, ld);
        ALLOC(rc_count, 4);
        if (cudaMallocHost(&h->rc_host, 4 * sizeof(int32_t)) != cudaSuccess) {
            g_create_err = "pinned host allocation failed";
            return LSS_ERR_CUDA;
        }
        memset(h->rc_host, 0, 4 * sizeof(int32_t));
        if (cudaEventCreateWithFlags(&h->rc_ev, cudaEventDisableTiming) != cudaSuccess) {
            g_create_err = "event creation failed";
            return LSS_ERR_CUDA;
        }
    } else {
        ALLOC(B0T_hi, (size_t)h->N * h->CKpad);
        ALLOC(B0T_lo, (size_t)h->N * h->CKpad);
    }
    // tf32 template splits: the FP32 path's scores, and the BF16 path's re-check
    const int Tpad32 = tc_plan(T, TC_TF32X3).Tpad;
    ALLOC(Up_hi, (size_t)Tpad32 * h->CKpad);
    ALLOC(Up_lo, (size_t)Tpad32 * h->CKpad);
    ALLOC(Uw_hi, (size_t)Tpad32 * h->CKpad);
    ALLOC(Uw_lo, (size_t)Tpad32 * h->CKpad);
    ALLOC(U, (size_t)T * K * C);
    const bool hp_fft = h->hpL >= 0 && h->hpL <= 1024;
    if (hp_fft) {
        ALLOC(hpH, 4096);
        ALLOC(hpTw, 4096);
    }
    ALLOC(R, (size_t)K * K * (2 * nt - 1));
    ALLOC(B, (size_t)T * ld);
    ALLOC(nm, T);
    ALLOC(ctcP, (size_t)T * T * L2);
    ALLOC(wave, (size_t)T * C * nt);
    ALLOC(wpca, (size_t)K * nt);
    ALLOC(Ucc, (size_t)std::max(nC, 1) * T * K);
    ALLOC(iCC, (size_t)std::max(nC, 1) * C);
    ALLOC(iU, T);
    ALLOC(Xres, (size_t)C * ld);
    ALLOC(tF, (size_t)cap * std::max(nC * K, 1));
    ALLOC(cfmax, ld);
    ALLOC(imax, ld);
    ALLOC(colkey, 2 * ld);
    h->mp_nb = (T + MPB_ROWS - 1) / MPB_ROWS;
    // the block-skipping rounds pay off from a few hundred templates on (more
    // rows per block far from a spike); below, updating every row is faster
    h->mp_skip = T >= 600;
    ALLOC(mp_perm, (size_t)h->mp_nb * MPB_ROWS);
    ALLOC(mp_cmaxr, (size_t)T * T);
    ALLOC(mp_rowof, T);
    {
        const int64_t passes = ((T + 15) / 16 * 16 + 255) / 256;  // the score GEMM's template passes
        ALLOC(sc_part_keys, (size_t)(passes * ld));
        ALLOC(sc_part, (size_t)(4 * passes * ld));
    }
    ALLOC(mp_ctcq, (size_t)T * T * L2);
    ALLOC(mp_bkey, (size_t)h->mp_nb * ld);
    ALLOC(mp_phase, 6);
    // 4 int4 per list entry
    ALLOC(mp_ent, (size_t)mp_blocks_list_entries(ld, nt, T, h->mp_grid) * 4);
    ALLOC(mp_ent_cnt, (size_t)h->mp_grid);
    ALLOC(mp_bmin, (size_t)h->mp_nb * ld);
    ALLOC(blk_cnt, 4096);
    ALLOC(blk_x, ld);
    ALLOC(blk_y, ld);
    ALLOC(blk_amp, ld);
    ALLOC(sp_x, cap);
    ALLOC(sp_y, cap);
    ALLOC(sp_amp, cap);
    ALLOC(sp_round, cap);
    ALLOC(round_start, cfg->max_rounds + 2);
    ALLOC(counters, 4);
    ALLOC(status, 1);
    ALLOC(bar, 2);
    ALLOC(rec_time, cap);
    ALLOC(rec_tmpl, cap);
    ALLOC(rec_slot, cap);
    ALLOC(rec_amp, cap);
    ALLOC(rec_pc, (size_t)cap * std::max(nC * K, 1));
    ALLOC(rec_count, 1);
#undef ALLOC

    // ctc[i, j, l] -> ctcP[j, i, l], streamed through a host staging row
    {
        std::vector<float> row((size_t)T * L2);
        for (int j = 0; j < T; ++j) {
            for (int i = 0; i < T; ++i)
                std::memcpy(&row[(size_t)i * L2], t->ctc + ((size_t)i * T + j) * L2, L2 * sizeof(float));
            CK(cudaMemcpy(h->ctcP.p + (size_t)j * T * L2, row.data(), row.size() * sizeof(float),
                          cudaMemcpyHostToDevice));
        }
    }
    std::vector<int32_t> cmap(C);
    for (int c = 0; c < C; ++c) cmap[c] = t->chan_map ? t->chan_map[c] : c;
    CK(cudaMemcpy(h->chan_map.p, cmap.data(), C * sizeof(int32_t), cudaMemcpyHostToDevice));
    if (!taps.empty()) CK(cudaMemcpy(h->taps.p, taps.data(), taps.size() * sizeof(float), cudaMemcpyHostToDevice));
    if (bf16) {
        // U_p as the bf16 split hi = bf16(x), lo = bf16(x - hi), [Tpad, CKpad] with zero padding
        std::vector<__nv_bfloat16> u16((size_t)plan.Tpad * h->CKpad, __float2bfloat16(0.f)), u16lo(u16);
        for (int i = 0; i < T; ++i)
            for (int e = 0; e < C * K; ++e) {
                const float x = up[(size_t)i * C * K + e];
                const __nv_bfloat16 hb = __float2bfloat16(x);
                u16[(size_t)i * h->CKpad + e] = hb;
                u16lo[(size_t)i * h->CKpad + e] = __float2bfloat16(x - __bfloat162float(hb));
            }
        CK(cudaMemcpy(h->Up16.p, u16.data(), u16.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->Up16lo.p, u16lo.data(), u16lo.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
        CK(cudaMemset(h->B0T.p, 0, (size_t)h->N * h->CKpad * sizeof(__nv_bfloat16)));
        CK(cudaMemset(h->B0T16lo.p, 0, (size_t)h->N * h->CKpad * sizeof(__nv_bfloat16)));
        const size_t rc_bytes = (size_t)(h->N + 127) / 128 * 128 * h->CKpad * sizeof(float);
        CK(cudaMemset(h->Pc_hi.p, 0, rc_bytes));
        CK(cudaMemset(h->Pc_lo.p, 0, rc_bytes));
    }
    {
        // U_p split into tf32 parts, each rounded half away like cvt.rna.tf32.f32:
        // hi = rna(x), lo = rna(x - hi)
        auto rna = [](float x) {
            uint32_t u;
            std::memcpy(&u, &x, 4);
            if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
            float r;
            std::memcpy(&r, &u, 4);
            return r;
        };
        std::vector<float> hi((size_t)Tpad32 * h->CKpad, 0.f), lo(hi.size(), 0.f);
        for (int i = 0; i < T; ++i)
            for (int e = 0; e < C * K; ++e) {
                const float x = up[(size_t)i * C * K + e];
                const float xh = rna(x);
                hi[(size_t)i * h->CKpad + e] = xh;
                lo[(size_t)i * h->CKpad + e] = rna(x - xh);
            }
        CK(cudaMemcpy(h->Up_hi.p, hi.data(), hi.size() * sizeof(float), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->Up_lo.p, lo.data(), lo.size() * sizeof(float), cudaMemcpyHostToDevice));
        if (!bf16) {
            CK(cudaMemset(h->B0T_hi.p, 0, (size_t)h->N * h->CKpad * sizeof(float)));
            CK(cudaMemset(h->B0T_lo.p, 0, (size_t)h->N * h->CKpad * sizeof(float)));
        }
    }
    CK(cudaMemcpy(h->nm.p, nmv.data(), T * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->wave.p, wave.data(), wave.size() * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->wpca.p, t->wpca, (size_t)K * nt * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->U.p, t->wall3, (size_t)T * K * C * sizeof(float), cudaMemcpyHostToDevice));
    if (hp_fft) {
        // g = taps wrapped around index 0 (circular correlation), H = conj(FFT(g))
        const int F = 4096, L = h->hpL;
        std::vector<std::complex<double>> g(F, 0.0);
        g[0] = taps[L];
        for (int d = 1; d <= L; ++d) {
            g[d] = taps[L + d];
            g[F - d] = taps[L - d];
        }
        fft_double(g);
        std::vector<float2> hv(F), tv(F);
        for (int k = 0; k < F; ++k) {
            hv[k] = make_float2((float)g[k].real(), (float)-g[k].imag());
            const double ang = -2.0 * M_PI * k / F;
            tv[k] = make_float2((float)std::cos(ang), (float)std::sin(ang));
        }
        CK(cudaMemcpy(h->hpH.p, hv.data(), F * sizeof(float2), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->hpTw.p, tv.data(), F * sizeof(float2), cudaMemcpyHostToDevice));
    }
    {
        // R[k, k', d] = sum_m wPCA[k, m] * wPCA[k', m + d], d = -(nt-1) .. nt-1
        const int nd = 2 * nt - 1;
        std::vector<float> r((size_t)K * K * nd);
        for (int k = 0; k < K; ++k)
            for (int k2 = 0; k2 < K; ++k2)
                for (int d = -(nt - 1); d <= nt - 1; ++d) {
                    double acc = 0.0;
                    for (int m = 0; m < nt; ++m)
                        if (m + d >= 0 && m + d < nt)
                            acc += (double)t->wpca[(size_t)k * nt + m] * t->wpca[(size_t)k2 * nt + m + d];
                    r[((size_t)k * K + k2) * nd + (d + nt - 1)] = (float)acc;
                }
        CK(cudaMemcpy(h->R.p, r.data(), r.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    if (bf16) {
        CK(cudaMemset(h->Uw16.p, 0, (size_t)plan.Tpad * h->CKpad * sizeof(__nv_bfloat16)));
        CK(cudaMemset(h->Uw16lo.p, 0, (size_t)plan.Tpad * h->CKpad * sizeof(__nv_bfloat16)));
    }
    CK(cudaMemset(h->Uw_hi.p, 0, (size_t)Tpad32 * h->CKpad * sizeof(float)));
    CK(cudaMemset(h->Uw_lo.p, 0, (size_t)Tpad32 * h->CKpad * sizeof(float)));
    if (nC > 0) {
        CK(cudaMemcpy(h->Ucc.p, t->Ucc, (size_t)nC * T * K * sizeof(float), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->iCC.p, t->iCC, (size_t)nC * C * sizeof(int64_t), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->iU.p, t->iU, (size_t)T * sizeof(int64_t), cudaMemcpyHostToDevice));
    }
    CK(cudaMemset(h->colkey.p, 0, 2 * ld * sizeof(unsigned long long)));
    CK(h->status_acc.alloc(1));
    h->dev_bytes += 256;
    CK(cudaMemset(h->status_acc.p, 0, sizeof(int32_t)));
    CK(cudaEventCreateWithFlags(&h->batch_ev, cudaEventDisableTiming));
    CK(cudaMemcpy(h->Wrot.p, t->whitening, (size_t)C * C * sizeof(float), cudaMemcpyHostToDevice));
    rc = set_mixing(h, t->drift);
    if (rc) { g_create_err = h->err; return rc; }
    rc = rebuild_mp_blocks(h);
    if (rc) { g_create_err = h->err; return rc; }
    // the set-up work is on the legacy stream; waiting for it alone leaves
    // other handles' non-blocking streams (a serving loop's probes) running
    CK(cudaStreamSynchronize(0));
    *out = hp.release();
    return LSS_OK;
}

void lss_destroy(lss_handle* h) { delete h; }

const char* lss_last_error(const lss_handle* h) { return h ? h->err.c_str() : g_create_err.c_str(); }

int lss_get_config(const lss_handle* h, lss_config* out) {
    if (!h || !out) return LSS_ERR_ARG;
    *out = h->cfg;
    return LSS_OK;
}

int lss_get_stats(const lss_handle* h, lss_stats* out) {
    if (!h || !out) return LSS_ERR_ARG;
    *out = h->stats;
    if (h->rc_pending) {
        // re-check counts of the last BF16 scoring, copied back asynchronously
        const cudaError_t e = cudaEventSynchronize(h->rc_ev);
        if (e != cudaSuccess) {
            lss::set_thread_error((std::string("lss_get_stats: ") + cudaGetErrorString(e)).c_str());
            return LSS_ERR_CUDA;
        }
        out->recheck_columns = h->rc_host[2];
        out->recheck_flips = h->rc_host[1];
        out->recheck_rescored = h->rc_host[0];
    }
    return LSS_OK;
}

int lss_set_round_kernel(lss_handle* h, int32_t skip_blocks) {
    if (!h || (skip_blocks != 0 && skip_blocks != 1)) return LSS_ERR_ARG;
    if (h->streaming) return h->fail(LSS_ERR_STATE, "handle is owned by a serving loop");
    h->mp_skip = skip_blocks != 0;
    return LSS_OK;
}

int lss_get_round_kernel(const lss_handle* h, int32_t* skip_blocks) {
    if (!h || !skip_blocks) return LSS_ERR_ARG;
    *skip_blocks = h->mp_skip ? 1 : 0;
    return LSS_OK;
}

int lss_set_drift(lss_handle* h, const float* M) {
    if (!h) return LSS_ERR_ARG;
    if (h->streaming) return h->fail(LSS_ERR_STATE, "handle is owned by a serving loop");
    CK(cudaSetDevice(h->cfg.device));
    return set_mixing(h, M);
}

}  // extern "C"

// ---------------------------------------------------------------- stages
// Ingest of one padded batch. Xout (may be null) receives the whitened,
// drift-corrected batch; *pre_out the highpassed batch before whitening.
// The rows of a batch that are read (Kilosort's batch layout): the first
// batch is NT + nt rows with the nt leading ones replicated, the last may be
// short, the others are NT + 2nt.
static int batch_map(lss_handle* h, const int16_t* raw, int64_t n_rows, int64_t ibatch, int64_t n_batches,
                     IngestMap& map) {
    if (!raw || n_rows <= 0) return h->fail(LSS_ERR_ARG, "empty raw batch");
    if (ibatch < 0 || n_batches <= 0 || ibatch >= n_batches) return h->fail(LSS_ERR_ARG, "ibatch out of range");
    const int64_t N = h->N;
    map = IngestMap{};
    if (ibatch == 0) {
        map.lead = h->nt;
        map.nsamp = std::min<int64_t>(n_rows, h->NT + h->nt);
        map.zero_tail = 1;
    } else if (ibatch == n_batches - 1) {
        map.lead = 0;
        map.nsamp = std::min<int64_t>(n_rows, N);
        map.zero_tail = 0;
    } else {
        if (n_rows < N)
            return h->fail(LSS_ERR_SHAPE, "a middle batch needs NT + 2*nt rows (" + std::to_string(N) + ")");
        map.lead = 0;
        map.nsamp = N;
        map.zero_tail = 0;
    }
    return LSS_OK;
}

static int run_filter(lss_handle* h, const int16_t* raw, int64_t n_rows, int64_t ibatch, int64_t n_batches,
                      int32_t raw_on_device, float* Xout, cudaStream_t s, const float** pre_out = nullptr) {
    IngestMap map;
    int rc = batch_map(h, raw, n_rows, ibatch, n_batches, map);
    if (rc) return rc;
    const int16_t* src = raw;
    h->mark(0, s);
    if (!raw_on_device) {
        CK(cudaMemcpyAsync(h->raw.p, raw, (size_t)map.nsamp * h->Cbin * sizeof(int16_t), cudaMemcpyHostToDevice, s));
        src = h->raw.p;
    }
    h->mark(1, s);
    return run_ingest(h, src, map, Xout, s, pre_out);
}

int lss::run_ingest(lss_handle* h, const int16_t* src, const IngestMap& map, float* Xout, cudaStream_t s,
                    const float** pre_out) {
    const int64_t N = h->N;
    const float sign = h->cfg.invert_sign ? -1.f : 1.f;
    CK(launch_chan_sums(src, h->Cbin, h->chan_map.p, h->C, N, map, h->sums.p, s));
    CK(launch_car(src, h->Cbin, h->chan_map.p, h->C, N, map, sign, h->sums.p, h->cfg.do_car, h->X1.p, h->ld, s));
    h->stats.launches += 2;
    h->mark(2, s);
    const float* pre = h->X1.p;
    if (h->hpL >= 0) {
        if (h->hpH.p)
            CK(launch_highpass_fft(h->X1.p, h->ld, h->C, N, h->hpL, h->hpH.p, h->hpTw.p, h->Xh.p, s));
        else
            CK(launch_highpass(h->X1.p, h->ld, h->C, N, h->taps.p, h->hpL, h->Xh.p, s));
        h->stats.launches += 1;
        pre = h->Xh.p;
    }
    h->mark(3, s);
    if (Xout) {
        CK(launch_sgemm(h->Mw.p, h->C, pre, h->ld, Xout, h->ld, h->C, (int)N, h->C, s));
        h->stats.launches += 1;
    }
    h->mark(4, s);
    if (pre_out) *pre_out = pre;
    return LSS_OK;
}

int lss::run_scores(lss_handle* h, const float* X, int64_t ldx, int64_t N, float* B, cudaStream_t s,
                   bool* maxima_ready, bool folded, bool rows_for_mp) {
    const int32_t* rowof = (rows_for_mp && h->mp_skip) ? h->mp_rowof.p : nullptr;
    if (h->cfg.precision == LSS_PREC_BF16_RECHECK) {
        CK(launch_pca_proj_t(X, ldx, h->C, N, h->wpca.p, h->K, h->nt, h->B0T.p, h->B0T16lo.p, h->CKpad, s, h->pn2.p));
        h->mark(5, s);
        TcExtra ex;
        ex.cf2 = h->cf2.p;
        ex.un = folded ? h->un_w.p : h->un_p.p;
        ex.pn2 = h->pn2.p;
        // |B - B_fp32| <= eps ||U_t|| ||P_s||: 3 * 2^-18 for the dropped lo*lo term
        // and the rounding of the lo parts, plus FP32 accumulation over CKpad
        // terms in both paths (CKpad * 2^-24 each)
        ex.eps = (float)(3.0 * std::ldexp(1.0, -18) * 1.01 + 2.0 * h->CKpad * std::ldexp(1.0, -24));
        ex.cf_lo = h->cf_lo.p;
        ex.cf_hi = h->cf_hi.p;
        ex.rowof = rowof;
        ex.part_keys = h->sc_part_keys.p;
        ex.part = h->sc_part.p;
        ex.part_cap = (int64_t)h->sc_part_keys.n;
        CK(launch_score_tc_bf16x3(h->B0T.p, h->B0T16lo.p, h->CKpad, (int)N, folded ? h->Uw16.p : h->Up16.p,
                                  folded ? h->Uw16lo.p : h->Up16lo.p, h->T, h->CKpad, h->nm.p, B, h->ld, h->cfmax.p,
                                  h->imax.p, h->nt, h->status.p, h->sm_count, s, ex));
        // FP32 re-check of the columns whose first-round decisions the BF16
        // error bound leaves open; the column list and its length stay on the
        // device
        const float th2 = h->cfg.th_learned * h->cfg.th_learned;
        CK(launch_recheck_select(h->cf_lo.p, h->cf_hi.p, h->cf2.p, h->cfmax.p, h->imax.p, (int)N, h->nt, th2,
                                 h->rc_cols.p, h->pre_cf.p, h->pre_im.p, h->rc_count.p, s));
        CK(launch_pca_proj_cols_tf32(X, ldx, h->C, N, h->wpca.p, h->K, h->nt, h->rc_cols.p, h->rc_count.p, (int)N,
                                     h->Pc_hi.p, h->Pc_lo.p, h->CKpad, 0, s));
        TcExtra ex2;
        ex2.rowmap = h->rc_cols.p;
        ex2.map_rows = 1;
        ex2.count_dev = h->rc_count.p;
        ex2.ncols = (int)N;
        ex2.rowof = rowof;
        ex2.keys = h->colkey.p;  // templates split over CTAs; free until the rounds start (they clear it)
        const int max_rows = (int)((N + 127) / 128 * 128);
        CK(launch_score_tc_tf32x3(h->Pc_hi.p, h->Pc_lo.p, h->CKpad, max_rows, folded ? h->Uw_hi.p : h->Up_hi.p,
                                  folded ? h->Uw_lo.p : h->Up_lo.p, h->T, h->CKpad, h->nm.p, B, h->ld, h->cfmax.p,
                                  h->imax.p, h->nt, h->status.p, h->sm_count, s, ex2));
        CK(launch_recheck_flips(h->cfmax.p, h->imax.p, h->rc_cols.p, h->pre_cf.p, h->pre_im.p, h->rc_count.p, (int)N,
                                th2, s));
        if (!h->capturing) {
            CK(cudaMemcpyAsync(h->rc_host, h->rc_count.p, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            CK(cudaEventRecord(h->rc_ev, s));
            h->rc_pending = true;
            h->last_scored = N;
        }
        h->stats.launches += 7 + (h->T > 256 ? 1 : 0);  // + the bounds finalize of a multi-pass GEMM
        h->mark(6, s);
        if (maxima_ready) *maxima_ready = true;
        return LSS_OK;
    }
    CK(launch_pca_proj_t_tf32(X, ldx, h->C, N, h->wpca.p, h->K, h->nt, h->B0T_hi.p, h->B0T_lo.p, h->CKpad, s));
    h->mark(5, s);
    TcExtra ex;
    ex.keys = h->colkey.p;  // free until the rounds start (they clear it)
    ex.rowof = rowof;
    CK(launch_score_tc_tf32x3(h->B0T_hi.p, h->B0T_lo.p, h->CKpad, (int)N, folded ? h->Uw_hi.p : h->Up_hi.p,
                              folded ? h->Uw_lo.p : h->Up_lo.p, h->T, h->CKpad, h->nm.p, B, h->ld, h->cfmax.p,
                              h->imax.p, h->nt, h->status.p, h->sm_count, s, ex));
    h->stats.launches += 2 + (h->T > 256 ? 1 : 0);  // + the key maxima of a multi-pass GEMM
    h->mark(6, s);
    if (maxima_ready) *maxima_ready = true;
    return LSS_OK;
}

int lss::enqueue_mp(lss_handle* h, int64_t N, cudaStream_t s, bool maxima_ready) {
    if (N <= 2 * h->nt) return h->fail(LSS_ERR_ARG, "batch shorter than 2*nt + 1 samples");
    MPArgs a{};
    a.B = h->B.p;
    a.ldb = h->ld;
    a.T = h->T;
    a.N = (int)N;
    a.nt = h->nt;
    a.th2 = h->cfg.th_learned * h->cfg.th_learned;
    a.nm = h->nm.p;
    a.ctcP = h->ctcP.p;
    a.cfmax = h->cfmax.p;
    a.imax = h->imax.p;
    a.colkey = h->colkey.p;
    a.ldk = h->ld;
    a.blk_cnt = h->blk_cnt.p;
    a.blk_x = h->blk_x.p;
    a.blk_y = h->blk_y.p;
    a.blk_amp = h->blk_amp.p;
    a.sp_x = h->sp_x.p;
    a.sp_y = h->sp_y.p;
    a.sp_amp = h->sp_amp.p;
    a.sp_round = h->sp_round.p;
    a.round_start = h->round_start.p;
    a.capacity = h->cfg.max_spikes;
    a.max_rounds = h->cfg.max_rounds;
    a.counters = h->counters.p;
    a.status = h->status.p;
    a.bar = h->bar.p;
    const int G = h->mp_grid;
    a.cols_per_blk = (int)((N + G - 1) / G);
    if (!maxima_ready) CK(cudaMemsetAsync(h->status.p, 0, sizeof(int32_t), s));
    CK(cudaMemsetAsync(h->counters.p, 0, 4 * sizeof(int32_t), s));
    CK(cudaMemsetAsync(h->mp_phase.p, 0, 6 * sizeof(unsigned long long), s));
    a.phase = h->mp_phase.p;
    if (h->mp_skip) {
        a.perm = h->mp_perm.p;
        a.nb = h->mp_nb;
        a.cmaxr = h->mp_cmaxr.p;
        a.bkey = h->mp_bkey.p;
        a.bmin = h->mp_bmin.p;
        a.ctcP = h->mp_ctcq.p;
        a.ment = h->mp_ent.p;
        a.ment_cnt = h->mp_ent_cnt.p;
        a.ment_cap = (int32_t)std::min<int64_t>(h->mp_ent.n / 4 / G, INT32_MAX);
        a.init_cols = 1;  // the rounds take their block maxima from the field itself
        CK(launch_mp_blocks(a, G, s));
    } else {
        a.init_cols = maxima_ready ? 0 : 1;
        CK(cudaMemsetAsync(h->colkey.p, 0, 2 * h->ld * sizeof(unsigned long long), s));
        CK(launch_mp(a, G, s));
    }
    h->stats.launches += 1;
    return LSS_OK;
}

// Runs the rounds on h->B (already holding the score field); returns spikes.
static int run_mp(lss_handle* h, int64_t N, int32_t* n_out, int32_t* rounds_out, cudaStream_t s,
                  bool maxima_ready = false) {
    int rc = enqueue_mp(h, N, s, maxima_ready);
    if (rc) return rc;
    int32_t hc[4], st = 0;
    CK(cudaMemcpyAsync(hc, h->counters.p, sizeof(hc), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h->mp_phase_host, h->mp_phase.p, sizeof(h->mp_phase_host), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&st, h->status.p, sizeof(st), cudaMemcpyDeviceToHost, s));
    h->mark(7, s);
    CK(cudaStreamSynchronize(s));
    if (st & STATUS_TIMEOUT) return h->fail(LSS_ERR_TIMEOUT, "matching pursuit grid barrier timed out");
    if (st & STATUS_LIST) return h->fail(LSS_ERR_CAPACITY, MSG_MP_LIST);
    if (st & STATUS_CAPACITY)
        return h->fail(LSS_ERR_CAPACITY, "more than max_spikes spikes in one batch");
    *n_out = hc[0];
    *rounds_out = hc[1];
    h->stats.rounds = hc[1];
    h->stats.spikes = hc[0];
    h->stats.mp_items_updated = hc[2];
    h->stats.mp_items = hc[3];
    h->set_phase_stats();
    return LSS_OK;
}

static int run_xres(lss_handle* h, const float* X, int64_t ldx, int64_t N, int rounds, float* Xres,
                    int64_t ldr, cudaStream_t s) {
    (void)ldr;
    CK(launch_xres(X, ldx, h->C, (int)N, h->nt, h->wave.p, h->sp_x.p, h->sp_y.p, h->sp_amp.p,
                   h->round_start.p, h->counters.p, rounds, Xres, h->status.p, s));
    h->stats.launches += 1;
    return LSS_OK;
}

int lss::enqueue_records(lss_handle* h, const RecordClock& rc_in, int32_t n_bound, bool with_pc, bool tf_ready,
                         int64_t* time, int32_t* tmpl, float* amp, float* pc, float* x, float* y, int32_t* clu,
                         int64_t cap, int64_t* count, cudaStream_t s) {
    RecordClock rc = rc_in;
    const int feat = h->nC * h->K;
    if (h->post) {
        PostArgs a = h->pa;
        a.tF = tf_ready ? h->tF.p : nullptr;
        CK(launch_post(a, rc, n_bound, h->rec_slot.p, count, s));
        rc.presorted = 1;
        h->stats.launches += 5;
    }
    CK(launch_records(h->sp_x.p, h->sp_y.p, h->sp_amp.p, with_pc ? h->tF.p : nullptr, h->rec_slot.p, n_bound, feat,
                      rc, time, tmpl, amp, pc, cap, count, s));
    h->stats.launches += (n_bound > 0) ? 2 : 1;
    if (h->post && (x || y || clu)) {
        CK(launch_post_write(h->pa, rc, h->rec_slot.p, n_bound, x, y, clu, cap, s));
        h->stats.launches += 1;
    }
    return LSS_OK;
}

extern "C" {

int lss_reset_postprocess(lss_handle* h) {
    if (!h) return LSS_ERR_ARG;
    if (!h->post) return LSS_OK;
    CK(cudaSetDevice(h->cfg.device));
    std::vector<int64_t> init(h->plast.n, -(int64_t(1) << 62));
    CK(cudaMemcpy(h->plast.p, init.data(), init.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
    return LSS_OK;
}

int lss_set_postprocess(lss_handle* h, const lss_post_config* pc) {
    if (!h) return LSS_ERR_ARG;
    if (h->streaming) return h->fail(LSS_ERR_STATE, "handle is owned by a serving loop");
    CK(cudaSetDevice(h->cfg.device));
    if (!pc) {
        h->post = false;
        return LSS_OK;
    }
    if (pc->n_clusters < 0 || pc->dt_samples < 0 || (pc->n_clusters > 0 && !pc->centroids_xy))
        return h->fail(LSS_ERR_ARG, "bad post-processing config");
    if ((pc->xc == nullptr) != (pc->yc == nullptr)) return h->fail(LSS_ERR_ARG, "give both xc and yc or neither");
    if (pc->xc && (h->nC <= 0 || !h->iCC.p)) return h->fail(LSS_ERR_STATE, "positions need iCC / iU / Ucc");
    if (pc->n_clusters > 0 && !pc->xc) return h->fail(LSS_ERR_ARG, "clusters need channel positions");
    if (h->nC > 16) return h->fail(LSS_ERR_ARG, "positions support at most 16 nearest channels");
    if (h->N >= (1 << 20) || h->cfg.max_spikes >= (1 << 20))
        return h->fail(LSS_ERR_ARG, "post-processing keys need batches and spike lists below 2^20");
    const int64_t nmax = h->cfg.max_spikes;
    const size_t sort_bytes = post_sort_bytes((int32_t)nmax);
    auto al = [&](auto& buf, size_t n) -> cudaError_t {
        if (buf.p) h->dev_bytes -= std::max<size_t>(buf.n, 1) * sizeof(*buf.p);
        buf.release();
        cudaError_t e = buf.alloc(n);
        if (e == cudaSuccess) h->dev_bytes += std::max<size_t>(n, 1) * sizeof(*buf.p);
        return e;
    };
    const int nclu = pc->n_clusters > 0 ? pc->n_clusters : h->T;
    CK(al(h->pk, 4 * (size_t)nmax));
    CK(al(h->psort, sort_bytes));
    CK(al(h->pkeep, (size_t)nmax));
    CK(al(h->plast, (size_t)nclu));
    CK(al(h->pxy, 2 * (size_t)nmax));
    CK(al(h->pclu, (size_t)nmax));
    CK(al(h->rec_x, (size_t)nmax));
    CK(al(h->rec_y, (size_t)nmax));
    CK(al(h->rec_clu, (size_t)nmax));
    CK(al(h->pcen, 2 * (size_t)std::max(pc->n_clusters, 1)));
    CK(al(h->pchan, 2 * (size_t)h->C));
    PostArgs a;
    a.sp_x = h->sp_x.p;
    a.sp_y = h->sp_y.p;
    a.nC = h->nC;
    a.K = h->K;
    a.C = h->C;
    a.iCC = h->iCC.p;
    a.iU = h->iU.p;
    if (pc->xc) {
        CK(cudaMemcpy(h->pchan.p, pc->xc, h->C * sizeof(float), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->pchan.p + h->C, pc->yc, h->C * sizeof(float), cudaMemcpyHostToDevice));
        a.xc = h->pchan.p;
        a.yc = h->pchan.p + h->C;
    }
    if (pc->n_clusters > 0) {
        std::vector<float> cx(pc->n_clusters), cy(pc->n_clusters);
        for (int i = 0; i < pc->n_clusters; ++i) {
            cx[i] = pc->centroids_xy[2 * i];
            cy[i] = pc->centroids_xy[2 * i + 1];
        }
        CK(cudaMemcpy(h->pcen.p, cx.data(), cx.size() * sizeof(float), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->pcen.p + pc->n_clusters, cy.data(), cy.size() * sizeof(float), cudaMemcpyHostToDevice));
        a.cen_x = h->pcen.p;
        a.cen_y = h->pcen.p + pc->n_clusters;
        a.n_clu = pc->n_clusters;
    }
    a.dt = pc->dt_samples;
    a.key_c = h->pk.p;
    a.key_c_sorted = h->pk.p + nmax;
    a.key_t = h->pk.p + 2 * nmax;
    a.key_t_sorted = h->pk.p + 3 * nmax;
    a.sort_tmp = h->psort.p;
    a.sort_bytes = sort_bytes;
    a.keep = h->pkeep.p;
    a.last_time = h->plast.p;
    a.px = h->pxy.p;
    a.py = h->pxy.p + nmax;
    a.clu = h->pclu.p;
    h->pa = a;
    h->post = true;
    return lss_reset_postprocess(h);
}

int lss_filter(lss_handle* h, const int16_t* raw, int64_t n_rows, int64_t ibatch, int64_t n_batches,
               int32_t raw_on_device, float* X_dev, void* stream) {
    if (!h || !X_dev) return LSS_ERR_ARG;
    if (h->streaming) return h->fail(LSS_ERR_STATE, "handle is owned by a serving loop");
    CK(cudaSetDevice(h->cfg.device));
    cudaStream_t s = (cudaStream_t)stream;
    CK(wait_mixing(h, s));
    // the GEMM writes rows of stride ld; the caller's buffer has stride N
    int rc = run_filter(h, raw, n_rows, ibatch, n_batches, raw_on_device, h->X.p, s);
    if (rc) return rc;
    CK(cudaMemcpy2DAsync(X_dev, h->N * sizeof(float), h->X.p, h->ld * sizeof(float), h->N * sizeof(float), h->C,
                         cudaMemcpyDeviceToDevice, s));
    CK(cudaStreamSynchronize(s));
    return LSS_OK;
}

int lss_scores(lss_handle* h, const float* X_dev, int64_t N, float* B_dev, void* stream) {
    if (!h || !X_dev || !B_dev) return LSS_ERR_ARG;
    if (h->streaming) return h->fail(LSS_ERR_STATE, "handle is owned by a serving loop");
    if (N <= 0 || N > h->N) return h->fail(LSS_ERR_ARG, "N out of range");
    CK(cudaSetDevice(h->cfg.device));
    cudaStream_t s = (cudaStream_t)stream;
    CK(wait_mixing(h, s));
    CK(cudaMemcpy2DAsync(h->X.p, h->ld * sizeof(float), X_dev, N * sizeof(float), N * sizeof(float), h->C,
                         cudaMemcpyDeviceToDevice, s));
    CK(cudaMemsetAsync(h->status.p, 0, sizeof(int32_t), s));
    int rc = run_scores(h, h->X.p, h->ld, N, h->B.p, s, nullptr, false, /*rows_for_mp=*/false);
    if (rc) return rc;
    CK(cudaMemcpy2DAsync(B_dev, N * sizeof(float), h->B.p, h->ld * sizeof(float), N * sizeof(float), h->T,
                         cudaMemcpyDeviceToDevice, s));
    int32_t st = 0;
    CK(cudaMemcpyAsync(&st, h->status.p, sizeof(st), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (st & STATUS_TIMEOUT) return h->fail(LSS_ERR_TIMEOUT, "score GEMM pipeline wait timed out");
    return LSS_OK;
}

static int match_common(lss_handle* h, int64_t N, const float* Xsrc, int64_t* st_dev, float* amps_dev,
                        float* xres_dev, int64_t capacity, int64_t* n_spikes, cudaStream_t s,
                        bool maxima_ready = false) {
    int32_t n = 0, rounds = 0;
    int rc = run_mp(h, N, &n, &rounds, s, maxima_ready);
    if (rc) return rc;
    if (n_spikes) *n_spikes = n;
    if (n > capacity) return h->fail(LSS_ERR_CAPACITY, "output capacity smaller than the spike count");
    if (st_dev && amps_dev && n > 0) {
        CK(launch_st_out(h->sp_x.p, h->sp_y.p, h->sp_amp.p, n, st_dev, amps_dev, s));
        h->stats.launches += 1;
    }
    if (xres_dev && Xsrc) {
        rc = run_xres(h, Xsrc, h->ld, N, rounds, h->Xres.p, h->ld, s);
        if (rc) return rc;
        CK(cudaMemcpy2DAsync(xres_dev, N * sizeof(float), h->Xres.p, h->ld * sizeof(float), N * sizeof(float), h->C,
                             cudaMemcpyDeviceToDevice, s));
    }
    int32_t st = 0;
    CK(cudaMemcpyAsync(&st, h->status.p, sizeof(st), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (st & STATUS_LIST) return h->fail(LSS_ERR_CAPACITY, "residual tile touched by more than 1024 spikes");
    return LSS_OK;
}

int lss_match(lss_handle* h, const float* X_dev, int64_t N, int64_t* st_dev, float* amps_dev, float* xres_dev,
              int64_t capacity, int64_t* n_spikes, void* stream) {
    if (!h || !X_dev) return LSS_ERR_ARG;
    if (h->streaming) return h->fail(LSS_ERR_STATE, "handle is owned by a serving loop");
    if (N <= 0 || N > h->N) return h->fail(LSS_ERR_ARG, "N out of range (1..NT+2nt)");
    CK(cudaSetDevice(h->cfg.device));
    cudaStream_t s = (cudaStream_t)stream;
    CK(wait_mixing(h, s));
    CK(cudaMemcpy2DAsync(h->X.p, h->ld * sizeof(float), X_dev, N * sizeof(float), N * sizeof(float), h->C,
                         cudaMemcpyDeviceToDevice, s));
    CK(cudaMemsetAsync(h->status.p, 0, sizeof(int32_t), s));
    bool ready = false;
    int rc = run_scores(h, h->X.p, h->ld, N, h->B.p, s, &ready);
    if (rc) return rc;
    return match_common(h, N, h->X.p, st_dev, amps_dev, xres_dev, capacity, n_spikes, s, ready);
}

int lss_match_scores(lss_handle* h, const float* B_dev, int64_t N, int64_t* st_dev, float* amps_dev,
                     int64_t capacity, int64_t* n_spikes, void* stream) {
    if (!h || !B_dev) return LSS_ERR_ARG;
    if (h->streaming) return h->fail(LSS_ERR_STATE, "handle is owned by a serving loop");
    if (N <= 0 || N > h->N) return h->fail(LSS_ERR_ARG, "N out of range (1..NT+2nt)");
    CK(cudaSetDevice(h->cfg.device));
    cudaStream_t s = (cudaStream_t)stream;
    CK(wait_mixing(h, s));
    if (h->mp_skip) {  // the block-skipping rounds read the rows in probe order
        CK(launch_gather_rows(B_dev, N, h->mp_perm.p, h->T, N, h->B.p, h->ld, s));
        h->stats.launches += 1;
    } else {
        CK(cudaMemcpy2DAsync(h->B.p, h->ld * sizeof(float), B_dev, N * sizeof(float), N * sizeof(float), h->T,
                             cudaMemcpyDeviceToDevice, s));
    }
    CK(cudaMemsetAsync(h->status.p, 0, sizeof(int32_t), s));
    return match_common(h, N, nullptr, st_dev, amps_dev, nullptr, capacity, n_spikes, s);
}

static int sort_batch_impl(lss_handle* h, const int16_t* raw, int64_t n_rows, int64_t ibatch, int64_t n_batches,
                           int32_t raw_on_device, lss_records* out, void* stream, int64_t* count_dev);

int lss_sort_batch(lss_handle* h, const int16_t* raw, int64_t n_rows, int64_t ibatch, int64_t n_batches,
                   int32_t raw_on_device, lss_records* out, void* stream) {
    return sort_batch_impl(h, raw, n_rows, ibatch, n_batches, raw_on_device, out, stream, nullptr);
}

int lss_sort_batch_async(lss_handle* h, const int16_t* raw, int64_t n_rows, int64_t ibatch, int64_t n_batches,
                         int32_t raw_on_device, lss_records* out, int64_t* count_dev, void* stream) {
    if (!h || !out || !count_dev) return LSS_ERR_ARG;
    if (!out->on_device) return h->fail(LSS_ERR_ARG, "asynchronous batches write device records");
    for (const void* p : {(const void*)out->time, (const void*)out->template_id, (const void*)out->amplitude,
                          (const void*)out->pc, (const void*)out->x_pos, (const void*)out->y_pos,
                          (const void*)out->cluster, (const void*)count_dev})
        if (!lss::device_accessible(p, h->cfg.device))
            return h->fail(LSS_ERR_ARG,
                           "asynchronous records and count must be memory of the handle's device or pinned host memory");
    return sort_batch_impl(h, raw, n_rows, ibatch, n_batches, raw_on_device, out, stream, count_dev);
}

int lss_sync(lss_handle* h, void* stream) {
    if (!h) return LSS_ERR_ARG;
    CK(cudaSetDevice(h->cfg.device));
    CK(cudaStreamSynchronize((cudaStream_t)stream));
    int32_t st = 0;
    CK(cudaMemcpy(&st, h->status_acc.p, sizeof(st), cudaMemcpyDeviceToHost));
    CK(cudaMemset(h->status_acc.p, 0, sizeof(st)));
    if (st & STATUS_TIMEOUT) return h->fail(LSS_ERR_TIMEOUT, "a bounded device-side wait timed out");
    if (st & STATUS_CAPACITY) return h->fail(LSS_ERR_CAPACITY, "more than max_spikes spikes in one batch");
    if (st & STATUS_LIST)
        return h->fail(LSS_ERR_CAPACITY, std::string(MSG_MP_LIST) + ", or a PC-feature neighbour list overflow");
    return LSS_OK;
}

}  // extern "C"

static int sort_batch_impl(lss_handle* h, const int16_t* raw, int64_t n_rows, int64_t ibatch, int64_t n_batches,
                           int32_t raw_on_device, lss_records* out, void* stream, int64_t* count_dev) {
    if (!h || !out) return LSS_ERR_ARG;
    if (h->streaming) return h->fail(LSS_ERR_STATE, "handle is owned by a serving loop");
    if (!out->time || !out->template_id || !out->amplitude) return h->fail(LSS_ERR_ARG, "null record arrays");
    CK(cudaSetDevice(h->cfg.device));
    // a pageable host pointer handed over as device memory would fault in the
    // kernels: refuse it here
    if (raw_on_device && !lss::device_accessible(raw, h->cfg.device))
        return h->fail(LSS_ERR_ARG, "raw_on_device rows must be memory of the handle's device or pinned host memory");
    if (out->on_device && !count_dev)
        for (const void* p : {(const void*)out->time, (const void*)out->template_id, (const void*)out->amplitude,
                              (const void*)out->pc, (const void*)out->x_pos, (const void*)out->y_pos,
                              (const void*)out->cluster})
            if (!lss::device_accessible(p, h->cfg.device))
                return h->fail(LSS_ERR_ARG,
                               "on_device records must be memory of the handle's device or pinned host memory");
    cudaStream_t s = (cudaStream_t)stream;
    CK(wait_mixing(h, s));
    // host rows of an asynchronous batch: upload on the handle's upload stream
    // into the free one of two device buffers; the batch's stream waits for
    // the upload, and the buffer is free again once the batch's ingest has
    // read it, so the next batch's upload runs under this batch's work
    int up_slot = -1;
    if (count_dev && !raw_on_device) {
        IngestMap map;
        int rc0 = batch_map(h, raw, n_rows, ibatch, n_batches, map);
        if (rc0) return rc0;
        if (!h->up_s) {
            CK(cudaStreamCreateWithFlags(&h->up_s, cudaStreamNonBlocking));
            for (int i = 0; i < 2; ++i) {
                CK(h->raw_up[i].alloc((size_t)h->N * h->Cbin));
                CK(cudaEventCreateWithFlags(&h->up_done[i], cudaEventDisableTiming));
                CK(cudaEventCreateWithFlags(&h->raw_free[i], cudaEventDisableTiming));
            }
        }
        up_slot = h->raw_next;
        h->raw_next ^= 1;
        CK(cudaStreamWaitEvent(h->up_s, h->raw_free[up_slot], 0));
        CK(cudaMemcpyAsync(h->raw_up[up_slot].p, raw, (size_t)map.nsamp * h->Cbin * sizeof(int16_t),
                           cudaMemcpyHostToDevice, h->up_s));
        CK(cudaEventRecord(h->up_done[up_slot], h->up_s));
        CK(cudaStreamWaitEvent(s, h->up_done[up_slot], 0));
        raw = h->raw_up[up_slot].p;
        raw_on_device = 1;
    }
    // the whitening / drift matrix is folded into the templates (set_mixing), so
    // the scores come from the highpassed batch directly
    const float* Xh = nullptr;
    int rc = run_filter(h, raw, n_rows, ibatch, n_batches, raw_on_device, nullptr, s, &Xh);
    if (rc) return rc;
    if (up_slot >= 0) CK(cudaEventRecord(h->raw_free[up_slot], s));
    CK(cudaMemsetAsync(h->status.p, 0, sizeof(int32_t), s));
    bool ready = false;
    rc = run_scores(h, Xh, h->ld, h->N, h->B.p, s, &ready, /*folded=*/true);
    if (rc) return rc;
    // rounds, features and records all read the spike count on the device:
    // the batch has one host synchronisation, at its end
    rc = enqueue_mp(h, h->N, s, ready);
    if (rc) return rc;
    h->mark(7, s);
    const int feat = h->nC * h->K;
    const bool want_pc = out->pc != nullptr && feat > 0;
    const bool need_tf = want_pc || (h->post && h->pa.xc != nullptr && feat > 0);
    const bool bf16 = h->cfg.precision == LSS_PREC_BF16_RECHECK;
    const int32_t n_bound = h->cfg.max_spikes;
    h->mark(8, s);
    if (need_tf) {
        // the projection rows of the score GEMM: tf32 parts (FP32 path) or bf16 parts (BF16 path)
        const int grid = std::min(n_bound, 16 * h->sm_count);
        CK(launch_pc_features_folded(Xh, h->ld, h->C, h->nt, h->K, h->nC, h->T, h->wpca.p, h->Mw.p, h->U.p, h->R.p,
                                     h->iCC.p, h->iU.p, h->Ucc.p, h->sp_x.p, h->sp_y.p, h->sp_amp.p,
                                     h->round_start.p, 0, grid, h->counters.p, h->tF.p, h->status.p,
                                     bf16 ? (const void*)h->B0T.p : (const void*)h->B0T_hi.p,
                                     bf16 ? (const void*)h->B0T16lo.p : (const void*)h->B0T_lo.p, bf16 ? 1 : 0,
                                     h->CKpad, s));
        h->stats.launches += 1;
    }
    h->mark(9, s);
    const int64_t cap = out->capacity;
    int64_t* d_time = out->on_device ? out->time : h->rec_time.p;
    int32_t* d_tmpl = out->on_device ? out->template_id : h->rec_tmpl.p;
    float* d_amp = out->on_device ? out->amplitude : h->rec_amp.p;
    float* d_pc = want_pc ? (out->on_device ? out->pc : h->rec_pc.p) : nullptr;
    const int64_t dcap = out->on_device ? cap : std::min<int64_t>(cap, h->cfg.max_spikes);
    RecordClock rclk;
    rclk.ibatch = ibatch;
    rclk.counters = h->counters.p;
    rclk.NT = h->NT;
    rclk.nt = h->nt;
    rclk.nt0min = h->cfg.nt0min;
    if (h->post && ibatch == 0) {
        int rc0 = lss_reset_postprocess(h);
        if (rc0) return rc0;
    }
    const bool want_post = h->post && (out->x_pos || out->y_pos || out->cluster);
    float* d_x = want_post && out->x_pos ? (out->on_device ? out->x_pos : h->rec_x.p) : nullptr;
    float* d_y = want_post && out->y_pos ? (out->on_device ? out->y_pos : h->rec_y.p) : nullptr;
    int32_t* d_clu = want_post && out->cluster ? (out->on_device ? out->cluster : h->rec_clu.p) : nullptr;
    rc = enqueue_records(h, rclk, n_bound, want_pc, need_tf, d_time, d_tmpl, d_amp, d_pc, d_x, d_y, d_clu, dcap,
                         count_dev ? count_dev : h->rec_count.p, s);
    if (rc) return rc;
    if (count_dev) {
        // asynchronous: errors accumulate for lss_sync; no host wait
        CK(launch_status_or(h->status.p, h->status_acc.p, s));
        h->stats.launches += 1;
        h->mark(10, s);
        CK(cudaEventRecord(h->batch_ev, s));
        return LSS_OK;
    }
    CK(cudaEventRecord(h->batch_ev, s));
    int64_t count = 0;
    int32_t st = 0, hc[4];
    CK(cudaMemcpyAsync(&count, h->rec_count.p, sizeof(count), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&st, h->status.p, sizeof(st), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hc, h->counters.p, sizeof(hc), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h->mp_phase_host, h->mp_phase.p, sizeof(h->mp_phase_host), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (st & STATUS_TIMEOUT) return h->fail(LSS_ERR_TIMEOUT, "a bounded device-side wait timed out");
    if (st & STATUS_CAPACITY) return h->fail(LSS_ERR_CAPACITY, "more than max_spikes spikes in one batch");
    if (st & STATUS_LIST)
        return h->fail(LSS_ERR_CAPACITY, std::string(MSG_MP_LIST) + ", or a PC-feature neighbour list overflow");
    h->stats.spikes = hc[0];
    h->stats.rounds = hc[1];
    h->stats.mp_items_updated = hc[2];
    h->stats.mp_items = hc[3];
    h->set_phase_stats();
    out->count = count;
    if (count > cap) return h->fail(LSS_ERR_CAPACITY, "record capacity smaller than the spike count");
    if (!out->on_device && count > 0) {
        CK(cudaMemcpyAsync(out->time, d_time, count * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(out->template_id, d_tmpl, count * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(out->amplitude, d_amp, count * sizeof(float), cudaMemcpyDeviceToHost, s));
        if (want_pc)
            CK(cudaMemcpyAsync(out->pc, d_pc, count * feat * sizeof(float), cudaMemcpyDeviceToHost, s));
        if (d_x) CK(cudaMemcpyAsync(out->x_pos, d_x, count * sizeof(float), cudaMemcpyDeviceToHost, s));
        if (d_y) CK(cudaMemcpyAsync(out->y_pos, d_y, count * sizeof(float), cudaMemcpyDeviceToHost, s));
        if (d_clu) CK(cudaMemcpyAsync(out->cluster, d_clu, count * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    }
    h->mark(10, s);
    CK(cudaStreamSynchronize(s));
    if (h->prof) {
        float* f = &h->times.h2d_ms;
        for (int i = 0; i < 10; ++i) cudaEventElapsedTime(&f[i], h->ev[i], h->ev[i + 1]);
        cudaEventElapsedTime(&h->times.total_ms, h->ev[0], h->ev[10]);
    }
    return LSS_OK;
}

extern "C" {

int lss_set_profiling(lss_handle* h, int32_t on) {
    if (!h) return LSS_ERR_ARG;
    CK(cudaSetDevice(h->cfg.device));
    if (on && !h->ev[0])
        for (auto& e : h->ev) CK(cudaEventCreate(&e));
    h->prof = on != 0;
    return LSS_OK;
}

int lss_get_stage_times(const lss_handle* h, lss_stage_times* out) {
    if (!h || !out) return LSS_ERR_ARG;
    if (!h->prof) return LSS_ERR_STATE;
    *out = h->times;
    return LSS_OK;
}

// ---------------------------------------------------------------- directory
static bool read_misc(const std::string& path, std::map<std::string, std::string>& kv) {
    std::ifstream in(path);
    if (!in) return false;
    std::string line;
    while (std::getline(in, line)) {
        const size_t p = line.find(':');
        if (p == std::string::npos) continue;
        std::string v = line.substr(p + 1);
        while (!v.empty() && (v.back() == '\r' || v.back() == ' ')) v.pop_back();
        kv[line.substr(0, p)] = v;
    }
    return true;
}

int lss_create_from_dir(const char* dir, const lss_config* overrides, lss_handle** out) {
    if (!dir || !out) { g_create_err = "null argument"; return LSS_ERR_ARG; }
    std::string d(dir);
    if (!d.empty() && d.back() != '/') d += '/';
    std::string err;
    auto load = [&](const char* name, NpyArray& a) -> bool {
        if (!npy_load(d + name, a, err)) { g_create_err = err; return false; }
        return true;
    };
    NpyArray aW, aP, aC, aWr, aDr, aHp, aICC, aIU, aUcc, aMap;
    if (!load("Wall3.npy", aW) || !load("wPCA.npy", aP) || !load("ctc.npy", aC)) return LSS_ERR_IO;
    if (!npy_load(d + "whitening_mat.npy", aWr, err) && !npy_load(d + "whiteningMat.npy", aWr, err)) {
        g_create_err = "whitening_mat.npy / whiteningMat.npy: " + err;
        return LSS_ERR_IO;
    }
    const bool have_drift = npy_load(d + "drift_matrix.npy", aDr, err);
    const bool have_hp = npy_load(d + "hp_filter.npy", aHp, err);
    const bool have_ext = npy_load(d + "iCC.npy", aICC, err) && npy_load(d + "iU.npy", aIU, err) &&
                          npy_load(d + "Ucc.npy", aUcc, err);
    const bool have_map = npy_load(d + "channel_map.npy", aMap, err) || npy_load(d + "channelMap.npy", aMap, err);
    if (aW.shape.size() != 3 || aP.shape.size() != 2 || aC.shape.size() != 3 || aWr.shape.size() != 2) {
        g_create_err = "Wall3 [T,K,C], wPCA [K,nt], ctc [T,T,2nt+1], whitening [C,C] expected";
        return LSS_ERR_SHAPE;
    }
    lss_config c{};
    c.n_templates = (int32_t)aW.shape[0];
    c.n_pcs = (int32_t)aW.shape[1];
    c.n_chan = (int32_t)aW.shape[2];
    c.nt = (int32_t)aP.shape[1];
    c.n_chan_bin = c.n_chan;
    c.batch_size = 60000;
    c.nt0min = 20;
    c.th_learned = 8.f;
    c.max_rounds = 100;
    c.max_spikes = 100000;
    c.do_car = 1;
    c.n_nearest = have_ext ? (int32_t)aICC.shape[0] : 0;
    std::map<std::string, std::string> kv;
    if (read_misc(d + "misc.txt", kv)) {
        if (kv.count("nt0min")) c.nt0min = std::stoi(kv["nt0min"]);
        if (kv.count("Th_learned")) c.th_learned = std::stof(kv["Th_learned"]);
        if (kv.count("numNearestChans") && have_ext && std::stoi(kv["numNearestChans"]) != c.n_nearest) {
            g_create_err = "misc.txt numNearestChans disagrees with iCC.npy";
            return LSS_ERR_SHAPE;
        }
    }
    if (overrides) {
        if (overrides->n_chan_bin) c.n_chan_bin = overrides->n_chan_bin;
        if (overrides->batch_size) c.batch_size = overrides->batch_size;
        if (overrides->nt0min) c.nt0min = overrides->nt0min;
        if (overrides->th_learned != 0.f) c.th_learned = overrides->th_learned;
        if (overrides->max_rounds) c.max_rounds = overrides->max_rounds;
        if (overrides->max_spikes) c.max_spikes = overrides->max_spikes;
        c.do_car = overrides->do_car;
        c.invert_sign = overrides->invert_sign;
        c.precision = overrides->precision;
        c.device = overrides->device;
    }
    const int64_t T = c.n_templates, K = c.n_pcs, C = c.n_chan, nt = c.nt;
    if (aP.shape[0] != K || aC.shape[0] != T || aC.shape[1] != T || aC.shape[2] != 2 * nt + 1 ||
        aWr.shape[0] != C || aWr.shape[1] != C) {
        g_create_err = "inconsistent shapes among Wall3, wPCA, ctc and whitening";
        return LSS_ERR_SHAPE;
    }
    std::vector<float> W, P, Cc, Wr, Dr, Hp, Ucc;
    std::vector<int64_t> iCC, iU, mp64;
    if (!npy_as_f32(aW, W, err) || !npy_as_f32(aP, P, err) || !npy_as_f32(aC, Cc, err) || !npy_as_f32(aWr, Wr, err)) {
        g_create_err = err;
        return LSS_ERR_SHAPE;
    }
    if (have_drift) {
        if (aDr.shape.size() != 2 || aDr.shape[0] != C || aDr.shape[1] != C) {
            g_create_err = "drift_matrix.npy must be [C, C]";
            return LSS_ERR_SHAPE;
        }
        if (!npy_as_f32(aDr, Dr, err)) { g_create_err = err; return LSS_ERR_SHAPE; }
        // the file holds M.T (run_online_spikes.py:532); recover M
        std::vector<float> M(Dr.size());
        for (int64_t i = 0; i < C; ++i)
            for (int64_t j = 0; j < C; ++j) M[i * C + j] = Dr[j * C + i];
        Dr.swap(M);
    }
    if (have_hp) {
        if (!npy_as_f32(aHp, Hp, err)) { g_create_err = err; return LSS_ERR_SHAPE; }
        c.hp_len = (int32_t)Hp.size();
    }
    if (have_ext) {
        if (!npy_as_i64(aICC, iCC, err) || !npy_as_i64(aIU, iU, err) || !npy_as_f32(aUcc, Ucc, err)) {
            g_create_err = err;
            return LSS_ERR_SHAPE;
        }
        if (aICC.shape.size() != 2 || aICC.shape[1] != C || (int64_t)iU.size() != T ||
            (int64_t)Ucc.size() != (int64_t)c.n_nearest * T * K) {
            g_create_err = "iCC [nC,C], iU [T], Ucc [nC,T,K] expected";
            return LSS_ERR_SHAPE;
        }
    }
    std::vector<int32_t> cmap;
    if (have_map) {
        if (!npy_as_i64(aMap, mp64, err)) { g_create_err = err; return LSS_ERR_SHAPE; }
        if ((int64_t)mp64.size() != C) { g_create_err = "channel map must have C entries"; return LSS_ERR_SHAPE; }
        cmap.assign(mp64.begin(), mp64.end());
        for (auto v : cmap) c.n_chan_bin = std::max<int32_t>(c.n_chan_bin, v + 1);
        if (overrides && overrides->n_chan_bin) c.n_chan_bin = overrides->n_chan_bin;
    }
    lss_tensors t{};
    t.wall3 = W.data();
    t.wpca = P.data();
    t.ctc = Cc.data();
    t.whitening = Wr.data();
    t.drift = have_drift ? Dr.data() : nullptr;
    t.hp_filter = have_hp ? Hp.data() : nullptr;
    t.iCC = have_ext ? iCC.data() : nullptr;
    t.iU = have_ext ? iU.data() : nullptr;
    t.Ucc = have_ext ? Ucc.data() : nullptr;
    t.chan_map = have_map ? cmap.data() : nullptr;
    return lss_create(&c, &t, out);
}

}  // extern "C"
