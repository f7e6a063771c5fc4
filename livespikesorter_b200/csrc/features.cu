// Residual, PC features and spike records of one batch.
//
// * Xres = X minus every accepted spike's waveform, applied in the order the
//   reference applies them (round by round; within a round the +-nt/2
//   windows of distinct peaks never overlap): template_matching.py:197.
// * PC features xfeat[i, j, k] = sum_m Xres[iCC[j, iU[y_i]], x_i + m - nt/2]
//   * wPCA[k, m] + amp_i * Ucc[j, y_i, k]: template_matching.py:50-51
//   (compute_xfeat_kernel, OnlineSpikesV2.cu:112-187, which indexes the
//   residual as [n, C] although it is stored [C, n]; this follows Kilosort).
// * records: time = (x - nt) + ibatch*NT - nt/2 + nt0min, dropping negative
//   times of batch 0 (template_matching.py:53-68), in run_matching order.
#include "lss_kernels.cuh"

#include <algorithm>

namespace lss {

// projection-row element as float: the FP32 path's tf32 parts or the BF16
// path's bf16 parts (hi + lo is the projection to 2^-23 or 2^-17 relative)
__device__ __forceinline__ float pval(const float* p) { return *p; }
__device__ __forceinline__ float pval(const __nv_bfloat16* p) { return __bfloat162float(*p); }

constexpr int XR_COLS = 128;
constexpr int XR_CH = 32;
constexpr int XR_LIST_MAX = 1024;

__global__ void __launch_bounds__(XR_COLS) k_xres(const float* __restrict__ X, int64_t ldx, int32_t C, int32_t N,
                                                  int32_t nt, const float* __restrict__ wave,
                                                  const int32_t* __restrict__ sp_x,
                                                  const int32_t* __restrict__ sp_y,
                                                  const float* __restrict__ sp_amp,
                                                  const int32_t* __restrict__ round_start, int32_t rounds,
                                                  float* __restrict__ Xres, int32_t* status) {
    __shared__ int l_x[XR_LIST_MAX], l_y[XR_LIST_MAX];
    __shared__ float l_a[XR_LIST_MAX];
    __shared__ int r_cnt[XR_COLS], r_off[XR_COLS + 1];
    const int h = nt / 2;
    const int s0 = blockIdx.x * XR_COLS;
    const int wlo = s0 - h, whi = s0 + XR_COLS - 1 + h;
    int nlist = 0;
    // spikes touching the tile, in round order; rounds handled XR_COLS at a time
    for (int rb = 0; rb < rounds; rb += XR_COLS) {
        const int r = rb + threadIdx.x;
        int lo = 0, cnt = 0;
        if (r < rounds) {
            int a = round_start[r], bnd = round_start[r + 1];
            int b2 = bnd;
            while (a < b2) {  // first spike with x >= wlo
                const int m = (a + b2) >> 1;
                if (sp_x[m] < wlo) a = m + 1; else b2 = m;
            }
            lo = a;
            int e = a;
            while (e < bnd && sp_x[e] <= whi) ++e;
            cnt = e - a;
        }
        r_cnt[threadIdx.x] = cnt;
        __syncthreads();
        if (threadIdx.x == 0) {
            int o = 0;
            for (int i = 0; i < XR_COLS; ++i) {
                r_off[i] = o;
                o += r_cnt[i];
            }
            r_off[XR_COLS] = o;
        }
        __syncthreads();
        for (int k = 0; k < cnt; ++k) {
            const int dst = nlist + r_off[threadIdx.x] + k;
            if (dst < XR_LIST_MAX) {
                l_x[dst] = sp_x[lo + k];
                l_y[dst] = sp_y[lo + k];
                l_a[dst] = sp_amp[lo + k];
            }
        }
        nlist += r_off[XR_COLS];
        __syncthreads();
    }
    if (nlist > XR_LIST_MAX) {
        if (threadIdx.x == 0) atomicOr(status, STATUS_LIST);
        nlist = XR_LIST_MAX;
    }
    const int s = s0 + threadIdx.x;
    if (s >= N) return;
    for (int c0 = 0; c0 < C; c0 += XR_CH) {
        const int nc = min(XR_CH, C - c0);
        float v[XR_CH];
#pragma unroll
        for (int k = 0; k < XR_CH; ++k) v[k] = (k < nc) ? X[(int64_t)(c0 + k) * ldx + s] : 0.f;
        for (int e = 0; e < nlist; ++e) {
            const int d = s - l_x[e];
            if (d < -h || d > h) continue;
            const float a = l_a[e];
            const float* wp = wave + ((int64_t)l_y[e] * C + c0) * nt + (d + h);
#pragma unroll
            for (int k = 0; k < XR_CH; ++k)
                if (k < nc) v[k] = __fsub_rn(v[k], __fmul_rn(a, wp[(int64_t)k * nt]));
        }
#pragma unroll
        for (int k = 0; k < XR_CH; ++k)
            if (k < nc) Xres[(int64_t)(c0 + k) * ldx + s] = v[k];
    }
}

cudaError_t launch_xres(const float* X, int64_t ldx, int32_t C, int32_t N, int32_t nt, const float* wave,
                        const int32_t* sp_x, const int32_t* sp_y, const float* sp_amp,
                        const int32_t* round_start, const int32_t* counters, int32_t rounds,
                        float* Xres, int32_t* status, cudaStream_t s) {
    (void)counters;
    const int grid = (N + XR_COLS - 1) / XR_COLS;
    k_xres<<<grid, XR_COLS, 0, s>>>(X, ldx, C, N, nt, wave, sp_x, sp_y, sp_amp, round_start, rounds, Xres,
                                     status);
    return cudaGetLastError();
}

// Records: one CTA computes every kept spike's output slot with ballot scans
// (spikes aligned before the recording start are dropped, which only happens
// in the first batch), then a grid writes the slots and their PC features.
//
// Record time t = (x - nt) + ibatch * NT + shift - nt/2 + nt0min
// (template_matching.py:54-59; shift = 0 for Kilosort's batches). With
// rc.counters the spike count is read from the device, with rc.ibatch_dev the
// batch index too, and with rc.slots > 0 batch b writes slot b % slots of
// output arrays that hold `slots` batches of `capacity` records each (the
// streaming loop's result rings).
__device__ __forceinline__ int64_t rec_time(int x, int64_t ibatch, const RecordClock& rc) {
    return (int64_t)(x - rc.nt) + ibatch * (int64_t)rc.NT + rc.shift - rc.nt / 2 + rc.nt0min;
}

__global__ void __launch_bounds__(1024) k_records_scan(const int32_t* __restrict__ sp_x, int32_t n, RecordClock rc,
                                                       int32_t* __restrict__ slot, int64_t* out_count) {
    __shared__ int wsum[32];
    __shared__ int s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (rc.counters) n = rc.counters[0];
    const int64_t ibatch = rc.ibatch_dev ? *rc.ibatch_dev : rc.ibatch;
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();
    for (int c0 = 0; c0 < n; c0 += 1024) {
        const int i = c0 + threadIdx.x;
        bool keep = false;
        if (i < n) keep = rec_time(sp_x[i], ibatch, rc) >= 0;
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) wsum[warp] = __popc(bal);
        __syncthreads();
        if (warp == 0) {
            const int c = wsum[lane];
            int inc = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += u;
            }
            wsum[lane] = inc - c;
        }
        __syncthreads();
        if (i < n) slot[i] = keep ? s_base + wsum[warp] + __popc(bal & ((1u << lane) - 1u)) : -1;
        __syncthreads();
        if (threadIdx.x == 1023) s_base += wsum[31] + __popc(bal);
        __syncthreads();
    }
    if (threadIdx.x == 0) out_count[rc.slots > 0 ? ibatch % rc.slots : 0] = s_base;
}

__global__ void k_records_write(const int32_t* __restrict__ sp_x, const int32_t* __restrict__ sp_y,
                                const float* __restrict__ sp_amp, const float* __restrict__ tF,
                                const int32_t* __restrict__ slot, int32_t n, int32_t feat_len, RecordClock rc,
                                int64_t* out_time, int32_t* out_tmpl, float* out_amp, float* out_pc,
                                int64_t capacity) {
    if (rc.counters) n = rc.counters[0];
    const int64_t ibatch = rc.ibatch_dev ? *rc.ibatch_dev : rc.ibatch;
    const int64_t base = rc.slots > 0 ? (ibatch % rc.slots) * capacity : 0;
    const int row = 3 + feat_len;  // time, template, amplitude, features
    const int64_t total = (int64_t)n * row;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / row;
        const int f = (int)(e % row);
        const int o = slot[i];
        if (o < 0 || o >= capacity) continue;
        const int64_t q = base + o;
        if (f == 0) out_time[q] = rec_time(sp_x[i], ibatch, rc);
        else if (f == 1) out_tmpl[q] = sp_y[i];
        else if (f == 2) out_amp[q] = sp_amp[i];
        else if (out_pc && tF) out_pc[q * feat_len + (f - 3)] = tF[i * feat_len + (f - 3)];
    }
}

cudaError_t launch_records(const int32_t* sp_x, const int32_t* sp_y, const float* sp_amp, const float* tF,
                           int32_t* slot, int32_t n, int32_t feat_len, const RecordClock& rc, int64_t* out_time,
                           int32_t* out_tmpl, float* out_amp, float* out_pc, int64_t capacity, int64_t* out_count,
                           cudaStream_t s) {
    // n: the spike count, or (rc.counters != null) an upper bound that sizes the write grid
    if (!rc.presorted) k_records_scan<<<1, 1024, 0, s>>>(sp_x, n, rc, slot, out_count);
    const int64_t total = (int64_t)n * (3 + (tF ? feat_len : 0));
    if (total > 0) {
        const int64_t blocks = std::min<int64_t>((total + 255) / 256, rc.counters ? 1184 : INT32_MAX);
        k_records_write<<<(unsigned)blocks, 256, 0, s>>>(sp_x, sp_y, sp_amp, tF, slot, n, tF ? feat_len : 0, rc,
                                                         out_time, out_tmpl, out_amp, tF ? out_pc : nullptr,
                                                         capacity);
    }
    return cudaGetLastError();
}

__global__ void k_st_out(const int32_t* __restrict__ sp_x, const int32_t* __restrict__ sp_y,
                         const float* __restrict__ sp_amp, int32_t n, int64_t* st, float* amps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    st[2 * (int64_t)i] = sp_x[i];
    st[2 * (int64_t)i + 1] = sp_y[i];
    amps[i] = sp_amp[i];
}

cudaError_t launch_st_out(const int32_t* sp_x, const int32_t* sp_y, const float* sp_amp, int32_t n,
                          int64_t* st, float* amps, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_st_out<<<(n + 255) / 256, 256, 0, s>>>(sp_x, sp_y, sp_amp, n, st, amps);
    return cudaGetLastError();
}



// ---------------------------------------------------------------------------
// PC features without a residual array (used by lss_sort_batch, where the
// whitening is folded into the templates). With Xh the highpassed batch and
// Mw = M @ Wrot, Kilosort's
//   xfeat[i, j, k] = sum_m Xres[ch, x_i + m - nt/2] * wPCA[k, m] + amp_i * Ucc[j, y_i, k]
// (template_matching.py:50-51, ch = iCC[j, iU[y_i]]) is evaluated as
//   sum_c' Mw[ch, c'] * sum_m wPCA[k, m] Xh[c', x_i + m - nt/2]
//   - sum_{spikes i', |x_i - x_i'| < nt} amp_i' * sum_k' U[y_i', k', ch] * R[k, k', x_i - x_i']
//   + amp_i * Ucc[j, y_i, k]
// with R[k, k', d] = sum_m wPCA[k, m] wPCA[k', m + d] (the waveform of spike i'
// projected on the basis at lag d). Same linear algebra, different order.
// One CTA per spike; channels are staged 64 at a time.
// ---------------------------------------------------------------------------
constexpr int FT_CH = 64;
constexpr int FT_LIST = 512;
constexpr int FT_NQ = 32;  // neighbours per staged chunk

template <typename PT>
__device__ __forceinline__ void pc_features_one(
    int i, int rounds, const float* __restrict__ Xh, int64_t ldx, int32_t C, int32_t nt, int32_t K, int32_t nC,
    int32_t T, const float* __restrict__ wpca, const float* __restrict__ Mw, const float* __restrict__ U,
    const float* __restrict__ R, const int64_t* __restrict__ iCC, const int64_t* __restrict__ iU,
    const float* __restrict__ Ucc, const int32_t* __restrict__ sp_x, const int32_t* __restrict__ sp_y,
    const float* __restrict__ sp_amp, const int32_t* __restrict__ round_start, float* __restrict__ tF,
    int32_t* status, const PT* __restrict__ Phi, const PT* __restrict__ Plo, int64_t ldp) {
    extern __shared__ float sm[];
    const int ntp = nt + 1;
    float* ws = sm;                          // [K][nt]
    float* xs = ws + K * nt;                 // [FT_CH][ntp]
    float* pc = xs + FT_CH * ntp;            // [FT_CH][K]
    float* mw = pc + FT_CH * K;              // [nC][FT_CH]
    // the projection-row path reuses the front of the buffer (see below)
    const int front = max(K * nt + FT_CH * ntp + FT_CH * K + nC * FT_CH, C * K + nC * C + 4 * nC * K);
    float* acc = sm + front;                 // [nC*K]
    __shared__ int s_ch[64];
    __shared__ int l_x[FT_LIST], l_y[FT_LIST];
    __shared__ float l_a[FT_LIST];
    __shared__ int s_n;
    __shared__ int s_cnt[256];
    const int x = sp_x[i], y = sp_y[i];
    const int h = nt / 2;
    for (int e = threadIdx.x; e < K * nt; e += blockDim.x) ws[e] = wpca[e];
    if (threadIdx.x < nC) s_ch[threadIdx.x] = (int)iCC[(int64_t)threadIdx.x * C + iU[y]];
    for (int e = threadIdx.x; e < nC * K; e += blockDim.x) acc[e] = 0.f;
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    // neighbours (any round, round order) whose waveform window overlaps this
    // spike's window; rounds are scanned blockDim.x at a time
    for (int rb = 0; rb < rounds; rb += blockDim.x) {
        const int r = rb + threadIdx.x;
        int lo = 0, cnt = 0;
        if (r < rounds) {
            const int b = round_start[r + 1];
            int hi2 = b;
            lo = round_start[r];
            while (lo < hi2) {
                const int m = (lo + hi2) >> 1;
                if (sp_x[m] <= x - nt) lo = m + 1; else hi2 = m;
            }
            int e = lo;
            while (e < b && sp_x[e] < x + nt) ++e;
            cnt = e - lo;
        }
        // exclusive prefix of the counts over the block (warp scans, then the
        // warp totals), offset by the entries listed so far
        {
            const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
            int inc = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += u;
            }
            __shared__ int s_wtot[8];
            if (lane == 31) s_wtot[wp] = inc;
            __syncthreads();
            int before = s_n;
            for (int w2 = 0; w2 < wp; ++w2) before += s_wtot[w2];
            s_cnt[threadIdx.x] = before + inc - cnt;
            __syncthreads();
            if (threadIdx.x == blockDim.x - 1) s_n = before + inc;
            __syncthreads();
        }
        for (int q = 0; q < cnt; ++q) {
            const int slot = s_cnt[threadIdx.x] + q;
            if (slot < FT_LIST) {
                l_x[slot] = sp_x[lo + q];
                l_y[slot] = sp_y[lo + q];
                l_a[slot] = sp_amp[lo + q];
            }
        }
        __syncthreads();
    }
    if (Phi) {
        // the spike's projection row P[x, :] = hi + lo and the nC rows of Mw,
        // then each (j, k) dot product split over 4 threads, combined in order
        float* prow = sm;                  // [C*K]
        float* mwr = prow + C * K;         // [nC][C]
        float* red = mwr + nC * C;         // [4*nC*K]
        __syncthreads();
        const int64_t o = (int64_t)x * ldp;
        for (int e = threadIdx.x; e < C * K; e += blockDim.x) prow[e] = __fadd_rn(pval(Phi + o + e), pval(Plo + o + e));
        for (int e = threadIdx.x; e < nC * C; e += blockDim.x) {
            const int j = e / C, c = e % C;
            mwr[e] = Mw[(int64_t)s_ch[j] * C + c];
        }
        __syncthreads();
        for (int e = threadIdx.x; e < 4 * nC * K; e += blockDim.x) {
            const int f = e >> 2, part = e & 3;
            const int j = f / K, k = f % K;
            float v = 0.f;
            for (int c = part; c < C; c += 4) v = fmaf(mwr[j * C + c], prow[c * K + k], v);
            red[e] = v;
        }
        __syncthreads();
        for (int f = threadIdx.x; f < nC * K; f += blockDim.x)
            acc[f] = __fadd_rn(__fadd_rn(red[4 * f], red[4 * f + 1]), __fadd_rn(red[4 * f + 2], red[4 * f + 3]));
    }
    for (int c0 = 0; c0 < (Phi ? 0 : C); c0 += FT_CH) {
        const int nc = min(FT_CH, C - c0);
        __syncthreads();
        if (Phi) {
            // projection row of the score GEMM: P[x, c*K + k] = hi + lo (to 2^-23 relative)
            const int64_t o = (int64_t)x * ldp + (int64_t)c0 * K;
            for (int e = threadIdx.x; e < nc * K; e += blockDim.x) pc[e] = __fadd_rn(pval(Phi + o + e), pval(Plo + o + e));
        } else {
            for (int e = threadIdx.x; e < nc * nt; e += blockDim.x) {
                const int c = e / nt, m = e % nt;
                xs[c * ntp + m] = Xh[(int64_t)(c0 + c) * ldx + x - h + m];
            }
        }
        for (int e = threadIdx.x; e < nC * nc; e += blockDim.x) {
            const int j = e / nc, c = e % nc;
            mw[j * FT_CH + c] = Mw[(int64_t)s_ch[j] * C + c0 + c];
        }
        __syncthreads();
        if (!Phi) {
            for (int e = threadIdx.x; e < nc * K; e += blockDim.x) {
                const int c = e / K, k = e % K;
                float p = 0.f;
                for (int m = 0; m < nt; ++m) p = fmaf(ws[k * nt + m], xs[c * ntp + m], p);
                pc[c * K + k] = p;
            }
            __syncthreads();
        }
        for (int e = threadIdx.x; e < nC * K; e += blockDim.x) {
            const int j = e / K, k = e % K;
            float v = acc[e];
            for (int c = 0; c < nc; ++c) v = fmaf(mw[j * FT_CH + c], pc[c * K + k], v);
            acc[e] = v;
        }
    }
    __syncthreads();
    const int nl = min(s_n, FT_LIST);
    if (threadIdx.x == 0 && s_n > FT_LIST) atomicOr(status, STATUS_LIST);
    // neighbours' projected waveforms, FT_NQ at a time:
    //   contrib[q][j][k] = sum_k' U[y_q, k', ch_j] * R[k, k', x - x_q]
    // all loads of a chunk are independent, then each (j, k) sums its column
    // over q in list order
    float* contrib = acc + nC * K;  // [FT_NQ][nC*K]
    const int F = nC * K;
    const int nd = 2 * nt - 1;
    float v = 0.f;
    const int e_own = threadIdx.x;  // (j, k) owned by this thread when < F
    if (e_own < F) v = acc[e_own];
    for (int q0 = 0; q0 < nl; q0 += FT_NQ) {
        const int nq = min(FT_NQ, nl - q0);
        __syncthreads();
        for (int task = threadIdx.x; task < nq * F; task += blockDim.x) {
            const int q = task / F, f = task % F;
            const int j = f / K, k = f % K;
            const int d = x - l_x[q0 + q];
            const float* rk = R + ((int64_t)k * K) * nd + (d + nt - 1);
            const float* uy = U + (int64_t)l_y[q0 + q] * K * C + s_ch[j];
            float sub = 0.f;
            for (int kk = 0; kk < K; ++kk) sub = fmaf(__ldg(uy + (int64_t)kk * C), __ldg(rk + (int64_t)kk * nd), sub);
            contrib[q * F + f] = sub;
        }
        __syncthreads();
        if (e_own < F)
            for (int q = 0; q < nq; ++q) v = __fsub_rn(v, __fmul_rn(l_a[q0 + q], contrib[q * F + e_own]));
    }
    if (e_own < F) {
        const int j = e_own / K, k = e_own % K;
        v = __fadd_rn(v, __fmul_rn(sp_amp[i], Ucc[((int64_t)j * T + y) * K + k]));
        tF[(int64_t)i * F + e_own] = v;
    }
}

// Warp per spike (projection-row path, nC = NCC and K = KPC known at compile
// time): lane l sums channels l, l + 32, ... of every (j, k) feature, the 32
// partial sums are combined by a butterfly, then each lane owns one or two
// features for the neighbour corrections (list order) and the amp * Ucc term.
constexpr int FW_LIST = 256;  // neighbours per spike (all rounds, within +-nt)
template <int KPC, int NCC, typename PT>
__global__ void __launch_bounds__(256, 2) k_pc_features_warp(
    int32_t C, int32_t nt, int32_t T, const float* __restrict__ Mw, const float* __restrict__ U,
    const float* __restrict__ R, const int64_t* __restrict__ iCC, const int64_t* __restrict__ iU,
    const float* __restrict__ Ucc, const int32_t* __restrict__ sp_x, const int32_t* __restrict__ sp_y,
    const float* __restrict__ sp_amp, const int32_t* __restrict__ round_start, int32_t rounds, int32_t n,
    const int32_t* __restrict__ counters, float* __restrict__ tF, int32_t* status, const PT* __restrict__ Phi,
    const PT* __restrict__ Plo, int64_t ldp) {
    constexpr int F = NCC * KPC;
    __shared__ int s_lx[8][FW_LIST], s_ly[8][FW_LIST];
    __shared__ float s_la[8][FW_LIST];
    if (counters) {
        n = counters[0];
        rounds = counters[1];
    }
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    const int nd = 2 * nt - 1;
    for (int i = blockIdx.x * 8 + wl; i < n; i += gridDim.x * 8) {
        const int x = sp_x[i], y = sp_y[i];
        const int64_t u = iU[y];
        int chl = 0;  // lane j < NCC holds channel j's index
        if (lane < NCC) chl = (int)iCC[(int64_t)lane * C + u];
        int ch[NCC];
#pragma unroll
        for (int j = 0; j < NCC; ++j) ch[j] = __shfl_sync(0xffffffffu, chl, j);
        // ---- sum over channels: acc[j][k] = sum_c Mw[ch_j, c] * P[x, c*K + k]
        float acc[NCC][KPC];
#pragma unroll
        for (int j = 0; j < NCC; ++j)
#pragma unroll
            for (int k = 0; k < KPC; ++k) acc[j][k] = 0.f;
        const int64_t o = (int64_t)x * ldp;
        for (int c = lane; c < C; c += 32) {
            float pv[KPC];
#pragma unroll
            for (int k = 0; k < KPC; ++k) pv[k] = __fadd_rn(pval(Phi + o + c * KPC + k), pval(Plo + o + c * KPC + k));
#pragma unroll
            for (int j = 0; j < NCC; ++j) {
                const float mv = __ldg(Mw + (int64_t)ch[j] * C + c);
#pragma unroll
                for (int k = 0; k < KPC; ++k) acc[j][k] = fmaf(mv, pv[k], acc[j][k]);
            }
        }
#pragma unroll
        for (int j = 0; j < NCC; ++j)
#pragma unroll
            for (int k = 0; k < KPC; ++k) {
                float v = acc[j][k];
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
                acc[j][k] = v;  // every lane holds the total
            }
        // ---- neighbours (any round, round order) whose window overlaps x's
        int nl = 0;
        for (int rb = 0; rb < rounds; rb += 32) {
            const int r = rb + lane;
            int lo = 0, cnt = 0;
            if (r < rounds) {
                const int b = round_start[r + 1];
                int hi2 = b;
                lo = round_start[r];
                while (lo < hi2) {
                    const int m = (lo + hi2) >> 1;
                    if (sp_x[m] <= x - nt) lo = m + 1; else hi2 = m;
                }
                int e = lo;
                while (e < b && sp_x[e] < x + nt) ++e;
                cnt = e - lo;
            }
            int inc = cnt;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int v2 = __shfl_up_sync(0xffffffffu, inc, off);
                if (lane >= off) inc += v2;
            }
            const int base = nl + inc - cnt;
            for (int q = 0; q < cnt; ++q) {
                const int slot = base + q;
                if (slot < FW_LIST) {
                    s_lx[wl][slot] = sp_x[lo + q];
                    s_ly[wl][slot] = sp_y[lo + q];
                    s_la[wl][slot] = sp_amp[lo + q];
                }
            }
            nl += __shfl_sync(0xffffffffu, inc, 31);
        }
        __syncwarp();
        if (nl > FW_LIST) {
            if (lane == 0) atomicOr(status, STATUS_LIST);
            nl = FW_LIST;
        }
        // ---- each lane finishes features f = lane and lane + 32
#pragma unroll
        for (int h2 = 0; h2 < 2; ++h2) {
            const int f = lane + 32 * h2;
            if (f >= F) break;
            const int j = f / KPC, k = f % KPC;
            float v = 0.f;
#pragma unroll
            for (int jj = 0; jj < NCC; ++jj)
#pragma unroll
                for (int kk = 0; kk < KPC; ++kk)
                    if (jj * KPC + kk == f) v = acc[jj][kk];
            int chj = 0;
#pragma unroll
            for (int jj = 0; jj < NCC; ++jj)
                if (jj == j) chj = ch[jj];
            for (int q = 0; q < nl; ++q) {
                const int d = x - s_lx[wl][q];
                const float* rk = R + ((int64_t)k * KPC) * nd + (d + nt - 1);
                const float* uy = U + (int64_t)s_ly[wl][q] * KPC * C + chj;
                float sub = 0.f;
#pragma unroll
                for (int kk = 0; kk < KPC; ++kk) sub = fmaf(__ldg(uy + (int64_t)kk * C), __ldg(rk + (int64_t)kk * nd), sub);
                v = __fsub_rn(v, __fmul_rn(s_la[wl][q], sub));
            }
            v = __fadd_rn(v, __fmul_rn(sp_amp[i], Ucc[((int64_t)j * T + y) * KPC + k]));
            tF[(int64_t)i * F + f] = v;
        }
        __syncwarp();
    }
}

// CTA per spike, grid-stride over the spikes; with counters != null the spike
// and round counts are read from the matching pursuit's device counters
// (graph-captured batches, whose launch does not know them).
template <typename PT>
__global__ void __launch_bounds__(256) k_pc_features_folded(
    const float* __restrict__ Xh, int64_t ldx, int32_t C, int32_t nt, int32_t K, int32_t nC, int32_t T,
    const float* __restrict__ wpca, const float* __restrict__ Mw, const float* __restrict__ U,
    const float* __restrict__ R, const int64_t* __restrict__ iCC, const int64_t* __restrict__ iU,
    const float* __restrict__ Ucc, const int32_t* __restrict__ sp_x, const int32_t* __restrict__ sp_y,
    const float* __restrict__ sp_amp, const int32_t* __restrict__ round_start, int32_t rounds, int32_t n,
    const int32_t* __restrict__ counters, float* __restrict__ tF, int32_t* status, const PT* __restrict__ Phi,
    const PT* __restrict__ Plo, int64_t ldp) {
    if (counters) {
        n = counters[0];
        rounds = counters[1];
    }
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        pc_features_one(i, rounds, Xh, ldx, C, nt, K, nC, T, wpca, Mw, U, R, iCC, iU, Ucc, sp_x, sp_y, sp_amp,
                        round_start, tF, status, Phi, Plo, ldp);
        __syncthreads();
    }
}

template <typename PT>
static cudaError_t launch_pcf(const float* Xh, int64_t ldx, int32_t C, int32_t nt, int32_t K, int32_t nC, int32_t T,
                              const float* wpca, const float* Mw, const float* U, const float* R, const int64_t* iCC,
                              const int64_t* iU, const float* Ucc, const int32_t* sp_x, const int32_t* sp_y,
                              const float* sp_amp, const int32_t* round_start, int32_t rounds, int32_t n,
                              const int32_t* counters, float* tF, int32_t* status, const PT* Phi, const PT* Plo,
                              int64_t ldp, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (Phi && K == 6 && nC == 10) {
        // warp per spike; n: the spike count or (counters) the grid bound in spikes
        const int grid = (n + 7) / 8;
        k_pc_features_warp<6, 10, PT><<<grid, 256, 0, s>>>(C, nt, T, Mw, U, R, iCC, iU, Ucc, sp_x, sp_y, sp_amp,
                                                           round_start, rounds, n, counters, tF, status, Phi, Plo,
                                                           ldp);
        return cudaGetLastError();
    }
    if (nC * K > 256) return cudaErrorInvalidValue;  // one (j, k) per thread
    const size_t front = std::max<size_t>((size_t)K * nt + (size_t)FT_CH * (nt + 1) + (size_t)FT_CH * K +
                                              (size_t)nC * FT_CH,
                                          (size_t)C * K + (size_t)nC * C + 4 * (size_t)nC * K);
    const size_t smem = sizeof(float) * (front + (size_t)nC * K + (size_t)FT_NQ * nC * K);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(k_pc_features_folded<PT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // n: the spike count, or (counters != null) the grid size
    k_pc_features_folded<PT><<<n, 256, smem, s>>>(Xh, ldx, C, nt, K, nC, T, wpca, Mw, U, R, iCC, iU, Ucc, sp_x,
                                                  sp_y, sp_amp, round_start, rounds, n, counters, tF, status, Phi, Plo,
                                                  ldp);
    return cudaGetLastError();
}

cudaError_t launch_pc_features_folded(const float* Xh, int64_t ldx, int32_t C, int32_t nt, int32_t K, int32_t nC,
                                      int32_t T, const float* wpca, const float* Mw, const float* U, const float* R,
                                      const int64_t* iCC, const int64_t* iU, const float* Ucc, const int32_t* sp_x,
                                      const int32_t* sp_y, const float* sp_amp, const int32_t* round_start,
                                      int32_t rounds, int32_t n, const int32_t* counters, float* tF,
                                      int32_t* status, const void* Phi, const void* Plo, int32_t p_bf16, int64_t ldp,
                                      cudaStream_t s) {
    if (p_bf16)
        return launch_pcf<__nv_bfloat16>(Xh, ldx, C, nt, K, nC, T, wpca, Mw, U, R, iCC, iU, Ucc, sp_x, sp_y, sp_amp,
                                         round_start, rounds, n, counters, tF, status,
                                         static_cast<const __nv_bfloat16*>(Phi),
                                         static_cast<const __nv_bfloat16*>(Plo), ldp, s);
    return launch_pcf<float>(Xh, ldx, C, nt, K, nC, T, wpca, Mw, U, R, iCC, iU, Ucc, sp_x, sp_y, sp_amp, round_start,
                             rounds, n, counters, tF, status, static_cast<const float*>(Phi),
                             static_cast<const float*>(Plo), ldp, s);
}

// acc |= *st (errors of asynchronous batches, collected until lss_sync)
__global__ void k_status_or(const int32_t* st, int32_t* acc) {
    if (*st) atomicOr(acc, *st);
}

cudaError_t launch_status_or(const int32_t* st, int32_t* acc, cudaStream_t s) {
    k_status_or<<<1, 1, 0, s>>>(st, acc);
    return cudaGetLastError();
}

}  // namespace lss
