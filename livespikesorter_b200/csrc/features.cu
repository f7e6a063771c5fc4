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

namespace lss {

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

// One CTA per spike; thread (j, k) computes one feature.
__global__ void k_pc_features(const float* __restrict__ Xres, int64_t ldx, int32_t nt, int32_t K, int32_t nC,
                              int32_t C, int32_t T, const float* __restrict__ wpca,
                              const int64_t* __restrict__ iCC, const int64_t* __restrict__ iU,
                              const float* __restrict__ Ucc, const int32_t* __restrict__ sp_x,
                              const int32_t* __restrict__ sp_y, const float* __restrict__ sp_amp,
                              float* __restrict__ tF) {
    const int i = blockIdx.x;
    const int f = threadIdx.x;
    if (f >= nC * K) return;
    const int j = f / K, k = f % K;
    const int x = sp_x[i], y = sp_y[i];
    const int64_t ch = iCC[(int64_t)j * C + iU[y]];
    const float* xr = Xres + ch * ldx + (x - nt / 2);
    const float* w = wpca + (int64_t)k * nt;
    float acc = 0.f;
    for (int m = 0; m < nt; ++m) acc = fmaf(xr[m], w[m], acc);
    const float off = __fmul_rn(sp_amp[i], Ucc[((int64_t)j * T + y) * K + k]);
    tF[(int64_t)i * nC * K + f] = __fadd_rn(acc, off);
}

cudaError_t launch_pc_features(const float* Xres, int64_t ldx, int32_t nt, int32_t K, int32_t nC,
                               int32_t C, int32_t T, const float* wpca, const int64_t* iCC,
                               const int64_t* iU, const float* Ucc, const int32_t* sp_x,
                               const int32_t* sp_y, const float* sp_amp, const int32_t* counters,
                               int32_t n, float* tF, cudaStream_t s) {
    (void)counters;
    if (n <= 0) return cudaSuccess;
    const int threads = ((nC * K + 31) / 32) * 32;
    k_pc_features<<<n, threads, 0, s>>>(Xres, ldx, nt, K, nC, C, T, wpca, iCC, iU, Ucc, sp_x, sp_y, sp_amp, tF);
    return cudaGetLastError();
}

// Single-CTA ordered compaction of the batch's spikes into caller records.
__global__ void __launch_bounds__(1024) k_records(const int32_t* __restrict__ sp_x,
                                                  const int32_t* __restrict__ sp_y,
                                                  const float* __restrict__ sp_amp,
                                                  const float* __restrict__ tF, int32_t n, int32_t feat_len,
                                                  int64_t ibatch, int32_t nt, int32_t NT, int32_t nt0min,
                                                  int64_t* out_time, int32_t* out_tmpl, float* out_amp,
                                                  float* out_pc, int64_t capacity, int64_t* out_count) {
    __shared__ int scan[1024];
    __shared__ int64_t s_base;
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();
    for (int c0 = 0; c0 < n; c0 += 1024) {
        const int i = c0 + threadIdx.x;
        int keep = 0;
        int64_t t = 0;
        if (i < n) {
            const int x = sp_x[i];
            keep = !(ibatch == 0 && (x - nt - nt / 2 + nt0min) < 0);
            t = (int64_t)(x - nt) + ibatch * (int64_t)NT - nt / 2 + nt0min;
        }
        scan[threadIdx.x] = keep;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            const int v = (threadIdx.x >= off) ? scan[threadIdx.x - off] : 0;
            __syncthreads();
            scan[threadIdx.x] += v;
            __syncthreads();
        }
        if (keep) {
            const int64_t o = s_base + scan[threadIdx.x] - 1;
            if (o < capacity) {
                out_time[o] = t;
                out_tmpl[o] = sp_y[i];
                out_amp[o] = sp_amp[i];
                if (out_pc && tF)
                    for (int f = 0; f < feat_len; ++f) out_pc[o * feat_len + f] = tF[(int64_t)i * feat_len + f];
            }
        }
        __syncthreads();
        if (threadIdx.x == 1023) s_base += scan[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out_count = s_base;
}

cudaError_t launch_records(const int32_t* sp_x, const int32_t* sp_y, const float* sp_amp, const float* tF,
                           const int32_t* counters, int32_t n, int32_t feat_len, int64_t ibatch, int32_t nt,
                           int32_t NT, int32_t nt0min, int64_t* out_time, int32_t* out_tmpl,
                           float* out_amp, float* out_pc, int64_t capacity, int64_t* out_count,
                           cudaStream_t s) {
    (void)counters;
    k_records<<<1, 1024, 0, s>>>(sp_x, sp_y, sp_amp, tF, n, feat_len, ibatch, nt, NT, nt0min, out_time,
                                 out_tmpl, out_amp, out_pc, capacity, out_count);
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

}  // namespace lss
