// Reconstruction of a batch from its spikes and the templates, and the
// reconstruction's adjoint (lss_recon_forward / lss_recon_backward).
//
// Kilosort subtracts each accepted spike from the batch as
//   Xres[:, x_i + m - nt/2] -= a_i * sum_k U[y_i, k, :] wPCA[k, m]
// (template_matching.py:195-198, the einsum('ijk,jl->kil', U[iY], W) term), so
// the reconstruction is
//   R[c, s] = sum_i a_i sum_k U[y_i, k, c] wPCA[k, s - x_i + nt/2].
// With the assignments (x_i, y_i, a_i) fixed, R is linear in U and in wPCA;
// for an upstream gradient G = dL/dR the adjoint is
//   P_i[k, c]   = sum_m wPCA[k, m] G[c, x_i + m - nt/2]   (the temporal-basis
//                 convolution of G, recomputed per spike: nothing is stored
//                 by the forward pass)
//   dL/dU[t]    = sum_{i: y_i = t} a_i P_i
//   dL/dwPCA    = sum_i a_i sum_c U[y_i, :, c] G[c, x_i + (.) - nt/2]
//   dL/da_i     = sum_{k, c} U[y_i, k, c] P_i[k, c]
// Both passes are deterministic: the forward gathers per output column over
// the spikes in time order, the backward runs one CTA per template over that
// template's spikes in a fixed order and reduces dL/dwPCA over templates in
// template order. F = float or double (the finite-difference checks run the
// same kernels in FP64).
#include <cuda_runtime.h>

#include <cstdint>

#include "lss.h"
#include "lss_kernels.cuh"

namespace lss {

constexpr int RF_COLS = 128;   // output columns per CTA
constexpr int RF_CH = 32;      // channels per CTA
constexpr int RF_SP = 8;       // spikes staged per step
constexpr int RB_CH = 32;      // channels per backward chunk
constexpr int RB_THREADS = 256;

__device__ __forceinline__ int lower_bound_i(const int32_t* a, int n, int v) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// xs/ys/as: spikes sorted by x.
template <typename F>
__global__ void __launch_bounds__(RF_COLS) k_recon_fwd(const F* __restrict__ U, const F* __restrict__ W, int K, int C,
                                                       int nt, const int32_t* __restrict__ xs,
                                                       const int32_t* __restrict__ ys, const F* __restrict__ as,
                                                       int n, F* __restrict__ R, int64_t N) {
    extern __shared__ unsigned char rf_smem[];
    F* Ws = reinterpret_cast<F*>(rf_smem);       // [K][nt]
    F* Us = Ws + K * nt;                          // [RF_SP][K][RF_CH]
    __shared__ int s_x[RF_SP];
    __shared__ F s_a[RF_SP];
    const int h = nt / 2;
    const int64_t t0 = (int64_t)blockIdx.x * RF_COLS;
    const int c0 = blockIdx.y * RF_CH;
    const int nc = min(RF_CH, C - c0);
    const int64_t col = t0 + threadIdx.x;
    for (int e = threadIdx.x; e < K * nt; e += blockDim.x) Ws[e] = W[e];
    // spikes whose window [x - h, x - h + nt) meets [t0, t0 + RF_COLS)
    const int lo = lower_bound_i(xs, n, (int)(t0 - (nt - 1 - h)));
    const int hi = lower_bound_i(xs, n, (int)(t0 + RF_COLS + h));
    F acc[RF_CH];
#pragma unroll
    for (int c = 0; c < RF_CH; ++c) acc[c] = F(0);
    for (int i0 = lo; i0 < hi; i0 += RF_SP) {
        const int ns = min(RF_SP, hi - i0);
        __syncthreads();
        for (int e = threadIdx.x; e < ns * K * RF_CH; e += blockDim.x) {
            const int q = e / (K * RF_CH), r = e % (K * RF_CH);
            const int k = r / RF_CH, c = r % RF_CH;
            Us[e] = (c < nc) ? U[((int64_t)ys[i0 + q] * K + k) * C + c0 + c] : F(0);
        }
        if (threadIdx.x < ns) {
            s_x[threadIdx.x] = xs[i0 + threadIdx.x];
            s_a[threadIdx.x] = as[i0 + threadIdx.x];
        }
        __syncthreads();
        for (int q = 0; q < ns; ++q) {
            const int m = (int)(col - s_x[q] + h);
            if (m < 0 || m >= nt) continue;
            const F a = s_a[q];
            const F* uq = Us + q * K * RF_CH;
#pragma unroll
            for (int c = 0; c < RF_CH; ++c) {
                F w = F(0);
                for (int k = 0; k < K; ++k) w += uq[k * RF_CH + c] * Ws[k * nt + m];
                acc[c] += a * w;
            }
        }
    }
    if (col < N)
        for (int c = 0; c < nc; ++c) R[(int64_t)(c0 + c) * N + col] = acc[c];
}

// One CTA per template t; order[tstart[t] .. tstart[t+1]) are its spikes.
template <typename F>
__global__ void __launch_bounds__(RB_THREADS) k_recon_bwd(const F* __restrict__ U, const F* __restrict__ W, int K,
                                                          int C, int nt, const int32_t* __restrict__ x,
                                                          const F* __restrict__ amp, const int32_t* __restrict__ order,
                                                          const int32_t* __restrict__ tstart, const F* __restrict__ G,
                                                          int64_t N, F* __restrict__ dU, F* __restrict__ Qt,
                                                          F* __restrict__ damp) {
    extern __shared__ unsigned char rb_smem[];
    F* Ws = reinterpret_cast<F*>(rb_smem);        // [K][nt]
    F* Ut = Ws + K * nt;                           // [K][C]  U[t]
    F* dUt = Ut + K * C;                           // [K][C]  accumulated dU[t]
    F* Qa = dUt + K * C;                           // [K][nt] accumulated a_i * Q_i
    F* win = Qa + K * nt;                          // [RB_CH][nt + 1]
    F* red = win + RB_CH * (nt + 1);               // [RB_THREADS]
    const int t = blockIdx.x;
    const int h = nt / 2;
    const int ntp = nt + 1;
    for (int e = threadIdx.x; e < K * nt; e += blockDim.x) {
        Ws[e] = W[e];
        Qa[e] = F(0);
    }
    for (int e = threadIdx.x; e < K * C; e += blockDim.x) {
        Ut[e] = U[(int64_t)t * K * C + e];
        dUt[e] = F(0);
    }
    const int j0 = tstart[t], j1 = tstart[t + 1];
    for (int j = j0; j < j1; ++j) {
        const int i = order[j];
        const int xi = x[i];
        const F ai = amp[i];
        F dsum = F(0);  // this thread's share of dL/da_i
        for (int c0 = 0; c0 < C; c0 += RB_CH) {
            const int nc = min(RB_CH, C - c0);
            __syncthreads();
            for (int e = threadIdx.x; e < nc * nt; e += blockDim.x) {
                const int c = e / nt, m = e % nt;
                const int64_t s = (int64_t)xi + m - h;
                win[c * ntp + m] = (s >= 0 && s < N) ? G[(int64_t)(c0 + c) * N + s] : F(0);
            }
            __syncthreads();
            // P_i[k, c] for the chunk: dU and dL/da_i
            for (int e = threadIdx.x; e < nc * K; e += blockDim.x) {
                const int c = e / K, k = e % K;
                F p = F(0);
                for (int m = 0; m < nt; ++m) p += Ws[k * nt + m] * win[c * ntp + m];
                dUt[k * C + c0 + c] += ai * p;
                dsum += Ut[k * C + c0 + c] * p;
            }
            // Q_i[k, m] over the chunk's channels (each (k, m) owned by one thread)
            for (int e = threadIdx.x; e < K * nt; e += blockDim.x) {
                const int k = e / nt, m = e % nt;
                F q = F(0);
                for (int c = 0; c < nc; ++c) q += Ut[k * C + c0 + c] * win[c * ntp + m];
                Qa[e] += ai * q;
            }
        }
        // dL/da_i: fixed-order tree reduction of the threads' shares
        red[threadIdx.x] = dsum;
        __syncthreads();
        for (int w = RB_THREADS / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0 && damp) damp[i] = red[0];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < K * C; e += blockDim.x) dU[(int64_t)t * K * C + e] = dUt[e];
    for (int e = threadIdx.x; e < K * nt; e += blockDim.x) Qt[(int64_t)t * K * nt + e] = Qa[e];
}

template <typename F>
__global__ void k_reduce_templates(const F* __restrict__ Qt, int T, int KN, F* __restrict__ dW) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= KN) return;
    F s = F(0);
    for (int t = 0; t < T; ++t) s += Qt[(int64_t)t * KN + e];
    dW[e] = s;
}

template <typename F>
static cudaError_t recon_fwd(const void* U, const void* W, int K, int C, int nt, const int32_t* xs, const int32_t* ys,
                             const void* as, int n, void* R, int64_t N, cudaStream_t s) {
    const size_t smem = sizeof(F) * ((size_t)K * nt + (size_t)RF_SP * K * RF_CH);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_recon_fwd<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((unsigned)((N + RF_COLS - 1) / RF_COLS), (unsigned)((C + RF_CH - 1) / RF_CH));
    k_recon_fwd<F><<<grid, RF_COLS, smem, s>>>(static_cast<const F*>(U), static_cast<const F*>(W), K, C, nt, xs, ys,
                                               static_cast<const F*>(as), n, static_cast<F*>(R), N);
    return cudaGetLastError();
}

template <typename F>
static cudaError_t recon_bwd(const void* U, const void* W, int T, int K, int C, int nt, const int32_t* x,
                             const void* amp, const int32_t* order, const int32_t* tstart, const void* G, int64_t N,
                             void* dU, void* dW, void* damp, void* work, cudaStream_t s) {
    const size_t smem = sizeof(F) * (2 * (size_t)K * nt + 2 * (size_t)K * C + (size_t)RB_CH * (nt + 1) + RB_THREADS);
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_recon_bwd<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_recon_bwd<F><<<T, RB_THREADS, smem, s>>>(static_cast<const F*>(U), static_cast<const F*>(W), K, C, nt, x,
                                               static_cast<const F*>(amp), order, tstart, static_cast<const F*>(G),
                                               N, static_cast<F*>(dU), static_cast<F*>(work), static_cast<F*>(damp));
    const int KN = K * nt;
    k_reduce_templates<F><<<(KN + 255) / 256, 256, 0, s>>>(static_cast<const F*>(work), T, KN, static_cast<F*>(dW));
    return cudaGetLastError();
}

}  // namespace lss

using namespace lss;

static int recon_args_ok(int32_t dtype, int32_t T, int32_t K, int32_t C, int32_t nt, int64_t n, int64_t N) {
    if (dtype != 0 && dtype != 1) return 0;
    if (T <= 0 || K <= 0 || K > 16 || C <= 0 || nt <= 0 || nt > 255 || n < 0 || n > INT32_MAX || N <= 0) return 0;
    return 1;
}

extern "C" {

int lss_recon_forward(int32_t dtype, const void* U, const void* wPCA, int32_t T, int32_t K, int32_t C, int32_t nt,
                      const int32_t* x_sorted, const int32_t* y, const void* amp, int64_t n, void* R, int64_t N,
                      void* stream) {
    if (!recon_args_ok(dtype, T, K, C, nt, n, N) || !U || !wPCA || !R || (n > 0 && (!x_sorted || !y || !amp))) {
        lss::set_thread_error("lss_recon_forward: bad argument");
        return LSS_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const cudaError_t e = dtype == 0 ? recon_fwd<float>(U, wPCA, K, C, nt, x_sorted, y, amp, (int)n, R, N, s)
                                     : recon_fwd<double>(U, wPCA, K, C, nt, x_sorted, y, amp, (int)n, R, N, s);
    if (e != cudaSuccess) {
        lss::set_thread_error(cudaGetErrorString(e));
        return LSS_ERR_CUDA;
    }
    return LSS_OK;
}

int lss_recon_backward(int32_t dtype, const void* U, const void* wPCA, int32_t T, int32_t K, int32_t C, int32_t nt,
                       const int32_t* x, const void* amp, const int32_t* order_by_template,
                       const int32_t* template_start, const void* dR, int64_t N, void* dU, void* dwPCA, void* damp,
                       void* work, void* stream) {
    if (!recon_args_ok(dtype, T, K, C, nt, 0, N) || !U || !wPCA || !x || !amp || !order_by_template ||
        !template_start || !dR || !dU || !dwPCA || !work) {
        lss::set_thread_error("lss_recon_backward: bad argument");
        return LSS_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const cudaError_t e =
        dtype == 0 ? recon_bwd<float>(U, wPCA, T, K, C, nt, x, amp, order_by_template, template_start, dR, N, dU,
                                      dwPCA, damp, work, s)
                   : recon_bwd<double>(U, wPCA, T, K, C, nt, x, amp, order_by_template, template_start, dR, N, dU,
                                       dwPCA, damp, work, s);
    if (e != cudaSuccess) {
        lss::set_thread_error(cudaGetErrorString(e));
        return LSS_ERR_CUDA;
    }
    return LSS_OK;
}

}  // extern "C"
