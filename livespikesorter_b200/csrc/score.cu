// Temporal-basis projection of the filtered batch:
//   B0[c*K + k, s] = sum_m wPCA[k, m] * X[c, s + m - nt/2]   (zero outside [0, N))
// which is conv1d(X.unsqueeze(1), W.unsqueeze(1), padding=nt//2) of
// kilosort/template_matching.py:145 (conv1d kernel, myGPUhelpers.cu:355-399).
// The row order (c, k) lets the score GEMM contract over c*K + k with the
// template matrix permuted once at set-up to U_p[t, c*K + k] = U[t, k, c].
//
// CTA: one channel, PJ_TILE outputs for all K components; thread: 8
// consecutive samples x K components with a sliding register window (one
// shared load of X per 8*K FMAs).
#include "lss_kernels.cuh"

#include <cuda_bf16.h>

namespace lss {

constexpr int PJ_TILE = 1024;
constexpr int PJ_THREADS = PJ_TILE / 8;

template <int KPC>
__global__ void __launch_bounds__(PJ_THREADS) k_pca_proj(const float* __restrict__ X, int64_t ldx, int64_t N,
                                                         const float* __restrict__ wpca, int32_t nt,
                                                         float* __restrict__ B0, int64_t ldb0) {
    extern __shared__ float sm[];
    const int ntp = (nt + 7) & ~7;
    float* ws = sm;                  // [KPC][ntp]
    float* xs = sm + KPC * ntp;      // [PJ_TILE + ntp + 8]
    const int c = blockIdx.y;
    const int64_t s0 = (int64_t)blockIdx.x * PJ_TILE;
    const int half = nt / 2;
    for (int e = threadIdx.x; e < KPC * ntp; e += blockDim.x) {
        const int k = e / ntp, m = e % ntp;
        ws[e] = (m < nt) ? wpca[k * nt + m] : 0.f;
    }
    const float* xrow = X + (int64_t)c * ldx;
    const int nx = PJ_TILE + ntp + 8;
    for (int p = threadIdx.x; p < nx; p += blockDim.x) {
        const int64_t g = s0 - half + p;
        xs[p] = (g >= 0 && g < N) ? xrow[g] : 0.f;
    }
    __syncthreads();
    float acc[KPC][8];
#pragma unroll
    for (int k = 0; k < KPC; ++k)
#pragma unroll
        for (int r = 0; r < 8; ++r) acc[k][r] = 0.f;
    const int o = threadIdx.x * 8;
    float w[16];
#pragma unroll
    for (int r = 0; r < 8; ++r) w[r] = xs[o + r];
    for (int mb = 0; mb < ntp; mb += 8) {
#pragma unroll
        for (int r = 0; r < 8; ++r) w[8 + r] = xs[o + mb + 8 + r];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
#pragma unroll
            for (int k = 0; k < KPC; ++k) {
                const float t = ws[k * ntp + mb + u];
#pragma unroll
                for (int r = 0; r < 8; ++r) acc[k][r] = fmaf(t, w[r + u], acc[k][r]);
            }
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) w[r] = w[8 + r];
    }
#pragma unroll
    for (int k = 0; k < KPC; ++k) {
        float* row = B0 + ((int64_t)c * KPC + k) * ldb0;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int64_t s = s0 + o + r;
            if (s < N) row[s] = acc[k][r];
        }
    }
}

template <int KPC>
static cudaError_t launch_pj(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t nt,
                             float* B0, int64_t ldb0, cudaStream_t s) {
    const int ntp = (nt + 7) & ~7;
    const size_t smem = sizeof(float) * ((size_t)KPC * ntp + PJ_TILE + ntp + 8);
    dim3 grid((unsigned)((N + PJ_TILE - 1) / PJ_TILE), (unsigned)C);
    k_pca_proj<KPC><<<grid, PJ_THREADS, smem, s>>>(X, ldx, N, wpca, nt, B0, ldb0);
    return cudaGetLastError();
}

cudaError_t launch_pca_proj(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t K,
                            int32_t nt, float* B0, int64_t ldb0, cudaStream_t s) {
    switch (K) {
        case 1: return launch_pj<1>(X, ldx, C, N, wpca, nt, B0, ldb0, s);
        case 2: return launch_pj<2>(X, ldx, C, N, wpca, nt, B0, ldb0, s);
        case 3: return launch_pj<3>(X, ldx, C, N, wpca, nt, B0, ldb0, s);
        case 4: return launch_pj<4>(X, ldx, C, N, wpca, nt, B0, ldb0, s);
        case 5: return launch_pj<5>(X, ldx, C, N, wpca, nt, B0, ldb0, s);
        case 6: return launch_pj<6>(X, ldx, C, N, wpca, nt, B0, ldb0, s);
        case 7: return launch_pj<7>(X, ldx, C, N, wpca, nt, B0, ldb0, s);
        case 8: return launch_pj<8>(X, ldx, C, N, wpca, nt, B0, ldb0, s);
        default: return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------
// Transposed projection for the tensor-core score GEMM:
//   B0T[s, c*K + k] = bf16( sum_m wPCA[k, m] * X[c, s + m - nt/2] )
// rows = samples (the GEMM's M), columns = (channel, component) (its K),
// row stride ldk (a multiple of 64, the pad columns stay zero). CTA: 64
// samples x 64 channels; the bf16 tile is staged in shared memory and written
// as 2*64*K-byte row segments.
// ---------------------------------------------------------------------------
constexpr int PT_S = 64;    // samples per CTA
constexpr int PT_C = 64;    // channels per CTA

template <int KPC>
__global__ void __launch_bounds__(256) k_pca_proj_t(const float* __restrict__ X, int64_t ldx, int32_t C, int64_t N,
                                                    const float* __restrict__ wpca, int32_t nt,
                                                    __nv_bfloat16* __restrict__ B0T, int64_t ldk) {
    extern __shared__ float sm[];
    const int ntp = (nt + 7) & ~7;
    const int xw = PT_S + ntp + 8;                 // staged samples per channel row
    float* ws = sm;                                // [KPC][ntp]
    float* xs = ws + KPC * ntp;                    // [PT_C][xw]
    __nv_bfloat16* out = reinterpret_cast<__nv_bfloat16*>(xs + PT_C * xw);  // [PT_S][PT_C*KPC]
    const int64_t s0 = (int64_t)blockIdx.x * PT_S;
    const int c0 = blockIdx.y * PT_C;
    const int nc = min(PT_C, C - c0);
    const int half = nt / 2;
    for (int e = threadIdx.x; e < KPC * ntp; e += blockDim.x) {
        const int k = e / ntp, m = e % ntp;
        ws[e] = (m < nt) ? wpca[k * nt + m] : 0.f;
    }
    for (int e = threadIdx.x; e < PT_C * xw; e += blockDim.x) {
        const int c = e / xw, p = e % xw;
        const int64_t g = s0 - half + p;
        xs[e] = (c < nc && g >= 0 && g < N) ? X[(int64_t)(c0 + c) * ldx + g] : 0.f;
    }
    __syncthreads();
    // task = (channel, 8-sample group)
    for (int task = threadIdx.x; task < PT_C * (PT_S / 8); task += blockDim.x) {
        const int c = task % PT_C, sg = task / PT_C;
        const float* xr = xs + c * xw + sg * 8;
        float acc[KPC][8];
#pragma unroll
        for (int k = 0; k < KPC; ++k)
#pragma unroll
            for (int r = 0; r < 8; ++r) acc[k][r] = 0.f;
        float w[16];
#pragma unroll
        for (int r = 0; r < 8; ++r) w[r] = xr[r];
        for (int mb = 0; mb < ntp; mb += 8) {
#pragma unroll
            for (int r = 0; r < 8; ++r) w[8 + r] = xr[mb + 8 + r];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
#pragma unroll
                for (int k = 0; k < KPC; ++k) {
                    const float t = ws[k * ntp + mb + u];
#pragma unroll
                    for (int r = 0; r < 8; ++r) acc[k][r] = fmaf(t, w[r + u], acc[k][r]);
                }
            }
#pragma unroll
            for (int r = 0; r < 8; ++r) w[r] = w[8 + r];
        }
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
            for (int k = 0; k < KPC; ++k) out[(sg * 8 + r) * (PT_C * KPC) + c * KPC + k] = __float2bfloat16_rn(acc[k][r]);
    }
    __syncthreads();
    // row segments: PT_S rows of nc*KPC bf16 each
    const int seg = nc * KPC;
    for (int e = threadIdx.x; e < PT_S * seg; e += blockDim.x) {
        const int r = e / seg, j = e % seg;
        const int64_t s = s0 + r;
        if (s < N) B0T[s * ldk + (int64_t)c0 * KPC + j] = out[r * (PT_C * KPC) + j];
    }
}

template <int KPC>
static cudaError_t launch_pjt(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t nt,
                              __nv_bfloat16* B0T, int64_t ldk, cudaStream_t s) {
    const int ntp = (nt + 7) & ~7;
    const size_t smem = sizeof(float) * ((size_t)KPC * ntp + (size_t)PT_C * (PT_S + ntp + 8)) +
                        sizeof(__nv_bfloat16) * (size_t)PT_S * PT_C * KPC;
    cudaFuncSetAttribute(k_pca_proj_t<KPC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid((unsigned)((N + PT_S - 1) / PT_S), (unsigned)((C + PT_C - 1) / PT_C));
    k_pca_proj_t<KPC><<<grid, 256, smem, s>>>(X, ldx, C, N, wpca, nt, B0T, ldk);
    return cudaGetLastError();
}

cudaError_t launch_pca_proj_t(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t K,
                              int32_t nt, __nv_bfloat16* B0T, int64_t ldk, cudaStream_t s) {
    switch (K) {
        case 1: return launch_pjt<1>(X, ldx, C, N, wpca, nt, B0T, ldk, s);
        case 2: return launch_pjt<2>(X, ldx, C, N, wpca, nt, B0T, ldk, s);
        case 3: return launch_pjt<3>(X, ldx, C, N, wpca, nt, B0T, ldk, s);
        case 4: return launch_pjt<4>(X, ldx, C, N, wpca, nt, B0T, ldk, s);
        case 5: return launch_pjt<5>(X, ldx, C, N, wpca, nt, B0T, ldk, s);
        case 6: return launch_pjt<6>(X, ldx, C, N, wpca, nt, B0T, ldk, s);
        case 7: return launch_pjt<7>(X, ldx, C, N, wpca, nt, B0T, ldk, s);
        case 8: return launch_pjt<8>(X, ldx, C, N, wpca, nt, B0T, ldk, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace lss
