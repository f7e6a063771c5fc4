// FP32 SIMT GEMM, C[M,N] = A[M,K] @ B[K,N], all row-major.
//
// Used by the FP32 parity path for the whitening/drift product
// ((M @ Wrot) @ X, kilosort/io.py:782-789; cublasSgemm in
// OnlineSpikesV2.cu:767-778) and the template score GEMM
// (einsum('ijk,kjl->il'), template_matching.py:146;
// cross_correlation_kernel, myGPUhelpers.cu:262-336).
// Each output is a single FP32 FMA chain over k in ascending order, so the
// result is deterministic and independent of the launch shape.
//
// Tiling: 128x128 CTA tile, BK = 8, 256 threads, 8x8 outputs per thread
// (two 4x4 quadrants 64 apart so shared-memory reads are conflict-free
// float4s), register prefetch of the next k-slab while the current one is
// consumed from the other shared-memory buffer.
#include "lss_kernels.cuh"

#include <cuda_bf16.h>

namespace lss {

constexpr int GBM = 128, GBN = 128, GBK = 8;

__global__ void __launch_bounds__(256) k_sgemm(const float* __restrict__ A, int64_t lda,
                                               const float* __restrict__ B, int64_t ldb,
                                               float* __restrict__ Cm, int64_t ldc, int M, int N, int K) {
    __shared__ __align__(16) float As[2][GBK][GBM];
    __shared__ __align__(16) float Bs[2][GBK][GBN];
    const int tid = threadIdx.x;
    const int m0 = blockIdx.y * GBM;
    const int n0 = blockIdx.x * GBN;
    const int tx = tid & 15, ty = tid >> 4;

    // global->register staging: A slab 128x8 (4 per thread), B slab 8x128 (4 per thread)
    float ra[4], rb[4];
    auto load_slab = [&](int k0) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int idx = tid + 256 * i;
            const int kk = idx & 7, mm = idx >> 3;
            const int gm = m0 + mm, gk = k0 + kk;
            ra[i] = (gm < M && gk < K) ? A[(int64_t)gm * lda + gk] : 0.f;
            const int nn = idx & 127, kb = idx >> 7;
            const int gn = n0 + nn, gkb = k0 + kb;
            rb[i] = (gn < N && gkb < K) ? B[(int64_t)gkb * ldb + gn] : 0.f;
        }
    };
    auto store_slab = [&](int buf) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int idx = tid + 256 * i;
            As[buf][idx & 7][idx >> 3] = ra[i];
            Bs[buf][idx >> 7][idx & 127] = rb[i];
        }
    };

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

    const int nslab = (K + GBK - 1) / GBK;
    load_slab(0);
    store_slab(0);
    __syncthreads();
    for (int t = 0; t < nslab; ++t) {
        const int buf = t & 1;
        if (t + 1 < nslab) load_slab((t + 1) * GBK);
#pragma unroll
        for (int kk = 0; kk < GBK; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 4 + 64]);
            const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4]);
            const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4 + 64]);
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        if (t + 1 < nslab) store_slab(buf ^ 1);
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int gm = m0 + ty * 4 + (i & 3) + (i >> 2) * 64;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int gn = n0 + tx * 4 + (j & 3) + (j >> 2) * 64;
            if (gn < N) Cm[(int64_t)gm * ldc + gn] = acc[i][j];
        }
    }
}

// Small products (the C x C drift/whitening product, the folded templates)
// give the 128x128 tiling a handful of CTAs; they run on 64x64 tiles instead
// (BK = 16, 4x4 outputs per thread). Each output is the same FMA chain over
// k in ascending order, so the two tilings give identical bits.
constexpr int SBM = 64, SBN = 64, SBK = 16;

struct StorePlain {
    float* Cm;
    int64_t ldc;
    __device__ void operator()(int m, int n, float v) const { Cm[(int64_t)m * ldc + n] = v; }
};

// Folded-template layout of the score GEMM: row m = t*K + k, column n = c'
// goes to [t, c'*K + k] of a row-stride-ldk array, as the bf16 split
// hi = bf16(v), lo = bf16(v - hi) or as the tf32 split hi = rna(v),
// lo = rna(v - hi) (both exact tf32 values).
struct StoreFolded {
    int K;
    int64_t ldk;
    __nv_bfloat16* out16;
    __nv_bfloat16* out16lo;
    float* hi;
    float* lo;
    __device__ void operator()(int m, int n, float v) const {
        const int t = m / K, k = m - (m / K) * K;
        const int64_t o = (int64_t)t * ldk + (int64_t)n * K + k;
        if (out16) {
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            out16[o] = h;
            if (out16lo) out16lo[o] = __float2bfloat16_rn(__fsub_rn(v, __bfloat162float(h)));
        }
        if (hi) {
            uint32_t r;
            asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
            const float h = __uint_as_float(r);
            hi[o] = h;
            asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(__fsub_rn(v, h)));
            lo[o] = __uint_as_float(r);
        }
    }
};

template <class Store>
__global__ void __launch_bounds__(256) k_sgemm64(const float* __restrict__ A, int64_t lda,
                                                 const float* __restrict__ B, int64_t ldb, int M, int N, int K,
                                                 Store store) {
    __shared__ __align__(16) float As[SBK][SBM];
    __shared__ __align__(16) float Bs[SBK][SBN];
    const int tid = threadIdx.x;
    const int m0 = blockIdx.y * SBM, n0 = blockIdx.x * SBN;
    const int tx = tid & 15, ty = tid >> 4;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    for (int k0 = 0; k0 < K; k0 += SBK) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int idx = tid + 256 * i;                 // 0 .. 1023
            const int kk = idx & (SBK - 1), mm = idx >> 4;  // A slab: 64 rows x 16 k
            const int gm = m0 + mm, gk = k0 + kk;
            As[kk][mm] = (gm < M && gk < K) ? A[(int64_t)gm * lda + gk] : 0.f;
            const int nn = idx & (SBN - 1), kb = idx >> 6;  // B slab: 16 k x 64 columns
            const int gn = n0 + nn, gkb = k0 + kb;
            Bs[kb][nn] = (gn < N && gkb < K) ? B[(int64_t)gkb * ldb + gn] : 0.f;
        }
        __syncthreads();
        const int kn = min(SBK, K - k0);
#pragma unroll
        for (int kk = 0; kk < SBK; ++kk) {
            if (kk < kn) {  // no terms past K: the chain is exactly k = 0 .. K-1
                const float4 a = *reinterpret_cast<const float4*>(&As[kk][ty * 4]);
                const float4 b = *reinterpret_cast<const float4*>(&Bs[kk][tx * 4]);
                const float av[4] = {a.x, a.y, a.z, a.w};
                const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gm = m0 + ty * 4 + i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int gn = n0 + tx * 4 + j;
            if (gn < N) store(gm, gn, acc[i][j]);
        }
    }
}

cudaError_t launch_sgemm(const float* A, int64_t lda, const float* B, int64_t ldb, float* Cm, int64_t ldc,
                         int M, int N, int K, cudaStream_t s) {
    // fewer 128x128 tiles than a B200 has SMs: 64x64 tiles
    const int64_t big_ctas = (int64_t)((N + GBN - 1) / GBN) * ((M + GBM - 1) / GBM);
    if (big_ctas < 148) {
        dim3 grid((N + SBN - 1) / SBN, (M + SBM - 1) / SBM);
        k_sgemm64<StorePlain><<<grid, 256, 0, s>>>(A, lda, B, ldb, M, N, K, StorePlain{Cm, ldc});
        return cudaGetLastError();
    }
    dim3 grid((N + GBN - 1) / GBN, (M + GBM - 1) / GBM);
    k_sgemm<<<grid, 256, 0, s>>>(A, lda, B, ldb, Cm, ldc, M, N, K);
    return cudaGetLastError();
}

cudaError_t launch_sgemm_folded(const float* U, const float* Mw, int32_t T, int32_t K, int32_t C, int64_t ldk,
                                __nv_bfloat16* out16, __nv_bfloat16* out16lo, float* hi, float* lo, cudaStream_t s) {
    // rows t*K + k of U [T, K, C] (row-major, stride C) times Mw [C, C]
    dim3 grid((C + SBN - 1) / SBN, (T * K + SBM - 1) / SBM);
    k_sgemm64<StoreFolded><<<grid, 256, 0, s>>>(U, C, Mw, C, T * K, C, C, StoreFolded{K, ldk, out16, out16lo, hi, lo});
    return cudaGetLastError();
}

}  // namespace lss
