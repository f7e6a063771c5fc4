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

cudaError_t launch_sgemm(const float* A, int64_t lda, const float* B, int64_t ldb, float* Cm, int64_t ldc,
                         int M, int N, int K, cudaStream_t s) {
    dim3 grid((N + GBN - 1) / GBN, (M + GBM - 1) / GBM);
    k_sgemm<<<grid, 256, 0, s>>>(A, lda, B, ldb, Cm, ldc, M, N, K);
    return cudaGetLastError();
}

}  // namespace lss
