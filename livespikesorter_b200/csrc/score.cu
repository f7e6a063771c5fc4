// Temporal-basis projection of the filtered batch:
//   B0[c*K + k, s] = sum_m wPCA[k, m] * X[c, s + m - nt/2]   (zero outside [0, N))
// which is conv1d(X.unsqueeze(1), W.unsqueeze(1), padding=nt//2) of
// kilosort/template_matching.py:145 (conv1d kernel, myGPUhelpers.cu:355-399).
// The row order (c, k) lets the score GEMM contract over c*K + k with the
// template matrix permuted once at set-up to U_p[t, c*K + k] = U[t, k, c].
#include "lss_kernels.cuh"

#include <cuda_bf16.h>

namespace lss {

// ---------------------------------------------------------------------------
// Transposed projection for the tensor-core score GEMM:
//   B0T[s, c*K + k] = sum_m wPCA[k, m] * X[c, s + m - nt/2]
// rows = samples (the GEMM's M), columns = (channel, component) (its K), row
// stride ldk (a multiple of the GEMM's k-block; pad columns stay zero). The
// BF16 path stores bf16; the FP32 path stores the tf32 split hi = rna(x),
// lo = x - hi (exact in fp32) in two fp32 arrays. CTA: 64 samples x PC
// channels, staged in shared memory and written as contiguous row segments.
// ---------------------------------------------------------------------------
constexpr int PT_S = 64;    // samples per CTA

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Thread = (channel, 8-sample group) with the channel fastest across a warp,
// so the K values a thread writes per sample land next to its neighbours'
// and a warp writes 32*K contiguous outputs per sample row.
template <int KPC, int PC, bool TF32, int NTP>
__global__ void __launch_bounds__(256) k_pca_proj_t(const float* __restrict__ X, int64_t ldx, int32_t C, int64_t N,
                                                    const float* __restrict__ wpca, int32_t nt, void* __restrict__ out0,
                                                    float* __restrict__ out_lo, int64_t ldk,
                                                    const int32_t* __restrict__ tiles, const int32_t* __restrict__ ntiles) {
    extern __shared__ float sm[];
    // tiles != null: CTA x projects sample tile tiles[x] into output rows x*PT_S.. (the first *ntiles entries)
    if (tiles && (int)blockIdx.x >= *ntiles) return;
    const int64_t s0 = tiles ? (int64_t)tiles[blockIdx.x] * PT_S : (int64_t)blockIdx.x * PT_S;
    const int64_t o0 = (int64_t)blockIdx.x * PT_S;
    const int ntp = NTP ? NTP : (nt + 7) & ~7;     // taps padded to 8 (zero weights)
    const int xw = PT_S + ntp + 9;                 // staged samples per channel row (odd: no bank conflicts)
    float* ws = sm;                                // [KPC][ntp]
    float* xs = ws + KPC * ntp;                    // [PC][xw]
    float* stage = xs + PC * xw + ((PC * xw) & 3 ? 4 - ((PC * xw) & 3) : 0);  // [PT_S][PC*KPC], 16-byte aligned
    const int c0 = blockIdx.y * PC;
    const int nc = min(PC, C - c0);
    const int half = nt / 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for (int k = warp; k < KPC; k += nwarps)
        for (int m = lane; m < ntp; m += 32) ws[k * ntp + m] = (m < nt) ? wpca[k * nt + m] : 0.f;
    for (int c = warp; c < PC; c += nwarps) {
        const float* xrow = X + (int64_t)(c0 + c) * ldx;
        for (int p = lane; p < xw; p += 32) {
            const int64_t g = s0 - half + p;
            xs[c * xw + p] = (c < nc && g >= 0 && g < N) ? xrow[g] : 0.f;
        }
    }
    __syncthreads();
    for (int task = threadIdx.x; task < PC * (PT_S / 8); task += blockDim.x) {
        const int c = task % PC, sg = task / PC;
        if (c >= nc) continue;
        const float* xr = xs + c * xw + sg * 8;
        float acc[KPC][8];
#pragma unroll
        for (int k = 0; k < KPC; ++k)
#pragma unroll
            for (int r = 0; r < 8; ++r) acc[k][r] = 0.f;
        float w[16];
#pragma unroll
        for (int r = 0; r < 8; ++r) w[r] = xr[r];
        // every accumulator sums its taps in ascending order (one fmaf each)
#pragma unroll(NTP ? NTP / 8 : 1)
        for (int mb = 0; mb < ntp; mb += 8) {
#pragma unroll
            for (int r = 0; r < 8; ++r) w[8 + r] = xr[mb + 8 + r];
#pragma unroll
            for (int k = 0; k < KPC; ++k) {
                const float4 wa = *reinterpret_cast<const float4*>(ws + k * ntp + mb);
                const float4 wb = *reinterpret_cast<const float4*>(ws + k * ntp + mb + 4);
                const float tk[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
#pragma unroll
                for (int u = 0; u < 8; ++u)
#pragma unroll
                    for (int r = 0; r < 8; ++r) acc[k][r] = fmaf(tk[u], w[r + u], acc[k][r]);
            }
#pragma unroll
            for (int r = 0; r < 8; ++r) w[r] = w[8 + r];
        }
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
            for (int k = 0; k < KPC; ++k) stage[(sg * 8 + r) * (PC * KPC) + c * KPC + k] = acc[k][r];
    }
    __syncthreads();
    // rows of nc*KPC outputs, written as 16-byte vectors (ldk and c0*KPC are
    // multiples of 4, so every vector is aligned); one warp per sample row
    const int seg = nc * KPC;
    const int nv4 = seg / 4;
    for (int r = warp; r < PT_S; r += nwarps) {
        const int64_t s = s0 + r;
        if (s >= N) continue;
        const int64_t orow = (o0 + r) * ldk + (int64_t)c0 * KPC;
        const float* srow = stage + r * (PC * KPC);
        for (int q = lane; q < nv4; q += 32) {
            const float4 v = *reinterpret_cast<const float4*>(srow + 4 * q);
            const int64_t o = orow + 4 * q;
            if (TF32) {
                const float4 hi = make_float4(tf32_rna(v.x), tf32_rna(v.y), tf32_rna(v.z), tf32_rna(v.w));
                const float4 lo = make_float4(__fsub_rn(v.x, hi.x), __fsub_rn(v.y, hi.y), __fsub_rn(v.z, hi.z),
                                              __fsub_rn(v.w, hi.w));
                *reinterpret_cast<float4*>(static_cast<float*>(out0) + o) = hi;
                *reinterpret_cast<float4*>(out_lo + o) = lo;
            } else {
                __nv_bfloat16* d = static_cast<__nv_bfloat16*>(out0) + o;
                d[0] = __float2bfloat16_rn(v.x);
                d[1] = __float2bfloat16_rn(v.y);
                d[2] = __float2bfloat16_rn(v.z);
                d[3] = __float2bfloat16_rn(v.w);
            }
        }
        // tail (seg not a multiple of 4)
        for (int j = 4 * nv4 + lane; j < seg; j += 32) {
            const float v = srow[j];
            if (TF32) {
                const float hi = tf32_rna(v);
                static_cast<float*>(out0)[orow + j] = hi;
                out_lo[orow + j] = __fsub_rn(v, hi);
            } else {
                static_cast<__nv_bfloat16*>(out0)[orow + j] = __float2bfloat16_rn(v);
            }
        }
    }
}

template <int KPC, bool TF32>
static cudaError_t launch_pjt(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t nt,
                              void* out0, float* out_lo, int64_t ldk, const int32_t* tiles, const int32_t* ntiles,
                              cudaStream_t s) {
    constexpr int PC = 32;
    const int ntp = (nt + 7) & ~7;
    const size_t smem = sizeof(float) * ((size_t)KPC * ntp + (size_t)PC * (PT_S + ntp + 9) + 4 + (size_t)PT_S * PC * KPC);
    dim3 grid((unsigned)((N + PT_S - 1) / PT_S), (unsigned)((C + PC - 1) / PC));
    if (ntp == 64) {  // nt = 57..64 (Kilosort's 61): taps fully unrolled
        auto kern = k_pca_proj_t<KPC, PC, TF32, 64>;
        if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, 256, smem, s>>>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles);
    } else {
        auto kern = k_pca_proj_t<KPC, PC, TF32, 0>;
        if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, 256, smem, s>>>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles);
    }
    return cudaGetLastError();
}

template <bool TF32>
static cudaError_t pjt_dispatch(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t K,
                                int32_t nt, void* out0, float* out_lo, int64_t ldk, const int32_t* tiles,
                                const int32_t* ntiles, cudaStream_t s) {
    switch (K) {
        case 1: return launch_pjt<1, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, s);
        case 2: return launch_pjt<2, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, s);
        case 3: return launch_pjt<3, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, s);
        case 4: return launch_pjt<4, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, s);
        case 5: return launch_pjt<5, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, s);
        case 6: return launch_pjt<6, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, s);
        case 7: return launch_pjt<7, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, s);
        case 8: return launch_pjt<8, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_pca_proj_t(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t K,
                              int32_t nt, __nv_bfloat16* B0T, int64_t ldk, cudaStream_t s) {
    return pjt_dispatch<false>(X, ldx, C, N, wpca, K, nt, B0T, nullptr, ldk, nullptr, nullptr, s);
}

cudaError_t launch_pca_proj_t_tf32(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t K,
                                   int32_t nt, float* hi, float* lo, int64_t ldk, cudaStream_t s) {
    return pjt_dispatch<true>(X, ldx, C, N, wpca, K, nt, hi, lo, ldk, nullptr, nullptr, s);
}

cudaError_t launch_pca_proj_tiles_tf32(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t K,
                                       int32_t nt, const int32_t* tiles, const int32_t* ntiles, float* hi, float* lo,
                                       int64_t ldk, cudaStream_t s) {
    return pjt_dispatch<true>(X, ldx, C, N, wpca, K, nt, hi, lo, ldk, tiles, ntiles, s);
}

// Templates with the whitening folded in, in the score GEMM's layout:
//   U_w[t, c'*K + k] = sum_c U[t, k, c] * Mw[c, c']       (Mw = M @ Wrot)
// so that sum_kk U_w[t, kk] * P[s, kk] over the projection P of the
// un-whitened batch equals the score of the whitened batch. Stored as bf16
// (BF16 path) or as a tf32 hi/lo split (FP32 path), rows [Tpad, ldk]. The
// product is the 64x64-tile FP32 GEMM with a store into that layout; every
// output sums over c in order.
cudaError_t launch_build_uw(const float* U, const float* Mw, int32_t T, int32_t K, int32_t C, int64_t ldk,
                            __nv_bfloat16* out16, float* hi, float* lo, cudaStream_t s) {
    return launch_sgemm_folded(U, Mw, T, K, C, ldk, out16, hi, lo, s);
}


// ---------------------------------------------------------------------------
// FP32 re-check of the BF16 path's near decisions (first round).
//
// A column s needs its FP32 score when its BF16 maximum Cf could be above the
// threshold (best >= Th^2 (1 - m)) and a decision taken on it lies within the
// relative margin m = 1/16:
//   * the threshold itself: |best - Th^2| <= m Th^2;
//   * the runner-up template: second >= best (1 - m);
//   * the peak test: best is within m of the window maximum and another column
//     of the window is within m of best.
// (BF16 rounding of both GEMM operands moves Cf by about 1% at the scores
// spikes have, so m is several times the error.) Selection works on 64-sample
// tiles (the projection's CTA width): a tile holding any such column is listed,
// projected in FP32 by the FP32 path's own projection kernel, split into tf32
// hi/lo and re-scored by the 3xTF32 GEMM through the tile list, which
// overwrites the tile's scores and column maxima with the FP32 path's values.
// Counts stay on the device: count[0] = listed tiles, count[1] = flips,
// count[2] = near-decision columns.
// ---------------------------------------------------------------------------
constexpr float RECHECK_MARGIN = 1.f / 16.f;
constexpr int RS_TILE = 256;
static_assert(RECHECK_TILE == PT_S, "re-check tiles are projection CTA tiles");
static_assert(RS_TILE % RECHECK_TILE == 0, "selection CTAs cover whole re-check tiles");

__global__ void __launch_bounds__(RS_TILE) k_recheck_select(const float* __restrict__ cfmax, const float* __restrict__ cf2,
                                                            const int32_t* __restrict__ imax, int32_t N, int32_t nt,
                                                            float th2, int32_t* __restrict__ tiles,
                                                            float* __restrict__ pre_cf, int32_t* __restrict__ pre_im,
                                                            int32_t* __restrict__ count) {
    constexpr int NTL = RS_TILE / RECHECK_TILE;
    __shared__ float v[RS_TILE + 2 * 256];
    __shared__ int flag[NTL], slot[NTL];
    const int s0 = blockIdx.x * RS_TILE;
    for (int p = threadIdx.x; p < RS_TILE + 2 * nt; p += blockDim.x) {
        const int s = s0 - nt + p;
        v[p] = (s >= 0 && s < N) ? cfmax[s] : -1.f;
    }
    if (threadIdx.x < NTL) flag[threadIdx.x] = 0;
    __syncthreads();
    const int s = s0 + threadIdx.x;
    const float best = v[threadIdx.x + nt];
    bool sel = false;
    if (s < N) {
        const float m = RECHECK_MARGIN;
        if (best >= th2 * (1.f - m)) {
            float wmax = best, other = -1.f;
            for (int d = -nt; d <= nt; ++d) {
                if (d == 0) continue;
                const float u = v[threadIdx.x + nt + d];
                wmax = fmaxf(wmax, u);
                other = fmaxf(other, u);
            }
            const bool near_thr = fabsf(best - th2) <= m * th2;
            const bool near_tmpl = cf2[s] >= best * (1.f - m);
            const bool near_peak = best >= wmax * (1.f - m) && other >= best * (1.f - m);
            sel = near_thr || near_tmpl || near_peak;
        }
    }
    const unsigned bal = __ballot_sync(0xffffffffu, sel);
    if (bal) {
        if ((threadIdx.x & 31) == 0) atomicAdd(count + 2, __popc(bal));
        flag[threadIdx.x / RECHECK_TILE] = 1;
    }
    __syncthreads();
    if (threadIdx.x < NTL) {
        int sl = -1;
        if (flag[threadIdx.x]) {
            sl = atomicAdd(count, 1);
            tiles[sl] = s0 / RECHECK_TILE + threadIdx.x;
        }
        slot[threadIdx.x] = sl;
    }
    __syncthreads();
    const int sl = slot[threadIdx.x / RECHECK_TILE];
    if (sl >= 0) {
        const int64_t r = (int64_t)sl * RECHECK_TILE + threadIdx.x % RECHECK_TILE;
        pre_cf[r] = (s < N) ? best : 0.f;
        pre_im[r] = (s < N) ? imax[s] : 0;
    }
}

cudaError_t launch_recheck_select(const float* cfmax, const float* cf2, const int32_t* imax, int32_t N, int32_t nt,
                                  float th2, int32_t* tiles, float* pre_cf, int32_t* pre_im, int32_t* count,
                                  cudaStream_t s) {
    if (nt > 256) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(count, 0, 4 * sizeof(int32_t), s);
    if (e != cudaSuccess) return e;
    k_recheck_select<<<(N + RS_TILE - 1) / RS_TILE, RS_TILE, 0, s>>>(cfmax, cf2, imax, N, nt, th2, tiles, pre_cf,
                                                                    pre_im, count);
    return cudaGetLastError();
}

// Decisions the FP32 re-check changed: the best template, or the side of the
// threshold the column maximum falls on.
__global__ void k_recheck_flips(const float* __restrict__ cfmax, const int32_t* __restrict__ imax,
                                const int32_t* __restrict__ tiles, const float* __restrict__ pre_cf,
                                const int32_t* __restrict__ pre_im, const int32_t* __restrict__ count, int32_t N,
                                float th2, int32_t* flips) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= count[0] * RECHECK_TILE) return;
    const int s = tiles[r / RECHECK_TILE] * RECHECK_TILE + r % RECHECK_TILE;
    if (s >= N) return;
    if (imax[s] != pre_im[r] || ((cfmax[s] > th2) != (pre_cf[r] > th2))) atomicAdd(flips, 1);
}

cudaError_t launch_recheck_flips(const float* cfmax, const int32_t* imax, const int32_t* tiles, const float* pre_cf,
                                 const int32_t* pre_im, int32_t* count, int32_t N, float th2, cudaStream_t s) {
    const int rows = (N + RECHECK_TILE - 1) / RECHECK_TILE * RECHECK_TILE;
    k_recheck_flips<<<(rows + 255) / 256, 256, 0, s>>>(cfmax, imax, tiles, pre_cf, pre_im, count, N, th2, count + 1);
    return cudaGetLastError();
}

}  // namespace lss
