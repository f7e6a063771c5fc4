// Temporal-basis projection of the filtered batch:
//   B0[c*K + k, s] = sum_m wPCA[k, m] * X[c, s + m - nt/2]   (zero outside [0, N))
// which is conv1d(X.unsqueeze(1), W.unsqueeze(1), padding=nt//2) of
// kilosort/template_matching.py:145 (conv1d kernel, myGPUhelpers.cu:355-399).
// The row order (c, k) lets the score GEMM contract over c*K + k with the
// template matrix permuted once at set-up to U_p[t, c*K + k] = U[t, k, c].
#include "lss_kernels.cuh"

#include <cuda_bf16.h>

#include <algorithm>

namespace lss {

// ---------------------------------------------------------------------------
// Transposed projection for the tensor-core score GEMM:
//   B0T[s, c*K + k] = sum_m wPCA[k, m] * X[c, s + m - nt/2]
// rows = samples (the GEMM's M), columns = (channel, component) (its K), row
// stride ldk (a multiple of the GEMM's k-block; pad columns stay zero). The
// BF16 path stores bf16; the FP32 path stores the tf32 split hi = rna(x),
// lo = rna(x - hi) in two fp32 arrays: both parts exact tf32 values, so the
// tensor core's tf32 reading of them drops nothing and the split errs by at
// most 2^-23 |x|, unbiased (a plain x - hi would be truncated by the MMA,
// always toward zero). CTA: 64 samples x PC
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
__global__ void __launch_bounds__(256, KPC <= 6 ? 3 : 2) k_pca_proj_t(const float* __restrict__ X, int64_t ldx, int32_t C, int64_t N,
                                                    const float* __restrict__ wpca, int32_t nt, void* __restrict__ out0,
                                                    void* __restrict__ out_lo, int64_t ldk,
                                                    const int32_t* __restrict__ tiles, const int32_t* __restrict__ ntiles,
                                                    float* __restrict__ norm2) {
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
    if constexpr (NTP > 0 && PC % 8 == 0) {
        // fixed tap count: a warp's channel rows loaded into registers first, so
        // that all of them are in flight at once, then stored (256 threads)
        constexpr int XW = PT_S + NTP + 9, NP = (XW + 31) / 32, NCW = PC / 8;
        float v[NCW][NP];
#pragma unroll
        for (int i = 0; i < NCW; ++i) {
            const int c = warp + 8 * i;
            const float* xrow = X + (int64_t)(c0 + c) * ldx;
#pragma unroll
            for (int j = 0; j < NP; ++j) {
                const int pp = lane + 32 * j;
                const int64_t g = s0 - half + pp;
                v[i][j] = (pp < XW && c < nc && g >= 0 && g < N) ? xrow[g] : 0.f;
            }
        }
#pragma unroll
        for (int i = 0; i < NCW; ++i)
#pragma unroll
            for (int j = 0; j < NP; ++j) {
                const int pp = lane + 32 * j;
                if (pp < XW) xs[(warp + 8 * i) * XW + pp] = v[i][j];
            }
    } else {
        for (int c = warp; c < PC; c += nwarps) {
            const float* xrow = X + (int64_t)(c0 + c) * ldx;
            for (int p = lane; p < xw; p += 32) {
                const int64_t g = s0 - half + p;
                xs[c * xw + p] = (c < nc && g >= 0 && g < N) ? xrow[g] : 0.f;
            }
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
                const float4 lo = make_float4(tf32_rna(__fsub_rn(v.x, hi.x)), tf32_rna(__fsub_rn(v.y, hi.y)),
                                              tf32_rna(__fsub_rn(v.z, hi.z)), tf32_rna(__fsub_rn(v.w, hi.w)));
                *reinterpret_cast<float4*>(static_cast<float*>(out0) + o) = hi;
                *reinterpret_cast<float4*>(static_cast<float*>(out_lo) + o) = lo;
            } else {
                // bf16 split: hi = bf16(x), lo = bf16(x - hi), 4 values per 8-byte store
                const float vv[4] = {v.x, v.y, v.z, v.w};
                __align__(8) __nv_bfloat16 hb[4], lb[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    hb[u] = __float2bfloat16_rn(vv[u]);
                    lb[u] = __float2bfloat16_rn(__fsub_rn(vv[u], __bfloat162float(hb[u])));
                }
                *reinterpret_cast<uint2*>(static_cast<__nv_bfloat16*>(out0) + o) = *reinterpret_cast<const uint2*>(hb);
                if (out_lo)
                    *reinterpret_cast<uint2*>(static_cast<__nv_bfloat16*>(out_lo) + o) = *reinterpret_cast<const uint2*>(lb);
            }
        }
        // tail (seg not a multiple of 4)
        for (int j = 4 * nv4 + lane; j < seg; j += 32) {
            const float v = srow[j];
            if (TF32) {
                const float hi = tf32_rna(v);
                static_cast<float*>(out0)[orow + j] = hi;
                static_cast<float*>(out_lo)[orow + j] = tf32_rna(__fsub_rn(v, hi));
            } else {
                const __nv_bfloat16 h = __float2bfloat16_rn(v);
                static_cast<__nv_bfloat16*>(out0)[orow + j] = h;
                if (out_lo)
                    static_cast<__nv_bfloat16*>(out_lo)[orow + j] = __float2bfloat16_rn(__fsub_rn(v, __bfloat162float(h)));
            }
        }
        if (norm2) {
            // this channel group's share of ||P[s, :]||^2 (the FP32 values, before rounding)
            float q = 0.f;
            for (int j = lane; j < seg; j += 32) q = fmaf(srow[j], srow[j], q);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
            if (lane == 0) atomicAdd(norm2 + s, q);
        }
    }
}

template <int KPC, bool TF32>
static cudaError_t launch_pjt(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t nt,
                              void* out0, void* out_lo, int64_t ldk, const int32_t* tiles, const int32_t* ntiles,
                              float* norm2, cudaStream_t s) {
    constexpr int PC = 32;
    const int ntp = (nt + 7) & ~7;
    const size_t smem = sizeof(float) * ((size_t)KPC * ntp + (size_t)PC * (PT_S + ntp + 9) + 4 + (size_t)PT_S * PC * KPC);
    dim3 grid((unsigned)((N + PT_S - 1) / PT_S), (unsigned)((C + PC - 1) / PC));
    if (ntp == 64) {  // nt = 57..64 (Kilosort's 61): taps fully unrolled
        auto kern = k_pca_proj_t<KPC, PC, TF32, 64>;
        if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, 256, smem, s>>>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, norm2);
    } else {
        auto kern = k_pca_proj_t<KPC, PC, TF32, 0>;
        if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, 256, smem, s>>>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, norm2);
    }
    return cudaGetLastError();
}

template <bool TF32>
static cudaError_t pjt_dispatch(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t K,
                                int32_t nt, void* out0, void* out_lo, int64_t ldk, const int32_t* tiles,
                                const int32_t* ntiles, float* norm2, cudaStream_t s) {
    if (norm2) {
        const cudaError_t e = cudaMemsetAsync(norm2, 0, sizeof(float) * N, s);
        if (e != cudaSuccess) return e;
    }
    switch (K) {
        case 1: return launch_pjt<1, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, norm2, s);
        case 2: return launch_pjt<2, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, norm2, s);
        case 3: return launch_pjt<3, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, norm2, s);
        case 4: return launch_pjt<4, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, norm2, s);
        case 5: return launch_pjt<5, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, norm2, s);
        case 6: return launch_pjt<6, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, norm2, s);
        case 7: return launch_pjt<7, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, norm2, s);
        case 8: return launch_pjt<8, TF32>(X, ldx, C, N, wpca, nt, out0, out_lo, ldk, tiles, ntiles, norm2, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_pca_proj_t(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t K,
                              int32_t nt, __nv_bfloat16* B0T_hi, __nv_bfloat16* B0T_lo, int64_t ldk, cudaStream_t s,
                              float* norm2) {
    return pjt_dispatch<false>(X, ldx, C, N, wpca, K, nt, B0T_hi, B0T_lo, ldk, nullptr, nullptr, norm2, s);
}

cudaError_t launch_pca_proj_t_tf32(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t K,
                                   int32_t nt, float* hi, float* lo, int64_t ldk, cudaStream_t s) {
    return pjt_dispatch<true>(X, ldx, C, N, wpca, K, nt, hi, lo, ldk, nullptr, nullptr, nullptr, s);
}


// Templates with the whitening folded in, in the score GEMM's layout:
//   U_w[t, c'*K + k] = sum_c U[t, k, c] * Mw[c, c']       (Mw = M @ Wrot)
// so that sum_kk U_w[t, kk] * P[s, kk] over the projection P of the
// un-whitened batch equals the score of the whitened batch. Stored as bf16
// (BF16 path) or as a tf32 hi/lo split (FP32 path), rows [Tpad, ldk]. The
// product is the 64x64-tile FP32 GEMM with a store into that layout; every
// output sums over c in order.
cudaError_t launch_build_uw(const float* U, const float* Mw, int32_t T, int32_t K, int32_t C, int64_t ldk,
                            __nv_bfloat16* out16, __nv_bfloat16* out16lo, float* hi, float* lo, cudaStream_t s) {
    return launch_sgemm_folded(U, Mw, T, K, C, ldk, out16, out16lo, hi, lo, s);
}


// ---------------------------------------------------------------------------
// FP32 re-check of the BF16 path (first round), column by column.
//
// Every BF16 score is within dB = 2^-7 ||U_t|| ||P_s|| of the FP32 path's
// (bf16 rounding of both operands moves each product by at most 2^-8 of its
// magnitude, sum |U||P| <= ||U|| ||P||, and both paths accumulate in FP32 with
// errors far below that). From it the BF16 GEMM's epilogue gives each column
// an interval [lo, hi] that holds its column maximum of Cf in both paths (the
// BF16 best template's), and ch, the largest upper bound of Cf over the other
// templates. With W(x) the +-nt window of column x (without x):
//   * x can be a peak in either path only if it is a candidate:
//       hi(x) > Th^2 and no v in W(x) has lo(v) > hi(x);
//   * a candidate's decisions are open when lo(x) <= Th^2 (threshold),
//     ch(x) >= lo(x) (best template) or some v in W(x) has hi(v) >= lo(x)
//     (window maximum);
//   * listed: every candidate with an open decision, and every column v whose
//     hi(v) reaches lo(x) of a candidate x with an open window maximum.
// Listed columns are projected with the FP32 path's arithmetic and re-scored
// by its 3xTF32 GEMM through the list, which overwrites their scores with the
// FP32 path's values. Every first-round decision then equals the FP32 path's:
// an unlisted non-candidate is beaten by a neighbour, an unlisted candidate
// strictly beats its window and the threshold with a strictly best template,
// in both paths, and every open comparison involves FP32 values only. Edge
// columns are exactly zero in both paths and never listed. count[0] = listed
// columns, count[1] = decisions the re-check changed, count[2] = listed.
// ---------------------------------------------------------------------------
constexpr int RS_COLS = 256;
constexpr int RS_MAX_NT = 128;

__global__ void __launch_bounds__(RS_COLS) k_recheck_select(const float* __restrict__ cf_lo,
                                                            const float* __restrict__ cf_hi,
                                                            const float* __restrict__ ch,
                                                            const float* __restrict__ cfmax,
                                                            const int32_t* __restrict__ imax, int32_t N, int32_t nt,
                                                            float th2, int32_t* __restrict__ cols,
                                                            float* __restrict__ pre_cf, int32_t* __restrict__ pre_im,
                                                            int32_t* __restrict__ count) {
    // columns s0 - 2nt .. s0 + RS_COLS + 2nt (p = s - s0 + 2nt)
    __shared__ float lo_s[RS_COLS + 4 * RS_MAX_NT], hi_s[RS_COLS + 4 * RS_MAX_NT];
    __shared__ unsigned char openmax[RS_COLS + 2 * RS_MAX_NT];  // p - nt: candidate with an open window maximum
    const int s0 = blockIdx.x * RS_COLS;
    const int span = RS_COLS + 4 * nt;
    for (int p = threadIdx.x; p < span; p += blockDim.x) {
        const int s = s0 - 2 * nt + p;
        const bool in = s >= nt && s < N - nt;  // edge and outside columns: exactly zero
        lo_s[p] = in ? cf_lo[s] : 0.f;
        hi_s[p] = in ? cf_hi[s] : 0.f;
    }
    __syncthreads();
    // candidates and their open window maxima for columns s0 - nt .. s0 + RS_COLS + nt
    for (int p = nt + threadIdx.x; p < RS_COLS + 3 * nt; p += blockDim.x) {
        const float lo = lo_s[p], hi = hi_s[p];
        float wlo = 0.f, whi = 0.f;
        for (int d = 1; d <= nt; ++d) {
            wlo = fmaxf(wlo, fmaxf(lo_s[p - d], lo_s[p + d]));
            whi = fmaxf(whi, fmaxf(hi_s[p - d], hi_s[p + d]));
        }
        const bool cand = hi > th2 && !(wlo > hi);
        openmax[p - nt] = cand && whi >= lo;
    }
    __syncthreads();
    const int s = s0 + threadIdx.x;
    bool sel = false;
    if (s >= nt && s < N - nt) {
        const int p = threadIdx.x + 2 * nt;
        const float lo = lo_s[p], hi = hi_s[p];
        float wlo = 0.f;
        for (int d = 1; d <= nt; ++d) wlo = fmaxf(wlo, fmaxf(lo_s[p - d], lo_s[p + d]));
        const bool cand = hi > th2 && !(wlo > hi);
        sel = cand && (lo <= th2 || ch[s] >= lo || openmax[p - nt]);
        for (int d = -nt; d <= nt && !sel; ++d)
            if (d != 0 && openmax[p + d - nt] && hi >= lo_s[p + d]) sel = true;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, sel);
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == 0 && bal) {
        base = atomicAdd(count, __popc(bal));
        atomicAdd(count + 2, __popc(bal));
    }
    base = __shfl_sync(0xffffffffu, base, 0);
    if (sel) {
        const int i = base + __popc(bal & ((1u << lane) - 1u));
        cols[i] = s;
        pre_cf[i] = cfmax[s];
        pre_im[i] = imax[s];
    }
}

cudaError_t launch_recheck_select(const float* cf_lo, const float* cf_hi, const float* ch, const float* cfmax,
                                  const int32_t* imax, int32_t N, int32_t nt, float th2, int32_t* cols, float* pre_cf,
                                  int32_t* pre_im, int32_t* count, cudaStream_t s) {
    if (nt > RS_MAX_NT) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(count, 0, 4 * sizeof(int32_t), s);
    if (e != cudaSuccess) return e;
    k_recheck_select<<<(N + RS_COLS - 1) / RS_COLS, RS_COLS, 0, s>>>(cf_lo, cf_hi, ch, cfmax, imax, N, nt, th2, cols,
                                                                    pre_cf, pre_im, count);
    return cudaGetLastError();
}

// FP32 projection of the listed columns (tf32 split), with k_pca_proj_t's
// arithmetic: every output sums its (zero-padded) taps in ascending order with
// one fmaf each, so the rows equal the FP32 path's. Column cols[i] goes to row
// i (scatter = 0) or to row cols[i] (scatter = 1: a batch-sized array). A CTA
// takes a (column, chunk of PCOL_CH channels) at a time and stages the chunk's
// window of PCOL_CH channels x ntp samples in shared memory (coalesced loads,
// 8 per thread in flight) before the dot products.
constexpr int PCOL_CH = 64;
template <int KPC>
__global__ void __launch_bounds__(256) k_pca_proj_cols(const float* __restrict__ X, int64_t ldx, int32_t C, int64_t N,
                                                       const float* __restrict__ wpca, int32_t nt, int32_t ntp,
                                                       const int32_t* __restrict__ cols,
                                                       const int32_t* __restrict__ count, float* __restrict__ hi,
                                                       float* __restrict__ lo, int64_t ldk, int32_t scatter) {
    extern __shared__ float sm[];
    const int xw = ntp + 1;           // odd row strides: no bank conflicts across k or c
    float* ws = sm;                   // [KPC][ntp + 1]
    float* xs = sm + KPC * xw;        // [PCOL_CH][ntp + 1]
    for (int e = threadIdx.x; e < KPC * ntp; e += blockDim.x) {
        const int k = e / ntp, m = e % ntp;
        ws[k * xw + m] = (m < nt) ? wpca[k * nt + m] : 0.f;
    }
    const int n = *count;
    const int half = nt / 2;
    const int nchunk = (C + PCOL_CH - 1) / PCOL_CH;
    // one work item per (listed column, chunk of PCOL_CH channels)
    for (int it = blockIdx.x; it < n * nchunk; it += gridDim.x) {
        const int i = it / nchunk, c0 = (it - i * nchunk) * PCOL_CH;
        const int64_t s = cols[i];
        const int64_t row = scatter ? s : (int64_t)i;
        {
            const int nc = min(PCOL_CH, C - c0);
            __syncthreads();
            // staged 8 elements per thread at a time (loads before stores)
            for (int e0 = threadIdx.x; e0 < nc * ntp; e0 += 8 * (int)blockDim.x) {
                float v[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int e = e0 + u * (int)blockDim.x;
                    const int c = e / ntp, m = e % ntp;
                    const int64_t g = s - half + m;
                    v[u] = (e < nc * ntp && g >= 0 && g < N) ? X[(int64_t)(c0 + c) * ldx + g] : 0.f;
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int e = e0 + u * (int)blockDim.x;
                    if (e < nc * ntp) xs[(e / ntp) * xw + e % ntp] = v[u];
                }
            }
            __syncthreads();
            for (int e = threadIdx.x; e < nc * KPC; e += blockDim.x) {
                const int c = e / KPC, k = e % KPC;
                const float* xr = xs + c * xw;
                const float* wk = ws + k * xw;
                float acc = 0.f;
                for (int m = 0; m < ntp; ++m) acc = fmaf(wk[m], xr[m], acc);
                const int64_t o = row * ldk + (int64_t)(c0 + c) * KPC + k;
                const float h = tf32_rna(acc);
                hi[o] = h;
                lo[o] = tf32_rna(__fsub_rn(acc, h));
            }
        }
    }
}

template <int KPC>
static cudaError_t launch_cols(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t nt,
                               const int32_t* cols, const int32_t* count, int32_t max_cols, float* hi, float* lo,
                               int64_t ldk, int32_t scatter, cudaStream_t s) {
    const int ntp = (nt + 7) & ~7;
    const size_t smem = sizeof(float) * ((size_t)KPC * (ntp + 1) + (size_t)PCOL_CH * (ntp + 1));
    if (smem > 48 * 1024) return cudaErrorInvalidValue;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)max_cols * ((C + PCOL_CH - 1) / PCOL_CH),
                                                                   8 * sms));
    k_pca_proj_cols<KPC><<<grid, 256, smem, s>>>(X, ldx, C, N, wpca, nt, ntp, cols, count, hi, lo, ldk, scatter);
    return cudaGetLastError();
}

cudaError_t launch_pca_proj_cols_tf32(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t K,
                                      int32_t nt, const int32_t* cols, const int32_t* count, int32_t max_cols, float* hi,
                                      float* lo, int64_t ldk, int32_t scatter, cudaStream_t s) {
    switch (K) {
        case 1: return launch_cols<1>(X, ldx, C, N, wpca, nt, cols, count, max_cols, hi, lo, ldk, scatter, s);
        case 2: return launch_cols<2>(X, ldx, C, N, wpca, nt, cols, count, max_cols, hi, lo, ldk, scatter, s);
        case 3: return launch_cols<3>(X, ldx, C, N, wpca, nt, cols, count, max_cols, hi, lo, ldk, scatter, s);
        case 4: return launch_cols<4>(X, ldx, C, N, wpca, nt, cols, count, max_cols, hi, lo, ldk, scatter, s);
        case 5: return launch_cols<5>(X, ldx, C, N, wpca, nt, cols, count, max_cols, hi, lo, ldk, scatter, s);
        case 6: return launch_cols<6>(X, ldx, C, N, wpca, nt, cols, count, max_cols, hi, lo, ldk, scatter, s);
        case 7: return launch_cols<7>(X, ldx, C, N, wpca, nt, cols, count, max_cols, hi, lo, ldk, scatter, s);
        case 8: return launch_cols<8>(X, ldx, C, N, wpca, nt, cols, count, max_cols, hi, lo, ldk, scatter, s);
        default: return cudaErrorInvalidValue;
    }
}

// Decisions the FP32 re-check changed: the best template, or the side of the
// threshold the column maximum falls on.
__global__ void k_recheck_flips(const float* __restrict__ cfmax, const int32_t* __restrict__ imax,
                                const int32_t* __restrict__ cols, const float* __restrict__ pre_cf,
                                const int32_t* __restrict__ pre_im, const int32_t* __restrict__ count, float th2,
                                int32_t* flips) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count[0]) return;
    const int s = cols[i];
    if (imax[s] != pre_im[i] || ((cfmax[s] > th2) != (pre_cf[i] > th2))) atomicAdd(flips, 1);
}

cudaError_t launch_recheck_flips(const float* cfmax, const int32_t* imax, const int32_t* cols, const float* pre_cf,
                                 const int32_t* pre_im, int32_t* count, int32_t N, float th2, cudaStream_t s) {
    k_recheck_flips<<<(N + 255) / 256, 256, 0, s>>>(cfmax, imax, cols, pre_cf, pre_im, count, th2, count + 1);
    return cudaGetLastError();
}

// un[t] = ||hi[t, :] + lo[t, :]|| (rows of the tf32-split template operand,
// summed in double, rounded up): the template norms of the BF16 error bound
__global__ void k_row_norms(const float* __restrict__ hi, const float* __restrict__ lo, int32_t T, int64_t ld,
                            float* __restrict__ un) {
    const int t = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= T) return;
    double q = 0.0;
    for (int64_t e = lane; e < ld; e += 32) {
        const double v = (double)hi[t * ld + e] + (double)lo[t * ld + e];
        q += v * v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
    if (lane == 0) un[t] = __double2float_ru(__dsqrt_ru(q));
}

cudaError_t launch_row_norms(const float* hi, const float* lo, int32_t T, int64_t ld, float* un, cudaStream_t s) {
    k_row_norms<<<(T + 7) / 8, 256, 0, s>>>(hi, lo, T, ld, un);
    return cudaGetLastError();
}

}  // namespace lss
