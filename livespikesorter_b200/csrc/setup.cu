// One-time set-up on the GPU in FP64: hot swap of the templates and drift
// matrices without Python (lss_set_templates, lss_set_drift_model,
// lss_set_drift_shift).
//
// * Template cross-correlations (kilosort/template_matching.py:110-121,
//   prepare_matching):
//     WtW[k, m, l] = sum_q wPCA[k, q + nt - l] wPCA[m, q]   (the flipped
//                    autocorrelation of the basis, l = 0 .. 2nt)
//     UtU[(i,k), (j,m)] = sum_c U[i, k, c] U[j, m, c]
//     ctc[i, j, l] = sum_{k,m} UtU[(i,k), (j,m)] WtW[k, m, l]
//   computed in FP64 and rounded once to FP32 (Kilosort computes it in FP32).
// * Energies nm (template_matching.py:141), the nearest-channel tables iU and
//   Ucc (template_matching.py:20-26, with iCC given), the GEMM's template
//   operands, template waveforms and the basis correlation R are rebuilt from
//   U and wPCA with the same arithmetic lss_create uses, so a swapped-in
//   template set sorts exactly as a handle created with it would.
// * Drift interpolation (kilosort/preprocessing.py:44-69, one block):
//     M = Kyx iKxx,  Kyx[a, b] = exp(-|p_a - dshift e_y - p_b|^2 / (2 sig^2))
//   with iKxx = (Kxx + 0.01 I)^-1 (datashift.py:213-219) computed once on the
//   host in FP64.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "lss.h"
#include "lss_handle.h"
#include "lss_kernels.cuh"

namespace lss {

// nm[t] = double sum, in (k, c) order, of the FP32 squares; iU[t] = first
// channel with the largest sum over k of the FP32 squares (torch.argmax).
__global__ void k_nm_iu(const float* __restrict__ U, int T, int K, int C, float* __restrict__ nm,
                        int64_t* __restrict__ iU) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const float* u = U + (int64_t)t * K * C;
    double acc = 0.0;
    for (int e = 0; e < K * C; ++e) acc += (double)__fmul_rn(u[e], u[e]);
    nm[t] = (float)acc;
    if (iU) {
        float best = -1.f;
        int bi = 0;
        for (int c = 0; c < C; ++c) {
            float s = 0.f;
            for (int k = 0; k < K; ++k) s = __fadd_rn(s, __fmul_rn(u[k * C + c], u[k * C + c]));
            if (s > best) {
                best = s;
                bi = c;
            }
        }
        iU[t] = bi;
    }
}

__global__ void k_ucc(const float* __restrict__ U, const int64_t* __restrict__ iCC, const int64_t* __restrict__ iU,
                      int nC, int T, int K, int C, float* __restrict__ Ucc) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nC * T * K) return;
    const int j = e / (T * K), r = e % (T * K), t = r / K, k = r % K;
    const int64_t ch = iCC[(int64_t)j * C + iU[t]];
    Ucc[e] = U[((int64_t)t * K + k) * C + ch];
}

// GEMM operands U_p[t, c*K + k] = U[t, k, c]: tf32 split hi = rna(x),
// lo = rna(x - hi) (the bit rounding lss_create uses) and the bf16 split
// hi = bf16(x), lo = bf16(x - hi).
__global__ void k_up(const float* __restrict__ U, int T, int K, int C, int64_t ldk, float* __restrict__ hi,
                     float* __restrict__ lo, __nv_bfloat16* __restrict__ b16, __nv_bfloat16* __restrict__ b16lo) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)T * C * K) return;
    const int t = (int)(e / ((int64_t)C * K)), r = (int)(e % ((int64_t)C * K)), c = r / K, k = r % K;
    const float x = U[((int64_t)t * K + k) * C + c];
    uint32_t u = __float_as_uint(x);
    if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
    const float xh = __uint_as_float(u);
    uint32_t v = __float_as_uint(__fsub_rn(x, xh));
    if ((v & 0x7f800000u) != 0x7f800000u) v = (v + 0x1000u) & 0xffffe000u;
    hi[(int64_t)t * ldk + r] = xh;
    lo[(int64_t)t * ldk + r] = __uint_as_float(v);
    if (b16) {
        const __nv_bfloat16 hb = __float2bfloat16_rn(x);
        b16[(int64_t)t * ldk + r] = hb;
        b16lo[(int64_t)t * ldk + r] = __float2bfloat16_rn(__fsub_rn(x, __bfloat162float(hb)));
    }
}

// wave[t, c, m] = sum_k U[t, k, c] wPCA[k, m] (double, k order)
__global__ void k_wave(const float* __restrict__ U, const float* __restrict__ W, int T, int K, int C, int nt,
                       float* __restrict__ wave) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)T * C * nt) return;
    const int t = (int)(e / ((int64_t)C * nt)), r = (int)(e % ((int64_t)C * nt)), c = r / nt, m = r % nt;
    double acc = 0.0;
    for (int k = 0; k < K; ++k) acc += (double)U[((int64_t)t * K + k) * C + c] * (double)W[k * nt + m];
    wave[e] = (float)acc;
}

// R[k, k2, d] = sum_m wPCA[k, m] wPCA[k2, m + d] (double, m order) and
// WtW[k, m, l] = sum_q wPCA[k, q + nt - l] wPCA[m, q] (double)
__global__ void k_basis(const float* __restrict__ W, int K, int nt, float* __restrict__ R, double* __restrict__ WtW) {
    const int nd = 2 * nt - 1, L2 = 2 * nt + 1;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < K * K * nd) {
        const int k = e / (K * nd), r = e % (K * nd), k2 = r / nd, d = r % nd - (nt - 1);
        double acc = 0.0;
        for (int m = 0; m < nt; ++m)
            if (m + d >= 0 && m + d < nt) acc += (double)W[k * nt + m] * (double)W[k2 * nt + m + d];
        R[e] = (float)acc;
    }
    if (e < K * K * L2) {
        const int k = e / (K * L2), r = e % (K * L2), m = r / L2, l = r % L2;
        double acc = 0.0;
        for (int q = 0; q < nt; ++q) {
            const int p = q + nt - l;
            if (p >= 0 && p < nt) acc += (double)W[k * nt + p] * (double)W[m * nt + q];
        }
        WtW[e] = acc;
    }
}

// UtU = A A^T, A = U viewed as [T*K, C] (FP64 accumulate), 64x64 tiles.
constexpr int UT = 64;
__global__ void __launch_bounds__(256) k_utu(const float* __restrict__ A, int M, int C, double* __restrict__ out) {
    __shared__ double sa[16][UT + 1], sb[16][UT + 1];
    const int r0 = blockIdx.y * UT, c0 = blockIdx.x * UT;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    double acc[4][4] = {};
    for (int k0 = 0; k0 < C; k0 += 16) {
        for (int e = threadIdx.x; e < 16 * UT; e += 256) {
            const int kk = e / UT, rr = e % UT;
            sa[kk][rr] = (r0 + rr < M && k0 + kk < C) ? (double)A[(int64_t)(r0 + rr) * C + k0 + kk] : 0.0;
            sb[kk][rr] = (c0 + rr < M && k0 + kk < C) ? (double)A[(int64_t)(c0 + rr) * C + k0 + kk] : 0.0;
        }
        __syncthreads();
        for (int kk = 0; kk < 16; ++kk)
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] = fma(sa[kk][ty * 4 + a], sb[kk][tx * 4 + b], acc[a][b]);
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int r = r0 + ty * 4 + a, c = c0 + tx * 4 + b;
            if (r < M && c < M) out[(int64_t)r * M + c] = acc[a][b];
        }
}

// ctcP[j, i, l] = (float) sum_{k,m} UtU[(i,k),(j,m)] WtW[k,m,l]; CTA = one i,
// eight j, threads over l.
constexpr int CJ = 8;
__global__ void k_ctc(const double* __restrict__ UtU, const double* __restrict__ WtW, int T, int K, int nt,
                      float* __restrict__ ctcP) {
    extern __shared__ double cs[];
    const int L2 = 2 * nt + 1;
    double* w = cs;                    // [K*K][L2]
    double* u = cs + K * K * L2;       // [CJ][K*K]
    const int i = blockIdx.y, j0 = blockIdx.x * CJ;
    const int nj = min(CJ, T - j0);
    const int M = T * K;
    for (int e = threadIdx.x; e < K * K * L2; e += blockDim.x) w[e] = WtW[e];
    for (int e = threadIdx.x; e < nj * K * K; e += blockDim.x) {
        const int q = e / (K * K), r = e % (K * K), k = r / K, m = r % K;
        u[e] = UtU[(int64_t)(i * K + k) * M + (j0 + q) * K + m];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nj * L2; e += blockDim.x) {
        const int q = e / L2, l = e % L2;
        double acc = 0.0;
        for (int km = 0; km < K * K; ++km) acc = fma(u[q * K * K + km], w[km * L2 + l], acc);
        ctcP[((int64_t)(j0 + q) * T + i) * L2 + l] = (float)acc;
    }
}

// M[a, b] = sum_c Kyx[a, c] iKxx[c, b], Kyx from the channel positions (FP64)
__global__ void k_drift(const double* __restrict__ xc, const double* __restrict__ yc, const double* __restrict__ iK,
                        int C, double dshift, double sig, float* __restrict__ M) {
    const int a = blockIdx.y, b = blockIdx.x * blockDim.x + threadIdx.x;
    extern __shared__ double kr[];  // Kyx row a
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        const double dx = xc[a] - xc[c], dy = (yc[a] - dshift) - yc[c];
        kr[c] = exp(-(dx * dx + dy * dy) / (2.0 * sig * sig));
    }
    __syncthreads();
    if (b >= C) return;
    double acc = 0.0;
    for (int c = 0; c < C; ++c) acc = fma(kr[c], iK[(int64_t)c * C + b], acc);
    M[(int64_t)a * C + b] = (float)acc;
}

}  // namespace lss

using namespace lss;

#define SCK(call)                                                                    \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) return h->cuda_fail(e_, #call);                       \
    } while (0)

namespace {

template <typename T>
struct Tmp {
    T* p = nullptr;
    ~Tmp() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t n) { return cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T)); }
};

// (A + 0.01 I)^-1 for a symmetric positive definite A (Cholesky, FP64)
bool spd_inverse(std::vector<double>& A, int n) {
    std::vector<double> L((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j) {
        double d = A[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) d -= L[(size_t)j * n + k] * L[(size_t)j * n + k];
        if (!(d > 0.0)) return false;
        const double ljj = std::sqrt(d);
        L[(size_t)j * n + j] = ljj;
        for (int i = j + 1; i < n; ++i) {
            double s = A[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) s -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
            L[(size_t)i * n + j] = s / ljj;
        }
    }
    // inverse of L (lower), then A^-1 = L^-T L^-1
    std::vector<double> Li((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j) {
        Li[(size_t)j * n + j] = 1.0 / L[(size_t)j * n + j];
        for (int i = j + 1; i < n; ++i) {
            double s = 0.0;
            for (int k = j; k < i; ++k) s -= L[(size_t)i * n + k] * Li[(size_t)k * n + j];
            Li[(size_t)i * n + j] = s / L[(size_t)i * n + i];
        }
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = 0.0;
            for (int k = i; k < n; ++k) s += Li[(size_t)k * n + i] * Li[(size_t)k * n + j];
            A[(size_t)i * n + j] = s;
            A[(size_t)j * n + i] = s;
        }
    return true;
}

}  // namespace

extern "C" {

int lss_set_templates(lss_handle* h, const float* U, const float* wPCA) {
    if (!h || !U) return LSS_ERR_ARG;
    if (h->streaming) return h->fail(LSS_ERR_STATE, "handle is owned by a serving loop");
    SCK(cudaSetDevice(h->cfg.device));
    const int T = h->T, K = h->K, C = h->C, nt = h->nt, nC = h->nC;
    const int L2 = 2 * nt + 1, nd = 2 * nt - 1;
    cudaStream_t s = 0;
    SCK(cudaMemcpy(h->U.p, U, (size_t)T * K * C * sizeof(float), cudaMemcpyHostToDevice));
    if (wPCA) SCK(cudaMemcpy(h->wpca.p, wPCA, (size_t)K * nt * sizeof(float), cudaMemcpyHostToDevice));
    Tmp<double> wtw, utu;
    SCK(wtw.alloc((size_t)K * K * L2));
    SCK(utu.alloc((size_t)T * K * T * K));
    const int nb = std::max(K * K * nd, K * K * L2);
    k_basis<<<(nb + 255) / 256, 256, 0, s>>>(h->wpca.p, K, nt, h->R.p, wtw.p);
    k_nm_iu<<<(T + 127) / 128, 128, 0, s>>>(h->U.p, T, K, C, h->nm.p, nC > 0 ? h->iU.p : nullptr);
    if (nC > 0) k_ucc<<<(nC * T * K + 255) / 256, 256, 0, s>>>(h->U.p, h->iCC.p, h->iU.p, nC, T, K, C, h->Ucc.p);
    const int64_t nup = (int64_t)T * C * K;
    const bool bf16 = h->cfg.precision == LSS_PREC_BF16_RECHECK;
    k_up<<<(unsigned)((nup + 255) / 256), 256, 0, s>>>(h->U.p, T, K, C, h->CKpad, h->Up_hi.p, h->Up_lo.p,
                                                       bf16 ? h->Up16.p : nullptr, bf16 ? h->Up16lo.p : nullptr);
    h->un_p_stale = true;  // the plain templates changed
    const int64_t nw = (int64_t)T * C * nt;
    k_wave<<<(unsigned)((nw + 255) / 256), 256, 0, s>>>(h->U.p, h->wpca.p, T, K, C, nt, h->wave.p);
    const int M = T * K;
    k_utu<<<dim3((M + UT - 1) / UT, (M + UT - 1) / UT), 256, 0, s>>>(h->U.p, M, C, utu.p);
    const size_t smem = sizeof(double) * ((size_t)K * K * L2 + (size_t)CJ * K * K);
    if (smem > 48 * 1024) SCK(cudaFuncSetAttribute(k_ctc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_ctc<<<dim3((T + CJ - 1) / CJ, T), 128, smem, s>>>(utu.p, wtw.p, T, K, nt, h->ctcP.p);
    SCK(cudaGetLastError());
    h->stats.launches += 7 + (nC > 0);
    SCK(cudaStreamSynchronize(s));
    // energies must stay positive for the rounds' division
    std::vector<float> nmv(T);
    SCK(cudaMemcpy(nmv.data(), h->nm.p, T * sizeof(float), cudaMemcpyDeviceToHost));
    for (int i = 0; i < T; ++i)
        if (!(nmv[i] > 0.f) || !std::isfinite(nmv[i]))
            return h->fail(LSS_ERR_ARG, "template " + std::to_string(i) + " has zero or non-finite energy");
    // the rounds' template order and |ctc| maxima, and the whitening-folded
    // operands, follow the new templates
    const int rc = rebuild_mp_blocks(h);
    if (rc) return rc;
    return rebuild_uw(h);
}

int lss_set_drift_model(lss_handle* h, const float* xc, const float* yc, float sig_interp) {
    if (!h || !xc || !yc || !(sig_interp > 0.f)) return LSS_ERR_ARG;
    const int C = h->C;
    std::vector<double> x(C), y(C), A((size_t)C * C);
    for (int c = 0; c < C; ++c) {
        x[c] = xc[c];
        y[c] = yc[c];
    }
    const double s2 = 2.0 * (double)sig_interp * (double)sig_interp;
    for (int a = 0; a < C; ++a)
        for (int b = 0; b < C; ++b) {
            const double dx = x[a] - x[b], dy = y[a] - y[b];
            A[(size_t)a * C + b] = std::exp(-(dx * dx + dy * dy) / s2) + (a == b ? 0.01 : 0.0);
        }
    if (!spd_inverse(A, C)) return h->fail(LSS_ERR_ARG, "channel kernel matrix is not positive definite");
    SCK(cudaSetDevice(h->cfg.device));
    h->dm_pos.release();
    h->dm_ik.release();
    SCK(h->dm_pos.alloc(2 * (size_t)C));
    SCK(h->dm_ik.alloc((size_t)C * C));
    SCK(cudaMemcpy(h->dm_pos.p, x.data(), C * sizeof(double), cudaMemcpyHostToDevice));
    SCK(cudaMemcpy(h->dm_pos.p + C, y.data(), C * sizeof(double), cudaMemcpyHostToDevice));
    SCK(cudaMemcpy(h->dm_ik.p, A.data(), A.size() * sizeof(double), cudaMemcpyHostToDevice));
    h->dm_sig = sig_interp;
    return LSS_OK;
}

int lss_set_drift_shift(lss_handle* h, double dshift) {
    if (!h) return LSS_ERR_ARG;
    if (!h->dm_ik.p) return h->fail(LSS_ERR_STATE, "lss_set_drift_model first");
    SCK(cudaSetDevice(h->cfg.device));
    if (h->streaming) return h->fail(LSS_ERR_STATE, "handle is owned by a serving loop");
    const int C = h->C;
    k_drift<<<dim3((C + 127) / 128, C), 128, C * sizeof(double), 0>>>(h->dm_pos.p, h->dm_pos.p + C, h->dm_ik.p, C,
                                                                    dshift, (double)h->dm_sig, h->Mdrift.p);
    SCK(cudaGetLastError());
    h->stats.launches += 1;
    return mix_device_drift(h);
}

}  // extern "C"
