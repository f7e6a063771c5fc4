// Ingest of one padded batch: int16 rows -> channel mean removal -> median
// common-average reference -> circular highpass.
//
// Semantics follow kilosort/io.py:584-637 (padded_batch_to_torch) and
// io.py:757-777 (BinaryFiltered.filter up to the whitening); the whitening and
// drift GEMM runs in gemm_fp32.cu. LiveSpikeSorter's equivalents are
// meanRemove / median_remove_kernel / highpassFilter
// (myGPUhelpers.cu:98-118,471-534; OnlineSpikesV2.cu:976-1026).
//
// HBM layout: raw int16 [n_rows, ld_raw] (the file's interleaved rows), output
// float [C, ldx] channel-major with time contiguous, so every later stage reads
// 128-byte rows.
#include "lss_kernels.cuh"

namespace lss {

__device__ __forceinline__ int64_t src_row(int64_t s, const IngestMap& m, int64_t base) {
    if (m.base_dev) {
        const int64_t r = base + s;
        return r < 0 ? 0 : r % m.ring_rows;
    }
    int64_t j = s - m.lead;
    if (j < 0) j = 0;
    if (j >= m.nsamp) {
        if (m.zero_tail) return -1;
        j = m.nsamp - 1;
    }
    return j;
}

// Per-channel integer sums over the padded batch (exact: raw samples are
// integers, so the mean is the correctly rounded quotient of an exact sum).
// Grid: one CTA per 256 columns; a warp per column at a time with channels
// lane + 32q in registers (all of a column's loads in flight), per-lane int
// sums combined across the CTA's warps in shared memory, one 64-bit atomic
// per channel and CTA.
template <int NQ>
__global__ void __launch_bounds__(256) k_chan_sums(const int16_t* __restrict__ raw, int32_t ld_raw,
                                                   const int32_t* __restrict__ chan_map, int32_t C, int64_t N,
                                                   IngestMap map, long long* __restrict__ sums) {
    __shared__ int part[8][NQ * 32];
    const int64_t s0 = (int64_t)blockIdx.x * 256;
    const int64_t s1 = min(N, s0 + 256);
    const int64_t base = map.base_dev ? *map.base_dev : 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int acc[NQ];
    int ch[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        const int c = lane + 32 * q;
        acc[q] = 0;
        ch[q] = (c < C) ? (chan_map ? chan_map[c] : c) : 0;
    }
    for (int64_t sc = s0 + warp; sc < s1; sc += 8) {
        const int64_t r = src_row(sc, map, base);
        if (r < 0) continue;
        const int16_t* row = raw + r * ld_raw;
#pragma unroll
        for (int q = 0; q < NQ; ++q)
            if (lane + 32 * q < C) acc[q] += row[ch[q]];
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) part[warp][lane + 32 * q] = acc[q];
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        int t = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) t += part[w][c];
        atomicAdd((unsigned long long*)&sums[c], (unsigned long long)(long long)t);
    }
}

template <int NQ>
static void launch_sums_t(const int16_t* raw, int32_t ld_raw, const int32_t* chan_map, int32_t C, int64_t N,
                          IngestMap map, long long* sums, cudaStream_t s) {
    const int grid = (int)((N + 255) / 256);
    k_chan_sums<NQ><<<grid, 256, 0, s>>>(raw, ld_raw, chan_map, C, N, map, sums);
}

cudaError_t launch_chan_sums(const int16_t* raw, int32_t ld_raw, const int32_t* chan_map, int32_t C,
                             int64_t N, IngestMap map, long long* sums, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(sums, 0, sizeof(long long) * C, s);
    if (e != cudaSuccess) return e;
    const int nq = (C + 31) / 32;
    if (nq <= 2) launch_sums_t<2>(raw, ld_raw, chan_map, C, N, map, sums, s);
    else if (nq <= 4) launch_sums_t<4>(raw, ld_raw, chan_map, C, N, map, sums, s);
    else if (nq <= 8) launch_sums_t<8>(raw, ld_raw, chan_map, C, N, map, sums, s);
    else if (nq <= 12) launch_sums_t<12>(raw, ld_raw, chan_map, C, N, map, sums, s);
    else if (nq <= 16) launch_sums_t<16>(raw, ld_raw, chan_map, C, N, map, sums, s);
    else if (nq <= 24) launch_sums_t<24>(raw, ld_raw, chan_map, C, N, map, sums, s);
    else launch_sums_t<32>(raw, ld_raw, chan_map, C, N, map, sums, s);
    return cudaGetLastError();
}

// Order-preserving float -> uint32 key.
__device__ __forceinline__ uint32_t fkey(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unkey(uint32_t k) {
    uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

// CAR tile: 32 time columns x C channels staged in shared memory. Each warp
// finds the lower median (sorted index (C-1)/2, torch.median's choice) of a
// column by a 32-step bitwise select on order-preserving keys held in
// registers (NQ = keys per lane >= C/32; padding keys are the largest value),
// then the tile is written back as 128-byte channel rows.
constexpr int CAR_COLS = 32;
template <int NQ>
__global__ void __launch_bounds__(256) k_car(const int16_t* __restrict__ raw, int32_t ld_raw,
                                             const int32_t* __restrict__ chan_map, int32_t C,
                                             int64_t N, IngestMap map, float sign,
                                             const long long* __restrict__ sums, int do_car,
                                             float* __restrict__ X1, int64_t ldx) {
    extern __shared__ float sm[];
    float* tile = sm;                                  // [C][CAR_COLS + 1]
    float* mean = sm + (size_t)C * (CAR_COLS + 1);     // [C]
    const int64_t s0 = (int64_t)blockIdx.x * CAR_COLS;
    const int ncol = (int)min((int64_t)CAR_COLS, N - s0);
    const double invN = 1.0 / (double)N;
    const int64_t base = map.base_dev ? *map.base_dev : 0;
    for (int c = threadIdx.x; c < C; c += blockDim.x)
        mean[c] = (float)((double)sign * (double)sums[c] * invN);
    __syncthreads();
    // a warp per time column: its channels lane + 32q in registers (all loads
    // of the column in flight at once), mean removed, the lower median found
    // on the keys, and the referenced values parked in the tile for the
    // channel-major write below
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t kth = (uint32_t)((C - 1) / 2);
    for (int j = warp; j < CAR_COLS; j += blockDim.x >> 5) {
        const int64_t r = (j < ncol) ? src_row(s0 + j, map, base) : -1;
        float v[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const int c = lane + 32 * q;
            const int ch = (c < C) ? (chan_map ? chan_map[c] : c) : 0;
            const float x = (c < C && r >= 0) ? sign * (float)raw[r * ld_raw + ch] : 0.f;
            v[q] = (c < C && j < ncol) ? __fsub_rn(x, mean[c]) : 0.f;
        }
        float mj = 0.f;
        if (do_car && j < ncol) {
            uint32_t key[NQ];
#pragma unroll
            for (int q = 0; q < NQ; ++q) key[q] = (lane + 32 * q < C) ? fkey(v[q]) : 0xFFFFFFFFu;
            uint32_t res = 0;
            for (int b = 31; b >= 0; --b) {
                const uint32_t trial = res | ((1u << b) - 1u);
                uint32_t cnt = 0;
#pragma unroll
                for (int q = 0; q < NQ; ++q) cnt += (key[q] <= trial);
                cnt = __reduce_add_sync(0xffffffffu, cnt);
                if (cnt < kth + 1) res |= (1u << b);
            }
            mj = unkey(res);
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const int c = lane + 32 * q;
            if (c < C) tile[c * (CAR_COLS + 1) + j] = do_car ? __fsub_rn(v[q], mj) : v[q];
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < C * CAR_COLS; idx += blockDim.x) {
        const int j = idx % CAR_COLS, c = idx / CAR_COLS;
        if (j < ncol) {
            X1[(int64_t)c * ldx + s0 + j] = tile[c * (CAR_COLS + 1) + j];
        }
    }
}

template <int NQ>
static cudaError_t launch_car_t(const int16_t* raw, int32_t ld_raw, const int32_t* chan_map, int32_t C, int64_t N,
                                IngestMap map, float sign, const long long* sums, int do_car, float* X1, int64_t ldx,
                                cudaStream_t s) {
    const size_t smem = sizeof(float) * ((size_t)C * (CAR_COLS + 1) + C + CAR_COLS);
    cudaFuncSetAttribute(k_car<NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    const int grid = (int)((N + CAR_COLS - 1) / CAR_COLS);
    k_car<NQ><<<grid, 256, smem, s>>>(raw, ld_raw, chan_map, C, N, map, sign, sums, do_car, X1, ldx);
    return cudaGetLastError();
}

cudaError_t launch_car(const int16_t* raw, int32_t ld_raw, const int32_t* chan_map, int32_t C, int64_t N,
                       IngestMap map, float sign, const long long* sums, int do_car, float* X1,
                       int64_t ldx, cudaStream_t s) {
    const int nq = (C + 31) / 32;
    if (nq <= 2) return launch_car_t<2>(raw, ld_raw, chan_map, C, N, map, sign, sums, do_car, X1, ldx, s);
    if (nq <= 4) return launch_car_t<4>(raw, ld_raw, chan_map, C, N, map, sign, sums, do_car, X1, ldx, s);
    if (nq <= 8) return launch_car_t<8>(raw, ld_raw, chan_map, C, N, map, sign, sums, do_car, X1, ldx, s);
    if (nq <= 12) return launch_car_t<12>(raw, ld_raw, chan_map, C, N, map, sign, sums, do_car, X1, ldx, s);
    if (nq <= 16) return launch_car_t<16>(raw, ld_raw, chan_map, C, N, map, sign, sums, do_car, X1, ldx, s);
    if (nq <= 24) return launch_car_t<24>(raw, ld_raw, chan_map, C, N, map, sign, sums, do_car, X1, ldx, s);
    return launch_car_t<32>(raw, ld_raw, chan_map, C, N, map, sign, sums, do_car, X1, ldx, s);
}

// Circular highpass: Xh[c, i] = sum_{d=-L..L} taps[d+L] * X1[c, (i+d) mod N].
// This equals fftshift(real(ifft(fft(X) * conj(fft(h_N))))) of
// kilosort/preprocessing.py:138-154 + io.py:771-774 with the impulse response
// truncated where its tail mass is below 2^-30 of its L1 norm (the host picks
// L; the tail then contributes less than the FP32 rounding of the transform).
// CTA: one channel, HP_TILE outputs; thread: 8 consecutive outputs with a
// sliding register window over the staged input.
constexpr int HP_TILE = 1024;
constexpr int HP_THREADS = HP_TILE / 8;
__global__ void __launch_bounds__(HP_THREADS) k_highpass(const float* __restrict__ X1, int64_t ldx, int64_t N,
                                                         const float* __restrict__ taps, int32_t L,
                                                         float* __restrict__ Xh) {
    extern __shared__ float sm[];
    const int ntap = 2 * L + 1;
    const int ntap_pad = (ntap + 7) & ~7;
    float* tp = sm;                      // [ntap_pad] (zero padded)
    float* xs = sm + ntap_pad;           // [HP_TILE + ntap_pad + 8]
    const int c = blockIdx.y;
    const int64_t i0 = (int64_t)blockIdx.x * HP_TILE;
    const float* xrow = X1 + (int64_t)c * ldx;
    for (int e = threadIdx.x; e < ntap_pad; e += blockDim.x) tp[e] = (e < ntap) ? taps[e] : 0.f;
    const int nx = HP_TILE + ntap_pad + 8;
    for (int p = threadIdx.x; p < nx; p += blockDim.x) {
        int64_t g = i0 - L + p;
        g %= N;
        if (g < 0) g += N;
        xs[p] = xrow[g];
    }
    __syncthreads();
    float acc[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) acc[r] = 0.f;
    const int o = threadIdx.x * 8;
    float w[16];
#pragma unroll
    for (int r = 0; r < 8; ++r) w[r] = xs[o + r];
    for (int eb = 0; eb < ntap_pad; eb += 8) {
#pragma unroll
        for (int r = 0; r < 8; ++r) w[8 + r] = xs[o + eb + 8 + r];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const float t = tp[eb + u];
#pragma unroll
            for (int r = 0; r < 8; ++r) acc[r] = fmaf(t, w[r + u], acc[r]);
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) w[r] = w[8 + r];
    }
    float* yrow = Xh + (int64_t)c * ldx;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int64_t i = i0 + o + r;
        if (i < N) yrow[i] = acc[r];
    }
}

cudaError_t launch_highpass(const float* X1, int64_t ldx, int32_t C, int64_t N, const float* taps, int32_t L,
                            float* Xh, cudaStream_t s) {
    const int ntap_pad = ((2 * L + 1) + 7) & ~7;
    const size_t smem = sizeof(float) * ((size_t)ntap_pad + HP_TILE + ntap_pad + 8);
    static bool attr_done = false;
    if (!attr_done) {
        cudaFuncSetAttribute(k_highpass, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr_done = true;
    }
    dim3 grid((unsigned)((N + HP_TILE - 1) / HP_TILE), (unsigned)C);
    k_highpass<<<grid, HP_THREADS, smem, s>>>(X1, ldx, N, taps, L, Xh);
    return cudaGetLastError();
}



// ---------------------------------------------------------------------------
// The same circular highpass by overlap-save FFT convolution (used when the
// truncated impulse response has L <= 1024). One CTA filters two channels at
// once as the real and imaginary parts of a 4096-point complex signal (the
// filter is real, so both come out of one transform): the block x[start-L ..
// start-L+4096) (indices mod N) is transformed by a radix-16 Stockham FFT in
// shared memory, multiplied by H = conj(FFT(g)) where g holds the taps wrapped
// around index 0 (a circular correlation), and transformed back; its outputs
// L .. 4096-L-1 are exact (their taps never wrap inside the block).
// ---------------------------------------------------------------------------
constexpr int HF = 4096;

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                       __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

// Shared-memory index with one pad slot per 16 points (radix-16 passes write
// with stride 16: the pad spreads those writes over the banks).
__device__ __forceinline__ int pad16(int i) { return i + (i >> 4); }
constexpr int HFP = HF + HF / 16;

__device__ __forceinline__ void dft4(float2& x0, float2& x1, float2& x2, float2& x3) {
    const float2 s02 = make_float2(x0.x + x2.x, x0.y + x2.y), d02 = make_float2(x0.x - x2.x, x0.y - x2.y);
    const float2 s13 = make_float2(x1.x + x3.x, x1.y + x3.y), d13 = make_float2(x1.x - x3.x, x1.y - x3.y);
    x0 = make_float2(s02.x + s13.x, s02.y + s13.y);
    x1 = make_float2(d02.x + d13.y, d02.y - d13.x);  // d02 - i*d13
    x2 = make_float2(s02.x - s13.x, s02.y - s13.y);
    x3 = make_float2(d02.x - d13.y, d02.y + d13.x);  // d02 + i*d13
}

// In-register 16-point forward DFT, natural order in and out (n = 4 n1 + n2,
// k = k1 + 4 k2: four 4-point DFTs, twiddles exp(-2 pi i n2 k1 / 16), four
// more 4-point DFTs).
__device__ __forceinline__ void dft16(float2 v[16]) {
    const float c1 = 0.92387953251128674f, s1 = 0.38268343236508977f, r2 = 0.70710678118654752f;
    const float2 W[10] = {{1.f, 0.f}, {c1, -s1}, {r2, -r2}, {s1, -c1}, {0.f, -1.f},
                          {-s1, -c1}, {-r2, -r2}, {-c1, -s1}, {-1.f, 0.f}, {-c1, s1}};
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) dft4(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
    // v[4 k1 + n2] now holds y[n2][k1]
#pragma unroll
    for (int n2 = 1; n2 < 4; ++n2)
#pragma unroll
        for (int k1 = 1; k1 < 4; ++k1) v[4 * k1 + n2] = cmul(v[4 * k1 + n2], W[n2 * k1]);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    // v[4 k1 + k2] holds X[k1 + 4 k2]: transpose to natural order
    float2 t[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) t[k1 + 4 * k2] = v[4 * k1 + k2];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = t[i];
}

// One radix-16 Stockham pass (L = 1, 16, 256 known at compile time), in
// place: one butterfly per thread (blockDim.x == HF / 16), every thread reads
// its 16 inputs before any thread writes. One buffer instead of two lets four
// CTAs share an SM.
template <int L>
__device__ __forceinline__ void fft16_pass(float2* a, const float2* __restrict__ tw) {
    constexpr int step = HF / (16 * L);
    constexpr int lg = (L == 1) ? 0 : (L == 16) ? 4 : 8;
    const int j = threadIdx.x;
    const int k = j & (L - 1), m = j >> lg;
    float2 v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = a[pad16(j + (HF / 16) * i)];
    if (L > 1) {
#pragma unroll
        for (int i = 1; i < 16; ++i) v[i] = cmul(v[i], __ldg(tw + ((i * k * step) & (HF - 1))));
    }
    dft16(v);
    __syncthreads();
    const int base = m * 16 * L + k;
#pragma unroll
    for (int i = 0; i < 16; ++i) a[pad16(base + L * i)] = v[i];
    __syncthreads();
}

constexpr int HF_THREADS = HF / 16;

__global__ void __launch_bounds__(HF_THREADS, 4) k_highpass_fft(const float* __restrict__ X1, int64_t ldx, int32_t C,
                                                               int64_t N, int32_t L, const float2* __restrict__ H,
                                                               const float2* __restrict__ tw, float* __restrict__ Xh) {
    extern __shared__ float2 A[];  // [HFP]: one padded 4096-point buffer, transformed in place
    const int c1 = 2 * blockIdx.y, c2 = c1 + 1;
    const bool two = c2 < C;
    const int64_t start = (int64_t)blockIdx.x * (HF - 2 * L);
    const float* x1 = X1 + (int64_t)c1 * ldx;
    const float* x2 = X1 + (int64_t)(two ? c2 : c1) * ldx;
    // 4 samples per thread loaded before they are stored (8 loads in flight)
    static_assert(HF % (4 * HF_THREADS) == 0, "whole groups of 4 samples per thread");
#pragma unroll
    for (int i0 = 0; i0 < HF / HF_THREADS; i0 += 4) {
        float v1[4], v2[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int n = threadIdx.x + (i0 + u) * HF_THREADS;
            int64_t g = start - L + n;  // circular index (the modulo only near the ends)
            if (g < 0 || g >= N) {
                g %= N;
                if (g < 0) g += N;
            }
            v1[u] = x1[g];
            v2[u] = two ? x2[g] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) A[pad16(threadIdx.x + (i0 + u) * HF_THREADS)] = make_float2(v1[u], v2[u]);
    }
    __syncthreads();
    fft16_pass<1>(A, tw);
    fft16_pass<16>(A, tw);
    fft16_pass<256>(A, tw);
    // conj(Z * H): the second forward transform then gives conj(F * y)
    for (int n = threadIdx.x; n < HF; n += HF_THREADS) {
        const float2 z = cmul(A[pad16(n)], __ldg(H + n));
        A[pad16(n)] = make_float2(z.x, -z.y);
    }
    __syncthreads();
    fft16_pass<1>(A, tw);
    fft16_pass<16>(A, tw);
    fft16_pass<256>(A, tw);
    const float inv = 1.f / (float)HF;
    for (int n = L + threadIdx.x; n < HF - L; n += HF_THREADS) {
        const int64_t i = start + (n - L);
        if (i >= N) break;
        const float2 r = A[pad16(n)];
        Xh[(int64_t)c1 * ldx + i] = r.x * inv;
        if (two) Xh[(int64_t)c2 * ldx + i] = -r.y * inv;
    }
}

cudaError_t launch_highpass_fft(const float* X1, int64_t ldx, int32_t C, int64_t N, int32_t L, const float2* H,
                                const float2* tw, float* Xh, cudaStream_t s) {
    if (L > 1024) return cudaErrorInvalidValue;
    const size_t smem = HFP * sizeof(float2);
    cudaFuncSetAttribute(k_highpass_fft, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid((unsigned)((N + (HF - 2 * L) - 1) / (HF - 2 * L)), (unsigned)((C + 1) / 2));
    k_highpass_fft<<<grid, HF_THREADS, smem, s>>>(X1, ldx, C, N, L, H, tw, Xh);
    return cudaGetLastError();
}

}  // namespace lss
