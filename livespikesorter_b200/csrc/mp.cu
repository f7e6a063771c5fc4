// Greedy matching pursuit as one persistent, cooperatively launched kernel.
//
// Semantics: kilosort/template_matching.py:157-198 (run_matching's round
// loop), which LiveSpikeSorter re-implements as
// kilosortMatchingPursuit (OnlineSpikesV2.cu:873-971) with host round trips
// every round; here the rounds never leave the device.
//
// One round r:
//   P  (peak pick)  Cf = relu(B)^2 / nm with the first and last nt columns
//      zeroed; Cfmax, imax = max / first argmax over templates;
//      Cmax = max_pool1d(Cfmax, 2nt+1, stride 1, pad nt);
//      peaks = (Cmax > Th^2) & (|Cmax - Cfmax| < 1e-9), in time order.
//      Each CTA owns W consecutive columns; column maxima are kept in
//      cfmax/imax and refreshed from `colkey` where the previous round's
//      update touched them.
//   C0 (compact)    every CTA scans the per-CTA peak counts, writes its peaks
//      at their global time-ordered slots with amp = B[y, x] / nm[y], and
//      clears its columns' colkey.
//   U  (update)     B[:, x + (-nt..nt)] -= amp * ctc[:, y, :] for the even
//      spikes of the round, then for the odd ones. Every column is owned by
//      the first spike whose window covers it; for each element the owner
//      applies the last even spike's term and then the last odd spike's term,
//      which is what the two index_put passes of the reference produce. The
//      products and differences are single-rounded FP32 (__fmul_rn/__fsub_rn),
//      so the score field stays bit-identical to the reference's given the same
//      input field. The touched columns' new maxima go to colkey through a
//      64-bit atomicMax on (Cf bits << 32 | ~t), i.e. larger score first and
//      smaller template index on ties (torch.max's first-index rule).
// A grid barrier separates the phases; it spins at most ~2 s before setting
// STATUS_TIMEOUT and returning, so the kernel can never hang the device.
// Everything another CTA writes during the kernel is read with ld.global.cg
// (L2), never through the non-coherent L1.
#include "lss_kernels.cuh"

#include <cfloat>

namespace lss {

constexpr int MP_THREADS = 512;
constexpr int MP_COLS = 128;
constexpr int MP_GROUPS = MP_THREADS / MP_COLS;
constexpr int MP_LIST_MAX = 32;
constexpr unsigned MP_SPIN_LIMIT = 1u << 24;

__device__ __forceinline__ bool grid_sync(unsigned int* bar, int32_t* status) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* vgen = bar + 1;
        const unsigned int gen = *vgen;
        __threadfence();
        const unsigned int arrived = atomicAdd(bar, 1u);
        int ok = 1;
        if (arrived == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            unsigned int spins = 0;
            while (*vgen == gen) {
                if ((++spins & 255u) == 0u && (*(volatile int32_t*)status & STATUS_TIMEOUT)) {
                    ok = 0;
                    break;
                }
                if (spins > MP_SPIN_LIMIT) {
                    atomicOr(status, STATUS_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(128);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ float cf_of(float b, float nmv) {
    const float r = fmaxf(b, 0.f);
    return __fdiv_rn(__fmul_rn(r, r), nmv);
}

__device__ __forceinline__ unsigned long long pack_key(float cf, int t) {
    return ((unsigned long long)__float_as_uint(cf) << 32) | (unsigned long long)(0xFFFFFFFFu - (unsigned)t);
}

// Reduce (best, idx) over the MP_GROUPS row groups of a 128-column strip.
// Returns the winner in the group-0 thread of each column.
__device__ __forceinline__ void group_reduce(float& best, int& bi, float* sb, int* si) {
    const int col = threadIdx.x % MP_COLS, g = threadIdx.x / MP_COLS;
    sb[g * MP_COLS + col] = best;
    si[g * MP_COLS + col] = bi;
    __syncthreads();
    if (g == 0) {
#pragma unroll
        for (int h = 1; h < MP_GROUPS; ++h) {
            const float v = sb[h * MP_COLS + col];
            const int ix = si[h * MP_COLS + col];
            if (v > best || (v == best && ix < bi)) {
                best = v;
                bi = ix;
            }
        }
    }
    __syncthreads();
}

struct ListEnt {
    int x, y, par;
    float amp;
};

__global__ void __launch_bounds__(MP_THREADS, 1) k_mp(MPArgs a) {
    extern __shared__ float smem[];
    __shared__ float s_best[MP_THREADS];
    __shared__ int s_idx[MP_THREADS];
    __shared__ int s_scan[MP_THREADS];
    __shared__ ListEnt s_list[MP_LIST_MAX];
    __shared__ int s_nlist, s_total, s_off, s_cnt;

    const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
    const int N = a.N, T = a.T, nt = a.nt, L2 = 2 * nt + 1;
    const int W = a.cols_per_blk;
    const int lo = b * W, hi = min(N, lo + W);
    const int col = tid % MP_COLS, grp = tid / MP_COLS;

    // ---- initial column maxima of the score field
    if (a.init_cols) {
        for (int c0 = lo; c0 < hi; c0 += MP_COLS) {
            const int s = c0 + col;
            float best = -1.f;
            int bi = 0;
            const bool edge = (s < nt) || (s >= N - nt);
            if (s < hi && !edge) {
                for (int t = grp; t < T; t += MP_GROUPS) {
                    const float cf = cf_of(__ldcg(a.B + (int64_t)t * a.ldb + s), __ldg(a.nm + t));
                    if (cf > best) {
                        best = cf;
                        bi = t;
                    }
                }
            }
            group_reduce(best, bi, s_best, s_idx);
            if (grp == 0 && s < hi) {
                a.cfmax[s] = edge ? 0.f : best;
                a.imax[s] = edge ? 0 : bi;
            }
        }
    }
    if (!grid_sync(a.bar, a.status)) return;

    float* vals = smem;  // [W + 2nt]
    int base = 0;
    int r = 0;
    for (; r < a.max_rounds; ++r) {
        // ---- P: refresh owned maxima, stage the pooled window, pick peaks
        const int nv = (hi - lo) + 2 * nt;
        for (int p = tid; p < nv; p += MP_THREADS) {
            const int s = lo - nt + p;
            float v = -INFINITY;
            if (s >= 0 && s < N) {
                const unsigned long long k = __ldcg(a.colkey + s);
                if (k) {
                    v = __uint_as_float((unsigned)(k >> 32));
                    if (s >= lo && s < hi) {
                        a.cfmax[s] = v;
                        a.imax[s] = (int)(0xFFFFFFFFu - (unsigned)(k & 0xFFFFFFFFull));
                    }
                } else {
                    v = __ldcg(a.cfmax + s);
                }
            }
            vals[p] = v;
        }
        __syncthreads();
        if (tid == 0) s_cnt = 0;
        __syncthreads();
        for (int c0 = lo; c0 < hi; c0 += MP_THREADS) {
            const int s = c0 + tid;
            int flag = 0;
            if (s < hi) {
                const int p = s - lo + nt;
                float cm = vals[p - nt];
                for (int d = -nt + 1; d <= nt; ++d) cm = fmaxf(cm, vals[p + d]);
                const float v = vals[p];
                flag = (cm > a.th2) && (fabsf(__fsub_rn(cm, v)) < 1e-9f);
            }
            // ordered block compaction
            s_scan[tid] = flag;
            __syncthreads();
            for (int off = 1; off < MP_THREADS; off <<= 1) {
                const int v = (tid >= off) ? s_scan[tid - off] : 0;
                __syncthreads();
                s_scan[tid] += v;
                __syncthreads();
            }
            if (flag) {
                const int k = s_cnt + s_scan[tid] - 1;
                a.blk_x[lo + k] = s;
                a.blk_y[lo + k] = __ldcg(a.imax + s);
            }
            __syncthreads();
            if (tid == MP_THREADS - 1) s_cnt += s_scan[tid];
            __syncthreads();
        }
        if (tid == 0) a.blk_cnt[b] = s_cnt;
        if (!grid_sync(a.bar, a.status)) return;

        // ---- C0: global time order, amplitudes, records
        {
            int v = 0;
            for (int i = tid; i < G; i += MP_THREADS) v += (i < b) ? __ldcg(a.blk_cnt + i) : 0;
            int tot = 0;
            for (int i = tid; i < G; i += MP_THREADS) tot += __ldcg(a.blk_cnt + i);
            s_scan[tid] = v;
            s_best[tid] = __int_as_float(tot);
            __syncthreads();
            if (tid == 0) {
                int o = 0, t2 = 0;
                for (int i = 0; i < MP_THREADS; ++i) {
                    o += s_scan[i];
                    t2 += __float_as_int(s_best[i]);
                }
                s_off = o;
                s_total = t2;
            }
            __syncthreads();
        }
        const int total = s_total;
        if (total == 0) break;
        if (base + total > a.capacity) {
            if (tid == 0) atomicOr(a.status, STATUS_CAPACITY);
            break;
        }
        {
            const int cnt = __ldcg(a.blk_cnt + b);
            for (int k = tid; k < cnt; k += MP_THREADS) {
                const int i = base + s_off + k;
                const int x = __ldcg(a.blk_x + lo + k);
                const int y = __ldcg(a.blk_y + lo + k);
                a.sp_x[i] = x;
                a.sp_y[i] = y;
                a.sp_amp[i] = __fdiv_rn(__ldcg(a.B + (int64_t)y * a.ldb + x), __ldg(a.nm + y));
                if (a.sp_round) a.sp_round[i] = r;
            }
            if (b == 0 && tid == 0) a.round_start[r] = base;
            for (int s = lo + tid; s < hi; s += MP_THREADS)
                if (__ldcg(a.colkey + s)) a.colkey[s] = 0ull;
        }
        if (!grid_sync(a.bar, a.status)) return;

        // ---- U: subtract the round's spikes from the score field
        {
            const int tb_min = 16;
            int nrb = (T + 63) / 64;
            const int want = (2 * G + total - 1) / total;
            if (want > nrb) nrb = want;
            const int nrb_max = (T + tb_min - 1) / tb_min;
            if (nrb > nrb_max) nrb = nrb_max;
            const int tb = (T + nrb - 1) / nrb;
            const int items = total * nrb;
            for (int it = b; it < items; it += G) {
                const int q = it / nrb, rb = it % nrb;
                const int i = base + q;
                const int xi = __ldcg(a.sp_x + i);
                int lo_own = xi - nt;
                if (q > 0) lo_own = max(lo_own, __ldcg(a.sp_x + i - 1) + nt + 1);
                lo_own = max(lo_own, 0);
                const int hi_own = min(xi + nt, N - 1);
                if (tid == 0) {
                    int n = 0;
                    for (int j = i; j < base + total; ++j) {
                        const int xj = __ldcg(a.sp_x + j);
                        if (xj > xi + 2 * nt) break;
                        if (n == MP_LIST_MAX) {
                            atomicOr(a.status, STATUS_LIST);
                            break;
                        }
                        s_list[n].x = xj;
                        s_list[n].y = __ldcg(a.sp_y + j);
                        s_list[n].amp = __ldcg(a.sp_amp + j);
                        s_list[n].par = (j - base) & 1;
                        ++n;
                    }
                    s_nlist = n;
                }
                __syncthreads();
                const int nl = s_nlist;
                const int t0 = rb * tb, t1 = min(T, t0 + tb);
                for (int c0 = lo_own; c0 <= hi_own; c0 += MP_COLS) {
                    const int s = c0 + col;
                    float best = -1.f;
                    int bi = 0;
                    const bool active = s <= hi_own;
                    const bool edge = (s < nt) || (s >= N - nt);
                    if (active) {
                        int e0 = -1, e1 = -1;
                        for (int e = 0; e < nl; ++e) {
                            if (s_list[e].x > s + nt) break;
                            if (s_list[e].par) e1 = e; else e0 = e;
                        }
                        const float* c0p = nullptr;
                        const float* c1p = nullptr;
                        float a0 = 0.f, a1 = 0.f;
                        if (e0 >= 0) {
                            c0p = a.ctcP + (int64_t)s_list[e0].y * T * L2 + (s - s_list[e0].x + nt);
                            a0 = s_list[e0].amp;
                        }
                        if (e1 >= 0) {
                            c1p = a.ctcP + (int64_t)s_list[e1].y * T * L2 + (s - s_list[e1].x + nt);
                            a1 = s_list[e1].amp;
                        }
                        for (int t = t0 + grp; t < t1; t += MP_GROUPS) {
                            float* bp = a.B + (int64_t)t * a.ldb + s;
                            float v = __ldcg(bp);
                            if (c0p) v = __fsub_rn(v, __fmul_rn(a0, __ldg(c0p + (int64_t)t * L2)));
                            if (c1p) v = __fsub_rn(v, __fmul_rn(a1, __ldg(c1p + (int64_t)t * L2)));
                            __stcg(bp, v);
                            if (!edge) {
                                const float cf = cf_of(v, __ldg(a.nm + t));
                                if (cf > best) {
                                    best = cf;
                                    bi = t;
                                }
                            }
                        }
                    }
                    group_reduce(best, bi, s_best, s_idx);
                    if (grp == 0 && active && !edge && t1 > t0)
                        atomicMax(a.colkey + s, pack_key(best, bi));
                }
                __syncthreads();
            }
        }
        base += total;
        if (!grid_sync(a.bar, a.status)) return;
    }
    if (b == 0 && tid == 0) {
        a.counters[0] = base;
        a.counters[1] = r;
        a.round_start[r] = base;
    }
}

int mp_max_grid(int device) {
    int sms = 0, occ = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mp, MP_THREADS, 48 * 1024);
    if (occ < 1) occ = 1;
    if (occ > 1) occ = 1;
    return sms * occ;
}

cudaError_t launch_mp(MPArgs a, int grid, cudaStream_t s) {
    const size_t smem = sizeof(float) * ((size_t)a.cols_per_blk + 2 * a.nt + 8);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_mp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    cudaMemsetAsync(a.bar, 0, 2 * sizeof(unsigned int), s);
    void* args[] = {&a};
    return cudaLaunchCooperativeKernel((void*)k_mp, dim3(grid), dim3(MP_THREADS), args, smem, s);
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the rounds (lss_mp_rounds_noalloc).
//
// Some callers cannot allocate device memory once they are running: a plugin
// inside an acquisition host that owns the GPU's memory, a process whose
// device memory is reserved up front by another allocator, or a real-time loop
// that may not take cudaMalloc's implicit synchronisation. For them the
// rounds' working memory (column maxima, update keys, per-CTA peak lists,
// round offsets, counters and the grid barrier) lives in one fixed array
// compiled into this library. Every GPU that loads the library holds the array
// (about 1.6 MB) until the process exits. All calls share it, so calls whose
// work overlaps on the GPU (two streams or two host threads at once) race and
// must be serialised by the caller. Each call clears the parts that must start
// at zero; the rest is fully written before it is read.
// ---------------------------------------------------------------------------
constexpr int NA_MAX_N = 65536;      // LSS_NOALLOC_MAX_SAMPLES
constexpr int NA_MAX_GRID = 1024;
constexpr int NA_MAX_ROUNDS = 1000;
constexpr size_t na_align(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t NA_OFF_CFMAX = 0;
constexpr size_t NA_OFF_IMAX = na_align(NA_OFF_CFMAX + sizeof(float) * NA_MAX_N);
constexpr size_t NA_OFF_COLKEY = na_align(NA_OFF_IMAX + sizeof(int32_t) * NA_MAX_N);
constexpr size_t NA_OFF_BLKX = na_align(NA_OFF_COLKEY + sizeof(unsigned long long) * NA_MAX_N);
constexpr size_t NA_OFF_BLKY = na_align(NA_OFF_BLKX + sizeof(int32_t) * NA_MAX_N);
constexpr size_t NA_OFF_BLKCNT = na_align(NA_OFF_BLKY + sizeof(int32_t) * NA_MAX_N);
constexpr size_t NA_OFF_RSTART = na_align(NA_OFF_BLKCNT + sizeof(int32_t) * NA_MAX_GRID);
constexpr size_t NA_OFF_ZERO = na_align(NA_OFF_RSTART + sizeof(int32_t) * (NA_MAX_ROUNDS + 2));
// zero-initialised tail: counters[4], status, pad, barrier[2]
constexpr size_t NA_ZERO_BYTES = 256;
constexpr size_t NA_BYTES = NA_OFF_ZERO + NA_ZERO_BYTES;

static __device__ __align__(256) unsigned char g_mp_scratch[NA_BYTES];

}  // namespace lss

#include <mutex>

#include "../../include/lss.h"

namespace {
std::mutex g_na_mutex;
unsigned char* g_na_base[256] = {};  // device address of g_mp_scratch, per device ordinal
}  // namespace

extern "C" int lss_mp_rounds_noalloc(float* B_dev, int64_t ldb, int32_t n_templates, int32_t n_samples,
                                     int32_t nt, float th_learned, const float* nm_dev,
                                     const float* ctc_permuted_dev, int32_t max_rounds, int32_t capacity,
                                     int32_t* spike_x, int32_t* spike_y, float* spike_amp, int32_t* n_spikes,
                                     int32_t* n_rounds, void* stream) {
    using namespace lss;
    if (!B_dev || !nm_dev || !ctc_permuted_dev || !spike_x || !spike_y || !spike_amp || !n_spikes || !n_rounds) {
        set_thread_error("lss_mp_rounds_noalloc: null pointer argument");
        return LSS_ERR_ARG;
    }
    if (n_samples > NA_MAX_N) {
        set_thread_error("lss_mp_rounds_noalloc: n_samples exceeds LSS_NOALLOC_MAX_SAMPLES (65536)");
        return LSS_ERR_ARG;
    }
    if (n_templates <= 0 || nt <= 0 || nt % 2 == 0 || n_samples <= 2 * nt || ldb < n_samples) {
        set_thread_error("lss_mp_rounds_noalloc: need n_templates > 0, odd nt, n_samples > 2*nt, ldb >= n_samples");
        return LSS_ERR_ARG;
    }
    if (max_rounds <= 0 || max_rounds > NA_MAX_ROUNDS || capacity <= 0 || !(th_learned > 0.f)) {
        set_thread_error("lss_mp_rounds_noalloc: need 0 < max_rounds <= 1000, capacity > 0, th_learned > 0");
        return LSS_ERR_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 256) {
        set_thread_error("lss_mp_rounds_noalloc: no current CUDA device");
        return LSS_ERR_CUDA;
    }
    unsigned char* base = nullptr;
    {
        // one-time set-up per device: the device address of the scratch array
        std::lock_guard<std::mutex> lock(g_na_mutex);
        if (!g_na_base[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_mp_scratch);
            if (e != cudaSuccess) {
                set_thread_error(cudaGetErrorString(e));
                return LSS_ERR_CUDA;
            }
            g_na_base[dev] = static_cast<unsigned char*>(p);
        }
        base = g_na_base[dev];
    }
    const int G = mp_max_grid(dev);
    if (G > NA_MAX_GRID) {
        set_thread_error("lss_mp_rounds_noalloc: device has more SMs than the scratch supports");
        return LSS_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    MPArgs a{};
    a.B = B_dev;
    a.ldb = ldb;
    a.T = n_templates;
    a.N = n_samples;
    a.nt = nt;
    a.th2 = th_learned * th_learned;
    a.nm = nm_dev;
    a.ctcP = ctc_permuted_dev;
    a.cfmax = reinterpret_cast<float*>(base + NA_OFF_CFMAX);
    a.imax = reinterpret_cast<int32_t*>(base + NA_OFF_IMAX);
    a.colkey = reinterpret_cast<unsigned long long*>(base + NA_OFF_COLKEY);
    a.blk_x = reinterpret_cast<int32_t*>(base + NA_OFF_BLKX);
    a.blk_y = reinterpret_cast<int32_t*>(base + NA_OFF_BLKY);
    a.blk_cnt = reinterpret_cast<int32_t*>(base + NA_OFF_BLKCNT);
    a.round_start = reinterpret_cast<int32_t*>(base + NA_OFF_RSTART);
    int32_t* zero = reinterpret_cast<int32_t*>(base + NA_OFF_ZERO);
    a.counters = zero;           // [4]
    a.status = zero + 4;         // [1]
    a.bar = reinterpret_cast<unsigned int*>(zero + 8);  // [2]
    a.sp_x = spike_x;
    a.sp_y = spike_y;
    a.sp_amp = spike_amp;
    a.sp_round = nullptr;
    a.capacity = capacity;
    a.max_rounds = max_rounds;
    a.cols_per_blk = (n_samples + G - 1) / G;
    a.rows_per_item = 64;
    a.init_cols = 1;
    if ((e = cudaMemsetAsync(a.colkey, 0, sizeof(unsigned long long) * n_samples, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(zero, 0, NA_ZERO_BYTES, s)) != cudaSuccess ||
        (e = launch_mp(a, G, s)) != cudaSuccess) {
        set_thread_error(cudaGetErrorString(e));
        return LSS_ERR_CUDA;
    }
    int32_t hc[8] = {0};
    if ((e = cudaMemcpyAsync(hc, zero, sizeof(hc), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
        set_thread_error(cudaGetErrorString(e));
        return LSS_ERR_CUDA;
    }
    const int32_t st = hc[4];
    *n_spikes = hc[0];
    *n_rounds = hc[1];
    if (st & STATUS_TIMEOUT) {
        set_thread_error("lss_mp_rounds_noalloc: grid barrier timed out");
        return LSS_ERR_TIMEOUT;
    }
    if (st & (STATUS_CAPACITY | STATUS_LIST)) {
        set_thread_error("lss_mp_rounds_noalloc: more spikes than capacity, or a 2*nt window with over 32 peaks");
        return LSS_ERR_CAPACITY;
    }
    return LSS_OK;
}
