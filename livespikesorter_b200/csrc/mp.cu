// Greedy matching pursuit as one persistent, cooperatively launched kernel.
//
// Semantics: kilosort/template_matching.py:157-198 (run_matching's round
// loop), which LiveSpikeSorter re-implements as
// kilosortMatchingPursuit (OnlineSpikesV2.cu:873-971) with host round trips
// every round; here the rounds never leave the device.
//
// One round r has two phases separated by grid barriers:
//   P  (peaks)   Cf = relu(B)^2 / nm with the first and last nt columns
//      zeroed; Cfmax, imax = max / first argmax over templates;
//      Cmax = max_pool1d(Cfmax, 2nt+1, stride 1, pad nt);
//      peaks = (Cmax > Th^2) & (|Cmax - Cfmax| < 1e-9), in time order.
//      Each CTA owns W consecutive columns. Column maxima live in cfmax/imax
//      and are refreshed from the update keys of the previous round. The CTA
//      writes its peaks (column, template, amp = B[y, x] / nm[y]) in column
//      order to its region of the per-CTA lists.
//   U  (update)  every CTA prefix-sums the per-CTA peak counts, so the round's
//      spikes have a global time order without another barrier. Then
//      B[:, x + (-nt..nt)] -= amp * ctc[:, y, :] for the even spikes of the
//      round, then for the odd ones. Every column is owned by the first spike
//      whose window covers it; for each element the owner applies the last
//      even spike's term and then the last odd spike's term, which is what the
//      two index_put passes of the reference produce. Products and differences
//      are single-rounded FP32 (__fmul_rn/__fsub_rn), so the score field stays
//      bit-identical to the reference's given the same input field. The new
//      column maxima go to the round's key buffer through a 64-bit atomicMax on
//      (Cf bits << 32 | ~t): larger score first, smaller template index on ties
//      (torch.max's first-index rule). The key buffers alternate by round
//      parity; each CTA clears its columns of the buffer the next round writes.
// Work items of U are (spike, block of template rows, chunk of 32 owned
// columns), each run by one warp without any barrier: a lane owns one column
// and streams its rows eight at a time.
// The grid barrier spins at most ~2 s before setting STATUS_TIMEOUT and
// returning, so the kernel can never hang the device. Everything another CTA
// writes during the kernel is read with ld.global.cg (L2), never through the
// non-coherent L1.
#include "lss_kernels.cuh"
#include "mp_common.cuh"

#include <algorithm>
#include <cfloat>
#include <climits>

namespace lss {

constexpr int MP_THREADS = 512;
static_assert(MP_LIST == 31, "MSG_MP_LIST names the list length");
constexpr int MP_MAX_GRID = 1024;
// U-phase work items: at least MP_ITEMS_PER_WARP items per warp and at most
// MP_ROWS_PER_ITEM template rows per item (whole 8-row batches)
#ifndef MP_ITEMS_PER_WARP
#define MP_ITEMS_PER_WARP 2
#endif
#ifndef MP_ROWS_PER_ITEM
#define MP_ROWS_PER_ITEM 128
#endif
__global__ void __launch_bounds__(MP_THREADS, 1) k_mp(MPArgs a) {
    extern __shared__ float smem[];
    __shared__ int s_pref[MP_MAX_GRID + 1];
    __shared__ int s_wcnt[MP_THREADS / 32];
    __shared__ int s_cnt, s_total;

    const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int N = a.N, T = a.T, nt = a.nt, L2 = 2 * nt + 1;
    const int W = a.cols_per_blk;
    const int lo = min(N, b * W), hi = min(N, lo + W);
    const int64_t ldk = a.ldk;

    float* vals = smem;                                        // [W + 2nt]
    int* ivals = reinterpret_cast<int*>(smem + W + 2 * nt);   // [W]
    float* s_nm = smem + 2 * W + 2 * nt;                       // [T]
    float* s_inv = s_nm + T;                                   // [T]
    for (int t = tid; t < T; t += MP_THREADS) {
        const float v = __ldg(a.nm + t);
        s_nm[t] = v;
        s_inv[t] = __frcp_rn(v);
    }
    __syncthreads();

    // ---- initial column maxima of the score field
    if (a.init_cols) {
        for (int s = lo + tid; s < hi; s += MP_THREADS) {
            const bool edge = (s < nt) || (s >= N - nt);
            ColMax m;
            if (!edge) column_best(a.B, a.ldb, s_nm, s_inv, s, 0, T, m);
            a.cfmax[s] = edge ? 0.f : m.best;
            a.imax[s] = edge ? 0 : m.bi;
        }
    }
    if (!grid_sync(a.bar, a.status)) return;
    __shared__ unsigned long long s_clk[5];
    PhaseClock clk{s_clk};
    if (tid == 0) clk.start();
    int base = 0;
    int r = 0;
    for (; r < a.max_rounds; ++r) {
        unsigned long long* kprev = a.colkey + (int64_t)((r + 1) & 1) * ldk;  // written last round
        unsigned long long* knext = a.colkey + (int64_t)(r & 1) * ldk;        // written this round

        // ---- P: refresh owned maxima, stage the pooled window, pick peaks
        const int nv = (hi - lo) + 2 * nt;
        for (int p = tid; p < nv; p += MP_THREADS) {
            const int s = lo - nt + p;
            float v = -INFINITY;
            if (s >= 0 && s < N) {
                const unsigned long long k = __ldcg(kprev + s);
                const bool own = (s >= lo && s < hi);
                if (k) {
                    v = __uint_as_float((unsigned)(k >> 32));
                    if (own) {
                        const int ix = (int)(0xFFFFFFFFu - (unsigned)(k & 0xFFFFFFFFull));
                        a.cfmax[s] = v;
                        a.imax[s] = ix;
                        ivals[s - lo] = ix;
                    }
                } else {
                    v = __ldcg(a.cfmax + s);
                    if (own) ivals[s - lo] = __ldcg(a.imax + s);
                }
            }
            vals[p] = v;
        }
        if (tid == 0) s_cnt = 0;
        __syncthreads();
        for (int c0 = lo; c0 < hi; c0 += MP_THREADS) {
            const int s = c0 + tid;
            bool flag = false;
            if (s < hi) {
                const int p = s - lo + nt;
                float cm = vals[p - nt];
                for (int d = -nt + 1; d <= nt; ++d) cm = fmaxf(cm, vals[p + d]);
                flag = (cm > a.th2) && (fabsf(__fsub_rn(cm, vals[p])) < 1e-9f);
            }
            const unsigned bal = __ballot_sync(0xffffffffu, flag);
            if (lane == 0) s_wcnt[warp] = __popc(bal);
            __syncthreads();
            if (warp == 0) {
                const int c = (lane < MP_THREADS / 32) ? s_wcnt[lane] : 0;
                const int inc = warp_inc_scan(c, lane);
                if (lane < MP_THREADS / 32) s_wcnt[lane] = inc - c;  // exclusive
                if (lane == MP_THREADS / 32 - 1) s_total = inc;
            }
            __syncthreads();
            if (flag) {
                const int k = s_cnt + s_wcnt[warp] + __popc(bal & ((1u << lane) - 1u));
                const int y = ivals[s - lo];
                a.blk_x[lo + k] = s;
                a.blk_y[lo + k] = y;
                a.blk_amp[lo + k] = __fdiv_rn(__ldcg(a.B + (int64_t)y * a.ldb + s), s_nm[y]);
            }
            __syncthreads();
            if (tid == 0) s_cnt += s_total;
        }
        __syncthreads();
        if (tid == 0) a.blk_cnt[b] = s_cnt;
        if (tid == 0) clk.lap(0);
        if (!grid_sync(a.bar, a.status)) return;
        if (tid == 0) clk.lap(1);

        // ---- U: global order of the round's spikes, records, score update
        {
            int carry = 0;
            for (int c0 = 0; c0 < G; c0 += MP_THREADS) {
                const int i = c0 + tid;
                const int c = (i < G) ? __ldcg(a.blk_cnt + i) : 0;
                const int inc = warp_inc_scan(c, lane);
                if (lane == 31) s_wcnt[warp] = inc;
                __syncthreads();
                if (warp == 0) {
                    const int wc = (lane < MP_THREADS / 32) ? s_wcnt[lane] : 0;
                    const int winc = warp_inc_scan(wc, lane);
                    if (lane < MP_THREADS / 32) s_wcnt[lane] = winc - wc;
                    if (lane == MP_THREADS / 32 - 1) s_total = winc;
                }
                __syncthreads();
                if (i < G) s_pref[i] = carry + s_wcnt[warp] + inc - c;
                carry += s_total;
                __syncthreads();
            }
            if (tid == 0) s_pref[G] = carry;
            __syncthreads();
        }
        const int total = s_pref[G];
        if (total == 0) break;
        if (base + total > a.capacity) {
            if (tid == 0) atomicOr(a.status, STATUS_CAPACITY);
            break;
        }
        {
            const int cnt = s_pref[b + 1] - s_pref[b];
            for (int k = tid; k < cnt; k += MP_THREADS) {
                const int i = base + s_pref[b] + k;
                a.sp_x[i] = __ldcg(a.blk_x + lo + k);
                a.sp_y[i] = __ldcg(a.blk_y + lo + k);
                a.sp_amp[i] = __ldcg(a.blk_amp + lo + k);
                if (a.sp_round) a.sp_round[i] = r;
            }
            if (b == 0 && tid == 0) a.round_start[r] = base;
            for (int s = lo + tid; s < hi; s += MP_THREADS) kprev[s] = 0ull;  // next round's key buffer
        }
        {
            // Work items are (spike, block of template rows, chunk of 32 owned
            // columns), each run by one warp on its own: lane L holds spike
            // q - 1 + L of the round (lane 0 the previous spike), whose
            // windows may cover the owned columns; no barrier inside the phase.
            const int NW = MP_THREADS / 32;
            const int wid = b * NW + warp, wtot = G * NW;
            const int nch = (2 * nt + 1 + 31) / 32;
            int nrb = (MP_ITEMS_PER_WARP * wtot + total * nch - 1) / (total * nch);
            nrb = max(nrb, (T + MP_ROWS_PER_ITEM - 1) / MP_ROWS_PER_ITEM);
            nrb = min(nrb, (T + 7) / 8);
            const int tb = ((T + nrb - 1) / nrb + 7) & ~7;  // whole 8-row batches
            nrb = (T + tb - 1) / tb;
            const int per_spike = nrb * nch;
            const int items = total * per_spike;
            auto fetch = [&](int it2, int& x, int& y, float& amp) {
                const int j = it2 / per_spike - 1 + lane;
                x = INT_MAX;
                y = 0;
                amp = 0.f;
                if (it2 < items && j >= 0 && j < total) {
                    int lo2 = 0, hi2 = G;  // region c with s_pref[c] <= j < s_pref[c+1]
                    while (hi2 - lo2 > 1) {
                        const int m = (lo2 + hi2) >> 1;
                        if (s_pref[m] <= j) lo2 = m; else hi2 = m;
                    }
                    const int idx = lo2 * W + (j - s_pref[lo2]);
                    x = __ldcg(a.blk_x + idx);
                    y = __ldcg(a.blk_y + idx);
                    amp = __ldcg(a.blk_amp + idx);
                }
            };
            int fx = 0, fy = 0;
            float fa = 0.f;
            fetch(wid, fx, fy, fa);
            for (int it = wid; it < items; it += wtot) {
                const int q = it / per_spike, rem = it % per_spike, rb = rem / nch, ch = rem % nch;
                const int x = fx, y = fy;
                const float amp = fa;
                fetch(it + wtot, fx, fy, fa);  // the next item's list loads are in flight meanwhile
                const int j = q - 1 + lane;
                const int xi = __shfl_sync(0xffffffffu, x, 1);
                const int xprev = __shfl_sync(0xffffffffu, x, 0);
                const bool ok = lane >= 1 && j < total && x <= xi + 2 * nt;
                const int nl = __popc(__ballot_sync(0xffffffffu, ok));
                if (lane == 0 && ch == 0 && rb == 0 && nl == MP_LIST && q + MP_LIST < total)
                    atomicOr(a.status, STATUS_LIST);
                const int lo_own = max(max(xi - nt, (q > 0 ? xprev : INT_MIN / 2) + nt + 1), 0);
                const int hi_own = min(xi + nt, N - 1);
                if (lo_own + ch * 32 > hi_own) continue;  // warp-uniform: nothing owned in this chunk
                const int s = lo_own + ch * 32 + lane;
                const bool active = s <= hi_own;
                // last even and last odd spike of the list whose window covers s
                int e0 = -1, e1 = -1;
                for (int e = 0; e < nl; ++e) {
                    const int ex = __shfl_sync(0xffffffffu, x, e + 1);
                    if (active && ex <= s + nt) {
                        if ((q + e) & 1) e1 = e; else e0 = e;
                    }
                }
                const int x0 = __shfl_sync(0xffffffffu, x, max(e0, 0) + 1);
                const int y0 = __shfl_sync(0xffffffffu, y, max(e0, 0) + 1);
                const float a0s = __shfl_sync(0xffffffffu, amp, max(e0, 0) + 1);
                const int x1 = __shfl_sync(0xffffffffu, x, max(e1, 0) + 1);
                const int y1 = __shfl_sync(0xffffffffu, y, max(e1, 0) + 1);
                const float a1s = __shfl_sync(0xffffffffu, amp, max(e1, 0) + 1);
                if (!active) continue;
                const float* c0p = nullptr;
                const float* c1p = nullptr;
                float a0 = 0.f, a1 = 0.f;
                if (e0 >= 0) {
                    c0p = a.ctcP + (int64_t)y0 * T * L2 + (s - x0 + nt);
                    a0 = a0s;
                }
                if (e1 >= 0) {
                    c1p = a.ctcP + (int64_t)y1 * T * L2 + (s - x1 + nt);
                    a1 = a1s;
                }
                const int t0 = rb * tb, t1 = min(T, t0 + tb);
                const bool edge = (s < nt) || (s >= N - nt);
                ColMax m;
                const uint64_t pk = policy_keep(), ps = policy_stream();
                float* bp = a.B + (int64_t)t0 * a.ldb + s;
                const float* p0 = c0p ? c0p + (int64_t)t0 * L2 : nullptr;
                const float* p1 = c1p ? c1p + (int64_t)t0 * L2 : nullptr;
                const int64_t ldb = a.ldb;
                int t = t0;
                // software pipelined: the next eight rows' loads are issued
                // before the current eight are updated (the rows of a column
                // belong to this lane alone); two buffers used alternately, so
                // no register copy has to wait for loads in flight
                auto issue = [&](int dt, float (&lv)[8], float (&l0)[8], float (&l1)[8]) {
#pragma unroll
                    for (int u = 0; u < 8; ++u) lv[u] = ld_keep(bp + (dt + u) * ldb, pk);
#pragma unroll
                    for (int u = 0; u < 8; ++u) l0[u] = p0 ? ld_stream(p0 + (dt + u) * L2, ps) : 0.f;
#pragma unroll
                    for (int u = 0; u < 8; ++u) l1[u] = p1 ? ld_stream(p1 + (dt + u) * L2, ps) : 0.f;
                };
                auto update = [&](const float (&v)[8], const float (&w0)[8], const float (&w1)[8]) {
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        float xv = v[u];
                        if (p0) xv = __fsub_rn(xv, __fmul_rn(a0, w0[u]));
                        if (p1) xv = __fsub_rn(xv, __fmul_rn(a1, w1[u]));
                        st_keep(bp + u * ldb, xv, pk);
                        if (!edge) m.consider(xv, s_nm[t + u], s_inv[t + u], t + u);
                    }
                    bp += 8 * ldb;
                    if (p0) p0 += 8 * L2;
                    if (p1) p1 += 8 * L2;
                    t += 8;
                };
                float va[8], w0a[8], w1a[8], vb[8], w0b[8], w1b[8];
                if (t + 8 <= t1) issue(0, va, w0a, w1a);
                while (t + 8 <= t1) {
                    if (t + 16 <= t1) issue(8, vb, w0b, w1b);
                    update(va, w0a, w1a);
                    if (t + 8 > t1) break;
                    if (t + 16 <= t1) issue(8, va, w0a, w1a);
                    update(vb, w0b, w1b);
                }
                for (; t < t1; ++t, bp += ldb) {
                    float xv = ld_keep(bp, pk);
                    if (p0) { xv = __fsub_rn(xv, __fmul_rn(a0, ld_stream(p0, ps))); p0 += L2; }
                    if (p1) { xv = __fsub_rn(xv, __fmul_rn(a1, ld_stream(p1, ps))); p1 += L2; }
                    st_keep(bp, xv, pk);
                    if (!edge) m.consider(xv, s_nm[t], s_inv[t], t);
                }
                if (!edge && t1 > t0) atomicMax(knext + s, pack_key(m.best, m.bi));
            }
        }
        base += total;
        if (tid == 0) clk.lap(2);
        if (!grid_sync(a.bar, a.status)) return;
        if (tid == 0) clk.lap(3);
    }
    if (tid == 0) {
        clk.lap(2);  // the last round's update phase, or its empty tail
        clk.flush(a.phase);
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
    return std::min(sms * occ, MP_MAX_GRID);
}

size_t mp_smem_bytes(int cols_per_blk, int nt, int T) {
    return sizeof(float) * ((size_t)cols_per_blk + 2 * nt) + sizeof(int) * (size_t)cols_per_blk +
           sizeof(float) * 2 * (size_t)T + 16;
}

cudaError_t launch_mp(MPArgs a, int grid, cudaStream_t s) {
    if (grid > MP_MAX_GRID) return cudaErrorInvalidValue;
    const size_t smem = mp_smem_bytes(a.cols_per_blk, a.nt, a.T);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_mp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    cudaMemsetAsync(a.bar, 0, 2 * sizeof(unsigned int), s);
    // cooperative (all CTAs co-resident for the grid barrier); the launch-attribute
    // form is also valid inside stream capture
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(grid);
    lc.blockDim = dim3(MP_THREADS);
    lc.dynamicSmemBytes = smem;
    lc.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    return cudaLaunchKernelEx(&lc, k_mp, a);
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
// (about 2.3 MB) until the process exits. All calls share it, so calls whose
// work overlaps on the GPU (two streams or two host threads at once) race and
// must be serialised by the caller. Each call clears the parts that must start
// at zero; the rest is fully written before it is read.
// ---------------------------------------------------------------------------
constexpr int NA_MAX_N = 65536;      // LSS_NOALLOC_MAX_SAMPLES
constexpr int NA_MAX_ROUNDS = 1000;
constexpr size_t na_align(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t NA_OFF_CFMAX = 0;
constexpr size_t NA_OFF_IMAX = na_align(NA_OFF_CFMAX + sizeof(float) * NA_MAX_N);
constexpr size_t NA_OFF_COLKEY = na_align(NA_OFF_IMAX + sizeof(int32_t) * NA_MAX_N);
constexpr size_t NA_OFF_BLKX = na_align(NA_OFF_COLKEY + 2 * sizeof(unsigned long long) * NA_MAX_N);
constexpr size_t NA_OFF_BLKY = na_align(NA_OFF_BLKX + sizeof(int32_t) * NA_MAX_N);
constexpr size_t NA_OFF_BLKAMP = na_align(NA_OFF_BLKY + sizeof(int32_t) * NA_MAX_N);
constexpr size_t NA_OFF_BLKCNT = na_align(NA_OFF_BLKAMP + sizeof(float) * NA_MAX_N);
constexpr size_t NA_OFF_RSTART = na_align(NA_OFF_BLKCNT + sizeof(int32_t) * MP_MAX_GRID);
constexpr size_t NA_OFF_ZERO = na_align(NA_OFF_RSTART + sizeof(int32_t) * (NA_MAX_ROUNDS + 2));
// zero-initialised tail: counters[4], status, pad, barrier[2]
constexpr size_t NA_ZERO_BYTES = 256;
constexpr size_t NA_BYTES = NA_OFF_ZERO + NA_ZERO_BYTES;

static __device__ __align__(256) unsigned char g_mp_scratch[NA_BYTES];

}  // namespace lss

#include <mutex>

#include "lss.h"

namespace {
std::mutex g_na_mutex;
// device address of g_mp_scratch, per device ordinal, looked up on the first
// call on that device; a cudaDeviceReset ends the context the address belongs
// to, so a process that resets a device must not call this entry point again
unsigned char* g_na_base[256] = {};
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
    // every array the kernel dereferences must be memory of the current
    // device (or pinned host memory): a pageable host array or another GPU's
    // buffer would fault in the kernel, so it is refused before any launch
    for (const void* p : {(const void*)B_dev, (const void*)nm_dev, (const void*)ctc_permuted_dev,
                          (const void*)spike_x, (const void*)spike_y, (const void*)spike_amp})
        if (!device_accessible(p, dev)) {
            set_thread_error("lss_mp_rounds_noalloc: arrays must be memory of the current device or pinned host memory");
            return LSS_ERR_ARG;
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
    a.ldk = NA_MAX_N;
    a.blk_x = reinterpret_cast<int32_t*>(base + NA_OFF_BLKX);
    a.blk_y = reinterpret_cast<int32_t*>(base + NA_OFF_BLKY);
    a.blk_amp = reinterpret_cast<float*>(base + NA_OFF_BLKAMP);
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
    a.init_cols = 1;
    if ((e = cudaMemsetAsync(a.colkey, 0, sizeof(unsigned long long) * n_samples, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(a.colkey + NA_MAX_N, 0, sizeof(unsigned long long) * n_samples, s)) != cudaSuccess ||
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
    if (st & STATUS_CAPACITY) {
        set_thread_error("lss_mp_rounds_noalloc: more spikes than capacity");
        return LSS_ERR_CAPACITY;
    }
    if (st & STATUS_LIST) {
        set_thread_error(MSG_MP_LIST);
        return LSS_ERR_CAPACITY;
    }
    return LSS_OK;
}
