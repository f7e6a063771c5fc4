// Post-processing of a batch's spikes before they are emitted: positions,
// cluster assignment, duplicate removal and time order.
//
// * Position (kilosort/postprocessing.py:33-46, compute_spike_positions;
//   LiveSpikeSorter compute_spike_positions_kernel, OnlineSpikesV2.cu:189-244):
//   the PC-feature energy of each of the spike's nC nearest channels,
//   normalised to 1, weights those channels' coordinates.
// * Cluster (OnlineSpikesV2::closestCluster, OnlineSpikesV2.cu:1028-1043): the
//   nearest cluster centroid by Euclidean distance, first index on ties. (The
//   reference loops over its template count instead of its centroid count;
//   here the loop covers exactly the centroids given.)
// * Duplicates (kilosort/postprocessing.py:10-31, remove_duplicates, applied
//   per cluster to time-ordered spikes; OnlineSpikesV2::saveSpikes,
//   OnlineSpikesV2.cu:1131-1164): a spike closer than dt samples to the last
//   kept spike of its cluster is dropped. The last kept time per cluster is
//   carried from batch to batch, so a stream is deduplicated as a whole.
// * Order: records are emitted sorted by time, ties in matching order (the
//   order saveSpikes' sorted insertion produces).
//
// The spike count may live on the device (graph-captured batches): keys of
// the unused tail are all-ones so they sort last, and every sort covers the
// fixed bound.
#include <cub/device/device_radix_sort.cuh>

#include "lss_kernels.cuh"

namespace lss {

constexpr unsigned long long KEY_NONE = ~0ull;

__device__ __forceinline__ int64_t post_time(int x, int64_t ibatch, const RecordClock& rc) {
    return (int64_t)(x - rc.nt) + ibatch * (int64_t)rc.NT + rc.shift - rc.nt / 2 + rc.nt0min;
}

__global__ void k_post_keys(PostArgs a, RecordClock rc, int32_t n_max) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_max) return;
    const int n = rc.counters ? rc.counters[0] : n_max;
    const int64_t ibatch = rc.ibatch_dev ? *rc.ibatch_dev : rc.ibatch;
    if (i >= n) {
        a.key_c[i] = KEY_NONE;
        a.key_t[i] = KEY_NONE;
        return;
    }
    const int x = a.sp_x[i], y = a.sp_y[i];
    float px = 0.f, py = 0.f;
    if (a.tF && a.xc) {
        float mass[16];
        float tot = 0.f;
        for (int j = 0; j < a.nC; ++j) {
            float m = 0.f;
            for (int k = 0; k < a.K; ++k) {
                const float v = a.tF[((int64_t)i * a.nC + j) * a.K + k];
                m = __fadd_rn(m, __fmul_rn(v, v));
            }
            mass[j] = m;
            tot = __fadd_rn(tot, m);
        }
        const int64_t u = a.iU[y];
        for (int j = 0; j < a.nC; ++j) {
            const float w = tot > 0.f ? __fdiv_rn(mass[j], tot) : 0.f;
            const int64_t ch = a.iCC[(int64_t)j * a.C + u];
            px = __fadd_rn(px, __fmul_rn(a.xc[ch], w));
            py = __fadd_rn(py, __fmul_rn(a.yc[ch], w));
        }
    }
    int clu = y;
    if (a.n_clu > 0) {
        float best = 3.402823466e38f;
        clu = 0;
        for (int c = 0; c < a.n_clu; ++c) {
            const float dx = __fsub_rn(px, a.cen_x[c]), dy = __fsub_rn(py, a.cen_y[c]);
            const float d = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
            if (d < best) {
                best = d;
                clu = c;
            }
        }
    }
    a.px[i] = px;
    a.py[i] = py;
    a.clu[i] = clu;
    a.keep[i] = 0;
    const bool valid = post_time(x, ibatch, rc) >= 0;  // the first batch drops negative times
    a.key_c[i] = valid ? ((unsigned long long)clu << 40) | ((unsigned long long)x << 20) | (unsigned long long)i
                       : KEY_NONE;
    a.key_t[i] = valid ? ((unsigned long long)x << 20) | (unsigned long long)i : KEY_NONE;
}

// One thread per cluster segment of the (cluster, time, index)-sorted keys.
__global__ void k_post_dedup(PostArgs a, RecordClock rc, int32_t n_max) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_max) return;
    const unsigned long long kj = a.key_c_sorted[j];
    if (kj == KEY_NONE) return;
    const unsigned long long cj = kj >> 40;
    if (j > 0 && (a.key_c_sorted[j - 1] >> 40) == cj) return;  // not a segment start
    const int64_t ibatch = rc.ibatch_dev ? *rc.ibatch_dev : rc.ibatch;
    int64_t last = a.last_time[cj];
    for (int q = j; q < n_max; ++q) {
        const unsigned long long kq = a.key_c_sorted[q];
        if (kq == KEY_NONE || (kq >> 40) != cj) break;
        const int i = (int)(kq & 0xFFFFFull);
        const int x = (int)((kq >> 20) & 0xFFFFFull);
        const int64_t t = post_time(x, ibatch, rc);
        if (a.dt <= 0 || t >= last + a.dt) {
            a.keep[i] = 1;
            last = t;
        }
    }
    a.last_time[cj] = last;
}

// Output slots in time order (one CTA).
__global__ void __launch_bounds__(1024) k_post_slots(PostArgs a, RecordClock rc, int32_t n_max, int32_t* slot,
                                                     int64_t* out_count) {
    __shared__ int wsum[32];
    __shared__ int s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = rc.counters ? rc.counters[0] : n_max;
    const int64_t ibatch = rc.ibatch_dev ? *rc.ibatch_dev : rc.ibatch;
    if (threadIdx.x == 0) s_base = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) slot[i] = -1;
    __syncthreads();
    for (int c0 = 0; c0 < n; c0 += 1024) {
        const int j = c0 + threadIdx.x;
        int i = -1;
        if (j < n) {
            const unsigned long long k = a.key_t_sorted[j];
            if (k != KEY_NONE) i = (int)(k & 0xFFFFFull);
        }
        const bool keep = i >= 0 && a.keep[i];
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) wsum[warp] = __popc(bal);
        __syncthreads();
        if (warp == 0) {
            const int c = wsum[lane];
            int inc = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += u;
            }
            wsum[lane] = inc - c;
        }
        __syncthreads();
        if (keep) slot[i] = s_base + wsum[warp] + __popc(bal & ((1u << lane) - 1u));
        __syncthreads();
        if (threadIdx.x == 1023) s_base += wsum[31] + __popc(bal);
        __syncthreads();
    }
    if (threadIdx.x == 0) out_count[rc.slots > 0 ? ibatch % rc.slots : 0] = s_base;
}

size_t post_sort_bytes(int32_t n_max) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, bytes, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                   n_max);
    return bytes;
}

cudaError_t launch_post(const PostArgs& a, const RecordClock& rc, int32_t n_max, int32_t* slot, int64_t* out_count,
                        cudaStream_t s) {
    if (a.nC > 16) return cudaErrorInvalidValue;
    if (n_max <= 0) {
        // nothing to sort: the count is zero (host-known batch index here)
        return cudaMemsetAsync(out_count + (rc.slots > 0 ? rc.ibatch % rc.slots : 0), 0, sizeof(int64_t), s);
    }
    const int grid = (n_max + 255) / 256;
    k_post_keys<<<grid, 256, 0, s>>>(a, rc, n_max);
    size_t bytes = a.sort_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortKeys(a.sort_tmp, bytes, a.key_c, a.key_c_sorted, n_max, 0, 64, s);
    if (e != cudaSuccess) return e;
    k_post_dedup<<<grid, 256, 0, s>>>(a, rc, n_max);
    bytes = a.sort_bytes;
    e = cub::DeviceRadixSort::SortKeys(a.sort_tmp, bytes, a.key_t, a.key_t_sorted, n_max, 0, 64, s);
    if (e != cudaSuccess) return e;
    k_post_slots<<<1, 1024, 0, s>>>(a, rc, n_max, slot, out_count);
    return cudaGetLastError();
}

__global__ void k_post_write(const PostArgs a, const RecordClock rc, const int32_t* slot, int32_t n_max,
                             float* out_x, float* out_y, int32_t* out_clu, int64_t capacity) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = rc.counters ? rc.counters[0] : n_max;
    if (i >= n || i >= n_max) return;
    const int o = slot[i];
    if (o < 0 || o >= capacity) return;
    const int64_t ibatch = rc.ibatch_dev ? *rc.ibatch_dev : rc.ibatch;
    const int64_t q = (rc.slots > 0 ? (ibatch % rc.slots) * capacity : 0) + o;
    if (out_x) out_x[q] = a.px[i];
    if (out_y) out_y[q] = a.py[i];
    if (out_clu) out_clu[q] = a.clu[i];
}

cudaError_t launch_post_write(const PostArgs& a, const RecordClock& rc, const int32_t* slot, int32_t n_max,
                              float* out_x, float* out_y, int32_t* out_clu, int64_t capacity, cudaStream_t s) {
    if (n_max <= 0 || (!out_x && !out_y && !out_clu)) return cudaSuccess;
    k_post_write<<<(n_max + 255) / 256, 256, 0, s>>>(a, rc, slot, n_max, out_x, out_y, out_clu, capacity);
    return cudaGetLastError();
}

}  // namespace lss
