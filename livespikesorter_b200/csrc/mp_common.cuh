// Device helpers shared by the two matching-pursuit kernels (mp.cu: the
// rounds over the whole score field; mp_blocks.cu: the rounds that skip
// template-row blocks whose update leaves every score unchanged).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lss_kernels.cuh"

namespace lss {

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
                ++spins;
                if ((spins & 255u) == 0u && (*(volatile int32_t*)status & STATUS_TIMEOUT)) {
                    ok = 0;
                    break;
                }
                if (spins > MP_SPIN_LIMIT) {
                    atomicOr(status, STATUS_TIMEOUT);
                    ok = 0;
                    break;
                }
                if (spins > 64) __nanosleep(32);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// L2 residency: the score field is read-modify-written every round and fits
// in L2 for a few hundred templates, while each spike's ctc slice is read once
// per spike, so the field is kept (evict_last) and ctc streamed (evict_first).
__device__ __forceinline__ uint64_t policy_keep() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t policy_stream() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ float ld_keep(const float* a, uint64_t pol) {
    float v;
    asm volatile("ld.global.cg.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ void st_keep(float* a, float v, uint64_t pol) {
    asm volatile("st.global.cg.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(a), "f"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ float ld_stream(const float* a, uint64_t pol) {
    float v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
    return v;
}


// Predicated store (no branch around it), so that the rows of a batch stay
// in one basic block and their chains interleave.
__device__ __forceinline__ void st_keep_if(float* a, float v, bool p, uint64_t pol) {
    asm volatile(
        "{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t"
        "@q st.global.cg.L2::cache_hint.f32 [%0], %1, %3;\n\t}" ::"l"(a),
        "f"(v), "r"((int)p), "l"(pol)
        : "memory");
}
// Asynchronous 4-byte copy global -> shared (skipped where p is false), and
// its group commit / wait. The copies go through L1 (cp.async of 4 bytes has
// only the .ca form); rows that other CTAs updated in an earlier round are
// visible because every round ends at a grid barrier whose gpu-scope fences
// order those writes before this CTA's later reads.
__device__ __forceinline__ void cp_async4_if(uint32_t dst, const float* src, bool p, uint64_t pol) {
    asm volatile(
        "{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t"
        "@q cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 4, %3;\n\t}" ::"r"(dst),
        "l"(src), "r"((int)p), "l"(pol)
        : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Phase clock of the rounds (thread 0 of each CTA): time in the peak phase,
// waiting at the grid barrier after it, in the update phase and waiting after
// it, summed over the rounds; added to phase[0..3] (sums over CTAs) with the
// slowest CTA's peak and update totals in phase[4], phase[5].
// The clock lives in shared memory (s: time of the last lap, then the four
// sums), so that no register is held for it across the rounds.
struct PhaseClock {
    unsigned long long* s;  // [5] shared
    __device__ __forceinline__ static unsigned long long now() {
        unsigned long long v;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
        return v;
    }
    __device__ __forceinline__ void start() {
        s[0] = now();
        for (int i = 1; i < 5; ++i) s[i] = 0;
    }
    __device__ __forceinline__ void lap(int i) {
        const unsigned long long u = now();
        s[1 + i] += u - s[0];
        s[0] = u;
    }
    __device__ __forceinline__ void flush(unsigned long long* phase) const {
        if (!phase) return;
        for (int i = 0; i < 4; ++i) atomicAdd(phase + i, s[1 + i]);
        atomicMax(phase + 4, s[1]);
        atomicMax(phase + 5, s[3]);
    }
};

__device__ __forceinline__ float cf_of(float b, float nmv) {
    const float r = fmaxf(b, 0.f);
    return __fdiv_rn(__fmul_rn(r, r), nmv);
}

__device__ __forceinline__ unsigned long long pack_key(float cf, int t) {
    return ((unsigned long long)__float_as_uint(cf) << 32) | (unsigned long long)(0xFFFFFFFFu - (unsigned)t);
}


// Running maximum of Cf = fl(fl(r*r) / nm) (r = relu(b)) with the first index
// on ties. The correctly rounded quotient is formed only for candidates:
// a = fl(fl(r*r) * fl(1/nm)) is within 3.01 ulp of it, so a < best*(1 - 8 ulp)
// proves the exact value is below best (checked only while best is a normal
// number, where the relative bounds hold).
struct ColMax {
    float best = -1.f;
    float thr = -1.f;  // rounded-down best * (1 - 2^-21)
    int bi = 0;
    __device__ __forceinline__ void consider(float b, float nmv, float inv, int t) {
        const float r = fmaxf(b, 0.f);
        const float sq = __fmul_rn(r, r);
        if (__fmul_rn(sq, inv) < thr) return;
        const float cf = __fdiv_rn(sq, nmv);
        if (cf > best) {
            best = cf;
            bi = t;
            thr = (cf >= 1e-30f) ? __fmul_rd(cf, 0.99999952316f) : -1.f;
        }
    }
};

// Best Cf of column s over rows [t0, t1), loads issued eight rows at a time.
__device__ __forceinline__ void column_best(const float* __restrict__ B, int64_t ldb, const float* s_nm,
                                            const float* s_inv, int s, int t0, int t1, ColMax& m) {
    const float* bp = B + (int64_t)t0 * ldb + s;
    int t = t0;
    for (; t + 8 <= t1; t += 8, bp += 8 * ldb) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = __ldcg(bp + u * ldb);
#pragma unroll
        for (int u = 0; u < 8; ++u) m.consider(v[u], s_nm[t + u], s_inv[t + u], t + u);
    }
    for (; t < t1; ++t, bp += ldb) m.consider(__ldcg(bp), s_nm[t], s_inv[t], t);
}

// Inclusive warp scan.
__device__ __forceinline__ int warp_inc_scan(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    return v;
}

}  // namespace lss
