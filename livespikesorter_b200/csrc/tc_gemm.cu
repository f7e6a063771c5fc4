// Template scores on the 5th-generation tensor cores (tcgen05), BF16 inputs,
// FP32 accumulation in tensor memory:
//   B[t, s] = sum_kk B0T[s, kk] * U_p[t, kk]      (kk = c*K + k)
// i.e. einsum('ijk,kjl->il', U, conv1d(X, wPCA)) of
// kilosort/template_matching.py:145-146 (cross_correlation_kernel,
// myGPUhelpers.cu:262-336, in the reference).
//
// Shape: samples are the MMA's M (128 per tile, one TMEM lane each), templates
// its N (up to 512 TMEM columns per pass; several passes when T > 512), the
// (channel, component) pairs its K (64 per pipeline stage = one 128-byte
// swizzle row of bf16). Both operands are K-major, loaded by TMA with 128B
// swizzle into a multi-stage shared-memory ring guarded by mbarriers.
//
// Warp roles (192 threads): warp 0 issues TMA, warp 1 owns TMEM and issues the
// MMAs (one elected lane), warps 2-5 drain the accumulator: each thread owns
// one sample (TMEM lane), so the stores of B[t, s] for a fixed template are
// 128-byte coalesced across a warp, and the same thread forms the column
// maximum of Cf = relu(B)^2 / nm over all templates (the matching pursuit's
// first Cfmax / imax), exactly as the rounds' kernel does.
//
// Every mbarrier wait is bounded; on expiry the CTA raises an abort flag,
// drains what it issued and frees its tensor memory before returning.
#include "lss_kernels.cuh"

#include <cuda.h>

#include <algorithm>
#include <cstdio>

namespace lss {
namespace tc {

constexpr int BM = 128;               // samples per tile
constexpr int MAX_NP = 512;           // templates per pass (TMEM columns)
constexpr int SPLIT_W = 128;          // templates per work item in split mode
constexpr int MAPPED_SPLIT_W = 64;    // ... for a re-check of a few mapped rows
constexpr int THREADS = 192;

// Element kinds of the score GEMM (TcOp).
//  BF16  : one MMA term, 128-byte rows (64 bf16 per k-block), 128B swizzle.
//  TF32x3: FP32-class accuracy from tf32 splits x = hi + lo:
//          D += A_hi B_hi + A_hi B_lo + A_lo B_hi, 64-byte rows (16 floats per
//          k-block), 64B swizzle; A and B each have a hi and a lo tile.
//  BF16x3: the same three terms with bf16 splits hi = bf16(x), lo = bf16(x - hi)
//          (about 2^-16 relative per product), 64-byte rows (32 bf16 per
//          k-block), 64B swizzle: half the operand bytes and tensor time of
//          TF32x3.
template <int OP>
struct Kind {
    static constexpr bool SPLIT = OP != TC_BF16;                   // hi and lo tiles per operand
    static constexpr uint32_t ROW = SPLIT ? 64u : 128u;            // bytes per operand row in a stage
    static constexpr int BKE = OP == TC_TF32X3 ? 16 : (OP == TC_BF16X3 ? 32 : 64);  // elements per k-block
    static constexpr int SUB = ROW / 32;                           // 32-byte MMA K steps per k-block
    static constexpr int PARTS = SPLIT ? 2 : 1;
    static constexpr uint32_t A_TILE = BM * ROW;                   // bytes of one A tile
    static constexpr uint32_t ATOM = 8 * ROW;                      // swizzle atom (8 rows)
    static constexpr uint64_t LAYOUT = SPLIT ? 4 : 2;              // UMMA layout: SWIZZLE_64B / SWIZZLE_128B
    static constexpr uint32_t FMT = OP == TC_TF32X3 ? 2u : 1u;     // operand format: TF32 (2) or BF16 (1)
};

struct Args {
    int N, T, Tpad, KB;
    int box_rows, nbox_max, stages, b_rows;
    int nacc;                 // accumulator buffers in TMEM (2 when a pass fits in 256 columns)
    float* Bout;
    int64_t ldb;
    const float* nm;
    float* cfmax;
    int32_t* imax;
    int nt;
    int32_t* status;
    const int32_t* rowmap;    // GEMM row r scores sample rowmap[r / map_rows] * map_rows + r % map_rows (null: r)
    int map_rows;
    const int32_t* count_dev; // rows = min(N, count_dev[0] * map_rows) (null: N)
    const int32_t* rowof;     // template t's score row is Bout row rowof[t] (null: t)
    int ncols;                // samples in the batch (edge columns are the first/last nt)
    float* cf2;               // runner-up Cf of each column (null: not tracked)
    int pass_w;               // templates per pass (<= MAX_NP)
    unsigned long long* keys; // split mode: one work item per (sample tile, pass); column maxima are
                              // combined as atomicMax of (Cf bits << 32 | ~t) (null: a CTA owns whole rows)
    // error bounds (BF16 path): |B - B_fp32| <= eps * un[t] * sqrt(pn2[s]) per score; per column
    // the epilogue writes cf_lo (lower bound of the best template's Cf), cf_hi (upper bound of
    // the column maximum) and, in cf2, the largest upper bound of any other template
    const float* un;
    const float* pn2;
    float eps;
    float* cf_lo;
    float* cf_hi;
    // split mode with error bounds: per (pass, column) partials, finished by
    // k_bounds_finalize: part_keys [npass][ncols] best key of the pass; part
    // [npass][4][ncols] lo of the pass's best, largest hi, its template, second hi
    unsigned long long* part_keys;
    float* part;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait (about 2 s of wall time); false when the CTA is aborting or
// the budget expired (then the abort flag and STATUS_TIMEOUT are raised).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag,
                                          int32_t* status) {
    const uint64_t t0 = globaltimer();
    for (uint32_t i = 0;; ++i) {
        if (mbar_try(bar, parity)) return true;
        if ((i & 255u) == 255u) {
            if (*abort_flag) return false;
            if (globaltimer() - t0 > 2000000000ull) break;
        }
    }
    *abort_flag = 1;
    atomicOr(status, STATUS_TIMEOUT);
    return false;
}

// Wait (bounded, no abort check) for a phase that is known to complete.
__device__ __forceinline__ void mbar_drain(uint32_t bar, uint32_t parity) {
    const uint64_t t0 = globaltimer();
    while (!mbar_try(bar, parity) && globaltimer() - t0 < 2000000000ull) {
    }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// K-major operand with swizzled rows: 8-row atoms of ATOM bytes.
template <int OP>
__device__ __forceinline__ uint64_t operand_desc(uint32_t addr) {
    using KD = Kind<OP>;
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(KD::ATOM >> 4) << 32) |
           ((uint64_t)1 << 46) | (KD::LAYOUT << 61);
}

// Instruction descriptor: F32 accumulator, BF16 (1) or TF32 (2) operands,
// both K-major, M = 128.
template <int OP>
__device__ __forceinline__ uint32_t instr_desc(int n) {
    const uint32_t fmt = Kind<OP>::FMT;
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

template <int OP>
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                    uint32_t accumulate) {
    if constexpr (OP == TC_TF32X3) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
            : "memory");
    }
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void st_keep(float* a, float v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(a), "f"(v), "l"(pol) : "memory");
}

// Running column maximum of Cf with the rounds kernel's exact rule, plus the
// runner-up (to within the 3-ulp reciprocal approximation) when asked for.
struct ColMax {
    float best = -1.f;
    float thr = -1.f;
    float second = -1.f;
    int bi = 0;
    template <bool SECOND>
    __device__ __forceinline__ void consider(float b, float nmv, float inv, int t) {
        const float r = fmaxf(b, 0.f);
        const float sq = __fmul_rn(r, r);
        const float approx = __fmul_rn(sq, inv);
        if (approx < thr) {
            if (SECOND) second = fmaxf(second, approx);
            return;
        }
        const float cf = __fdiv_rn(sq, nmv);
        if (cf > best) {
            if (SECOND) second = fmaxf(second, best);
            best = cf;
            bi = t;
            thr = (cf >= 1e-30f) ? __fmul_rd(cf, 0.99999952316f) : -1.f;
        } else if (SECOND) {
            second = fmaxf(second, cf);
        }
    }
};

// Stage layout: [A_hi | A_lo] [B_hi rows | B_lo rows] (lo tiles only for the split kinds).
template <int OP>
__global__ void __launch_bounds__(THREADS, 1)
    k_score_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmAlo,
               const __grid_constant__ CUtensorMap tmB, const __grid_constant__ CUtensorMap tmBlo, Args a) {
    using KD = Kind<OP>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t a_bytes = KD::PARTS * KD::A_TILE;
    const uint32_t b_part = (uint32_t)a.b_rows * KD::ROW;
    const uint32_t stage_bytes = a_bytes + KD::PARTS * b_part;
    uint8_t* tail = smem + (size_t)a.stages * stage_bytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(tail);  // full[S], empty[S], acc_full[2], acc_empty[2], drain
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * a.stages + 5);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    float* s_nm = reinterpret_cast<float*>(tmem_slot + 4);
    float* s_inv = s_nm + a.Tpad;
    float* s_un = s_inv + a.Tpad;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t s0 = smem_u32(smem);
    auto full_bar = [&](int s) { return smem_u32(bars + s); };
    auto empty_bar = [&](int s) { return smem_u32(bars + a.stages + s); };
    auto accf_bar = [&](int i) { return smem_u32(bars + 2 * a.stages + i); };
    auto acce_bar = [&](int i) { return smem_u32(bars + 2 * a.stages + 2 + i); };
    const uint32_t drain_bar = smem_u32(bars + 2 * a.stages + 4);

    if (threadIdx.x == 0) {
        for (int s = 0; s < a.stages; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(accf_bar(i), 1);
            mbar_init(acce_bar(i), 4);
        }
        mbar_init(drain_bar, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int t = threadIdx.x; t < a.Tpad; t += THREADS) {
        const float v = (t < a.T) ? a.nm[t] : 1.f;
        s_nm[t] = v;
        s_inv[t] = __frcp_rn(v);
        s_un[t] = (a.un && t < a.T) ? a.un[t] : 0.f;
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(MAX_NP)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    const int rows = a.count_dev ? min(a.N, a.count_dev[0] * a.map_rows) : a.N;
    const int ntiles = (rows + BM - 1) / BM;
    const int PW = a.pass_w;
    const int npass = (a.Tpad + PW - 1) / PW;
    const bool split = a.keys != nullptr || a.part_keys != nullptr;
    const int items = split ? ntiles * npass : ntiles;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer
            int stage = 0;
            uint32_t ph = 0;
            uint32_t last_ph[8];
            bool pending[8] = {false, false, false, false, false, false, false, false};
            bool ok = true;
            for (int it = blockIdx.x; it < items && ok; it += gridDim.x) {
                const int tile = split ? it / npass : it;
                const int pb = split ? it % npass : 0, pe = split ? pb + 1 : npass;
                for (int p = pb; p < pe && ok; ++p) {
                    const int np = min(PW, a.Tpad - p * PW);
                    const int nbox = (np + a.box_rows - 1) / a.box_rows;
                    const uint32_t bytes = KD::PARTS * (KD::A_TILE + (uint32_t)nbox * a.box_rows * KD::ROW);
                    for (int kb = 0; kb < a.KB; ++kb) {
                        if (!mbar_wait(empty_bar(stage), ph ^ 1u, abort_flag, a.status)) { ok = false; break; }
                        const uint32_t sa = s0 + stage * stage_bytes;
                        const uint32_t sb = sa + a_bytes;
                        const int kx = kb * KD::BKE;
                        mbar_expect_tx(full_bar(stage), bytes);
                        tma_load_2d(sa, &tmA, kx, tile * BM, full_bar(stage));
                        if (KD::SPLIT) tma_load_2d(sa + KD::A_TILE, &tmAlo, kx, tile * BM, full_bar(stage));
                        for (int bx = 0; bx < nbox; ++bx) {
                            const int row = p * PW + bx * a.box_rows;
                            tma_load_2d(sb + bx * a.box_rows * KD::ROW, &tmB, kx, row, full_bar(stage));
                            if (KD::SPLIT) tma_load_2d(sb + b_part + bx * a.box_rows * KD::ROW, &tmBlo, kx, row, full_bar(stage));
                        }
                        last_ph[stage] = ph;
                        pending[stage] = true;
                        if (++stage == a.stages) { stage = 0; ph ^= 1u; }
                    }
                }
            }
            if (!ok) {
                // aborting: let every load this thread issued land before the CTA exits
                for (int s = 0; s < a.stages; ++s)
                    if (pending[s]) mbar_drain(full_bar(s), last_ph[s]);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer
            int stage = 0;
            uint32_t ph = 0;
            uint32_t acc_ph[2] = {0, 0};
            int acc = 0;
            bool ok = true;
            for (int it = blockIdx.x; it < items && ok; it += gridDim.x) {
                const int pb = split ? it % npass : 0, pe = split ? pb + 1 : npass;
                for (int p = pb; p < pe && ok; ++p) {
                    const int np = min(PW, a.Tpad - p * PW);
                    if (!mbar_wait(acce_bar(acc), acc_ph[acc] ^ 1u, abort_flag, a.status)) { ok = false; break; }
                    fence_after();
                    const uint32_t dcol = tmem + (uint32_t)(acc * 256);
                    for (int kb = 0; kb < a.KB; ++kb) {
                        if (!mbar_wait(full_bar(stage), ph, abort_flag, a.status)) { ok = false; break; }
                        fence_after();
                        const uint32_t sa = s0 + stage * stage_bytes;
                        const uint32_t sb = sa + a_bytes;
#pragma unroll
                        for (int ks = 0; ks < KD::SUB; ++ks) {
                            const uint32_t ko = ks * 32;
                            const uint64_t ad = operand_desc<OP>(sa + ko);
                            for (int c = 0; c < np; c += 256) {
                                const int n = min(256, np - c);
                                const uint32_t idesc = instr_desc<OP>(n);
                                const uint64_t bd = operand_desc<OP>(sb + (uint32_t)c * KD::ROW + ko);
                                const uint32_t acc_on = (kb | ks) != 0;
                                if (KD::SPLIT) {
                                    const uint64_t adl = operand_desc<OP>(sa + KD::A_TILE + ko);
                                    const uint64_t bdl = operand_desc<OP>(sb + b_part + (uint32_t)c * KD::ROW + ko);
                                    mma<OP>(dcol + (uint32_t)c, adl, bd, idesc, acc_on);   // A_lo B_hi
                                    mma<OP>(dcol + (uint32_t)c, ad, bdl, idesc, 1u);      // A_hi B_lo
                                    mma<OP>(dcol + (uint32_t)c, ad, bd, idesc, 1u);       // A_hi B_hi
                                } else {
                                    mma<OP>(dcol + (uint32_t)c, ad, bd, idesc, acc_on);
                                }
                            }
                        }
                        mma_commit(empty_bar(stage));
                        if (++stage == a.stages) { stage = 0; ph ^= 1u; }
                    }
                    if (!ok) break;
                    mma_commit(accf_bar(acc));
                    acc_ph[acc] ^= 1u;
                    acc = (acc + 1) % a.nacc;
                }
            }
            if (!ok) {
                *abort_flag = 1;
                // aborting: wait for every MMA already issued before the memory is released
                mma_commit(drain_bar);
                mbar_drain(drain_bar, 0);
            }
        }
    } else {
        // ---------------- epilogue: warps 2..5, one sample per thread
        const int q = warp & 3;  // TMEM lane quarter this warp may access
        // the score field is re-read by the matching pursuit right after: keep it in L2
        uint64_t pol;
        asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
        const int row = q * 32 + lane;
        uint32_t acc_ph[2] = {0, 0};
        int acc = 0;
        bool ok = true;
        for (int it = blockIdx.x; it < items && ok; it += gridDim.x) {
            const int tile = split ? it / npass : it;
            const int pb = split ? it % npass : 0, pe = split ? pb + 1 : npass;
            const int gr = tile * BM + row;
            const int n = (a.rowmap && gr < rows) ? a.rowmap[gr / a.map_rows] * a.map_rows + gr % a.map_rows : gr;
            const bool valid = gr < rows && n < a.ncols;
            const bool edge = (n < a.nt) || (n >= a.ncols - a.nt);
            const bool bounds = a.un != nullptr;
            const bool second = a.cf2 != nullptr && !bounds;
            ColMax m;
            // bound of this column's score errors per unit template norm
            const float epsp = (bounds && valid) ? __fmul_ru(a.eps, __fsqrt_ru(a.pn2[n])) : 0.f;
            float lo_best = 0.f, hi1 = 0.f, hi2 = 0.f;
            int thi1 = -1;
            for (int p = pb; p < pe; ++p) {
                const int np = min(PW, a.Tpad - p * PW);
                if (!mbar_wait(accf_bar(acc), acc_ph[acc], abort_flag, a.status)) { ok = false; break; }
                fence_after();
                const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * 256);
                for (int c = 0; c < np; c += 16) {
                    uint32_t r[16];
                    tmem_ld16(tbase + (uint32_t)c, r);
                    const int t0 = p * PW + c;
                    if (valid) {
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            const int t = t0 + j;
                            if (t < a.T) {
                                const float v = __uint_as_float(r[j]);
                                const int orow = a.rowof ? __ldg(a.rowof + t) : t;
                                st_keep(a.Bout + (int64_t)orow * a.ldb + n, v, pol);
                                if (!edge) {
                                    if (second) m.consider<true>(v, s_nm[t], s_inv[t], t);
                                    else m.consider<false>(v, s_nm[t], s_inv[t], t);
                                    if (bounds) {
                                        // Cf of the FP32 path lies in [lo, hi]: B within +-dB,
                                        // directed rounding, then a margin for the
                                        // reciprocal and the rounded squares
                                        const float dB = __fmul_ru(epsp, s_un[t]);
                                        const float bh = fmaxf(__fadd_ru(v, dB), 0.f);
                                        const float bl = fmaxf(__fsub_rd(v, dB), 0.f);
                                        const float hi = __fmul_ru(__fmul_ru(__fmul_ru(bh, bh), s_inv[t]), 1.000001f);
                                        const float lo = __fmul_rd(__fmul_rd(__fmul_rd(bl, bl), s_inv[t]), 0.999999f);
                                        if (m.bi == t) lo_best = lo;  // t just became the best
                                        if (hi > hi1) {
                                            hi2 = hi1;
                                            hi1 = hi;
                                            thi1 = t;
                                        } else {
                                            hi2 = fmaxf(hi2, hi);
                                        }
                                    }
                                }
                            }
                        }
                    }
                }
                fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(acce_bar(acc));
                acc_ph[acc] ^= 1u;
                acc = (acc + 1) % a.nacc;
            }
            if (ok && valid) {
                if (split && bounds) {
                    const int64_t nc = a.ncols;
                    const float cf = edge ? 0.f : fmaxf(m.best, 0.f);
                    const uint32_t t = edge ? 0u : (uint32_t)m.bi;
                    a.part_keys[pb * nc + n] = ((unsigned long long)__float_as_uint(cf) << 32) | (unsigned long long)(~t);
                    a.part[(pb * 4 + 0) * nc + n] = edge ? 0.f : lo_best;
                    a.part[(pb * 4 + 1) * nc + n] = edge ? 0.f : hi1;
                    a.part[(pb * 4 + 2) * nc + n] = __int_as_float(edge ? -1 : thi1);
                    a.part[(pb * 4 + 3) * nc + n] = edge ? 0.f : hi2;
                } else if (split) {
                    const float cf = edge ? 0.f : fmaxf(m.best, 0.f);
                    const uint32_t t = edge ? 0u : (uint32_t)m.bi;
                    atomicMax(a.keys + n, ((unsigned long long)__float_as_uint(cf) << 32) | (unsigned long long)(~t));
                } else {
                    a.cfmax[n] = edge ? 0.f : m.best;
                    a.imax[n] = edge ? 0 : m.bi;
                    if (second) a.cf2[n] = edge ? 0.f : m.second;
                    if (bounds) {
                        a.cf2[n] = edge ? 0.f : ((thi1 == m.bi) ? hi2 : hi1);
                        a.cf_lo[n] = edge ? 0.f : lo_best;
                        a.cf_hi[n] = edge ? 0.f : hi1;
                    }
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(MAX_NP) : "memory");
    }
}

// Split mode: column maxima from the combined keys (the keys are left for the
// next user to clear).
__global__ void k_keys_to_maxima(const unsigned long long* __restrict__ keys, int N, float* __restrict__ cfmax,
                                 int32_t* __restrict__ imax) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const unsigned long long k = keys[n];
    cfmax[n] = __uint_as_float((uint32_t)(k >> 32));
    imax[n] = (int32_t)(~(uint32_t)k);
}

// Split mode with error bounds: per column, the passes' partials combined into
// what the unsplit epilogue writes: the best (Cf, first template) over the
// passes, the lower bound of that template's Cf, the largest upper bound and,
// in cf2, the largest upper bound of any other template.
__global__ void k_bounds_finalize(const unsigned long long* __restrict__ part_keys, const float* __restrict__ part,
                                  int npass, int N, int nt, float* __restrict__ cfmax, int32_t* __restrict__ imax,
                                  float* __restrict__ cf_lo, float* __restrict__ cf_hi, float* __restrict__ cf2) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    unsigned long long best = 0ull;
    int pbest = 0;
    for (int p = 0; p < npass; ++p) {
        const unsigned long long k = part_keys[(int64_t)p * N + n];
        if (k > best) {
            best = k;
            pbest = p;
        }
    }
    const int tb = (int)(~(uint32_t)best);
    float hi = 0.f, other = 0.f;
    for (int p = 0; p < npass; ++p) {
        const float h1 = part[((int64_t)p * 4 + 1) * N + n];
        const int t1 = __float_as_int(part[((int64_t)p * 4 + 2) * N + n]);
        const float h2 = part[((int64_t)p * 4 + 3) * N + n];
        hi = fmaxf(hi, h1);
        other = fmaxf(other, (t1 == tb) ? h2 : h1);
    }
    const bool edge = (n < nt) || (n >= N - nt);
    cfmax[n] = edge ? 0.f : __uint_as_float((uint32_t)(best >> 32));
    imax[n] = edge ? 0 : tb;
    cf_lo[n] = edge ? 0.f : part[((int64_t)pbest * 4 + 0) * N + n];
    cf_hi[n] = edge ? 0.f : hi;
    cf2[n] = edge ? 0.f : other;
}

// The same for the mapped columns of a re-check (rowmap, count on the device).
__global__ void k_keys_to_maxima_mapped(const unsigned long long* __restrict__ keys, const int32_t* __restrict__ rowmap,
                                        const int32_t* __restrict__ count_dev, int map_rows, int max_rows,
                                        float* __restrict__ cfmax, int32_t* __restrict__ imax) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= min(max_rows, count_dev[0] * map_rows)) return;
    const int n = rowmap[i / map_rows] * map_rows + i % map_rows;
    const unsigned long long k = keys[n];
    cfmax[n] = __uint_as_float((uint32_t)(k >> 32));
    imax[n] = (int32_t)(~(uint32_t)k);
}

}  // namespace tc

// ---------------------------------------------------------------- host side
typedef CUresult (*PFN_encodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                    const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                    CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_encodeTiled get_encode() {
    static PFN_encodeTiled fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_encodeTiled>(p);
    }
    return fn;
}

// 2-D tensor [rows, cols] (cols contiguous, row pitch in elements) of the
// kind's element type, box [box_rows, one swizzled row]: 128 B rows with 128B
// swizzle (BF16) or 64 B rows with 64B swizzle (TF32x3, BF16x3).
static bool make_map(CUtensorMap* m, const void* base, int64_t rows, int64_t cols, int64_t pitch, int box_rows,
                     int op) {
    PFN_encodeTiled enc = get_encode();
    if (!enc) return false;
    const bool f32 = op == TC_TF32X3;
    const int64_t esz = f32 ? 4 : 2;
    if ((reinterpret_cast<uintptr_t>(base) & 15) || ((pitch * esz) & 15) || box_rows < 8 || box_rows > 256 ||
        (box_rows & 7))
        return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(pitch * esz)};
    cuuint32_t box[2] = {(cuuint32_t)(op == TC_BF16 ? 64 : 64 / esz), (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1u, 1u};
    return enc(m, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base),
               dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               op == TC_BF16 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

TcPlan tc_plan(int T, int op, int pass_w) {
    TcPlan p{};
    p.Tpad = (T + 15) / 16 * 16;
    p.pass_w = std::min(pass_w, tc::MAX_NP);
    const int np0 = std::min(p.pass_w, p.Tpad);
    p.box_rows = (np0 <= 256) ? np0 : ((np0 + 1) / 2 + 7) / 8 * 8;
    int b_rows = 0;  // largest pass rounded up to whole boxes
    for (int off = 0; off < p.Tpad; off += p.pass_w) {
        const int np = std::min(p.pass_w, p.Tpad - off);
        b_rows = std::max(b_rows, (np + p.box_rows - 1) / p.box_rows * p.box_rows);
    }
    p.b_rows = b_rows;
    const size_t row = op == TC_BF16 ? 128 : 64, parts = op == TC_BF16 ? 1 : 2;
    const size_t stage = parts * (tc::BM * row + (size_t)b_rows * row);
    const size_t tail = 8 * (2 * 4 + 5) + 16 + 12 * (size_t)p.Tpad;
    const size_t budget = 227 * 1024 - 1024 - tail;
    p.stages = (int)std::min<size_t>(4, budget / stage);
    p.nacc = (np0 <= 256) ? 2 : 1;
    p.smem = 1024 + (size_t)p.stages * stage + 8 * (2 * p.stages + 5) + 16 + 12 * (size_t)p.Tpad;
    p.kblock = op == TC_TF32X3 ? 16 : (op == TC_BF16X3 ? 32 : 64);
    return p;
}

template <int OP>
static cudaError_t launch_tc(const void* A, const void* Alo, int64_t ldk, int N, const void* Bm, const void* Blo, int T,
                             int CKpad, const float* nm, float* Bout, int64_t ldb, float* cfmax, int32_t* imax, int nt,
                             int32_t* status, int grid, cudaStream_t s, const TcExtra& ex) {
    // Few sample tiles (short streaming batches): one work item per (tile,
    // pass of SPLIT_W templates) so that more SMs share the templates; the
    // column maxima are then combined through 64-bit keys.
    // A re-check of mapped rows (rowmap, count on the device) is usually one
    // or two tiles: its templates are split the same way, in narrower passes.
    const int ntiles = (N + tc::BM - 1) / tc::BM;
    // templates in passes of at most 256 TMEM columns (equal widths): two
    // accumulators alternate, so one pass's epilogue drains while the next
    // pass's MMAs run, and the smaller stages leave room for four of them
    const int tpad = (T + 15) / 16 * 16;
    const int npass = (tpad + 255) / 256;
    const int even_w = ((tpad + npass - 1) / npass + 15) / 16 * 16;
    const bool split_map = ex.keys && ex.rowmap && ex.count_dev && !ex.cf2 && !ex.un && T > tc::MAPPED_SPLIT_W;
    const bool split_short = ex.keys && !ex.cf2 && !ex.un && !ex.rowmap && 2 * ntiles < grid && T > tc::SPLIT_W;
    // Several passes over a full batch: one work item per (tile, pass), so that
    // a tile's passes run on consecutive CTAs at the same time and its sample
    // operand is read from DRAM once (tile by tile the passes would stream it
    // once per pass, and 148 tiles in flight do not fit the L2); column maxima
    // through keys, or per-pass partials for the error bounds.
    const bool bounds_part = ex.un && ex.part_keys && ex.part && (int64_t)npass * N <= ex.part_cap;
    const bool split_pass = !split_map && !split_short && !ex.rowmap && npass > 1 &&
                            ((ex.keys && !ex.cf2 && !ex.un) || bounds_part);
    const bool split = split_map || split_short || split_pass;
    const bool part_mode = split_pass && bounds_part;
    const TcPlan p = tc_plan(T, OP, split_map ? tc::MAPPED_SPLIT_W : (split_short ? tc::SPLIT_W : even_w));
    if (p.stages < 2 || CKpad % p.kblock) return cudaErrorInvalidValue;
    CUtensorMap ma, malo, mb, mblo;
    if (!make_map(&ma, A, N, CKpad, ldk, tc::BM, OP) || !make_map(&mb, Bm, p.Tpad, CKpad, CKpad, p.box_rows, OP))
        return cudaErrorInvalidValue;
    if (tc::Kind<OP>::SPLIT) {
        if (!make_map(&malo, Alo, N, CKpad, ldk, tc::BM, OP) ||
            !make_map(&mblo, Blo, p.Tpad, CKpad, CKpad, p.box_rows, OP))
            return cudaErrorInvalidValue;
    } else {
        malo = ma;
        mblo = mb;
    }
    tc::Args a{};
    a.N = N;
    a.T = T;
    a.Tpad = p.Tpad;
    a.KB = CKpad / p.kblock;
    a.box_rows = p.box_rows;
    a.stages = p.stages;
    a.b_rows = p.b_rows;
    a.nacc = p.nacc;
    a.Bout = Bout;
    a.ldb = ldb;
    a.nm = nm;
    a.cfmax = cfmax;
    a.imax = imax;
    a.nt = nt;
    a.status = status;
    a.rowmap = ex.rowmap;
    a.map_rows = ex.map_rows;
    a.count_dev = ex.count_dev;
    a.rowof = ex.rowof;
    a.ncols = ex.rowmap ? ex.ncols : N;
    a.cf2 = ex.cf2;
    a.pass_w = p.pass_w;
    a.keys = (split && !part_mode) ? ex.keys : nullptr;
    a.part_keys = part_mode ? ex.part_keys : nullptr;
    a.part = part_mode ? ex.part : nullptr;
    a.un = (split && !part_mode) ? nullptr : ex.un;
    a.pn2 = ex.pn2;
    a.eps = ex.eps;
    a.cf_lo = ex.cf_lo;
    a.cf_hi = ex.cf_hi;
    if (a.un && (!a.pn2 || !a.cf2 || !a.cf_lo || !a.cf_hi || ex.rowmap)) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(tc::k_score_tc<OP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem);
    if (e != cudaSuccess) return e;
    const int items = split ? ntiles * ((p.Tpad + p.pass_w - 1) / p.pass_w) : ntiles;
    if (split && !part_mode) {
        e = cudaMemsetAsync(ex.keys, 0, (size_t)(split_map ? ex.ncols : N) * sizeof(unsigned long long), s);
        if (e != cudaSuccess) return e;
    }
    tc::k_score_tc<OP><<<std::min(grid, items), tc::THREADS, p.smem, s>>>(ma, malo, mb, mblo, a);
    if (part_mode)
        tc::k_bounds_finalize<<<(N + 255) / 256, 256, 0, s>>>(ex.part_keys, ex.part, (p.Tpad + p.pass_w - 1) / p.pass_w, N,
                                                              nt, cfmax, imax, ex.cf_lo, ex.cf_hi, ex.cf2);
    else if (split_map)
        tc::k_keys_to_maxima_mapped<<<(N + 255) / 256, 256, 0, s>>>(ex.keys, ex.rowmap, ex.count_dev, ex.map_rows, N,
                                                                    cfmax, imax);
    else if (split)
        tc::k_keys_to_maxima<<<(N + 255) / 256, 256, 0, s>>>(ex.keys, N, cfmax, imax);
    return cudaGetLastError();
}

cudaError_t launch_score_tc(const __nv_bfloat16* B0T, int64_t ldk, int N, const __nv_bfloat16* Up, int T, int CKpad,
                            const float* nm, float* Bout, int64_t ldb, float* cfmax, int32_t* imax, int nt,
                            int32_t* status, int grid, cudaStream_t s, const TcExtra& ex) {
    return launch_tc<TC_BF16>(B0T, nullptr, ldk, N, Up, nullptr, T, CKpad, nm, Bout, ldb, cfmax, imax, nt, status, grid,
                              s, ex);
}

cudaError_t launch_score_tc_bf16x3(const __nv_bfloat16* B0T_hi, const __nv_bfloat16* B0T_lo, int64_t ldk, int N,
                                   const __nv_bfloat16* Up_hi, const __nv_bfloat16* Up_lo, int T, int CKpad,
                                   const float* nm, float* Bout, int64_t ldb, float* cfmax, int32_t* imax, int nt,
                                   int32_t* status, int grid, cudaStream_t s, const TcExtra& ex) {
    return launch_tc<TC_BF16X3>(B0T_hi, B0T_lo, ldk, N, Up_hi, Up_lo, T, CKpad, nm, Bout, ldb, cfmax, imax, nt, status,
                                grid, s, ex);
}

cudaError_t launch_score_tc_tf32x3(const float* B0T_hi, const float* B0T_lo, int64_t ldk, int N, const float* Up_hi,
                                   const float* Up_lo, int T, int CKpad, const float* nm, float* Bout, int64_t ldb,
                                   float* cfmax, int32_t* imax, int nt, int32_t* status, int grid, cudaStream_t s,
                                   const TcExtra& ex) {
    return launch_tc<TC_TF32X3>(B0T_hi, B0T_lo, ldk, N, Up_hi, Up_lo, T, CKpad, nm, Bout, ldb, cfmax, imax, nt, status,
                                grid, s, ex);
}

}  // namespace lss
