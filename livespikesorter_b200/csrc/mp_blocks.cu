// Greedy matching pursuit that skips template-row blocks whose update is an
// exact no-op. Same rounds, same arithmetic and the same spikes, amplitudes
// and final score field as k_mp (mp.cu) and Kilosort's round loop
// (kilosort/template_matching.py:157-198, LiveSpikeSorter's
// kilosortMatchingPursuit, OnlineSpikesV2.cu:873-971).
//
// Why most of the update can be skipped. A spike (x, y, a) changes score
// B[t, s] to fl(B - fl(a * ctc[t, y, s - x + nt])). For |B| in [2^e, 2^(e+1))
// the neighbouring floats are at least 2^(e-24) away, so any |d| < 2^(e-25)
// leaves fl(B - d) == B bit for bit. Templates far apart on the probe have
// cross-correlations many orders of magnitude below the scores they would
// change (on a 384-channel probe with 800 templates, two thirds of the
// (spike chunk, row block) updates are such no-ops), so:
//   * template rows are grouped into blocks of MPB_ROWS templates that lie
//     close together on the probe (perm: templates ordered by the centre of
//     mass of their channel energy);
//   * per block and column the kernel keeps bmin = min over the block's rows
//     of |B| and bkey = max over the rows of (Cf bits << 32 | ~t), exact for
//     the current field;
//   * for a (spike segment, 32-column chunk) and a block, row r needs spike
//     e's term only if fl(|a_e| * cmaxr[y_e][t_r]) >= thr, thr being a quarter
//     ulp of the smallest bmin over the warp's columns (cmaxr = max over lags
//     of |ctc|); a block where no row needs a term is skipped (its scores,
//     bmin and bkey are provably unchanged); in a processed block a row's
//     term is applied where its bound says it may change the score, and a
//     row's second term also wherever its first was applied (the bound was
//     taken on the field before the first term);
//   * the peak phase takes each column's maximum over the block keys.
// Everything that is computed is computed exactly as in k_mp: single-rounded
// products and differences (__fmul_rn / __fsub_rn), Cf = fl(fl(r*r)/nm), the
// largest Cf with the smallest template index on ties (torch.max), the two
// interleaved passes per round (last even spike's term, then the last odd
// spike's, per element).
//
// Score rows are kept in probe order (row r holds template perm[r]; the score
// GEMM writes them so, and ctc comes as a copy with each spike template's
// rows in that order), so a block's rows are contiguous.
//
// Round structure and bounded grid barriers follow k_mp: the peak phase owns
// W consecutive columns per CTA; the update phase prefix-sums the per-CTA
// peak counts for the round's time order. The update then runs in two steps
// split by a grid barrier: the decisions for every (spike segment, 32-column
// chunk, group of blocks) item, an equal range of items per warp, append the
// blocks to process to their CTA's list; then every CTA takes an equal range
// of all lists' entries, its warps take them one at a time from a shared
// counter, and stream their rows through a ring of stages in shared memory
// filled by asynchronous copies a few batches ahead. Every wait
// is bounded (STATUS_TIMEOUT).
#include "lss_kernels.cuh"
#include "mp_common.cuh"

#include <algorithm>
#include <cfloat>
#include <climits>

namespace lss {

constexpr int MPB_THREADS = 512;
constexpr int MPB_MAX_GRID = 1024;
constexpr int MPB_GROUP = 4;  // row blocks per update work item
constexpr int MPB_SPK = 3;    // spikes of a chunk's list that get row masks
constexpr int WPB = MPB_THREADS / 32;  // warps per CTA
constexpr int BPB = MPB_ROWS / 8;     // 8-row batches per block
static_assert(MPB_SPK == 3, "list entries hold three spikes");
constexpr unsigned FULL = 0xffffffffu;

// 2^(e - 25) for v in [2^e, 2^(e+1)) (v >= 0): any |d| below it leaves
// fl(v' - d) == v' for every v' with |v'| >= v. Zero when v is zero,
// subnormal, tiny, infinite or NaN (nothing is then skipped).
__device__ __forceinline__ float quarter_ulp(float v) {
    const unsigned e = (__float_as_uint(v) >> 23) & 0xFFu;
    return (e > 25u && e < 255u) ? __uint_as_float((e - 25u) << 23) : 0.f;
}

// Running max of Cf over score rows in probe order (row r holds template
// perm[r]): larger Cf first, smaller template index on ties (torch.max's
// first index). The correctly rounded quotient is formed only for candidates
// (see ColMax in mp_common.cuh).
struct ColMaxRows {
    float best = -1.f;
    float thr = -1.f;
    int br = -1;
    __device__ __forceinline__ void consider(float b, float nmv, float inv, int r, const int* perm) {
        const float x = fmaxf(b, 0.f);
        const float sq = __fmul_rn(x, x);
        if (__fmul_rn(sq, inv) < thr) return;
        const float cf = __fdiv_rn(sq, nmv);
        if (cf > best || (cf == best && perm[r] < perm[br])) {
            best = cf;
            br = r;
            thr = (cf >= 1e-30f) ? __fmul_rd(cf, 0.99999952316f) : -1.f;
        }
    }
    __device__ __forceinline__ unsigned long long key(const int* perm) const {
        return pack_key(best, br >= 0 ? perm[br] : 0);
    }
};

template <int NST>
__global__ void __launch_bounds__(MPB_THREADS, 1) k_mp_blocks(MPArgs a) {
    extern __shared__ float smem[];
    __shared__ int s_pref[MPB_MAX_GRID + 1];
    __shared__ int s_wcnt[MPB_THREADS / 32];
    __shared__ int s_cnt, s_total, s_ecnt, s_enext;

    const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int NW = G * WPB, gw = b * WPB + warp;  // warps of the grid, this warp's rank
    const int N = a.N, T = a.T, nt = a.nt, L2 = 2 * nt + 1, nb = a.nb;
    const int W = a.cols_per_blk;
    const int lo = min(N, b * W), hi = min(N, lo + W);
    const int64_t ldk = a.ldk, ldb = a.ldb;
    const int ldb_i = (int)a.ldb;  // < 2^31 (checked at launch): row offsets as one 32x32->64 multiply-add

    float* vals = smem;                                       // [W + 2nt]
    int* ivals = reinterpret_cast<int*>(smem + W + 2 * nt);  // [W]
    // score rows are in probe order: row r holds template perm[r], template t
    // is row s_rowof[t]; nm and 1/nm by row
    float* s_nm = smem + 2 * W + 2 * nt;                      // [T] by row
    float* s_inv = s_nm + T;                                  // [T] by row
    int* s_perm = reinterpret_cast<int*>(s_inv + T);          // [nb * MPB_ROWS]
    int* s_rowof = s_perm + nb * MPB_ROWS;                    // [T]
    // per warp: NST stages of 3 x 8 rows x 32 columns (16-byte aligned)
    float* ring = smem + ((2 * W + 2 * nt + 2 * T + nb * MPB_ROWS + T + 3) & ~3);
    for (int i = tid; i < nb * MPB_ROWS; i += MPB_THREADS) {
        const int t = __ldg(a.perm + i);
        s_perm[i] = t;
        if (i < T) {
            const float v = __ldg(a.nm + t);
            s_nm[i] = v;
            s_inv[i] = __frcp_rn(v);
            s_rowof[t] = i;
        }
    }
    __syncthreads();
    const uint64_t pk = policy_keep(), ps = policy_stream();

    // ---- block keys and minima of the owned columns for the initial field
    {
        const int ncol = hi - lo;
        for (int w = tid; w < ncol * nb; w += MPB_THREADS) {
            const int bb = w / ncol, s = lo + (w - bb * ncol);
            const int r0 = bb * MPB_ROWS, nr = min(MPB_ROWS, T - r0);
            ColMaxRows m;
            float mn = INFINITY;
            for (int r = 0; r < nr; r += 16) {
                float v[16];
#pragma unroll
                for (int u = 0; u < 16; ++u)
                    v[u] = (r + u < nr) ? ld_keep(a.B + (int64_t)(r0 + r + u) * ldb + s, pk) : 0.f;
#pragma unroll
                for (int u = 0; u < 16; ++u)
                    if (r + u < nr) {
                        mn = fminf(mn, fabsf(v[u]));
                        m.consider(v[u], s_nm[r0 + r + u], s_inv[r0 + r + u], r0 + r + u, s_perm);
                    }
            }
            a.bkey[bb * ldk + s] = m.key(s_perm);
            a.bmin[bb * ldk + s] = mn;
        }
    }
    if (!grid_sync(a.bar, a.status)) return;
    __shared__ unsigned long long s_clk[5];
    PhaseClock clk{s_clk};
    if (tid == 0) clk.start();

    int base = 0;
    int r = 0;
    int n_items = 0, n_proc = 0;  // per warp, lane 0: update work items seen and processed
    for (; r < a.max_rounds; ++r) {
        // ---- P: column maxima from the block keys, pooled window, peaks
        const int nv = (hi - lo) + 2 * nt;
        for (int p = tid; p < nv; p += MPB_THREADS) {
            const int s = lo - nt + p;
            float v = -INFINITY;
            if (s >= 0 && s < N) {
                const bool own = (s >= lo && s < hi);
                if (s < nt || s >= N - nt) {
                    v = 0.f;  // Cf[:, :nt] = Cf[:, -nt:] = 0
                    if (own) ivals[s - lo] = 0;
                } else {
                    // the block keys of the column, 32 loads in flight at a time
                    unsigned long long k = 0ull;
                    for (int b0 = 0; b0 < nb; b0 += 32) {
                        unsigned long long kk[32];
#pragma unroll
                        for (int u = 0; u < 32; ++u) kk[u] = (b0 + u < nb) ? __ldcg(a.bkey + (b0 + u) * ldk + s) : 0ull;
#pragma unroll
                        for (int u = 0; u < 32; ++u) k = max(k, kk[u]);
                    }
                    v = __uint_as_float((unsigned)(k >> 32));
                    if (own) ivals[s - lo] = (int)(0xFFFFFFFFu - (unsigned)(k & 0xFFFFFFFFull));
                }
            }
            vals[p] = v;
        }
        if (tid == 0) {
            s_cnt = 0;
            s_ecnt = 0;
        }
        __syncthreads();
        for (int c0 = lo; c0 < hi; c0 += MPB_THREADS) {
            const int s = c0 + tid;
            bool flag = false;
            if (s < hi) {
                const int p = s - lo + nt;
                float cm = vals[p - nt];
                for (int d = -nt + 1; d <= nt; ++d) cm = fmaxf(cm, vals[p + d]);
                flag = (cm > a.th2) && (fabsf(__fsub_rn(cm, vals[p])) < 1e-9f);
            }
            const unsigned bal = __ballot_sync(FULL, flag);
            if (lane == 0) s_wcnt[warp] = __popc(bal);
            __syncthreads();
            if (warp == 0) {
                const int c = (lane < MPB_THREADS / 32) ? s_wcnt[lane] : 0;
                const int inc = warp_inc_scan(c, lane);
                if (lane < MPB_THREADS / 32) s_wcnt[lane] = inc - c;
                if (lane == MPB_THREADS / 32 - 1) s_total = inc;
            }
            __syncthreads();
            if (flag) {
                const int k = s_cnt + s_wcnt[warp] + __popc(bal & ((1u << lane) - 1u));
                const int y = ivals[s - lo];
                a.blk_x[lo + k] = s;
                a.blk_y[lo + k] = y;
                const int ry = s_rowof[y];
                a.blk_amp[lo + k] = __fdiv_rn(__ldcg(a.B + (int64_t)ry * ldb + s), s_nm[ry]);
            }
            __syncthreads();
            if (tid == 0) s_cnt += s_total;
        }
        __syncthreads();
        if (tid == 0) a.blk_cnt[b] = s_cnt;
        if (tid == 0) clk.lap(0);
        if (!grid_sync(a.bar, a.status)) return;
        if (tid == 0) clk.lap(1);

        // ---- U: global order of the round's spikes, records, block updates
        // s_pref[c] = sum of cnt[0, c) over the grid's CTAs, s_pref[G] = total
        auto prefix_counts = [&](const int32_t* cnt) {
            int carry = 0;
            for (int c0 = 0; c0 < G; c0 += MPB_THREADS) {
                const int i = c0 + tid;
                const int c = (i < G) ? __ldcg(cnt + i) : 0;
                const int inc = warp_inc_scan(c, lane);
                if (lane == 31) s_wcnt[warp] = inc;
                __syncthreads();
                if (warp == 0) {
                    const int wc = (lane < WPB) ? s_wcnt[lane] : 0;
                    const int winc = warp_inc_scan(wc, lane);
                    if (lane < WPB) s_wcnt[lane] = winc - wc;
                    if (lane == WPB - 1) s_total = winc;
                }
                __syncthreads();
                if (i < G) s_pref[i] = carry + s_wcnt[warp] + inc - c;
                carry += s_total;
                __syncthreads();
            }
            if (tid == 0) s_pref[G] = carry;
            __syncthreads();
        };
        prefix_counts(a.blk_cnt);
        const int total = s_pref[G];
        if (total == 0) break;
        if (base + total > a.capacity) {
            if (tid == 0) atomicOr(a.status, STATUS_CAPACITY);
            break;
        }
        const int nch = (L2 + 31) / 32;
        const int ngr = (nb + MPB_GROUP - 1) / MPB_GROUP;
        const int per_spike = nch * ngr;
        const int items = total * per_spike;
        {
            const int cnt = s_pref[b + 1] - s_pref[b];
            for (int k = tid; k < cnt; k += MPB_THREADS) {
                const int i = base + s_pref[b] + k;
                a.sp_x[i] = __ldcg(a.blk_x + lo + k);
                a.sp_y[i] = __ldcg(a.blk_y + lo + k);
                a.sp_amp[i] = __ldcg(a.blk_amp + lo + k);
                if (a.sp_round) a.sp_round[i] = r;
            }
            if (b == 0 && tid == 0) a.round_start[r] = base;
        }
        // Work items (spike q, chunk ch, group g): the columns of spike q's
        // segment [max(x_q - nt, x_{q-1} + nt + 1), x_q + nt], 32 at a time
        // (lane = column), and the row blocks g*MPB_GROUP.. of the group; an
        // equal range of consecutive items per warp of the grid. An item's
        // decisions name the blocks to process; in list mode each becomes an
        // entry of the CTA's list and the lists are processed after a grid
        // barrier, an equal share of all entries per warp (decisions take one
        // round trip per item, a processed block four batches of rows, so
        // separating them balances both); otherwise the item's blocks are
        // processed where they are decided.
        const bool use_list =
            a.ment != nullptr && (int64_t)((items + NW - 1) / NW) * WPB * MPB_GROUP <= (int64_t)a.ment_cap;
        {
            // lane L holds spike q - 1 + L of the round
            auto fetch = [&](int q2, int& fx, int& fy, float& fa) {
                const int j = q2 - 1 + lane;
                fx = INT_MAX;
                fy = 0;
                fa = 0.f;
                if (j >= 0 && j < total) {
                    int lo2 = 0, hi2 = G;  // region c with s_pref[c] <= j < s_pref[c+1]
                    while (hi2 - lo2 > 1) {
                        const int m = (lo2 + hi2) >> 1;
                        if (s_pref[m] <= j) lo2 = m; else hi2 = m;
                    }
                    const int idx = lo2 * W + (j - s_pref[lo2]);
                    fx = __ldcg(a.blk_x + idx);
                    fy = __ldcg(a.blk_y + idx);
                    fa = __ldcg(a.blk_amp + idx);
                }
            };
            int x = INT_MAX, y = 0, cur_q = -1;
            float amp = 0.f;
            const int it_hi = (int)((int64_t)items * (gw + 1) / NW);
            for (int it = (int)((int64_t)items * gw / NW); it < it_hi; ++it) {
                const int q = it / per_spike, rem = it - q * per_spike, ch = rem / ngr, g = rem - ch * ngr;
                if (q != cur_q) {
                    cur_q = q;
                    fetch(q, x, y, amp);
                }
                const int xi = __shfl_sync(FULL, x, 1);
                const int xprev = __shfl_sync(FULL, x, 0);
                const bool ok = lane >= 1 && (q - 1 + lane) < total && x <= xi + 2 * nt;
                const int nl = __popc(__ballot_sync(FULL, ok));
                if (lane == 0 && ch == 0 && g == 0 && nl == MP_LIST && q + MP_LIST < total)
                    atomicOr(a.status, STATUS_LIST);
                const int lo_own = max(max(xi - nt, (q > 0 ? xprev : INT_MIN / 2) + nt + 1), 0);
                const int hi_own = min(xi + nt, N - 1);
                if (lo_own + ch * 32 > hi_own) continue;  // warp-uniform: nothing owned in this chunk
                const int s = lo_own + ch * 32 + lane;
                const bool active = s <= hi_own;
                // last even and last odd spike of the list whose window covers s
                int e0 = -1, e1 = -1;
                for (int e = 0; e < nl; ++e) {
                    const int ex = __shfl_sync(FULL, x, e + 1);
                    if (active && ex <= s + nt) {
                        if ((q + e) & 1) e1 = e; else e0 = e;
                    }
                }
                // the first MPB_SPK spikes of the list (nearly always the only ones
                // a chunk meets): template and |amplitude| for the row masks
                int ye[MPB_SPK];
                float fae[MPB_SPK];
#pragma unroll
                for (int e = 0; e < MPB_SPK; ++e) {
                    ye[e] = __shfl_sync(FULL, y, e + 1);
                    fae[e] = fabsf(__shfl_sync(FULL, amp, e + 1));
                }
                // ---- decisions for the group's blocks, all loads in one round trip.
                // thr: a quarter ulp of the smallest |B| the block holds in any of
                // the warp's columns; row r of block b needs spike e's term only if
                // fl(|a_e| * max_l |ctc[r, y_e, l]|) >= thr (otherwise the term
                // leaves every score of the row bit for bit unchanged).
                const int bg0 = g * MPB_GROUP, nbg = min(MPB_GROUP, nb - bg0);
                float bmv[MPB_GROUP], cmv[MPB_GROUP][MPB_SPK];
#pragma unroll
                for (int j = 0; j < MPB_GROUP; ++j) {
                    const int bb = bg0 + j;
                    const int tr = (j < nbg && bb * MPB_ROWS + lane < T) ? bb * MPB_ROWS + lane : -1;
                    bmv[j] = (j < nbg && active) ? __ldcg(a.bmin + bb * ldk + s) : 0.f;
#pragma unroll
                    for (int e = 0; e < MPB_SPK; ++e)
                        cmv[j][e] = (tr >= 0 && e < nl) ? __ldg(a.cmaxr + (int64_t)ye[e] * T + tr) : 0.f;
                }
                // me[j][e]: the rows of block j that need spike e's term (lane =
                // row in the ballot); per column, the rows that need its even term
                // (m0) and its odd term (m1); bit j of procm: block j is processed
                unsigned me[MPB_GROUP][MPB_SPK];
                auto masks = [&](int j, unsigned& m0, unsigned& m1) {
                    m0 = (e0 >= MPB_SPK) ? FULL : 0u;
                    m1 = (e1 >= MPB_SPK) ? FULL : 0u;
#pragma unroll
                    for (int jj = 0; jj < MPB_GROUP; ++jj)
                        if (jj == j) {
#pragma unroll
                            for (int e = 0; e < MPB_SPK; ++e) {
                                if (e0 == e) m0 = me[jj][e];
                                if (e1 == e) m1 = me[jj][e];
                            }
                        }
                    if (e0 < 0) m0 = 0u;
                    // after a term that changes the score the second is always applied
                    m1 = (e1 >= 0) ? (m1 | m0) : 0u;
                };
                unsigned procm = 0u;
#pragma unroll
                for (int j = 0; j < MPB_GROUP; ++j) {
                    const float thr_l = active ? quarter_ulp(bmv[j]) : FLT_MAX;
                    const float thr = __uint_as_float(__reduce_min_sync(FULL, __float_as_uint(thr_l)));
#pragma unroll
                    for (int e = 0; e < MPB_SPK; ++e)
                        me[j][e] = __ballot_sync(FULL, e < nl && !(__fmul_rn(fae[e], cmv[j][e]) < thr));
                    unsigned m0, m1;
                    masks(j, m0, m1);
                    if (j < nbg && __any_sync(FULL, active && (m0 | m1) != 0u)) procm |= 1u << j;
                }
                n_items += nbg;
                n_proc += __popc(procm);
                if (procm == 0u) continue;
                if (use_list && __all_sync(FULL, e0 < MPB_SPK && e1 < MPB_SPK)) {
                    // one entry per processed block: chunk, block, the first
                    // MPB_SPK spikes of the list and their row masks
                    int slot = 0;
                    if (lane == 0) slot = atomicAdd(&s_ecnt, __popc(procm));
                    slot = __shfl_sync(FULL, slot, 0);
                    int xe[MPB_SPK];
                    float ae[MPB_SPK];
#pragma unroll
                    for (int e = 0; e < MPB_SPK; ++e) {
                        xe[e] = __shfl_sync(FULL, x, e + 1);
                        ae[e] = __shfl_sync(FULL, amp, e + 1);
                    }
                    int4* dst = a.ment + ((int64_t)b * a.ment_cap + slot) * 4;
                    int k = 0;
#pragma unroll
                    for (int j = 0; j < MPB_GROUP; ++j) {
                        if (!((procm >> j) & 1u)) continue;
                        int4 w;
                        if (lane == 0)
                            w = make_int4(lo_own + ch * 32, hi_own, bg0 + j, min(nl, MPB_SPK) | ((q & 1) << 8));
                        else if (lane == 1)
                            w = make_int4((int)me[j][0], (int)me[j][1], (int)me[j][2], xe[0]);
                        else if (lane == 2)
                            w = make_int4(xe[1], xe[2], ye[0], ye[1]);
                        else
                            w = make_int4(ye[2], __float_as_int(ae[0]), __float_as_int(ae[1]), __float_as_int(ae[2]));
                        if (lane < 4) __stcg(dst + 4 * k + lane, w);
                        ++k;
                    }
                    continue;
                }
                // not listed (a spike list longer than the entries hold, or lists
                // too short for the round): the processed blocks' rows here, 8 at
                // a time
                const int x0 = __shfl_sync(FULL, x, max(e0, 0) + 1);
                const int y0 = __shfl_sync(FULL, y, max(e0, 0) + 1);
                const float a0 = __shfl_sync(FULL, amp, max(e0, 0) + 1);
                const int x1 = __shfl_sync(FULL, x, max(e1, 0) + 1);
                const int y1 = __shfl_sync(FULL, y, max(e1, 0) + 1);
                const float a1 = __shfl_sync(FULL, amp, max(e1, 0) + 1);
                const float* c0p = a.ctcP + (int64_t)y0 * T * L2 + (s - x0 + nt);
                const float* c1p = a.ctcP + (int64_t)y1 * T * L2 + (s - x1 + nt);
                for (int j = 0; j < nbg; ++j) {
                    if (!((procm >> j) & 1u)) continue;
                    unsigned m0, m1;
                    masks(j, m0, m1);
                    const int bb = bg0 + j, r0 = bb * MPB_ROWS, nr = min(MPB_ROWS, T - r0);
                    ColMaxRows m;
                    float mn = INFINITY;
                    for (int rb = 0; rb < BPB; ++rb) {
                        float v[8], w0[8], w1[8];
#pragma unroll
                        for (int u = 0; u < 8; ++u) {
                            const int rr = rb * 8 + u;
                            const bool ld = active && rr < nr;
                            const int64_t t = r0 + rr;
                            v[u] = ld ? ld_keep(a.B + t * ldb + s, pk) : 0.f;
                            w0[u] = (ld && ((m0 >> rr) & 1u)) ? ld_stream(c0p + t * L2, ps) : 0.f;
                            w1[u] = (ld && ((m1 >> rr) & 1u)) ? ld_stream(c1p + t * L2, ps) : 0.f;
                        }
#pragma unroll
                        for (int u = 0; u < 8; ++u) {
                            const int rr = rb * 8 + u;
                            if (!active || rr >= nr) continue;
                            const int t = r0 + rr;
                            float xv = v[u];
                            if ((m0 >> rr) & 1u) xv = __fsub_rn(xv, __fmul_rn(a0, w0[u]));
                            if ((m1 >> rr) & 1u) xv = __fsub_rn(xv, __fmul_rn(a1, w1[u]));
                            if (__float_as_uint(xv) != __float_as_uint(v[u]))
                                st_keep(a.B + (int64_t)t * ldb + s, xv, pk);
                            mn = fminf(mn, fabsf(xv));
                            m.consider(xv, s_nm[t], s_inv[t], t, s_perm);
                        }
                    }
                    if (active) {
                        a.bkey[bb * ldk + s] = m.key(s_perm);
                        a.bmin[bb * ldk + s] = mn;
                    }
                }
            }
        }
        if (use_list) {
            // ---- the CTAs' lists: an equal range of all entries per warp, their
            // rows fetched NST - 1 batches ahead into this warp's ring in shared
            // memory (asynchronous copies, no registers held for rows in flight)
            __syncthreads();
            if (tid == 0) {
                a.ment_cnt[b] = s_ecnt;
                clk.lap(2);
            }
            if (!grid_sync(a.bar, a.status)) return;
            if (tid == 0) clk.lap(3);
            prefix_counts(a.ment_cnt);
            const int n = s_pref[G];
            // this CTA's equal range of all entries, handed to its warps one
            // entry at a time from a shared counter (each warp starts with one)
            const int c_lo = (int)((int64_t)n * b / G), c_hi = (int)((int64_t)n * (b + 1) / G);
            if (tid == 0) s_enext = c_lo + WPB;
            __syncthreads();
            const int e_first = c_lo + warp;
            if (e_first < c_hi) {
                struct Ent {
                    int4 w0, w1, w2, w3;
                };
                // this lane's column of an entry: its row masks, terms and ctc rows
                struct St {
                    int s, bb;  // s < 0: the lane's column is past the chunk's segment
                    unsigned m0, m1;
                    float a0, a1;
                    const float* c0p;
                    const float* c1p;
                };
                auto ld_ent = [&](int e, Ent& E) {
                    int lo2 = 0, hi2 = G;  // list c with s_pref[c] <= e < s_pref[c+1]
                    while (hi2 - lo2 > 1) {
                        const int m = (lo2 + hi2) >> 1;
                        if (s_pref[m] <= e) lo2 = m; else hi2 = m;
                    }
                    const int4* p = a.ment + ((int64_t)lo2 * a.ment_cap + (e - s_pref[lo2])) * 4;
                    E.w0 = __ldcg(p);
                    E.w1 = __ldcg(p + 1);
                    E.w2 = __ldcg(p + 2);
                    E.w3 = __ldcg(p + 3);
                };
                auto make = [&](const Ent& E, St& S) {
                    const int col = E.w0.x + lane;
                    const bool act = col <= E.w0.y;
                    S.s = act ? col : -1;
                    S.bb = E.w0.z;
                    const int nlq = E.w0.w & 0xFF, qp = (E.w0.w >> 8) & 1;
                    const int xs[MPB_SPK] = {E.w1.w, E.w2.x, E.w2.y};
                    const int ys[MPB_SPK] = {E.w2.z, E.w2.w, E.w3.x};
                    const float as[MPB_SPK] = {__int_as_float(E.w3.y), __int_as_float(E.w3.z), __int_as_float(E.w3.w)};
                    const unsigned ms[MPB_SPK] = {(unsigned)E.w1.x, (unsigned)E.w1.y, (unsigned)E.w1.z};
                    int e0 = -1, e1 = -1;
#pragma unroll
                    for (int e = 0; e < MPB_SPK; ++e)
                        if (e < nlq && act && xs[e] <= col + nt) {
                            if ((qp + e) & 1) e1 = e; else e0 = e;
                        }
                    unsigned m0 = 0u, m1 = 0u;
                    int x0 = xs[0], y0 = ys[0], x1 = xs[0], y1 = ys[0];
                    float a0 = as[0], a1 = as[0];
#pragma unroll
                    for (int e = 0; e < MPB_SPK; ++e) {
                        if (e0 == e) {
                            m0 = ms[e];
                            x0 = xs[e];
                            y0 = ys[e];
                            a0 = as[e];
                        }
                        if (e1 == e) {
                            m1 = ms[e];
                            x1 = xs[e];
                            y1 = ys[e];
                            a1 = as[e];
                        }
                    }
                    S.m0 = m0;
                    S.m1 = (e1 >= 0) ? (m1 | m0) : 0u;
                    S.a0 = a0;
                    S.a1 = a1;
                    S.c0p = a.ctcP + (int64_t)y0 * T * L2 + (col - x0 + nt);
                    S.c1p = a.ctcP + (int64_t)y1 * T * L2 + (col - x1 + nt);
                };
                // this warp's ring of NST stages in shared memory, stage =
                // [B rows | even-term ctc rows | odd-term ctc rows][8][32 lanes]
                const uint32_t ring_s = (uint32_t)__cvta_generic_to_shared(ring + warp * NST * 3 * 8 * 32);
                const float* ring_w = ring + warp * NST * 3 * 8 * 32 + lane;
                auto issue = [&](const St& S, int rb, int stage) {
                    const int r0 = S.bb * MPB_ROWS, nr = min(MPB_ROWS, T - r0);
                    const bool act = S.s >= 0;
                    const uint32_t d = ring_s + (uint32_t)(stage * 3 * 8 * 32 + lane) * 4u;
                    const unsigned m0b = S.m0 >> (rb * 8), m1b = S.m1 >> (rb * 8);
                    const float* bcol = a.B + S.s;
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const bool ld = act && rb * 8 + u < nr;
                        const int t = r0 + rb * 8 + u;
                        cp_async4_if(d + (uint32_t)u * 128u, bcol + (int64_t)t * ldb_i, ld, pk);
                        cp_async4_if(d + (uint32_t)(8 + u) * 128u, S.c0p + (int64_t)t * L2, ld && ((m0b >> u) & 1u), ps);
                        cp_async4_if(d + (uint32_t)(16 + u) * 128u, S.c1p + (int64_t)t * L2, ld && ((m1b >> u) & 1u), ps);
                    }
                };
                Ent En;
                St scur, siss;  // the entry being updated, the entry being fetched
                ld_ent(e_first, En);
                make(En, siss);
                scur = siss;
                int n_ent = 1;  // entries this warp has taken so far
                // flat batch j of the warp's entries into stage j % NST; the
                // fetch runs NST - 1 batches ahead of the update (less than one
                // entry, so at most two entries are live); entering an entry,
                // it takes the next one and loads its words
                static_assert(NST - 1 < BPB, "the fetch may run at most one entry ahead");
                auto fetch_batch = [&](int j) {
                    const int rb = j % BPB;
                    if (rb == 0) {
                        if (j > 0) make(En, siss);
                        int e2 = 0;
                        if (lane == 0) e2 = atomicAdd(&s_enext, 1);
                        e2 = __shfl_sync(FULL, e2, 0);
                        if (e2 < c_hi) {
                            ld_ent(e2, En);
                            ++n_ent;
                        }
                    }
                    issue(siss, rb, j % NST);
                };
#pragma unroll
                for (int j = 0; j < NST - 1; ++j) {
                    if (j < n_ent * BPB) fetch_batch(j);
                    cp_async_commit();
                }
                ColMaxRows m;
                float mn = INFINITY;
                for (int k = 0; k < n_ent * BPB; ++k) {
                    if (k + NST - 1 < n_ent * BPB) fetch_batch(k + NST - 1);
                    cp_async_commit();
                    cp_async_wait<NST - 1>();  // batch k has landed (this lane's own copies)
                    const int rb = k % BPB;
                    if (rb == 0 && k > 0) scur = siss;
                    const float* stg = ring_w + (k % NST) * 3 * 8 * 32;
                    const int r0 = scur.bb * MPB_ROWS, nr = min(MPB_ROWS, T - r0);
                    const bool act = scur.s >= 0;
                    // the eight rows' updates without branches (selects and
                    // predicated stores; rows not fetched are never selected),
                    // then the rare Cf candidates
                    float xs[8], ap[8];
                    const unsigned m0b = scur.m0 >> (rb * 8), m1b = scur.m1 >> (rb * 8);
                    float* bcol = a.B + scur.s;
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const bool okr = act && rb * 8 + u < nr;
                        const int t = r0 + rb * 8 + u;
                        const float v = stg[u * 32], w0 = stg[(8 + u) * 32], w1 = stg[(16 + u) * 32];
                        const float y0 = __fsub_rn(v, __fmul_rn(scur.a0, w0));
                        const float xa = ((m0b >> u) & 1u) ? y0 : v;
                        const float y1 = __fsub_rn(xa, __fmul_rn(scur.a1, w1));
                        const float xv = ((m1b >> u) & 1u) ? y1 : xa;
                        st_keep_if(bcol + (int64_t)t * ldb_i, xv, okr && __float_as_uint(xv) != __float_as_uint(v), pk);
                        mn = okr ? fminf(mn, fabsf(xv)) : mn;
                        const float rl = fmaxf(xv, 0.f);
                        ap[u] = okr ? __fmul_rn(__fmul_rn(rl, rl), s_inv[min(t, T - 1)]) : -INFINITY;
                        xs[u] = xv;
                    }
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const int t = r0 + rb * 8 + u;
                        if (ap[u] >= m.thr) m.consider(xs[u], s_nm[t], s_inv[t], t, s_perm);
                    }
                    if (rb == BPB - 1) {  // the entry's block: its key and minimum in this column
                        if (act) {
                            a.bkey[scur.bb * ldk + scur.s] = m.key(s_perm);
                            a.bmin[scur.bb * ldk + scur.s] = mn;
                        }
                        m = ColMaxRows();
                        mn = INFINITY;
                    }
                }
                cp_async_wait<0>();
            }
        }
        base += total;
        if (tid == 0) clk.lap(2);
        if (!grid_sync(a.bar, a.status)) return;
        if (tid == 0) clk.lap(3);
    }
    if (lane == 0 && n_items) {
        atomicAdd(a.counters + 2, n_proc);
        atomicAdd(a.counters + 3, n_items);
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

int mp_blocks_max_grid(int device) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return std::min(sms, MPB_MAX_GRID);
}

static size_t mpb_smem_bytes(int cols_per_blk, int nt, int T, int nb, int nst) {
    const size_t base = ((size_t)2 * cols_per_blk + 2 * nt + 3 * (size_t)T + (size_t)nb * MPB_ROWS + 3) & ~(size_t)3;
    return sizeof(float) * (base + (size_t)WPB * nst * 3 * 8 * 32);
}

template <int NST>
static cudaError_t launch_nst(const MPArgs& a, int grid, size_t smem, cudaStream_t s) {
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_mp_blocks<NST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(grid);
    lc.blockDim = dim3(MPB_THREADS);
    lc.dynamicSmemBytes = smem;
    lc.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    return cudaLaunchKernelEx(&lc, k_mp_blocks<NST>, a);
}

int64_t mp_blocks_list_entries(int64_t N, int nt, int T, int grid) {
    // the rounds' largest peak count when peaks are nt + 1 apart, its items,
    // the largest share of one CTA, MPB_GROUP entries per item
    const int64_t peaks = (N + nt) / (nt + 1);
    const int64_t items = peaks * ((2 * nt + 1 + 31) / 32) * (((T + MPB_ROWS - 1) / MPB_ROWS + MPB_GROUP - 1) / MPB_GROUP);
    const int64_t nw = (int64_t)std::max(grid, 1) * WPB;
    return (int64_t)std::max(grid, 1) * ((items + nw - 1) / nw) * WPB * MPB_GROUP;
}

cudaError_t launch_mp_blocks(MPArgs a, int grid, cudaStream_t s) {
    if (grid > MPB_MAX_GRID || !a.perm || !a.cmaxr || !a.bkey || !a.bmin || (a.ment && (!a.ment_cnt || a.ment_cap < 0)) ||
        a.nb != (a.T + MPB_ROWS - 1) / MPB_ROWS || a.ldb > INT_MAX || (int64_t)a.T * (2 * a.nt + 1) > INT_MAX)
        return cudaErrorInvalidValue;
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa{};
    e = cudaFuncGetAttributes(&fa, k_mp_blocks<2>);
    if (e != cudaSuccess) return e;
    const size_t room = (size_t)optin - fa.sharedSizeBytes;
    // the deepest ring of fetched rows that fits (4, 3 or 2 stages per warp)
    int nst = 4;
    while (nst > 2 && mpb_smem_bytes(a.cols_per_blk, a.nt, a.T, a.nb, nst) > room) --nst;
    const size_t smem = mpb_smem_bytes(a.cols_per_blk, a.nt, a.T, a.nb, nst);
    if (smem > room) return cudaErrorInvalidValue;
    e = cudaMemsetAsync(a.bar, 0, 2 * sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    if (nst == 4) return launch_nst<4>(a, grid, smem, s);
    if (nst == 3) return launch_nst<3>(a, grid, smem, s);
    return launch_nst<2>(a, grid, smem, s);
}

// ctcQ[y, r, :] = ctcP[y, perm[r], :]: each spike template's cross-correlation
// rows in the score rows' probe order (a warp per row, lags by lane)
__global__ void k_permute_ctc(const float* __restrict__ ctcP, const int32_t* __restrict__ perm, int T, int L2,
                              float* __restrict__ ctcQ) {
    const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= (int64_t)T * T) return;
    const int64_t y = row / T;
    const int r = (int)(row - y * T);
    const float* src = ctcP + (y * T + __ldg(perm + r)) * L2;
    float* dst = ctcQ + row * L2;
    for (int l = lane; l < L2; l += 32) dst[l] = __ldg(src + l);
}

cudaError_t launch_permute_ctc(const float* ctcP, const int32_t* perm, int32_t T, int32_t L2, float* ctcQ,
                               cudaStream_t s) {
    const int64_t rows = (int64_t)T * T;
    k_permute_ctc<<<(unsigned)((rows + 7) / 8), 256, 0, s>>>(ctcP, perm, T, L2, ctcQ);
    return cudaGetLastError();
}

// dst row r = src row perm[r] (N columns each)
__global__ void k_gather_rows(const float* __restrict__ src, int64_t lds, const int32_t* __restrict__ perm,
                              int64_t N, float* __restrict__ dst, int64_t ldd) {
    const int r = blockIdx.y;
    const float* sp = src + (int64_t)__ldg(perm + r) * lds;
    float* dp = dst + (int64_t)r * ldd;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x)
        dp[n] = __ldg(sp + n);
}

cudaError_t launch_gather_rows(const float* src, int64_t lds, const int32_t* perm, int32_t rows, int64_t N,
                               float* dst, int64_t ldd, cudaStream_t s) {
    if (rows <= 0 || N <= 0) return cudaSuccess;
    const unsigned gx = (unsigned)std::min<int64_t>((N + 255) / 256, 64);
    k_gather_rows<<<dim3(gx, (unsigned)rows), 256, 0, s>>>(src, lds, perm, N, dst, ldd);
    return cudaGetLastError();
}

// cmaxr[y, t] = max over lags of |ctcP[y, t, :]| (one warp per row); a NaN
// lag makes the row's maximum infinite, so that nothing touching it is skipped
__global__ void k_ctc_row_max(const float* __restrict__ ctcP, int64_t rows, int L2, float* __restrict__ cmaxr) {
    const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= rows) return;
    const float* p = ctcP + row * L2;
    float m = 0.f;
    for (int l = lane; l < L2; l += 32) {
        const float v = __ldg(p + l);
        m = (v != v) ? INFINITY : fmaxf(m, fabsf(v));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
    if (lane == 0) cmaxr[row] = m;
}

cudaError_t launch_ctc_row_max(const float* ctcP, int32_t T, int32_t L2, float* cmaxr, cudaStream_t s) {
    const int64_t rows = (int64_t)T * T;
    k_ctc_row_max<<<(unsigned)((rows + 7) / 8), 256, 0, s>>>(ctcP, rows, L2, cmaxr);
    return cudaGetLastError();
}

}  // namespace lss
