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
// change (on a 384-channel probe about three quarters of all (row, spike)
// updates are such no-ops), so:
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
//     bmin and bkey are provably unchanged); in a processed block the terms
//     that are no-ops are skipped row by row, the second term only where the
//     first left the score unchanged;
//   * the peak phase takes each column's maximum over the block keys.
// Everything that is computed is computed exactly as in k_mp: single-rounded
// products and differences (__fmul_rn / __fsub_rn), Cf = fl(fl(r*r)/nm), the
// largest Cf with the smallest template index on ties (torch.max), the two
// interleaved passes per round (last even spike's term, then the last odd
// spike's, per element).
//
// Round structure, work split and bounded grid barriers follow k_mp: the peak
// phase owns W consecutive columns per CTA; the update phase prefix-sums the
// per-CTA peak counts for the round's time order; update work items are
// split into per-CTA slices of equal estimated cost (template bands) and
// handed to the CTA's warps through a shared counter, and a warp runs the
// rows of an item's processed blocks through one software pipeline; every
// wait is bounded (STATUS_TIMEOUT).
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
constexpr int MPB_MAX_SPK = 2048;  // spikes per round the cost-balanced split holds (else: equal item counts)
constexpr unsigned FULL = 0xffffffffu;

// 2^(e - 25) for v in [2^e, 2^(e+1)) (v >= 0): any |d| below it leaves
// fl(v' - d) == v' for every v' with |v'| >= v. Zero when v is zero,
// subnormal, tiny, infinite or NaN (nothing is then skipped).
__device__ __forceinline__ float quarter_ulp(float v) {
    const unsigned e = (__float_as_uint(v) >> 23) & 0xFFu;
    return (e > 25u && e < 255u) ? __uint_as_float((e - 25u) << 23) : 0.f;
}

// Running max of Cf over rows visited in any order: larger Cf first, smaller
// template index on ties (torch.max's first index). The correctly rounded
// quotient is formed only for candidates (see ColMax in mp_common.cuh).
struct ColMaxAny {
    float best = -1.f;
    float thr = -1.f;
    int bi = INT_MAX;
    __device__ __forceinline__ void consider(float b, float nmv, float inv, int t) {
        const float r = fmaxf(b, 0.f);
        const float sq = __fmul_rn(r, r);
        if (__fmul_rn(sq, inv) < thr) return;
        const float cf = __fdiv_rn(sq, nmv);
        if (cf > best || (cf == best && t < bi)) {
            best = cf;
            bi = t;
            thr = (cf >= 1e-30f) ? __fmul_rd(cf, 0.99999952316f) : -1.f;
        }
    }
};

__global__ void __launch_bounds__(MPB_THREADS, 1) k_mp_blocks(MPArgs a) {
    extern __shared__ float smem[];
    __shared__ int s_pref[MPB_MAX_GRID + 1];
    __shared__ int s_wcnt[MPB_THREADS / 32];
    __shared__ int s_cnt, s_total, s_next, s_end;

    const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int N = a.N, T = a.T, nt = a.nt, L2 = 2 * nt + 1, nb = a.nb;
    const int W = a.cols_per_blk;
    const int lo = min(N, b * W), hi = min(N, lo + W);
    const int64_t ldk = a.ldk, ldb = a.ldb;

    float* vals = smem;                                       // [W + 2nt]
    int* ivals = reinterpret_cast<int*>(smem + W + 2 * nt);  // [W]
    float* s_nm = smem + 2 * W + 2 * nt;                      // [T]
    float* s_inv = s_nm + T;                                  // [T]
    int* s_perm = reinterpret_cast<int*>(s_inv + T);          // [nb * MPB_ROWS]
    int* s_cost = s_perm + nb * MPB_ROWS;                     // [MPB_MAX_SPK] spike costs, then their prefix
    int* s_band = s_cost + MPB_MAX_SPK;                       // [MPB_MAX_SPK] band lo | hi << 16 per spike
    for (int t = tid; t < T; t += MPB_THREADS) {
        const float v = __ldg(a.nm + t);
        s_nm[t] = v;
        s_inv[t] = __frcp_rn(v);
    }
    for (int i = tid; i < nb * MPB_ROWS; i += MPB_THREADS) s_perm[i] = __ldg(a.perm + i);
    __syncthreads();
    const uint64_t pk = policy_keep(), ps = policy_stream();

    // ---- block keys and minima of the owned columns for the initial field
    {
        const int ncol = hi - lo;
        for (int w = tid; w < ncol * nb; w += MPB_THREADS) {
            const int bb = w / ncol, s = lo + (w - bb * ncol);
            const int r0 = bb * MPB_ROWS, nr = min(MPB_ROWS, T - r0);
            ColMaxAny m;
            float mn = INFINITY;
            for (int r = 0; r < nr; r += 16) {
                float v[16];
#pragma unroll
                for (int u = 0; u < 16; ++u)
                    v[u] = (r + u < nr) ? ld_keep(a.B + (int64_t)s_perm[r0 + r + u] * ldb + s, pk) : 0.f;
#pragma unroll
                for (int u = 0; u < 16; ++u)
                    if (r + u < nr) {
                        const int t = s_perm[r0 + r + u];
                        mn = fminf(mn, fabsf(v[u]));
                        m.consider(v[u], s_nm[t], s_inv[t], t);
                    }
            }
            a.bkey[bb * ldk + s] = pack_key(m.best, m.bi);
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
                    // the block keys of the column, 16 loads in flight at a time
                    unsigned long long k = 0ull;
                    for (int b0 = 0; b0 < nb; b0 += 16) {
                        unsigned long long kk[16];
#pragma unroll
                        for (int u = 0; u < 16; ++u) kk[u] = (b0 + u < nb) ? __ldcg(a.bkey + (b0 + u) * ldk + s) : 0ull;
#pragma unroll
                        for (int u = 0; u < 16; ++u) k = max(k, kk[u]);
                    }
                    v = __uint_as_float((unsigned)(k >> 32));
                    if (own) ivals[s - lo] = (int)(0xFFFFFFFFu - (unsigned)(k & 0xFFFFFFFFull));
                }
            }
            vals[p] = v;
        }
        if (tid == 0) s_cnt = 0;
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
                a.blk_amp[lo + k] = __fdiv_rn(__ldcg(a.B + (int64_t)y * ldb + s), s_nm[y]);
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
        {
            int carry = 0;
            for (int c0 = 0; c0 < G; c0 += MPB_THREADS) {
                const int i = c0 + tid;
                const int c = (i < G) ? __ldcg(a.blk_cnt + i) : 0;
                const int inc = warp_inc_scan(c, lane);
                if (lane == 31) s_wcnt[warp] = inc;
                __syncthreads();
                if (warp == 0) {
                    const int wc = (lane < MPB_THREADS / 32) ? s_wcnt[lane] : 0;
                    const int winc = warp_inc_scan(wc, lane);
                    if (lane < MPB_THREADS / 32) s_wcnt[lane] = winc - wc;
                    if (lane == MPB_THREADS / 32 - 1) s_total = winc;
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
        // ---- this CTA's share of the update items, balanced by estimated cost:
        // an item (spike q, chunk ch, group g) costs 1 (its decisions) plus 4
        // per block of the group inside spike q's template band (the blocks
        // its cross-correlations can reach); every CTA prefix-sums the spikes'
        // costs and takes the items of an equal slice of the total
        if (total <= MPB_MAX_SPK) {
            for (int q = tid; q < total; q += MPB_THREADS) {
                int lo2 = 0, hi2 = G;
                while (hi2 - lo2 > 1) {
                    const int m = (lo2 + hi2) >> 1;
                    if (s_pref[m] <= q) lo2 = m; else hi2 = m;
                }
                const int y = __ldcg(a.blk_y + lo2 * W + (q - s_pref[lo2]));
                const int bl = __ldg(a.band_lo + y), bh = __ldg(a.band_hi + y);
                s_band[q] = (bl & 0xFFFF) | (bh << 16);
                s_cost[q] = nch * (ngr + 4 * max(0, bh - bl + 1));
            }
            __syncthreads();
            // inclusive prefix of s_cost[0, total): 4 consecutive entries per thread
            {
                int v4[4], sum = 0;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int q = 4 * tid + u;
                    v4[u] = q < total ? s_cost[q] : 0;
                    sum += v4[u];
                }
                const int inc = warp_inc_scan(sum, lane);
                if (lane == 31) s_wcnt[warp] = inc;
                __syncthreads();
                if (warp == 0) {
                    const int wc = (lane < MPB_THREADS / 32) ? s_wcnt[lane] : 0;
                    const int winc = warp_inc_scan(wc, lane);
                    if (lane < MPB_THREADS / 32) s_wcnt[lane] = winc - wc;
                }
                __syncthreads();
                int run = s_wcnt[warp] + inc - sum;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int q = 4 * tid + u;
                    run += v4[u];
                    if (q < total) s_cost[q] = run;
                }
            }
            __syncthreads();
            if (tid == 0) {
                const int64_t ctot = s_cost[total - 1];
                // first item whose cumulative cost exceeds c
                auto item_at = [&](int64_t c) -> int {
                    if (c >= ctot) return items;
                    int lo2 = 0, hi2 = total - 1;  // first q with s_cost[q] > c
                    while (lo2 < hi2) {
                        const int m = (lo2 + hi2) >> 1;
                        if (s_cost[m] > c) hi2 = m; else lo2 = m + 1;
                    }
                    int64_t acc = lo2 > 0 ? s_cost[lo2 - 1] : 0;
                    const int bl = s_band[lo2] & 0xFFFF, bh = s_band[lo2] >> 16;
                    for (int k = 0; k < per_spike; ++k) {
                        const int g0 = (k % ngr) * MPB_GROUP;
                        acc += 1 + 4 * max(0, min(bh, g0 + MPB_GROUP - 1) - max(bl, g0) + 1);
                        if (acc > c) return lo2 * per_spike + k;
                    }
                    return (lo2 + 1) * per_spike;
                };
                s_next = item_at(ctot * b / G);
                s_end = (b == G - 1) ? items : item_at(ctot * (b + 1) / G);
            }
        } else if (tid == 0) {
            const int per_cta = (items + G - 1) / G;
            s_next = min(items, b * per_cta);
            s_end = min(items, (b + 1) * per_cta);
        }
        __syncthreads();
        {
            // Work items (spike q, chunk ch, group g): the columns of spike q's
            // segment [max(x_q - nt, x_{q-1} + nt + 1), x_q + nt], 32 at a time
            // (lane = column), and the row blocks g*MPB_GROUP.. of the group;
            // the CTA's warps take them from a shared counter. Lane L holds
            // spike q - 1 + L of the round.
            const int it_end = s_end;
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
            for (;;) {
                int it = 0;
                if (lane == 0) it = atomicAdd(&s_next, 1);
                it = __shfl_sync(FULL, it, 0);
                if (it >= it_end) break;
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
                const int x0 = __shfl_sync(FULL, x, max(e0, 0) + 1);
                const int y0 = __shfl_sync(FULL, y, max(e0, 0) + 1);
                const float a0 = __shfl_sync(FULL, amp, max(e0, 0) + 1);
                const int x1 = __shfl_sync(FULL, x, max(e1, 0) + 1);
                const int y1 = __shfl_sync(FULL, y, max(e1, 0) + 1);
                const float a1 = __shfl_sync(FULL, amp, max(e1, 0) + 1);
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
                // fl(|a_e| * max_l |ctc[t_r, y_e, l]|) >= thr (otherwise the term
                // leaves every score of the row bit for bit unchanged).
                const int bg0 = g * MPB_GROUP, nbg = min(MPB_GROUP, nb - bg0);
                float bmv[MPB_GROUP], cmv[MPB_GROUP][MPB_SPK];
#pragma unroll
                for (int j = 0; j < MPB_GROUP; ++j) {
                    const int bb = bg0 + j;
                    const int tr = (j < nbg) ? s_perm[bb * MPB_ROWS + lane] : -1;
                    bmv[j] = (j < nbg && active) ? __ldcg(a.bmin + bb * ldk + s) : 0.f;
#pragma unroll
                    for (int e = 0; e < MPB_SPK; ++e)
                        cmv[j][e] = (tr >= 0 && e < nl) ? __ldg(a.cmaxr + (int64_t)ye[e] * T + tr) : 0.f;
                }
                // per block j: the rows that need this lane's even term (m0) and odd
                // term (m1), packed 32 bits per block; bit j of procm: block j is processed
                unsigned long long m0p[(MPB_GROUP + 1) / 2], m1p[(MPB_GROUP + 1) / 2];
#pragma unroll
                for (int i = 0; i < (MPB_GROUP + 1) / 2; ++i) m0p[i] = m1p[i] = 0ull;
                unsigned procm = 0u;
#pragma unroll
                for (int j = 0; j < MPB_GROUP; ++j) {
                    const float thr_l = active ? quarter_ulp(bmv[j]) : FLT_MAX;
                    const float thr = __uint_as_float(__reduce_min_sync(FULL, __float_as_uint(thr_l)));
                    unsigned m0 = (e0 >= MPB_SPK) ? 0xffffffffu : 0u, m1 = (e1 >= MPB_SPK) ? 0xffffffffu : 0u;
#pragma unroll
                    for (int e = 0; e < MPB_SPK; ++e) {
                        const unsigned me = __ballot_sync(FULL, e < nl && !(__fmul_rn(fae[e], cmv[j][e]) < thr));
                        if (e0 == e) m0 = me;
                        if (e1 == e) m1 = me;
                    }
                    if (e0 < 0) m0 = 0u;
                    // after a term that changes the score the second is always applied
                    m1 = (e1 >= 0) ? (m1 | m0) : 0u;
                    if (j < nbg && __any_sync(FULL, active && (m0 | m1) != 0u)) procm |= 1u << j;
                    m0p[j / 2] |= (unsigned long long)m0 << (32 * (j & 1));
                    m1p[j / 2] |= (unsigned long long)m1 << (32 * (j & 1));
                }
                n_items += nbg;
                const float* c0p = a.ctcP + (int64_t)y0 * T * L2 + (s - x0 + nt);
                const float* c1p = a.ctcP + (int64_t)y1 * T * L2 + (s - x1 + nt);
                n_proc += __popc(procm);
                if (!active || procm == 0u) continue;
                // the processed blocks' rows in 8-row batches through one
                // software pipeline: the next batch's loads are issued before
                // the current batch is updated, across block boundaries
                auto masks = [&](int j, unsigned& m0, unsigned& m1) {
                    unsigned long long p0 = m0p[0], p1 = m1p[0];
#pragma unroll
                    for (int i = 1; i < (MPB_GROUP + 1) / 2; ++i)
                        if (j / 2 == i) {
                            p0 = m0p[i];
                            p1 = m1p[i];
                        }
                    m0 = (unsigned)(p0 >> (32 * (j & 1)));
                    m1 = (unsigned)(p1 >> (32 * (j & 1)));
                };
                // batch k of the sequence: block j = k-th set bit group, rows rb*8..
                const int nbt = __popc(procm) * (MPB_ROWS / 8);
                auto batch_of = [&](int k, int& j, int& rb) {
                    int left = k / (MPB_ROWS / 8);
                    unsigned pm = procm;
                    for (int i = 0; i < left; ++i) pm &= pm - 1u;
                    j = __ffs(pm) - 1;
                    rb = k % (MPB_ROWS / 8);
                };
                float v[8], w0[8], w1[8];
                auto load = [&](int k, float (&lv)[8], float (&l0)[8], float (&l1)[8]) {
                    int j, rb;
                    batch_of(k, j, rb);
                    unsigned m0, m1;
                    masks(j, m0, m1);
                    const int r0 = (bg0 + j) * MPB_ROWS, nr = min(MPB_ROWS, T - r0);
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const int rr = rb * 8 + u;
                        const int t = rr < nr ? s_perm[r0 + rr] : -1;
                        lv[u] = t >= 0 ? ld_keep(a.B + (int64_t)t * ldb + s, pk) : 0.f;
                        l0[u] = (t >= 0 && ((m0 >> rr) & 1u)) ? ld_stream(c0p + (int64_t)t * L2, ps) : 0.f;
                        l1[u] = (t >= 0 && ((m1 >> rr) & 1u)) ? ld_stream(c1p + (int64_t)t * L2, ps) : 0.f;
                    }
                };
                load(0, v, w0, w1);
                ColMaxAny m;
                float mn = INFINITY;
                for (int k = 0; k < nbt; ++k) {
                    float nv[8], nw0[8], nw1[8];
                    if (k + 1 < nbt) load(k + 1, nv, nw0, nw1);
                    int j, rb;
                    batch_of(k, j, rb);
                    unsigned m0, m1;
                    masks(j, m0, m1);
                    const int bb = bg0 + j, r0 = bb * MPB_ROWS, nr = min(MPB_ROWS, T - r0);
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const int rr = rb * 8 + u;
                        if (rr >= nr) continue;
                        const int t = s_perm[r0 + rr];
                        float xv = v[u];
                        if ((m0 >> rr) & 1u) xv = __fsub_rn(xv, __fmul_rn(a0, w0[u]));
                        if ((m1 >> rr) & 1u) xv = __fsub_rn(xv, __fmul_rn(a1, w1[u]));
                        if (__float_as_uint(xv) != __float_as_uint(v[u])) st_keep(a.B + (int64_t)t * ldb + s, xv, pk);
                        mn = fminf(mn, fabsf(xv));
                        m.consider(xv, s_nm[t], s_inv[t], t);
                    }
                    if (rb == MPB_ROWS / 8 - 1) {  // last batch of the block: its key and minimum
                        a.bkey[bb * ldk + s] = pack_key(m.best, m.bi);
                        a.bmin[bb * ldk + s] = mn;
                        m = ColMaxAny();
                        mn = INFINITY;
                    }
                    if (k + 1 < nbt) {
#pragma unroll
                        for (int u = 0; u < 8; ++u) {
                            v[u] = nv[u];
                            w0[u] = nw0[u];
                            w1[u] = nw1[u];
                        }
                    }
                }
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

static size_t mpb_smem_bytes(int cols_per_blk, int nt, int T, int nb) {
    return sizeof(float) * ((size_t)cols_per_blk + 2 * nt) + sizeof(int) * (size_t)cols_per_blk +
           sizeof(float) * 2 * (size_t)T + sizeof(int) * (size_t)nb * MPB_ROWS + sizeof(int) * 2 * MPB_MAX_SPK + 16;
}

cudaError_t launch_mp_blocks(MPArgs a, int grid, cudaStream_t s) {
    if (grid > MPB_MAX_GRID || !a.perm || !a.cmaxr || !a.bkey || !a.bmin || !a.band_lo || !a.band_hi ||
        a.nb != (a.T + MPB_ROWS - 1) / MPB_ROWS)
        return cudaErrorInvalidValue;
    const size_t smem = mpb_smem_bytes(a.cols_per_blk, a.nt, a.T, a.nb);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_mp_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = cudaMemsetAsync(a.bar, 0, 2 * sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
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
    return cudaLaunchKernelEx(&lc, k_mp_blocks, a);
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
