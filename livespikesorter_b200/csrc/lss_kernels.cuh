// Internal declarations shared by the kernel translation units and the host
// orchestration (lss_api.cpp). Launchers return cudaError_t of the launch.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace lss {

// Where column s of the padded batch X [C, N] comes from in the raw rows
// (kilosort/io.py:584-637): row = clamp(s - lead, 0, nsamp-1); columns at or
// past lead + nsamp are zero when zero_tail (batch 0) and replicate the last
// row otherwise (last batch).
// Batch column s reads raw row src_row(s): Kilosort's padded batch
// (io.py:584-637) with `lead` replicated leading rows and the tail replicated
// or zero. With base_dev set the rows come from a ring of ring_rows rows
// instead: column s is stream row *base_dev + s (rows before the stream start
// replicate row 0), stored at ring index row % ring_rows.
struct IngestMap {
    int64_t lead = 0;
    int64_t nsamp = 0;
    int32_t zero_tail = 0;
    const int64_t* base_dev = nullptr;
    int64_t ring_rows = 0;
};

// ---- ingest (ingest.cu) ----
cudaError_t launch_chan_sums(const int16_t* raw, int32_t ld_raw, const int32_t* chan_map, int32_t C,
                             int64_t N, IngestMap map, long long* sums, cudaStream_t s);
cudaError_t launch_car(const int16_t* raw, int32_t ld_raw, const int32_t* chan_map, int32_t C, int64_t N,
                       IngestMap map, float sign, const long long* sums, int do_car, float* X1,
                       int64_t ldx, cudaStream_t s);
cudaError_t launch_highpass(const float* X1, int64_t ldx, int32_t C, int64_t N, const float* taps, int32_t L,
                            float* Xh, cudaStream_t s);
// overlap-save FFT form (L <= 1024): H = conj(FFT_4096(taps wrapped around 0)), tw[k] = exp(-2 pi i k / 4096)
cudaError_t launch_highpass_fft(const float* X1, int64_t ldx, int32_t C, int64_t N, int32_t L, const float2* H,
                                const float2* tw, float* Xh, cudaStream_t s);

// ---- dense FP32 GEMM (gemm_fp32.cu): C[M,N] = A[M,K] @ B[K,N], row-major ----
cudaError_t launch_sgemm(const float* A, int64_t lda, const float* B, int64_t ldb, float* Cm, int64_t ldc,
                         int M, int N, int K, cudaStream_t s);
// rows t*K + k of U [T, K, C] times Mw [C, C], stored as the score GEMM's
// folded templates ([t, c'*K + k], bf16 or tf32 hi/lo)
cudaError_t launch_sgemm_folded(const float* U, const float* Mw, int32_t T, int32_t K, int32_t C, int64_t ldk,
                                __nv_bfloat16* out16, __nv_bfloat16* out16lo, float* hi, float* lo, cudaStream_t s);

// ---- temporal basis projection (score.cu) ----
// transposed bf16 variant for the tensor-core GEMM: B0T[s, c*K + k], row stride ldk
// bf16 split (hi, lo = bf16(x - hi)) of the projection for the BF16x3 GEMM;
// norm2 (optional, [N]): ||B0T[s, :]||^2 of the FP32 values before rounding
cudaError_t launch_pca_proj_t(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t K,
                              int32_t nt, __nv_bfloat16* B0T_hi, __nv_bfloat16* B0T_lo, int64_t ldk, cudaStream_t s,
                              float* norm2 = nullptr);

// ---- tensor-core score GEMM (tc_gemm.cu) ----
struct TcPlan {
    int Tpad;      // templates rounded up to 16 (the MMA's N granularity)
    int box_rows;  // template rows per TMA box
    int b_rows;    // template rows of one shared-memory stage
    int stages;
    int nacc;      // accumulator buffers in tensor memory
    size_t smem;
    int kblock;    // K elements per pipeline stage
    int pass_w;    // templates per pass
};
// element kinds of the score GEMM (tc_gemm.cu)
enum TcOp : int { TC_BF16 = 0, TC_TF32X3 = 1, TC_BF16X3 = 2 };
TcPlan tc_plan(int T, int op, int pass_w = 512);
// Optional epilogue behaviour of the score GEMM.
struct TcExtra {
    // GEMM row r scores sample rowmap[r / map_rows] * map_rows + r % map_rows
    // (re-check tiles); rows beyond count_dev[0] * map_rows are skipped
    const int32_t* rowmap = nullptr;
    int map_rows = 1;
    const int32_t* count_dev = nullptr;
    int ncols = 0;                    // batch samples when rowmap is set
    float* cf2 = nullptr;             // runner-up Cf per sample
    unsigned long long* keys = nullptr;  // [N] scratch: lets short batches split templates over CTAs
    // BF16 error bounds: un[t] = ||template row t||, pn2[s] = ||projection row s||^2; with them the
    // epilogue writes cf_lo / cf_hi (bounds of the FP32 path's best Cf) and, in cf2, the largest
    // upper bound of any other template, for |B - B_fp32| <= eps * un[t] * sqrt(pn2[s])
    const float* un = nullptr;
    const float* pn2 = nullptr;
    float eps = 0.f;
    float* cf_lo = nullptr;
    float* cf_hi = nullptr;
    // error bounds over a full batch in several template passes: scratch for
    // the per-(pass, column) partials (part_cap = passes x columns it holds);
    // without it such a batch is scored tile by tile
    unsigned long long* part_keys = nullptr;
    float* part = nullptr;  // 4 x part_cap
    int64_t part_cap = 0;
    // score rows in another order: template t's row of B is rowof[t] (the
    // block-skipping rounds keep rows in probe order); null: row t
    const int32_t* rowof = nullptr;
};
// B[t, s] (row stride ldb) = sum_kk B0T[s, kk] * Up[t, kk] with B0T [N, ldk] and Up [Tpad, CKpad]
// bf16, CKpad a multiple of 64; also writes the column maxima cfmax/imax of Cf.
cudaError_t launch_score_tc(const __nv_bfloat16* B0T, int64_t ldk, int N, const __nv_bfloat16* Up, int T, int CKpad,
                            const float* nm, float* Bout, int64_t ldb, float* cfmax, int32_t* imax, int nt,
                            int32_t* status, int grid, cudaStream_t s, const TcExtra& ex = TcExtra());
// BF16x3: operands split into bf16 hi = bf16(x), lo = bf16(x - hi); three bf16
// MMAs per k-step (hi*hi, hi*lo, lo*hi) with FP32 accumulation, about 2^-16
// relative per product
cudaError_t launch_score_tc_bf16x3(const __nv_bfloat16* B0T_hi, const __nv_bfloat16* B0T_lo, int64_t ldk, int N,
                                   const __nv_bfloat16* Up_hi, const __nv_bfloat16* Up_lo, int T, int CKpad,
                                   const float* nm, float* Bout, int64_t ldb, float* cfmax, int32_t* imax, int nt,
                                   int32_t* status, int grid, cudaStream_t s, const TcExtra& ex = TcExtra());
// FP32-class variant (3xTF32): operands split into tf32 hi + lo parts stored as fp32.
cudaError_t launch_score_tc_tf32x3(const float* B0T_hi, const float* B0T_lo, int64_t ldk, int N, const float* Up_hi,
                                   const float* Up_lo, int T, int CKpad, const float* nm, float* Bout, int64_t ldb,
                                   float* cfmax, int32_t* imax, int nt, int32_t* status, int grid, cudaStream_t s,
                                   const TcExtra& ex = TcExtra());
// transposed projection split into tf32 hi/lo parts (fp32 containers) for the 3xTF32 GEMM
cudaError_t launch_pca_proj_t_tf32(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t K,
                                   int32_t nt, float* hi, float* lo, int64_t ldk, cudaStream_t s);

// U_w[t, c'*K + k] = sum_c U[t,k,c] Mw[c,c'] in GEMM layout: bf16 split (out16, out16lo) and/or tf32
// hi/lo (a null pointer skips that form)
cudaError_t launch_build_uw(const float* U, const float* Mw, int32_t T, int32_t K, int32_t C, int64_t ldk,
                            __nv_bfloat16* out16, __nv_bfloat16* out16lo, float* hi, float* lo, cudaStream_t s);

// FP32 re-check of the BF16 path (score.cu): columns whose first-round
// decisions the BF16 error bound leaves open, their FP32 projection rows and
// the count of decisions the re-check changed
cudaError_t launch_recheck_select(const float* cf_lo, const float* cf_hi, const float* ch, const float* cfmax,
                                  const int32_t* imax, int32_t N, int32_t nt, float th2, int32_t* cols, float* pre_cf,
                                  int32_t* pre_im, int32_t* count, cudaStream_t s);
// FP32 projection rows (tf32 split) of the columns cols[0 .. *count) (at most
// max_cols): row i of hi / lo, or row cols[i] when scatter is set
cudaError_t launch_pca_proj_cols_tf32(const float* X, int64_t ldx, int32_t C, int64_t N, const float* wpca, int32_t K,
                                      int32_t nt, const int32_t* cols, const int32_t* count, int32_t max_cols, float* hi,
                                      float* lo, int64_t ldk, int32_t scatter, cudaStream_t s);
cudaError_t launch_recheck_flips(const float* cfmax, const int32_t* imax, const int32_t* cols, const float* pre_cf,
                                 const int32_t* pre_im, int32_t* count, int32_t N, float th2, cudaStream_t s);
// un[t] = ||hi[t, :] + lo[t, :]|| over rows of length ld
cudaError_t launch_row_norms(const float* hi, const float* lo, int32_t T, int64_t ld, float* un, cudaStream_t s);

// ---- matching pursuit (mp.cu) ----
struct MPArgs {
    float* B;                 // [T, ldb] score field, updated in place
    int64_t ldb;
    int32_t T, N, nt;
    float th2;                // Th * Th
    const float* nm;          // [T]
    const float* ctcP;        // [T(j), T(i), 2nt+1] = ctc.permute(1,0,2)
    float* cfmax;             // [N] column maxima
    int32_t* imax;            // [N] first argmax template of each column
    unsigned long long* colkey;  // [2, ldk] update keys, alternating by round parity; zero at launch
    int64_t ldk;
    int32_t* blk_cnt;         // [G] peaks per CTA
    int32_t* blk_x;           // [N] per-CTA peak lists (CTA b at b*W)
    int32_t* blk_y;           // [N]
    float* blk_amp;           // [N]
    int32_t* sp_x;            // [capacity] spikes in run_matching order
    int32_t* sp_y;
    float* sp_amp;
    int32_t* sp_round;        // may be null
    int32_t* round_start;     // [max_rounds + 2]
    int32_t capacity;
    int32_t max_rounds;
    int32_t* counters;        // [0]=spikes [1]=rounds
    int32_t* status;          // error bits (STATUS_*)
    unsigned int* bar;        // [2] grid barrier count / generation, zero at launch
    int32_t cols_per_blk;     // W
    int32_t init_cols;        // 1: compute column maxima of B before round 0
    unsigned long long* phase = nullptr;    // [6] phase clock of the rounds (PhaseClock), zero at launch; may be null
    // block-skipping rounds (mp_blocks.cu) only: the score rows of B are in
    // probe order (row r holds template perm[r]) and grouped in blocks of
    // MPB_ROWS; ctcP then points at ctcQ [T(spike template), T(row), 2nt+1]
    const int32_t* perm = nullptr;          // [nb * MPB_ROWS] template of each row, -1 past T
    int32_t nb = 0;                         // row blocks
    const float* cmaxr = nullptr;           // [T(spike template), T(row)] max |ctc| over lags
    unsigned long long* bkey = nullptr;     // [nb, ldk] per block and column: max (Cf bits << 32 | ~t)
    float* bmin = nullptr;                  // [nb, ldk] per block and column: min |B|
    int4* ment = nullptr;                   // [G * ment_cap * 4] per-CTA lists of blocks to process (64-byte
                                            // entries); null: blocks are processed where they are decided
    int32_t* ment_cnt = nullptr;            // [G] entries per list
    int32_t ment_cap = 0;                   // entries per list
};
enum : int32_t { STATUS_TIMEOUT = 1, STATUS_CAPACITY = 2, STATUS_LIST = 4 };
cudaError_t launch_mp(MPArgs a, int grid, cudaStream_t s);
// the same rounds, skipping (spike, row block) updates that provably leave
// every score of the block unchanged; needs perm, nb, cmaxr, bkey, bmin
constexpr int MPB_ROWS = 32;
cudaError_t launch_mp_blocks(MPArgs a, int grid, cudaStream_t s);
int mp_blocks_max_grid(int device);
// entries the lists of a grid of `grid` CTAs hold in all (ment_cap = that / grid
// keeps every round of at most (N + nt) / (nt + 1) peaks in list mode)
int64_t mp_blocks_list_entries(int64_t N, int nt, int T, int grid);
// cmaxr[y, t] = max over lags of |ctcP[y, t, :]| (infinite where a lag is NaN)
cudaError_t launch_ctc_row_max(const float* ctcP, int32_t T, int32_t L2, float* cmaxr, cudaStream_t s);
// ctcQ[y, r, :] = ctcP[y, perm[r], :] (the block-skipping rounds' copy, rows in probe order)
cudaError_t launch_permute_ctc(const float* ctcP, const int32_t* perm, int32_t T, int32_t L2, float* ctcQ,
                               cudaStream_t s);
// dst row r = src row perm[r], N columns
cudaError_t launch_gather_rows(const float* src, int64_t lds, const int32_t* perm, int32_t rows, int64_t N,
                               float* dst, int64_t ldd, cudaStream_t s);
int mp_max_grid(int device);
void set_thread_error(const char* msg);
// true when kernels on `device` may dereference p (that device's memory,
// managed or pinned host memory) or p is null
bool device_accessible(const void* p, int device);
// the rounds' per-column spike lists hold MP_LIST spikes; more peaks than that
// whose windows reach one column in one round overflow them (STATUS_LIST)
constexpr int MP_LIST = 31;
constexpr const char* MSG_MP_LIST = "more than 31 peaks within 2*nt samples of one another in one round";
cudaError_t launch_status_or(const int32_t* st, int32_t* acc, cudaStream_t s);

// ---- residual and PC features (features.cu); n = spikes of the batch ----
cudaError_t launch_xres(const float* X, int64_t ldx, int32_t C, int32_t N, int32_t nt, const float* wave,
                        const int32_t* sp_x, const int32_t* sp_y, const float* sp_amp,
                        const int32_t* round_start, const int32_t* counters, int32_t rounds,
                        float* Xres, int32_t* status, cudaStream_t s);
// slot: scratch [n] for the output position of each spike
struct RecordClock {
    int32_t presorted = 0;                 // output slots already computed (post-processing)
    int64_t ibatch = 0;                    // batch index (host value) ...
    const int64_t* ibatch_dev = nullptr;   // ... or read from the device
    const int32_t* counters = nullptr;     // spike count read from the device (counters[0])
    int64_t shift = 0;                     // extra sample offset of the batch window
    int32_t NT = 0, nt = 0, nt0min = 0;
    int32_t slots = 0;                     // > 0: outputs are rings of `slots` batches
};
// ---- post-processing (post.cu): positions, clusters, duplicates, time order ----
struct PostArgs {
    const int32_t* sp_x = nullptr;
    const int32_t* sp_y = nullptr;
    const float* tF = nullptr;             // [n, nC, K] PC features (null: no positions)
    int nC = 0, K = 0, C = 0;
    const int64_t* iCC = nullptr;
    const int64_t* iU = nullptr;
    const float* xc = nullptr;             // channel coordinates (null: no positions)
    const float* yc = nullptr;
    const float* cen_x = nullptr;          // cluster centroids (n_clu = 0: cluster = template)
    const float* cen_y = nullptr;
    int n_clu = 0;
    int dt = 0;                            // duplicate window in samples (0: off)
    unsigned long long* key_c = nullptr;   // [n_max] scratch keys and their sorted copies
    unsigned long long* key_c_sorted = nullptr;
    unsigned long long* key_t = nullptr;
    unsigned long long* key_t_sorted = nullptr;
    void* sort_tmp = nullptr;
    size_t sort_bytes = 0;
    uint8_t* keep = nullptr;               // [n_max]
    int64_t* last_time = nullptr;          // [clusters] last kept time, carried across batches
    float* px = nullptr;                   // [n_max] per-spike position and cluster
    float* py = nullptr;
    int32_t* clu = nullptr;
};
size_t post_sort_bytes(int32_t n_max);
cudaError_t launch_post(const PostArgs& a, const RecordClock& rc, int32_t n_max, int32_t* slot, int64_t* out_count,
                        cudaStream_t s);
cudaError_t launch_post_write(const PostArgs& a, const RecordClock& rc, const int32_t* slot, int32_t n_max,
                              float* out_x, float* out_y, int32_t* out_clu, int64_t capacity, cudaStream_t s);

cudaError_t launch_records(const int32_t* sp_x, const int32_t* sp_y, const float* sp_amp, const float* tF,
                           int32_t* slot, int32_t n, int32_t feat_len, const RecordClock& rc, int64_t* out_time,
                           int32_t* out_tmpl, float* out_amp, float* out_pc, int64_t capacity, int64_t* out_count,
                           cudaStream_t s);
// PC features from the highpassed batch (or, when Phi is given, the projection rows
// P = Phi + Plo [N, ldp] of the score GEMM: fp32 tf32 parts, or bf16 parts when
// p_bf16) and the folded whitening (no residual array)
cudaError_t launch_pc_features_folded(const float* Xh, int64_t ldx, int32_t C, int32_t nt, int32_t K, int32_t nC,
                                      int32_t T, const float* wpca, const float* Mw, const float* U, const float* R,
                                      const int64_t* iCC, const int64_t* iU, const float* Ucc, const int32_t* sp_x,
                                      const int32_t* sp_y, const float* sp_amp, const int32_t* round_start,
                                      int32_t rounds, int32_t n, const int32_t* counters, float* tF,
                                      int32_t* status, const void* Phi, const void* Plo, int32_t p_bf16, int64_t ldp,
                                      cudaStream_t s);
cudaError_t launch_st_out(const int32_t* sp_x, const int32_t* sp_y, const float* sp_amp, int32_t n,
                          int64_t* st, float* amps, cudaStream_t s);

}  // namespace lss
