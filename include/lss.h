/*
 * lss.h - C ABI of the B200-native per-batch spike-sorting hot path.
 *
 * A drop-in for the sorting path of LiveSpikeSorter's V2 sorter
 * (src/SpikeSorter/OnlineSpikesV2.{h,cu}) and of the Kilosort4 template
 * matching it mirrors (kilosort/template_matching.py, kilosort/io.py).
 * Plain C types only: pointers, sizes and status codes. No exception crosses
 * this boundary and nothing here calls exit().
 *
 * Thread safety: one handle per probe stream; distinct handles may be used
 * from distinct threads concurrently. A single handle is not re-entrant.
 * Streams are passed as `void*` (a cudaStream_t; NULL = legacy default stream).
 */
#ifndef LSS_H_
#define LSS_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (replace _RUN_ERROR / _CUDA_CALL exceptions and loader exit(),
 * src/Helpers/Utils.h:41-64, OnlineSpikesV2.cu:437-441). */
#define LSS_OK            0
#define LSS_ERR_ARG       1   /* invalid argument / unsupported value       */
#define LSS_ERR_IO        2   /* file missing, unreadable or malformed .npy */
#define LSS_ERR_SHAPE     3   /* tensor dtype or shape mismatch             */
#define LSS_ERR_CUDA      4   /* CUDA runtime error                         */
#define LSS_ERR_CAPACITY  5   /* spike or record buffer too small           */
#define LSS_ERR_TIMEOUT   6   /* a bounded device-side wait gave up         */
#define LSS_ERR_STATE     7   /* call out of order (e.g. no drift matrix)   */
#define LSS_ERR_BUSY      8   /* no probe slot or device memory free now    */

/* Score precision of the template-matching GEMM. */
#define LSS_PREC_FP32          0  /* FP32 scores (parity path)                        */
#define LSS_PREC_BF16_RECHECK  1  /* BF16 tcgen05 GEMM + FP32 recheck of near ties    */

typedef struct lss_handle lss_handle;

/* Shapes and hyper-parameters. Mirrors the sorter's members
 * (OnlineSpikesV2.h:84-102) and the Kilosort ops entries it reads
 * (misc.txt parsing at OnlineSpikesV2.cu:435-457). */
typedef struct lss_config {
    int32_t n_chan;        /* C: channels after chan_map                        */
    int32_t n_chan_bin;    /* channels per raw int16 row (>= n_chan)            */
    int32_t n_templates;   /* T: rows of Wall3 (unclu_T)                        */
    int32_t n_pcs;         /* K: temporal basis size                            */
    int32_t nt;            /* template length in samples (M)                    */
    int32_t n_nearest;     /* nC: channels per PC feature                       */
    int32_t batch_size;    /* NT: samples per batch (padded batch = NT + 2*nt)  */
    int32_t nt0min;        /* trough alignment sample                           */
    float   th_learned;    /* Th: score threshold is Th*Th                      */
    int32_t max_rounds;    /* matching-pursuit round cap (Kilosort: 100)        */
    int32_t max_spikes;    /* per-batch spike capacity (Kilosort: 100000)       */
    int32_t do_car;        /* subtract the per-sample median across channels    */
    int32_t invert_sign;   /* multiply raw data by -1                           */
    int32_t precision;     /* LSS_PREC_*                                        */
    int32_t device;        /* CUDA device ordinal                               */
    int32_t hp_len;        /* taps in hp_filter (0 = no highpass)               */
} lss_config;

/* Host tensors, row-major, float32 unless noted. Kilosort export names
 * (src/Python/run_online_spikes.py:548-576). The library copies them. */
typedef struct lss_tensors {
    const float*   wall3;      /* U          [T, K, C]                              */
    const float*   wpca;       /* wPCA       [K, nt]                                */
    const float*   ctc;        /* ctc        [T, T, 2*nt+1]  (ctc[i, j, l])         */
    const float*   whitening;  /* Wrot       [C, C]                                 */
    const float*   drift;      /* M          [C, C] or NULL (identity)              */
    const float*   hp_filter;  /* hp_filter  [hp_len] or NULL                       */
    const int64_t* iCC;        /* iCC        [nC, C]                                */
    const int64_t* iU;         /* iU         [T]                                    */
    const float*   Ucc;        /* Ucc        [nC, T, K]                             */
    const int32_t* chan_map;   /* chan_map   [C] or NULL (identity)                 */
    const float*   nm;         /* template energies [T] or NULL (computed)          */
} lss_tensors;

/* Caller-owned spike records of one batch (OnlineSpikesPayload's Times /
 * Templates / Amplitudes, onlineSpikesPayload.h:8-48, plus Kilosort's tF).
 * `count` is written on return; on LSS_ERR_CAPACITY it holds the required size. */
typedef struct lss_records {
    int64_t* time;         /* [capacity] absolute sample, Kilosort convention     */
    int32_t* template_id;  /* [capacity]                                           */
    float*   amplitude;    /* [capacity]                                           */
    float*   pc;           /* [capacity, nC, K] or NULL                            */
    int64_t  capacity;
    int64_t  count;
    int32_t  on_device;    /* 1: the arrays are device pointers                    */
    /* filled only when post-processing is on (lss_set_postprocess); may be NULL */
    float*   x_pos;        /* [capacity] spike position (compute_spike_positions)  */
    float*   y_pos;        /* [capacity]                                           */
    int32_t* cluster;      /* [capacity] nearest cluster centroid (or template)    */
} lss_records;

/* Post-processing of every batch's spikes (off by default):
 *  - position from the PC-feature energy on the nC nearest channels
 *    (kilosort/postprocessing.py:33-46; OnlineSpikesV2.cu:189-244), needs xc/yc;
 *  - cluster = nearest of n_clusters centroids [n_clusters, 2] (x, y), first
 *    index on ties (OnlineSpikesV2::closestCluster, OnlineSpikesV2.cu:1028-1043,
 *    with the reference's cluster_centroids.npy); n_clusters = 0: cluster = template;
 *  - removal of spikes closer than dt_samples to the last kept spike of their
 *    cluster (kilosort/postprocessing.py:10-31; OnlineSpikesV2::saveSpikes,
 *    OnlineSpikesV2.cu:1131-1164), carried from batch to batch (reset by a
 *    first batch, ibatch = 0, or lss_reset_postprocess); dt_samples = 0: off;
 *  - records in time order (ties in matching order).
 * Pass NULL to switch it off. */
typedef struct lss_post_config {
    const float* xc;            /* [n_chan] channel x (um), or NULL */
    const float* yc;            /* [n_chan] channel y (um), or NULL */
    const float* centroids_xy;  /* [n_clusters, 2] or NULL           */
    int32_t n_clusters;
    int32_t dt_samples;         /* Kilosort's duplicate_spike_bins (7 at 30 kHz) */
} lss_post_config;
int  lss_set_postprocess(lss_handle* h, const lss_post_config* post);
int  lss_reset_postprocess(lss_handle* h);

/* Construction. Replaces OnlineSpikesV2::OnlineSpikesV2 / initializeSorter /
 * initializeStaticMemory (OnlineSpikesV2.cu:247-280, 321-352, 470-608): all
 * device memory is allocated here, none per batch. */
int  lss_create(const lss_config* cfg, const lss_tensors* tensors, lss_handle** out);

/* Reads an LSS input directory (Wall3.npy, wPCA.npy, ctc.npy, whitening_mat.npy
 * or whiteningMat.npy, drift_matrix.npy, hp_filter.npy, iCC.npy, iU.npy,
 * Ucc.npy, channel_map.npy, misc.txt), honouring each .npy header's
 * fortran_order flag (the reference's cnpy ignores it, cnpy.cpp:181-184, and
 * drift_matrix.npy is written in Fortran order). `overrides` may be NULL;
 * otherwise its do_car, invert_sign, precision and device are used as given
 * and its other non-zero fields replace values read from the directory. */
int  lss_create_from_dir(const char* dir, const lss_config* overrides, lss_handle** out);

void lss_destroy(lss_handle* h);

/* Last error message of this handle, or of the calling thread's last failed
 * create when h is NULL. */
const char* lss_last_error(const lss_handle* h);

/* Reads back the effective configuration. */
int  lss_get_config(const lss_handle* h, lss_config* out);

/* Per-batch drift interpolation matrix M [C, C] (host pointer); the filter
 * applies (M @ Wrot) @ X as kilosort/io.py:782-789 does. NULL = identity. */
int  lss_set_drift(lss_handle* h, const float* M);

/* Ingest of one padded batch, kilosort/io.py:584-637 + 757-790:
 * raw = the int16 rows [n_rows, n_chan_bin] that padded_batch_to_torch reads
 * for batch `ibatch` of `n_batches` (device pointer if raw_on_device, else
 * host), out X_dev = filtered, whitened, drift-corrected f32 [C, NT + 2*nt]
 * (row stride NT + 2*nt). Replaces the preprocessing block of
 * OnlineSpikesV2::runSpikeSorting (OnlineSpikesV2.cu:738-778). */
int  lss_filter(lss_handle* h, const int16_t* raw, int64_t n_rows, int64_t ibatch,
                int64_t n_batches, int32_t raw_on_device, float* X_dev, void* stream);

/* Template matching on a filtered batch, kilosort/template_matching.py:128-202
 * (run_matching) and OnlineSpikesV2::kilosortMatchingPursuit
 * (OnlineSpikesV2.h:56, OnlineSpikesV2.cu:873-971). X_dev f32 [C, N] (row
 * stride N). Outputs (device pointers, run_matching order = round-major,
 * time-minor): st_dev int64 [capacity, 2] (sample, template), amps_dev f32
 * [capacity], xres_dev f32 [C, N] or NULL. *n_spikes = spikes found. */
int  lss_match(lss_handle* h, const float* X_dev, int64_t N, int64_t* st_dev, float* amps_dev,
               float* xres_dev, int64_t capacity, int64_t* n_spikes, void* stream);

/* The matching-pursuit rounds alone on a given score field B_dev f32 [T, N]
 * (template_matching.py:157-198), for parity checks of the rounds in isolation
 * from the score GEMM. B_dev is not modified. */
int  lss_match_scores(lss_handle* h, const float* B_dev, int64_t N, int64_t* st_dev,
                      float* amps_dev, int64_t capacity, int64_t* n_spikes, void* stream);

/* Which kernel runs the matching-pursuit rounds of this handle (identical
 * spikes, amplitudes and score field either way; a performance choice, no
 * counterpart in the reference): 0 = every template row of every spike window
 * is updated; 1 = template rows are grouped in blocks along the probe and a
 * block whose update provably leaves every score unchanged (terms below a
 * quarter ulp of the block's smallest score) is skipped. The default is 1 from
 * 600 templates up (measured on a B200, 384 channels: 7.40 vs 7.75 ms of rounds
 * per 2-s batch at 800 templates, 2.43 vs 2.15 ms at 400), else 0. */
int  lss_set_round_kernel(lss_handle* h, int32_t skip_blocks);
/* The handle's rounds kernel (1: block-skipping, 0: every row). */
int  lss_get_round_kernel(const lss_handle* h, int32_t* skip_blocks);

/* The same matching-pursuit rounds for callers that cannot allocate device
 * memory (an acquisition host that owns the GPU's memory, a process whose
 * memory another allocator reserved up front, a real-time loop that must not
 * take cudaMalloc's synchronisation). No counterpart in the reference.
 * Allocates nothing: its working memory is a fixed array inside the library
 * (about 2.3 MB, held on every GPU that loads the library until exit), sized
 * for at most LSS_NOALLOC_MAX_SAMPLES columns; larger batches are rejected
 * with LSS_ERR_ARG. Needs no handle; runs on the calling thread's current
 * device. The first call on a device looks up the array's device address, so
 * make that first call before any stream capture; the address is kept for the
 * life of the process, so do not call this again after cudaDeviceReset on that
 * device. All calls share the array: calls that overlap on the GPU race, so
 * serialise them. Every array must be memory of the current device or pinned
 * host memory (LSS_ERR_ARG otherwise, before any launch).
 * B_dev f32 [T, ldb] is the score field and is updated in place;
 * nm_dev f32 [T]; ctc_permuted_dev f32 [T, T, 2nt+1] = ctc.permute(1,0,2)
 * (the reference's ctc_permuted.npy). Outputs: spike_x / spike_y / spike_amp
 * (device, [capacity]) in run_matching order; *n_spikes and *n_rounds on the host. */
#define LSS_NOALLOC_MAX_SAMPLES 65536
int  lss_mp_rounds_noalloc(float* B_dev, int64_t ldb, int32_t n_templates, int32_t n_samples,
                           int32_t nt, float th_learned, const float* nm_dev,
                           const float* ctc_permuted_dev, int32_t max_rounds, int32_t capacity,
                           int32_t* spike_x, int32_t* spike_y, float* spike_amp,
                           int32_t* n_spikes, int32_t* n_rounds, void* stream);

/* Score field B f32 [T, N] of a filtered batch (template_matching.py:145-146). */
int  lss_scores(lss_handle* h, const float* X_dev, int64_t N, float* B_dev, void* stream);

/* One batch end to end: ingest (a), scores (b), matching pursuit (c), PC
 * features (d), time conversion and first-batch negative-time drop
 * (template_matching.py:46-73). Records are in run_matching order. Rows with
 * raw_on_device = 1 and records with out->on_device = 1 must be device or
 * pinned host memory (LSS_ERR_ARG otherwise). */
int  lss_sort_batch(lss_handle* h, const int16_t* raw, int64_t n_rows, int64_t ibatch,
                    int64_t n_batches, int32_t raw_on_device, lss_records* out, void* stream);

/* lss_sort_batch without any host wait, for pipelined submission: the
 * records must be device-accessible (device arrays, or pinned host memory,
 * which the kernels then write across the bus; out->on_device = 1), the
 * record count is written to count_dev (device or pinned memory) when the
 * batch's work finishes, and errors are collected until lss_sync (which waits
 * for the stream and returns the first error seen). Batches on one stream run
 * in order; drift changes between them (lss_set_drift) wait for the batch
 * before. Host rows (raw_on_device = 0) are uploaded on the handle's own
 * stream into one of two device buffers while the previous batch computes;
 * pinned rows must stay unchanged until the batch has finished. */
int  lss_sort_batch_async(lss_handle* h, const int16_t* raw, int64_t n_rows, int64_t ibatch,
                          int64_t n_batches, int32_t raw_on_device, lss_records* out, int64_t* count_dev,
                          void* stream);
int  lss_sync(lss_handle* h, void* stream);

/* Statistics of the last lss_match / lss_sort_batch: rounds run and spikes;
 * for the BF16 path, of the last scoring: columns whose decisions lay within
 * the re-check margin, decisions (best template or threshold side) the FP32
 * re-check changed, and columns re-scored in FP32 (whole 64-sample tiles). */
typedef struct lss_stats {
    int32_t rounds;
    int64_t spikes;
    int64_t recheck_columns;
    int64_t recheck_flips;
    int64_t launches;      /* kernels this handle has launched since creation */
    int64_t recheck_rescored;
    /* matching-pursuit update work items (spike segment x template-row block x
     * 32 columns) of the last synchronous batch, and how many of them changed
     * any score: the others were skipped as exact no-ops */
    int64_t mp_items;
    int64_t mp_items_updated;
    /* the rounds' time split, per CTA of the rounds kernel (mean over CTAs,
     * summed over the rounds of the last synchronous batch): peak phase,
     * waiting at the grid barrier after it, update phase, waiting after it;
     * and the slowest CTA's peak and update totals */
    int64_t mp_peak_ns, mp_peak_wait_ns, mp_update_ns, mp_update_wait_ns;
    int64_t mp_peak_max_ns, mp_update_max_ns;
} lss_stats;
int  lss_get_stats(const lss_handle* h, lss_stats* out);

/* Per-stage device time of the last lss_sort_batch, from CUDA events recorded
 * on the call's stream while profiling is on (the Timer scopes of
 * OnlineSpikesV2.cu:719-964, whose print is disabled at Timer.h:15). */
typedef struct lss_stage_times {
    float h2d_ms;       /* raw rows host -> device                      */
    float ingest_ms;    /* channel sums + mean + median CAR             */
    float highpass_ms;  /* circular highpass                            */
    float whiten_ms;    /* (M @ Wrot) @ X                               */
    float project_ms;   /* temporal-basis projection                    */
    float score_ms;     /* template score GEMM                          */
    float mp_ms;        /* matching-pursuit rounds (+ count read-back)  */
    float xres_ms;      /* residual                                     */
    float feature_ms;   /* PC features                                  */
    float records_ms;   /* record compaction + device -> host copies    */
    float total_ms;
} lss_stage_times;
int  lss_set_profiling(lss_handle* h, int32_t on);
int  lss_get_stage_times(const lss_handle* h, lss_stage_times* out);

/* ------------------------------------------------------------------------
 * One-time set-up on the GPU in FP64 (hot swap without Python).
 * lss_set_templates: new U [T, K, C] (same shapes) and optionally a new
 * wPCA [K, nt]; rebuilds nm, ctc (prepare_matching,
 * template_matching.py:110-121, in FP64 rounded to FP32), iU and Ucc
 * (template_matching.py:20-26, with the handle's iCC), the score GEMM's
 * operands, template waveforms and the basis correlations.
 * lss_set_drift_model: channel positions [C] and the interpolation width
 * (datashift.py:213-219: iKxx = (Kxx + 0.01 I)^-1, FP64 on the host, once);
 * lss_set_drift_shift: M = Kyx iKxx for a vertical shift in um
 * (preprocessing.py:44-69, one block) on the GPU, then as lss_set_drift. */
int  lss_set_templates(lss_handle* h, const float* U, const float* wPCA);
int  lss_set_drift_model(lss_handle* h, const float* xc, const float* yc, float sig_interp);
int  lss_set_drift_shift(lss_handle* h, double dshift);

/* ------------------------------------------------------------------------
 * Output formats of the reference's consumers (host records, host code).
 * lss_format_spike_lines: spikeOutput.txt lines "time,template,amplitude,y\n"
 * (OnlineSpikesV2::writeSpikesToFile, OnlineSpikesV2.cu:1117-1124) with time
 * + recording_offset, the template id or (use_cluster) the cluster, floats as
 * %g; y = y_pos or 0. lss_serialize_payload: the decoder's
 * OnlineSpikesPayload (onlineSpikesPayload.h:8-48) in cereal's binary
 * archive layout, `long` fields long_bytes (4 for the reference's Windows
 * build, 8 for LP64) wide. Both write at most cap bytes into buf (NULL: size
 * only) and return the full length, or -1 on bad arguments; a short buffer
 * gets a prefix (whole lines and a terminating NUL for the spike lines). */
int64_t lss_format_spike_lines(const lss_records* rec, int64_t recording_offset, int32_t use_cluster, char* buf,
                               int64_t cap);
int64_t lss_serialize_payload(const lss_records* rec, int64_t recording_offset, int64_t stream_sample_ct,
                              double vrms, float p2p, int64_t process_time, int32_t long_bytes, int32_t use_cluster,
                              uint8_t* buf, int64_t cap);

/* ------------------------------------------------------------------------
 * Reconstruction and its adjoint, for refining U and the temporal basis by
 * gradient on residual energy with the spike assignments held fixed. No
 * counterpart in the reference (Kilosort's reconstruction is the residual
 * update of template_matching.py:195-198; its templates are learned offline).
 *   R[c, s] = sum_i amp_i sum_k U[y_i, k, c] wPCA[k, s - x_i + nt/2]
 * dtype 0 = float32, 1 = float64 (every floating-point array in that type).
 * U [T, K, C], wPCA [K, nt], R / dR [C, N] row-major, device memory.
 * lss_recon_forward needs the spikes sorted by x (x_sorted and y, amp in the
 * same order). lss_recon_backward takes the spikes in any order plus
 * order_by_template (spike indices grouped by template) and
 * template_start [T + 1] (template t's spikes are
 * order_by_template[template_start[t] .. template_start[t+1])); it writes
 * dU [T, K, C], dwPCA [K, nt] and, when damp is not null, dL/damp [n]; work
 * holds T * K * nt elements. Both are deterministic.
 * ---------------------------------------------------------------------- */
int  lss_recon_forward(int32_t dtype, const void* U, const void* wPCA, int32_t T, int32_t K, int32_t C, int32_t nt,
                       const int32_t* x_sorted, const int32_t* y, const void* amp, int64_t n, void* R, int64_t N,
                       void* stream);
int  lss_recon_backward(int32_t dtype, const void* U, const void* wPCA, int32_t T, int32_t K, int32_t C, int32_t nt,
                        const int32_t* x, const void* amp, const int32_t* order_by_template,
                        const int32_t* template_start, const void* dR, int64_t N, void* dU, void* dwPCA,
                        void* damp, void* work, void* stream);

/* ------------------------------------------------------------------------
 * Streaming serving loop. No counterpart in the reference as an API: there
 * each probe runs its own OnlineSpikesV2 object on its own thread
 * (main.cpp:77-85), whose runSpikeSorting loop (OnlineSpikesV2.cu:632-820)
 * fetches the latest window from the acquisition socket, sorts it with
 * synchronous copies and writes spikeOutput.txt.
 *
 * Here one server owns a device and admits probe streams while device memory
 * and probe slots allow (LSS_ERR_BUSY otherwise: retry after a release). Each
 * probe has its own sorter handle (its own templates and T), CUDA stream,
 * device ring of raw int16 rows and one CUDA graph, captured at admission,
 * that sorts one batch of cfg->batch_size (= NT) samples end to end with no
 * host synchronisation. Probes' graphs run concurrently on the device.
 *
 * Stream batch b (b = 0, 1, ...) is launched as soon as its NT-sample block
 * has arrived: its window is stream rows [b*NT - 2nt, (b+1)*NT) (rows before
 * the stream start replicate row 0) and it sorts samples [b*NT - nt,
 * (b+1)*NT - nt), i.e. Kilosort's batch semantics on the stream delayed by nt
 * samples, so no batch waits for the next block. Record times are stream
 * samples in Kilosort's convention (trough-aligned: + nt0min - nt/2);
 * negative times are dropped. Results land in pinned host memory written by
 * the device; arrival-to-emit latency is measured from the arrival time given
 * to lss_server_push for the block's last row to the moment the server sees
 * the batch's completion event (in lss_server_poll, or in a push that waits
 * for the batch's slot).
 * ---------------------------------------------------------------------- */
typedef struct lss_server lss_server;

int  lss_server_create(int32_t device, int64_t memory_budget_bytes, int32_t max_probes, lss_server** out);
void lss_server_destroy(lss_server* s);
/* Admits a probe: creates its handle from (cfg, t), applies the drift matrix
 * M [C, C] and the post-processing when given, allocates its ring (`depth` batches in flight) and
 * result ring (`capacity` records per batch) and captures its graph.
 * LSS_ERR_BUSY when no slot is free or the handle would exceed the budget. */
int  lss_server_admit(lss_server* s, const lss_config* cfg, const lss_tensors* t, const float* drift_M,
                      const lss_post_config* post, int32_t depth, int64_t capacity, int32_t* probe);
/* Appends n_rows raw int16 rows [n_rows, n_chan_bin] (host) to the probe's
 * stream; every completed NT-row block launches its batch. arrival_ns: host
 * CLOCK_MONOTONIC time the rows arrived (<= 0: now). Blocks only when `depth`
 * batches are already in flight. */
int  lss_server_push(lss_server* s, int32_t probe, const int16_t* rows, int64_t n_rows, int64_t arrival_ns);
/* Oldest finished batch's records into `out` (host arrays); *batch = its
 * index, or -1 when none is finished (wait = 0) or none is in flight. */
int  lss_server_poll(lss_server* s, int32_t probe, lss_records* out, int64_t* batch, int32_t wait);
/* Waits for the probe's batches and frees its slot; finished batches not yet
 * polled are dropped. Its device and pinned memory are freed by a later
 * admission that needs the room (released + admitted + the largest probe so
 * far over the budget) or by lss_server_destroy: a free waits for the whole
 * device, which the other probes' batches would see as latency. */
int  lss_server_release(lss_server* s, int32_t probe);
/* Replaces the probe's drift matrix after its in-flight batches finish. */
int  lss_server_set_drift(lss_server* s, int32_t probe, const float* drift_M);
/* Arrival-to-emit latency percentiles (ms) over the probe's polled batches. */
int  lss_server_latency(lss_server* s, int32_t probe, double* p50_ms, double* p99_ms, int64_t* batches);
/* Every polled batch's arrival-to-emit latency (ms), in batch order: up to
 * capacity values into out_ms, *n = how many there are. */
int  lss_server_latencies(lss_server* s, int32_t probe, double* out_ms, int64_t capacity, int64_t* n);
/* The same latencies split in four (ms, 4 per batch, batch order, up to
 * capacity batches; *n = how many batches there are): arrival -> graph launch
 * (host), launch -> the batch's first kernel starts (queued behind the
 * stream's or the device's other work), first kernel start -> last kernel
 * end (device), last kernel end -> completion seen. The parts sum to the
 * latency; the device times are mapped to the host clock by an offset taken
 * at admission (error a few us). */
int  lss_server_latency_parts(lss_server* s, int32_t probe, double* out_ms, int64_t capacity, int64_t* n);
/* Device memory held by admitted probes (released ones not counted) and the
 * budget, in bytes. */
int  lss_server_memory(lss_server* s, int64_t* used, int64_t* budget);

#ifdef __cplusplus
}
#endif
#endif /* LSS_H_ */
