// Internal: the sorter handle behind the C ABI (include/lss.h) and the
// stage functions shared by the batch entry points (lss_api.cpp) and the
// streaming loop (serve.cpp). Every device buffer is allocated once by
// lss_create; the stages only enqueue work on the caller's stream.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "lss.h"
#include "lss_kernels.cuh"

namespace lss {

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t alloc(size_t count) {
        n = count;
        return cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(count, 1) * sizeof(T));
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
    }
};

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

}  // namespace lss

using lss::DevBuf;

struct lss_handle {
    lss_config cfg{};
    std::string err;
    int C = 0, Cbin = 0, T = 0, K = 0, nt = 0, nC = 0, NT = 0, N = 0;
    int64_t ld = 0;
    int hpL = -1;  // FIR half length; -1 = no highpass
    int mp_grid = 0;
    size_t dev_bytes = 0;                        // device memory allocated by lss_create
    std::vector<float> h_hp;
    lss_stats stats{};
    bool prof = false;
    bool capturing = false;                      // inside a graph capture: no host-side copies or timing events
    bool streaming = false;                      // owned by a serving loop: the batch entry points are refused
    cudaEvent_t ev[11] = {};
    lss_stage_times times{};

    void mark(int i, cudaStream_t s) {
        if (prof) cudaEventRecord(ev[i], s);
    }

    DevBuf<int16_t> raw;
    DevBuf<int32_t> chan_map;
    DevBuf<long long> sums;
    DevBuf<float> taps, Mw, Wrot, Mdrift, X1, Xh, X, B, nm, ctcP, wave, wpca, Ucc, Xres, tF;
    DevBuf<int64_t> iCC, iU;
    DevBuf<float> cfmax;
    DevBuf<int32_t> imax, blk_cnt, blk_x, blk_y, sp_x, sp_y, sp_round, round_start, counters, status;
    DevBuf<float> sp_amp, blk_amp;
    DevBuf<unsigned long long> colkey;
    // block-skipping rounds (mp_blocks.cu): template rows in blocks of
    // MPB_ROWS ordered along the probe, |ctc| maxima, per-block column state
    bool un_p_stale = true;                      // plain-template norms (BF16 bound) need recomputing
    bool mp_skip = false;                        // rounds kernel: block-skipping (mp_blocks.cu) or full (mp.cu)
    int mp_nb = 0;
    DevBuf<int32_t> mp_perm;
    DevBuf<float> mp_cmaxr, mp_bmin;
    DevBuf<unsigned long long> mp_bkey;
    DevBuf<unsigned long long> mp_phase;         // [6] phase clock of the rounds kernel
    DevBuf<int4> mp_ent;                         // block-skipping rounds: per-CTA lists of blocks to process
    DevBuf<int32_t> mp_ent_cnt;                  // [grid] entries per list
    DevBuf<int32_t> mp_rowof;                    // [T] score row of each template in probe order
    DevBuf<unsigned long long> sc_part_keys;     // [passes, ld] score GEMM: per-pass best keys (error-bound split)
    DevBuf<float> sc_part;                       // [passes, 4, ld] per-pass bound partials
    DevBuf<float> mp_ctcq;                       // [T, T, 2nt+1] ctc rows in probe order
    // BF16 path (BF16x3 GEMM): projection and templates as bf16 hi / lo splits
    DevBuf<__nv_bfloat16> B0T, B0T16lo, Up16, Up16lo;
    DevBuf<float> B0T_hi, B0T_lo, Up_hi, Up_lo;  // FP32 path (3xTF32): tf32 hi/lo splits
    DevBuf<__nv_bfloat16> Uw16, Uw16lo;          // templates with the whitening folded in (BF16 path)
    DevBuf<float> Uw_hi, Uw_lo;                  // ... (FP32 path)
    DevBuf<float> U, R;                          // U [T,K,C]; R [K,K,2nt-1] basis lag correlations
    DevBuf<float2> hpH, hpTw;                    // highpass spectrum and twiddles (FFT form)
    // BF16 re-check: largest other upper bound of Cf, bounds of the best Cf, saved maxima,
    // projection rows of the listed columns, ||P_s||^2, template norms (folded / plain)
    DevBuf<float> cf2, cf_lo, cf_hi, pre_cf, Pc_hi, Pc_lo, pn2, un_w, un_p;
    DevBuf<int32_t> rc_cols, pre_im, rc_count;   // ... listed columns, saved argmax, [columns, flips, columns]
    int32_t* rc_host = nullptr;                  // pinned copy of rc_count (read by lss_get_stats)
    cudaEvent_t rc_ev = nullptr;                 // recorded after that copy
    cudaEvent_t mix_ev = nullptr;                // recorded after the whitening-folded templates are rebuilt
    cudaEvent_t batch_ev = nullptr;              // recorded after each batch's work (template rebuilds wait for it)
    // pinned staging of drift matrices: a ring, so that a caller submitting
    // batches ahead waits for the upload M_PIN_SLOTS matrices back, not the last
    static constexpr int M_PIN_SLOTS = 16;
    float* m_pin = nullptr;                      // [M_PIN_SLOTS][C][C]
    cudaEvent_t m_pin_ev[M_PIN_SLOTS] = {};      // recorded after each slot's last upload
    int m_pin_next = 0;
    DevBuf<int32_t> status_acc;                  // errors of asynchronous batches since the last lss_sync
    bool rc_pending = false;
    int64_t last_scored = 0;                     // samples of the last BF16 scoring
    int CKpad = 0;
    int sm_count = 0;
    DevBuf<unsigned int> bar;
    DevBuf<int64_t> rec_time, rec_count;
    DevBuf<int32_t> rec_tmpl, rec_slot;
    // post-processing (positions, clusters, duplicates, time order)
    bool post = false;
    lss::PostArgs pa;
    DevBuf<unsigned long long> pk;               // 4 key arrays of max_spikes
    DevBuf<unsigned char> psort, pkeep;
    DevBuf<int64_t> plast;
    DevBuf<float> pxy, pcen, pchan;              // per-spike x|y, centroids x|y, channel x|y
    DevBuf<int32_t> pclu;
    DevBuf<float> rec_x, rec_y;                  // host-records staging of x, y, cluster
    DevBuf<int32_t> rec_clu;
    // drift model on the device: channel positions (x | y) and (Kxx + 0.01 I)^-1, FP64
    DevBuf<double> dm_pos, dm_ik;
    float dm_sig = 20.f;
    DevBuf<float> rec_amp, rec_pc;
    // asynchronous batches from host memory: the rows are uploaded on their
    // own stream into one of two device buffers, so that a batch's upload
    // overlaps the work of the batch before it
    DevBuf<int16_t> raw_up[2];
    cudaStream_t up_s = nullptr;
    cudaEvent_t up_done[2] = {}, raw_free[2] = {};
    int raw_next = 0;

    unsigned long long mp_phase_host[6] = {};    // host copy of mp_phase after a synchronous batch
    void set_phase_stats() {
        const int64_t g = std::max(1, mp_grid);
        stats.mp_peak_ns = (int64_t)(mp_phase_host[0] / g);
        stats.mp_peak_wait_ns = (int64_t)(mp_phase_host[1] / g);
        stats.mp_update_ns = (int64_t)(mp_phase_host[2] / g);
        stats.mp_update_wait_ns = (int64_t)(mp_phase_host[3] / g);
        stats.mp_peak_max_ns = (int64_t)mp_phase_host[4];
        stats.mp_update_max_ns = (int64_t)mp_phase_host[5];
    }

    int fail(int code, const std::string& m) {
        err = m;
        return code;
    }
    int cuda_fail(cudaError_t e, const char* where) {
        err = std::string(where) + ": " + cudaGetErrorString(e);
        return LSS_ERR_CUDA;
    }
    ~lss_handle() {
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess && dev != cfg.device) cudaSetDevice(cfg.device);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (up_s) cudaStreamSynchronize(up_s);
        for (int i = 0; i < 2; ++i) {
            raw_up[i].release();
            if (up_done[i]) cudaEventDestroy(up_done[i]);
            if (raw_free[i]) cudaEventDestroy(raw_free[i]);
        }
        if (up_s) cudaStreamDestroy(up_s);
        raw.release(); chan_map.release(); sums.release(); taps.release(); Mw.release(); Wrot.release(); Mdrift.release();
        X1.release(); Xh.release(); X.release(); B.release();
        nm.release(); ctcP.release(); wave.release(); wpca.release(); Ucc.release(); Xres.release();
        tF.release(); iCC.release(); iU.release(); cfmax.release(); imax.release(); blk_cnt.release();
        blk_x.release(); blk_y.release(); sp_x.release(); sp_y.release(); sp_round.release();
        round_start.release(); counters.release(); status.release(); sp_amp.release(); blk_amp.release(); colkey.release();
        mp_perm.release(); mp_cmaxr.release(); mp_phase.release(); mp_ent.release(); mp_ent_cnt.release(); mp_rowof.release(); mp_ctcq.release(); sc_part_keys.release(); sc_part.release(); mp_bmin.release(); mp_bkey.release();
        bar.release(); rec_time.release(); rec_count.release(); rec_tmpl.release(); rec_slot.release(); rec_amp.release();
        rec_pc.release(); B0T.release(); B0T16lo.release(); Up16.release(); Up16lo.release();
        B0T_hi.release(); B0T_lo.release(); Up_hi.release(); Up_lo.release();
        Uw16.release(); Uw16lo.release(); Uw_hi.release(); Uw_lo.release(); U.release(); R.release(); hpH.release(); hpTw.release();
        cf2.release(); cf_lo.release(); cf_hi.release(); pre_cf.release(); Pc_hi.release(); Pc_lo.release();
        pn2.release(); un_w.release(); un_p.release(); rc_cols.release(); pre_im.release();
        rc_count.release();
        pk.release(); psort.release(); pkeep.release(); plast.release(); pxy.release(); pcen.release();
        pchan.release(); pclu.release(); rec_x.release(); rec_y.release(); rec_clu.release();
        dm_pos.release(); dm_ik.release();
        if (rc_ev) cudaEventDestroy(rc_ev);
        if (mix_ev) cudaEventDestroy(mix_ev);
        if (batch_ev) cudaEventDestroy(batch_ev);
        for (cudaEvent_t e : m_pin_ev)
            if (e) cudaEventDestroy(e);
        if (m_pin) cudaFreeHost(m_pin);
        status_acc.release();
        if (rc_host) cudaFreeHost(rc_host);
    }
};

#define CK(call)                                                   \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return h->cuda_fail(e_, #call);     \
    } while (0)

namespace lss {

// Ingest (channel sums, CAR, highpass; optional whitening into Xout) of the
// batch whose raw rows `src` (device) are read through `map`.
int run_ingest(lss_handle* h, const int16_t* src, const IngestMap& map, float* Xout, cudaStream_t s,
               const float** pre_out);
// Projection and score GEMM of X [C, ldx] into B; *maxima_ready when the
// column maxima were fused into the GEMM. rows_for_mp: B rows in the order
// the selected rounds kernel reads (probe order for the block-skipping one).
int run_scores(lss_handle* h, const float* X, int64_t ldx, int64_t N, float* B, cudaStream_t s,
               bool* maxima_ready = nullptr, bool folded = false, bool rows_for_mp = true);
// Whitening-folded template operands from U and Mw (after a template or drift change).
int rebuild_uw(lss_handle* h);
// Orders stream s after the last template / drift rebuild (no host wait).
inline cudaError_t wait_mixing(lss_handle* h, cudaStream_t s) {
    return h->mix_ev ? cudaStreamWaitEvent(s, h->mix_ev, 0) : cudaSuccess;
}
// Template order and |ctc| maxima of the block-skipping rounds (after the
// templates or ctc change; synchronous).
int rebuild_mp_blocks(lss_handle* h);
// Mw = Mdrift @ Wrot with Mdrift already on the device, then rebuild_uw.
int mix_device_drift(lss_handle* h);
// Matching-pursuit rounds on h->B, enqueued only (counts stay on the device).
int enqueue_mp(lss_handle* h, int64_t N, cudaStream_t s, bool maxima_ready);
// Record slots / count for the batch's spikes (post-processing when on, else
// the matching order with the first-batch drop), then the records themselves.
// n_bound: the spike count, or an upper bound when rc reads it from the device.
int enqueue_records(lss_handle* h, const RecordClock& rc, int32_t n_bound, bool with_pc, bool tf_ready,
                    int64_t* time, int32_t* tmpl, float* amp, float* pc, float* x, float* y, int32_t* clu,
                    int64_t cap, int64_t* count, cudaStream_t s);

}  // namespace lss
