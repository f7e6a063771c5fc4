// Streaming serving loop (lss_server_* in include/lss.h).
//
// The reference runs one OnlineSpikesV2 object per probe on its own host
// thread (main.cpp:77-85); each loop iteration of runSpikeSorting
// (OnlineSpikesV2.cu:632-820) fetches the latest window, copies it to the
// device synchronously, sorts it and copies the spikes back. Here a server
// owns one device and admits several probe streams; each probe's batch is a
// CUDA graph (captured once per probe, i.e. per batch length and template
// set) that reads its window straight from a device ring of raw rows and
// writes its records into pinned host memory, so a batch costs one H2D copy
// of the new block, one graph launch and one event, and batches of
// different probes overlap on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "lss.h"
#include "lss_handle.h"
#include "lss_kernels.cuh"

namespace lss {

// Per-batch summary the graph's last kernel writes to pinned host memory.
struct StreamMail {
    int64_t batch;
    int32_t spikes, rounds, status, pad;
    int64_t t_begin, t_end;  // device global timer (ns) at the graph's first and last kernel
};

__device__ __forceinline__ int64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return (int64_t)t;
}

// Clock ping through mapped pinned memory: the kernel announces itself
// (ping[0] = 5), waits for the host's go (ping[0] == 1), reads the global timer
// at once, stores it in ping[1] and answers (ping[0] = 2). The wait gives up
// after 1 s of device time (ping[0] = 3, no timestamp).
__global__ void k_clock_ping(volatile int64_t* ping) {
    ping[0] = 5;
    __threadfence_system();
    const int64_t t0 = global_timer_ns();
    while (ping[0] != 1) {
        if (global_timer_ns() - t0 > 1000000000ll) {
            ping[0] = 3;
            return;
        }
    }
    ping[1] = global_timer_ns();
    __threadfence_system();
    ping[0] = 2;
}

// state[0] = batch index (starts at -1), state[1] = first stream row of the
// batch window, state[2] = device time at which the batch's work began.
__global__ void k_stream_begin(int64_t* state, int64_t NT, int64_t lead) {
    const int64_t b = state[0] + 1;
    state[0] = b;
    state[1] = b * NT - lead;
    state[2] = global_timer_ns();
}

__global__ void k_stream_end(const int64_t* state, const int32_t* counters, const int32_t* status, StreamMail* mail,
                             int32_t slots) {
    const int64_t b = state[0];
    StreamMail m;
    m.batch = b;
    m.spikes = counters[0];
    m.rounds = counters[1];
    m.status = *status;
    m.pad = 0;
    m.t_begin = state[2];
    m.t_end = global_timer_ns();
    mail[b % slots] = m;
}

static int64_t now_ns() {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

}  // namespace lss

using namespace lss;

namespace {

// One in-flight batch. Its completion is an event recorded behind the
// batch's graph and queried by the thread that polls: a host callback in the
// stream would hold the stream's next batch back until the driver's callback
// thread had run it, and that thread was seen to run tens of ms late.
struct Slot {
    cudaEvent_t ev = nullptr;
    int64_t batch = -1;
    int64_t arrival_ns = 0;
    int64_t launch_ns = 0;
    int64_t emit_ns = 0;
};

struct Result {
    int64_t batch = -1;
    int32_t status = 0;
    int64_t count = 0;
    std::vector<int64_t> time;
    std::vector<int32_t> tmpl;
    std::vector<float> amp;
    std::vector<float> pc;
    std::vector<float> x, y;
    std::vector<int32_t> clu;
};

template <typename T>
struct HostBuf {
    T* p = nullptr;
    T* d = nullptr;  // device alias of mapped memory
    cudaError_t alloc(size_t n, bool mapped) {
        cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T),
                                      mapped ? cudaHostAllocMapped : cudaHostAllocDefault);
        if (e != cudaSuccess) return e;
        std::memset(p, 0, std::max<size_t>(n, 1) * sizeof(T));
        if (mapped) return cudaHostGetDevicePointer(reinterpret_cast<void**>(&d), p, 0);
        return cudaSuccess;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = d = nullptr;
    }
};

struct Probe {
    lss_handle* h = nullptr;
    cudaStream_t s = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t NT = 0, nt = 0, Cbin = 0, R = 0, D = 0, cap = 0, feat = 0;
    DevBuf<int16_t> ring;
    DevBuf<int64_t> state;
    HostBuf<int16_t> staging;                  // D blocks of NT rows
    HostBuf<int64_t> o_time, o_count;
    HostBuf<int32_t> o_tmpl;
    HostBuf<float> o_amp, o_pc, o_x, o_y;
    HostBuf<int32_t> o_clu;
    HostBuf<StreamMail> mail;
    std::unique_ptr<Slot[]> slots;
    int64_t fill = 0;                          // rows in the block being assembled
    int64_t next = 0;                          // next batch to launch
    int64_t harvest = 0;                       // next batch to harvest
    std::deque<Result> ready;
    std::vector<double> lat_ms;
    std::vector<double> parts_ms;              // 4 per batch, lss_server_latency_parts
    int64_t gpu_offset_ns = 0;                 // host steady clock - device global timer
    size_t bytes = 0;
    std::mutex m;
    std::string err;

    int fail(int code, const std::string& msg) {
        err = msg;
        lss::set_thread_error(msg.c_str());
        return code;
    }
    ~Probe() {
        if (s) cudaStreamSynchronize(s);
        for (int64_t i = 0; slots && i < D; ++i)
            if (slots[i].ev) cudaEventDestroy(slots[i].ev);
        if (exec) cudaGraphExecDestroy(exec);
        if (s) cudaStreamDestroy(s);
        ring.release();
        state.release();
        staging.release();
        o_time.release();
        o_count.release();
        o_tmpl.release();
        o_amp.release();
        o_pc.release();
        o_x.release();
        o_y.release();
        o_clu.release();
        mail.release();
        if (h) lss_destroy(h);
    }
};

#define PCK(call)                                                                   \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) return p->fail(LSS_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

// The batch's device work, enqueued on p->s (captured into the probe's graph).
int enqueue_stream_batch(Probe* p) {
    lss_handle* h = p->h;
    cudaStream_t s = p->s;
    k_stream_begin<<<1, 1, 0, s>>>(p->state.p, p->NT, 2 * p->nt);
    PCK(cudaGetLastError());
    IngestMap map;
    map.base_dev = p->state.p + 1;
    map.ring_rows = p->R;
    const float* Xh = nullptr;
    int rc = run_ingest(h, p->ring.p, map, nullptr, s, &Xh);
    if (rc) return p->fail(rc, h->err);
    PCK(cudaMemsetAsync(h->status.p, 0, sizeof(int32_t), s));
    bool ready = false;
    rc = run_scores(h, Xh, h->ld, h->N, h->B.p, s, &ready, /*folded=*/true);
    if (rc) return p->fail(rc, h->err);
    rc = enqueue_mp(h, h->N, s, ready);
    if (rc) return p->fail(rc, h->err);
    const bool bf16 = h->cfg.precision == LSS_PREC_BF16_RECHECK;
    if (p->feat > 0) {
        const int grid = (int)std::min<int64_t>(p->cap, 2 * (int64_t)h->sm_count);
        PCK(launch_pc_features_folded(Xh, h->ld, h->C, h->nt, h->K, h->nC, h->T, h->wpca.p, h->Mw.p, h->U.p,
                                      h->R.p, h->iCC.p, h->iU.p, h->Ucc.p, h->sp_x.p, h->sp_y.p, h->sp_amp.p,
                                      h->round_start.p, 0, grid, h->counters.p, h->tF.p, h->status.p,
                                      bf16 ? (const void*)h->B0T.p : (const void*)h->B0T_hi.p,
                                      bf16 ? (const void*)h->B0T16lo.p : (const void*)h->B0T_lo.p, bf16 ? 1 : 0,
                                      h->CKpad, s));
    }
    RecordClock rclk;
    rclk.ibatch_dev = p->state.p;
    rclk.counters = h->counters.p;
    rclk.shift = -p->nt;
    rclk.NT = (int32_t)p->NT;
    rclk.nt = (int32_t)p->nt;
    rclk.nt0min = h->cfg.nt0min;
    rclk.slots = (int32_t)p->D;
    rc = enqueue_records(h, rclk, (int32_t)std::min<int64_t>(p->cap, h->cfg.max_spikes), p->feat > 0, p->feat > 0,
                         p->o_time.d, p->o_tmpl.d, p->o_amp.d, p->feat > 0 ? p->o_pc.d : nullptr, p->o_x.d, p->o_y.d,
                         p->o_clu.d, p->cap, p->o_count.d, s);
    if (rc) return p->fail(rc, h->err);
    k_stream_end<<<1, 1, 0, s>>>(p->state.p, h->counters.p, h->status.p, p->mail.d, (int32_t)p->D);
    PCK(cudaGetLastError());
    return LSS_OK;
}

int capture(Probe* p) {
    lss_handle* h = p->h;
    const bool prof = h->prof;
    h->prof = false;
    h->capturing = true;
    cudaGraph_t g = nullptr;
    PCK(cudaStreamBeginCapture(p->s, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_stream_batch(p);
    const cudaError_t e = cudaStreamEndCapture(p->s, &g);
    h->capturing = false;
    h->prof = prof;
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return p->fail(LSS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(&p->exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return p->fail(LSS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
    // one launch on the zeroed ring (no spikes) so that the stream's first
    // batch does not pay for the graph's upload and first-launch set-up; the
    // stream state is reset afterwards
    PCK(cudaGraphUpload(p->exec, p->s));
    PCK(cudaGraphLaunch(p->exec, p->s));
    const int64_t init[2] = {-1, 0};
    PCK(cudaMemcpyAsync(p->state.p, init, sizeof(init), cudaMemcpyHostToDevice, p->s));
    PCK(cudaStreamSynchronize(p->s));
    const StreamMail m0 = p->mail.p[0];
    if (m0.status != 0 || m0.spikes != 0)
        return p->fail(LSS_ERR_STATE, "warm-up launch of the stream graph did not come back clean");
    return LSS_OK;
}

// Offset from the device's global timer to the host's steady clock. In each
// of a few pings (k_clock_ping) the device reads its timer at a host moment
// between t_go (the host wrote the go flag) and t_seen (the host saw the
// answer), so offset = that moment - timestamp lies in [t_go - g, t_seen - g];
// the ping with the narrowest bracket (a few us: two transfers over the bus)
// gives the midpoint. With that bound, device timestamps map to host times
// that keep the launch -> device start -> device end -> seen order.
int calibrate_clock(Probe* p) {
    struct Ping {
        HostBuf<int64_t> b;
        ~Ping() { b.release(); }
    } ping;
    PCK(ping.b.alloc(2, true));
    volatile int64_t* hp = ping.b.p;
    int64_t best = INT64_MAX;
    for (int i = 0; i < 16; ++i) {
        hp[0] = 0;
        hp[1] = 0;
        k_clock_ping<<<1, 1, 0, p->s>>>(ping.b.d);
        PCK(cudaGetLastError());
        const int64_t w0 = lss::now_ns();
        bool started = false;
        while (lss::now_ns() - w0 < 1000000000ll)
            if (hp[0] == 5) { started = true; break; }
        const int64_t t_go = lss::now_ns();
        hp[0] = 1;
        int64_t t_seen = 0;
        while (started && lss::now_ns() - t_go < 1000000000ll)
            if (hp[0] == 2) { t_seen = lss::now_ns(); break; }
        PCK(cudaStreamSynchronize(p->s));
        if (!t_seen || hp[0] != 2) continue;  // the device gave up waiting: no sample
        const int64_t g = hp[1];
        if (t_seen - t_go < best) {
            best = t_seen - t_go;
            p->gpu_offset_ns = t_go + (t_seen - t_go) / 2 - g;
        }
    }
    if (best == INT64_MAX) return p->fail(LSS_ERR_CUDA, "device clock calibration got no answer");
    return LSS_OK;
}

// Moves the oldest in-flight batch's results into p->ready (waits for it when
// `wait`). Caller holds p->m through `lk`. Returns LSS_OK (possibly nothing
// moved when !wait), or an error.
int harvest_one(Probe* p, std::unique_lock<std::mutex>& lk, bool wait) {
    if (p->harvest >= p->next) return LSS_OK;
    Slot& sl = p->slots[p->harvest % p->D];
    // the device work is bounded (every wait in the kernels gives up), so
    // this wait ends; 60 s covers a cold first launch
    const auto t0 = std::chrono::steady_clock::now();
    cudaError_t q;
    while ((q = cudaEventQuery(sl.ev)) == cudaErrorNotReady) {
        if (!wait) return LSS_OK;
        if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(60))
            return p->fail(LSS_ERR_TIMEOUT, "stream batch did not finish within 60 s");
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    if (q != cudaSuccess) return p->fail(LSS_ERR_CUDA, std::string("stream batch: ") + cudaGetErrorString(q));
    sl.emit_ns = lss::now_ns();
    const int64_t k = p->harvest % p->D;
    const StreamMail mail = p->mail.p[k];
    Result r;
    r.batch = sl.batch;
    r.status = mail.status;
    if (mail.batch != sl.batch) r.status |= 1 << 30;  // mailbox out of step: report as a state error
    r.count = p->o_count.p[k];
    const int64_t n = std::min<int64_t>(r.count, p->cap);
    r.time.assign(p->o_time.p + k * p->cap, p->o_time.p + k * p->cap + n);
    r.tmpl.assign(p->o_tmpl.p + k * p->cap, p->o_tmpl.p + k * p->cap + n);
    r.amp.assign(p->o_amp.p + k * p->cap, p->o_amp.p + k * p->cap + n);
    if (p->feat > 0)
        r.pc.assign(p->o_pc.p + (k * p->cap) * p->feat, p->o_pc.p + (k * p->cap + n) * p->feat);
    if (p->o_x.p) {
        r.x.assign(p->o_x.p + k * p->cap, p->o_x.p + k * p->cap + n);
        r.y.assign(p->o_y.p + k * p->cap, p->o_y.p + k * p->cap + n);
        r.clu.assign(p->o_clu.p + k * p->cap, p->o_clu.p + k * p->cap + n);
    }
    p->lat_ms.push_back((double)(sl.emit_ns - sl.arrival_ns) * 1e-6);
    // the host and device clocks drift apart by a few ppm: each batch brackets
    // the offset between launch - t_begin (the device began after the host
    // launched) and emit - t_end (the host saw completion after the device
    // ended); the estimate is pulled into that bracket when it has drifted out
    p->gpu_offset_ns = std::max(p->gpu_offset_ns, sl.launch_ns - mail.t_begin);
    p->gpu_offset_ns = std::min(p->gpu_offset_ns, sl.emit_ns - mail.t_end);
    const int64_t beg = mail.t_begin + p->gpu_offset_ns, end = mail.t_end + p->gpu_offset_ns;
    const double parts[4] = {(double)(sl.launch_ns - sl.arrival_ns) * 1e-6, (double)(beg - sl.launch_ns) * 1e-6,
                             (double)(end - beg) * 1e-6, (double)(sl.emit_ns - end) * 1e-6};
    p->parts_ms.insert(p->parts_ms.end(), parts, parts + 4);
    p->harvest += 1;
    p->ready.push_back(std::move(r));
    return LSS_OK;
}

int launch_block(Probe* p, int64_t arrival_ns) {
    const int64_t b = p->next;
    const int64_t k = b % p->D;
    PCK(cudaMemcpyAsync(p->ring.p + ((b * p->NT) % p->R) * p->Cbin, p->staging.p + k * p->NT * p->Cbin,
                        (size_t)(p->NT * p->Cbin) * sizeof(int16_t), cudaMemcpyHostToDevice, p->s));
    Slot& sl = p->slots[k];
    sl.batch = b;
    sl.launch_ns = lss::now_ns();
    sl.arrival_ns = arrival_ns > 0 ? arrival_ns : sl.launch_ns;
    PCK(cudaGraphLaunch(p->exec, p->s));
    PCK(cudaEventRecord(sl.ev, p->s));
    p->next = b + 1;
    return LSS_OK;
}

}  // namespace

struct lss_server {
    int device = 0;
    int64_t budget = 0, used = 0;
    std::vector<std::unique_ptr<Probe>> probes;
    // Released probes, kept whole until an admission needs their room or the
    // server is destroyed: freeing device and pinned memory waits for the
    // whole device and holds the driver up, which would show as latency on
    // every other probe's batches.
    std::vector<std::unique_ptr<Probe>> retired;
    int64_t retired_bytes = 0;
    int64_t largest = 0;  // bytes of the largest probe admitted so far
    std::mutex m;
};

namespace {
void free_retired(lss_server* s) {
    s->retired.clear();
    s->retired_bytes = 0;
}
}  // namespace

extern "C" {

int lss_server_create(int32_t device, int64_t memory_budget_bytes, int32_t max_probes, lss_server** out) {
    if (!out || max_probes <= 0 || memory_budget_bytes <= 0) {
        lss::set_thread_error("lss_server_create: bad argument");
        return LSS_ERR_ARG;
    }
    auto* s = new lss_server;
    s->device = device;
    s->budget = memory_budget_bytes;
    s->probes.resize(max_probes);
    *out = s;
    return LSS_OK;
}

void lss_server_destroy(lss_server* s) {
    if (!s) return;
    cudaSetDevice(s->device);
    s->probes.clear();
    free_retired(s);
    delete s;
}

int lss_server_admit(lss_server* s, const lss_config* cfg, const lss_tensors* t, const float* drift_M,
                     const lss_post_config* post, int32_t depth, int64_t capacity, int32_t* probe) {
    if (!s || !cfg || !t || !probe || depth < 1 || depth > 64 || capacity <= 0) {
        lss::set_thread_error("lss_server_admit: bad argument");
        return LSS_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(s->m);
    int slot = -1;
    for (size_t i = 0; i < s->probes.size(); ++i)
        if (!s->probes[i]) { slot = (int)i; break; }
    if (slot < 0) {
        lss::set_thread_error("no probe slot free");
        return LSS_ERR_BUSY;
    }
    if (cfg->device != s->device) {
        lss::set_thread_error("probe config names another device than the server's");
        return LSS_ERR_ARG;
    }
    cudaSetDevice(s->device);
    if (!s->retired.empty() && s->used + s->retired_bytes + s->largest > s->budget) free_retired(s);
    auto p = std::make_unique<Probe>();
    int rc = lss_create(cfg, t, &p->h);
    if (rc) return rc;
    lss_handle* h = p->h;
    p->NT = h->NT;
    p->nt = h->nt;
    p->Cbin = h->Cbin;
    p->D = depth;
    p->cap = capacity;
    p->feat = (h->nC > 0 && h->iCC.p) ? (int64_t)h->nC * h->K : 0;
    // ring: the oldest in-flight window plus the blocks written behind it
    const int64_t win = p->NT + 2 * p->nt;
    p->R = ((win + p->NT - 1) / p->NT + depth) * p->NT;
    const size_t ring_bytes = (size_t)p->R * p->Cbin * sizeof(int16_t);
    p->bytes = h->dev_bytes + ring_bytes + 3 * sizeof(int64_t);
    if (s->used + (int64_t)p->bytes > s->budget) {
        lss::set_thread_error("device memory budget exhausted");
        return LSS_ERR_BUSY;  // p's destructor frees the handle
    }
    auto cfail = [&](cudaError_t e, const char* what) {
        lss::set_thread_error((std::string(what) + ": " + cudaGetErrorString(e)).c_str());
        return LSS_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&p->s, cudaStreamNonBlocking)) != cudaSuccess) return cfail(e, "stream");
    if ((e = p->ring.alloc((size_t)p->R * p->Cbin)) != cudaSuccess) return cfail(e, "ring");
    if ((e = p->state.alloc(3)) != cudaSuccess) return cfail(e, "state");
    const int64_t init[2] = {-1, 0};
    if ((e = cudaMemcpy(p->state.p, init, sizeof(init), cudaMemcpyHostToDevice)) != cudaSuccess)
        return cfail(e, "state");
    if ((e = cudaMemset(p->ring.p, 0, ring_bytes)) != cudaSuccess) return cfail(e, "ring");
    if ((e = p->staging.alloc((size_t)depth * p->NT * p->Cbin, false)) != cudaSuccess) return cfail(e, "staging");
    if ((e = p->o_time.alloc((size_t)depth * capacity, true)) != cudaSuccess) return cfail(e, "records");
    if ((e = p->o_tmpl.alloc((size_t)depth * capacity, true)) != cudaSuccess) return cfail(e, "records");
    if ((e = p->o_amp.alloc((size_t)depth * capacity, true)) != cudaSuccess) return cfail(e, "records");
    if ((e = p->o_pc.alloc((size_t)depth * capacity * std::max<int64_t>(p->feat, 1), true)) != cudaSuccess)
        return cfail(e, "records");
    if ((e = p->o_count.alloc((size_t)depth, true)) != cudaSuccess) return cfail(e, "records");
    if ((e = p->mail.alloc((size_t)depth, true)) != cudaSuccess) return cfail(e, "mailbox");
    p->slots.reset(new Slot[depth]);
    for (int i = 0; i < depth; ++i)
        if ((e = cudaEventCreateWithFlags(&p->slots[i].ev, cudaEventDisableTiming)) != cudaSuccess)
            return cfail(e, "event");
    if (drift_M) {
        rc = lss_set_drift(h, drift_M);
        if (rc) {
            lss::set_thread_error(h->err.c_str());
            return rc;
        }
    }
    if (h->mix_ev && (e = cudaEventSynchronize(h->mix_ev)) != cudaSuccess) return cfail(e, "template rebuild");
    if (post) {
        rc = lss_set_postprocess(h, post);
        if (rc) {
            lss::set_thread_error(h->err.c_str());
            return rc;
        }
        if ((e = p->o_x.alloc((size_t)depth * capacity, true)) != cudaSuccess) return cfail(e, "records");
        if ((e = p->o_y.alloc((size_t)depth * capacity, true)) != cudaSuccess) return cfail(e, "records");
        if ((e = p->o_clu.alloc((size_t)depth * capacity, true)) != cudaSuccess) return cfail(e, "records");
        p->bytes = h->dev_bytes + ring_bytes + 3 * sizeof(int64_t);
        if (s->used + (int64_t)p->bytes > s->budget) {
            lss::set_thread_error("device memory budget exhausted");
            return LSS_ERR_BUSY;
        }
    }
    // every admitted probe's rounds kernel (a cooperative grid, one CTA per
    // SM) must fit beside the others': at most SMs / max_probes CTAs each
    h->mp_grid = std::max(1, std::min(h->mp_grid, h->sm_count / (int)s->probes.size()));
    // short stream batches: the block-skipping rounds' extra grid barrier per
    // round costs more latency than the rows it skips (measured on a B200, 800
    // templates, 300-sample blocks: p99 2.66 ms against about 2 ms), so every
    // row is updated
    h->mp_skip = false;
    h->streaming = true;
    rc = capture(p.get());
    if (!rc) rc = calibrate_clock(p.get());
    if (rc) {
        lss::set_thread_error(p->err.c_str());
        return rc;
    }
    if (s->used + s->retired_bytes + (int64_t)p->bytes > s->budget) free_retired(s);
    s->used += (int64_t)p->bytes;
    s->largest = std::max<int64_t>(s->largest, (int64_t)p->bytes);
    s->probes[slot] = std::move(p);
    *probe = slot;
    return LSS_OK;
}

static Probe* get_probe(lss_server* s, int32_t probe) {
    if (!s || probe < 0 || probe >= (int32_t)s->probes.size()) return nullptr;
    return s->probes[probe].get();
}

int lss_server_push(lss_server* s, int32_t probe, const int16_t* rows, int64_t n_rows, int64_t arrival_ns) {
    Probe* p = get_probe(s, probe);
    if (!p || (!rows && n_rows > 0) || n_rows < 0) {
        lss::set_thread_error("lss_server_push: bad probe or rows");
        return LSS_ERR_ARG;
    }
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(p->m);
    while (n_rows > 0) {
        if (p->fill == 0 && p->next - p->harvest >= p->D) {
            // the staging block and result slot of batch next - D are reused:
            // that batch must have finished and been moved out
            int rc = harvest_one(p, lk, true);
            if (rc) return rc;
        }
        const int64_t take = std::min(n_rows, p->NT - p->fill);
        std::memcpy(p->staging.p + ((p->next % p->D) * p->NT + p->fill) * p->Cbin, rows,
                    (size_t)(take * p->Cbin) * sizeof(int16_t));
        p->fill += take;
        rows += take * p->Cbin;
        n_rows -= take;
        if (p->fill == p->NT) {
            int rc = launch_block(p, arrival_ns);
            if (rc) return rc;
            p->fill = 0;
        }
    }
    return LSS_OK;
}

int lss_server_poll(lss_server* s, int32_t probe, lss_records* out, int64_t* batch, int32_t wait) {
    Probe* p = get_probe(s, probe);
    if (!p || !out || !batch) {
        lss::set_thread_error("lss_server_poll: bad argument");
        return LSS_ERR_ARG;
    }
    if (out->on_device) {
        lss::set_thread_error("lss_server_poll: records are returned in host memory");
        return LSS_ERR_ARG;
    }
    std::unique_lock<std::mutex> lk(p->m);
    *batch = -1;
    out->count = 0;
    if (p->ready.empty()) {
        int rc = harvest_one(p, lk, wait != 0);
        if (rc) return rc;
    }
    if (p->ready.empty()) return LSS_OK;
    Result r = std::move(p->ready.front());
    p->ready.pop_front();
    *batch = r.batch;
    out->count = r.count;
    if (r.status & STATUS_TIMEOUT) {
        lss::set_thread_error("a bounded device-side wait gave up in this batch");
        return LSS_ERR_TIMEOUT;
    }
    if (r.status & (STATUS_CAPACITY | STATUS_LIST)) {
        lss::set_thread_error("spike list capacity exceeded in this batch");
        return LSS_ERR_CAPACITY;
    }
    if (r.status & (1 << 30)) {
        lss::set_thread_error("stream mailbox out of step");
        return LSS_ERR_STATE;
    }
    if (r.count > p->cap || r.count > out->capacity) {
        lss::set_thread_error("record capacity smaller than the batch's spike count");
        return LSS_ERR_CAPACITY;
    }
    if (!out->time || !out->template_id || !out->amplitude) {
        lss::set_thread_error("null record arrays");
        return LSS_ERR_ARG;
    }
    std::copy(r.time.begin(), r.time.end(), out->time);
    std::copy(r.tmpl.begin(), r.tmpl.end(), out->template_id);
    std::copy(r.amp.begin(), r.amp.end(), out->amplitude);
    if (out->pc && p->feat > 0) std::copy(r.pc.begin(), r.pc.end(), out->pc);
    if (out->x_pos && !r.x.empty()) std::copy(r.x.begin(), r.x.end(), out->x_pos);
    if (out->y_pos && !r.y.empty()) std::copy(r.y.begin(), r.y.end(), out->y_pos);
    if (out->cluster && !r.clu.empty()) std::copy(r.clu.begin(), r.clu.end(), out->cluster);
    return LSS_OK;
}

int lss_server_release(lss_server* s, int32_t probe) {
    if (!get_probe(s, probe)) {
        lss::set_thread_error("lss_server_release: bad probe");
        return LSS_ERR_ARG;
    }
    cudaSetDevice(s->device);
    std::lock_guard<std::mutex> lk(s->m);
    std::unique_ptr<Probe> p = std::move(s->probes[probe]);
    s->used -= (int64_t)p->bytes;
    if (p->s && cudaStreamSynchronize(p->s) != cudaSuccess) {
        p.reset();  // a failed stream: free now
        return LSS_OK;
    }
    s->retired_bytes += (int64_t)p->bytes;
    s->retired.push_back(std::move(p));
    return LSS_OK;
}

int lss_server_set_drift(lss_server* s, int32_t probe, const float* drift_M) {
    Probe* p = get_probe(s, probe);
    if (!p || !drift_M) {
        lss::set_thread_error("lss_server_set_drift: bad argument");
        return LSS_ERR_ARG;
    }
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(p->m);
    while (p->harvest < p->next) {
        int rc = harvest_one(p, lk, true);
        if (rc) return rc;
    }
    p->h->streaming = false;
    int rc = lss_set_drift(p->h, drift_M);
    if (!rc && p->h->mix_ev && cudaEventSynchronize(p->h->mix_ev) != cudaSuccess) rc = LSS_ERR_CUDA;
    p->h->streaming = true;
    if (rc) lss::set_thread_error(p->h->err.c_str());
    return rc;
}

int lss_server_latency(lss_server* s, int32_t probe, double* p50_ms, double* p99_ms, int64_t* batches) {
    Probe* p = get_probe(s, probe);
    if (!p || !p50_ms || !p99_ms || !batches) {
        lss::set_thread_error("lss_server_latency: bad argument");
        return LSS_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(p->m);
    std::vector<double> v = p->lat_ms;
    *batches = (int64_t)v.size();
    if (v.empty()) {
        *p50_ms = *p99_ms = 0.0;
        return LSS_OK;
    }
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) {
        const double pos = q * (double)(v.size() - 1);
        const size_t i = (size_t)pos;
        const double f = pos - (double)i;
        return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
    };
    *p50_ms = pct(0.50);
    *p99_ms = pct(0.99);
    return LSS_OK;
}

int lss_server_latencies(lss_server* s, int32_t probe, double* out_ms, int64_t capacity, int64_t* n) {
    Probe* p = get_probe(s, probe);
    if (!p || !n || (capacity > 0 && !out_ms)) {
        lss::set_thread_error("lss_server_latencies: bad argument");
        return LSS_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(p->m);
    *n = (int64_t)p->lat_ms.size();
    for (int64_t i = 0; i < std::min<int64_t>(capacity, *n); ++i) out_ms[i] = p->lat_ms[i];
    return LSS_OK;
}

int lss_server_latency_parts(lss_server* s, int32_t probe, double* out_ms, int64_t capacity, int64_t* n) {
    Probe* p = get_probe(s, probe);
    if (!p || !n || (capacity > 0 && !out_ms)) {
        lss::set_thread_error("lss_server_latency_parts: bad argument");
        return LSS_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(p->m);
    *n = (int64_t)p->parts_ms.size() / 4;
    const int64_t m = std::min<int64_t>(capacity, *n) * 4;
    for (int64_t i = 0; i < m; ++i) out_ms[i] = p->parts_ms[i];
    return LSS_OK;
}

int lss_server_memory(lss_server* s, int64_t* used, int64_t* budget) {
    if (!s || !used || !budget) return LSS_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->m);
    *used = s->used;
    *budget = s->budget;
    return LSS_OK;
}

}  // extern "C"
