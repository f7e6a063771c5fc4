// Output formats the reference's consumers read (lss_format_spike_lines,
// lss_serialize_payload).
//
// * spikeOutput.txt: one line per spike, "time,template,amplitude,y"
//   (OnlineSpikesV2::writeSpikesToFile, OnlineSpikesV2.cu:1117-1124), the
//   values written by std::ostream's default formatting (integers in decimal,
//   floats as %g with 6 significant digits). The reference prints the y of the
//   spike at the same position of its per-batch position array, which after
//   its sorted insertion belongs to another spike; here each record prints its
//   own y.
// * OnlineSpikesPayload (src/Networking/onlineSpikesPayload.h:8-48), the UDP
//   message to the decoder, in the layout cereal's BinaryOutputArchive gives
//   it: fields in declaration order, no padding, scalars in native
//   (little-endian) byte order, each std::vector as a uint64 element count
//   followed by its elements. `long` is 4 bytes in the reference's Windows
//   build (LLP64) and 8 on LP64 systems, so its width is a parameter.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "lss.h"

namespace lss {
void set_thread_error(const char* msg);
}

namespace {

struct Writer {
    uint8_t* buf;
    int64_t cap;
    int64_t len = 0;
    void raw(const void* p, size_t n) {
        if (buf && len + (int64_t)n <= cap) std::memcpy(buf + len, p, n);
        len += (int64_t)n;
    }
    void i64_as(int64_t v, int bytes) {
        if (bytes == 4) {
            const int32_t w = (int32_t)v;
            raw(&w, 4);
        } else {
            raw(&v, 8);
        }
    }
    void u64(uint64_t v) { raw(&v, 8); }
};

}  // namespace

extern "C" {

int64_t lss_format_spike_lines(const lss_records* rec, int64_t recording_offset, int32_t use_cluster, char* buf,
                               int64_t cap) {
    if (!rec || rec->count < 0 || rec->on_device) {
        lss::set_thread_error("lss_format_spike_lines: host records expected");
        return -1;
    }
    if (rec->count > 0 && (!rec->time || !rec->template_id || !rec->amplitude)) {
        lss::set_thread_error("lss_format_spike_lines: null record arrays");
        return -1;
    }
    if (use_cluster && rec->count > 0 && !rec->cluster) {
        lss::set_thread_error("lss_format_spike_lines: no cluster array");
        return -1;
    }
    // whole lines are copied while they fit with room for the terminator;
    // the return value is always the full length
    int64_t len = 0, written = 0;
    char line[128];
    for (int64_t i = 0; i < rec->count; ++i) {
        const int64_t id = use_cluster ? rec->cluster[i] : rec->template_id[i];
        const double y = rec->y_pos ? (double)rec->y_pos[i] : 0.0;
        const int n = std::snprintf(line, sizeof(line), "%lld,%lld,%g,%g\n",
                                    (long long)(recording_offset + rec->time[i]), (long long)id,
                                    (double)rec->amplitude[i], y);
        if (n < 0) return -1;
        if (buf && written == len && len + n < cap) {
            std::memcpy(buf + len, line, (size_t)n);
            written += n;
        }
        len += n;
    }
    if (buf && cap > 0) buf[written] = '\0';
    return len;
}

int64_t lss_serialize_payload(const lss_records* rec, int64_t recording_offset, int64_t stream_sample_ct,
                              double vrms, float p2p, int64_t process_time, int32_t long_bytes, int32_t use_cluster,
                              uint8_t* buf, int64_t cap) {
    if (!rec || rec->count < 0 || rec->on_device || (long_bytes != 4 && long_bytes != 8)) {
        lss::set_thread_error("lss_serialize_payload: host records and long_bytes 4 or 8 expected");
        return -1;
    }
    if (rec->count > 0 && (!rec->time || !rec->template_id || !rec->amplitude || (use_cluster && !rec->cluster))) {
        lss::set_thread_error("lss_serialize_payload: null record arrays");
        return -1;
    }
    Writer w{buf, cap};
    const uint64_t n = (uint64_t)rec->count;
    w.i64_as(recording_offset, long_bytes);
    w.i64_as(stream_sample_ct, long_bytes);
    w.u64(n);  // Times
    for (uint64_t i = 0; i < n; ++i) w.i64_as(rec->time[i], long_bytes);
    w.u64(n);  // Templates
    for (uint64_t i = 0; i < n; ++i) w.i64_as(use_cluster ? rec->cluster[i] : rec->template_id[i], long_bytes);
    w.u64(n);  // Amplitudes
    if (n) w.raw(rec->amplitude, n * sizeof(float));
    w.raw(&vrms, sizeof(double));
    w.raw(&p2p, sizeof(float));
    w.i64_as(process_time, long_bytes);
    // decoder-to-GUI fields, unused on this hop (zero)
    w.i64_as(0, long_bytes);  // eventStreamSampleCt
    const int16_t z16 = 0;
    for (int i = 0; i < 4; ++i) w.raw(&z16, 2);  // predictLabel, label, nTrials, nCorrect
    const double z64 = 0.0;
    w.raw(&z64, 8);  // confidence
    return w.len;
}

}  // extern "C"
