"""Output formats (host code, no GPU): spikeOutput.txt lines and the
decoder's OnlineSpikesPayload in cereal's binary archive layout."""
import struct

import numpy as np


def _rec():
    return dict(time=np.array([100, 250, 251], np.int64), template=np.array([3, 0, 7], np.int32),
                amplitude=np.array([12.3456789, 0.5, 1e-7], np.float32),
                cluster=np.array([1, 1, 2], np.int32), y=np.array([480.0, 20.5, 3840.25], np.float32))


def test_spike_lines_match_ostream_formatting():
    from livespikesorter_b200.output import spike_lines
    r = _rec()
    txt = spike_lines(r, recording_offset=1000)
    want = ''.join(f'{1000 + t},{y},{float(a):g},{float(p):g}\n'
                   for t, y, a, p in zip(r['time'], r['template'], r['amplitude'], r['y']))
    assert txt == want
    assert txt.splitlines()[0] == '1100,3,12.3457,480'
    assert spike_lines(r, use_cluster=True).splitlines()[2].split(',')[1] == '2'
    assert spike_lines(dict(time=np.zeros(0, np.int64), template=np.zeros(0, np.int32),
                            amplitude=np.zeros(0, np.float32))) == ''


def test_payload_layout_and_round_trip():
    from livespikesorter_b200.output import parse_payload, payload
    r = _rec()
    for lb in (4, 8):
        b = payload(r, recording_offset=7, stream_sample_ct=123456, vrms=2.5, p2p=9.0, process_time=42,
                    long_bytes=lb, use_cluster=True)
        n = len(r['time'])
        assert len(b) == 2 * lb + 3 * 8 + 2 * n * lb + 4 * n + 8 + 4 + lb + lb + 8 + 8
        p = parse_payload(b, lb)
        assert p['recordingOffset'] == 7 and p['streamSampleCt'] == 123456
        assert np.array_equal(p['Times'], r['time']) and np.array_equal(p['Templates'], r['cluster'])
        assert np.array_equal(p['Amplitudes'], r['amplitude'])
        assert (p['VRMS'], p['P2P'], p['processTime'], p['confidence']) == (2.5, 9.0, 42, 0.0)
    # one spike, Windows `long`: offset, count, first time at fixed positions
    b = payload(dict(time=np.array([5], np.int64), template=np.array([9], np.int32),
                     amplitude=np.array([1.5], np.float32)), recording_offset=-3, long_bytes=4)
    assert len(b) == 80
    assert struct.unpack_from('<iiQi', b, 0) == (-3, 0, 1, 5)
    assert struct.unpack_from('<Qi', b, 20) == (1, 9)


def test_short_buffers_and_bad_arguments():
    import ctypes
    from livespikesorter_b200 import _lib
    from livespikesorter_b200.output import _records, spike_lines
    lib = _lib.load()
    r = _rec()
    full = spike_lines(r)
    rec, keep = _records(r)
    # a buffer that holds the first line and a half: the first line, NUL-terminated, full length returned
    first = full.splitlines(keepends=True)[0]
    cap = len(first) + 5
    buf = ctypes.create_string_buffer(b'\xff' * cap, cap)
    assert lib.lss_format_spike_lines(rec, 0, 0, buf, cap) == len(full)
    assert buf.value.decode() == first
    assert lib.lss_format_spike_lines(rec, 0, 0, buf, 0) == len(full)  # nothing written
    # payload into a short buffer: a prefix of the full payload, nothing past cap
    n = lib.lss_serialize_payload(rec, 0, 0, 0.0, 0.0, 0, 4, 0, None, 0)
    whole = (ctypes.c_uint8 * n)()
    assert lib.lss_serialize_payload(rec, 0, 0, 0.0, 0.0, 0, 4, 0, whole, n) == n
    part = (ctypes.c_uint8 * (n + 8))(*([0xAB] * (n + 8)))
    assert lib.lss_serialize_payload(rec, 0, 0, 0.0, 0.0, 0, 4, 0, part, 30) == n
    assert bytes(part)[30:] == b'\xab' * (n + 8 - 30)
    k = max(i for i in range(31) if bytes(part)[:i] == bytes(whole)[:i])
    assert bytes(part)[k:30] == b'\xab' * (30 - k)           # a field that did not fit is not started
    # bad arguments: -1 and a message
    assert lib.lss_serialize_payload(rec, 0, 0, 0.0, 0.0, 0, 3, 0, None, 0) == -1
    assert b'long_bytes' in lib.lss_last_error(None)
    dev = _lib.LssRecords(time=rec.time, template_id=rec.template_id, amplitude=rec.amplitude, pc=None,
                          capacity=3, count=3, on_device=1)
    assert lib.lss_format_spike_lines(dev, 0, 0, None, 0) == -1
    nocl = _lib.LssRecords(time=rec.time, template_id=rec.template_id, amplitude=rec.amplitude, pc=None,
                           capacity=3, count=3, on_device=0)
    assert lib.lss_format_spike_lines(nocl, 0, 1, None, 0) == -1   # clusters asked for, none given
    del keep
