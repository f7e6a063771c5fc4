"""The reference's output formats for a batch's records.

``spike_lines`` writes spikeOutput.txt lines (OnlineSpikesV2::writeSpikesToFile,
OnlineSpikesV2.cu:1117-1124) and ``payload`` the decoder's OnlineSpikesPayload
(src/Networking/onlineSpikesPayload.h:8-48) in cereal's binary archive layout,
both through ``lss_format_spike_lines`` / ``lss_serialize_payload`` in the
library. ``parse_payload`` reads a payload back (for tests and consumers).
"""
from __future__ import annotations

import ctypes
import struct

import numpy as np

from . import _lib
from ._lib import LssRecords


def _records(rec: dict):
    t = np.ascontiguousarray(rec['time'], np.int64)
    y = np.ascontiguousarray(rec['template'], np.int32)
    a = np.ascontiguousarray(rec['amplitude'], np.float32)
    c = None if rec.get('cluster') is None else np.ascontiguousarray(rec['cluster'], np.int32)
    yp = None if rec.get('y') is None else np.ascontiguousarray(rec['y'], np.float32)
    keep = (t, y, a, c, yp)
    r = LssRecords(time=t.ctypes.data, template_id=y.ctypes.data, amplitude=a.ctypes.data, pc=None,
                   capacity=len(t), count=len(t), on_device=0, x_pos=None,
                   y_pos=None if yp is None else yp.ctypes.data, cluster=None if c is None else c.ctypes.data)
    return r, keep


def spike_lines(rec: dict, recording_offset: int = 0, use_cluster: bool = False) -> str:
    lib = _lib.load()
    r, keep = _records(rec)
    n = lib.lss_format_spike_lines(r, recording_offset, int(use_cluster), None, 0)
    if n < 0:
        raise _lib.LssError(_lib.LSS_ERR_ARG, (lib.lss_last_error(None) or b'').decode())
    buf = ctypes.create_string_buffer(n + 1)
    lib.lss_format_spike_lines(r, recording_offset, int(use_cluster), buf, n + 1)
    del keep
    return buf.value.decode()


def payload(rec: dict, recording_offset: int = 0, stream_sample_ct: int = 0, vrms: float = 0.0, p2p: float = 0.0,
            process_time: int = 0, long_bytes: int = 4, use_cluster: bool = False) -> bytes:
    lib = _lib.load()
    r, keep = _records(rec)
    args = (recording_offset, stream_sample_ct, vrms, p2p, process_time, long_bytes, int(use_cluster))
    n = lib.lss_serialize_payload(r, *args, None, 0)
    if n < 0:
        raise _lib.LssError(_lib.LSS_ERR_ARG, (lib.lss_last_error(None) or b'').decode())
    buf = (ctypes.c_uint8 * n)()
    lib.lss_serialize_payload(r, *args, buf, n)
    del keep
    return bytes(buf)


def parse_payload(b: bytes, long_bytes: int = 4) -> dict:
    """Reads an OnlineSpikesPayload written in cereal's binary layout."""
    L = 'i' if long_bytes == 4 else 'q'
    off = 0

    def take(fmt):
        nonlocal off
        v = struct.unpack_from('<' + fmt, b, off)
        off += struct.calcsize('<' + fmt)
        return v

    out = {}
    out['recordingOffset'], out['streamSampleCt'] = take(L + L)
    for name, f in (('Times', L), ('Templates', L), ('Amplitudes', 'f')):
        (n,) = take('Q')
        out[name] = np.array(take(f'{n}{f}'), dtype={'i': np.int32, 'q': np.int64, 'f': np.float32}[f])
    (out['VRMS'],) = take('d')
    (out['P2P'],) = take('f')
    (out['processTime'],) = take(L)
    (out['eventStreamSampleCt'],) = take(L)
    out['predictLabel'], out['label'], out['nTrials'], out['nCorrect'] = take('hhhh')
    (out['confidence'],) = take('d')
    if off != len(b):
        raise ValueError(f'{len(b) - off} trailing bytes')
    return out
