"""ctypes binding of ``include/lss.h`` (the C ABI in ``liblss_b200.so``).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as ct
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / 'liblss_b200.so'

(LSS_OK, LSS_ERR_ARG, LSS_ERR_IO, LSS_ERR_SHAPE, LSS_ERR_CUDA, LSS_ERR_CAPACITY, LSS_ERR_TIMEOUT, LSS_ERR_STATE,
 LSS_ERR_BUSY) = range(9)
LSS_PREC_FP32, LSS_PREC_BF16_RECHECK = 0, 1

# every entry point declared in include/lss.h
EXPORTS = ('lss_create', 'lss_create_from_dir', 'lss_destroy', 'lss_last_error', 'lss_get_config',
           'lss_set_drift', 'lss_filter', 'lss_match', 'lss_match_scores', 'lss_scores',
           'lss_sort_batch', 'lss_get_stats', 'lss_set_profiling', 'lss_get_stage_times',
           'lss_mp_rounds_noalloc', 'lss_set_round_kernel', 'lss_get_round_kernel', 'lss_server_create', 'lss_server_destroy', 'lss_server_admit',
           'lss_server_push', 'lss_server_poll', 'lss_server_release', 'lss_server_set_drift',
           'lss_server_latency', 'lss_server_memory', 'lss_recon_forward', 'lss_recon_backward',
           'lss_set_postprocess', 'lss_reset_postprocess', 'lss_format_spike_lines', 'lss_serialize_payload',
           'lss_set_templates', 'lss_set_drift_model', 'lss_set_drift_shift', 'lss_server_latencies',
           'lss_server_latency_parts',
           'lss_sort_batch_async', 'lss_sync')


class LssConfig(ct.Structure):
    _fields_ = [('n_chan', ct.c_int32), ('n_chan_bin', ct.c_int32), ('n_templates', ct.c_int32),
                ('n_pcs', ct.c_int32), ('nt', ct.c_int32), ('n_nearest', ct.c_int32),
                ('batch_size', ct.c_int32), ('nt0min', ct.c_int32), ('th_learned', ct.c_float),
                ('max_rounds', ct.c_int32), ('max_spikes', ct.c_int32), ('do_car', ct.c_int32),
                ('invert_sign', ct.c_int32), ('precision', ct.c_int32), ('device', ct.c_int32),
                ('hp_len', ct.c_int32)]


class LssTensors(ct.Structure):
    _fields_ = [('wall3', ct.c_void_p), ('wpca', ct.c_void_p), ('ctc', ct.c_void_p),
                ('whitening', ct.c_void_p), ('drift', ct.c_void_p), ('hp_filter', ct.c_void_p),
                ('iCC', ct.c_void_p), ('iU', ct.c_void_p), ('Ucc', ct.c_void_p),
                ('chan_map', ct.c_void_p), ('nm', ct.c_void_p)]


class LssRecords(ct.Structure):
    _fields_ = [('time', ct.c_void_p), ('template_id', ct.c_void_p), ('amplitude', ct.c_void_p),
                ('pc', ct.c_void_p), ('capacity', ct.c_int64), ('count', ct.c_int64),
                ('on_device', ct.c_int32), ('x_pos', ct.c_void_p), ('y_pos', ct.c_void_p),
                ('cluster', ct.c_void_p)]


class LssPostConfig(ct.Structure):
    _fields_ = [('xc', ct.c_void_p), ('yc', ct.c_void_p), ('centroids_xy', ct.c_void_p),
                ('n_clusters', ct.c_int32), ('dt_samples', ct.c_int32)]


class LssStats(ct.Structure):
    _fields_ = [('rounds', ct.c_int32), ('spikes', ct.c_int64), ('recheck_columns', ct.c_int64),
                ('recheck_flips', ct.c_int64), ('launches', ct.c_int64), ('recheck_rescored', ct.c_int64),
                ('mp_items', ct.c_int64), ('mp_items_updated', ct.c_int64),
                ('mp_peak_ns', ct.c_int64), ('mp_peak_wait_ns', ct.c_int64), ('mp_update_ns', ct.c_int64),
                ('mp_update_wait_ns', ct.c_int64), ('mp_peak_max_ns', ct.c_int64), ('mp_update_max_ns', ct.c_int64)]


STAGES = ('h2d_ms', 'ingest_ms', 'highpass_ms', 'whiten_ms', 'project_ms', 'score_ms', 'mp_ms', 'xres_ms',
          'feature_ms', 'records_ms', 'total_ms')


class LssStageTimes(ct.Structure):
    _fields_ = [(n, ct.c_float) for n in STAGES]


class LssError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f'lss error {code}: {msg}')
        self.code = code


_lib = None


def load() -> ct.CDLL:
    """Load ``liblss_b200.so`` (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f'{LIB_PATH} is missing; run `python -m livespikesorter_b200.build` '
                          '(the sorter has no CPU fallback)')
    lib = ct.CDLL(str(LIB_PATH))
    P, I64, I32 = ct.c_void_p, ct.c_int64, ct.c_int32
    sig = {
        'lss_create': ([ct.POINTER(LssConfig), ct.POINTER(LssTensors), ct.POINTER(P)], ct.c_int),
        'lss_create_from_dir': ([ct.c_char_p, ct.POINTER(LssConfig), ct.POINTER(P)], ct.c_int),
        'lss_destroy': ([P], None),
        'lss_last_error': ([P], ct.c_char_p),
        'lss_get_config': ([P, ct.POINTER(LssConfig)], ct.c_int),
        'lss_set_drift': ([P, P], ct.c_int),
        'lss_filter': ([P, P, I64, I64, I64, I32, P, P], ct.c_int),
        'lss_match': ([P, P, I64, P, P, P, I64, ct.POINTER(I64), P], ct.c_int),
        'lss_match_scores': ([P, P, I64, P, P, I64, ct.POINTER(I64), P], ct.c_int),
        'lss_scores': ([P, P, I64, P, P], ct.c_int),
        'lss_sort_batch': ([P, P, I64, I64, I64, I32, ct.POINTER(LssRecords), P], ct.c_int),
        'lss_sort_batch_async': ([P, P, I64, I64, I64, I32, ct.POINTER(LssRecords), P, P], ct.c_int),
        'lss_sync': ([P, P], ct.c_int),
        'lss_get_stats': ([P, ct.POINTER(LssStats)], ct.c_int),
        'lss_set_profiling': ([P, I32], ct.c_int),
        'lss_get_stage_times': ([P, ct.POINTER(LssStageTimes)], ct.c_int),
        'lss_set_round_kernel': ([P, I32], ct.c_int),
        'lss_get_round_kernel': ([P, ct.POINTER(ct.c_int32)], ct.c_int),
        'lss_mp_rounds_noalloc': ([P, I64, I32, I32, I32, ct.c_float, P, P, I32, I32, P, P, P,
                                   ct.POINTER(I32), ct.POINTER(I32), P], ct.c_int),
        'lss_server_create': ([I32, I64, I32, ct.POINTER(P)], ct.c_int),
        'lss_server_destroy': ([P], None),
        'lss_server_admit': ([P, ct.POINTER(LssConfig), ct.POINTER(LssTensors), P, ct.POINTER(LssPostConfig), I32,
                              I64, ct.POINTER(I32)], ct.c_int),
        'lss_set_postprocess': ([P, ct.POINTER(LssPostConfig)], ct.c_int),
        'lss_reset_postprocess': ([P], ct.c_int),
        'lss_set_templates': ([P, P, P], ct.c_int),
        'lss_set_drift_model': ([P, P, P, ct.c_float], ct.c_int),
        'lss_set_drift_shift': ([P, ct.c_double], ct.c_int),
        'lss_format_spike_lines': ([ct.POINTER(LssRecords), I64, I32, P, I64], I64),
        'lss_serialize_payload': ([ct.POINTER(LssRecords), I64, I64, ct.c_double, ct.c_float, I64, I32, I32, P,
                                   I64], I64),
        'lss_server_push': ([P, I32, P, I64, I64], ct.c_int),
        'lss_server_poll': ([P, I32, ct.POINTER(LssRecords), ct.POINTER(I64), I32], ct.c_int),
        'lss_server_release': ([P, I32], ct.c_int),
        'lss_server_set_drift': ([P, I32, P], ct.c_int),
        'lss_server_latency': ([P, I32, ct.POINTER(ct.c_double), ct.POINTER(ct.c_double), ct.POINTER(I64)],
                               ct.c_int),
        'lss_server_memory': ([P, ct.POINTER(I64), ct.POINTER(I64)], ct.c_int),
        'lss_server_latencies': ([P, I32, P, I64, ct.POINTER(I64)], ct.c_int),
        'lss_server_latency_parts': ([P, I32, P, I64, ct.POINTER(I64)], ct.c_int),
        'lss_recon_forward': ([I32, P, P, I32, I32, I32, I32, P, P, P, I64, P, I64, P], ct.c_int),
        'lss_recon_backward': ([I32, P, P, I32, I32, I32, I32, P, P, P, P, P, I64, P, P, P, P, P], ct.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def check(rc: int, handle=None):
    if rc != LSS_OK:
        msg = load().lss_last_error(handle)
        raise LssError(rc, msg.decode() if msg else '')
