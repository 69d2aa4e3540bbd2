"""ctypes binding of libtqb200.so (include/turboquant_b200.h).

The library is loaded from this directory; there is no fallback: without the
built library (or without an sm_100 GPU for the compute calls) every call
fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtqb200.so")

TQ_OK = 0
TQ_ERR_INVALID_ARGUMENT = 1
TQ_ERR_CUDA = 2
TQ_ERR_OUT_OF_MEMORY = 3
TQ_ERR_NO_DEVICE = 4
TQ_ERR_TIMEOUT = 5
TQ_ERR_BUSY = 6
TQ_ERR_NOT_SUPPORTED = 7

PRECISION = {"fp32": 0, "split_bf16": 1, "split_tf32": 2, "reference": 3, "split_bf16_decoded": 4}

# Every symbol include/turboquant_b200.h declares.
EXPORTS = (
    "tq_last_error", "tq_version", "tq_space_create", "tq_space_destroy", "tq_space_get_info",
    "tq_space_tables", "tq_space_quantize", "tq_encode_batch", "tq_distance_1_to_n", "tq_distance_m_to_n",
    "tq_distance_m_to_n_symmetric", "tq_encode_batch_device", "tq_prepare_queries_device", "tq_prepare_query",
    "tq_distance_1_to_n_device", "tq_distance_1_to_n_prepared_device",
    "tq_distance_1_to_n_device_noalloc", "tq_distance_m_to_n_device",
    "tq_distance_m_to_n_symmetric_device", "tq_index_create", "tq_index_create_ex", "tq_index_destroy",
    "tq_server_create", "tq_server_create_ex", "tq_server_submit", "tq_request_wait", "tq_request_done",
    "tq_request_release", "tq_server_get_stats", "tq_server_reset_stats", "tq_server_tuning", "tq_server_tuning_times", "tq_topk_variant_shape",
    "tq_server_destroy", "tq_selftest_bounded_wait", "tq_space_take_device_status", "tq_space_scan_timer",
    "tq_space_scan_timer_read",
    "tq_rotated_coords_batch", "tq_rotated_coords_batch_device",
    "tq_distance_m_to_n_symmetric_qjl", "tq_distance_m_to_n_symmetric_qjl_device",
    "tq_prepare_symmetric_query", "tq_distance_1_to_n_symmetric_full",
    "tq_distance_1_to_n_symmetric_full_device",
)

SYM_VARIANT = {"light": 0, "full": 1, "full_prepared": 2}


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_uint64), ("rejected", C.c_uint64), ("completed", C.c_uint64),
        ("batches", C.c_uint64), ("rows", C.c_uint64), ("queued_rows", C.c_size_t),
        ("slots", C.c_int), ("max_rows", C.c_int), ("candidates", C.c_int),
        ("fallback_rows", C.c_uint64), ("bound_violations", C.c_uint64),
        ("pool_rows", C.c_size_t), ("pool_used_rows", C.c_size_t), ("scan_pass_rows", C.c_uint64),
        ("list_pass_rows", C.c_uint64),
    ]


class ServerParams(C.Structure):
    _fields_ = [
        ("k", C.c_int), ("max_rows", C.c_int), ("slots", C.c_int), ("kernel_variant", C.c_int),
        ("queue_rows", C.c_size_t), ("candidates", C.c_int), ("bound_scale", C.c_float),
        ("memory_budget", C.c_size_t),
    ]


class SpaceInfo(C.Structure):
    _fields_ = [
        ("dim", C.c_size_t), ("padded_dim", C.c_size_t), ("packed_bytes", C.c_size_t),
        ("code_size", C.c_size_t), ("bits_per_coord", C.c_int), ("num_levels", C.c_int),
        ("padded", C.c_int), ("num_threads", C.c_int), ("device", C.c_int),
        ("rot_seed", C.c_uint64), ("qjl_seed", C.c_uint64), ("scale", C.c_float),
    ]


class TQError(RuntimeError):
    """A failure reported by libtqb200 (CUDA error, out of memory, no device...)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


_LIB = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libtqb200.so not found at {LIB_PATH}: build it with "
            "`make -C turboquant-space_b200` (or __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    vp, sz, fp, u8p = C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p
    st = C.c_int
    L.tq_last_error.restype = C.c_char_p
    L.tq_version.restype = C.c_char_p
    L.tq_space_create.restype = st
    L.tq_space_create.argtypes = [sz, C.c_int, C.c_uint64, C.c_uint64, C.c_int, C.c_int,
                                  C.POINTER(vp)]
    L.tq_space_destroy.restype = None
    L.tq_space_destroy.argtypes = [vp]
    L.tq_space_get_info.restype = st
    L.tq_space_get_info.argtypes = [vp, C.POINTER(SpaceInfo)]
    L.tq_space_tables.restype = st
    L.tq_space_tables.argtypes = [vp, fp, fp, fp, fp]
    L.tq_space_quantize.restype = st
    L.tq_space_quantize.argtypes = [vp, fp, sz, u8p]
    L.tq_encode_batch.restype = st
    L.tq_encode_batch.argtypes = [vp, fp, sz, u8p]
    L.tq_distance_1_to_n.restype = st
    L.tq_distance_1_to_n.argtypes = [vp, fp, u8p, sz, fp]
    L.tq_distance_m_to_n.restype = st
    L.tq_distance_m_to_n.argtypes = [vp, fp, sz, u8p, sz, fp, C.c_int]
    L.tq_distance_m_to_n_symmetric.restype = st
    L.tq_distance_m_to_n_symmetric.argtypes = [vp, u8p, sz, u8p, sz, fp, C.c_int]
    L.tq_encode_batch_device.restype = st
    L.tq_encode_batch_device.argtypes = [vp, fp, sz, u8p, vp]
    L.tq_prepare_queries_device.restype = st
    L.tq_prepare_queries_device.argtypes = [vp, fp, sz, fp, fp, fp, vp]
    L.tq_prepare_query.restype = st
    L.tq_prepare_query.argtypes = [vp, fp, fp, fp, fp]
    L.tq_distance_1_to_n_device.restype = st
    L.tq_distance_1_to_n_device.argtypes = [vp, fp, u8p, sz, fp, vp]
    L.tq_distance_1_to_n_prepared_device.restype = st
    L.tq_distance_1_to_n_prepared_device.argtypes = [vp, fp, fp, fp, u8p, sz, fp, vp]
    L.tq_distance_1_to_n_device_noalloc.restype = st
    L.tq_distance_1_to_n_device_noalloc.argtypes = [vp, fp, u8p, sz, fp, vp]
    L.tq_distance_m_to_n_device.restype = st
    L.tq_distance_m_to_n_device.argtypes = [vp, fp, sz, u8p, sz, fp, C.c_int, vp]
    L.tq_distance_m_to_n_symmetric_device.restype = st
    L.tq_distance_m_to_n_symmetric_device.argtypes = [vp, u8p, sz, u8p, sz, fp, C.c_int, vp]
    L.tq_index_create_ex.restype = st
    L.tq_index_create_ex.argtypes = [vp, u8p, sz, C.c_int, C.c_int, C.POINTER(vp)]
    L.tq_index_create.restype = st
    L.tq_index_create.argtypes = [vp, u8p, sz, C.c_int, C.POINTER(vp)]
    L.tq_index_destroy.restype = None
    L.tq_index_destroy.argtypes = [vp]
    L.tq_server_create_ex.restype = st
    L.tq_server_create_ex.argtypes = [vp, C.POINTER(ServerParams), C.POINTER(vp)]
    L.tq_server_create.restype = st
    L.tq_server_create.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, sz, C.POINTER(vp)]
    L.tq_server_submit.restype = st
    L.tq_server_submit.argtypes = [vp, fp, sz, C.POINTER(vp)]
    L.tq_request_wait.restype = st
    L.tq_request_wait.argtypes = [vp, C.c_int, fp, vp, C.POINTER(C.c_double)]
    L.tq_request_done.restype = C.c_int
    L.tq_request_done.argtypes = [vp]
    L.tq_request_release.restype = None
    L.tq_request_release.argtypes = [vp]
    L.tq_server_get_stats.restype = st
    L.tq_server_get_stats.argtypes = [vp, C.POINTER(ServerStats), fp, sz, C.POINTER(C.c_size_t)]
    L.tq_server_reset_stats.restype = st
    L.tq_server_reset_stats.argtypes = [vp]
    L.tq_server_tuning_times.restype = st
    L.tq_server_tuning_times.argtypes = [vp, vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(C.c_int)]
    L.tq_topk_variant_shape.restype = st
    L.tq_topk_variant_shape.argtypes = [C.c_int, vp]
    L.tq_server_tuning.restype = st
    L.tq_server_tuning.argtypes = [vp, vp, vp, vp, C.c_int, C.POINTER(C.c_int)]
    L.tq_selftest_bounded_wait.restype = st
    L.tq_selftest_bounded_wait.argtypes = [C.c_int, C.c_int]
    L.tq_space_scan_timer.restype = st
    L.tq_space_scan_timer.argtypes = [vp, C.c_int]
    L.tq_space_scan_timer_read.restype = st
    L.tq_space_scan_timer_read.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]
    L.tq_space_take_device_status.restype = st
    L.tq_space_take_device_status.argtypes = [vp, C.POINTER(C.c_int)]
    L.tq_rotated_coords_batch.restype = st
    L.tq_rotated_coords_batch.argtypes = [vp, fp, sz, fp]
    L.tq_rotated_coords_batch_device.restype = st
    L.tq_rotated_coords_batch_device.argtypes = [vp, fp, sz, fp, vp]
    L.tq_distance_m_to_n_symmetric_qjl.restype = st
    L.tq_distance_m_to_n_symmetric_qjl.argtypes = [vp, u8p, sz, u8p, sz, fp, C.c_int, C.c_int]
    L.tq_distance_m_to_n_symmetric_qjl_device.restype = st
    L.tq_distance_m_to_n_symmetric_qjl_device.argtypes = [vp, u8p, sz, u8p, sz, fp, C.c_int,
                                                          C.c_int, vp]
    L.tq_prepare_symmetric_query.restype = st
    L.tq_prepare_symmetric_query.argtypes = [vp, u8p, fp, fp, fp]
    L.tq_distance_1_to_n_symmetric_full.restype = st
    L.tq_distance_1_to_n_symmetric_full.argtypes = [vp, fp, fp, fp, u8p, sz, fp]
    L.tq_distance_1_to_n_symmetric_full_device.restype = st
    L.tq_distance_1_to_n_symmetric_full_device.argtypes = [vp, fp, fp, fp, u8p, sz, fp, vp]
    L.tq_server_destroy.restype = None
    L.tq_server_destroy.argtypes = [vp]
    _LIB = L
    return L


def check(status: int) -> None:
    if status == TQ_OK:
        return
    msg = lib().tq_last_error().decode(errors="replace")
    if status == TQ_ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    if status == TQ_ERR_OUT_OF_MEMORY:
        raise MemoryError(msg)
    raise TQError(status, msg)
