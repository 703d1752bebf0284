"""ctypes binding of libmt_b200.so (declarations mirror include/mt_masstree.h)."""
import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libmt_b200.so")

_u32 = ctypes.c_uint32
_u64 = ctypes.c_uint64
_p = ctypes.c_void_p
_int = ctypes.c_int

# name -> (restype, argtypes)
SIGNATURES = {
    "mt_create": (_int, [ctypes.POINTER(_p), ctypes.c_float, _u32]),
    "mt_create_bytes": (_int, [ctypes.POINTER(_p), _u64, _u32]),
    "mt_destroy": (_int, [_p]),
    "mt_set_tile_size": (_int, [_p, _u32]),
    "mt_set_write_tile_size": (_int, [_p, _u32]),
    "mt_set_blocks_per_sm": (_int, [_p, _u32]),
    "mt_set_scan_tile_size": (_int, [_p, _u32]),
    "mt_set_lock_wait": (_int, [_p, _u32]),
    "mt_set_upderase_tile_size": (_int, [_p, _u32]),
    "mt_inject_node_lock": (_int, [_p, _u32, _int]),
    "mt_find": (_int, [_p, _p, _u32, _p, _p, _u32, _p, _u32, _u32, _p]),
    "mt_insert": (_int, [_p, _p, _u32, _p, _p, _u32, _p, _u32, _p, _u32, _p]),
    "mt_update": (_int, [_p, _p, _u32, _p, _p, _u32, _p, _u32, _p, _u32, _p]),
    "mt_erase": (_int, [_p, _p, _u32, _p, _u32, _p, _u32, _p]),
    "mt_scan": (_int, [_p, _p, _p, _u32, _u32, _u32, _p, _p, _p, _p, _u32, _p, _p, _p, _u32, _p]),
    "mt_mixed_batch": (_int, [_p, _p, _p, _u32, _p, _p, _u32, _p, _p, _u32, _u32, _p]),
    "mt_mixed_batch_noalloc": (_int, [_p, _p, _p, _u32, _p, _p, _u32, _p, _p, _u32, _p]),
    "mt_mixed_batch_host": (_int, [_p, _p, _p, _u32, _p, _p, _u32, _p, _p, _u32, _u32, _u32, _p]),
    "mt_batches_reserve": (_int, [_p, _u32, _u64]),
    "mt_mixed_batches": (_int, [_p, _p, _u32, _u32, _u32, _u32, _p]),
    "mt_sync": (_int, [_p, _p]),
    "mt_stats": (_int, [_p, _p]),
    "mt_reclaim": (_int, [_p, _p]),
    "mt_status_string": (ctypes.c_char_p, [_int]),
    "mt_validate": (_int, [_p, ctypes.POINTER(_u64), ctypes.c_char_p, ctypes.c_size_t]),
    "mt_selftest_line_atomicity": (_int, [_u32, _u32, _u32, ctypes.POINTER(_u64), ctypes.POINTER(_u64)]),
    "mt_serve": (_int, [_p, _p, _p, _p]),
    "mt_device_view": (_int, [_p, _p, ctypes.c_size_t]),
    "mt_server_start": (_int, [_p, _p, ctypes.POINTER(_p)]),
    "mt_server_submit": (_int, [_p, _p, _p, _p, _p, _p, _p, _u32, ctypes.POINTER(_u64)]),
    "mt_server_poll": (_int, [_p, _u64, ctypes.POINTER(_int), ctypes.POINTER(_u64)]),
    "mt_server_stop": (_int, [_p]),
    "mt_server_stats": (_int, [_p, _p]),
    "mt_set_group_hash_bits": (_int, [_p, _u32]),
}


class MtStats(ctypes.Structure):
    _fields_ = [
        ("total_slabs", _u64),
        ("used_slabs", _u64),
        ("free_slabs", _u64),
        ("limbo_slabs", _u64),
        ("num_shards", _u32),
        ("tile_size", _u32),
        ("device_error", _u32),
        ("device_error_count", _u32),
        ("device_error_site", _u32),
        ("reserved", _u32),
    ]


class MtServePlan(ctypes.Structure):
    _fields_ = [
        ("types", _p),
        ("keys", _p),
        ("key_lengths", _p),
        ("values", _p),
        ("value_lengths", _p),
        ("results", _p),
        ("max_key_length", _u32),
        ("max_value_length", _u32),
        ("request_first_op", _p),
        ("request_num_ops", _p),
        ("arrival_ns", _p),
        ("num_requests", _u32),
        ("mode", _u32),
        ("chunk_ops", _u32),
        ("epoch_us", _u32),
        ("memory_budget", ctypes.c_float),
        ("reserved", _u32),
    ]


class MtServerConfig(ctypes.Structure):
    _fields_ = [
        ("max_key_length", _u32),
        ("max_value_length", _u32),
        ("max_ops_in_flight", _u32),
        ("max_requests_in_flight", _u32),
        ("chunk_ops", _u32),
        ("epoch_us", _u32),
        ("memory_budget", ctypes.c_float),
        ("reserved", _u32),
    ]


class MtServeStats(ctypes.Structure):
    _fields_ = [
        ("wall_ns", _u64),
        ("requests_done", _u64),
        ("ops_done", _u64),
        ("admission_waits", _u64),
        ("stage_ns", _u64 * 4),
    ]


class MtServerStats(ctypes.Structure):
    _fields_ = [
        ("requests", _u64),
        ("ops", _u64),
        ("queued_ns", _u64),
        ("upload_ns", _u64),
        ("device_ns", _u64),
        ("deliver_ns", _u64),
        ("max_latency_ns", _u64),
        ("reserved", _u64),
    ]


_lib = None


def load():
    """Load the CUDA library; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m indexingpu_b200.build` "
                "(there is no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
