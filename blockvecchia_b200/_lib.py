"""ctypes binding of libbv_b200.so (include/bv.h).

The library is built in-tree by blockvecchia_b200.build; importing this module
never falls back to anything else: a missing or unloadable library raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbv_b200.so")

BV_OK = 0
BV_E_INVALID = -1
BV_E_CUDA = -2
BV_E_NOMEM = -3
BV_E_NODEVICE = -4
BV_E_TOOLARGE = -5
BV_E_TIMEOUT = -6
BV_PREC_FP64 = 0
BV_PREC_MIXED = 1
BV_LARGE_AUTO = 0
BV_LARGE_STREAMED = 1
BV_LARGE_SLAB = 2
BV_SCHED_AUTO = 0
BV_SCHED_BUCKETED = 1
BV_SCHED_PERSISTENT = 2
BV_SCHED_STREAMED = 3
BV_FAIL_NEGINF = 0
BV_FAIL_CONTINUE = 1
BV_ST_COND_FAIL = 1
BV_ST_SCHUR_FAIL = 2
BV_ST_FP32_FALLBACK = 4
BV_ST_NONFINITE = 8

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)

# Every function include/bv.h declares, with its ctypes signature.
EXPORTS = {
    "bv_default_opts": (None, [C.c_void_p]),
    "bv_abi_sizes": (C.c_int, [C.POINTER(C.c_size_t), C.c_int]),
    "bv_create": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "bv_destroy": (None, [C.c_void_p]),
    "bv_llh": (C.c_double, [C.c_uint, _D, _D, C.c_void_p]),
    "bv_llh_eval": (C.c_int, [C.c_void_p, _D, _D]),
    "bv_block_llk": (C.c_int, [C.c_void_p, _D, C.c_int]),
    "bv_block_status": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint), C.c_int]),
    "bv_get_status": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bv_iterations": (C.c_int, [C.c_void_p]),
    "bv_last_error": (C.c_char_p, []),
    "bv_llh_host": (C.c_int, [C.c_void_p, _D, _D, _D, _I, _D, _D]),
    "bv_knn": (C.c_int, [_D, _D, C.c_int, C.c_int, C.c_int, _I, _D, _D, _I, C.c_int]),
    "bv_knn_subset": (C.c_int, [_D, _D, _D, C.c_int, C.c_int, C.c_int, _I, _D, _D, _D,
                                C.POINTER(C.c_ubyte), _I, C.c_int]),
    "bv_knn_ex": (C.c_int, [_D, _D, _D, C.c_int, C.c_int, C.c_int, _I, _D, _D, _D,
                            C.POINTER(C.c_ubyte), C.c_int, _I, C.c_int]),
    "bv_knn3": (C.c_int, [_D, _D, _D, C.c_int, C.c_int, C.c_int, _I, _D, _D, _D, _I, C.c_int]),
    "bv_layout_build": (C.c_int, [_D, _D, _D, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                  _I, _I, _D, _D, _D, _D, _D, _I, _I]),
    "bv_layout_from_clusters": (C.c_int, [_D, _D, _D, C.c_int, C.c_int, _I, _D, _D, C.c_int,
                                          _I, _I, _D, _D, _D, _D, _D, _I, _I]),
    "bv_kmeans": (C.c_int, [_D, _D, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _I, _D, _D]),
    "bv_generate_xy": (C.c_int, [C.c_int, C.c_int, _D, _D]),
    "bv_generate_xyt": (C.c_int, [C.c_int, C.c_int, C.c_int, _D, _D, _D]),
    "bv_layout_build3": (C.c_int, [_D, _D, _D, _D, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_int, _I, _I, _D, _D, _D, _D, _D, _D, _D, _I, _I]),
    "bv_layout_build_ex": (C.c_int, [_D, _D, _D, _D, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                     C.c_int, C.c_int, _I, _I, _D, _D, _D, _D, _D, _D, _D, _I, _I]),
    "bv_layout_from_clusters_ex": (C.c_int, [_D, _D, _D, _D, C.c_int, C.c_int, _I, _D, _D, _D,
                                             C.c_int, C.c_int, _I, _I, _D, _D, _D, _D, _D, _D, _D,
                                             _I, _I]),
    "bv_order_centroids": (C.c_int, [C.c_int, C.c_int, _D, _D, _D]),
    "bv_shard_blocks": (C.c_int, [_I, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_ubyte)]),
    "bv_get_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "bv_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bv_llh_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_int, C.c_int, C.c_int, _D, C.c_double, C.c_void_p,
                                 C.POINTER(C.c_uint), C.c_void_p]),
    "bv_server_default_opts": (None, [C.c_void_p]),
    "bv_server_create": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "bv_server_destroy": (None, [C.c_void_p]),
    "bv_server_open_job": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, _I]),
    "bv_server_open_job_ex": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, _I]),
    "bv_server_job_admitted": (C.c_int, [C.c_void_p, C.c_int, _I]),
    "bv_server_close_job": (C.c_int, [C.c_void_p, C.c_int]),
    "bv_server_submit": (C.c_int, [C.c_void_p, C.c_int, _D, C.POINTER(C.c_longlong)]),
    "bv_server_wait": (C.c_int, [C.c_void_p, C.c_longlong, _D, _D, C.c_int]),
    "bv_server_get_stats": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bv_server_reset_stats": (C.c_int, [C.c_void_p]),
}


class BvLayout(C.Structure):
    _fields_ = [("n", C.c_int), ("bc", C.c_int), ("cs", C.c_int),
                ("batchNum", _I), ("batchNumAccum", _I),
                ("x", _D), ("y", _D), ("obs", _D), ("knn_idx", _I),
                ("cx", _D), ("cy", _D), ("z", _D), ("cz", _D)]


class BvOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("kernel", C.c_int), ("dist_scale", C.c_double),
                ("device", C.c_int), ("on_failure", C.c_int), ("print_iter", C.c_int),
                ("use_graph", C.c_int), ("schedule", C.c_int), ("mixed_tol", C.c_double),
                ("shard_count", C.c_int), ("shard_index", C.c_int), ("large_blocks", C.c_int),
                ("nugget", C.c_int), ("earth", C.c_int), ("tune", C.c_int),
                ("mixed_fp32", C.c_int)]


class BvStatus(C.Structure):
    _fields_ = [("blocks", C.c_int), ("cond_fail", C.c_int), ("schur_fail", C.c_int),
                ("fp32_fallback", C.c_int), ("nonfinite", C.c_int), ("flags_or", C.c_uint),
                ("llk", C.c_double), ("device_ms", C.c_double), ("kernel_ms", C.c_double),
                ("failed", C.c_int), ("launches", C.c_int), ("streamed_blocks", C.c_int),
                ("streamed_threads", C.c_int), ("streamed_variant", C.c_int),
                ("tune_ms", C.c_double * 6)]


class BvJobOpts(C.Structure):
    _fields_ = [("dist_scale", C.c_double), ("nugget", C.c_int)]


class BvServerOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget", C.c_size_t), ("max_batch", C.c_int),
                ("on_failure", C.c_int), ("max_inflight", C.c_int)]


class BvServerStats(C.Structure):
    _fields_ = [("evals", C.c_longlong), ("batches", C.c_longlong), ("mean_batch", C.c_double),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("max_ms", C.c_double),
                ("bytes_in_use", C.c_size_t), ("hbm_budget", C.c_size_t),
                ("jobs_admitted", C.c_int), ("jobs_waiting", C.c_int)]


class BvError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libbv_b200 error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load libbv_b200.so (building it first if it is absent and nvcc exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build()
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in EXPORTS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != BV_OK:
        msg = lib().bv_last_error()
        raise BvError(rc, msg.decode() if msg else "")


def dp(a):
    return a.ctypes.data_as(_D)


def ip(a):
    return a.ctypes.data_as(_I)
