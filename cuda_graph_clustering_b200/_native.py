"""ctypes binding of libccb.so (the C ABI declared in include/ccb.h).

The library is built in-tree by ``python -m cuda_graph_clustering_b200.build`` (or
``__graft_entry__.build()``).  Loading fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libccb.so")

CCB_OK = 0
CCB_ERR_INVALID = 1
CCB_ERR_DEVICE_MEMORY = 2
CCB_ERR_CUDA = 3
CCB_ERR_TIMEOUT = 4
CCB_ERR_STATE = 5
CCB_ERR_CANCELLED = 6

LS_AUTO, LS_GLOBAL, LS_SHARED, LS_WIDE = 0, 1, 2, 3
MAX_CLUSTERS = 64
MAX_VERTICES_NARROW = 32767
MAX_VERTICES_WIDE = 1 << 20


class CcbParams(C.Structure):
    _fields_ = [("k", C.c_int32), ("population", C.c_int32), ("tournament", C.c_int32),
                ("iterations", C.c_int32), ("early_stop", C.c_int32), ("perturbation", C.c_double),
                ("gww", C.c_double), ("threads", C.c_int32), ("seed", C.c_uint64),
                ("time_limit_sec", C.c_double), ("verbose", C.c_int32), ("ls_kernel", C.c_int32)]


class CcbResult(C.Structure):
    _fields_ = [("objective", C.c_int64), ("iterations_done", C.c_int32), ("clusters_used", C.c_int32),
                ("seconds", C.c_double), ("local_searches", C.c_int64), ("accepted_moves", C.c_int64)]


class CcbKernelStats(C.Structure):
    _fields_ = [("descent_ms", C.c_double), ("rebuild_ms", C.c_double), ("record_ms", C.c_double),
                ("other_ms", C.c_double), ("descent_launches", C.c_int64), ("rebuild_launches", C.c_int64),
                ("record_launches", C.c_int64), ("other_launches", C.c_int64)]


class CcbTuningEntry(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n_min", C.c_int32), ("n_max", C.c_int32), ("k_min", C.c_int32),
                ("k_max", C.c_int32), ("use_kind", C.c_int32), ("threads", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("max_slots", C.c_int32)]


_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)
_vp = C.c_void_p

# name -> (restype, argtypes); the exported surface of include/ccb.h
SIGNATURES = {
    "ccb_last_error": (C.c_char_p, []),
    "ccb_params_init": (None, [C.POINTER(CcbParams)]),
    "ccb_pbils_solve": (C.c_int, [_vp, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(CcbParams), _vp,
                                  C.POINTER(CcbResult)]),
    "ccb_neighborhood_solve": (C.c_int, [_vp, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(CcbParams),
                                         C.c_int32, _vp, C.POINTER(CcbResult)]),
    "ccb_graph_upload": (C.c_int, [_vp, C.c_uint32, C.c_uint32, C.c_uint64, _vp, C.POINTER(_vp)]),
    "ccb_graph_from_device": (C.c_int, [_vp, C.c_uint32, C.c_uint32, C.c_uint64, _vp, C.POINTER(_vp)]),
    "ccb_graph_size": (C.c_int, [_vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    "ccb_graph_destroy": (None, [_vp]),
    "ccb_solver_create": (C.c_int, [_vp, C.POINTER(CcbParams), C.POINTER(_vp)]),
    "ccb_solver_pbils": (C.c_int, [_vp, C.POINTER(CcbParams), _vp, _vp, C.POINTER(CcbResult)]),
    "ccb_solver_neighborhood": (C.c_int, [_vp, C.POINTER(CcbParams), C.c_int32, _vp, _vp, C.POINTER(CcbResult)]),
    "ccb_solver_describe": (C.c_char_p, [_vp]),
    "ccb_solver_destroy": (None, [_vp]),
    "ccb_solver_set_profiling": (C.c_int, [_vp, C.c_int32]),
    "ccb_solver_set_rebuild": (C.c_int, [_vp, C.c_int32]),
    "ccb_solver_stats": (C.c_int, [_vp, C.POINTER(CcbKernelStats)]),
    "ccb_graph_generate_erdos_renyi": (C.c_int, [C.c_uint32, C.c_double, C.c_uint64, _vp, C.POINTER(_vp)]),
    "ccb_graph_load_tags": (C.c_int, [C.c_char_p, C.c_char_p, C.c_double, C.c_uint32, C.c_uint64, _vp,
                                      C.POINTER(_vp)]),
    "ccb_graph_generate_planted": (C.c_int, [C.c_uint32, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                             C.c_uint64, _vp, C.POINTER(_vp), _vp]),
    "ccb_graph_download": (C.c_int, [_vp, _vp, C.c_uint32]),
    "ccb_batch_create": (C.c_int, [C.POINTER(_vp)]),
    "ccb_batch_add": (C.c_int, [_vp, _vp, C.POINTER(CcbParams), C.POINTER(C.c_int32)]),
    "ccb_batch_run": (C.c_int, [_vp]),
    "ccb_batch_result": (C.c_int, [_vp, C.c_int32, _vp, C.POINTER(CcbResult)]),
    "ccb_batch_describe": (C.c_char_p, [_vp]),
    "ccb_batch_set_engine": (C.c_int, [_vp, C.c_int32, C.c_double]),
    "ccb_batch_withhold": (C.c_int, [_vp, C.c_int32]),
    "ccb_batch_destroy": (None, [_vp]),
    "ccb_release_cache": (None, []),
    "ccb_tuning_set": (C.c_int, [C.POINTER(CcbTuningEntry), C.c_int32]),
    "ccb_tuning_get": (C.c_int, [C.POINTER(CcbTuningEntry), C.c_int32, C.POINTER(C.c_int32)]),
    "ccb_server_create": (C.c_int, [C.c_uint64, C.c_int32, C.POINTER(_vp)]),
    "ccb_server_submit": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(CcbParams),
                                    C.POINTER(C.c_int32)]),
    "ccb_server_submit_generated": (C.c_int, [_vp, C.c_int32, C.c_uint32, C.c_double, C.c_double, C.c_double,
                                              C.c_int32, C.c_uint64, C.POINTER(CcbParams), C.POINTER(C.c_int32)]),
    "ccb_server_step": (C.c_int, [_vp, _i32p, C.c_int32, C.POINTER(C.c_int32)]),
    "ccb_server_status": (C.c_int, [_vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_uint64)]),
    "ccb_server_result": (C.c_int, [_vp, C.c_int32, C.POINTER(C.c_int32), _vp, C.POINTER(CcbResult)]),
    "ccb_server_cancel": (C.c_int, [_vp, C.c_int32, C.POINTER(C.c_int32)]),
    "ccb_server_destroy": (None, [_vp]),
    "ccb_evaluate_labelings": (C.c_int, [_vp, C.c_uint32, C.c_uint32, C.c_uint64, C.c_int32, C.c_int32, _vp, _vp,
                                         _vp, _vp, _vp]),
    "ccb_evaluate_labelings_noalloc": (C.c_int, [_vp, C.c_uint32, C.c_uint32, C.c_uint64, C.c_int32, C.c_int32,
                                                 _vp, _vp, _vp, _vp, _vp]),
    "ccb_evaluate_labelings_tensor": (C.c_int, [_vp, C.c_uint32, C.c_uint32, C.c_uint64, C.c_int32, C.c_int32,
                                                _vp, _vp, _vp, _vp, _vp]),
    "ccb_generate_erdos_renyi": (C.c_uint64, [_vp, ]),  # argtypes set below (mixed scalar types)
    "ccb_generate_planted": (C.c_uint64, []),
}

_lib = None


def library_path() -> str:
    return LIB_PATH


def lib() -> C.CDLL:
    """The loaded libccb.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libccb.so not built at {LIB_PATH}: run python -m cuda_graph_clustering_b200.build")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    L.ccb_generate_erdos_renyi.argtypes = [C.c_uint32, C.c_double, C.c_uint64, _vp, C.c_uint32]
    L.ccb_generate_planted.argtypes = [C.c_uint32, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                       C.c_uint64, _vp, C.c_uint32, _vp]
    _lib = L
    return L


def last_error() -> str:
    return lib().ccb_last_error().decode()


class CcbError(RuntimeError):
    """A nonzero ccb status; the message is the one the reference's std::runtime_error carries."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def check(status: int) -> None:
    if status != CCB_OK:
        raise CcbError(status, last_error())
