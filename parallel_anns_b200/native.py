"""ctypes binding of the C ABI in include/panns_b200.h (libpanns_b200.so).

There is no CPU fallback: a missing or unloadable library, or no usable GPU,
raises. The library is built in-tree by ``parallel_anns_b200.build``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

PANNS_OK = 0
ERRORS = {
    -1: "EINVAL", -2: "EIO", -3: "ENOMEM", -4: "ECUDA", -5: "ESTATE", -6: "EDEVICE",
}

MODE_NSG_SEQ, MODE_TOP_M, MODE_PSS_V5, MODE_EFANNA = 0, 1, 2, 3
DIST_NORM_IP, DIST_L2 = 0, 1
STORE_FP32, STORE_BF16, STORE_FP8 = 0, 1, 2

# Every function declared in include/panns_b200.h.
EXPORTS = [
    "panns_last_error", "panns_version", "panns_open", "panns_close", "panns_set_base",
    "panns_load_fvecs_base", "panns_set_queries", "panns_load_fvecs_queries", "panns_set_graph",
    "panns_load_nsg", "panns_info", "panns_prepare_init_ids", "panns_rand_seed",
    "panns_efanna_init_ids", "panns_search", "panns_search_host", "panns_search_device",
    "panns_recall", "panns_load_true_nn", "panns_search_static", "panns_ground_truth",
    # include/panns_learned.h
    "panns_mlp_param_count", "panns_mlp_loss_grad", "panns_mlp_forward", "panns_mlp_train",
    "panns_kmeans", "panns_set_learned", "panns_learned_record",
    # include/panns_build.h
    "panns_build_nsg", "panns_build_nsg_ex", "panns_build_nsg_cells", "panns_graph_cells", "panns_graph_info",
    "panns_graph_copy", "panns_graph_save_nsg", "panns_graph_free",
    "panns_efanna_build",
]


class PannsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


FLAG_CUDA_GRAPH = 1
FLAG_LEARNED = 2


class SearchParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in
                ("mode", "distance", "K", "L", "M", "T", "L_local", "X", "warps_per_block", "storage",
                 "flags")] + [("L_query", ctypes.c_void_p), ("blocks_per_sm", ctypes.c_uint32),
                              ("warps_per_query", ctypes.c_uint32)]


class MlpTrainParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("d", "R", "T", "batch", "epochs", "seed")] + [
        (n, ctypes.c_float) for n in ("lr", "beta1", "beta2", "eps", "weight_decay", "lambda_L")]


class LearnedParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("E", "L_init", "L_min", "use_L")] + [
        (n, ctypes.c_float) for n in ("L_scale", "L_exp", "min_conf")]


class Stats(ctypes.Structure):
    _fields_ = [("n_dist", ctypes.c_uint64), ("n_expand", ctypes.c_uint64),
                ("n_edges", ctypes.c_uint64), ("n_iter", ctypes.c_uint64),
                ("kernel_ms", ctypes.c_double), ("total_ms", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def library_path() -> str:
    return _build.SO


def load(build_if_missing: bool = True):
    """Load libpanns_b200.so (building it if it is missing or stale)."""
    global _lib
    if _lib is not None:
        return _lib
    path = os.environ.get("PANNS_B200_LIB") or _build.SO  # another build of the same library
    if build_if_missing and path == _build.SO:
        _build.build()
    if not os.path.exists(path):
        raise PannsError(-4, f"native library not built: {path}")
    L = ctypes.CDLL(path)
    P = ctypes.c_void_p
    u32 = ctypes.c_uint32
    i32 = ctypes.c_int
    L.panns_last_error.restype = ctypes.c_char_p
    L.panns_version.restype = u32
    L.panns_open.argtypes = [ctypes.POINTER(P), i32]
    L.panns_close.argtypes = [P]
    L.panns_set_base.argtypes = [P, P, u32, u32, u32]
    L.panns_load_fvecs_base.argtypes = [P, ctypes.c_char_p, u32]
    L.panns_set_queries.argtypes = [P, P, u32, u32]
    L.panns_load_fvecs_queries.argtypes = [P, ctypes.c_char_p]
    L.panns_set_graph.argtypes = [P, u32, u32, P, P, u32]
    L.panns_load_nsg.argtypes = [P, ctypes.c_char_p]
    L.panns_info.argtypes = [P, P, P, P, P, P]
    L.panns_prepare_init_ids.argtypes = [P, u32, P]
    L.panns_rand_seed.argtypes = [P, u32]
    L.panns_efanna_init_ids.argtypes = [P, u32, u32, P, P]
    L.panns_search.argtypes = [P, ctypes.POINTER(SearchParams), P, u32, u32, P, ctypes.POINTER(Stats)]
    L.panns_search_host.argtypes = [P, ctypes.POINTER(SearchParams), P, u32, P, P,
                                    ctypes.POINTER(Stats)]
    L.panns_search_device.argtypes = [P, ctypes.POINTER(SearchParams), P, u32, P, P, P,
                                      ctypes.POINTER(Stats)]
    L.panns_recall.argtypes = [P, u32, u32, P, u32, u32, u32, ctypes.POINTER(ctypes.c_double)]
    L.panns_search_static.argtypes = [P, ctypes.POINTER(SearchParams), P, u32, P, P]
    L.panns_ground_truth.argtypes = [P, P, u32, u32, P, P]
    L.panns_load_true_nn.argtypes = [ctypes.c_char_p, P, P, P, P]
    L.panns_mlp_param_count.argtypes = [u32, u32]
    L.panns_mlp_param_count.restype = ctypes.c_uint64
    L.panns_mlp_loss_grad.argtypes = [i32, u32, u32, u32, P, P, P, P, u32, ctypes.c_float, P,
                                      ctypes.POINTER(ctypes.c_double)]
    L.panns_mlp_forward.argtypes = [i32, u32, u32, P, P, u32, P]
    L.panns_mlp_train.argtypes = [i32, ctypes.POINTER(MlpTrainParams), P, P, P, u32, P, P]
    L.panns_kmeans.argtypes = [P, u32, u32, u32, P, P, P]
    L.panns_set_learned.argtypes = [P, P, u32, P, ctypes.POINTER(LearnedParams)]
    L.panns_learned_record.argtypes = [P, u32, P]
    L.panns_build_nsg.argtypes = [i32, P, u32, u32, u32, u32, ctypes.POINTER(P)]
    L.panns_build_nsg_ex.argtypes = [i32, P, u32, u32, u32, u32, u32, ctypes.POINTER(P)]
    L.panns_build_nsg_cells.argtypes = [i32, P, u32, u32, u32, u32, u32, u32, u32, u32, u32, u32, ctypes.POINTER(P)]
    L.panns_graph_cells.argtypes = [P, P, P, P, P]
    L.panns_graph_info.argtypes = [P, P, P, P, P, P]
    L.panns_graph_copy.argtypes = [P, P, P, P]
    L.panns_graph_save_nsg.argtypes = [P, ctypes.c_char_p]
    L.panns_graph_free.argtypes = [P]
    L.panns_efanna_build.argtypes = [i32, P, u32, u32, P, u32, u32, u32, u32, u32, ctypes.POINTER(P)]
    for name in EXPORTS:
        getattr(L, name).restype = getattr(L, name).restype or ctypes.c_int
    L.panns_last_error.restype = ctypes.c_char_p
    L.panns_version.restype = u32
    _lib = L
    return L


def check(rc: int):
    if rc != PANNS_OK:
        msg = load().panns_last_error()
        raise PannsError(rc, msg.decode() if msg else "")
    return rc


def ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)
