"""ctypes binding of libhnswgpu.so (the C ABI declared in include/hnswgpu.h).

The library is loaded from this package directory.  There is no fallback: if
it has not been built (``python -m hnsw_rabitq_b200.build``) or cannot be
loaded, every use raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhnswgpu.so")

OK = 0
ERR_ARG, ERR_IO, ERR_FORMAT, ERR_CUDA, ERR_NOMEM, ERR_LABEL, ERR_STATE, ERR_KERNEL, ERR_UNSUPPORTED = \
    -1, -2, -3, -4, -5, -6, -7, -8, -9
SPACE_L2, SPACE_IP, SPACE_COSINE, SPACE_L2_UINT8 = 0, 1, 2, 3
DEVICE_PTRS = 0x1
TRACE = 0x2
EXACT_TIES = 0x4
LEARNED_STOP = 0x8
EXACT_SCAN = 0x10
REPLAY_ALL = 0x20
TERM_FEATURES = 16
TERM_HIDDEN = 64
TERM_PARAMS = 5345
PREC_FP32, PREC_BF16, PREC_FP8 = 0, 1, 2
STATUS_TIMEOUT = 0x1
STATUS_OVERFLOW = 0x2

# Every function the header declares, with its ctypes signature.
P, U64, U32, I32 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int32


class Info(C.Structure):
    _fields_ = [("count", U64), ("max_elements", U64), ("dim", U64), ("M", U64), ("maxM", U64), ("maxM0", U64),
                ("ef_construction", U64), ("ef", U64), ("num_deleted", U64), ("maxlevel", I32),
                ("enterpoint", U32), ("space", I32), ("is_bruteforce", I32), ("device_bytes", U64)]


class SearchOpts(C.Structure):
    _fields_ = [("flags", U32), ("precision", U32), ("ef", U64), ("allow", P), ("trace", P), ("stream", P),
                ("rerank", U32), ("filter", U32)]


class TermTrainOpts(C.Structure):
    _fields_ = [("epochs", U32), ("batch", U32), ("lr", C.c_float), ("pos_weight", C.c_float),
                ("weight_decay", C.c_float), ("reserved", U32), ("seed", U64)]


class ServerOpts(C.Structure):
    _fields_ = [("max_inflight", U32), ("max_batch", U32), ("smem_budget", U64)]


class Request(C.Structure):
    _fields_ = [("k", U32), ("ef", U32), ("filter", I32), ("flags", U32), ("precision", U32), ("rerank", U32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", U64), ("completed", U64), ("batches", U64), ("mean_batch", C.c_double),
                ("p50_us", C.c_double), ("p99_us", C.c_double), ("mean_us", C.c_double), ("max_us", C.c_double)]


SIGNATURES = {
    "hnswgpu_last_error": (C.c_char_p, []),
    "hnswgpu_version": (C.c_char_p, []),
    "hnswgpu_load_hnsw": (C.c_int, [C.c_char_p, C.c_int, U64, U64, C.c_int, C.POINTER(P)]),
    "hnswgpu_load_hnsw_buffer": (C.c_int, [P, U64, C.c_int, U64, U64, C.c_int, C.POINTER(P)]),
    "hnswgpu_load_bf": (C.c_int, [C.c_char_p, C.c_int, U64, C.c_int, C.POINTER(P)]),
    "hnswgpu_create_bf": (C.c_int, [C.c_int, U64, P, P, U64, U64, C.c_int, C.POINTER(P)]),
    "hnswgpu_free": (C.c_int, [P]),
    "hnswgpu_build_traversal_copy": (C.c_int, [P, U32]),
    "hnswgpu_get_info": (C.c_int, [P, C.POINTER(Info)]),
    "hnswgpu_set_ef": (C.c_int, [P, U64]),
    "hnswgpu_get_labels": (C.c_int, [P, P]),
    "hnswgpu_mark_deleted": (C.c_int, [P, U64]),
    "hnswgpu_unmark_deleted": (C.c_int, [P, U64]),
    "hnswgpu_search": (C.c_int, [P, P, U64, U64, C.POINTER(SearchOpts), P, P, P]),
    "hnswgpu_get_status": (C.c_int, [P, C.POINTER(U32)]),
    "hnswgpu_search_noalloc": (C.c_int, [P, P, U64, U64, U64, U32, P, P, P, P, P]),
    "hnswgpu_noalloc_get_status": (C.c_int, [C.c_int, P, C.POINTER(U32)]),
    "hnswgpu_filter_create": (C.c_int, [P, P, C.POINTER(U32)]),
    "hnswgpu_load_hnsw_multivector": (C.c_int, [C.c_char_p, U64, U64, C.c_int, C.POINTER(P)]),
    "hnswgpu_search_multivector": (C.c_int, [P, P, U64, U64, U64, U64, P, P, P]),
    "hnswgpu_filter_destroy": (C.c_int, [P, U32]),
    "hnswgpu_save_hnsw": (C.c_int, [P, C.c_char_p]),
    "hnswgpu_selftest_wait_timeout": (C.c_int, [C.c_int, C.POINTER(U32)]),
    "hnswgpu_search_epsilon": (C.c_int, [P, P, U64, C.c_float, U64, U64, C.POINTER(SearchOpts), P, P, P]),
    "hnswgpu_set_termination_model": (C.c_int, [P, P, U32, C.c_float]),
    "hnswgpu_search_checkpoints": (C.c_int, [P, P, U64, U64, C.POINTER(SearchOpts), U32, U32, U32, P, P, P, P, P, P,
                                             P]),
    "hnswgpu_term_train": (C.c_int, [C.c_int, P, P, U64, C.POINTER(TermTrainOpts), P, P]),
    "hnswgpu_term_loss_grad": (C.c_int, [C.c_int, P, P, P, U64, C.c_float, P, P]),
    "hnswgpu_term_logits": (C.c_int, [C.c_int, P, P, U64, P]),
    "hnswgpu_fp64_distances": (C.c_int, [P, P, U64, P, U64, P]),
    "hnswgpu_server_create": (C.c_int, [P, C.POINTER(ServerOpts), C.POINTER(P)]),
    "hnswgpu_server_add_filter": (C.c_int, [P, P, C.POINTER(I32)]),
    "hnswgpu_server_submit": (C.c_int, [P, P, C.POINTER(Request), C.POINTER(U64)]),
    "hnswgpu_server_wait": (C.c_int, [P, U64, P, P, P, P]),
    "hnswgpu_server_replay": (C.c_int, [P, P, U64, P, P, U32, P, P, P, P]),
    "hnswgpu_server_get_stats": (C.c_int, [P, C.POINTER(ServerStats), C.c_int]),
    "hnswgpu_server_destroy": (C.c_int, [P]),
}

_lib = None


class HnswGpuError(RuntimeError):
    """A C-ABI call failed; ``code`` is its HNSWGPU_ERR_* status."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def lib():
    """The loaded library (raises if it is missing: there is no CPU path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m hnsw_rabitq_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != OK:
        raise HnswGpuError(rc, lib().hnswgpu_last_error().decode())
