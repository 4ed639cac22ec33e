"""ctypes binding of libwmd_b200.so (the C ABI declared in include/wmd_b200.h).

Loading fails loudly when the library is missing: there is no Python or CPU
fallback for any solve.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwmd_b200.so")

c_u64 = ctypes.c_uint64
c_f64p = ctypes.POINTER(ctypes.c_double)
c_f32p = ctypes.POINTER(ctypes.c_float)
c_u64p = ctypes.POINTER(ctypes.c_uint64)
c_i64p = ctypes.POINTER(ctypes.c_int64)

STATUS = {
    0: "WMD_OK", 1: "WMD_ERR_INVALID_ARG", 2: "WMD_ERR_INVALID_INPUT",
    3: "WMD_ERR_OUT_OF_MEMORY", 4: "WMD_ERR_CUDA", 5: "WMD_ERR_NO_DEVICE",
    6: "WMD_ERR_UNSUPPORTED", 7: "WMD_ERR_DEVICE_TIMEOUT",
}

CDIST_MODES = {"fp32": 0, "bf16": 1, "fp16": 2, "tf32x3": 3, "f16x3": 4}


class WMDError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        self.name = STATUS.get(status, f"status {status}")
        super().__init__(f"{self.name}: {message}")


class CSR(ctypes.Structure):
    """Mirror of puma_csr_double_t (common.h:38-46)."""
    _fields_ = [("num_rows", c_u64), ("num_cols", c_u64), ("nnz", c_u64),
                ("row_ptr", c_u64p), ("col_inds", c_u64p), ("vals", c_f64p)]


class CSC(ctypes.Structure):
    """Mirror of puma_csc_double_t (common.h:49-57)."""
    _fields_ = [("num_rows", c_u64), ("num_cols", c_u64), ("nnz", c_u64),
                ("col_ptr", c_u64p), ("row_inds", c_u64p), ("vals", c_f64p)]


# (name, restype, argtypes) for every entry point of include/wmd_b200.h.
_SIGS = [
    ("wmd_sinkhorn_fused", ctypes.c_int,
     [c_f64p, c_f64p, c_f64p, ctypes.c_double, ctypes.c_int, c_u64, c_u64,
      c_u64, ctypes.POINTER(CSR)]),
    ("wmd_sinkhorn_nonfused", ctypes.c_int,
     [c_f64p, c_f64p, c_f64p, ctypes.c_double, ctypes.c_int, c_u64, c_u64,
      c_u64, ctypes.POINTER(CSR)]),
    ("wmd_sinkhorn_fused_csc", ctypes.c_int,
     [c_f64p, c_f64p, c_f64p, ctypes.c_double, ctypes.c_int, c_u64, c_u64,
      c_u64, ctypes.POINTER(CSC)]),
    ("wmd_sinkhorn_nonfused_csc", ctypes.c_int,
     [c_f64p, c_f64p, c_f64p, ctypes.c_double, ctypes.c_int, c_u64, c_u64,
      c_u64, ctypes.POINTER(CSC)]),
    ("wmd_create", ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]),
    ("wmd_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("wmd_set_embeddings_f64", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, c_u64, c_u64, ctypes.c_int]),
    ("wmd_set_embeddings_f32", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, c_u64, c_u64, ctypes.c_int]),
    ("wmd_set_embeddings_bf16", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, c_u64, c_u64, ctypes.c_int]),
    ("wmd_set_targets_csc", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(CSC)]),
    ("wmd_set_targets_csr", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(CSR)]),
    ("wmd_set_cdist_mode", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("wmd_set_solve_precision", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("wmd_set_solve_order", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("wmd_set_batch_mode", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64]),
    ("wmd_last_batch_groups", ctypes.c_int, [ctypes.c_void_p]),
    ("wmd_solve_shape_choices", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    ("wmd_group_shape_choices", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    ("wmd_solve_shape_name", ctypes.c_char_p, [ctypes.c_int]),
    ("wmd_set_autotune", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("wmd_set_relaxation", ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    ("wmd_autotune_choices", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    ("wmd_block_shape_name", ctypes.c_char_p, [ctypes.c_int]),
    ("wmd_set_block_shape", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("wmd_ws_param_count", ctypes.c_uint64, [ctypes.c_uint64]),
    ("wmd_ws_init_params", ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, c_f32p]),
    ("wmd_ws_build_training_set", ctypes.c_int,
     [ctypes.c_void_p, c_u64p, c_u64p, c_f64p, ctypes.c_uint64, ctypes.c_double,
      ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double, ctypes.c_int,
      ctypes.c_uint64, c_u64p, c_u64p, c_f64p]),
    ("wmd_ws_train", ctypes.c_int,
     [ctypes.c_void_p, c_f32p, ctypes.c_int, ctypes.c_uint64, ctypes.c_float,
      ctypes.c_uint64, c_f64p]),
    ("wmd_ws_loss_grad", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_uint64, c_f32p, c_f32p, c_i64p, ctypes.c_uint64, c_f32p,
      c_f64p, c_f32p]),
    ("wmd_ws_get_training_set", ctypes.c_int,
     [ctypes.c_void_p, c_f32p, c_f32p, c_i64p, ctypes.POINTER(ctypes.c_uint32),
      ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_int32)]),
    ("wmd_set_warm_start", ctypes.c_int, [ctypes.c_void_p, c_f32p]),
    ("wmd_mtx_header", ctypes.c_int, [ctypes.c_char_p, c_u64p, c_u64p, c_u64p]),
    ("wmd_read_mtx", ctypes.c_int,
     [ctypes.c_char_p, ctypes.c_uint64, c_u64p, c_u64p, c_f64p, c_u64p]),
    ("wmd_read_vecs", ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_uint64, c_f64p]),
    ("wmd_read_r", ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint64, c_f64p]),
    ("wmd_edges_to_csc", ctypes.c_int,
     [ctypes.c_void_p, c_u64p, c_u64p, c_f64p, ctypes.c_uint64, ctypes.c_uint64,
      ctypes.c_uint64, c_u64p, c_u64p, c_f64p]),
    ("wmd_set_targets_edges", ctypes.c_int,
     [ctypes.c_void_p, c_u64p, c_u64p, c_f64p, ctypes.c_uint64, ctypes.c_uint64,
      ctypes.c_uint64]),
    ("wmd_ws_init_scalings", ctypes.c_int,
     [ctypes.c_void_p, c_f64p, ctypes.c_double, c_f32p, c_u64p]),
    ("wmd_query_dense", ctypes.c_int,
     [ctypes.c_void_p, c_f64p, ctypes.c_double, ctypes.c_int, c_f64p]),
    ("wmd_query_dense_device", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, c_u64, ctypes.c_double, ctypes.c_int,
      ctypes.c_void_p]),
    ("wmd_check", ctypes.c_int, [ctypes.c_void_p]),
    ("wmd_selftest_bounded_wait", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    ("wmd_probe_roofline", ctypes.c_int,
     [ctypes.c_int, ctypes.c_uint64, c_f64p, c_f64p]),
    ("wmd_stream", ctypes.c_void_p, [ctypes.c_void_p]),
    ("wmd_last_launch_count", ctypes.c_int, [ctypes.c_void_p]),
    ("wmd_query_topk", ctypes.c_int,
     [ctypes.c_void_p, c_f64p, ctypes.c_double, ctypes.c_int, ctypes.c_uint32,
      ctypes.POINTER(ctypes.c_uint32), c_f64p]),
    ("wmd_topk_device", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, c_u64, ctypes.c_uint32, ctypes.c_void_p,
      ctypes.c_void_p]),
    ("wmd_query_batch", ctypes.c_int,
     [ctypes.c_void_p, c_u64p, c_u64p, c_f64p, c_u64, ctypes.c_double,
      ctypes.c_int, c_f64p, ctypes.POINTER(ctypes.c_int)]),
    ("wmd_set_tolerance", ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    ("wmd_last_iterations", ctypes.c_int,
     [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    ("wmd_set_timing", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("wmd_stage_times", ctypes.c_int,
     [ctypes.c_void_p, c_f32p, c_f32p, c_f32p]),
    ("wmd_sinkhorn_noalloc", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, c_u64, c_u64, ctypes.c_void_p,
      ctypes.c_void_p, ctypes.c_void_p, c_u64, c_u64, c_u64, ctypes.c_double,
      ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    ("wmd_status_string", ctypes.c_char_p, [ctypes.c_int]),
    ("wmd_last_error", ctypes.c_char_p, []),
    ("wmd_abi_version", ctypes.c_int, []),
    ("wmd_dropin_h2d_bytes", ctypes.c_uint64, []),
]

_lib = None


def lib():
    """Load libwmd_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with "
                f"`python {os.path.join(HERE, 'build.py')}`")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_names():
    return [s[0] for s in _SIGS]


def check(status: int):
    if status != 0:
        msg = lib().wmd_last_error().decode(errors="replace")
        raise WMDError(status, msg)
