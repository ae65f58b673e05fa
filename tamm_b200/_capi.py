"""ctypes binding of libtamm_b200.so (the C ABI in include/tamm_b200.h).

The library is built in-tree by tamm_b200/build.py.  Loading fails loudly when it
is missing: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtamm_b200.so")

TB_OK = 0
TB_ERR_INVALID = 1
TB_ERR_NOT_IMPLEMENTED = 2
TB_ERR_NO_MEMORY = 3
TB_ERR_CUDA = 4
TB_ERR_TIMEOUT = 5
TB_ERR_DEVICE = 6
TB_ERR_STATE = 7

TB_MODE_FP64 = 0
TB_MODE_INT8 = 1
TB_MODE_BF16X3 = 2
# element functions of tb_sched_map
TB_MAP_COPY, TB_MAP_SCALE, TB_MAP_SET, TB_MAP_SQUARE, TB_MAP_SQRT = 0, 1, 2, 3, 4
TB_MAP_LOG, TB_MAP_LOG10, TB_MAP_INVERSE, TB_MAP_POW, TB_MAP_ABS = 5, 6, 7, 8, 9

i64p = C.POINTER(C.c_int64)
i32p = C.POINTER(C.c_int32)
ip = C.POINTER(C.c_int)
dp = C.POINTER(C.c_double)
vp = C.c_void_p
h = C.c_void_p  # opaque handles


class tb_stats(C.Structure):
    _fields_ = [("flops", C.c_double), ("int8_ops", C.c_double), ("slices_min", C.c_int),
                ("slices_max", C.c_int), ("scratch_bytes", C.c_int64), ("split_ms", C.c_double),
                ("gemm_ms", C.c_double), ("mode", C.c_int), ("tile_n", C.c_int), ("flops_run", C.c_double),
                ("int8_ops_alg", C.c_double)]


# callbacks of lambda tensors (tb_block_fn, tb_batch_fn)
BLOCK_FN = C.CFUNCTYPE(C.c_int, i64p, C.c_int, i64p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p)
BATCH_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p)


class tb_labeled(C.Structure):
    _fields_ = [("tensor", h), ("labels", ip), ("label_tis", C.POINTER(h))]


# name -> argtypes (every function returns int status unless noted)
PROTOS = {
    "tb_last_error": [C.c_char_p, C.c_size_t],
    "tb_version": [ip, ip],
    "tb_block_multiply": [C.c_double, vp, i64p, ip, C.c_int, vp, i64p, ip, C.c_int, C.c_double, vp,
                          i64p, ip, C.c_int, C.c_int, C.c_int, vp],
    "tb_block_assign": [vp, i64p, ip, C.c_int, C.c_double, vp, i64p, ip, C.c_int, C.c_int, vp],
    "tb_block_multiply_int8_noalloc": [C.c_double, vp, i64p, ip, C.c_int, vp, i64p, ip, C.c_int, vp, i64p, ip,
                                       C.c_int, C.c_int, vp],
    "tb_fill": [vp, C.c_int64, C.c_double, C.c_int, vp],
    "tb_axpby": [C.c_double, vp, C.c_double, vp, C.c_int64, vp],
    "tb_norm2": [vp, C.c_int64, dp, vp],
    "tb_dot": [vp, vp, C.c_int64, dp, vp],
    "tb_fill_random": [vp, C.c_int64, C.c_uint64, C.c_uint64, C.c_int, C.c_double, C.c_double, vp],
    "tb_plan_contraction": [ip, C.c_int, ip, C.c_int, ip, C.c_int, C.c_int, C.c_double, C.c_int,
                            C.POINTER(h)],
    "tb_plan_destroy": [h],
    "tb_worklist_build": [h, C.c_int64, i64p, i32p, i64p, i64p, i64p, i32p, i32p, C.POINTER(h)],
    "tb_worklist_destroy": [h],
    "tb_worklist_info": [h, i64p, dp],
    "tb_contract": [h, h, C.c_double, vp, vp, vp, vp],
    "tb_plan_stats": [h, C.POINTER(tb_stats)],
    "tb_ctx_create": [C.c_int, C.c_int64, C.POINTER(h)],
    "tb_ctx_destroy": [h],
    "tb_ctx_set_precision": [h, C.c_int, C.c_double, C.c_int],
    "tb_ctx_stream": [h, C.POINTER(vp)],
    "tb_ctx_synchronize": [h],
    "tb_ctx_arena_info": [h, i64p, i64p, i64p],
    "tb_is_create": [C.c_int64, C.c_int, C.POINTER(C.c_char_p), ip, i64p, C.c_int, ip, ip, i64p,
                     C.POINTER(h)],
    "tb_is_destroy": [h],
    "tb_tis_create": [h, C.c_int64, i64p, C.c_int64, C.POINTER(h)],
    "tb_tis_named": [h, C.c_char_p, C.POINTER(h)],
    "tb_tis_subrange": [h, C.c_int64, C.c_int64, C.POINTER(h)],
    "tb_tis_num_tiles": [h, i64p],
    "tb_tis_tiles": [h, i64p, ip, i64p],
    "tb_tis_destroy": [h],
    "tb_tensor_create": [C.c_int, C.POINTER(h), ip, C.POINTER(h)],
    "tb_tensor_create_spin_sizes": [C.c_int, C.POINTER(h), C.c_int, C.c_int, C.POINTER(h)],
    "tb_tensor_allocate": [h, h],
    "tb_tensor_deallocate": [h],
    "tb_tensor_destroy": [h],
    "tb_tensor_info": [h, ip, i64p, i64p],
    "tb_tensor_block_table": [h, i64p, i64p],
    "tb_tensor_data": [h, C.POINTER(vp)],
    "tb_tensor_set_read_only": [h, C.c_int],
    "tb_tensor_record_use": [h],
    "tb_ctx_set_digit_cache": [h, C.c_int64],
    "tb_ctx_digit_cache_info": [h, i64p, i64p],
    "tb_tis_create_dependent": [h, C.c_int, C.POINTER(h), C.c_int64, i64p, C.POINTER(h), C.POINTER(h)],
    "tb_tensor_create_dependent": [C.c_int, C.POINTER(h), ip, ip, C.POINTER(h)],
    "tb_tensor_create_lambda": [C.c_int, C.POINTER(h), ip, C.c_void_p, C.c_void_p, C.POINTER(h)],
    "tb_tensor_create_built": [C.c_int, C.POINTER(h), ip, C.c_void_p, C.c_void_p, C.POINTER(h)],
    "tb_tensor_set_batch_bytes": [h, C.c_int64],
    "tb_tensor_space": [h, C.c_int, C.POINTER(h)],
    "tb_tensor_read_only_info": [h, ip, i64p, i64p],
    "tb_tensor_is_non_zero": [h, i64p, ip],
    "tb_tensor_block_size": [h, i64p, i64p],
    "tb_tensor_block_dims": [h, i64p, i64p],
    "tb_tensor_locate": [h, i64p, i64p],
    "tb_tensor_get": [h, i64p, dp, C.c_int64],
    "tb_tensor_put": [h, i64p, dp, C.c_int64],
    "tb_tensor_add": [h, i64p, dp, C.c_int64],
    "tb_tensor_write": [h, dp, C.c_int64],
    "tb_tensor_read": [h, dp, C.c_int64],
    "tb_tensor_norm": [h, dp],
    "tb_sched_create": [h, C.POINTER(h)],
    "tb_sched_destroy": [h],
    "tb_sched_set": [h, tb_labeled, C.c_double, C.c_int],
    "tb_sched_add": [h, tb_labeled, C.c_double, tb_labeled, C.c_int],
    "tb_sched_mult": [h, tb_labeled, C.c_double, tb_labeled, tb_labeled, C.c_int],
    "tb_mult_info": [tb_labeled, tb_labeled, tb_labeled, i64p, i64p, dp],
    "tb_sched_execute": [h, C.c_int, C.c_int],
    "tb_sched_profile": [h, i64p, dp, dp, C.c_int64],
    "tb_sched_clear": [h],
    "tb_sched_map": [h, tb_labeled, tb_labeled, C.c_int, C.c_double],
    "tb_sched_mult_n": [h, tb_labeled, C.c_double, C.POINTER(tb_labeled), C.c_int, C.c_int],
    "tb_opmin_order": [tb_labeled, C.POINTER(tb_labeled), C.c_int, i64p, dp],
    "tb_sched_release": [h],
    "tb_sched_op_stats": [h, C.c_int64, C.POINTER(tb_stats)],
    "tb_tensor_attach": [h, h, vp, C.c_int64],
    "tb_tensor_save": [h, C.c_char_p],
    "tb_ctx_join": [h],
    "tb_ctx_alloc": [h, C.c_int64, C.POINTER(vp)],
    "tb_ctx_free": [h, vp],
    "tb_tensor_write_async": [h, dp, C.c_int64],
    "tb_tensor_read_async": [h, dp, C.c_int64],
    "tb_sched_execute_async": [h],
    "tb_sched_wait": [h],
    "tb_tensor_load": [h, C.c_char_p],
    "tb_sched_set_owner": [h, C.c_int, C.c_int],
    "tb_mult_owned": [tb_labeled, tb_labeled, tb_labeled, C.c_int, C.c_int, i64p, dp, i64p, C.c_int64],
    "tb_sched_dot": [h, C.c_int, C.c_double, tb_labeled, tb_labeled],
    "tb_sched_norm": [h, C.c_int, C.c_double, tb_labeled],
    "tb_sched_scalars": [h, dp, C.c_int],
    "tb_sched_denom": [h, tb_labeled, C.c_double, tb_labeled, dp, C.c_int64, dp],
    "tb_sched_denom_energy": [h, C.c_int, C.c_double, tb_labeled, dp, C.c_int64, dp],
    "tb_sched_mult_energy": [h, C.c_int, C.c_double, tb_labeled, C.c_double, tb_labeled, tb_labeled, dp, C.c_int64,
                             dp],
    "tb_sched_set_scalar": [h, C.c_int, C.c_double],
    "tb_sched_autotune": [h, C.c_int],
    "tb_sched_tune_info": [h, C.c_int64, ip, ip, ip, ip, ip, dp, C.c_int],
    "tb_sched_graph_create": [h, C.POINTER(h)],
    "tb_graph_launch": [h],
    "tb_graph_sync": [h],
    "tb_graph_destroy": [h],
    "tb_tape_create": [h, C.c_int64, C.POINTER(h)],
    "tb_tape_destroy": [h],
    "tb_tape_leaf": [h, h, h],
    "tb_tape_contract": [h, tb_labeled, C.c_double, tb_labeled, tb_labeled],
    "tb_tape_dot": [h, C.c_double, tb_labeled, tb_labeled, dp],
    "tb_tape_backward": [h],
    "tb_tape_info": [h, i64p, dp, i64p, i64p],
    "tb_tape_reset": [h],
}

_lib = None


class TambError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{msg} (status {code})")
        self.code = code


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with tamm_b200/build.py "
                              "(there is no fallback implementation)")
        L = C.CDLL(LIB_PATH)
        for name, args in PROTOS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.tb_status_string.argtypes = [C.c_int]
        L.tb_status_string.restype = C.c_char_p
        _lib = L
    return _lib


def last_error():
    buf = C.create_string_buffer(1024)
    lib().tb_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(status):
    if status != TB_OK:
        raise TambError(status, last_error() or lib().tb_status_string(status).decode())
    return status


def call(name, *args):
    return check(getattr(lib(), name)(*args))
