"""ctypes binding of the C ABI declared in include/ltg.h.

Loads the in-tree libtensor_b200/_lib/libltg.so.  There is no fallback: if the
library is missing or cannot be loaded, importing the operations raises.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libltg.so")

c_i32p = C.POINTER(C.c_int32)
c_i64p = C.POINTER(C.c_int64)
c_dblp = C.POINTER(C.c_double)
c_vp = C.c_void_p

LTG_OK = 0
ERRORS = {
    1: "LTG_ERR_BAD_ARG", 2: "LTG_ERR_BAD_DIMS", 3: "LTG_ERR_SYMMETRY",
    4: "LTG_ERR_UNSUPPORTED", 5: "LTG_ERR_OOM", 6: "LTG_ERR_CUDA",
    7: "LTG_ERR_TIMEOUT", 8: "LTG_ERR_STATE",
}
MODE_PLAIN_FP64, MODE_OZAKI_BF16, MODE_OZAKI_FP8, MODE_OZAKI_INT8, MODE_OZAKI_CRT = 0, 1, 2, 3, 4


class ltg_bt_spec(C.Structure):
    _fields_ = [
        ("order", C.c_int32),
        ("dims", c_i64p),
        ("nsplit", c_i32p),
        ("splits", c_i64p),
        ("nperm", C.c_int32),
        ("perm", c_i32p),
        ("perm_coeff", c_dblp),
        ("has_part", C.c_int32),
        ("part_pdims", c_i64p),
        ("npart_forbidden", C.c_int64),
        ("part_forbidden", c_i64p),
        ("has_label", C.c_int32),
        ("label_nirrep", C.c_int32),
        ("labels", c_i32p),
        ("label_nintr", C.c_int32),
        ("label_intr", c_i32p),
    ]


# name -> (restype, argtypes)
_SIGS = {
    "ltg_last_error": (C.c_char_p, []),
    "ltg_version": (C.c_int, []),
    "ltg_ctx_create": (C.c_int, [C.c_int, C.POINTER(c_vp)]),
    "ltg_ctx_destroy": (C.c_int, [c_vp]),
    "ltg_ctx_synchronize": (C.c_int, [c_vp]),
    "ltg_ctx_stream": (C.c_int, [c_vp, C.POINTER(c_vp)]),
    "ltg_ctx_set_host_threads": (C.c_int, [c_vp, C.c_int]),
    "ltg_ctx_set_wait_limit": (C.c_int, [c_vp, C.c_uint64]),
    "ltg_ctx_wait_limit": (C.c_int, [c_vp, C.POINTER(C.c_uint64)]),
    "ltg_ctx_launch_count": (C.c_int, [c_vp, c_i64p]),
    "ltg_bt_create": (C.c_int, [c_vp, C.POINTER(ltg_bt_spec), C.POINTER(c_vp)]),
    "ltg_bt_create_permuted": (C.c_int, [c_vp, c_i32p, C.POINTER(c_vp)]),
    "ltg_bt_create_sum_space": (C.c_int, [C.c_int32, C.POINTER(c_vp), c_i32p, C.POINTER(c_vp)]),
    "ltg_bt_create_symmetrized": (C.c_int, [c_vp, C.c_int32, c_i32p, C.c_int32, C.POINTER(c_vp)]),
    "ltg_symmetrize": (C.c_int, [c_vp, C.c_double, C.c_int32, c_i32p, C.c_int32, c_vp, C.c_int32, C.c_double]),
    "ltg_contract2_make_symmetrized": (C.c_int, [c_vp, C.c_int32, c_i32p, C.c_int32, C.POINTER(c_vp)]),
    "ltg_contract2_symmetrized": (C.c_int, [c_vp, c_vp, C.c_int32, C.c_int32, C.c_double, C.c_int32, c_i32p,
                                            C.c_int32, C.c_double, C.c_double, C.c_double]),
    "ltg_bt_destroy": (C.c_int, [c_vp]),
    "ltg_bt_info": (C.c_int, [c_vp, c_i32p, c_i64p, c_i64p]),
    "ltg_bt_blocks": (C.c_int, [c_vp, c_i64p, c_i64p, c_i64p]),
    "ltg_bt_bidims": (C.c_int, [c_vp, c_i64p]),
    "ltg_bt_block_dims": (C.c_int, [c_vp, c_i64p, c_i64p]),
    "ltg_bt_nonzero": (C.c_int, [c_vp, c_i64p, C.c_int64, c_i64p]),
    "ltg_bt_orbit": (C.c_int, [c_vp, C.c_int64, c_i64p, c_i32p, c_dblp, c_i32p]),
    "ltg_bt_upload": (C.c_int, [c_vp, c_dblp]),
    "ltg_bt_download": (C.c_int, [c_vp, c_dblp]),
    "ltg_bt_upload_block": (C.c_int, [c_vp, c_i64p, c_dblp]),
    "ltg_bt_download_block": (C.c_int, [c_vp, c_i64p, c_dblp]),
    "ltg_bt_upload_async": (C.c_int, [c_vp, c_vp]),
    "ltg_bt_download_async": (C.c_int, [c_vp, c_vp]),
    "ltg_bt_set_zero": (C.c_int, [c_vp]),
    "ltg_bt_mark_nonzero": (C.c_int, [c_vp]),
    "ltg_bt_zero_block": (C.c_int, [c_vp, c_i64p]),
    "ltg_bt_fill_seeded": (C.c_int, [c_vp, C.c_uint64, C.c_double]),
    "ltg_bt_fill_seeded_host": (C.c_int, [c_vp, C.c_uint64, C.c_double, c_dblp]),
    "ltg_bt_device_ptr": (C.c_int, [c_vp, C.POINTER(c_vp)]),
    "ltg_contract2_create": (C.c_int, [c_vp, C.c_int32, C.c_int32, C.c_int32, c_i32p, c_i32p,
                                       c_vp, c_vp, C.POINTER(c_vp)]),
    "ltg_contract2_make_result": (C.c_int, [c_vp, C.POINTER(c_vp)]),
    "ltg_plan_schedule": (C.c_int, [c_vp, c_i64p, C.c_int64, c_i64p]),
    "ltg_plan_pairs": (C.c_int, [c_vp, C.c_int64, c_i64p, C.c_int64, c_i64p]),
    "ltg_plan_flops": (C.c_int, [c_vp, c_dblp]),
    "ltg_contract2": (C.c_int, [c_vp, c_vp, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                C.c_double, C.c_int32, C.c_double]),
    "ltg_plan_destroy": (C.c_int, [c_vp]),
    "ltg_contract2_set_tile": (C.c_int, [c_vp, C.c_int32]),
    "ltg_schedule_cache_set_capacity": (C.c_int, [C.c_int64]),
    "ltg_schedule_cache_stats": (C.c_int, [c_i64p, c_i64p, c_i64p]),
    "ltg_contract2_set_split_k": (C.c_int, [c_vp, C.c_int32]),
    "ltg_contract2_set_grouping": (C.c_int, [c_vp, C.c_int32]),
    "ltg_contract2_set_fused_split": (C.c_int, [c_vp, C.c_int32]),
    "ltg_contract2_set_crt_bound": (C.c_int, [c_vp, C.c_int32]),
    "ltg_contract2_set_crt_stage": (C.c_int, [c_vp, C.c_int32]),
    "ltg_contract2_group_info": (C.c_int, [c_vp, c_vp, c_i64p, c_i64p, c_dblp, c_dblp]),
    "ltg_contract2_set_crt_rows": (C.c_int, [c_vp, C.c_int32]),
    "ltg_contract2_autotune": (C.c_int, [c_vp, c_vp, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                         C.c_double, C.c_int32]),
    "ltg_plan_tiles": (C.c_int, [c_vp, c_i64p, c_i64p, c_i32p, C.c_int64, c_i64p]),
    "ltg_copy": (C.c_int, [c_vp, c_i32p, C.c_double, c_vp, C.c_int32, C.c_double]),
    "ltg_add": (C.c_int, [C.c_int32, C.POINTER(c_vp), c_i32p, c_dblp, c_vp, C.c_int32, C.c_double]),
    "ltg_dotprod": (C.c_int, [c_vp, c_i32p, c_vp, c_i32p, c_dblp]),
    "ltg_dotprod_async": (C.c_int, [c_vp, c_i32p, c_vp, c_i32p, c_vp]),
    "ltg_dot_noalloc": (C.c_int, [c_vp, c_vp, C.c_int64, c_vp, c_dblp]),
    "ltg_contract2_split_bytes": (C.c_int, [c_vp, c_vp, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                            C.c_double, C.c_int32, C.c_double, c_i64p, c_i64p]),
    "ltg_ctx_set_timing": (C.c_int, [c_vp, C.c_int32]),
    "ltg_ctx_kernel_times": (C.c_int, [c_vp, c_dblp, c_i64p]),
    "ltg_scale": (C.c_int, [c_vp, C.c_double]),
    "ltg_denominator": (C.c_int, [c_vp, c_dblp, C.c_int32]),
    "ltg_graph_begin": (C.c_int, [c_vp]),
    "ltg_graph_end": (C.c_int, [c_vp, C.POINTER(c_vp)]),
    "ltg_graph_launch": (C.c_int, [c_vp]),
    "ltg_graph_destroy": (C.c_int, [c_vp]),
    "ltg_plan_export_tasks": (C.c_int, [c_vp, c_vp, c_i64p, C.c_int64, c_i64p]),
    "ltg_plan_contract2_upload": (C.c_int, [c_vp, c_vp, c_vp, c_i64p, C.c_int64, C.POINTER(c_vp)]),
    "ltg_bt_alloc": (C.c_int, [c_vp, C.POINTER(ltg_bt_spec), C.POINTER(c_vp)]),
    "ltg_bt_free": (C.c_int, [c_vp]),
    "ltg_bt_upload_blocks": (C.c_int, [c_vp, c_dblp]),
    "ltg_bt_download_blocks": (C.c_int, [c_vp, c_dblp]),
    "ltg_plan_free": (C.c_int, [c_vp]),
    "ltg_copy_perm": (C.c_int, [c_vp, c_i32p, C.c_double, c_vp, C.c_int32, C.c_double]),
    "ltg_add_perm_n": (C.c_int, [C.c_int32, C.POINTER(c_vp), c_i32p, c_dblp, c_vp, C.c_int32, C.c_double]),
    "ltg_last_error_string": (C.c_char_p, []),
}

# words per task record of ltg_plan_export_tasks / ltg_plan_contract2_upload
LTG_TASK_WORDS = 43

_lib = None


def lib():
    """Loads libltg.so (raises OSError if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: run `python -m libtensor_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def declared_symbols():
    return sorted(_SIGS)


class LtgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def check(status):
    if status != LTG_OK:
        raise LtgError(status, lib().ltg_last_error().decode(errors="replace"))
    return status
