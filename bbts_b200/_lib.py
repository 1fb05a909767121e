"""ctypes binding of libbbts_b200.so (the C ABI declared in include/bbts_b200.h).

The library is loaded from the package directory; if it is missing the import
fails loudly -- there is no CPU fallback for any entry point.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbbts_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        "bbts_b200: native library %s is missing; build it with `python bbts_b200/build.py`" % LIB_PATH)

lib = C.CDLL(LIB_PATH)

vp, i32, i64, f32, u64, sz = C.c_void_p, C.c_int, C.c_longlong, C.c_float, C.c_ulonglong, C.c_size_t
pf = C.c_void_p  # device pointers are passed as integers


class TcProblem(C.Structure):
    """Mirror of bbx_tc_problem_t."""
    _fields_ = [("a", vp), ("b", vp), ("c", vp), ("bias", vp),
                ("m", i32), ("n", i32), ("k", i32),
                ("trans_a", i32), ("trans_b", i32), ("flags", i32),
                ("lda", i64), ("ldb", i64), ("ldc", i64),
                ("alpha", f32), ("beta", f32)]


# name -> (restype, argtypes); the order matches include/bbts_b200.h
SIGNATURES = {
    "bbx_version": (C.c_char_p, []),
    "bbx_last_error": (i32, [C.c_char_p, sz]),
    "bbx_num_sms": (i32, []),
    "bbx_check_device_status": (i32, [vp, C.POINTER(C.c_uint32)]),
    "bbx_matmul_f32": (i32, [pf, pf, pf, i32, i32, i32, i64, i64, i64, i32, i32, f32, f32, pf, i32,
                             i32, i64, i64, i64, vp]),
    "bbx_matmul_tc": (i32, [i32, C.POINTER(TcProblem), i32, i32, vp]),
    "bbx_tc_plan_create": (i32, [i32, C.POINTER(TcProblem), i32, i32, C.POINTER(vp)]),
    "bbx_tc_plan_launch": (i32, [vp, vp]),
    "bbx_tc_plan_destroy": (i32, [vp]),
    "bbx_tc_plan_tile_n": (i32, [vp]),
    "bbx_dag_profile": (i32, [vp, vp, i32, vp, vp, vp, vp, vp, C.POINTER(i32)]),
    "bbx_add_f32": (i32, [pf, pf, pf, i64, vp]),
    "bbx_reduce_f32": (i32, [C.POINTER(vp), i32, pf, i64, i32, vp]),
    "bbx_unary_f32": (i32, [i32, pf, pf, i64, f32, vp]),
    "bbx_binary_f32": (i32, [i32, pf, pf, pf, i64, f32, f32, vp]),
    "bbx_bias_add_f32": (i32, [pf, pf, pf, i32, i32, i32, vp]),
    "bbx_colsum_f32": (i32, [pf, pf, i32, i32, i64, i32, vp]),
    "bbx_cast": (i32, [i32, pf, i32, pf, i64, vp]),
    "bbx_relu_split": (i32, [pf, vp, vp, i64, vp]),
    "bbx_quantize_e4m3": (i32, [i32, pf, pf, i32, i32, i32, pf, vp]),
    "bbx_quantize_e4m3_batched": (i32, [i32, C.POINTER(vp), C.POINTER(vp), i32, i32, i32, i32, pf, vp]),
    "bbx_quantize_e4m3_batched_noalloc": (i32, [i32, C.POINTER(vp), C.POINTER(vp), i32, i32, i32, i32, pf, vp]),
    "bbx_fill_philox": (i32, [i32, pf, i64, u64, i32, f32, f32, vp]),
    "bbx_softmax_ce_f32": (i32, [pf, pf, pf, pf, i32, i32, i64, f32, vp]),
    "bbx_permute": (i32, [pf, i32, C.POINTER(i64), C.POINTER(i32), i32, pf, vp]),
    "bbx_contraction": (i32, [pf, i32, C.POINTER(i64), C.POINTER(i32), pf, i32, C.POINTER(i64),
                              C.POINTER(i32), pf, i32, C.POINTER(i32), f32, i32, vp]),
    "bbx_cu_reduction": (i32, [pf, i32, C.POINTER(i64), i32, f32, C.POINTER(i32), i32, pf, vp]),
    "bbx_cu_ew": (i32, [pf, i32, C.POINTER(i64), i32, f32, f32, C.POINTER(i32), pf, vp]),
    "bbx_cu_ewb": (i32, [pf, i32, C.POINTER(i64), C.POINTER(i32), pf, i32, C.POINTER(i64), C.POINTER(i32), i32,
                         f32, f32, pf, C.POINTER(i32), C.POINTER(i64), vp]),
    "bbx_cu_expand": (i32, [pf, C.POINTER(i32), i32, pf, vp]),
    "bbx_stream_group": (i32, [vp, i32, vp]),
    "bbx_stream_plan_create": (i32, [vp, i32, C.POINTER(vp)]),
    "bbx_stream_plan_launch": (i32, [vp, vp]),
    "bbx_stream_plan_destroy": (i32, [vp]),
    "bbx_stream_plan_bulk": (i32, [vp]),
    # runtime
    "bbx_rt_create": (i32, [C.POINTER(vp)]),
    "bbx_rt_destroy": (i32, [vp]),
    "bbx_rt_stream": (i32, [vp, C.POINTER(vp)]),
    "bbx_rt_fmt_id": (i32, [vp, C.c_char_p]),
    "bbx_rt_find_impl": (i32, [vp, C.c_char_p, C.c_char_p, C.c_char_p, i32, C.POINTER(i32), C.POINTER(i32)]),
    "bbx_rt_impl_name": (i32, [vp, i32, i32, C.c_char_p, sz]),
    "bbx_rt_complexity": (i32, [vp, i32, i32, C.POINTER(C.c_uint32), i32, vp, i32, C.POINTER(u64)]),
    "bbx_rt_tensor_put": (i32, [vp, i32, vp, vp, sz, i32]),
    "bbx_rt_tensor_get": (i32, [vp, i32, vp, vp, sz, i32]),
    "bbx_rt_tensor_payload": (i32, [vp, i32, C.POINTER(vp), C.POINTER(sz)]),
    "bbx_rt_tensor_count": (i32, [vp]),
    "bbx_rt_tensor_remove": (i32, [vp, i32]),
    "bbx_rt_queue_apply": (i32, [vp, i32, i32, i32, C.POINTER(C.c_uint32), i32, C.POINTER(i32), i32,
                                 C.POINTER(i32), i32]),
    "bbx_rt_queue_reduce": (i32, [vp, i32, i32, i32, C.POINTER(C.c_uint32), i32, C.POINTER(i32), i32, i32]),
    "bbx_rt_queue_delete": (i32, [vp, i32, C.POINTER(i32), i32]),
    "bbx_rt_clear_commands": (i32, [vp]),
    "bbx_rt_load_sbbts": (i32, [vp, C.c_char_p, C.POINTER(i32)]),
    "bbx_rt_load_bbts": (i32, [vp, C.c_char_p, C.POINTER(i32)]),
    "bbx_rt_save_bbts": (i32, [vp, C.c_char_p]),
    "bbx_rt_num_commands": (i32, [vp]),
    "bbx_rt_run": (i32, [vp, i32]),
    "bbx_rt_record": (i32, [vp, i32, vp, vp, vp, i32, C.POINTER(i32)]),
    "bbx_rt_set_workers": (i32, [vp, i32]),
    "bbx_rt_set_storage_budget": (i32, [vp, C.c_ulonglong, C.c_ulonglong, C.c_char_p]),
    "bbx_rt_spill_stats": (i32, [vp, C.POINTER(C.c_ulonglong), i32]),
    "bbx_rt_set_hint_predictor": (i32, [vp, C.c_double, C.c_double]),
    "bbx_dag_build": (i32, [vp, i32, i32, C.POINTER(vp)]),
    "bbx_dag_launch": (i32, [vp, vp]),
    "bbx_dag_destroy": (i32, [vp]),
    "bbx_dag_stats": (i32, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(i32), C.POINTER(i32),
                            C.POINTER(i32), C.POINTER(i32), C.POINTER(sz)]),
    "bbx_dag_tensor": (i32, [vp, i32, C.POINTER(vp), vp]),
    "bbx_dag_read": (i32, [vp, i32, vp, sz]),
    "bbx_stream_plan_create_kernel": (i32, [vp, i32, i32, C.POINTER(vp)]),
    "bbx_rt_set_dag_stream_kernel": (i32, [vp, i32]),
    "bbx_dag_register_waves": (i32, [vp]),
    "bbx_dag_write": (i32, [vp, i32, vp, sz, i32, vp]),
    "bbx_dag_fetch": (i32, [vp, i32, vp, sz, i32, vp]),
    "bbx_dag_group_tiles": (i32, [vp, i32, vp, C.POINTER(i32)]),
    # learned cost model
    "bbx_mlp_create": (i32, [u64, C.POINTER(vp)]),
    "bbx_mlp_destroy": (i32, [vp]),
    "bbx_mlp_set_norm": (i32, [vp, vp, vp]),
    "bbx_mlp_train": (i32, [vp, vp, vp, i32, i32, i32, f32, C.POINTER(f32)]),
    "bbx_mlp_predict": (i32, [vp, vp, i32, vp]),
    "bbx_mlp_loss_grad": (i32, [vp, vp, vp, i32, C.POINTER(f32), vp]),
    "bbx_mlp_num_params": (i32, []),
    "bbx_mlp_get_params": (i32, [vp, vp]),
    "bbx_mlp_set_params": (i32, [vp, vp]),
    "bbx_rt_set_predictor": (i32, [vp, vp]),
    "bbx_tile_record": (i32, [i32]),
    "bbx_tile_samples": (i32, [vp, vp, i32, C.POINTER(i32)]),
    "bbx_rt_set_tile_predictor": (i32, [vp, vp]),
}

for _name, (_res, _args) in SIGNATURES.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args


class BbxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("bbts_b200 error %d: %s" % (code, msg))
        self.code = code


def last_error():
    buf = C.create_string_buffer(2048)
    lib.bbx_last_error(buf, 2048)
    return buf.value.decode(errors="replace")


def check(rc):
    if rc != 0:
        raise BbxError(rc, last_error())
    return rc


def exported_symbols():
    """All bbx_* names the C header declares (parsed from include/bbts_b200.h)."""
    import re
    hdr = os.path.join(os.path.dirname(_HERE), "include", "bbts_b200.h")
    names = []
    for line in open(hdr):
        m = re.match(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_\s\*]*?\b(bbx_[a-z0-9_]+)\s*\(", line)
        if m:
            names.append(m.group(1))
    return names
