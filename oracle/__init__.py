"""ctypes view of the CPU oracle (oracle/_build/liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg. The product package never imports this module.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")


def _load():
    if not os.path.exists(LIB_PATH):
        import subprocess
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return C.CDLL(LIB_PATH)


lib = _load()
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
i32, i64, f32, f64, u64 = C.c_int, C.c_longlong, C.c_float, C.c_double, C.c_ulonglong

lib.oracle_add.argtypes = [_fp, _fp, _fp, i64]
lib.oracle_reduce_fold.argtypes = [C.POINTER(C.c_void_p), i32, _fp, i64]
lib.oracle_reduce_f64.argtypes = [C.POINTER(C.c_void_p), i32, _dp, i64]
lib.oracle_unary.argtypes = [i32, _fp, _fp, i64, f32]
lib.oracle_binary.argtypes = [i32, _fp, _fp, _fp, i64, f32, f32]
lib.oracle_bias_add.argtypes = [_fp, _fp, _fp, i32, i32, i32]
lib.oracle_colsum.argtypes = [_fp, _fp, i32, i32, i64, i32]
lib.oracle_softmax_ce_f64.argtypes = [_fp, _ip, _dp, C.c_void_p, i32, i32, i64, f64]
lib.oracle_matmul_f64.argtypes = [_fp, _fp, _dp, i32, i32, i32, i64, i64, i64, i32, i32]
lib.oracle_sgemm_mt.argtypes = [_fp, _fp, _fp, i32, i32, i32, i64, i64, i64, i32, i32, i32]
lib.oracle_contraction_f64.argtypes = [_fp, i32, _i64p, _ip, _fp, i32, _i64p, _ip, _dp, i32, _ip, f64]
lib.oracle_philox.argtypes = [u64, i64, _u32p]
lib.oracle_uniform.argtypes = [u64, i64, f32, f32, _fp]


def _f32(x):
    return np.ascontiguousarray(x, dtype=np.float32)


def add(a, b):
    a, b = _f32(a), _f32(b)
    c = np.empty_like(a)
    lib.oracle_add(a, b, c, a.size)
    return c


def reduce_fold(inputs):
    ins = [_f32(x) for x in inputs]
    out = np.empty_like(ins[0])
    arr = (C.c_void_p * len(ins))(*[x.ctypes.data for x in ins])
    lib.oracle_reduce_fold(arr, len(ins), out, out.size)
    return out


def reduce_f64(inputs):
    ins = [_f32(x) for x in inputs]
    out = np.empty(ins[0].shape, dtype=np.float64)
    arr = (C.c_void_p * len(ins))(*[x.ctypes.data for x in ins])
    lib.oracle_reduce_f64(arr, len(ins), out, out.size)
    return out


def unary(op, x, p=0.0):
    x = _f32(x)
    out = np.empty_like(x)
    lib.oracle_unary(op, x, out, x.size, p)
    return out


def binary(op, a, b, ca=1.0, cb=1.0):
    a, b = _f32(a), _f32(b)
    out = np.empty_like(a)
    lib.oracle_binary(op, a, b, out, a.size, ca, cb)
    return out


def bias_add(x, bias, relu=False):
    x, bias = _f32(x), _f32(bias)
    out = np.empty_like(x)
    lib.oracle_bias_add(x, bias, out, x.shape[0], x.shape[1], int(relu))
    return out


def colsum(x, init=None):
    x = _f32(x)
    out = _f32(init).copy() if init is not None else np.zeros(x.shape[1], np.float32)
    lib.oracle_colsum(x, out, x.shape[0], x.shape[1], x.shape[1], int(init is not None))
    return out


def softmax_ce_f64(z, y, grad_scale=1.0, want_grad=True):
    z = _f32(z)
    y = np.ascontiguousarray(y, dtype=np.int32)
    rows, cols = z.shape
    loss = np.empty(rows, np.float64)
    grad = np.empty((rows, cols), np.float64) if want_grad else None
    lib.oracle_softmax_ce_f64(z, y, loss, grad.ctypes.data if want_grad else None, rows, cols, cols, grad_scale)
    return loss, grad


def matmul_f64(a, b, trans_a=False, trans_b=False):
    a, b = _f32(a), _f32(b)
    m = a.shape[1] if trans_a else a.shape[0]
    k = a.shape[0] if trans_a else a.shape[1]
    n = b.shape[0] if trans_b else b.shape[1]
    c = np.empty((m, n), np.float64)
    lib.oracle_matmul_f64(a, b, c, m, n, k, a.shape[1], b.shape[1], n, int(trans_a), int(trans_b))
    return c


def sgemm(a, b, trans_a=False, trans_b=False, threads=1):
    a, b = _f32(a), _f32(b)
    m = a.shape[1] if trans_a else a.shape[0]
    k = a.shape[0] if trans_a else a.shape[1]
    n = b.shape[0] if trans_b else b.shape[1]
    c = np.empty((m, n), np.float32)
    lib.oracle_sgemm_mt(a, b, c, m, n, k, a.shape[1], b.shape[1], n, int(trans_a), int(trans_b), threads)
    return c


def contraction_f64(lhs, dims_l, modes_l, rhs, dims_r, modes_r, modes_o, alpha=1.0):
    ext = {}
    for d, m in zip(dims_l, modes_l):
        ext[m] = d
    for d, m in zip(dims_r, modes_r):
        ext[m] = d
    nout = int(np.prod([ext[m] for m in modes_o])) if modes_o else 1
    out = np.empty(nout, np.float64)
    lib.oracle_contraction_f64(_f32(lhs).ravel(), len(dims_l), np.asarray(dims_l, np.int64), np.asarray(modes_l, np.int32),
                               _f32(rhs).ravel(), len(dims_r), np.asarray(dims_r, np.int64), np.asarray(modes_r, np.int32),
                               out, len(modes_o), np.asarray(modes_o if modes_o else [0], np.int32), alpha)
    return out


def philox(seed, ngroups):
    out = np.empty(4 * ngroups, np.uint32)
    lib.oracle_philox(seed, ngroups, out)
    return out


def uniform(seed, n, lo, hi):
    out = np.empty(n, np.float32)
    lib.oracle_uniform(seed, n, lo, hi, out)
    return out
