"""Torch-facing wrappers over the C ABI for tests and benchmarks.

torch supplies device memory and the current CUDA stream; every computation is
done by the library's own kernels through the C ABI (no torch math here).
"""
import ctypes as C

from ._lib import lib, check, TcProblem

F32, BF16, E4M3 = 0, 1, 2
U_RELU, U_RELU_DIF, U_SIGMOID_REF, U_SIGMOID, U_EXP, U_SQUARE, U_SQRT, U_ADD_SCALAR, U_SCALE = range(9)
B_ADD, B_WEIGHTED, B_HADAMARD, B_MAX, B_MIN, B_SUB, B_DIV = range(7)
EPI_RELU, EPI_OUT_BF16, EPI_BIAS, EPI_BETA, EPI_C_COLMAJOR = 1, 2, 4, 8, 32


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _dtype_code(t):
    import torch
    return {torch.float32: F32, torch.bfloat16: BF16, torch.float8_e4m3fn: E4M3}[t.dtype]


def matmul_f32(a, b, c, trans_a=False, trans_b=False, alpha=1.0, beta=0.0, bias=None, relu=False):
    """c = alpha*op(a)@op(b) + beta*c (+bias)(relu); 2-D or batched 3-D row-major tensors."""
    batched = a.dim() == 3
    A = a if batched else a.unsqueeze(0)
    B = b if batched else b.unsqueeze(0)
    Cc = c if batched else c.unsqueeze(0)
    m = A.shape[2] if trans_a else A.shape[1]
    k = A.shape[1] if trans_a else A.shape[2]
    n = B.shape[1] if trans_b else B.shape[2]
    check(lib.bbx_matmul_f32(_p(A), _p(B), _p(Cc), m, n, k, A.stride(1), B.stride(1), Cc.stride(1),
                             int(trans_a), int(trans_b), alpha, beta, _p(bias), int(relu), A.shape[0],
                             A.stride(0), B.stride(0), Cc.stride(0), _stream()))
    return c


def tc_problem(a, b, c, trans_a=False, trans_b=False, alpha=1.0, beta=0.0, bias=None, relu=False,
               c_colmajor=False):
    """c_colmajor: c holds C column-major, i.e. the n x m tensor C^T row-major."""
    import torch
    m = a.shape[1] if trans_a else a.shape[0]
    k = a.shape[0] if trans_a else a.shape[1]
    n = b.shape[0] if trans_b else b.shape[1]
    flags = (EPI_RELU if relu else 0) | (EPI_BIAS if bias is not None else 0) | \
            (EPI_BETA if beta != 0.0 else 0) | (EPI_OUT_BF16 if c.dtype == torch.bfloat16 else 0) | \
            (EPI_C_COLMAJOR if c_colmajor else 0)
    return TcProblem(a.data_ptr(), b.data_ptr(), c.data_ptr(), bias.data_ptr() if bias is not None else None,
                     m, n, k, int(trans_a), int(trans_b), flags, a.stride(0), b.stride(0), c.stride(0),
                     alpha, beta)


def matmul_tc(problems, in_dtype=BF16, tile_n=0):
    arr = (TcProblem * len(problems))(*problems)
    check(lib.bbx_matmul_tc(in_dtype, arr, len(problems), tile_n, _stream()))


# Groups whose largest K is at most this run with eight epilogue warps (the variant the
# plan picks; `kTcEp8MaxK` / `kTc2Ep8MaxK` in csrc/gemm_tc.cuh): 1-SM tiles, the 2-SM pair.
TC_EP8_MAX_K = 512
TC2_EP8_MAX_K = 1024


class TcPlan:
    """A prepared grouped tensor-core matmul (tensor maps built once)."""

    def __init__(self, problems, in_dtype=BF16, tile_n=0):
        arr = (TcProblem * len(problems))(*problems)
        self.h = C.c_void_p()
        self.in_dtype = in_dtype
        self.trans = (bool(problems[0].trans_a), bool(problems[0].trans_b))
        self.max_k = max(int(p.k) for p in problems)
        check(lib.bbx_tc_plan_create(in_dtype, arr, len(problems), tile_n, C.byref(self.h)))

    def launch(self, stream=None):
        check(lib.bbx_tc_plan_launch(self.h, stream if stream is not None else _stream()))

    @property
    def tile_n(self):
        """128 / 256 (1-SM 128 x tile_n tiles) or 512 (2-SM 256 x 256 pair)."""
        return lib.bbx_tc_plan_tile_n(self.h)

    @property
    def kernel_name(self):
        tn = self.tile_n
        a = "MN-major A" if self.trans[0] else "K-major A"
        b = "K-major B" if self.trans[1] else "MN-major B"
        if tn == 512:
            epi = "8 epilogue warps" if self.max_k <= TC2_EP8_MAX_K else "4 epilogue warps"
            return "tc_gemm2_kernel<%s,%s,%s> (2-SM 256x256 pair, cta_group::2)" % (a, b, epi)
        epi = "8 epilogue warps" if self.max_k <= TC_EP8_MAX_K else "4 epilogue warps"
        return "tc_gemm_kernel<%d,%s,%s,%s,%s>" % (tn, a, b, "e4m3" if self.in_dtype == E4M3 else "bf16", epi)

    def close(self):
        if self.h:
            lib.bbx_tc_plan_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


S_SUM, S_UNARY, S_BINARY, S_CAST = range(4)


class StreamOp(C.Structure):
    """bbx_stream_op_t: one add / n-ary reduce / elementwise / cast block op."""
    _fields_ = [("kind", C.c_int), ("op", C.c_int), ("in_dtype", C.c_int), ("out_dtype", C.c_int),
                ("n_in", C.c_int), ("kahan", C.c_int), ("n", C.c_longlong), ("inp", C.c_void_p * 16),
                ("out", C.c_void_p), ("p0", C.c_float), ("p1", C.c_float)]


def stream_op(kind, inputs, out, op=0, kahan=True, p0=0.0, p1=0.0, n=None):
    """A StreamOp over flat tensors (all inputs of one dtype)."""
    o = StreamOp()
    o.kind, o.op, o.n_in, o.kahan = kind, op, len(inputs), int(kahan)
    o.in_dtype, o.out_dtype = _dtype_code(inputs[0]), _dtype_code(out)
    o.n = out.numel() if n is None else n
    for j, t in enumerate(inputs):
        o.inp[j] = t.data_ptr()
    o.out = out.data_ptr()
    o.p0, o.p1 = p0, p1
    return o


def stream_group(ops):
    """One grouped launch (or one per 8 ops) of independent streaming ops."""
    arr = (StreamOp * len(ops))(*ops)
    check(lib.bbx_stream_group(C.cast(arr, C.c_void_p), len(ops), _stream()))


class StreamPlan:
    """A grouped streaming launch built once (op table on the device) and replayed."""

    def __init__(self, ops):
        arr = (StreamOp * len(ops))(*ops)
        self.h = C.c_void_p()
        check(lib.bbx_stream_plan_create(C.cast(arr, C.c_void_p), len(ops), C.byref(self.h)))

    def launch(self, stream=None):
        check(lib.bbx_stream_plan_launch(self.h, stream if stream is not None else _stream()))

    @property
    def bulk(self):
        """True when the plan runs the bulk-staged (cp.async.bulk) kernel."""
        r = lib.bbx_stream_plan_bulk(self.h)
        check(min(r, 0))
        return r == 1

    def close(self):
        if self.h:
            check(lib.bbx_stream_plan_destroy(self.h))
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def add(a, b, c):
    check(lib.bbx_add_f32(_p(a), _p(b), _p(c), a.numel(), _stream()))
    return c


def reduce(inputs, out, kahan=True):
    arr = (C.c_void_p * len(inputs))(*[t.data_ptr() for t in inputs])
    check(lib.bbx_reduce_f32(arr, len(inputs), _p(out), out.numel(), int(kahan), _stream()))
    return out


def unary(op, x, out, param=0.0):
    check(lib.bbx_unary_f32(op, _p(x), _p(out), x.numel(), param, _stream()))
    return out


def binary(op, a, b, out, ca=1.0, cb=1.0):
    check(lib.bbx_binary_f32(op, _p(a), _p(b), _p(out), a.numel(), ca, cb, _stream()))
    return out


def bias_add(x, bias, out, relu=False):
    check(lib.bbx_bias_add_f32(_p(x), _p(bias), _p(out), x.shape[0], x.shape[1], int(relu), _stream()))
    return out


def colsum(x, out, accumulate=False):
    check(lib.bbx_colsum_f32(_p(x), _p(out), x.shape[0], x.shape[1], x.stride(0), int(accumulate), _stream()))
    return out


def relu_split(z, hi, lo):
    """hi = bf16(relu(z)), lo = bf16(relu(z) - hi) for an f32 tensor z."""
    check(lib.bbx_relu_split(_p(z), _p(hi), _p(lo), z.numel(), _stream()))
    return hi, lo


def cast(x, out):
    check(lib.bbx_cast(_dtype_code(x), _p(x), _dtype_code(out), _p(out), x.numel(), _stream()))
    return out


def quantize_e4m3(x, out, scale_out, transpose=False):
    rows, cols = x.shape
    check(lib.bbx_quantize_e4m3(_dtype_code(x), _p(x), _p(out), rows, cols, int(transpose),
                                _p(scale_out), _stream()))
    return out


def quantize_e4m3_batched(xs, outs, scales_out, transpose=False):
    """quantize_e4m3 over a list of equally shaped blocks in one call;
    scales_out: a device tensor of len(xs) floats."""
    rows, cols = xs[0].shape
    arr_in = (C.c_void_p * len(xs))(*[x.data_ptr() for x in xs])
    arr_out = (C.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
    check(lib.bbx_quantize_e4m3_batched(_dtype_code(xs[0]), arr_in, arr_out, len(xs), rows, cols, int(transpose),
                                        _p(scales_out), _stream()))
    return outs


def fill_philox(out, seed, dist=0, a=0.0, b=1.0):
    check(lib.bbx_fill_philox(_dtype_code(out), _p(out), out.numel(), seed, dist, a, b, _stream()))
    return out


def softmax_ce(logits, labels, loss, grad=None, grad_scale=1.0):
    rows, cols = logits.shape
    check(lib.bbx_softmax_ce_f32(_p(logits), _p(labels), _p(loss), _p(grad), rows, cols,
                                 logits.stride(0), grad_scale, _stream()))
    return loss


def permute(x, perm, out):
    rank = x.dim()
    dims = (C.c_longlong * rank)(*x.shape)
    pm = (C.c_int * rank)(*perm)
    check(lib.bbx_permute(_p(x), rank, dims, pm, _dtype_code(out), _p(out), _stream()))
    return out


def _ints(v, ctype=C.c_int):
    return (ctype * max(1, len(v)))(*v)


def cu_reduction(x, dims, op, alpha, ordering, out):
    """out (dims[ordering]...) = alpha * fold_op over the modes not in ordering
    (op 0 add, 1 max, 2 min, 3 mul); column-major FP32."""
    check(lib.bbx_cu_reduction(_p(x), len(dims), _ints(dims, C.c_longlong), op, alpha, _ints(ordering),
                               len(ordering), _p(out), _stream()))
    return out


def cu_ew(x, dims, uop, alpha, ordering, out, scalar=0.0):
    """out = alpha * uop(x) with output mode r = input mode ordering[r]."""
    check(lib.bbx_cu_ew(_p(x), len(dims), _ints(dims, C.c_longlong), uop, scalar, alpha, _ints(ordering), _p(out),
                        _stream()))
    return out


def cu_ewb(lhs, dims_l, ord_l, rhs, dims_r, ord_r, op, alpha, beta, out):
    """out = op(alpha * lhs, beta * rhs), broadcast over the output modes each
    side lacks; returns the output dims."""
    ro = C.c_int()
    do = (C.c_longlong * 4)()
    check(lib.bbx_cu_ewb(_p(lhs), len(dims_l), _ints(dims_l, C.c_longlong), _ints(ord_l), _p(rhs), len(dims_r),
                         _ints(dims_r, C.c_longlong), _ints(ord_r), op, alpha, beta, _p(out), C.byref(ro), do,
                         _stream()))
    return [do[i] for i in range(ro.value)]


def cu_expand(x, params5, out):
    """Zero `out`, then copy the box given per mode as (sz_in, sz_out, num,
    start_in, start_out)."""
    check(lib.bbx_cu_expand(_p(x), _ints(params5), len(params5) // 5, _p(out), _stream()))
    return out


def contraction(lhs, dims_l, modes_l, rhs, dims_r, modes_r, out, modes_o, alpha=1.0, precision=F32):
    """Column-major einsum (the cutensor format): tensors are flat device buffers."""
    dl = (C.c_longlong * len(dims_l))(*dims_l)
    ml = (C.c_int * len(modes_l))(*modes_l)
    dr = (C.c_longlong * len(dims_r))(*dims_r)
    mr = (C.c_int * len(modes_r))(*modes_r)
    mo = (C.c_int * max(1, len(modes_o)))(*modes_o)
    check(lib.bbx_contraction(_p(lhs), len(dims_l), dl, ml, _p(rhs), len(dims_r), dr, mr, _p(out),
                              len(modes_o), mo, alpha, precision, _stream()))
    return out
