"""The allocation-free FP8 quantisation entry point.

It serves callers that may not allocate device memory while they run (a
memory manager owning the whole GPU, latency paths where cudaMalloc would
synchronise, fixed-footprint deployments): its scratch is a fixed device
array inside the library. This file is collected last on purpose, so a run
that stops at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _quantize_noalloc(lib, ins, outs, scales, transpose, stream):
    arr_in = (C.c_void_p * len(ins))(*[t.data_ptr() for t in ins])
    arr_out = (C.c_void_p * len(outs))(*[t.data_ptr() for t in outs])
    rows, cols = ins[0].shape
    return lib.bbx_quantize_e4m3_batched_noalloc(0 if ins[0].dtype.itemsize == 4 else 1, arr_in, arr_out, len(ins),
                                                 rows, cols, int(transpose), C.c_void_p(scales.data_ptr()), stream)


@pytest.mark.parametrize("transpose", [False, True])
def test_noalloc_matches_allocating_entry_point(cuda, transpose):
    import torch
    from bbts_b200 import lib, last_error, ops
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(4)
    rows, cols = 384, 640
    for call in range(2):  # two calls in a row: the shared scratch must start clean each time
        count = 5 + call
        ins = [torch.from_numpy((rng.standard_normal((rows, cols)) * 10 ** rng.uniform(-2, 2)).astype(np.float32)).cuda()
               for _ in range(count)]
        shape = (cols, rows) if transpose else (rows, cols)
        outs = [torch.empty(shape, dtype=torch.float8_e4m3fn, device="cuda") for _ in range(count)]
        scales = torch.empty(count, device="cuda")
        rc = _quantize_noalloc(lib, ins, outs, scales, transpose, stream)
        assert rc == 0, last_error()
        for i in range(count):
            ref = torch.empty(shape, dtype=torch.float8_e4m3fn, device="cuda")
            ref_scale = torch.empty(1, device="cuda")
            ops.quantize_e4m3(ins[i], ref, ref_scale, transpose=transpose)
            torch.cuda.synchronize()
            # same kernels, same arithmetic: identical bytes and scales
            assert torch.equal(outs[i].view(torch.uint8), ref.view(torch.uint8))
            assert torch.equal(scales[i:i + 1], ref_scale)


def test_noalloc_rejects_too_many_blocks(cuda):
    import torch
    from bbts_b200 import lib, last_error
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    x = torch.zeros(16, 16, device="cuda")
    q = torch.empty(16, 16, dtype=torch.float8_e4m3fn, device="cuda")
    scales = torch.empty(1025, device="cuda")
    rc = _quantize_noalloc(lib, [x] * 1025, [q] * 1025, scales, False, stream)
    assert rc == -1
    assert "at most 1024" in last_error()
