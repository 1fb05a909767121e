"""cutensor-plugin block ops (reduction, ew, ewb, ewb_castable, expand) on the
GPU against the oracle: bit-exact except exp / sigmoid (<= 2 ulp-scale 1e-6
relative), through the C ABI and through the registered uds."""
import numpy as np
import pytest

import oracle.cutensor as oc
from conftest import rel_err

pytestmark = pytest.mark.gpu
F = np.float32


@pytest.fixture(scope="module")
def T(cuda):
    import torch
    from bbts_b200 import ops
    return torch, ops


@pytest.fixture(scope="module")
def R(cuda):
    from bbts_b200 import runtime, workloads
    return runtime, workloads


def _dev(torch, x):
    return torch.from_numpy(np.ascontiguousarray(x, F)).cuda()


def _host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _shape(rng, rank, lo=1, hi=40):
    return [int(v) for v in rng.integers(lo, hi, rank)]


@pytest.mark.parametrize("seed", range(8))
def test_reduction_bit_exact(T, seed):
    torch, ops = T
    rng = np.random.default_rng(seed)
    rank = 1 + seed % 4
    dims = _shape(rng, rank, 1, 24 if rank < 4 else 10)
    keep = int(rng.integers(0, rank + 1))
    ordering = [int(v) for v in rng.permutation(rank)[:keep]]
    x = rng.standard_normal(int(np.prod(dims))).astype(F)
    nout = int(np.prod([dims[m] for m in ordering])) if ordering else 1
    for op in range(4):
        out = torch.empty(nout, dtype=torch.float32, device="cuda")
        ops.cu_reduction(_dev(torch, x), dims, op, 0.5, ordering, out)
        assert np.array_equal(_host(out), oc.reduction(x, dims, op, 0.5, ordering)), (dims, ordering, op)


def test_reduction_signed_zero_and_nan_rules(T):
    torch, ops = T
    x = np.array([-0.0, 0.0, np.nan, 1.0, 1.0, np.nan], F)
    for op in (1, 2):
        out = torch.empty(3, dtype=torch.float32, device="cuda")
        ops.cu_reduction(_dev(torch, x), [2, 3], op, 1.0, [1], out)
        got, want = _host(out), oc.reduction(x, [2, 3], op, 1.0, [1])
        # NaN payloads are not compared: the GPU's alpha multiply returns the
        # canonical NaN where x86 keeps the input's payload
        assert np.array_equal(np.isnan(got), np.isnan(want)), (op, got, want)
        ok = ~np.isnan(want)
        assert np.array_equal(got[ok].view(np.uint32), want[ok].view(np.uint32)), (op, got, want)


@pytest.mark.parametrize("uop", range(7))
def test_ew_all_unary_ops(T, uop):
    torch, ops = T
    rng = np.random.default_rng(100 + uop)
    dims = [13, 7, 5]
    ordering = [2, 0, 1]  # a 3-cycle: output mode r is input mode ordering[r]
    x = rng.standard_normal(int(np.prod(dims))).astype(F)
    if uop == 5:
        x = np.abs(x)
    out = torch.empty(x.size, dtype=torch.float32, device="cuda")
    ops.cu_ew(_dev(torch, x), dims, uop, -1.25, ordering, out, scalar=0.375)
    want, od = oc.ew(x, dims, uop, -1.25, ordering, scalar=0.375)
    got = _host(out)
    if uop in (0, 1):
        assert rel_err(got, want) <= 1e-6
    else:
        assert np.array_equal(got, want)


@pytest.mark.parametrize("seed", range(10))
def test_ewb_broadcast_bit_exact(T, seed):
    torch, ops = T
    rng = np.random.default_rng(200 + seed)
    rank = 1 + seed % 4
    od = _shape(rng, rank, 1, 20 if rank < 4 else 9)
    ol = [int(v) for v in rng.permutation(rank)[:int(rng.integers(1, rank + 1))]]
    orr = [int(v) for v in rng.permutation(rank)[:int(rng.integers(1, rank + 1))]]
    if max(ol + orr) + 1 != rank:
        ol = list(range(rank))
    dl, dr = [od[m] for m in ol], [od[m] for m in orr]
    l = rng.standard_normal(int(np.prod(dl))).astype(F)
    r = rng.standard_normal(int(np.prod(dr))).astype(F) + F(3.0)
    for op in range(6):
        out = torch.empty(int(np.prod(od)), dtype=torch.float32, device="cuda")
        god = ops.cu_ewb(_dev(torch, l), dl, ol, _dev(torch, r), dr, orr, op, 1.5, -0.75, out)
        want, wod = oc.ewb(l, dl, ol, r, dr, orr, op, 1.5, -0.75)
        assert god == wod
        assert np.array_equal(_host(out), want), (ol, orr, op)


def test_ewb_rejects_bad_modes(T):
    torch, ops = T
    from bbts_b200._lib import BbxError
    a = torch.zeros(12, device="cuda")
    out = torch.zeros(64, device="cuda")
    with pytest.raises(BbxError, match="extents disagree"):
        ops.cu_ewb(a, [3, 4], [0, 1], a, [4, 3], [0, 1], 0, 1.0, 1.0, out)
    with pytest.raises(BbxError, match="ordering"):
        ops.cu_ewb(a, [3, 4], [0, 0], a, [3, 4], [0, 1], 0, 1.0, 1.0, out)


def test_expand_box_and_signed_zero(T):
    torch, ops = T
    rng = np.random.default_rng(7)
    x = rng.standard_normal(6 * 5 * 4).astype(F)
    x[0] = -0.0
    p = [6, 9, 4, 0, 3, 5, 5, 5, 0, 0, 4, 7, 2, 2, 1]
    out = torch.full((9 * 5 * 7,), 7.0, device="cuda")
    ops.cu_expand(_dev(torch, x), p, out)
    got = _host(out)
    assert np.array_equal(got.view(np.uint32), oc.expand(x, p).view(np.uint32))


def test_cutensor_uds_through_runtime(R):
    """The uds registered under the plugin's names run through the reservation
    station with the plugin's parameter layouts."""
    runtime, _ = R
    rt = runtime.Runtime()
    cf = rt.fmt("cutensor")
    rng = np.random.default_rng(3)
    dims = [6, 5, 4]
    x = rng.standard_normal(120).astype(F)
    y = rng.standard_normal(120).astype(F)
    rt.put(0, runtime.cutensor_meta(cf, dims), x)
    rt.put(1, runtime.cutensor_meta(cf, dims), y)
    rt.put(2, runtime.cutensor_meta(cf, [5]), rng.standard_normal(5).astype(F))
    one = ("cutensor",)
    rt.apply(rt.impl_named("reduction", "b200_reduction", one, one), [0], [10], params=[0, 2.0, 2, 0])
    rt.apply(rt.impl_named("ew", "b200_ew", one, one), [0], [11], params=[6, 0.5, 3.0, 1, 2, 0])
    rt.apply(rt.impl_named("ewb", "b200_ewb"), [0, 2], [12], params=[4, 1.0, 2.0, 3, 0, 1, 2, 1, 1])
    rt.apply(rt.impl_named("ewb_castable", "b200_ewb_castable"), [0, 1], [13], params=[1])
    rt.apply(rt.impl_named("expand", "b200_expand", one, one), [2], [14], params=[5, 8, 3, 1, 4])
    rt.run()
    get = lambda t: rt.get_bytes(t).view(np.float32)
    assert np.array_equal(get(10), oc.reduction(x, dims, 0, 2.0, [2, 0]))
    assert np.array_equal(get(11), oc.ew(x, dims, 6, 3.0, [1, 2, 0], scalar=0.5)[0])
    b = rt.get_bytes(2).view(np.float32)
    assert np.array_equal(get(12), oc.ewb(x, dims, [0, 1, 2], b, [5], [1], 4, 1.0, 2.0)[0])
    assert np.array_equal(get(13), oc.ewb_castable(x, y, dims, 1))
    assert np.array_equal(get(14), oc.expand(b, [5, 8, 3, 1, 4]))
    # the output metas carry the plugin's shapes
    import struct
    assert struct.unpack_from("<I4xqq", rt.meta(10), 4) == (2, 4, 6)
    assert struct.unpack_from("<I4xqqq", rt.meta(11), 4) == (3, 5, 4, 6)
    assert struct.unpack_from("<I4xqqq", rt.meta(12), 4) == (3, 6, 5, 4)
