"""The vectorised cutensor-plugin oracle against a per-index loop restatement
of the plugin's own checkers (libraries/cutensor/reduction.h:36-100,
ew.h:44-120, ewb.h:122-204, expand.h:41-140), which walk every index and
compute column-major offsets directly."""
import itertools

import numpy as np
import pytest

import oracle.cutensor as oc

F = np.float32


def _off(dims, idx):
    s, o = 1, 0
    for d, i in zip(dims, idx):
        o += s * i
        s *= d
    return o


def _loop_reduction(x, dims, op, alpha, ordering):
    fold = {0: lambda a, b: F(a + b), 1: lambda a, b: a if a > b else b,
            2: lambda a, b: a if a < b else b, 3: lambda a, b: F(a * b)}[op]
    dout = [dims[m] for m in ordering]
    ref, seen = np.zeros(int(np.prod(dout)) if dout else 1, F), set()
    # the checker walks the input column-major (mode 0 fastest), which visits
    # each output's elements with the first dropped mode fastest
    for idx in itertools.product(*[range(d) for d in reversed(dims)]):
        idx = idx[::-1]
        o = _off(dout, [idx[m] for m in ordering])
        v = x[_off(dims, idx)]
        ref[o] = fold(ref[o], v) if o in seen else v
        seen.add(o)
    return (F(alpha) * ref).astype(F)


def _loop_ewb(l, dl, ol, r, dr, orr, op, a, b):
    rank = 1 + max(ol + orr)
    od = [1] * rank
    for q, m in enumerate(ol):
        od[m] = dl[q]
    for q, m in enumerate(orr):
        od[m] = dr[q]
    out = np.zeros(int(np.prod(od)), F)
    for idx in itertools.product(*[range(d) for d in reversed(od)]):
        idx = idx[::-1]
        vl = F(F(a) * l[_off(dl, [idx[m] for m in ol])])
        vr = F(F(b) * r[_off(dr, [idx[m] for m in orr])])
        with np.errstate(all="ignore"):
            v = [vl + vr, vl if vl > vr else vr, vr if vl > vr else vl, vl * vr, vl - vr, vl / vr][op]
        out[_off(od, idx)] = v
    return out, od


@pytest.mark.parametrize("seed", range(6))
def test_reduction_matches_loop(seed):
    rng = np.random.default_rng(seed)
    rank = 1 + seed % 4
    dims = [int(v) for v in rng.integers(1, 5, rank)]
    keep = int(rng.integers(0, rank + 1))
    ordering = [int(v) for v in rng.permutation(rank)[:keep]]
    x = rng.standard_normal(int(np.prod(dims))).astype(F)
    for op in range(4):
        got = oc.reduction(x, dims, op, 0.75, ordering)
        assert np.array_equal(got, _loop_reduction(x, dims, op, 0.75, ordering)), (dims, ordering, op)


def test_reduction_min_keeps_plugin_tie_rule():
    # scalarMin(l, r) = l < r ? l : r: on (-0, +0) the later +0 wins
    x = np.array([-0.0, 0.0], F)
    assert np.signbit(oc.reduction(x, [2], 2, 1.0, []))[0] == False  # noqa: E712
    assert np.signbit(oc.reduction(x, [2], 1, 1.0, []))[0] == False  # noqa: E712


@pytest.mark.parametrize("seed", range(6))
def test_ew_permutes_like_out_meta(seed):
    rng = np.random.default_rng(10 + seed)
    rank = 1 + seed % 4
    dims = [int(v) for v in rng.integers(1, 5, rank)]
    ordering = [int(v) for v in rng.permutation(rank)]
    x = rng.standard_normal(int(np.prod(dims))).astype(F)
    got, od = oc.ew(x, dims, 2, 0.5, ordering)
    assert od == [dims[m] for m in ordering]
    out = np.zeros_like(got)
    for idx in itertools.product(*[range(d) for d in reversed(od)]):
        idx = idx[::-1]
        iin = [0] * rank
        for r, m in enumerate(ordering):
            iin[m] = idx[r]
        v = x[_off(dims, iin)]
        out[_off(od, idx)] = F(0.5) * F(v * v)
    assert np.array_equal(got, out)


@pytest.mark.parametrize("seed", range(8))
def test_ewb_matches_loop(seed):
    rng = np.random.default_rng(20 + seed)
    rank = 1 + seed % 4
    od = [int(v) for v in rng.integers(1, 4, rank)]
    ol = sorted(int(v) for v in rng.permutation(rank)[:int(rng.integers(1, rank + 1))])
    orr = [int(v) for v in rng.permutation(rank)[:int(rng.integers(1, rank + 1))]]
    if max(ol + orr) + 1 != rank:
        ol = list(range(rank))
    dl, dr = [od[m] for m in ol], [od[m] for m in orr]
    l = rng.standard_normal(int(np.prod(dl))).astype(F)
    r = rng.standard_normal(int(np.prod(dr))).astype(F)
    for op in range(6):
        got, god = oc.ewb(l, dl, ol, r, dr, orr, op, 1.5, -0.5)
        ref, rod = _loop_ewb(l, dl, ol, r, dr, orr, op, 1.5, -0.5)
        assert god == rod
        assert np.array_equal(got, ref), (ol, orr, op)


def test_expand_box():
    x = np.arange(12, dtype=F)  # 3 x 4 column-major
    p = [3, 5, 2, 1, 0, 4, 6, 3, 0, 2]
    got = oc.expand(x, p).reshape(5, 6, order="F")
    want = np.zeros((5, 6), F)
    a = x.reshape(3, 4, order="F")
    want[0:2, 2:5] = a[1:3, 0:3]
    assert np.array_equal(got, want)
