"""Pins the CPU oracle against the known-answer fixtures (no GPU needed)."""
import numpy as np
import pytest

import oracle
from conftest import golden


def test_add_known_answer_from_reference():
    # tests/test_builtin_ud.cc:32-71: a=row+col, b=2(row+col) -> 3(row+col) within 1e-4
    g = golden("add_kat.npz")
    out = oracle.add(g["a"], g["b"])
    assert out.shape == (100, 200)
    assert np.max(np.abs(out - g["expect"])) <= 1e-4
    assert np.array_equal(out, g["expect"])


@pytest.mark.parametrize("key", ["128x256x64", "200x136x96", "256x512x256", "130x70x40"])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_matmul_integer_exact(key, ta, tb):
    g = golden("matmul_int.npz")
    a, b, c = g[key + "_a"], g[key + "_b"], g[key + "_c"]
    A = np.ascontiguousarray(a.T) if ta else a
    B = np.ascontiguousarray(b.T) if tb else b
    assert np.array_equal(oracle.matmul_f64(A, B, bool(ta), bool(tb)), c.astype(np.float64))
    assert np.array_equal(oracle.sgemm(A, B, bool(ta), bool(tb), threads=2), c)


def test_reduce_fold_cancellation_exact():
    g = golden("reduce_cancel.npz")
    ins = list(g["inputs"])
    assert np.array_equal(oracle.reduce_fold(ins), g["expect"])
    assert np.array_equal(oracle.reduce_f64(ins), g["expect"].astype(np.float64))


def test_reduce_fold_is_left_fold():
    rng = np.random.default_rng(0)
    ins = [rng.standard_normal(1000).astype(np.float32) for _ in range(7)]
    ref = ins[0].copy()
    for x in ins[1:]:
        ref = (ref + x).astype(np.float32)  # matrix_add applied pairwise, left to right
    assert np.array_equal(oracle.reduce_fold(ins), ref)


def test_elementwise_known_answers():
    g = golden("elementwise.npz")
    a, b = g["a"], g["b"]
    assert np.array_equal(oracle.unary(0, a), g["relu"])
    assert np.array_equal(oracle.unary(1, a), g["relu_dif"])
    assert np.array_equal(oracle.binary(2, a, b), g["hadamard"])
    assert np.array_equal(oracle.binary(1, a, b, 2.0, -3.0), g["wsum"])
    assert np.array_equal(oracle.colsum(a), g["colsum_a"])


def test_sigmoid_matches_reference_formula():
    # dense_matrix_sigmoid.cc:67 computes 1/(1+exp(v)) (sigmoid of -v); the oracle keeps it.
    x = np.linspace(-8, 8, 101).astype(np.float32)
    ref = 1.0 / (1.0 + np.exp(x.astype(np.float64)))
    assert np.max(np.abs(oracle.unary(2, x) - ref)) < 1e-6
    ref_ok = 1.0 / (1.0 + np.exp(-x.astype(np.float64)))
    assert np.max(np.abs(oracle.unary(3, x) - ref_ok)) < 1e-6


@pytest.mark.parametrize("case", ["c1", "c2"])
def test_contraction_integer_exact(case):
    g = golden("contraction_int.npz")
    if case == "c1":
        I, J, K, L = g["c1_dims"]
        got = oracle.contraction_f64(g["c1_lhs"], [I, J, K], [0, 1, 2], g["c1_rhs"], [K, L], [2, 3], [0, 1, 3])
    else:
        B, I, K, J = g["c2_dims"]
        got = oracle.contraction_f64(g["c2_lhs"], [B, I, K], [0, 1, 2], g["c2_rhs"], [K, J, B], [2, 3, 0], [3, 1, 0])
    assert np.array_equal(got, g[case + "_out"].astype(np.float64))


def test_softmax_ce_f64_properties():
    rng = np.random.default_rng(5)
    z = rng.standard_normal((16, 10)).astype(np.float32)
    y = rng.integers(0, 10, 16)
    loss, grad = oracle.softmax_ce_f64(z, y)
    zz = z.astype(np.float64)
    p = np.exp(zz - zz.max(1, keepdims=True))
    p /= p.sum(1, keepdims=True)
    assert np.allclose(loss, -np.log(p[np.arange(16), y]), rtol=1e-12)
    assert np.allclose(grad.sum(1), 0.0, atol=1e-12)


def test_philox_uniform_statistics():
    u = oracle.uniform(1234, 1 << 16, -1.0, 1.0)
    assert u.min() >= -1.0 and u.max() < 1.0
    assert abs(u.mean()) < 0.02 and abs(u.var() - 1.0 / 3.0) < 0.02
    w = oracle.philox(1234, 8)
    assert len(set(w.tolist())) == 32  # distinct words
    assert not np.array_equal(oracle.philox(1, 4), oracle.philox(2, 4))
