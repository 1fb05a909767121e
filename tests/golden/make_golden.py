"""Generates the known-answer fixtures in tests/golden/ (run from the repo root:
`python tests/golden/make_golden.py`).

Every expected value here is computed with exact integer arithmetic (Python /
numpy int64), independent of the oracle and of the kernels:

* add_kat: the reference's own known-answer test for matrix_add
  (tests/test_builtin_ud.cc:32-71 of dcbdan/bbts): 100 x 200 blocks with
  a[r][c] = r + c, b[r][c] = 2(r + c), expected 3(r + c) within 1e-4.
* matmul_int: small-integer matrices whose products and partial sums are exact
  in FP32 (|entries| <= 4, K <= 256 keeps every partial sum below 2^24) and
  whose inputs are exact in BF16 and E4M3, for all four transpose combinations.
* reduce_cancel: integer blocks whose n-ary sum cancels to small values.
* contraction_int: 'ijk,kl->ijl' and a batched/permuted einsum on integer
  column-major tensors (the cutensor format), expected via int64 einsum.
* elementwise: relu / relu' / hadamard / weighted sum on values exact in FP32.
"""
import os

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))


def add_kat():
    r = np.arange(100)[:, None]
    c = np.arange(200)[None, :]
    a = (r + c).astype(np.float32)
    b = (2 * (r + c)).astype(np.float32)
    expect = (3 * (r + c)).astype(np.float32)
    np.savez_compressed(os.path.join(OUT, "add_kat.npz"), a=a, b=b, expect=expect)


def matmul_int():
    rng = np.random.default_rng(20240601)
    cases = {}
    for (m, n, k) in [(128, 256, 64), (200, 136, 96), (256, 512, 256), (130, 70, 40)]:
        a = rng.integers(-4, 5, size=(m, k)).astype(np.int64)
        b = rng.integers(-4, 5, size=(k, n)).astype(np.int64)
        cases["%dx%dx%d" % (m, n, k)] = (a, b, a @ b)
    payload = {}
    for key, (a, b, c) in cases.items():
        payload[key + "_a"] = a.astype(np.float32)
        payload[key + "_b"] = b.astype(np.float32)
        payload[key + "_c"] = c.astype(np.float32)
    np.savez_compressed(os.path.join(OUT, "matmul_int.npz"), **payload)


def reduce_cancel():
    rng = np.random.default_rng(7)
    base = rng.integers(-1000, 1000, size=(16, 64, 96)).astype(np.int64)
    base[-1] = -base[:-1].sum(axis=0) + rng.integers(-3, 4, size=(64, 96))
    expect = base.sum(axis=0)
    np.savez_compressed(os.path.join(OUT, "reduce_cancel.npz"), inputs=base.astype(np.float32),
             expect=expect.astype(np.float32))


def contraction_int():
    rng = np.random.default_rng(11)
    # 'ijk,kl->ijl' with modes i=0, j=1, k=2, l=3; column-major storage
    I, J, K, L = 33, 40, 24, 19
    lhs = rng.integers(-3, 4, size=(I, J, K)).astype(np.int64)
    rhs = rng.integers(-3, 4, size=(K, L)).astype(np.int64)
    out = np.einsum("ijk,kl->ijl", lhs, rhs)
    # batched + permuted: 'bik,kjb->jib' with b=0, i=1, k=2, j=3
    B, I2, K2, J2 = 3, 17, 20, 9
    lhs2 = rng.integers(-3, 4, size=(B, I2, K2)).astype(np.int64)
    rhs2 = rng.integers(-3, 4, size=(K2, J2, B)).astype(np.int64)
    out2 = np.einsum("bik,kjb->jib", lhs2, rhs2)
    f = lambda x: np.asfortranarray(x).ravel(order="F").astype(np.float32)
    np.savez_compressed(os.path.join(OUT, "contraction_int.npz"),
             c1_lhs=f(lhs), c1_rhs=f(rhs), c1_out=f(out), c1_dims=np.array([I, J, K, L]),
             c2_lhs=f(lhs2), c2_rhs=f(rhs2), c2_out=f(out2), c2_dims=np.array([B, I2, K2, J2]))


def elementwise():
    rng = np.random.default_rng(3)
    a = (rng.integers(-64, 65, size=(37, 53)) / 8.0).astype(np.float32)
    b = (rng.integers(-64, 65, size=(37, 53)) / 8.0).astype(np.float32)
    ai = (a * 8).astype(np.int64)
    bi = (b * 8).astype(np.int64)
    relu = np.where(ai > 0, ai, 0) / 8.0
    relu_dif = (ai > 0).astype(np.float64)
    had = (ai * bi) / 64.0
    wsum = (2 * ai - 3 * bi) / 8.0  # ca = 2, cb = -3
    np.savez_compressed(os.path.join(OUT, "elementwise.npz"), a=a, b=b, relu=relu.astype(np.float32),
             relu_dif=relu_dif.astype(np.float32), hadamard=had.astype(np.float32),
             wsum=wsum.astype(np.float32), colsum_a=(ai.sum(axis=0) / 8.0).astype(np.float32))


if __name__ == "__main__":
    add_kat()
    matmul_int()
    reduce_cancel()
    contraction_int()
    elementwise()
    print("fixtures written to", OUT)
