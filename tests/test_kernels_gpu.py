"""Parity of the CUDA block kernels (through the C ABI) against the CPU oracle."""
import zlib

import numpy as np
import pytest

import oracle
from conftest import golden, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T(cuda):
    import torch
    from bbts_b200 import ops
    return torch, ops


def dev(torch, x, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    return t.to(dtype) if dtype is not None else t


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.float().cpu().numpy() if t.dtype != torch.float32 else t.cpu().numpy()


def bf16_round(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(torch.bfloat16).float().numpy()


# ----------------------------------------------------------------- add / reduce
def test_add_known_answer(T):
    torch, ops = T
    g = golden("add_kat.npz")
    a, b = dev(torch, g["a"]), dev(torch, g["b"])
    ops.add(a, b, a)  # in place into input 0, as the reference test does
    out = host(a)
    assert np.max(np.abs(out - g["expect"])) <= 1e-4
    assert np.array_equal(out, g["expect"])


@pytest.mark.parametrize("n", [0, 1, 3, 1000, 1024 * 1024 + 5])
def test_add_bit_exact(T, n):
    torch, ops = T
    rng = np.random.default_rng(n)
    a = rng.standard_normal(n).astype(np.float32)
    b = rng.standard_normal(n).astype(np.float32)
    c = torch.empty(n, device="cuda")
    ops.add(dev(torch, a), dev(torch, b), c)
    assert np.array_equal(host(c), oracle.add(a, b))


@pytest.mark.parametrize("n_in", [1, 2, 4, 16, 33, 70])
def test_reduce_fold_bit_exact(T, n_in):
    torch, ops = T
    rng = np.random.default_rng(n_in)
    ins = [rng.standard_normal(4099).astype(np.float32) for _ in range(n_in)]
    out = torch.empty(4099, device="cuda")
    ops.reduce([dev(torch, x) for x in ins], out, kahan=False)
    assert np.array_equal(host(out), oracle.reduce_fold(ins))


@pytest.mark.parametrize("n_in", [2, 4, 16])
def test_reduce_kahan_vs_f64(T, n_in):
    torch, ops = T
    rng = np.random.default_rng(100 + n_in)
    shape = (1024, 1024)
    ins = [(rng.standard_normal(shape) * 10 ** rng.uniform(-3, 3)).astype(np.float32) for _ in range(n_in)]
    out = torch.empty(shape, device="cuda")
    ops.reduce([dev(torch, x) for x in ins], out, kahan=True)
    ref = oracle.reduce_f64(ins)
    assert rel_err(host(out), ref) <= 1e-6


def test_reduce_cancellation_exact(T):
    torch, ops = T
    g = golden("reduce_cancel.npz")
    out = torch.empty(g["expect"].shape, device="cuda")
    ops.reduce([dev(torch, x) for x in g["inputs"]], out, kahan=True)
    assert np.array_equal(host(out), g["expect"])


def test_reduce_in_place_alias(T):
    torch, ops = T
    rng = np.random.default_rng(9)
    ins = [rng.standard_normal(10000).astype(np.float32) for _ in range(4)]
    d = [dev(torch, x) for x in ins]
    ops.reduce(d, d[0], kahan=False)
    assert np.array_equal(host(d[0]), oracle.reduce_fold(ins))


# ----------------------------------------------------------------- grouped streaming ops
def _kahan_fold(ins):
    """Compensated left fold in f32 arithmetic, in the kernels' order."""
    a = ins[0].astype(np.float32).copy()
    comp = np.zeros_like(a)
    for b in ins[1:]:
        y = (b - comp).astype(np.float32)
        t = (a + y).astype(np.float32)
        comp = ((t - a) - y).astype(np.float32)
        a = t
    return a


def _stream_specs(seed, n_ops, sizes):
    """Seeded batch of independent ops: sums of 1..16 inputs (Kahan on/off),
    bit-exact unary / binary ops and casts, f32 or bf16 in and out."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_ops):
        kind = [0, 0, 0, 1, 2, 3][i % 6]
        n = int(sizes[i % len(sizes)])
        n_in = int(rng.integers(1, 17)) if kind == 0 else (2 if kind == 2 else 1)
        idt, odt = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        if kind == 3:
            odt = 1 - idt
        op = int(rng.choice([0, 1, 5, 7, 8])) if kind == 1 else int(rng.integers(0, 7)) if kind == 2 else 0
        xs = [rng.standard_normal(n).astype(np.float32) for _ in range(n_in)]
        specs.append(dict(kind=kind, op=op, idt=idt, odt=odt, kahan=bool(rng.integers(0, 2)), xs=xs, n=n))
    return specs


def _stream_materialise(torch, ops, specs, offset):
    """Device tensors for the specs, each starting `offset` elements into its
    allocation (offset 1 breaks 16-byte alignment: the register kernel)."""
    dt = {0: torch.float32, 1: torch.bfloat16}
    keep, outs, sops = [], [], []
    for sp in specs:
        ins = []
        for x in sp["xs"]:
            buf = torch.empty(sp["n"] + 16, dtype=dt[sp["idt"]], device="cuda")
            v = buf[offset:offset + sp["n"]]
            v.copy_(torch.from_numpy(x).to(dt[sp["idt"]]))
            keep.append(buf)
            ins.append(v)
        obuf = torch.full((sp["n"] + 16,), 7.0, dtype=dt[sp["odt"]], device="cuda")
        out = obuf[offset:offset + sp["n"]]
        keep.append(obuf)
        outs.append((out, obuf))
        sops.append(ops.stream_op(sp["kind"], ins, out, op=sp["op"], kahan=sp["kahan"], p0=0.3, p1=-1.7))
    return keep, outs, sops


def _stream_expect(torch, sp):
    """CPU result of one spec: inputs rounded to the input dtype, math in f32,
    result rounded to the output dtype."""
    rnd = (lambda a: a) if sp["idt"] == 0 else bf16_round
    xs = [rnd(x) for x in sp["xs"]]
    if sp["kind"] == 0:
        r = _kahan_fold(xs) if sp["kahan"] else oracle.reduce_fold(xs)
    elif sp["kind"] == 1:
        r = oracle.unary(sp["op"], xs[0], 0.3)
    elif sp["kind"] == 2:
        r = oracle.binary(sp["op"], xs[0], xs[1], 0.3, -1.7)
    else:
        r = xs[0]
    return r if sp["odt"] == 0 else bf16_round(r)


@pytest.mark.parametrize("sizes", [[1, 7, 8, 15, 64, 1000, 4099, 100003], [1024 * 1024, 1536 * 704, 129 * 131]])
def test_stream_group_bulk_and_register_paths(T, sizes):
    """The bulk-staged kernel (aligned pointers) and the register kernel
    (pointers offset by one element) give bit-identical results, equal to the
    CPU fold in the same order; bytes past each output stay untouched."""
    torch, ops = T
    specs = _stream_specs(len(sizes), 24, sizes)
    got = {}
    for offset in (0, 1):
        keep, outs, sops = _stream_materialise(torch, ops, specs, offset)
        plan = ops.StreamPlan(sops)
        assert plan.bulk == (offset == 0)
        plan.launch()
        res = [host(o) for o, _ in outs]
        guard = [host(b) for _, b in outs]
        # the one-shot (inline) launches give the same bits
        for o, _ in outs:
            o.fill_(0)
        ops.stream_group(sops)
        assert all(np.array_equal(r, host(o)) for r, (o, _) in zip(res, outs))
        for sp, g in zip(specs, guard):
            assert np.all(g[:offset] == 7.0) and np.all(g[offset + sp["n"]:] == 7.0)
        got[offset] = res
        plan.close()
        del keep
    for sp, a, b in zip(specs, got[0], got[1]):
        assert np.array_equal(a, b)
        assert np.array_equal(a, _stream_expect(torch, sp))


def test_stream_plan_many_items_replay(T):
    """Hundreds of items per CTA (every stage of the ring reused many times),
    replayed: results stay bit-exact against the CPU fold."""
    torch, ops = T
    specs = _stream_specs(77, 30, [1024 * 1024, 512 * 768 + 8, 333 * 1000])
    keep, outs, sops = _stream_materialise(torch, ops, specs, 0)
    plan = ops.StreamPlan(sops)
    assert plan.bulk
    for _ in range(3):
        plan.launch()
    for sp, (o, _) in zip(specs, outs):
        assert np.array_equal(host(o), _stream_expect(torch, sp))
    plan.close()


# ----------------------------------------------------------------- elementwise
@pytest.mark.parametrize("op", [0, 1, 5, 7, 8])
def test_unary_bit_exact(T, op):
    torch, ops = T
    x = np.random.default_rng(op).standard_normal(50001).astype(np.float32)
    out = torch.empty_like(dev(torch, x))
    ops.unary(op, dev(torch, x), out, 0.75)
    assert np.array_equal(host(out), oracle.unary(op, x, 0.75))


@pytest.mark.parametrize("op", [2, 3, 4, 6])
def test_unary_transcendental(T, op):
    torch, ops = T
    x = np.random.default_rng(op).standard_normal(50001).astype(np.float32)
    if op == 6:
        x = np.abs(x)
    out = torch.empty_like(dev(torch, x))
    ops.unary(op, dev(torch, x), out)
    got, ref = host(out), oracle.unary(op, x)
    # expf differs between libm and CUDA by at most a couple of ulp
    assert np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-30)) < 4e-7


@pytest.mark.parametrize("op", [0, 1, 2, 3, 4, 5, 6])
def test_binary_bit_exact(T, op):
    torch, ops = T
    rng = np.random.default_rng(op)
    a = rng.standard_normal(30003).astype(np.float32)
    b = rng.standard_normal(30003).astype(np.float32)
    out = torch.empty(30003, device="cuda")
    ops.binary(op, dev(torch, a), dev(torch, b), out, 0.3, -1.7)
    assert np.array_equal(host(out), oracle.binary(op, a, b, 0.3, -1.7))


def test_elementwise_golden(T):
    torch, ops = T
    g = golden("elementwise.npz")
    a, b = dev(torch, g["a"]), dev(torch, g["b"])
    out = torch.empty_like(a)
    assert np.array_equal(host(ops.unary(0, a, out)), g["relu"])
    assert np.array_equal(host(ops.unary(1, a, out)), g["relu_dif"])
    assert np.array_equal(host(ops.binary(2, a, b, out)), g["hadamard"])
    assert np.array_equal(host(ops.binary(1, a, b, out, 2.0, -3.0)), g["wsum"])
    cs = torch.empty(a.shape[1], device="cuda")
    assert np.array_equal(host(ops.colsum(a, cs)), g["colsum_a"])


def test_bias_add_and_colsum(T):
    torch, ops = T
    rng = np.random.default_rng(1)
    x = rng.standard_normal((333, 257)).astype(np.float32)
    bias = rng.standard_normal(257).astype(np.float32)
    out = torch.empty(333, 257, device="cuda")
    ops.bias_add(dev(torch, x), dev(torch, bias), out, relu=True)
    assert np.array_equal(host(out), oracle.bias_add(x, bias, relu=True))
    cs = dev(torch, bias.copy())
    ops.colsum(dev(torch, x), cs, accumulate=True)
    assert np.array_equal(host(cs), oracle.colsum(x, init=bias))


def test_softmax_ce(T):
    torch, ops = T
    rng = np.random.default_rng(2)
    z = (rng.standard_normal((300, 1024)) * 3).astype(np.float32)
    y = rng.integers(0, 1024, 300).astype(np.int32)
    loss = torch.empty(300, device="cuda")
    grad = torch.empty(300, 1024, device="cuda")
    ops.softmax_ce(dev(torch, z), dev(torch, y), loss, grad, grad_scale=1.0 / 300)
    l64, g64 = oracle.softmax_ce_f64(z, y, grad_scale=1.0 / 300)
    assert rel_err(host(loss), l64) < 1e-5
    assert rel_err(host(grad), g64) < 1e-5


def test_philox_fill_matches_oracle(T):
    torch, ops = T
    out = torch.empty(100003, device="cuda")
    ops.fill_philox(out, seed=0x1234_5678_9abc, dist=0, a=-1.0, b=1.0)
    assert np.array_equal(host(out), oracle.uniform(0x1234_5678_9abc, 100003, -1.0, 1.0))
    nrm = torch.empty(1 << 20, device="cuda")
    ops.fill_philox(nrm, seed=7, dist=1, a=0.0, b=1.0)
    v = host(nrm)
    assert abs(v.mean()) < 0.01 and abs(v.std() - 1.0) < 0.01


def test_cast_and_permute(T):
    torch, ops = T
    x = np.random.default_rng(4).standard_normal((7, 9, 11, 5)).astype(np.float32)
    out = torch.empty((11, 7, 5, 9), device="cuda")
    ops.permute(dev(torch, x), [2, 0, 3, 1], out)
    assert np.array_equal(host(out), np.transpose(x, (2, 0, 3, 1)))
    bf = torch.empty(x.size, dtype=torch.bfloat16, device="cuda")
    ops.cast(dev(torch, x.ravel()), bf)
    assert np.array_equal(host(bf), bf16_round(x.ravel()))


# ----------------------------------------------------------------- matmul FP32
@pytest.mark.parametrize("m,n,k", [(1024, 1024, 1024), (130, 70, 40), (1, 1, 1), (257, 129, 300)])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_matmul_f32_vs_f64(T, m, n, k, ta, tb):
    torch, ops = T
    rng = np.random.default_rng(m + n + k)
    a = rng.standard_normal((k, m) if ta else (m, k)).astype(np.float32)
    b = rng.standard_normal((n, k) if tb else (k, n)).astype(np.float32)
    c = torch.empty(m, n, device="cuda")
    ops.matmul_f32(dev(torch, a), dev(torch, b), c, bool(ta), bool(tb))
    ref = oracle.matmul_f64(a, b, bool(ta), bool(tb))
    assert rel_err(host(c), ref) <= 1e-5


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_matmul_vs_cpu_port_of_reference_sgemm(T, ta, tb):
    """The GPU block matmuls against the oracle's CPU port of the reference's
    block matmul (dense_matrix_mult.cc:78-82, cblas_sgemm RowMajor with the
    transpose flags) on the same seeded inputs: the FP32 SIMT path within
    1e-5 of the port's FP32 result, and the bf16 tensor-core path, on the
    bf16-rounded inputs, within 1e-5 of the port run on those inputs."""
    torch, ops = T
    rng = np.random.default_rng(100 + 2 * ta + tb)
    m, n, k = 512, 384, 640
    a = rng.uniform(-1, 1, (k, m) if ta else (m, k)).astype(np.float32)
    b = rng.uniform(-1, 1, (n, k) if tb else (k, n)).astype(np.float32)
    port = oracle.sgemm(a, b, bool(ta), bool(tb), threads=4)
    c = torch.empty(m, n, device="cuda")
    ops.matmul_f32(dev(torch, a), dev(torch, b), c, bool(ta), bool(tb))
    assert rel_err(host(c), port) <= 1e-5
    ab, bb = bf16_round(a), bf16_round(b)
    port16 = oracle.sgemm(ab, bb, bool(ta), bool(tb), threads=4)
    c16 = torch.empty(m, n, device="cuda")
    ops.matmul_tc([ops.tc_problem(dev(torch, ab, torch.bfloat16), dev(torch, bb, torch.bfloat16), c16,
                                  trans_a=bool(ta), trans_b=bool(tb))])
    assert rel_err(host(c16), port16) <= 1e-5


def test_matmul_f32_integer_exact(T):
    torch, ops = T
    g = golden("matmul_int.npz")
    for key in ["128x256x64", "200x136x96", "256x512x256", "130x70x40"]:
        a, b, cref = g[key + "_a"], g[key + "_b"], g[key + "_c"]
        c = torch.empty(cref.shape, device="cuda")
        ops.matmul_f32(dev(torch, a), dev(torch, b), c)
        assert np.array_equal(host(c), cref)


@pytest.mark.parametrize("n", [90, 96])  # 90: element-wise kernel; 96: the 16-byte-load kernel, float4 epilogue
def test_matmul_f32_epilogue_and_batch(T, n):
    torch, ops = T
    rng = np.random.default_rng(8)
    a = rng.standard_normal((3, 100, 64)).astype(np.float32)
    b = rng.standard_normal((3, 64, n)).astype(np.float32)
    c0 = rng.standard_normal((3, 100, n)).astype(np.float32)
    bias = rng.standard_normal(n).astype(np.float32)
    c = dev(torch, c0)
    ops.matmul_f32(dev(torch, a), dev(torch, b), c, alpha=0.5, beta=2.0, bias=dev(torch, bias), relu=True)
    ref = np.stack([oracle.matmul_f64(a[i], b[i]) for i in range(3)]) * 0.5 + 2.0 * c0 + bias
    ref = np.maximum(ref, 0)
    assert rel_err(host(c), ref) <= 1e-5


# ----------------------------------------------------------------- matmul tensor cores
@pytest.mark.parametrize("key", ["128x256x64", "200x136x96", "256x512x256", "130x70x40"])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("tile_n", [128, 256])
def test_matmul_tc_bf16_integer_exact(T, key, ta, tb, tile_n):
    torch, ops = T
    g = golden("matmul_int.npz")
    a, b, cref = g[key + "_a"], g[key + "_b"], g[key + "_c"]
    A = np.ascontiguousarray(a.T) if ta else a
    B = np.ascontiguousarray(b.T) if tb else b
    # pad pitches to 16 bytes
    def padded(x):
        rows, cols = x.shape
        p = (cols + 7) // 8 * 8
        buf = torch.zeros(rows, p, dtype=torch.bfloat16, device="cuda")
        buf[:, :cols] = dev(torch, x, torch.bfloat16)
        return buf[:, :cols]
    Ad, Bd = padded(A), padded(B)
    c = torch.full(cref.shape, -7.0, device="cuda")
    ops.matmul_tc([ops.tc_problem(Ad, Bd, c, bool(ta), bool(tb))], tile_n=tile_n)
    assert np.array_equal(host(c), cref)


@pytest.mark.parametrize("m,n,k", [(1024, 1024, 1024), (384, 640, 4096), (192, 320, 136)])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_matmul_tc_bf16_random_vs_f64(T, m, n, k, ta, tb):
    torch, ops = T
    rng = np.random.default_rng(m * 7 + n + k)
    a = rng.standard_normal((k, m) if ta else (m, k)).astype(np.float32)
    b = rng.standard_normal((n, k) if tb else (k, n)).astype(np.float32)
    ab, bb = bf16_round(a), bf16_round(b)
    c = torch.empty(m, n, device="cuda")
    ops.matmul_tc([ops.tc_problem(dev(torch, a, torch.bfloat16), dev(torch, b, torch.bfloat16), c,
                                  bool(ta), bool(tb))])
    # vs FP64 on the bf16-rounded inputs: only accumulation-order error remains
    assert rel_err(host(c), oracle.matmul_f64(ab, bb, bool(ta), bool(tb))) <= 1e-5
    # vs FP64 on the original FP32 inputs: the bf16 input rounding, within the 1e-2 budget
    assert rel_err(host(c), oracle.matmul_f64(a, b, bool(ta), bool(tb))) <= 1e-2


def test_matmul_tc_grouped_epilogues(T):
    torch, ops = T
    rng = np.random.default_rng(77)
    probs, refs, outs, keep = [], [], [], []
    shapes = [(256, 256, 128), (128, 384, 64), (300, 200, 72), (512, 128, 256), (64, 64, 64), (200, 520, 320)]
    for i, (m, n, k) in enumerate(shapes):
        a = bf16_round(rng.standard_normal((m, k)))
        b = bf16_round(rng.standard_normal((k, n)))
        c0 = rng.standard_normal((m, n)).astype(np.float32)
        bias = rng.standard_normal(n).astype(np.float32)
        A, B, Cd, Bi = dev(torch, a, torch.bfloat16), dev(torch, b, torch.bfloat16), dev(torch, c0), dev(torch, bias)
        keep += [A, B, Bi]
        relu = i % 2 == 0
        probs.append(ops.tc_problem(A, B, Cd, alpha=0.5, beta=1.5, bias=Bi, relu=relu))
        ref = 0.5 * oracle.matmul_f64(a, b) + 1.5 * c0 + bias
        refs.append(np.maximum(ref, 0) if relu else ref)
        outs.append(Cd)
    ops.matmul_tc(probs)  # 6 problems: carried in the kernel parameters
    for o, r in zip(outs, refs):
        assert rel_err(host(o), r) <= 1e-5


@pytest.mark.parametrize("tile_n", [128, 256, 512])
def test_matmul_tc_params_and_table_paths(T, tile_n):
    """Plans of up to 72 problems carry them (tensor maps included) in the
    kernel parameters, larger ones in a device table whose maps each CTA
    acquires before use: 72 and 73 problems of integer-valued blocks, ragged
    shapes, row- and column-major C and bias / relu epilogues, give every
    problem's exact int64 product, over three replays."""
    torch, ops = T
    rng = np.random.default_rng(91 + tile_n)
    for count in (72, 73):
        probs, checks, keep = [], [], []
        for i in range(count):
            m, n = int(rng.integers(1, 9)) * 64, int(rng.integers(1, 9)) * 64
            k = int(rng.choice([64, 128, 192]))
            a = rng.integers(-3, 4, (m, k)).astype(np.float32)
            b = rng.integers(-3, 4, (k, n)).astype(np.float32)
            bias = rng.integers(-8, 9, n).astype(np.float32) if i % 3 == 0 else None
            relu = i % 4 == 1
            colmajor = i % 5 == 2
            A, B = dev(torch, a, torch.bfloat16), dev(torch, b, torch.bfloat16)
            bt = dev(torch, bias) if bias is not None else None
            c = torch.full((n, m) if colmajor else (m, n), float("nan"), device="cuda")
            probs.append(ops.tc_problem(A, B, c, bias=bt, relu=relu, c_colmajor=colmajor))
            r = a.astype(np.int64) @ b.astype(np.int64)
            if bias is not None:
                r = r + bias.astype(np.int64)[None, :]
            if relu:
                r = np.maximum(r, 0)
            keep += [A, B, bt, c]
            checks.append((c, r.T if colmajor else r))
        plan = ops.TcPlan(probs, tile_n=tile_n)
        for _ in range(3):
            for c, _r in checks:
                c.fill_(float("nan"))
            plan.launch()
            for i, (c, want) in enumerate(checks):
                assert np.array_equal(host(c), want.astype(np.float64)), (count, i)
        plan.close()


def test_matmul_tc_bf16_output(T):
    torch, ops = T
    rng = np.random.default_rng(5)
    a = bf16_round(rng.standard_normal((256, 512)))
    b = bf16_round(rng.standard_normal((512, 384)))
    c = torch.empty(256, 384, dtype=torch.bfloat16, device="cuda")
    ops.matmul_tc([ops.tc_problem(dev(torch, a, torch.bfloat16), dev(torch, b, torch.bfloat16), c)])
    assert rel_err(host(c), oracle.matmul_f64(a, b)) <= 1e-2


def test_matmul_tc_plan_replay(T):
    torch, ops = T
    rng = np.random.default_rng(6)
    a = bf16_round(rng.standard_normal((512, 256)))
    b = bf16_round(rng.standard_normal((256, 512)))
    A, B = dev(torch, a, torch.bfloat16), dev(torch, b, torch.bfloat16)
    cs = [torch.empty(512, 512, device="cuda") for _ in range(5)]
    plan = ops.TcPlan([ops.tc_problem(A, B, c) for c in cs])
    ref = oracle.matmul_f64(a, b)
    for _ in range(3):
        for c in cs:
            c.zero_()
        plan.launch()
        for c in cs:
            assert rel_err(host(c), ref) <= 1e-5
    plan.close()


@pytest.mark.parametrize("k, tile_n", [(1024, 0), (256, 128), (256, 256)])
def test_matmul_fp8_per_block_scale(T, k, tile_n):
    """e4m3 blocks with per-block absmax scales; K = 256 runs the kernel with
    eight epilogue warps (every K at most 512), K = 1024 the four-warp one."""
    torch, ops = T
    rng = np.random.default_rng(12 + k + tile_n)
    m, n = 512, 512
    a = rng.uniform(-1, 1, (m, k)).astype(np.float32)
    b = rng.uniform(-1, 1, (k, n)).astype(np.float32)
    qa = torch.empty(m, k, dtype=torch.float8_e4m3fn, device="cuda")
    qb = torch.empty(n, k, dtype=torch.float8_e4m3fn, device="cuda")  # K-major via transpose
    sa = torch.empty(1, device="cuda")
    sb = torch.empty(1, device="cuda")
    ops.quantize_e4m3(dev(torch, a), qa, sa)
    ops.quantize_e4m3(dev(torch, b), qb, sb, transpose=True)
    c = torch.empty(m, n, device="cuda")
    scale = float(host(sa)[0] * host(sb)[0])
    ops.matmul_tc([ops.tc_problem(qa, qb, c, trans_b=True, alpha=scale)], in_dtype=ops.E4M3, tile_n=tile_n)
    # e4m3 keeps 3 mantissa bits (relative rounding error up to 2^-4 per input), so
    # the normwise error of a K=1024 dot product sits at a few percent: FP8 is
    # outside the 1e-2 budget, and the error is reported per block instead.
    assert rel_err(host(c), oracle.matmul_f64(a, b)) <= 6e-2
    # the same inputs dequantised exactly on the host give the kernel's own arithmetic
    deq_a = qa.float().cpu().numpy() * host(sa)[0]
    deq_b = qb.float().cpu().numpy().T * host(sb)[0]
    assert rel_err(host(c), oracle.matmul_f64(np.ascontiguousarray(deq_a), np.ascontiguousarray(deq_b))) <= 1e-5


def _quantize_ref(x, transpose):
    """Host restatement of the e4m3 quantisation: s = 448 / absmax (f32
    division), q = e4m3(x * s) rounded to nearest even with saturation at
    +-448 (torch's cast does not saturate, so the clamp comes first; values
    in (448, 464) round to 448 either way)."""
    import torch
    x = torch.as_tensor(x, dtype=torch.float32)
    amax = float(x.abs().max())
    s = np.float32(448.0) / np.float32(amax) if amax > 0 else np.float32(1.0)
    q = (x * torch.tensor(s, dtype=torch.float32)).clamp(-448.0, 448.0).to(torch.float8_e4m3fn)
    if transpose:
        q = q.t().contiguous()
    return q.view(torch.uint8), np.float32(amax) / np.float32(448.0) if amax > 0 else np.float32(1.0)


@pytest.mark.parametrize("shape,dtype,transpose,offset", [
    ((384, 640), "bf16", False, 0), ((384, 640), "bf16", True, 0),      # vector and tiled-transpose paths
    ((384, 640), "f32", False, 0), ((384, 640), "f32", True, 0),
    ((80, 264), "bf16", True, 0), ((4096, 4096), "bf16", True, 0),      # partial tiles; a full block
    ((37, 53), "bf16", False, 0), ((37, 53), "f32", True, 0),           # element-wise fallback
    ((64, 64), "f32", True, 1)])                                        # unaligned input -> fallback
def test_quantize_e4m3_paths(T, shape, dtype, transpose, offset):
    """Every dispatch path of the FP8 quantiser gives the host restatement's
    bytes and scale exactly."""
    torch, ops = T
    rng = np.random.default_rng(zlib.crc32(repr((shape, dtype, transpose, offset)).encode()))
    x = (rng.standard_normal(shape) * 3).astype(np.float32)
    tdt = torch.bfloat16 if dtype == "bf16" else torch.float32
    flat = torch.empty(x.size + offset, dtype=tdt, device="cuda")
    xd = flat[offset:].view(shape)
    xd.copy_(torch.from_numpy(x))
    out_shape = (shape[1], shape[0]) if transpose else shape
    q = torch.empty(out_shape, dtype=torch.float8_e4m3fn, device="cuda")
    scale = torch.empty(1, device="cuda")
    ops.quantize_e4m3(xd, q, scale, transpose=transpose)
    torch.cuda.synchronize()
    want, want_scale = _quantize_ref(xd.float().cpu(), transpose)
    assert torch.equal(q.view(torch.uint8).cpu(), want)
    assert float(scale.cpu()[0]) == float(want_scale)


@pytest.mark.parametrize("transpose", [False, True])
@pytest.mark.parametrize("count,unaligned", [(5, False), (70, False), (3, True)])
def test_quantize_e4m3_batched_matches_per_block(T, transpose, count, unaligned):
    """The batched entry point (one launch per pass per 64 blocks; 70 blocks
    take two) gives each block the bytes and scale of the per-block entry
    point; a batch with an unaligned block takes the element-wise kernels."""
    torch, ops = T
    rng = np.random.default_rng(count + 2 * int(transpose) + 4 * int(unaligned))
    rows, cols = 64, 96
    xs = []
    for i in range(count):
        x = torch.from_numpy((rng.standard_normal((rows, cols)) * 10 ** rng.uniform(-2, 2)).astype(np.float32))
        if unaligned and i == 1:
            flat = torch.empty(rows * cols + 1, device="cuda")
            d = flat[1:].view(rows, cols)
            d.copy_(x)
            xs.append(d)
        else:
            xs.append(x.cuda().to(torch.bfloat16))
    if unaligned:  # one element type per batch
        xs = [x.float() if x.dtype != torch.float32 else x for x in xs]
    shape = (cols, rows) if transpose else (rows, cols)
    outs = [torch.empty(shape, dtype=torch.float8_e4m3fn, device="cuda") for _ in range(count)]
    scales = torch.empty(count, device="cuda")
    ops.quantize_e4m3_batched(xs, outs, scales, transpose=transpose)
    for i in range(count):
        ref = torch.empty(shape, dtype=torch.float8_e4m3fn, device="cuda")
        ref_scale = torch.empty(1, device="cuda")
        ops.quantize_e4m3(xs[i], ref, ref_scale, transpose=transpose)
        torch.cuda.synchronize()
        assert torch.equal(outs[i].view(torch.uint8), ref.view(torch.uint8)), i
        assert torch.equal(scales[i:i + 1], ref_scale), i


# ----------------------------------------------------------------- contraction
@pytest.mark.parametrize("precision", [0, 1])
def test_contraction_golden(T, precision):
    torch, ops = T
    g = golden("contraction_int.npz")
    I, J, K, L = [int(v) for v in g["c1_dims"]]
    out = torch.empty(I * J * L, device="cuda")
    ops.contraction(dev(torch, g["c1_lhs"]), [I, J, K], [0, 1, 2], dev(torch, g["c1_rhs"]), [K, L], [2, 3],
                    out, [0, 1, 3], 1.0, precision)
    assert np.array_equal(host(out), g["c1_out"])
    B, I2, K2, J2 = [int(v) for v in g["c2_dims"]]
    out2 = torch.empty(B * I2 * J2, device="cuda")
    ops.contraction(dev(torch, g["c2_lhs"]), [B, I2, K2], [0, 1, 2], dev(torch, g["c2_rhs"]), [K2, J2, B], [2, 3, 0],
                    out2, [3, 1, 0], 1.0, precision)
    assert np.array_equal(host(out2), g["c2_out"])


@pytest.mark.parametrize("spec", [
    ([37, 45, 64], [0, 1, 2], [64, 129], [2, 3], [0, 1, 3]),      # ijk,kl->ijl
    ([50, 40], [0, 1], [40, 30], [1, 2], [2, 0]),                 # transposed output
    ([20, 30, 6], [0, 1, 2], [30, 25], [1, 3], [3, 0]),           # lhs-only mode summed
    ([8, 9], [0, 1], [10, 11], [2, 3], [0, 2, 1, 3]),             # outer product
    ([37, 64], [0, 2], [129, 64], [3, 2], [0, 3]),               # both operands staged MN-major
    ([24, 40, 5], [0, 2, 1], [33, 40, 5], [3, 2, 1], [0, 3, 1]),  # batched, both MN-major
])
@pytest.mark.parametrize("precision", [0, 1])
def test_contraction_random_vs_f64(T, spec, precision):
    torch, ops = T
    dl, ml, dr, mr, mo = spec
    rng = np.random.default_rng(len(dl) * 10 + len(mo))
    lhs = rng.standard_normal(int(np.prod(dl))).astype(np.float32)
    rhs = rng.standard_normal(int(np.prod(dr))).astype(np.float32)
    ext = dict(zip(ml, dl)); ext.update(zip(mr, dr))
    out = torch.empty(int(np.prod([ext[m] for m in mo])), device="cuda")
    ops.contraction(dev(torch, lhs), dl, ml, dev(torch, rhs), dr, mr, out, mo, 0.5, precision)
    if precision == 0:
        ref = oracle.contraction_f64(lhs, dl, ml, rhs, dr, mr, mo, 0.5)
        assert rel_err(host(out), ref) <= 1e-5
    else:
        ref = oracle.contraction_f64(lhs, dl, ml, rhs, dr, mr, mo, 0.5)
        assert rel_err(host(out), ref) <= 1e-2
        # with no mode summed inside a gather (every lhs / rhs mode is shared or
        # kept), the bf16 staging rounds the inputs themselves: against FP64 of
        # the rounded inputs only the f32 accumulation differs, so a
        # staging-layout slip cannot hide inside the bf16 budget
        if set(ml) <= set(mr) | set(mo) and set(mr) <= set(ml) | set(mo):
            ref_q = oracle.contraction_f64(bf16_round(lhs), dl, ml, bf16_round(rhs), dr, mr, mo, 0.5)
            assert rel_err(host(out), ref_q) <= 1e-5


# ----------------------------------------------------------------- 2-SM (cta_group::2) tile
@pytest.mark.parametrize("key", ["128x256x64", "200x136x96", "256x512x256", "130x70x40"])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_matmul_tc_2sm_integer_exact(T, key, ta, tb):
    torch, ops = T
    g = golden("matmul_int.npz")
    a, b, cref = g[key + "_a"], g[key + "_b"], g[key + "_c"]
    A = np.ascontiguousarray(a.T) if ta else a
    B = np.ascontiguousarray(b.T) if tb else b

    def padded(x):
        rows, cols = x.shape
        p = (cols + 7) // 8 * 8
        buf = torch.zeros(rows, p, dtype=torch.bfloat16, device="cuda")
        buf[:, :cols] = dev(torch, x, torch.bfloat16)
        return buf[:, :cols]
    c = torch.full(cref.shape, -7.0, device="cuda")
    ops.matmul_tc([ops.tc_problem(padded(A), padded(B), c, bool(ta), bool(tb))], tile_n=512)
    assert np.array_equal(host(c), cref)


@pytest.mark.parametrize("m,n,k", [(1024, 1024, 1024), (512, 768, 4096), (384, 640, 136)])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_matmul_tc_2sm_random_vs_1sm(T, m, n, k, ta, tb):
    torch, ops = T
    rng = np.random.default_rng(m + 3 * n + k)
    a = rng.standard_normal((k, m) if ta else (m, k)).astype(np.float32)
    b = rng.standard_normal((n, k) if tb else (k, n)).astype(np.float32)
    A, B = dev(torch, a, torch.bfloat16), dev(torch, b, torch.bfloat16)
    c2 = torch.empty(m, n, device="cuda")
    c1 = torch.empty(m, n, device="cuda")
    ops.matmul_tc([ops.tc_problem(A, B, c2, bool(ta), bool(tb))], tile_n=512)
    ops.matmul_tc([ops.tc_problem(A, B, c1, bool(ta), bool(tb))], tile_n=256)
    assert rel_err(host(c2), oracle.matmul_f64(bf16_round(a), bf16_round(b), bool(ta), bool(tb))) <= 1e-5
    assert rel_err(host(c2), host(c1)) <= 1e-6


def test_matmul_tc_2sm_grouped_epilogues(T):
    torch, ops = T
    rng = np.random.default_rng(78)
    probs, refs, outs, keep = [], [], [], []
    for i, (m, n, k) in enumerate([(256, 256, 128), (128, 384, 64), (300, 200, 72), (512, 128, 256),
                                   (64, 64, 64), (200, 520, 320), (1024, 1024, 512)]):
        a = bf16_round(rng.standard_normal((m, k)))
        b = bf16_round(rng.standard_normal((k, n)))
        c0 = rng.standard_normal((m, n)).astype(np.float32)
        bias = rng.standard_normal(n).astype(np.float32)
        A, B, Cd, Bi = dev(torch, a, torch.bfloat16), dev(torch, b, torch.bfloat16), dev(torch, c0), dev(torch, bias)
        keep += [A, B, Bi]
        relu = i % 2 == 1
        probs.append(ops.tc_problem(A, B, Cd, alpha=0.5, beta=1.5, bias=Bi, relu=relu))
        ref = 0.5 * oracle.matmul_f64(a, b) + 1.5 * c0 + bias
        refs.append(np.maximum(ref, 0) if relu else ref)
        outs.append(Cd)
    plan = ops.TcPlan(probs, tile_n=512)  # 7 problems: device table
    plan.launch()
    for o, r in zip(outs, refs):
        assert rel_err(host(o), r) <= 1e-5
    plan.close()


@pytest.mark.parametrize("tile_n", [256, 512])
def test_matmul_tc_mixed_store_paths(T, tile_n):
    """One group alternating outputs that are written by TMA stores (f32, pitch
    512 x 4 B) and outputs that are not (pitch 510 x 4 B is not a multiple of 16
    bytes): every CTA runs tiles of both kinds back to back through the same
    shared-memory slot, over three launches."""
    torch, ops = T
    rng = np.random.default_rng(31)
    probs, keep, refs = [], [], []
    for i in range(48):
        m, k = 256 + 64 * (i % 3), 128 + 64 * (i % 4)
        n = 512 if i % 2 == 0 else 510
        a = bf16_round(rng.standard_normal((m, k)))
        b = bf16_round(rng.standard_normal((k, n)))
        A = dev(torch, a, torch.bfloat16)
        B = torch.zeros(k, 512, dtype=torch.bfloat16, device="cuda")  # operand pitch stays 16-byte aligned
        B[:, :n] = dev(torch, b, torch.bfloat16)
        B = B[:, :n]
        c = torch.full((m, n), float("nan"), device="cuda")  # C pitch n: 2048 B or 2040 B
        keep += [A, B, c]
        probs.append(ops.tc_problem(A, B, c))
        refs.append(oracle.matmul_f64(a, b))
    plan = ops.TcPlan(probs, tile_n=tile_n)
    for _ in range(3):
        plan.launch()
        for i, ref in enumerate(refs):
            assert rel_err(host(keep[3 * i + 2]), ref) <= 1e-5, i
    plan.close()


@pytest.mark.parametrize("tile_n", [128, 256, 512])
@pytest.mark.parametrize("out_bf16", [False, True])
def test_matmul_tc_c_colmajor(T, tile_n, out_bf16):
    """Column-major C (BBX_EPI_C_COLMAJOR, the contraction lowering's skinny
    GEMMs), on the TMA-store path: integer-valued inputs make the f32
    accumulation exact, so every problem equals the int64 product, transposed
    in memory, and matches the row-major store of the same group bit for bit.
    Problems mix ragged m, n from 32 to 264, both layouts of A, and bias / relu
    epilogues; the 8 elements of pitch padding stay untouched."""
    torch, ops = T
    rng = np.random.default_rng(51 + tile_n)
    odt = torch.bfloat16 if out_bf16 else torch.float32
    col, row, keep, refs = [], [], [], []
    for i in range(36):
        m = int(rng.choice([40, 128, 200, 264, 520, 1032]))
        n = int(rng.choice([32, 64, 96, 200, 256, 264]))
        k = int(rng.choice([32, 64, 128, 192]))
        a = rng.integers(-3, 4, (m, k)).astype(np.float32)
        b = rng.integers(-3, 4, (k, n)).astype(np.float32)
        bias = rng.integers(-8, 9, n).astype(np.float32) if i % 3 == 0 else None
        relu = i % 4 == 1
        ta = i % 2 == 1
        mp = m + 8  # pitches along m: 16-byte multiples, with 8 elements of padding to watch
        if ta:  # A stored k x m (MN-major) with pitch mp
            A = torch.zeros(k, mp, dtype=torch.bfloat16, device="cuda")
            A[:, :m] = dev(torch, a.T.copy(), torch.bfloat16)
            A = A[:, :m]
        else:
            A = dev(torch, a, torch.bfloat16)
        B = dev(torch, b, torch.bfloat16)
        cbuf = torch.full((n, mp), float("nan"), dtype=odt, device="cuda")
        cc = cbuf[:, :m]
        cr = torch.full((m, n + (8 - n % 8) % 8), float("nan"), dtype=odt, device="cuda")[:, :n]
        bt = dev(torch, bias) if bias is not None else None
        keep += [A, B, cbuf, cc, cr, bt]
        col.append(ops.tc_problem(A, B, cc, trans_a=ta, bias=bt, relu=relu, c_colmajor=True))
        row.append(ops.tc_problem(A, B, cr, trans_a=ta, bias=bt, relu=relu))
        r = a.astype(np.int64) @ b.astype(np.int64)
        if bias is not None:
            r = r + bias.astype(np.int64)[None, :]
        if relu:
            r = np.maximum(r, 0)
        refs.append(r.astype(np.float64))
    for group in (col, row):
        by_layout = {}
        for i, q in enumerate(group):
            by_layout.setdefault(q.trans_a, []).append(i)
        for idx in by_layout.values():
            plan = ops.TcPlan([group[i] for i in idx], tile_n=tile_n)
            plan.launch()
            plan.close()
    for i, ref in enumerate(refs):
        cc, cr = keep[6 * i + 3], keep[6 * i + 4]
        got_c, got_r = host(cc), host(cr)
        want = bf16_round(ref) if out_bf16 else ref
        assert np.array_equal(got_c.T, want), i
        assert np.array_equal(got_c.T, got_r), i
        pad = host(keep[6 * i + 2])[:, cc.shape[1]:]
        assert np.all(np.isnan(pad)), i  # pitch padding untouched


def test_matmul_tc_padded_pitch_untouched(T):
    """C rows whose length is not a whole number of 16-byte pieces, inside a
    padded pitch: the epilogue must not write the padding (TMA stores clip in
    16-byte pieces, so such C takes the staged stores); column-major C of such
    a length goes through stores from registers, exact, padding untouched."""
    torch, ops = T
    from bbts_b200._lib import BbxError
    rng = np.random.default_rng(61)
    cases = [(300, 510, torch.float32), (300, 500, torch.bfloat16), (300, 504, torch.bfloat16),
             (131, 508, torch.float32)]
    for m, n, odt in cases:
        k = 128
        a = rng.integers(-3, 4, (m, k)).astype(np.float32)
        b = rng.integers(-3, 4, (k, n)).astype(np.float32)
        A = dev(torch, a, torch.bfloat16)
        Bp = torch.zeros(k, 512, dtype=torch.bfloat16, device="cuda")
        Bp[:, :n] = dev(torch, b, torch.bfloat16)
        cbuf = torch.full((m, 512), float("nan"), dtype=odt, device="cuda")
        c = cbuf[:, :n]
        plan = ops.TcPlan([ops.tc_problem(A, Bp[:, :n], c)], tile_n=256)
        plan.launch()
        plan.close()
        ref = a.astype(np.int64) @ b.astype(np.int64)
        want = bf16_round(ref.astype(np.float32)) if odt == torch.bfloat16 else ref
        got = host(cbuf)
        assert np.array_equal(got[:, :n], want), (m, n)
        assert np.all(np.isnan(got[:, n:])), (m, n)
    for m, n, ldc, odt in [(1031, 64, 1040, torch.float32), (1031, 96, 1031, torch.float32),
                           (333, 200, 340, torch.bfloat16), (77, 40, 77, torch.bfloat16)]:
        a = rng.integers(-3, 4, (m, 64)).astype(np.float32)
        b = rng.integers(-3, 4, (64, n)).astype(np.float32)
        A, B = dev(torch, a, torch.bfloat16), dev(torch, b, torch.bfloat16)
        cbuf = torch.full((n, ldc), float("nan"), dtype=odt, device="cuda")
        for tile in (128, 256, 512):
            cbuf.fill_(float("nan"))
            plan = ops.TcPlan([ops.tc_problem(A, B, cbuf[:, :m], c_colmajor=True)], tile_n=tile)
            plan.launch()
            plan.close()
            ref = a.astype(np.int64) @ b.astype(np.int64)
            want = bf16_round(ref.astype(np.float32)) if odt == torch.bfloat16 else ref
            got = host(cbuf)
            assert np.array_equal(got[:, :m].T, want), (m, n, ldc, tile)
            assert np.all(np.isnan(got[:, m:])), (m, n, ldc, tile)
    cf = torch.empty(40, 77, device="cuda")
    with pytest.raises(BbxError, match="beta"):
        ops.matmul_tc([ops.tc_problem(A, B, cf, beta=1.0, c_colmajor=True)])


@pytest.mark.parametrize("tile_n", [128, 256])
@pytest.mark.parametrize("kmax", [192, 1024])
def test_matmul_tc_colmajor_mixed_group(T, tile_n, kmax):
    """One grouped launch mixing column-major C whose m is a whole number of
    16-byte pieces (TMA boxes), column-major C of any m and any element-aligned
    base (the 1-SM kernel's cooperative 128-row column runs) and row-major C,
    with bias / relu and f32 or bf16 outputs. Integer-valued inputs make every
    product exact: each C equals its int64 product and nothing around it
    changes. kmax 192 runs the eight-epilogue-warp kernel, 1024 the four-warp
    one."""
    torch, ops = T
    rng = np.random.default_rng(71 + tile_n + kmax)
    probs, checks, keep = [], [], []
    for i in range(48):
        kind = i % 4  # 0 column-major TMA, 1 column-major ragged m, 2 column-major offset base, 3 row-major
        odt = torch.bfloat16 if (i // 4) % 2 else torch.float32
        q = 8 if odt == torch.bfloat16 else 4  # elements per 16-byte piece
        m = int(rng.integers(1, 48)) * q if kind == 0 else int(rng.integers(1, 700))
        if kind == 1 and m % q == 0:
            m += 1
        n = int(rng.integers(1, 300))
        k = kmax if i == 0 else int(rng.choice([32, 64, 96, 160, kmax]))
        a = rng.integers(-3, 4, (m, k)).astype(np.float32)
        b = rng.integers(-3, 4, (k, n)).astype(np.float32)
        bias = rng.integers(-8, 9, n).astype(np.float32) if i % 3 == 0 else None
        relu = i % 5 == 1
        A = dev(torch, a, torch.bfloat16)
        B = torch.zeros(k, (n + 7) // 8 * 8, dtype=torch.bfloat16, device="cuda")  # pitch: 16-byte multiple
        B[:, :n] = dev(torch, b, torch.bfloat16)
        B = B[:, :n]
        bt = dev(torch, bias) if bias is not None else None
        off = int(rng.integers(1, q)) if kind == 2 else 0
        if kind == 3:
            ld = n + int(rng.integers(0, 9))
            flat = torch.full((off + m * ld + 5,), float("nan"), dtype=odt, device="cuda")
            c = flat[off:off + m * ld].view(m, ld)[:, :n]
        else:
            ld = m + (int(rng.integers(0, 3)) * q if kind == 0 else int(rng.integers(0, 9)))
            flat = torch.full((off + n * ld + 5,), float("nan"), dtype=odt, device="cuda")
            c = flat[off:off + n * ld].view(n, ld)[:, :m]
        probs.append(ops.tc_problem(A, B, c, bias=bt, relu=relu, c_colmajor=kind != 3))
        r = a.astype(np.int64) @ b.astype(np.int64)
        if bias is not None:
            r = r + bias.astype(np.int64)[None, :]
        if relu:
            r = np.maximum(r, 0)
        want = bf16_round(r.astype(np.float32)) if odt == torch.bfloat16 else r.astype(np.float64)
        keep += [A, B, bt, flat, c]
        checks.append((flat, off, ld, m, n, kind, want))
    plan = ops.TcPlan(probs, tile_n=tile_n)
    for _ in range(2):
        plan.launch()
        for i, (flat, off, ld, m, n, kind, want) in enumerate(checks):
            got = host(flat)
            rows, cols = (m, n) if kind == 3 else (n, m)
            body = got[off:off + rows * ld].reshape(rows, ld)
            assert np.array_equal(body[:, :cols], want if kind == 3 else want.T), (i, kind, m, n, off)
            assert np.all(np.isnan(body[:, cols:])) and np.all(np.isnan(got[:off])), (i, kind, m, n, off)
            assert np.all(np.isnan(got[off + rows * ld:])), (i, kind, m, n, off)
    plan.close()
