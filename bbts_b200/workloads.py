"""Block-op DAG emitters: the command lists of the benchmark configurations.

* bmm      blocked matmul C = A.B on split x split grids (the DAG shape of
           applications/bmm/generate_bmm.cc:142-266: split^3 matrix_mult APPLYs,
           split^2 matrix_add REDUCEs, then DELETEs of the partial products)
* cpmm     cross-product blocked matmul: an (r x 1) grid times a (1 x c) grid
           (applications/cpmm/generate_cpmm.cc:228-274 without the shuffle)
* ffnn     one forward + backward step of a blocked 3-layer ReLU / softmax-CE
           network in the reference's ud style (applications/fnn/generate_ffnn.cc
           is the 2-layer original)
* random   seeded random DAGs of matmul / add / n-ary reduce / contraction ops

Each emitter registers its input blocks in a Runtime and queues the commands;
it returns a small description (tids of interesting tensors, algorithmic work).
"""
import numpy as np

from .runtime import cutensor_meta, dense_meta


def _rng(seed):
    return np.random.default_rng(seed)


class Emitter:
    def __init__(self, rt):
        self.rt = rt
        self.next_tid = 0
        self.flops = 0.0
        self.bytes = 0.0

    def tid(self):
        t = self.next_tid
        self.next_tid += 1
        return t


def _dtype_fmt(dtype):
    return {"f32": "dense", "bf16": "dense_bf16"}[dtype]


def fill_block(rt, tid, rows, cols, fmt, seed, dist="normal"):
    """Registers a rows x cols block filled on the device by the seeded Philox
    generator: N(0,1) (dist="normal") or U(-1,1) (dist="uniform")."""
    rt.put(tid, dense_meta(rt.fmt(fmt), rows, cols))
    d, a, b = (1, 0.0, 1.0) if dist == "normal" else (0, -1.0, 1.0)
    rt.fill_philox(tid, int(seed), d, a, b)


def put_block(rt, tid, arr, fmt):
    """Registers a host block in format `fmt` (dense f32 or dense_bf16)."""
    arr = np.ascontiguousarray(arr, np.float32)
    fid = rt.fmt(fmt)
    meta = dense_meta(fid, arr.shape[0], arr.shape[1])
    if fmt == "dense_bf16":
        import torch
        raw = torch.from_numpy(arr).to(torch.bfloat16).view(torch.int16).numpy()
        rt.put(tid, meta, raw)
    else:
        rt.put(tid, meta, arr)


def bmm(rt, n=4096, split=4, dtype="f32", out_dtype=None, seed=0, host=True, dist="normal"):
    """C = A.B, A and B n x n in split x split blocks. Returns dict with the
    A/B block tids, the C block tids and the host inputs (if host=True)."""
    e = Emitter(rt)
    fmt = _dtype_fmt(dtype)
    ofmt = _dtype_fmt(out_dtype or ("f32" if dtype == "bf16" else dtype))
    bs = n // split
    rng = _rng(seed)
    A, B, hostA, hostB = {}, {}, {}, {}
    for name, store, hstore in (("A", A, hostA), ("B", B, hostB)):
        for i in range(split):
            for j in range(split):
                t = e.tid()
                store[(i, j)] = t
                if host:
                    x = (rng.standard_normal((bs, bs)) if dist == "normal" else rng.uniform(-1, 1, (bs, bs))).astype(np.float32)
                    put_block(rt, t, x, fmt)
                    hstore[(i, j)] = x
                else:
                    fill_block(rt, t, bs, bs, fmt, seed=int(rng.integers(1 << 62)), dist=dist)
    mm = rt.impl("matrix_mult", [fmt, fmt], [ofmt])
    add = rt.impl("matrix_add", [ofmt, ofmt], [ofmt])
    parts, C = {}, {}
    for i in range(split):
        for j in range(split):
            for k in range(split):
                t = e.tid()
                rt.apply(mm, [A[(i, k)], B[(k, j)]], [t])
                parts.setdefault((i, j), []).append(t)
                e.flops += 2.0 * bs ** 3
    for i in range(split):
        for j in range(split):
            t = e.tid()
            rt.reduce(add, parts[(i, j)], t)
            C[(i, j)] = t
    rt.delete([t for v in parts.values() for t in v])
    return {"A": A, "B": B, "C": C, "hostA": hostA, "hostB": hostB, "flops": e.flops, "bs": bs, "split": split}


def cpmm_seeds(seed, rows, cols):
    """Philox seeds of the A row blocks and the B column blocks of cpmm."""
    return [seed + i for i in range(rows)], [seed + 1000 + j for j in range(cols)]


def cpmm(rt, rows=8, cols=8, bs=4096, dtype="bf16", seed=0):
    """C = A.B with A an (rows x 1) and B a (1 x cols) grid of bs x bs blocks
    (applications/cpmm/generate_cpmm.cc:228-274 on one node, without its
    shuffle): rows*cols independent matrix_mult APPLYs, no reduce, FP32
    output blocks. Inputs are U(-1,1) from the seeded Philox generator on the
    device (cpmm_seeds), rounded to the input format."""
    e = Emitter(rt)
    fmt = _dtype_fmt(dtype)
    sa, sb = cpmm_seeds(seed, rows, cols)
    A, B = {}, {}
    for i in range(rows):
        A[i] = e.tid()
        fill_block(rt, A[i], bs, bs, fmt, seed=sa[i], dist="uniform")
    for j in range(cols):
        B[j] = e.tid()
        fill_block(rt, B[j], bs, bs, fmt, seed=sb[j], dist="uniform")
    mm = rt.impl("matrix_mult", [fmt, fmt], ["dense"])
    C = {}
    for i in range(rows):
        for j in range(cols):
            t = e.tid()
            rt.apply(mm, [A[i], B[j]], [t])
            C[(i, j)] = t
            e.flops += 2.0 * bs ** 3
    return {"A": A, "B": B, "C": C, "flops": e.flops, "bs": bs, "seeds": (sa, sb), "fmt": fmt}


def ffnn(rt, batch=16384, d_in=8192, h1=8192, h2=4096, classes=1024, bs=2048, seed=0, host=False,
         dtype="bf16", split_a1=False):
    """One forward + backward step of a blocked 3-layer network:
    A1 = relu(X W1), A2 = relu(A1 W2), Z3 = A2 W3, loss = softmax-CE(Z3, labels);
    backward dW3 = A2^T G3, dA2 = G3 W3^T, dZ2 = dA2 * relu'(A2), dW2 = A1^T dZ2,
    dA1 = dZ2 W2^T, dZ1 = dA1 * relu'(A1), dW1 = X^T dZ1. Blocks are bs x bs
    (W3 / Z3 blocks bs x classes); X, W and activations are bf16, logits and
    weight gradients f32; every matmul over the block grid is split into block
    products plus a matrix_add REDUCE. Weights are N(0, 1/fan_in), X N(0, 1),
    labels uniform over the classes. Returns tids of the weights, dW blocks and
    per-row-block losses and the algorithmic FLOPs (2 * sum m n k).

    split_a1 (bf16 only): the first activation is kept as two bf16 blocks,
    hi = bf16(relu(Z1)) and lo = bf16(relu(Z1) - hi) (ud matrix_relu_split),
    and Z2 sums the products of both with W2. A bf16-rounded A1 moves enough
    layer-2 pre-activations across 0 to flip ~0.1 % of the layer-2 ReLU masks,
    which puts ~3 % of error into dW1 and dW2; hi + lo keeps ~16 bits. The
    extra products (2 * batch * h1 * h2 FLOP) are not counted as algorithmic
    FLOPs."""
    e = Emitter(rt)
    rng = _rng(seed)
    # dtype="f32" runs the same network on FP32 blocks (the plain path)
    B16, F32 = ("dense_bf16" if dtype == "bf16" else "dense"), "dense"
    R, KI, K1, K2 = batch // bs, d_in // bs, h1 // bs, h2 // bs
    mm_b = rt.impl("matrix_mult", [B16, B16], [B16])
    mm_f = rt.impl("matrix_mult", [B16, B16], [F32])
    add_b = rt.impl("matrix_add", [B16, B16], [B16])
    add_f = rt.impl("matrix_add", [F32, F32], [F32])
    relu = rt.impl("matrix_relu", [F32], [B16])  # f32 pre-activation -> bf16 activation
    drelu = rt.impl("matrix_relu_dif", [B16], [B16])
    had = rt.impl("matrix_matrix_hadamard", [B16, B16], [B16])
    sce = rt.impl("matrix_softmax_ce", [F32, "labels"], [B16, F32])
    split_a1 = split_a1 and dtype == "bf16"
    split = rt.impl("matrix_relu_split", [F32], [B16, B16]) if split_a1 else None
    host_vals = {}
    dead = []

    def inp(rows, cols, std):
        t = e.tid()
        if host:
            x = (rng.standard_normal((rows, cols)) * std).astype(np.float32)
            put_block(rt, t, x, B16)
            host_vals[t] = x
        else:
            rt.put(t, dense_meta(rt.fmt(B16), rows, cols))
            rt.fill_philox(t, int(rng.integers(1 << 62)), 1, 0.0, float(std))
        return t

    X = {(i, k): inp(bs, bs, 1.0) for i in range(R) for k in range(KI)}
    W1 = {(k, j): inp(bs, bs, 1.0 / np.sqrt(d_in)) for k in range(KI) for j in range(K1)}
    W2 = {(k, j): inp(bs, bs, 1.0 / np.sqrt(h1)) for k in range(K1) for j in range(K2)}
    W3 = {k: inp(bs, classes, 1.0 / np.sqrt(h2)) for k in range(K2)}
    labels = {}
    for i in range(R):
        t = e.tid()
        y = rng.integers(0, classes, bs).astype(np.int32)
        rt.put(t, dense_meta(rt.fmt("labels"), bs, 1), y)
        labels[i] = t
        host_vals[("y", i)] = y

    def blocked_mm(left, right, ni, nj, nk, out_impl, red_impl, ta=False, tb=False, m=bs, n=bs, k=bs,
                   lkey=None, rkey=None):
        """out[i,j] = sum_k op(left)[i,k] op(right)[k,j] as APPLYs + REDUCEs."""
        out = {}
        for i in range(ni):
            for j in range(nj):
                parts = []
                for kk in range(nk):
                    t = e.tid()
                    rt.apply(out_impl, [left(i, kk), right(kk, j)], [t], params=[bool(ta), bool(tb)])
                    e.flops += 2.0 * m * n * k
                    parts.append(t)
                if len(parts) == 1:
                    out[(i, j)] = parts[0]
                else:
                    t = e.tid()
                    rt.reduce(red_impl, parts, t)
                    dead.extend(parts)
                    out[(i, j)] = t
        return out

    def ew(impl, tids, params=()):
        t = e.tid()
        rt.apply(impl, tids, [t], params=list(params))
        return t

    # forward: pre-activations accumulate in f32 (so the ReLU masks come from
    # f32 values), activations are stored bf16 for the next tensor-core matmul
    Z1 = blocked_mm(lambda i, k: X[(i, k)], lambda k, j: W1[(k, j)], R, K1, KI, mm_f, add_f)
    if split_a1:
        A1, A1lo = {}, {}
        for key, t in Z1.items():
            hi, lo = e.tid(), e.tid()
            rt.apply(split, [t], [hi, lo])
            A1[key], A1lo[key] = hi, lo
    else:
        A1 = {key: ew(relu, [t]) for key, t in Z1.items()}
    dead.extend(Z1.values())
    if split_a1:
        # Z2[i, j] = sum over k of A1hi[i, k] W2[k, j] + A1lo[i, k] W2[k, j], one REDUCE in f32
        Z2 = {}
        for i in range(R):
            for j in range(K2):
                parts = []
                for kk in range(K1):
                    for src in (A1, A1lo):
                        t = e.tid()
                        rt.apply(mm_f, [src[(i, kk)], W2[(kk, j)]], [t], params=[False, False])
                        parts.append(t)
                    e.flops += 2.0 * bs * bs * bs
                t = e.tid()
                rt.reduce(add_f, parts, t)
                dead.extend(parts)
                Z2[(i, j)] = t
        dead.extend(A1lo.values())
    else:
        Z2 = blocked_mm(lambda i, k: A1[(i, k)], lambda k, j: W2[(k, j)], R, K2, K1, mm_f, add_f)
    A2 = {key: ew(relu, [t]) for key, t in Z2.items()}
    dead.extend(Z2.values())
    Z3 = blocked_mm(lambda i, k: A2[(i, k)], lambda k, j: W3[k], R, 1, K2, mm_f, add_f, n=classes)
    G3, loss = {}, {}
    for i in range(R):
        g, l = e.tid(), e.tid()
        rt.apply(sce, [Z3[(i, 0)], labels[i]], [g, l], params=[1.0 / batch])
        G3[i], loss[i] = g, l
    dead.extend(Z3.values())
    # backward
    dW3 = blocked_mm(lambda k, i: A2[(i, k)], lambda i, j: G3[i], K2, 1, R, mm_f, add_f, ta=True, n=classes)
    dA2 = blocked_mm(lambda i, j: G3[i], lambda j, k: W3[k], R, K2, 1, mm_b, add_b, tb=True, k=classes)
    M2 = {key: ew(drelu, [A2[key]]) for key in A2}
    dZ2 = {key: ew(had, [dA2[key], M2[key]]) for key in A2}
    dead.extend(list(dA2.values()) + list(M2.values()) + list(G3.values()))
    dW2 = blocked_mm(lambda k, i: A1[(i, k)], lambda i, j: dZ2[(i, j)], K1, K2, R, mm_f, add_f, ta=True)
    dA1 = blocked_mm(lambda i, j: dZ2[(i, j)], lambda j, k: W2[(k, j)], R, K1, K2, mm_b, add_b, tb=True)
    dead.extend(list(A2.values()) + list(dZ2.values()))
    M1 = {key: ew(drelu, [A1[key]]) for key in A1}
    dZ1 = {key: ew(had, [dA1[key], M1[key]]) for key in A1}
    dead.extend(list(dA1.values()) + list(M1.values()) + list(A1.values()))
    dW1 = blocked_mm(lambda k, i: X[(i, k)], lambda i, j: dZ1[(i, j)], KI, K1, R, mm_f, add_f, ta=True)
    dead.extend(dZ1.values())
    rt.delete(sorted(set(dead)))
    return {"X": X, "W1": W1, "W2": W2, "W3": W3, "labels": labels, "dW1": dW1, "dW2": dW2, "dW3": dW3,
            "loss": loss, "flops": e.flops, "host": host_vals, "bs": bs,
            "dims": (batch, d_in, h1, h2, classes), "split_a1": split_a1}


def random_dag(rt, n_ops=2000, depth=8, seed=0, dtype="bf16", lo=128, hi=2048, step=64,
               contraction_dims=(32, 256), mix=(0.60, 0.15, 0.15, 0.10), host=False, max_inputs=16,
               reuse=0.5):
    """Seeded random DAG: per level, ops drawn from the mix (matmul, add, n-ary
    reduce, contraction); every op reads at least one output of the previous
    level when one of a compatible shape exists, else fresh seeded inputs.
    matmul m,n,k uniform over multiples of `step` in [lo, hi]; add and reduce
    blocks m x n from the same grid; reduces take 2..max_inputs inputs;
    contraction 'ijk,kl->ijl' with i,j,k,l uniform in contraction_dims."""
    e = Emitter(rt)
    rng = _rng(seed)
    fmt = _dtype_fmt(dtype)
    odt = fmt
    mm_out_fmt = fmt
    mm = rt.impl("matrix_mult", [fmt, fmt], [mm_out_fmt])
    add = rt.impl("matrix_add", [fmt, fmt], [fmt])
    cfmt = rt.fmt("cutensor")
    # the bf16 DAG runs its contractions on the tensor cores too
    con = rt.impl_named("contraction", "b200_contraction_bf16" if dtype == "bf16" else "b200_contraction")
    sizes = np.arange(lo, hi + 1, step)
    dense_by_level = [[] for _ in range(depth + 1)]  # (tid, rows, cols)
    con_by_level = [[] for _ in range(depth + 1)]    # (tid, dims)
    readers = {}
    host_inputs = {}

    def fresh_dense(r, c):
        t = e.tid()
        if host:
            x = rng.standard_normal((r, c)).astype(np.float32)
            put_block(rt, t, x, fmt)
            host_inputs[t] = x
        else:
            fill_block(rt, t, r, c, fmt, seed=int(rng.integers(1 << 62)))
        return t

    def fresh_con(dims):
        t = e.tid()
        if host:
            x = rng.standard_normal(int(np.prod(dims))).astype(np.float32)
            rt.put(t, cutensor_meta(cfmt, dims), x)
            host_inputs[t] = x
        else:
            rt.put(t, cutensor_meta(cfmt, dims))
            rt.fill_philox(t, int(rng.integers(1 << 62)), 1, 0.0, 1.0)
        return t

    def pick(pool, pred):
        cands = [x for x in pool if pred(x)]
        return cands[rng.integers(len(cands))] if cands else None

    per_level = max(1, n_ops // depth)
    kinds = rng.choice(4, size=n_ops, p=np.asarray(mix) / np.sum(mix))
    ops = []
    for idx in range(n_ops):
        level = min(depth, 1 + idx // per_level)
        prev = dense_by_level[level - 1]
        earlier = [x for l in range(level) for x in dense_by_level[l]]
        kind = int(kinds[idx])
        t_out = e.tid()
        if kind == 0:  # matmul
            x = prev[rng.integers(len(prev))] if prev else None
            if x is None:
                m, k = int(rng.choice(sizes)), int(rng.choice(sizes))
                xa = fresh_dense(m, k)
            else:
                xa, m, k = x
            n = int(rng.choice(sizes))
            y = pick(earlier, lambda z: z[1] == k and z[2] == n) if rng.random() < reuse else None
            xb = y[0] if y else fresh_dense(k, n)
            rt.apply(mm, [xa, xb], [t_out])
            dense_by_level[level].append((t_out, m, n))
            e.flops += 2.0 * m * n * k
            ins = [xa, xb]
        elif kind in (1, 2):  # add / reduce
            x = prev[rng.integers(len(prev))] if prev else None
            if x is None:
                m, n = int(rng.choice(sizes)), int(rng.choice(sizes))
                xa = fresh_dense(m, n)
            else:
                xa, m, n = x
            cnt = 2 if kind == 1 else int(rng.integers(2, max_inputs + 1))
            ins = [xa]
            for _ in range(cnt - 1):
                y = pick(earlier, lambda z: z[1] == m and z[2] == n and z[0] not in ins) if rng.random() < reuse else None
                ins.append(y[0] if y else fresh_dense(m, n))
            if kind == 1:
                rt.apply(add, ins, [t_out])
            else:
                rt.reduce(add, ins, t_out)
            dense_by_level[level].append((t_out, m, n))
            e.bytes += (len(ins) + 1) * m * n * (2 if dtype == "bf16" else 4)
        else:  # contraction ijk,kl->ijl (modes i=0 j=1 k=2 l=3)
            cp = con_by_level[level - 1]
            c = cp[rng.integers(len(cp))] if cp else None
            if c is None:
                i_, j_, k_ = [int(v) for v in rng.integers(contraction_dims[0], contraction_dims[1] + 1, 3)]
                xl = fresh_con([i_, j_, k_])
            else:
                xl, (i_, j_, k_) = c[0], c[1][:3]
            l_ = int(rng.integers(contraction_dims[0], contraction_dims[1] + 1))
            xr = fresh_con([k_, l_])
            rt.apply(con, [xl, xr], [t_out], params=[3, 2, 3, 0, 1, 2, 2, 3, 0, 1, 3, 1.0])
            # the output (i, j, l) feeds later contractions as (i, j, k')
            con_by_level[level].append((t_out, [i_, j_, l_]))
            e.flops += 2.0 * i_ * j_ * k_ * l_
            ins = [xl, xr]
        for t in ins:
            readers[t] = idx
        ops.append((kind, ins, t_out))
    # delete every intermediate some later op reads (deferred until its last reader retires)
    produced = {t for _, _, t in ops}
    dead = sorted(t for t in readers if t in produced)
    if dead:
        rt.delete(dead)
    finals = sorted(produced - set(dead))
    return {"flops": e.flops, "bytes": e.bytes, "finals": finals, "n_ops": n_ops, "host_inputs": host_inputs,
            "ops": ops}
