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
    from ._lib import lib, check
    fid = rt.fmt(fmt)
    rt.put(tid, dense_meta(fid, rows, cols))
    ptr, _ = rt.payload(tid)
    dt = 1 if fmt == "dense_bf16" else 0
    d, a, b = (1, 0.0, 1.0) if dist == "normal" else (0, -1.0, 1.0)
    check(lib.bbx_fill_philox(dt, ptr, rows * cols, int(seed), d, a, b, rt.stream))


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


def cpmm(rt, rows=8, cols=8, bs=4096, dtype="bf16", seed=0, host=False):
    """C = A.B with A an (rows x 1) and B a (1 x cols) grid of bs x bs blocks:
    rows*cols independent matrix_mult ops, no reduce."""
    e = Emitter(rt)
    fmt = _dtype_fmt(dtype)
    rng = _rng(seed)
    A, B, hA, hB = {}, {}, {}, {}
    for i in range(rows):
        t = e.tid()
        x = rng.uniform(-1, 1, (bs, bs)).astype(np.float32)
        put_block(rt, t, x, fmt)
        A[i] = t
        if host:
            hA[i] = x
    for j in range(cols):
        t = e.tid()
        x = rng.uniform(-1, 1, (bs, bs)).astype(np.float32)
        put_block(rt, t, x, fmt)
        B[j] = t
        if host:
            hB[j] = x
    mm = rt.impl("matrix_mult", [fmt, fmt], ["dense"])
    C = {}
    for i in range(rows):
        for j in range(cols):
            t = e.tid()
            rt.apply(mm, [A[i], B[j]], [t])
            C[(i, j)] = t
            e.flops += 2.0 * bs ** 3
    return {"A": A, "B": B, "C": C, "hostA": hA, "hostB": hB, "flops": e.flops}


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
            from ._lib import lib, check
            rt.put(t, cutensor_meta(cfmt, dims))
            ptr, _ = rt.payload(t)
            check(lib.bbx_fill_philox(0, ptr, int(np.prod(dims)), int(rng.integers(1 << 62)), 1, 0.0, 1.0, rt.stream))
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
