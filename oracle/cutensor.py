"""CPU oracle for the "cutensor" plugin's element-wise / reduction block ops.

Test infrastructure only: the product path never imports this module.

Tensors are flat column-major FP32 arrays (mode 0 fastest), rank <= 4, as in
the plugin's tensor format (libraries/cutensor/cu.h:60-169). Each function
restates the checker the plugin compiles under CU_BARB_REFERENCE:

  reduction  libraries/cutensor/reduction.h:36-100 (params :13-21) and the
             fold order of its CPU op (:103-160): dropped modes first,
             first dropped mode fastest, left fold from the first element
  ew         libraries/cutensor/ew.h:44-120 (params :13-29, unary ops
             utils.h:69-91); output mode r is input mode ordering[r], the
             convention of the plugin's out-meta (ew.h:32-41) and of its GPU op
  ewb        libraries/cutensor/ewb.h:122-204 (params :13-46)
  ewb_castable libraries/cutensor/ewb_castable.h (same-shape ewb, alpha = beta = 1)
  expand     libraries/cutensor/expand.h:1-140

No golden vectors exist for these ops in the reference (nothing outside the
plugin calls them); parity rests on these restated checkers. Arithmetic is
float32 in the same order as the plugin's CPU path, so every op except exp /
sigmoid compares bit for bit.
"""
import numpy as np

F = np.float32


def _nd(flat, dims):
    return np.asarray(flat, F).reshape(tuple(dims), order="F") if len(dims) else np.asarray(flat, F).reshape(())


def _flat(a):
    return np.asarray(a, F).reshape(-1, order="F")


# reduction castable ops (utils.h:32-35)
def _fold(op, l, r):
    if op == 0:
        return (l + r).astype(F)
    if op == 1:
        return np.where(l > r, l, r).astype(F)
    if op == 2:
        return np.where(l < r, l, r).astype(F)
    if op == 3:
        return (l * r).astype(F)
    raise ValueError("reduction op must be 0..3")


def reduction(x, dims, op, alpha, ordering):
    """out (dims[ordering[r]]...) = alpha * left fold of op over the dropped modes."""
    dims = list(dims)
    a = _nd(x, dims)
    dropped = [m for m in range(len(dims)) if m not in ordering]
    # permute to (dropped..., kept in ordering order); column-major flatten of the
    # dropped block runs the first dropped mode fastest
    p = np.transpose(a, dropped + list(ordering)) if dims else a
    nagg = int(np.prod([dims[m] for m in dropped])) if dropped else 1
    nout = int(np.prod([dims[m] for m in ordering])) if ordering else 1
    flat = _flat(p).reshape(nout, nagg) if nagg and nout else np.zeros((nout, 0), F)
    acc = flat[:, 0].copy() if nagg else np.zeros(nout, F)
    for j in range(1, nagg):
        acc = _fold(op, acc, flat[:, j])
    return (F(alpha) * acc).astype(F)


def _unary(uop, v, scalar):
    v = np.asarray(v, F)
    with np.errstate(all="ignore"):
        if uop == 0:
            e = np.exp(v.astype(np.float64))
            return (e / (1.0 + e)).astype(F)
        if uop == 1:
            return np.exp(v.astype(np.float64)).astype(F)
        if uop == 2:
            return (v * v).astype(F)
        if uop == 3:
            return np.where(v > 0, v, F(0)).astype(F)
        if uop == 4:
            return np.where(v < 0, F(0), F(1)).astype(F)
        if uop == 5:
            return np.sqrt(v).astype(F)
        if uop == 6:
            return (v + F(scalar)).astype(F)
    raise ValueError("is not a valid unary op")


def ew(x, dims, uop, alpha, ordering, scalar=0.0):
    """out = alpha * uop(x), output mode r = input mode ordering[r]; returns (flat, out dims)."""
    dims = list(dims)
    a = _nd(x, dims)
    o = np.transpose(a, list(ordering)) if dims else a
    with np.errstate(all="ignore"):
        v = (F(alpha) * _unary(uop, o, scalar)).astype(F)
    return _flat(v), [dims[m] for m in ordering]


def _binary(op, l, r):
    with np.errstate(all="ignore"):
        if op == 0:
            return (l + r).astype(F)
        if op == 1:
            return np.where(l > r, l, r).astype(F)
        if op == 2:
            return np.where(l > r, r, l).astype(F)
        if op == 3:
            return (l * r).astype(F)
        if op == 4:
            return (l - r).astype(F)
        if op == 5:
            return (l / r).astype(F)
    raise ValueError("ewb op must be 0..5")


def ewb(lhs, dims_l, ord_l, rhs, dims_r, ord_r, op, alpha, beta):
    """out = op(alpha * lhs, beta * rhs) over the output modes; an input lacking
    an output mode is broadcast along it. Returns (flat, out dims)."""
    rank = 1 + max(list(ord_l) + list(ord_r)) if (ord_l or ord_r) else 0
    od = [1] * rank
    for q, m in enumerate(ord_l):
        od[m] = dims_l[q]
    for q, m in enumerate(ord_r):
        od[m] = dims_r[q]

    def spread(x, dims, ordr):
        a = _nd(x, dims)
        # move input mode q to output mode ordr[q], size-1 axes elsewhere
        order = sorted(range(len(ordr)), key=lambda q: ordr[q])
        a = np.transpose(a, order) if len(ordr) else a
        shape = [1] * rank
        for q in range(len(ordr)):
            shape[ordr[q]] = dims[q]
        return np.broadcast_to(a.reshape(shape, order="F") if rank else a, od)

    with np.errstate(all="ignore"):
        l = (F(alpha) * spread(lhs, dims_l, ord_l)).astype(F)
        r = (F(beta) * spread(rhs, dims_r, ord_r)).astype(F)
    return _flat(_binary(op, l, r)), od


def ewb_castable(lhs, rhs, dims, op):
    n = list(range(len(dims)))
    return ewb(lhs, dims, n, rhs, dims, n, op, 1.0, 1.0)[0]


def expand(x, params5):
    """Zeros of shape (sz_out...), then out[start_out + i] = in[start_in + i]
    for i in the box (num...)."""
    rank = len(params5) // 5
    sz_in = [params5[5 * i] for i in range(rank)]
    sz_out = [params5[5 * i + 1] for i in range(rank)]
    a = _nd(x, sz_in)
    o = np.zeros(sz_out, F)
    si = tuple(slice(params5[5 * i + 3], params5[5 * i + 3] + params5[5 * i + 2]) for i in range(rank))
    so = tuple(slice(params5[5 * i + 4], params5[5 * i + 4] + params5[5 * i + 2]) for i in range(rank))
    o[so] = a[si]
    return _flat(o)
