"""Writers for the reference's on-disk command programs.

* .bbts   binary parsed command list (src/commands/parsed_command.h:194-383):
          u64 count; per command i32 type, string ud name, u8 is_gpu, string
          lists of input / output types, (tid, node) lists stored as raw
          std::tuple<tid_t, node_id_t> (node first, then tid), raw 4-byte params.
* .sbbts  text compile source (src/commands/command_compiler.h:977-1027).

Emitters of the benchmark programs, single-node forms:
* bmm_bbts    applications/bmm/generate_bmm.cc: uniform APPLYs for the A and B
              blocks, split^3 matrix_mult APPLYs, split^2 matrix_add REDUCEs
              and one DELETE of the partial products;
* cpmm_bbts   applications/cpmm/generate_cpmm.cc:228-274 without its shuffles
              (one node owns every block): uniform APPLYs for an rows x k and a
              k x cols block grid, matrix_mult APPLYs, matrix_add REDUCEs over
              k when k > 1, DELETE of the partials;
* ffnn_bbts   the blocked FFN step of workloads.ffnn (the 3-layer, softmax-CE
              extension of applications/fnn/generate_ffnn.cc:202-380), recorded
              from the emitter with ProgramRecorder.
"""
import struct

APPLY, REDUCE, MOVE, DELETE = 0, 1, 2, 3


def _str(s):
    b = s.encode()
    return struct.pack("<Q", len(b)) + b


def _tids(lst):
    out = struct.pack("<Q", len(lst))
    for tid, node in lst:
        out += struct.pack("<ii", node, tid)
    return out


def _params(params):
    out = struct.pack("<Q", len(params))
    for p in params:
        if isinstance(p, float):
            out += struct.pack("<f", p)
        elif isinstance(p, bool):
            out += struct.pack("<I", int(p))
        else:
            out += struct.pack("<I", int(p) & 0xFFFFFFFF)
    return out


def write_bbts(path, commands):
    """commands: dicts {type, ud, in_types, out_types, is_gpu, inputs, outputs, params};
    inputs / outputs are lists of (tid, node)."""
    buf = struct.pack("<Q", len(commands))
    for c in commands:
        buf += struct.pack("<i", c["type"])
        buf += _str(c.get("ud", ""))
        buf += struct.pack("<B", 1 if c.get("is_gpu", False) else 0)
        buf += struct.pack("<Q", len(c.get("in_types", [])))
        for s in c.get("in_types", []):
            buf += _str(s)
        buf += struct.pack("<Q", len(c.get("out_types", [])))
        for s in c.get("out_types", []):
            buf += _str(s)
        buf += _tids(c.get("inputs", []))
        buf += _tids(c.get("outputs", []))
        buf += _params(c.get("params", []))
    with open(path, "wb") as f:
        f.write(buf)


def read_bbts(path):
    """Parses a .bbts file back into the command dicts write_bbts takes
    (params as raw 32-bit words)."""
    buf = open(path, "rb").read()
    pos = 0

    def take(fmt):
        nonlocal pos
        v = struct.unpack_from(fmt, buf, pos)
        pos += struct.calcsize(fmt)
        return v

    def string():
        nonlocal pos
        (n,) = take("<Q")
        s = buf[pos:pos + n].decode()
        pos += n
        return s

    def tids():
        (n,) = take("<Q")
        return [(tid, node) for node, tid in (take("<ii") for _ in range(n))]

    (count,) = take("<Q")
    out = []
    for _ in range(count):
        (kind,) = take("<i")
        ud = string()
        (gpu,) = take("<B")
        (n,) = take("<Q")
        ins = [string() for _ in range(n)]
        (n,) = take("<Q")
        outs = [string() for _ in range(n)]
        inputs, outputs = tids(), tids()
        (n,) = take("<Q")
        params = [take("<I")[0] for _ in range(n)]
        out.append({"type": kind, "ud": ud, "is_gpu": bool(gpu), "in_types": ins, "out_types": outs,
                    "inputs": inputs, "outputs": outputs, "params": params})
    if pos != len(buf):
        raise ValueError("%s: %d trailing bytes" % (path, len(buf) - pos))
    return out


def write_sbbts(path, specs, commands):
    """specs: [(id, ud_name, in_types, out_types)];
    commands: [(ud_id, "APPLY"|"REDUCE"|"DELETE", in_tids, out_tids, params)]."""
    lines = [str(len(specs))]
    for sid, name, ins, outs in specs:
        lines.append("%d %s %d %s %d %s" % (sid, name, len(ins), " ".join(ins), len(outs), " ".join(outs)))
    lines.append(str(len(commands)))
    for ud, kind, ins, outs, params in commands:
        ps = []
        for p in params:
            ps.append(("float %r" % p) if isinstance(p, float) else ("int %d" % int(p)))
        lines.append("%d %s %d %s %d %s %d %s" % (ud, kind, len(ins), " ".join(map(str, ins)), len(outs),
                                               " ".join(map(str, outs)), len(ps), " ".join(ps)))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def bmm_bbts(path, n, split, fmt="dense"):
    """The blocked-matmul program for one node; returns (A tids, B tids, C tids)."""
    bs = n // split
    cmds, tid = [], 0
    A, B = {}, {}
    for store in (A, B):
        for i in range(split):
            for j in range(split):
                cmds.append({"type": APPLY, "ud": "uniform", "in_types": [], "out_types": [fmt], "is_gpu": False,
                             "inputs": [], "outputs": [(tid, 0)], "params": [bs, bs, 0.0, 1.0]})
                store[(i, j)] = tid
                tid += 1
    parts = {}
    for i in range(split):
        for j in range(split):
            for k in range(split):
                cmds.append({"type": APPLY, "ud": "matrix_mult", "in_types": [fmt, fmt], "out_types": [fmt],
                             "is_gpu": True, "inputs": [(A[(i, k)], 0), (B[(k, j)], 0)], "outputs": [(tid, 0)]})
                parts.setdefault((i, j), []).append(tid)
                tid += 1
    C = {}
    for i in range(split):
        for j in range(split):
            cmds.append({"type": REDUCE, "ud": "matrix_add", "in_types": [fmt, fmt], "out_types": [fmt],
                         "is_gpu": True, "inputs": [(t, 0) for t in parts[(i, j)]], "outputs": [(tid, 0)]})
            C[(i, j)] = tid
            tid += 1
    cmds.append({"type": DELETE, "inputs": [(t, 0) for v in parts.values() for t in v]})
    write_bbts(path, cmds)
    return A, B, C


def cpmm_bbts(path, rows, cols, bs, k=1, fmt="dense_bf16", out_fmt="dense", seed=1000):
    """The cross-product blocked matmul program for one node: A is a rows x k
    grid and B a k x cols grid of bs x bs blocks, generated in-program by the
    uniform ud as U(-1, 1) with explicit Philox seeds (A block (i, kk): seed +
    i + 100 kk, B block (kk, j): seed + 1000 + j + 100 kk -- with k = 1 the
    seeds of workloads.cpmm_seeds); C[i, j] = sum over kk of A[i, kk] B[kk, j].
    Returns (A tids, B tids, C tids)."""
    cmds, tid = [], 0
    A, B = {}, {}
    for i in range(rows):
        for kk in range(k):
            cmds.append({"type": APPLY, "ud": "uniform", "in_types": [], "out_types": [fmt], "is_gpu": True,
                         "inputs": [], "outputs": [(tid, 0)], "params": [bs, bs, -1.0, 1.0, seed + i + 100 * kk]})
            A[(i, kk)] = tid
            tid += 1
    for kk in range(k):
        for j in range(cols):
            cmds.append({"type": APPLY, "ud": "uniform", "in_types": [], "out_types": [fmt], "is_gpu": True,
                         "inputs": [], "outputs": [(tid, 0)],
                         "params": [bs, bs, -1.0, 1.0, seed + 1000 + j + 100 * kk]})
            B[(kk, j)] = tid
            tid += 1
    parts, C = {}, {}
    for i in range(rows):
        for j in range(cols):
            for kk in range(k):
                cmds.append({"type": APPLY, "ud": "matrix_mult", "in_types": [fmt, fmt], "out_types": [out_fmt],
                             "is_gpu": True, "inputs": [(A[(i, kk)], 0), (B[(kk, j)], 0)], "outputs": [(tid, 0)]})
                parts.setdefault((i, j), []).append(tid)
                tid += 1
    for (i, j), ps in parts.items():
        if len(ps) == 1:
            C[(i, j)] = ps[0]
            continue
        cmds.append({"type": REDUCE, "ud": "matrix_add", "in_types": [out_fmt, out_fmt], "out_types": [out_fmt],
                     "is_gpu": True, "inputs": [(t, 0) for t in ps], "outputs": [(tid, 0)]})
        C[(i, j)] = tid
        tid += 1
    dead = [t for ps in parts.values() if len(ps) > 1 for t in ps]
    if dead:
        cmds.append({"type": DELETE, "inputs": [(t, 0) for t in dead]})
    write_bbts(path, cmds)
    return A, B, C


class ProgramRecorder:
    """Stands in for a Runtime in the workload emitters and records what they
    queue as .bbts command dicts (ud name and types instead of impl ids, as
    the program format stores them). Input blocks the emitter registers are
    recorded in `inputs` (tid -> meta, plus the Philox fill or host array)
    and are not part of the program: a node that runs it must hold them."""

    FORMATS = ("dense", "dense_bf16", "dense_e4m3", "ffnn_dense", "cutensor", "labels")

    def __init__(self):
        self.commands = []
        self.inputs = {}

    def fmt(self, name):
        return self.FORMATS.index(name)

    def impl(self, ud_name, in_types, out_types, gpu=True):
        return (ud_name, tuple(in_types), tuple(out_types), bool(gpu))

    def impl_named(self, ud_name, impl_name, in_types=("cutensor", "cutensor"), out_types=("cutensor",)):
        return self.impl(ud_name, in_types, out_types)

    def put(self, tid, meta, data=None, device_ptr=None, nbytes=None):
        self.inputs[tid] = {"meta": bytes(meta), "data": data}

    def fill_philox(self, tid, seed, dist=0, a=0.0, b=1.0):
        self.inputs[tid]["fill"] = (int(seed), int(dist), float(a), float(b))

    def _cmd(self, kind, impl, inputs, outputs, params):
        ud, ins, outs, gpu = impl
        self.commands.append({"type": kind, "ud": ud, "in_types": list(ins), "out_types": list(outs), "is_gpu": gpu,
                              "inputs": [(t, 0) for t in inputs], "outputs": [(t, 0) for t in outputs],
                              "params": list(params)})

    def apply(self, impl, inputs, outputs, params=(), cmd_id=None):
        self._cmd(APPLY, impl, inputs, outputs, params)

    def reduce(self, impl, inputs, output, params=(), cmd_id=None):
        self._cmd(REDUCE, impl, inputs, [output], params)

    def delete(self, tids, cmd_id=None):
        self.commands.append({"type": DELETE, "inputs": [(t, 0) for t in tids]})


def ffnn_bbts(path, **ffnn_args):
    """Writes the blocked FFN step (workloads.ffnn with `ffnn_args`) as a .bbts
    program. Its input blocks (X, W1, W2, W3 and the labels) are not created by
    the program: a runtime that loads it must hold them, e.g. registered by
    workloads.ffnn with the same arguments. Returns (the emitter's description,
    the recorded inputs)."""
    from . import workloads
    rec = ProgramRecorder()
    info = workloads.ffnn(rec, **ffnn_args)
    write_bbts(path, rec.commands)
    return info, rec.inputs
