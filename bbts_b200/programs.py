"""Writers for the reference's on-disk command programs.

* .bbts   binary parsed command list (src/commands/parsed_command.h:194-383):
          u64 count; per command i32 type, string ud name, u8 is_gpu, string
          lists of input / output types, (tid, node) lists stored as raw
          std::tuple<tid_t, node_id_t> (node first, then tid), raw 4-byte params.
* .sbbts  text compile source (src/commands/command_compiler.h:977-1027).

bmm_bbts() emits the single-node form of applications/bmm/generate_bmm.cc:
uniform APPLYs for the A and B blocks, split^3 matrix_mult APPLYs, split^2
matrix_add REDUCEs and one DELETE of the partial products.
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
