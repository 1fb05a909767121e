"""Per-group profile of a compiled random block-op DAG on one GPU.

Usage:
    python -m bbts_b200.dag_profile --ops 600 --mix 0,0,0,1 --tile 256 [--seed 7] [--stream-kernel 0]

Builds the random DAG of `workloads.random_dag` (the generator of the random-DAG workloads:
matmul / add / reduce / contraction mix over bf16 blocks), compiles it with the heuristic
schedule, replays the graph to time its makespan, then replays each group alone
(`bbx_dag_profile`) and prints one JSON line: the makespan, the DAG's FLOP rate and, per group
class and tile, the groups' count, time, FLOP rate and algorithmic bandwidth.

`--groups` adds one row per launch group (wave, kind, tile, time, rates). `--once` compiles and
launches the DAG once without timing or profiling: the form to run under a kernel profiler, where
the first `tc_gemm_kernel` launch is wave 0's tensor group.
"""
import argparse
import json

import torch

from . import runtime, workloads


def profile(n_ops, mix, tile, seed=7, depth=8, stream_kernel=0, reps=10, groups=False):
    rt = runtime.Runtime()
    rt.set_dag_stream_kernel(stream_kernel)
    info = workloads.random_dag(rt, n_ops=n_ops, depth=depth, seed=seed, dtype="bf16", mix=mix)
    torch.cuda.synchronize()
    dag = rt.build_dag(runtime.HEURISTIC, tile_n=tile)
    try:
        for _ in range(3):
            dag.launch()
        s = torch.cuda.ExternalStream(rt.stream.value)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            dag.launch()
        e1.record(s)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / reps
        agg = {}
        rows = []
        for g, t in zip(dag.profile(), dag.group_tiles()):
            rows.append({"wave": g["wave"], "kind": g["kind"], "tile": t, "ms": round(g["ms"], 4),
                         "gbs": round(g["bytes"] / g["ms"] / 1e6, 1) if g["ms"] else None,
                         "tflops": round(g["flops"] / g["ms"] / 1e9, 1) if g["ms"] else None})
            a = agg.setdefault(g["kind"] + ("_t%d" % t if t else ""), [0, 0.0, 0.0, 0.0])
            a[0] += 1
            a[1] += g["ms"]
            a[2] += g["flops"]
            a[3] += g["bytes"]
        out = {"n_ops": n_ops, "mix": list(mix), "tile": tile, "seed": seed,
                "makespan_ms": round(ms, 3), "tflops": round(info["flops"] / ms / 1e9, 1),
                "waves": dag.stats()["waves"], "register_waves": dag.register_waves(),
                "groups": {k: {"n": v[0], "ms": round(v[1], 3),
                               "tflops": round(v[2] / v[1] / 1e9, 1) if v[1] else None,
                               "gbs": round(v[3] / v[1] / 1e6, 1) if v[1] else None}
                           for k, v in sorted(agg.items())}}
        if groups:
            out["group_rows"] = rows
        return out
    finally:
        dag.close()
        rt.close()


def launch_once(n_ops, mix, tile, seed=7, depth=8):
    rt = runtime.Runtime()
    workloads.random_dag(rt, n_ops=n_ops, depth=depth, seed=seed, dtype="bf16", mix=mix)
    dag = rt.build_dag(runtime.HEURISTIC, tile_n=tile)
    try:
        dag.launch()
        torch.cuda.synchronize()
    finally:
        dag.close()
        rt.close()


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--ops", type=int, default=600)
    ap.add_argument("--mix", default="0.60,0.15,0.15,0.10",
                    help="fractions of matmul, add, reduce, contraction ops")
    ap.add_argument("--tile", type=int, default=-1, help="128 / 256 / 512, 0 = size rule, -1 = autotuned")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--depth", type=int, default=8)
    ap.add_argument("--stream-kernel", type=int, default=0, help="0 auto, 1 register, 2 per wave")
    ap.add_argument("--groups", action="store_true", help="one row per launch group")
    ap.add_argument("--once", action="store_true")
    a = ap.parse_args(argv)
    mix = tuple(float(x) for x in a.mix.split(","))
    if len(mix) != 4:
        raise SystemExit("--mix takes four fractions")
    if a.once:
        launch_once(a.ops, mix, a.tile, a.seed, a.depth)
        return
    print(json.dumps(profile(a.ops, mix, a.tile, a.seed, a.depth, a.stream_kernel, groups=a.groups)), flush=True)


if __name__ == "__main__":
    main()
