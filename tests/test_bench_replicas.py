"""Replica aggregation of bench.py on two gloo ranks (CPU): the job time is the
slowest rank's device time and the job throughput counts every rank's work."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, torch.device("cpu"))
        out[rank] = (ms, bench.job_tflops(8.796e12, world, ms))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_throughput():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]                      # every rank sees the job's time
    ms, tf = res[0]
    assert ms == 15.0                            # the slowest rank
    assert tf == pytest.approx(2 * 8.796e12 / 15e-3 / 1e12)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1, None) == 3.5
    assert bench.job_tflops(1e12, 1, 1000.0) == pytest.approx(1.0)


def test_cpu_step_sample():
    """The CPU baseline's step sample: every block product in order within the
    budget, C[0][0] returned for the cross-check, and a stop once the budget
    has passed (at least one product is always done)."""
    import numpy as np
    sys.path.insert(0, ROOT)
    import bench
    import oracle
    rng = np.random.default_rng(3)
    a = [rng.uniform(-1, 1, (64, 48)).astype(np.float32) for _ in range(2)]
    b = [rng.uniform(-1, 1, (48, 80)).astype(np.float32) for _ in range(3)]
    tf, done, dt, c00 = bench.cpu_step_tflops(a, b, threads=2)
    assert done == 6 and tf > 0 and dt > 0
    assert np.array_equal(c00, oracle.sgemm(a[0], b[0], threads=1))
    tf, done, dt, c00 = bench.cpu_step_tflops(a, b, threads=2, budget_s=0.0)
    assert done == 1 and c00 is not None


def test_reference_arm_line(capsys):
    """The reference arm on a tiny cpmm (2x2 grid of 64^2 blocks): a measured
    warm-up product, a bounded sample per step, one JSON line whose
    ms_per_step is a measured step (steps x ms_per_step fits the run) and
    whose cpu_baseline / e2e restate the line's value."""
    import json
    import time
    import types
    sys.path.insert(0, ROOT)
    import bench
    saved = bench.GRID, bench.BS, bench.REF_BUDGET_S
    bench.GRID, bench.BS, bench.REF_BUDGET_S = 2, 64, 0.05
    try:
        args = types.SimpleNamespace(gpus=1, steps=3, warmup=1)
        t0 = time.perf_counter()
        bench.run_reference(args)
        wall = time.perf_counter() - t0
    finally:
        bench.GRID, bench.BS, bench.REF_BUDGET_S = saved
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "TFLOP/s" and line["value"] > 0
    assert line["steps"] * line["ms_per_step"] * 1e-3 <= wall
    assert line["cpu_baseline"]["value"] == line["value"] == line["e2e"]["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"


def test_reference_inputs_are_the_device_fill_values():
    """The reference arm's inputs restate the device fill: Philox uniform in
    [-1, 1), rounded to bf16 (so exactly representable in bf16)."""
    import numpy as np
    import torch
    sys.path.insert(0, ROOT)
    import bench
    saved = bench.GRID, bench.BS
    bench.GRID, bench.BS = 2, 32
    try:
        a, b = bench.cpmm_block_inputs(bench.CPMM_SEED)
    finally:
        bench.GRID, bench.BS = saved
    assert len(a) == 2 and a[0].shape == (32, 32)
    x = torch.from_numpy(a[1])
    assert torch.equal(x.to(torch.bfloat16).float(), x)
    assert float(x.abs().max()) <= 1.0 and not np.array_equal(a[0], a[1])
