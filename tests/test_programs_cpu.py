"""Program emitters on the CPU: the .bbts files they write parse back into
the command lists of the reference's generators (single-node forms)."""
import collections

from bbts_b200 import programs


def test_cpmm_program_shape(tmp_path):
    path = str(tmp_path / "cpmm.bbts")
    A, B, C = programs.cpmm_bbts(path, rows=3, cols=2, bs=64, k=2, seed=1000)
    cmds = programs.read_bbts(path)
    kinds = collections.Counter((c["type"], c["ud"]) for c in cmds)
    assert kinds[(programs.APPLY, "uniform")] == 3 * 2 + 2 * 2
    assert kinds[(programs.APPLY, "matrix_mult")] == 3 * 2 * 2
    assert kinds[(programs.REDUCE, "matrix_add")] == 3 * 2
    assert kinds[(programs.DELETE, "")] == 1 and cmds[-1]["type"] == programs.DELETE
    # explicit seeds: A(i, kk) = seed + i + 100 kk; with k = 1 they are workloads.cpmm_seeds
    seeds = {c["outputs"][0][0]: c["params"][4] for c in cmds if c["ud"] == "uniform"}
    assert seeds[A[(2, 1)]] == 1000 + 2 + 100 and seeds[B[(1, 0)]] == 1000 + 1000 + 0 + 100
    reduce_out = {c["outputs"][0][0] for c in cmds if c["type"] == programs.REDUCE}
    assert reduce_out == set(C.values())
    path1 = str(tmp_path / "cpmm1.bbts")
    A1, B1, C1 = programs.cpmm_bbts(path1, rows=8, cols=8, bs=4096)
    cmds1 = programs.read_bbts(path1)
    assert len(cmds1) == 16 + 64 and all(c["type"] == programs.APPLY for c in cmds1)  # k = 1: no reduce, no delete
    assert [seeds1 for seeds1 in (c["params"][4] for c in cmds1[:8])] == [1000 + i for i in range(8)]


def test_ffnn_program_round_trip(tmp_path):
    path = str(tmp_path / "ffnn.bbts")
    info, inputs = programs.ffnn_bbts(path, batch=512, d_in=256, h1=256, h2=256, classes=128, bs=128, seed=3,
                                      dtype="bf16", split_a1=True)
    cmds = programs.read_bbts(path)
    uds = collections.Counter(c["ud"] for c in cmds)
    assert uds["matrix_softmax_ce"] == 512 // 128 and uds["matrix_relu_split"] == (512 // 128) * (256 // 128)
    assert uds["matrix_mult"] > 0 and uds["matrix_add"] > 0 and cmds[-1]["type"] == programs.DELETE
    # inputs are held by the node, not created by the program
    produced = {t for c in cmds for t, _ in c["outputs"]}
    assert not produced & set(inputs)
    read = {t for c in cmds for t, _ in c["inputs"]}
    assert set(inputs) <= read
    assert all("fill" in v or v["data"] is not None for v in inputs.values())
    programs.write_bbts(str(tmp_path / "again.bbts"), cmds)
    assert open(str(tmp_path / "again.bbts"), "rb").read() == open(path, "rb").read()


def test_cpmm_seed_formula_is_shared():
    """bench.py restates the cpmm input seeds on the host (its reference arm
    must not load the library); they must equal workloads.cpmm_seeds and the
    seeds cpmm_bbts writes into its uniform APPLYs."""
    import os
    import sys
    import tempfile
    from bbts_b200 import workloads
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    sa, sb = workloads.cpmm_seeds(bench.CPMM_SEED, bench.GRID, bench.GRID)
    assert sa == [bench.CPMM_SEED + i for i in range(bench.GRID)]
    assert sb == [bench.CPMM_SEED + 1000 + j for j in range(bench.GRID)]
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "c.bbts")
        programs.cpmm_bbts(path, rows=bench.GRID, cols=bench.GRID, bs=64, seed=bench.CPMM_SEED)
        seeds = [c["params"][4] for c in programs.read_bbts(path) if c["ud"] == "uniform"]
    assert seeds == sa + sb
