"""The C-ABI library loads and exports every symbol the public header declares (no GPU needed)."""
import ctypes
import os
import subprocess

import pytest

from conftest import ROOT


def test_library_exports_every_declared_symbol():
    from bbts_b200 import _lib
    names = _lib.exported_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(_lib.lib, n)]
    assert missing == []


def test_header_compiles_as_c():
    hdr = os.path.join(ROOT, "include", "bbts_b200.h")
    r = subprocess.run(["gcc", "-fsyntax-only", "-x", "c", "-std=c99", hdr], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_version_and_error_channel():
    from bbts_b200 import lib, last_error
    assert b"sm_100a" in lib.bbx_version()
    # argument validation happens before any CUDA call
    rc = lib.bbx_reduce_f32(None, 0, None, 10, 1, None)
    assert rc == -1
    assert "reduce" in last_error()


def test_no_cpu_fallback_symbols():
    # the product library must not contain the oracle
    from bbts_b200 import _lib
    for name in ("oracle_add", "oracle_matmul_f64", "oracle_sgemm_mt"):
        assert not hasattr(_lib.lib, name)


def test_tile_recording_api_without_a_gpu():
    # recording state and the sample buffer are host-side: on, no samples yet
    # (no DAG was built), off again
    from bbts_b200 import runtime
    runtime.tile_record(True)
    f, t = runtime.tile_samples()
    assert f.shape == (0, 12) and t.shape == (0,)
    runtime.tile_record(False)
    assert runtime.AUTOTUNE == -1 and runtime.LEARNED_TILES == -2


def test_host_arguments_rejected_before_cuda():
    # these entry points validate their arguments on the host and return an
    # error code with a message, without touching a device
    from bbts_b200 import lib, last_error
    assert lib.bbx_relu_split(None, None, None, 10, None) == -1
    assert "relu_split" in last_error()
    assert lib.bbx_stream_plan_bulk(None) == -1
    assert "stream plan" in last_error()
