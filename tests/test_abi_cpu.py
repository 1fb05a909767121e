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
