"""Builds and runs the C++ host tests (tests/cpp) against libbbts_b200.so (no GPU needed)."""
import os
import subprocess

from conftest import ROOT


def _build_and_run(name, tmp_path):
    src = os.path.join(ROOT, "tests", "cpp", name + ".cc")
    exe = os.path.join(str(tmp_path), name)
    lib_dir = os.path.join(ROOT, "bbts_b200")
    cmd = ["g++", "-std=c++17", "-O1", "-pthread", "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(ROOT, "bbts_b200", "csrc"), "-I" + os.path.join(ROOT, "bbts_b200", "csrc", "host"),
           "-I/usr/local/cuda/include", src, "-o", exe, "-L" + lib_dir, "-l:libbbts_b200.so",
           "-Wl,-rpath," + lib_dir]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_host_layer(tmp_path):
    out = _build_and_run("test_host", tmp_path)
    assert "all host tests passed" in out
