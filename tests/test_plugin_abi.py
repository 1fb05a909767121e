"""The plugin entry points against a stand-in reference node.

tests/cpp/ref_node_standin.cc restates the reference's plugin-facing classes
with the reference's member layout and defines (and exports) the node-side
member functions; it dlopen()s libbbts_b200.so RTLD_LOCAL | RTLD_NOW and calls
register_tensors / register_udfs through dlsym, as src/server/coordinator.cc:
509-532 does. The CPU test checks the registrations and the metadata
callbacks; the GPU test also runs impls on dense tensors the node allocated
itself (payload right after the 260-byte header, in managed memory).
"""
import os
import subprocess

import pytest

from conftest import ROOT

LIB = os.path.join(ROOT, "bbts_b200", "libbbts_b200.so")


def _standin(tmp_path):
    src = os.path.join(ROOT, "tests", "cpp", "ref_node_standin.cc")
    exe = os.path.join(str(tmp_path), "ref_node_standin")
    cmd = ["g++", "-std=c++17", "-O1", "-rdynamic", "-I/usr/local/cuda/include", src, "-o", exe,
           "-L/usr/local/cuda/lib64", "-lcudart", "-ldl", "-Wl,-rpath,/usr/local/cuda/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_reference_node_loads_the_plugin(tmp_path):
    r = subprocess.run([_standin(tmp_path), LIB], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "plugin boundary ok" in r.stdout


@pytest.mark.gpu
def test_reference_node_runs_impls_on_its_own_tensors(tmp_path, cuda):
    r = subprocess.run([_standin(tmp_path), LIB, "gpu"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "impls on node tensors ok" in r.stdout and "plugin boundary ok" in r.stdout
