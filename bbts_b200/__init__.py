"""bbts_b200: B200 (sm_100a) executor for BarbaTOS's tensor-block hot path.

The compute lives in libbbts_b200.so (CUDA kernels + C++ runtime behind the C
ABI of include/bbts_b200.h); this package is the Python view of that ABI used
by tests and benchmarks. Importing it fails if the native library is missing.
"""
from ._lib import lib, check, last_error, BbxError, TcProblem  # noqa: F401
from . import ops  # noqa: F401

__all__ = ["lib", "check", "last_error", "BbxError", "TcProblem", "ops"]
