"""B200-native Rayleigh-Chebyshev eigensolver (lowest eigenpairs of large sparse Hermitian operators).

The compute path is librcb200.so (hand-written sm_100a CUDA kernels behind a C ABI,
include/rc_b200.h). This package is the Python host layer over it:
  runtime   contexts, operators (CSR, stencil, callback), rc_solve and the kernel-level calls
  problems  the seeded synthetic operators of the benchmark configurations
"""
from . import _capi  # noqa: F401
from . import problems  # noqa: F401
from . import runtime  # noqa: F401

__all__ = ["runtime", "problems"]
