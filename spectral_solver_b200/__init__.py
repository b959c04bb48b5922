"""B200-native pseudo-spectral Taylor-Green RK3 step (drop-in backend for ovankerm/Spectral_solver).

The product is native: ``libsns_b200.so`` (sm_100a CUDA kernels behind the C ABI in
``include/sns_b200.h``) and ``libspectral_b200.so`` (the reference's C++ classes over that
ABI).  This Python package only binds the C ABI for tests and the benchmark.
"""
from ._lib import Batch, Fft3D, Server, Solver, SnsError, load  # noqa: F401

__all__ = ["Batch", "Fft3D", "Server", "Solver", "SnsError", "load"]
