"""B200-native fiber monodomain solver (OpenDiHu FastMonodomainSolver hot path).

The compute path is libfdm_b200.so (CUDA, sm_100a) behind the C ABI of include/fdm_b200.h; this package
is the settings harness and host-side operator API.
"""
from .solver import FastMonodomainSolver, FiberSystem, parse_settings, uniform_fibers  # noqa: F401

__all__ = ["FastMonodomainSolver", "FiberSystem", "parse_settings", "uniform_fibers"]
