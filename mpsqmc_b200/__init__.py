"""B200-native walker propagation for MPS-based projector QMC (the MPSQMC2 hot path).

The compute path is libmpsqmc_b200.so (hand-written sm_100a CUDA behind the C ABI in
include/mpsqmc_gpu.h); this package holds its ctypes binding and the host-side set-up.
"""
from . import problem
from .capi import Engine, MpsqmcError, load

__all__ = ["Engine", "MpsqmcError", "load", "problem"]
