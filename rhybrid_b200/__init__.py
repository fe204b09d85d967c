"""rhybrid_b200: B200-native (sm_100a) hot path of the RHybrid hybrid-PIC code.

The package holds the CUDA library (csrc/ -> librhgpu.so, C ABI in
include/rhgpu.h), its ctypes binding (abi), the host-side configuration and
initial state (config) and the Corsair-style driver (simulation).
"""
from . import abi, config  # noqa: F401

__all__ = ["abi", "config"]
