"""EU3D B200: a device-resident, sm_100a-native replacement for the per-step
hot path of the EU3D reactive Euler solver (flux sweeps, TimeAdv update,
decode and H2 chemistry), reached through the C ABI in include/eu3d_gpu.h.

Submodules:
  readers  -- the reference's mechanism/thermo/ctrl/grid file formats
  gpu      -- ctypes binding of the C ABI (DeviceFlowfield)
  cases    -- initial/boundary set-ups of the benchmark configurations
  build    -- nvcc recipe for libeu3d_gpu.so
"""
from . import readers  # noqa: F401

__all__ = ["readers", "gpu", "cases", "build"]
