"""gluedmd_b200 — B200-native (sm_100a) implementation of GLUED's per-step
enhanced-sampling hot path: CV evaluation -> MetaD / OPES bias -> chain-rule
force scatter into OpenMM's 2^32 fixed-point force buffer.

Layers:
  include/glued_b200.h     C ABI (the drop-in boundary)
  gluedmd_b200/csrc        CUDA kernels + C++ host (descriptor, plan, context, batch)
  gluedmd_b200.gluedplugin Python mirror of GLUED's SWIG module (GluedForce)
  gluedmd_b200.context     standalone System/Context harness over device buffers
"""
from ._native import GluedError, lib  # noqa: F401
from .gluedplugin import GluedForce, NativeContext  # noqa: F401

__all__ = ["GluedForce", "NativeContext", "GluedError", "lib"]
