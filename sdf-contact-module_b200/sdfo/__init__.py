"""sdfo: the SdfOracle hot path (SDF build, batched queries, penalty contact)
on NVIDIA B200 (sm_100a) through the libsdfo_cuda C ABI (include/sdfo.h).

Submodules:
  grid      SdfGrid -- build / query / load / save device grids
  autograd  sdf_query -- differentiable Trilinear / Tricubic queries
  contact   ContactBatch -- fused batched contact force + 6x6 pose Jacobian,
            the engine's culling and measure_pair; contact_force (autograd)
  be        BEStepper -- batched Backward-Euler contact steps
  io        SDFO 0.1.0 file format
  meshes    procedural meshes and quadrature
  workloads seeded synthetic inputs of the benchmark configurations
"""
from ._native import (CONTACT_AWARE, FIRST_ORDER, SECOND_ORDER, TRICUBIC, TRILINEAR, SdfoError,
                      library_path)
from ._native import load as load_library
from .grid import SdfGrid

__all__ = ["SdfGrid", "SdfoError", "FIRST_ORDER", "SECOND_ORDER", "TRILINEAR", "TRICUBIC",
           "CONTACT_AWARE", "library_path", "load_library"]
