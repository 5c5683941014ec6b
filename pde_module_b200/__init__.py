"""pde_module_b200: the finite-difference hot path of PDE_Module on B200 (sm_100a).

Drop-in module API (Laplacian, Grad, Divergence, GridBoundary, ImmersedBoundary,
ForwardEuler, the element-wise and absorbing-layer operators, the Runge-Kutta
integrators and their functional forms) over torch CUDA float32 tensors, backed by
the C ABI of include/pde_b200.h in ``_native/libpde_b200.so``.
"""
from . import _lib
from .FDM import (Laplacian, Grad, Divergence, GridBoundary, ImmersedBoundary, OuterProduct, scalarVectorMult,
                  FarField, ViscousDampingLayer)
from .time_step import (ForwardEuler, HeatRollout, HeatSolver, heat_rollout, FractionalStepLDC,
                        SlabFractionalStepLDC, WaveSolver,
                        wave_rollout,
                        BatchedHeatRollout, BatchedWaveRollout, RungeKatta1, RungeKatta2,
                        WeaklyCompressibleRK2, lid_driven_cavity_wc)
from .mesh import UniformGridMesh, create_structured_field, create_structured_warp_field

__all__ = ["Laplacian", "Grad", "Divergence", "GridBoundary", "ImmersedBoundary", "OuterProduct", "scalarVectorMult",
           "FarField", "ViscousDampingLayer", "ForwardEuler", "RungeKatta1", "RungeKatta2", "WeaklyCompressibleRK2",
           "lid_driven_cavity_wc", "HeatRollout",
           "FractionalStepLDC", "SlabFractionalStepLDC",
           "HeatSolver", "heat_rollout", "WaveSolver", "wave_rollout", "BatchedHeatRollout", "BatchedWaveRollout",
           "UniformGridMesh", "create_structured_field", "create_structured_warp_field"]
