"""bug_defense_b200 -- sm_100a implementation of the coupled laser-tissue epoch of
yudovsky/bug-defense (voxel Monte Carlo, bioheat stencil, boiling/char/ablation, plume).

Public names mirror the reference modules so callers can switch imports:

  simulation.voxel_mc_3d          -> bug_defense_b200.voxel_mc      (run_voxel_mc3d)
  simulation.voxel_mc_metal       -> bug_defense_b200.voxel_mc      (run_voxel_mc_metal, is_metal_available)
  simulation.voxel_thermal_metal  -> bug_defense_b200.thermal       (MetalThermalContext, run_thermal3d_substeps_metal)
  simulation.voxel_thermal_3d     -> bug_defense_b200.thermal       (VoxelThermalSolver3D)
  simulation.metal_ablation_solver-> bug_defense_b200.ablation      (MetalAblationContext)
  simulation.plume                -> bug_defense_b200.plume         (MultispectralPlumeField)
  simulation.coupled_ablation     -> bug_defense_b200.coupled       (CoupledAblationEngine)

All compute runs in libbugdef.so (CUDA, sm_100a) through the C ABI of include/bugdef.h.
"""
from ._device import is_gpu_available
from .voxel_mc import run_voxel_mc3d, run_voxel_mc_gpu, run_voxel_mc_metal
from .thermal import GpuThermalContext, MetalThermalContext, VoxelThermalSolver3D, run_thermal3d_substeps_gpu
from .ablation import GpuAblationContext, MetalAblationContext
from .plume import MultispectralPlumeField, PlumeField
from .coupled import CoupledAblationEngine, K_AIR, RHO_CP_AIR
from .phase import CHAR_STATE, compute_phase_map

is_metal_available = is_gpu_available

__all__ = [
    "is_gpu_available", "is_metal_available", "run_voxel_mc3d", "run_voxel_mc_gpu", "run_voxel_mc_metal",
    "GpuThermalContext", "MetalThermalContext", "VoxelThermalSolver3D", "run_thermal3d_substeps_gpu",
    "GpuAblationContext", "MetalAblationContext", "MultispectralPlumeField", "PlumeField",
    "CoupledAblationEngine", "K_AIR", "RHO_CP_AIR", "CHAR_STATE", "compute_phase_map",
]
