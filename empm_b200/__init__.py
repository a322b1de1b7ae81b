"""empm_b200 — B200-native (sm_100a) MLS-MPM substep for EMPM.

Drop-in for the Warp simulator of phys_sim/diff_simulator/warp_mpm: the
classes below keep the reference's names and call signatures; the substep
runs in hand-written CUDA kernels (libempm_b200.so, C ABI in
include/empm_b200.h). There is no CPU fallback.
"""
from .mpm_data_structure import (Dirichlet_collider, GridCollider, Impulse_modifier, MPMModelStruct, MPMStateStruct,
                                 ParticleVelocityModifier)
from .mpm_solver_diff import MPMWARPDiff
from .interface import (MPMDifferentiableSimulation, MPMDifferentiableSimulationClean,
                        MPMDifferentiableSimulationTrail, MPMDifferentiableSimulationWCheckpoint)
from .warp_mpm_wrapper import WarpMPMWrapper, material_gallery

__all__ = [
    "Dirichlet_collider", "GridCollider", "Impulse_modifier", "MPMModelStruct", "MPMStateStruct",
    "ParticleVelocityModifier", "MPMWARPDiff", "MPMDifferentiableSimulation", "MPMDifferentiableSimulationClean",
    "MPMDifferentiableSimulationTrail", "MPMDifferentiableSimulationWCheckpoint", "WarpMPMWrapper",
    "material_gallery",
]
