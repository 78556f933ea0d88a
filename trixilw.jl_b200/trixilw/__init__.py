"""trixilw: B200 (sm_100a) drop-in for TrixiLW.jl's Lax-Wendroff / MDRK right-hand side (TreeMesh{2},
compressible Euler, FP64). The compute runs in libtlw.so (CUDA, C ABI in include/tlw.h); this package is
the host-side mirror of the reference's Julia interface for that path."""
from ._lib import DomainError, TlwError, lib
from .adjoint import adjoint_solve, adjoint_step, adjoint_sweep, forward_record, lw_solve, solve_dts
from .batch import LWBatch, solve_lwfr_batch
from .curved_mesh import CurvedMesh, RefinedStructuredMesh, StructuredMesh, rotate_elements, rotate_state
from .equations import (CompressibleEulerEquations2D, CompressibleNavierStokesDiffusion2D, ConstantState,
                        DensityWave, FourQuadrantRiemann, GradientVariablesConservative, IsentropicVortex,
                        initial_condition_convergence_test, source_terms_convergence_test)
from .limiters import PositivityPreservingLimiterZhangShu, density, density_pressure, pressure
from .lwfr import LWIntegrator, LWSolution, l2_linf_errors, solve_lwfr
from .mesh import RefinedTreeMesh, TreeMesh
from .unstructured_mesh import UnstructuredMesh2D
from .semidiscretization import (LW, MDRK, DGSEM, Adaptive, Adiabatic, BoundaryConditionDirichlet,
                                 BoundaryConditionNavierStokesWall, CFLBased, FluxHLL, Isothermal, NoSlip,
                                 boundary_condition_slip_wall_horizontal, boundary_condition_slip_wall_vertical,
                                 FluxLaxFriedrichs, IndicatorHennemannGassner, SemidiscretizationHyperbolic,
                                 SemidiscretizationHyperbolicParabolic,
                                 VolumeIntegralFR, VolumeIntegralFRShockCapturing, FirstOrderReconstruction, MUSCLReconstruction, MUSCLHancockReconstruction,
                                 boundary_condition_periodic, flux_hll, flux_lax_friedrichs,
                                 get_time_discretization, lw_fourier_cfl, rhs, rhs_mdrk1, rhs_mdrk2,
                                 semidiscretize, trixi2lw)

__all__ = [
    "DomainError", "TlwError", "lib", "CompressibleEulerEquations2D", "ConstantState", "DensityWave",
    "FourQuadrantRiemann", "IsentropicVortex", "initial_condition_convergence_test",
    "source_terms_convergence_test", "LWIntegrator", "LWSolution", "l2_linf_errors", "solve_lwfr",
    "TreeMesh", "LW", "MDRK", "DGSEM", "Adaptive", "BoundaryConditionDirichlet", "CFLBased", "FluxHLL",
    "FluxLaxFriedrichs", "IndicatorHennemannGassner", "SemidiscretizationHyperbolic", "VolumeIntegralFR",
    "VolumeIntegralFRShockCapturing", "FirstOrderReconstruction", "MUSCLReconstruction", "MUSCLHancockReconstruction", "boundary_condition_periodic",
    "flux_hll", "flux_lax_friedrichs", "get_time_discretization", "lw_fourier_cfl", "rhs", "rhs_mdrk1",
    "rhs_mdrk2", "semidiscretize", "trixi2lw", "LWBatch", "solve_lwfr_batch",
    "adjoint_solve", "adjoint_step", "adjoint_sweep", "forward_record", "lw_solve", "solve_dts",
    "CurvedMesh", "RefinedStructuredMesh", "StructuredMesh", "rotate_elements", "rotate_state", "RefinedTreeMesh",
    "CompressibleNavierStokesDiffusion2D", "GradientVariablesConservative", "SemidiscretizationHyperbolicParabolic",
    "PositivityPreservingLimiterZhangShu", "density", "pressure", "density_pressure",
    "boundary_condition_slip_wall_vertical", "boundary_condition_slip_wall_horizontal", "NoSlip", "Adiabatic",
    "Isothermal", "BoundaryConditionNavierStokesWall", "UnstructuredMesh2D",
]
