"""dgm_in_rust_b200 -- B200-native (sm_100a) DG residual + SSP-RK3 time step of DGM_in_rust.

The hot path (volume integral, HLLC edge flux, boundary fluxes, inverse mass, KXRCF/WENO
limiter, SSP-RK3 stages, CFL time step, time-march loop) runs in hand-written CUDA kernels
behind the C ABI in include/dgm_b200.h.  This package is the Python host side: tables, mesh
processing and the reference-shaped Solver / SpatialDisc / TemperalDisc classes.
"""
from ._native import DgmError
from .basis_function import DubinerBasis, GaussPoints, default_rules
from .mesh import GmshParser, Mesh, RawMesh, freestream_quantity, naca0012_ogrid, process_mesh, write_gmsh
from .solver import (Batch, FlowParameters, InitialSolution, MeshParameters, Solver, SolverParameters, SpatialDisc,
                     TemperalDisc, build_solver, forces_to_coefficients, initial_state, reference_cfl, slot_capacity)

__all__ = [
    "DgmError", "DubinerBasis", "GaussPoints", "default_rules", "GmshParser", "Mesh", "RawMesh",
    "freestream_quantity", "naca0012_ogrid", "process_mesh", "write_gmsh", "FlowParameters", "InitialSolution",
    "MeshParameters", "Solver", "SolverParameters", "SpatialDisc", "TemperalDisc", "build_solver",
    "initial_state", "reference_cfl", "Batch", "forces_to_coefficients", "slot_capacity",
]
