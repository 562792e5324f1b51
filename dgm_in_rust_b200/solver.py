"""Host-side mirror of DGM_in_rust's solver objects, backed by the CUDA library.

Names, argument meaning and error behaviour follow the reference:

* :class:`SpatialDisc` -- ``compute_residuals(residuals, solutions)`` (src/spatial_disc.rs:27)
  and ``apply_limiter(solutions)`` (src/spatial_disc/limiter.rs:7);
* :class:`TemperalDisc` -- ``rk3(spatial_disc, residuals, solutions, time_step)``
  (src/temporal_disc/rk3.rs:7), ``time_march(spatial_disc, residuals, solutions)``
  (src/temporal_disc.rs:21), ``compute_time_step(solutions)`` (src/temporal_disc.rs:58);
* :class:`Solver` -- ``set_initial_solution()`` (src/solver.rs:45) and ``solve()``
  (src/solver.rs:80).

States are numpy float64 arrays shaped like the reference's ``Array<f64, Ix3>``
``[element][variable][basis]``.  Where the reference panics (negative density/pressure in
HLLC, an element with three boundary edges in WENO) these raise :class:`DgmError`.
"""
from __future__ import annotations

import ctypes
import dataclasses
import functools
import math

import numpy as np

from . import _native
from ._native import DgmError
from .basis_function import DubinerBasis, GaussPoints, default_rules
from .mesh import Mesh

__all__ = [
    "SolverParameters",
    "FlowParameters",
    "MeshParameters",
    "InitialSolution",
    "SpatialDisc",
    "TemperalDisc",
    "Solver",
    "reference_cfl",
    "initial_state",
    "Batch",
    "slot_capacity",
    "forces_to_coefficients",
]


def reference_cfl(order: int) -> float:
    """CFL formula of initialization.rs:29-33 (overrides the JSON value in the reference)."""
    p = float(order)
    return 1.0 * 1.0 / ((2.0 * p + 1.0) * (1.0 + 4.0 / (p + 2.0) ** 2.0))


@dataclasses.dataclass
class SolverParameters:
    """SolverParameters (src/solver.rs:10-20)."""

    cfl: float
    final_time: float
    final_step: int
    order_of_polynomials: int = 2
    number_of_cell_gp: int = 6
    number_of_edge_gp: int = 3
    number_of_equations: int = 4
    inviscid_flux_scheme: str = "hllc"

    @property
    def number_of_basis_functions(self) -> int:
        p = self.order_of_polynomials
        return (p + 1) * (p + 2) // 2

    def __post_init__(self):
        if self.inviscid_flux_scheme.lower() != "hllc":
            raise ValueError("Inviscid flux scheme not implemented")
        if self.number_of_equations != 4:
            raise ValueError("the Euler system has 4 equations")


@dataclasses.dataclass
class FlowParameters:
    """FlowParameters (src/solver.rs:27-31)."""

    hcr: float = 1.4
    gas_constant: float = 287.0
    prandtl_number: float = 0.72


@dataclasses.dataclass
class MeshParameters:
    """MeshParameters (src/solver.rs:21-26)."""

    number_of_elements: int
    number_of_edges: int
    number_of_vertices: int
    number_of_patches: int

    @staticmethod
    def of(mesh: Mesh) -> "MeshParameters":
        return MeshParameters(mesh.n_elements, mesh.n_edges, int(mesh.vertices.shape[0]),
                              int(mesh.patch_type.shape[0]))


@dataclasses.dataclass
class InitialSolution:
    """InitialSolution (src/io/initial_solution_parser.rs:4-10)."""

    density: float
    angle_of_attack: float
    mach_number: float
    pressure: float


def initial_state(mesh: Mesh, basis: DubinerBasis, gauss_points: GaussPoints, hcr: float,
                  init: InitialSolution) -> np.ndarray:
    """L2 projection of a uniform state onto the basis (Solver::set_initial_solution,
    src/solver.rs:45-79), same summation order as the reference."""
    rho, p = init.density, init.pressure
    c = math.sqrt(hcr * p / rho)
    a = init.angle_of_attack * (math.pi / 180.0)
    xv = init.mach_number * math.cos(a) * c
    yv = init.mach_number * math.sin(a) * c
    te = p / (hcr - 1.0) + 0.5 * rho * (xv * xv + yv * yv)
    q = np.array([rho, rho * xv, rho * yv, te])
    J = mesh.elem_jacob_det
    nb = basis.dof
    U = np.zeros((mesh.n_elements, 4, nb))
    for g in range(gauss_points.cell_gp_number):
        U += ((0.5 * J)[:, None, None] * gauss_points.cell_weights[g] * q[None, :, None]
              * basis.phis_cell_gps[g][None, None, :])
    U /= basis.mass_mat_diag[None, None, :] * 0.5 * J[:, None, None]
    return U


EDGE_FORMS = ("point", "pair", "staged", "point_r64")  # dgm_set_edge_variant's 0, 1, 2, 3


def _launch_config(L, ctx) -> dict:
    cfg = (ctypes.c_int32 * 3)()
    L.dgm_get_launch_config(ctx, cfg)
    staged, queue = ctypes.c_int32(0), ctypes.c_int32(0)
    L.dgm_get_limiter_variant(ctx, ctypes.byref(staged), None)
    L.dgm_get_limiter_schedule(ctx, ctypes.byref(queue), None)
    return {"edge_threads": cfg[0], "edge_blocks": cfg[1], "element_threads": cfg[2],
            "limiter_detector": "staged" if staged.value else "compact",
            "limiter_schedule": "queue" if queue.value else "barrier",
            "edge_form": EDGE_FORMS[L.dgm_get_edge_variant(ctx)],
            "limiter_grid": "one_per_sm" if L.dgm_get_limiter_grid(ctx) == 1 else "full"}


def _autotune(L, ctx, repeats: int) -> dict:
    best = (ctypes.c_double * 2)()
    st = L.dgm_autotune(ctx, int(repeats), best)
    if st != 0:
        raise DgmError(st, int(L.dgm_error_location(ctx)), "autotune")
    out = _launch_config(L, ctx)
    lim, sched = (ctypes.c_double * 2)(), (ctypes.c_double * 2)()
    L.dgm_get_limiter_variant(ctx, None, lim)
    L.dgm_get_limiter_schedule(ctx, None, sched)
    out.update({"edge_us": best[0], "element_us": best[1], "limiter_compact_us": lim[0], "limiter_staged_us": lim[1],
                "limiter_barrier_us": sched[0], "limiter_queue_us": sched[1]})
    return out


def _check_state(a: np.ndarray, ne: int, nb: int, name: str) -> None:
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or a.shape != (ne, 4, nb) or not a.flags.c_contiguous:
        raise ValueError(f"{name} must be a C-contiguous float64 array of shape ({ne}, 4, {nb})")


def _mesh_desc(m: Mesh, keep: list) -> "_native.MeshDesc":
    def f64(a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        return _native.dptr(a)

    def i64(a):
        a = np.ascontiguousarray(a, dtype=np.int64)
        keep.append(a)
        return _native.iptr(a)

    def i32(a):
        a = np.ascontiguousarray(a, dtype=np.int32)
        keep.append(a)
        return _native.i32ptr(a)

    return _native.MeshDesc(
        n_vertices=m.vertices.shape[0], n_elements=m.n_elements, n_edges=m.n_edges,
        n_patches=m.patch_type.shape[0], vertex_xy=f64(m.vertices), elem_vertices=i64(m.elem_vertices),
        elem_edges=i64(m.elem_edges), elem_neighbours=i64(m.elem_neighbours),
        elem_jacob_det=f64(m.elem_jacob_det), elem_circumradius=f64(m.elem_circumradius),
        elem_minimum_height=f64(m.elem_minimum_height), edge_elements=i64(m.edge_elements),
        edge_vertices=i64(m.edge_vertices), edge_in_cell=i64(m.edge_in_cell),
        edge_jacob_det=f64(m.edge_jacob_det), edge_normal=f64(m.edge_normal), edge_patch=i64(m.edge_patch),
        patch_type=i32(m.patch_type), patch_quantity=f64(m.patch_quantity),
        n_internal_edges=m.internal_edge_indices.shape[0], internal_edges=i64(m.internal_edge_indices),
        n_boundary_elements=m.boundary_element_indices.shape[0],
        boundary_elements=i64(m.boundary_element_indices))


def _tables_desc(basis: DubinerBasis, g: GaussPoints, keep: list) -> "_native.TablesDesc":
    def f64(a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        return _native.dptr(a)

    return _native.TablesDesc(
        order=basis.order, n_basis=basis.dof, n_cell_gp=g.cell_gp_number, n_edge_gp=g.edge_gp_number,
        n_deriv_keys=basis.nkeys, _pad=0, cell_weights=f64(g.cell_weights), edge_weights=f64(g.edge_weights),
        phi_cell=f64(basis.phis_cell_gps), phi_edge=f64(basis.phis_edge_gps),
        dphi_cell_ref=f64(basis.dphis_cell_gps), mass_diag=f64(basis.mass_mat_diag))


# fp64: the reference's arithmetic.  fp32: FP32 state, contractions, fluxes and stage updates
# (limiter, HLLC positivity checks, time step and diagnostics in FP64).  tf32 / tf32x3: as fp32,
# with the element pass's two basis contractions on the tensor cores (TF32 operands, FP32
# accumulation; tf32x3 splits each operand into a TF32 head and tail for FP32-level products).
# fp32_compute: FP64 state with the contractions, fluxes and residuals in FP32 (the stage
# combinations, limiter, positivity checks, time step and diagnostics in FP64).
PRECISIONS = {"fp64": 0, "fp32": 1, "tf32": 2, "tf32x3": 3, "fp32_compute": 4}


class SpatialDisc:
    """GPU-resident SpatialDisc (src/spatial_disc.rs:17-25).  Owns the device context.

    ``precision="fp64"`` reproduces the reference's arithmetic; ``"fp32"`` keeps the state and
    the bulk arithmetic in FP32 with the limiter, positivity checks and time step in FP64.
    """

    def __init__(self, mesh: Mesh, basis: DubinerBasis, gauss_points: GaussPoints,
                 flow_param: FlowParameters, mesh_param: MeshParameters, solver_param: SolverParameters,
                 limiter: bool = True, device: int = 0, precision: str = "fp64"):
        self.mesh = mesh
        self.basis = basis
        self.gauss_points = gauss_points
        self.flow_param = flow_param
        self.mesh_param = mesh_param
        self.solver_param = solver_param
        self.limiter = bool(limiter)
        self.precision = precision
        L = _native.lib()
        keep: list = []
        md = _mesh_desc(mesh, keep)
        td = _tables_desc(basis, gauss_points, keep)
        pr = _native.Params(hcr=flow_param.hcr, cfl=solver_param.cfl, final_time=solver_param.final_time,
                            final_step=solver_param.final_step, limiter=1 if limiter else 0, device=device,
                            precision=PRECISIONS[precision], _reserved=0)
        status = ctypes.c_int32(0)
        ctx = L.dgm_create(ctypes.byref(md), ctypes.byref(td), ctypes.byref(pr), ctypes.byref(status))
        if not ctx:
            raise DgmError(status.value, what="dgm_create")
        self._ctx = ctypes.c_void_p(ctx)
        self._lib = L
        self.ne = mesh.n_elements
        self.nb = basis.dof

    # ---- plumbing ----
    def _check(self, st: int, what: str) -> None:
        if st != 0:
            raise DgmError(st, int(self._lib.dgm_error_location(self._ctx)), what)

    @property
    def ctx(self):
        return self._ctx

    def close(self) -> None:
        if getattr(self, "_ctx", None):
            self._lib.dgm_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def new_state(self) -> np.ndarray:
        return np.zeros((self.ne, 4, self.nb))

    # ---- reference API ----
    def compute_residuals(self, residuals: np.ndarray, solutions: np.ndarray) -> None:
        """residuals = (residuals + volume + edge + boundary terms) / mass (spatial_disc.rs:27-39)."""
        _check_state(residuals, self.ne, self.nb, "residuals")
        _check_state(solutions, self.ne, self.nb, "solutions")
        self._check(self._lib.dgm_compute_residuals(self._ctx, _native.dptr(residuals), _native.dptr(solutions)),
                    "compute_residuals")

    def apply_limiter(self, solutions: np.ndarray) -> int:
        """KXRCF + WENO in place, reference element order (limiter.rs:7, weno.rs:86-269).
        Returns the number of limited cells."""
        _check_state(solutions, self.ne, self.nb, "solutions")
        n = ctypes.c_int64(0)
        self._check(self._lib.dgm_apply_limiter(self._ctx, _native.dptr(solutions), ctypes.byref(n)), "apply_limiter")
        return int(n.value)

    def cell_fields(self) -> np.ndarray:
        """[ne, 4] density, x velocity, y velocity, pressure of the resident state's mode-0
        coefficients, computed on the device with write_to_vtk's expressions
        (src/io/write_results.rs:33-61)."""
        out = np.zeros((self.ne, 4))
        self._check(self._lib.dgm_cell_fields(self._ctx, 0, _native.dptr(out)), "cell_fields")
        return out

    def diagnostics(self, use_residual: bool = False) -> np.ndarray:
        """[8]: integrals of rho, rho u, rho v, rho E; wall force Fx, Fy; sum of squared density
        residual coefficients (last residual written); element count.  FP64, deterministic."""
        out = np.zeros((1, 8))
        self._check(self._lib.dgm_diagnostics(self._ctx, 1 if use_residual else 0, _native.dptr(out)),
                    "diagnostics")
        return out[0]

    def enqueue_diagnostics(self, use_residual: bool = False) -> None:
        """Enqueue :meth:`diagnostics` behind the work on the stream, into a pinned host buffer."""
        self._check(self._lib.dgm_enqueue_diagnostics(self._ctx, 1 if use_residual else 0), "enqueue_diagnostics")

    def collected_diagnostics(self) -> np.ndarray:
        """The diagnostics of the last :meth:`enqueue_diagnostics` (waits for that copy only)."""
        out = np.zeros((1, 8))
        self._check(self._lib.dgm_collected_diagnostics(self._ctx, _native.dptr(out)), "collected_diagnostics")
        return out[0]

    def limiter_stats(self) -> tuple[int, int]:
        t, w = ctypes.c_int64(0), ctypes.c_int32(0)
        self._lib.dgm_limiter_stats(self._ctx, ctypes.byref(t), ctypes.byref(w))
        return int(t.value), int(w.value)

    # ---- launch configuration (no counterpart in the reference) ----
    @property
    def launch_config(self) -> dict:
        return _launch_config(self._lib, self._ctx)

    def set_launch_config(self, edge_threads: int, edge_blocks: int, element_threads: int) -> None:
        self._check(self._lib.dgm_set_launch_config(self._ctx, int(edge_threads), int(edge_blocks),
                                                    int(element_threads)), "set_launch_config")

    def set_edge_form(self, form) -> None:
        """Pick the edge pass's form: "point" (a thread per (slot, Gauss point)), "pair" (a lane pair
        per edge slot, each side's state loaded once), "staged" (a lane per point, the slots'
        records copied to shared memory first) or "point_r64" (the point form compiled for 64
        registers); all give the same fluxes.  A bool picks "pair" (True) or "point" (False)."""
        if isinstance(form, bool):
            form = "pair" if form else "point"
        if form not in EDGE_FORMS:
            raise ValueError(f"edge form must be one of {EDGE_FORMS}")
        self._check(self._lib.dgm_set_edge_variant(self._ctx, EDGE_FORMS.index(form)), "set_edge_form")

    def set_viscous(self, enable: bool = True, prandtl_number: float = 0.72, gas_constant: float = 287.0) -> None:
        """Evaluate the Navier-Stokes residual (BR2 lifting) instead of the Euler one: the
        reference's integrate_over_cell_ns / integrate_over_edges_ns / apply_bc_ns
        (spatial_disc.rs:70-160,212-348, boundary_condition.rs:121-413), which its compute_residuals
        keeps disabled (spatial_disc.rs:34-36).  FlowParameters::prandtl_number and gas_constant
        (parameters.json).  FP64 contexts only."""
        table = np.ascontiguousarray(self.basis.dphis_edge_gps, dtype=np.float64)
        self._check(self._lib.dgm_set_viscous(self._ctx, 1 if enable else 0, float(prandtl_number),
                                              float(gas_constant), _native.dptr(table)), "set_viscous")

    @property
    def viscous(self) -> bool:
        return bool(self._lib.dgm_get_viscous(self._ctx) == 1)

    def set_limiter_grid(self, one_per_sm: bool) -> None:
        """Run the limiter's cooperative wave kernel on one block per SM (cheaper grid barriers)
        or on every co-resident block (more warps for the reconstructions); same results."""
        self._check(self._lib.dgm_set_limiter_grid(self._ctx, 1 if one_per_sm else 0), "set_limiter_grid")

    def set_limiter_detector(self, staged: bool) -> None:
        """Pick the limiter's KXRCF detector form: staged loads (fewer memory round trips, more
        registers) or compact; both give the same flags.  The autotuner picks one per context."""
        self._check(self._lib.dgm_set_limiter_variant(self._ctx, 1 if staged else 0), "set_limiter_detector")

    def set_limiter_schedule(self, queue: bool) -> None:
        """Pick the limiter's schedule: a grid barrier between each wave's scan and its
        reconstructions, or a queue that lets finished scanners reconstruct while others still
        scan; both give bitwise identical results.  The autotuner picks one per context."""
        self._check(self._lib.dgm_set_limiter_schedule(self._ctx, 1 if queue else 0), "set_limiter_schedule")

    def autotune(self, repeats: int = 20) -> dict:
        """Time the candidate edge/element launch configurations and the limiter's detector forms
        and schedules on the resident state and keep the fastest (a state must have been uploaded).
        Returns the chosen configuration."""
        return _autotune(self._lib, self._ctx, repeats)


class TemperalDisc:
    """TemperalDisc (src/temporal_disc.rs:8-93): SSP-RK3 and the time-march loop on the GPU."""

    def __init__(self, spatial_disc: SpatialDisc):
        self._sd = spatial_disc
        self.solver_param = spatial_disc.solver_param

    @property
    def current_time(self) -> float:
        t, s = ctypes.c_double(0.0), ctypes.c_int64(0)
        self._sd._lib.dgm_get_clock(self._sd._ctx, ctypes.byref(t), ctypes.byref(s))
        return float(t.value)

    @property
    def current_step(self) -> int:
        t, s = ctypes.c_double(0.0), ctypes.c_int64(0)
        self._sd._lib.dgm_get_clock(self._sd._ctx, ctypes.byref(t), ctypes.byref(s))
        return int(s.value)

    def set_limits(self, final_time: float, final_step: int) -> None:
        """SolverParameters::final_time / final_step for the next time_march / advance."""
        self.solver_param.final_time = float(final_time)
        self.solver_param.final_step = int(final_step)
        self._sd._check(self._sd._lib.dgm_set_limits(self._sd._ctx, float(final_time), int(final_step)), "set_limits")

    def set_clock(self, current_time: float, current_step: int) -> None:
        self._sd._check(self._sd._lib.dgm_set_clock(self._sd._ctx, float(current_time), int(current_step)),
                        "set_clock")

    def compute_time_step(self, solutions: np.ndarray) -> float:
        _check_state(solutions, self._sd.ne, self._sd.nb, "solutions")
        dt = ctypes.c_double(0.0)
        self._sd._check(self._sd._lib.dgm_compute_time_step(self._sd._ctx, _native.dptr(solutions), ctypes.byref(dt)),
                        "compute_time_step")
        return float(dt.value)

    def rk3(self, spatial_disc: SpatialDisc, residuals: np.ndarray, solutions: np.ndarray, time_step: float) -> None:
        sd = spatial_disc
        _check_state(residuals, sd.ne, sd.nb, "residuals")
        _check_state(solutions, sd.ne, sd.nb, "solutions")
        sd._check(sd._lib.dgm_rk3(sd._ctx, _native.dptr(residuals), _native.dptr(solutions), float(time_step)), "rk3")

    def time_march(self, spatial_disc: SpatialDisc, residuals: np.ndarray, solutions: np.ndarray) -> None:
        sd = spatial_disc
        _check_state(residuals, sd.ne, sd.nb, "residuals")
        _check_state(solutions, sd.ne, sd.nb, "solutions")
        sd._check(sd._lib.dgm_time_march(sd._ctx, _native.dptr(residuals), _native.dptr(solutions)), "time_march")

    # ---- device-resident path ----
    def upload(self, solutions: np.ndarray) -> None:
        self._sd._check(self._sd._lib.dgm_upload_solutions(self._sd._ctx, _native.dptr(solutions)), "upload")

    def download(self, solutions: np.ndarray) -> None:
        self._sd._check(self._sd._lib.dgm_download_solutions(self._sd._ctx, _native.dptr(solutions)), "download")

    def set_initial_on_device(self, initial: "InitialSolution") -> None:
        """Solver::set_initial_solution (solver.rs:45-79) computed on the device into the resident
        state; bit-identical to :func:`initial_state` followed by :meth:`upload`."""
        self._sd._check(self._sd._lib.dgm_set_initial_solution(
            self._sd._ctx, float(initial.density), float(initial.angle_of_attack), float(initial.mach_number),
            float(initial.pressure)), "set_initial_solution")

    def advance(self, n_steps: int, with_residual: bool = False) -> None:
        f = self._sd._lib.dgm_advance_with_residual if with_residual else self._sd._lib.dgm_advance
        self._sd._check(f(self._sd._ctx, int(n_steps)), "advance")

    def synchronize(self) -> None:
        self._sd._check(self._sd._lib.dgm_synchronize(self._sd._ctx), "synchronize")

    def query(self) -> bool:
        """True once the enqueued steps have finished (raising their error, if any); False while
        they are still running.  Does not block."""
        st = int(self._sd._lib.dgm_query(self._sd._ctx))
        if st == _native.DGM_NOT_READY:
            return False
        self._sd._check(st, "query")
        return True


class Solver:
    """Solver (src/solver.rs:32-82): owns residuals/solutions and drives the time march."""

    def __init__(self, mesh: Mesh, basis: DubinerBasis, gauss_points: GaussPoints, flow_param: FlowParameters,
                 solver_param: SolverParameters, limiter: bool = True, device: int = 0, precision: str = "fp64"):
        self.mesh = mesh
        self.basis = basis
        self.gauss_points = gauss_points
        self.flow_param = flow_param
        self.solver_param = solver_param
        self.mesh_param = MeshParameters.of(mesh)
        self.spatial_disc = SpatialDisc(mesh, basis, gauss_points, flow_param, self.mesh_param, solver_param,
                                        limiter=limiter, device=device, precision=precision)
        self.temporal_disc = TemperalDisc(self.spatial_disc)
        self.residuals = self.spatial_disc.new_state()
        self.solutions = self.spatial_disc.new_state()

    def set_initial_solution(self, initial: InitialSolution) -> None:
        self.solutions[...] = initial_state(self.mesh, self.basis, self.gauss_points, self.flow_param.hcr, initial)

    def solve(self) -> None:
        self.temporal_disc.time_march(self.spatial_disc, self.residuals, self.solutions)

    def write_results(self, root: str = "outputfiles/solutions") -> str:
        """write_to_vtk after the time loop (temporal_disc.rs:56, write_results.rs:8-93): the
        resident state's cell fields, computed on the device, to root/step=<current_step>.vtk."""
        from .output import solution_path, write_to_vtk
        return write_to_vtk(solution_path(self.temporal_disc.current_step, root), self.mesh,
                            self.spatial_disc.cell_fields())

    def close(self) -> None:
        self.spatial_disc.close()


@functools.lru_cache(maxsize=None)
def default_tables(order: int):
    """(GaussPoints, DubinerBasis) of ``order`` with the default rules, built once per process
    (the tables are read-only once built; p = 3 takes ~0.1 s to expand)."""
    nq, ng = default_rules(order)
    g = GaussPoints(nq, ng)
    return g, DubinerBasis(order, g)


def build_solver(mesh: Mesh, order: int, hcr: float, cfl: float, final_time: float, final_step: int,
                 limiter: bool = True, device: int = 0, precision: str = "fp64") -> Solver:
    """Convenience: tables for ``order`` with the default rules, then a Solver."""
    nq, ng = default_rules(order)
    g, b = default_tables(order)
    sp = SolverParameters(cfl=cfl, final_time=final_time, final_step=final_step, order_of_polynomials=order,
                          number_of_cell_gp=nq, number_of_edge_gp=ng)
    return Solver(mesh, b, g, FlowParameters(hcr=hcr), sp, limiter=limiter, device=device, precision=precision)


def forces_to_coefficients(fx: float, fy: float, aoa_deg: float, rho: float, speed: float, chord: float = 1.0):
    """Lift and drag coefficients from the pressure force on the body (wind axes at ``aoa_deg``)."""
    a = aoa_deg * (math.pi / 180.0)
    q = 0.5 * rho * speed * speed * chord
    lift = -fx * math.sin(a) + fy * math.cos(a)
    drag = fx * math.cos(a) + fy * math.sin(a)
    return lift / q, drag / q


def slot_capacity(mesh) -> tuple:
    """The (elements, internal edges, boundary edges, patches) counts of a processed mesh: the
    least capacity of a batch slot that takes it."""
    return (int(mesh.n_elements), int(len(mesh.internal_edge_indices)),
            int(np.count_nonzero(mesh.edge_elements[:, 1] == -1)), int(len(mesh.patch_type)))


class Batch:
    """Many independent meshes advanced together: one launch per kernel of a step covers all of
    them (a disconnected union mesh on the device), each with its own time step, clock, loop
    bounds and status.  All share one polynomial order, hcr, precision and limiter setting.
    No counterpart in the reference (one mesh per run)."""

    def __init__(self, meshes: list, order, hcr: float, cfls, final_times, final_steps,
                 limiter: bool = True, device: int = 0, precision: str = "fp64", capacities=None):
        """``order``: one polynomial order for every mesh, or a list with each mesh's order -- with
        more than one order the context is a mixed batch (dgm_create_mixed: every kernel of a step
        is one launch over all orders; FP64 or FP32).  ``capacities`` (optional): per instance a
        (elements, internal edges, boundary edges, patches) room at least the mesh's, so that the
        slot can later take a larger mesh (:meth:`replace`); see :func:`slot_capacity`."""
        self.meshes = list(meshes)
        n = len(self.meshes)
        self.orders = [int(order)] * n if np.isscalar(order) else [int(p) for p in order]
        if len(self.orders) != n:
            raise ValueError("one order per mesh")
        self.tables = {p: default_tables(p) for p in sorted(set(self.orders))}
        self.mixed = len(self.tables) > 1
        self.gauss_points, self.basis = self.tables[self.orders[0]]
        keep: list = []
        mds = (_native.MeshDesc * n)(*[_mesh_desc(m, keep) for m in self.meshes])
        prs = (_native.Params * n)(*[
            _native.Params(hcr=hcr, cfl=float(cfls[i]), final_time=float(final_times[i]),
                           final_step=int(final_steps[i]), limiter=1 if limiter else 0, device=device,
                           precision=PRECISIONS[precision], _reserved=0) for i in range(n)])
        caps = None
        if capacities is not None:
            caps = (_native.SlotCapacity * n)(*[_native.SlotCapacity(*[int(x) for x in cap]) for cap in capacities])
        L = _native.lib()
        status = ctypes.c_int32(0)
        if self.mixed:
            tds = (_native.TablesDesc * 3)()
            for p, (g, b) in self.tables.items():
                tds[p - 1] = _tables_desc(b, g, keep)
            orders = (ctypes.c_int32 * n)(*self.orders)
            ctx = L.dgm_create_mixed(n, mds, orders, tds, prs, caps, ctypes.byref(status))
        else:
            td = _tables_desc(self.basis, self.gauss_points, keep)
            if caps is None:
                ctx = L.dgm_create_batch(n, mds, ctypes.byref(td), prs, ctypes.byref(status))
            else:
                ctx = L.dgm_create_batch_slots(n, mds, caps, ctypes.byref(td), prs, ctypes.byref(status))
        if not ctx:
            raise DgmError(status.value, what="dgm_create_mixed" if self.mixed else "dgm_create_batch")
        self._ctx = ctypes.c_void_p(ctx)
        self._lib = L
        self.n = n
        self.nb = self.basis.dof
        self.nbs = [self.tables[p][1].dof for p in self.orders]
        self.precision = precision
        self.hcr = hcr
        self.limiter = limiter
        self.device = device

    def capacity(self, i: int) -> tuple:
        """(elements, internal edges, boundary edges, patches) room of slot i."""
        cap = _native.SlotCapacity()
        self._check(self._lib.dgm_instance_capacity(self._ctx, i, ctypes.byref(cap)), "capacity")
        return (cap.elements, cap.internal_edges, cap.boundary_edges, cap.patches)

    def replace(self, i: int, mesh, cfl: float, final_time: float, final_step: int) -> None:
        """Put ``mesh`` (which must fit slot i's capacity) into slot i, with zeroed state and a
        reset clock, loop bounds and status; the other instances are untouched.  Waits for the
        context's stream first."""
        keep: list = []
        md = _mesh_desc(mesh, keep)
        pr = _native.Params(hcr=self.hcr, cfl=float(cfl), final_time=float(final_time), final_step=int(final_step),
                            limiter=1 if self.limiter else 0, device=self.device,
                            precision=PRECISIONS[self.precision], _reserved=0)
        self._check(self._lib.dgm_instance_replace(self._ctx, i, ctypes.byref(md), ctypes.byref(pr)), "replace")
        self.meshes[i] = mesh

    def _check(self, st: int, what: str) -> None:
        if st != 0:
            raise DgmError(st, int(self._lib.dgm_error_location(self._ctx)), what)

    @property
    def ctx(self):
        return self._ctx

    def close(self) -> None:
        if getattr(self, "_ctx", None):
            self._lib.dgm_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, i: int, solutions: np.ndarray) -> None:
        _check_state(solutions, self.meshes[i].n_elements, self.nbs[i], "solutions")
        self._check(self._lib.dgm_instance_upload(self._ctx, i, _native.dptr(solutions)), "upload")

    def set_initial(self, i: int, initial: "InitialSolution") -> None:
        """Solver::set_initial_solution for instance i, computed on the device."""
        self._check(self._lib.dgm_instance_set_initial(self._ctx, i, float(initial.density),
                                                       float(initial.angle_of_attack), float(initial.mach_number),
                                                       float(initial.pressure)), "set_initial")

    def download(self, i: int) -> np.ndarray:
        out = np.zeros((self.meshes[i].n_elements, 4, self.nbs[i]))
        self._check(self._lib.dgm_instance_download(self._ctx, i, _native.dptr(out)), "download")
        return out

    def advance(self, n_steps: int, with_residual: bool = False) -> None:
        f = self._lib.dgm_advance_with_residual if with_residual else self._lib.dgm_advance
        self._check(f(self._ctx, int(n_steps)), "advance")

    def synchronize(self) -> int:
        """Wait for the device; returns the first device status (0 = ok) without raising, since
        a failing instance stops alone (see state())."""
        return int(self._lib.dgm_synchronize(self._ctx))

    def query(self):
        """Non-blocking synchronize: None while steps are in flight, else the status that
        synchronize() would return."""
        st = int(self._lib.dgm_query(self._ctx))
        return None if st == _native.DGM_NOT_READY else st

    def device_bytes(self) -> int:
        return int(self._lib.dgm_device_bytes(self._ctx))

    @property
    def launch_config(self) -> dict:
        return _launch_config(self._lib, self._ctx)

    def autotune(self, repeats: int = 20) -> dict:
        """As SpatialDisc.autotune, for the whole batch (all instances' states uploaded).  A mixed
        batch runs fixed launch shapes and is not tuned (returns {})."""
        if self.mixed:
            return {}
        return _autotune(self._lib, self._ctx, repeats)

    def state(self, i: int):
        """(current_time, current_step, status, error_location) of instance i."""
        t, s, st, w = ctypes.c_double(), ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int64()
        self._lib.dgm_instance_state(self._ctx, i, ctypes.byref(t), ctypes.byref(s), ctypes.byref(st),
                                     ctypes.byref(w))
        return float(t.value), int(s.value), int(st.value), int(w.value)

    def set_instance(self, i: int, current_time: float, current_step: int, final_time: float,
                     final_step: int) -> None:
        self._check(self._lib.dgm_instance_set(self._ctx, i, float(current_time), int(current_step),
                                               float(final_time), int(final_step)), "set_instance")

    def cell_fields(self, i: int) -> np.ndarray:
        """[ne_i, 4] write_to_vtk cell fields of instance i (see SpatialDisc.cell_fields)."""
        out = np.zeros((self.meshes[i].n_elements, 4))
        self._check(self._lib.dgm_cell_fields(self._ctx, i, _native.dptr(out)), "cell_fields")
        return out

    def diagnostics(self, use_residual: bool = False) -> np.ndarray:
        """[n, 8]: integrals of rho, rho u, rho v, rho E; wall force Fx, Fy; sum of squared density
        residual coefficients; element count (FP64 on the device)."""
        out = np.zeros((self.n, 8))
        self._check(self._lib.dgm_diagnostics(self._ctx, 1 if use_residual else 0, _native.dptr(out)),
                    "diagnostics")
        return out

    def enqueue_diagnostics(self, use_residual: bool = False) -> None:
        """Enqueue :meth:`diagnostics` behind the work on the stream, into a pinned host buffer
        (not for mixed batches)."""
        self._check(self._lib.dgm_enqueue_diagnostics(self._ctx, 1 if use_residual else 0), "enqueue_diagnostics")

    def collected_diagnostics(self) -> np.ndarray:
        """[n, 8]: the diagnostics of the last :meth:`enqueue_diagnostics` (waits for that copy only)."""
        out = np.zeros((self.n, 8))
        self._check(self._lib.dgm_collected_diagnostics(self._ctx, _native.dptr(out)), "collected_diagnostics")
        return out
