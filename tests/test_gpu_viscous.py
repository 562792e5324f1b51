"""The Navier-Stokes (BR2) residual -- the reference's integrate_over_cell_ns, integrate_over_edges_ns
and apply_bc_ns (spatial_disc.rs:70-160,212-348, boundary_condition.rs:121-413), which its
compute_residuals keeps commented out (spatial_disc.rs:34-36) -- on the GPU against the oracle's
restatement of the same functions (parity with the Rust code unpinned: the reference never runs
them and ships no output of them).

Tolerances (FP64): residuals 1e-12 relative L2, the viscous part alone (NS residual minus Euler
residual) 1e-9, states after RK3 steps 1e-10, clocks 1e-14.  The gas constant is lowered so that
the Sutherland viscosity of the non-dimensional free stream (p = 1 / 1.4) is far above round-off:
1e-6 for the residuals (the viscous part then outweighs the inviscid one on the thin wall cells),
1e-3 for the time march (the viscous terms move the state by ~1e-6 in 3 steps; 1e-6 is unstable
at the inviscid CFL number).  With the reference's 287 they are ~1e-13 of the state.
"""
import ctypes

import numpy as np
import pytest

from conftest import airfoil_raw, rel_l2
from dgm_in_rust_b200 import (Batch, DgmError, InitialSolution, build_solver, default_rules, freestream_quantity,
                              initial_state, naca0012_ogrid, process_mesh)
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

FS = (1.25, 0.8, 1.0, 1.0 / 1.4)  # aoa, mach, rho, p
PR, RGAS, RGAS_MARCH = 0.72, 1e-6, 1e-3
MESHES = {"ogrid32x16": lambda: naca0012_ogrid(32, 16), "airfoil": airfoil_raw}


@pytest.fixture(autouse=True)
def _lib(built):
    return built


def _pair(raw, order, final_step=3, limiter=True):
    nq, ng = default_rules(order)
    mesh = process_mesh(raw, freestream_quantity(FS[1], FS[0], FS[2], FS[3], 1.4), 1.4)
    s = build_solver(mesh, order, 1.4, 0.1, 1.0e30, final_step, limiter=limiter)
    o = Oracle(raw=raw, order=order, ncell_gp=nq, nedge_gp=ng, cfl=0.1, final_time=1.0e30, final_step=final_step,
               limiter=limiter, threads=4, freestream=FS)
    U0 = initial_state(mesh, s.basis, s.gauss_points, 1.4, InitialSolution(FS[2], FS[0], FS[1], FS[3]))
    return s, o, U0


def _perturbed(U0, amp, seed):
    rng = np.random.default_rng(seed)
    U = U0.copy()
    U[:, :, 1:] += amp * rng.standard_normal(U[:, :, 1:].shape) * np.abs(U[:, :, :1])
    return U


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("mesh", sorted(MESHES))
def test_viscous_residual_matches_oracle(order, mesh):
    s, o, U0 = _pair(MESHES[mesh](), order)
    sd = s.spatial_disc
    U = _perturbed(U0, 0.02, order)
    out = {}
    for visc in (False, True):
        sd.set_viscous(visc, PR, RGAS)
        o.set_viscous(visc, PR, RGAS)
        assert sd.viscous == visc
        Ro, Rg = o.new_state(), sd.new_state()
        o.compute_residuals(Ro, U)
        sd.compute_residuals(Rg, U.copy())
        assert rel_l2(Rg, Ro) < 1e-12, visc
        out[visc] = (Rg, Ro)
    dg = out[True][0] - out[False][0]
    do = out[True][1] - out[False][1]
    assert rel_l2(do, out[False][1]) > 1e-6  # the viscous terms are present
    assert rel_l2(dg, do) < 1e-9
    s.close()
    o.close()


def test_viscous_time_march_matches_oracle():
    """Three SSP-RK3 steps of the NS residual with the limiter on (p = 2, 32 x 16 O-grid)."""
    s, o, U0 = _pair(naca0012_ogrid(32, 16), 2, final_step=3)
    s.spatial_disc.set_viscous(True, PR, RGAS_MARCH)
    o.set_viscous(True, PR, RGAS_MARCH)
    Uo, Ro = U0.copy(), o.new_state()
    to, so = o.time_march(Ro, Uo)
    Ug, Rg = U0.copy(), s.spatial_disc.new_state()
    s.temporal_disc.time_march(s.spatial_disc, Rg, Ug)
    assert so == s.temporal_disc.current_step == 3
    assert abs(s.temporal_disc.current_time - to) <= 1e-14 * to
    assert rel_l2(Ug, Uo) < 1e-10
    s.close()
    o.close()


def test_viscous_switch_and_refusals():
    """Switching the NS residual off gives the Euler context's residual bit for bit; FP32
    contexts and mixed batches refuse it."""
    raw = naca0012_ogrid(24, 12)
    s, _, U0 = _pair(raw, 2)
    U = _perturbed(U0, 0.02, 9)
    R0 = s.spatial_disc.new_state()
    s.spatial_disc.compute_residuals(R0, U.copy())
    s.spatial_disc.set_viscous(True, PR, RGAS)
    R1 = s.spatial_disc.new_state()
    s.spatial_disc.compute_residuals(R1, U.copy())
    s.spatial_disc.set_viscous(False)
    R2 = s.spatial_disc.new_state()
    s.spatial_disc.compute_residuals(R2, U.copy())
    assert not np.array_equal(R0, R1) and np.array_equal(R0, R2)
    with pytest.raises(DgmError):
        s.spatial_disc.set_viscous(True, -1.0, RGAS)
    s.close()
    mesh = process_mesh(raw, freestream_quantity(FS[1], FS[0], FS[2], FS[3], 1.4), 1.4)
    f = build_solver(mesh, 2, 1.4, 0.1, 1.0e30, 3, precision="fp32")
    with pytest.raises(DgmError):
        f.spatial_disc.set_viscous(True, PR, RGAS)
    f.close()
    m = Batch([mesh, process_mesh(naca0012_ogrid(16, 8), freestream_quantity(FS[1], FS[0], FS[2], FS[3], 1.4), 1.4)],
              [1, 2], 1.4, [0.1] * 2, [1.0e30] * 2, [3] * 2)
    table = np.zeros(3 * 4 * 10 * 2)
    assert m._lib.dgm_set_viscous(m.ctx, 1, PR, RGAS, table.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 7
    # DGM_BAD_ARG
    m.close()


def test_viscous_reference_configuration():
    """The reference's configured case (its airfoil.msh, p = 2, M 0.8, AoA 1.5 deg, rho 1, p 1e5,
    CFL 0.1) with the NS terms at its parameters (Prandtl 0.72, gas constant 287: T = 348 K):
    5 steps against the oracle at 1e-10, where the viscous terms move the state by ~3.5e-8."""
    ref_fs = (1.5, 0.8, 1.0, 100000.0)
    raw = airfoil_raw()
    mesh = process_mesh(raw, freestream_quantity(ref_fs[1], ref_fs[0], ref_fs[2], ref_fs[3], 1.4), 1.4)
    s = build_solver(mesh, 2, 1.4, 0.1, 1.0e30, 5)
    o = Oracle(raw=raw, order=2, cfl=0.1, final_time=1.0e30, final_step=5, threads=4, freestream=ref_fs)
    U0 = initial_state(mesh, s.basis, s.gauss_points, 1.4, InitialSolution(ref_fs[2], ref_fs[0], ref_fs[1], ref_fs[3]))
    s.spatial_disc.set_viscous(True, 0.72, 287.0)
    o.set_viscous(True, 0.72, 287.0)
    Uo, Ro = U0.copy(), o.new_state()
    to, so = o.time_march(Ro, Uo)
    Ug, Rg = U0.copy(), s.spatial_disc.new_state()
    s.temporal_disc.time_march(s.spatial_disc, Rg, Ug)
    assert so == s.temporal_disc.current_step == 5
    assert abs(s.temporal_disc.current_time - to) <= 1e-14 * to
    assert rel_l2(Ug, Uo) < 1e-10
    o.set_viscous(False)
    o.reset_clock()
    Ue, Re = U0.copy(), o.new_state()
    assert o.time_march(Re, Ue)[1] == 5
    assert rel_l2(Uo, Ue) > 1e-8  # the viscous terms count
    s.close()
    o.close()
