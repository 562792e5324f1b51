"""Batches (many meshes per launch), the FP32 precision mode and the FP64 diagnostics.

* A batch instance produces exactly (bit for bit) what the same mesh produces alone, including
  when instances stop at different steps or one instance fails.
* FP32 mode vs FP64: relative L2 density error <= 1e-5 and |dC_L|, |dC_D| <= 1e-4 after 200
  steps of the 64 x 32 O-grid (M 0.5, AoA 2 deg); the residual of a given state agrees with the
  oracle to 1e-5.
* Diagnostics (conserved totals, wall force) against numpy on the downloaded state.
"""
import math

import numpy as np
import pytest

from conftest import airfoil_raw, rel_l2
from dgm_in_rust_b200 import (Batch, DgmError, InitialSolution, build_solver, forces_to_coefficients,
                              freestream_quantity, initial_state, naca0012_ogrid, process_mesh)
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

REF_FS = (1.5, 0.8, 1.0, 100000.0)


@pytest.fixture(autouse=True)
def _lib(built):
    return built


def _case(raw, mach, aoa, rho=1.0, p=1.0 / 1.4):
    mesh = process_mesh(raw, freestream_quantity(mach, aoa, rho, p, 1.4), 1.4)
    return mesh, InitialSolution(rho, aoa, mach, p)


def _solo(mesh, init, steps, precision="fp64", order=2):
    s = build_solver(mesh, order, 1.4, 0.1, 1.0e30, steps, precision=precision)
    U = initial_state(mesh, s.basis, s.gauss_points, 1.4, init)
    R = np.zeros_like(U)
    s.temporal_disc.time_march(s.spatial_disc, R, U)
    t, st = s.temporal_disc.current_time, s.temporal_disc.current_step
    s.close()
    return U, t, st


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32_compute"])
def test_batch_instances_match_solo(precision):
    cases = [_case(naca0012_ogrid(32, 16), 0.5, 2.0), _case(naca0012_ogrid(48, 24, order="quad"), 0.8, 1.25),
             _case(airfoil_raw(), REF_FS[1], REF_FS[0], REF_FS[2], REF_FS[3])]
    steps = [4, 9, 7]
    b = Batch([m for m, _ in cases], 2, 1.4, [0.1] * 3, [1.0e30] * 3, steps, precision=precision)
    for i, (m, init) in enumerate(cases):
        b.upload(i, initial_state(m, b.basis, b.gauss_points, 1.4, init))
    b.advance(12)
    assert b.synchronize() == 0
    for i, (m, init) in enumerate(cases):
        U, t, st = _solo(m, init, steps[i], precision)
        bt, bs, bstat, _ = b.state(i)
        assert bstat == 0 and bs == st == steps[i] and bt == t
        assert np.array_equal(b.download(i), U)
    b.close()


def test_batch_error_stays_in_its_instance():
    cases = [_case(naca0012_ogrid(32, 16), 0.5, 2.0), _case(naca0012_ogrid(32, 16), 0.6, 1.0),
             _case(naca0012_ogrid(40, 20), 0.7, 0.0)]
    b = Batch([m for m, _ in cases], 2, 1.4, [0.1] * 3, [1.0e30] * 3, [5] * 3)
    for i, (m, init) in enumerate(cases):
        U = initial_state(m, b.basis, b.gauss_points, 1.4, init)
        if i == 1:
            U[5, 3, :] *= -1.0  # negative pressure in instance 1 only
        b.upload(i, U)
    b.advance(5)
    assert b.synchronize() == 2  # "Negative pressure found in HLLC!"
    assert b.state(1)[2] == 2
    for i in (0, 2):
        U, t, st = _solo(cases[i][0], cases[i][1], 5)
        assert b.state(i)[2] == 0 and b.state(i)[1] == 5
        assert np.array_equal(b.download(i), U)
    b.close()


@pytest.mark.parametrize("mode", ["fp32", "fp32_compute"])
def test_fp32_accuracy_vs_fp64(mode):
    """FP32 storage and arithmetic (fp32), and FP32 arithmetic on an FP64 state (fp32_compute):
    density relative L2 <= 1e-5 and |dC_L|, |dC_D| <= 1e-4 after 200 steps."""
    mesh, init = _case(naca0012_ogrid(64, 32), 0.5, 2.0)
    out = {}
    for prec in ("fp64", mode):
        s = build_solver(mesh, 2, 1.4, 0.1, 1.0e30, 200, precision=prec)
        U = initial_state(mesh, s.basis, s.gauss_points, 1.4, init)
        td = s.temporal_disc
        td.upload(U)
        td.advance(200)
        td.synchronize()
        V = np.zeros_like(U)
        td.download(V)
        d = s.spatial_disc.diagnostics()
        out[prec] = (V, forces_to_coefficients(d[4], d[5], 2.0, 1.0, 0.5))
        s.close()
    (V32, (cl32, cd32)), (V64, (cl64, cd64)) = out[mode], out["fp64"]
    assert rel_l2(V32[:, 0], V64[:, 0]) <= 1e-5
    assert abs(cl32 - cl64) <= 1e-4 and abs(cd32 - cd64) <= 1e-4


@pytest.mark.parametrize("mode", ["fp32", "fp32_compute"])
def test_fp32_residual_vs_oracle(mode):
    raw = naca0012_ogrid(64, 32)
    mesh, init = _case(raw, 0.8, 1.25)
    s = build_solver(mesh, 2, 1.4, 0.1, 1.0e30, 1, precision=mode)
    U = initial_state(mesh, s.basis, s.gauss_points, 1.4, init)
    rng = np.random.default_rng(3)
    U[:, :, 1:] += 0.02 * rng.standard_normal(U[:, :, 1:].shape) * np.abs(U[:, :, :1])
    Rg = np.zeros_like(U)
    s.spatial_disc.compute_residuals(Rg, U.copy())
    o = Oracle(raw=raw, order=2, freestream=(1.25, 0.8, 1.0, 1.0 / 1.4))
    Ro = o.new_state()
    o.compute_residuals(Ro, U)
    assert rel_l2(Rg, Ro) < 1e-5
    s.close()


def test_diagnostics_match_numpy():
    raw = naca0012_ogrid(32, 16)
    mesh, init = _case(raw, 0.5, 2.0)
    s = build_solver(mesh, 2, 1.4, 0.1, 1.0e30, 10)
    U = initial_state(mesh, s.basis, s.gauss_points, 1.4, init)
    R = np.zeros_like(U)
    s.temporal_disc.time_march(s.spatial_disc, R, U)
    d = s.spatial_disc.diagnostics(use_residual=True)
    area = 0.5 * mesh.elem_jacob_det
    assert np.allclose(d[0:4], (U[:, :, 0] * area[:, None]).sum(0), rtol=1e-13)
    assert np.isclose(d[6], (R[:, 0, :] ** 2).sum(), rtol=1e-12)
    assert d[7] == mesh.n_elements
    # wall force from the element traces
    phi_e, w = s.basis.phis_edge_gps, s.gauss_points.edge_weights
    F = np.zeros(2)
    for dd in np.nonzero(mesh.edge_elements[:, 1] == -1)[0]:
        if mesh.patch_type[mesh.edge_patch[dd]] != 0:
            continue
        e, k = mesh.edge_elements[dd, 0], mesh.edge_in_cell[dd, 0]
        n = mesh.edge_normal[dd] * (1.0 if mesh.elem_vertices[e, k] == mesh.edge_vertices[dd, 0] else -1.0)
        for g in range(len(w)):
            q = U[e] @ phi_e[k, g]
            p = 0.4 * (q[3] - 0.5 * (q[1] ** 2 + q[2] ** 2) / q[0])
            F += w[g] * p * n * 0.5 * mesh.edge_jacob_det[dd]
    assert np.allclose(d[4:6], F, rtol=1e-12, atol=1e-14)
    s.close()


def test_enqueued_diagnostics_equal_direct():
    """dgm_enqueue_diagnostics / dgm_collected_diagnostics (the serving loop's check path) return
    what dgm_diagnostics returns after the same steps, bit for bit; a mixed batch refuses them."""
    cases = [_case(naca0012_ogrid(32, 16), 0.5, 2.0), _case(naca0012_ogrid(40, 20), 0.7, 1.0)]
    b = Batch([m for m, _ in cases], 2, 1.4, [0.1] * 2, [1.0e30] * 2, [10 ** 6] * 2, precision="fp32")
    for i, (_, init) in enumerate(cases):
        b.set_initial(i, init)
    for n in (1, 9, 32):
        b.advance(n, with_residual=True)
        b.enqueue_diagnostics(use_residual=True)
        got = b.collected_diagnostics()
        assert b.synchronize() == 0
        assert np.array_equal(got, b.diagnostics(use_residual=True))
        assert got[:, 6].min() > 0.0
    b.close()
    m = Batch([cases[0][0], cases[1][0]], [1, 2], 1.4, [0.1] * 2, [1.0e30] * 2, [5] * 2)
    with pytest.raises(DgmError):
        m.enqueue_diagnostics()
    m.close()
