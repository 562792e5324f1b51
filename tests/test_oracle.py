"""Known-answer tests of the CPU oracle (the checker), derived from the mathematics of the
reference algorithm.  No GPU."""
import math

import numpy as np
import pytest

from conftest import rel_l2
from dgm_in_rust_b200 import (DubinerBasis, GaussPoints, freestream_quantity, naca0012_ogrid, process_mesh,
                              reference_cfl)
from dgm_in_rust_b200.basis_function import dubiner_basis, gauss_points_interval, gauss_points_triangle, mode_lk
from dgm_in_rust_b200.mesh import EdgeBlock, RawMesh
from oracle import oracle as orc

FS = (1.25, 0.8, 1.0, 1.0 / 1.4)


def square_mesh(n=6, name="Farfield", L=1.0):
    """n x n square split into counter-clockwise triangles, one boundary block around it."""
    xs = np.linspace(0.0, L, n + 1)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    v = np.stack([X.ravel(), Y.ravel()], 1)
    idx = lambda i, j: i * (n + 1) + j
    tris = []
    for i in range(n):
        for j in range(n):
            a, b, c, d = idx(i, j), idx(i + 1, j), idx(i + 1, j + 1), idx(i, j + 1)
            tris += [(a, b, c), (a, c, d)]
    ring = [idx(i, 0) for i in range(n)] + [idx(n, j) for j in range(n)] + \
           [idx(i, n) for i in range(n, 0, -1)] + [idx(0, j) for j in range(n, 0, -1)]
    pairs = np.array([(ring[k], ring[(k + 1) % len(ring)]) for k in range(len(ring))])
    return RawMesh(vertices=v, edge_blocks=[EdgeBlock(pairs, name)], element_blocks=[np.array(tris)])


@pytest.mark.parametrize("n,deg", [(3, 2), (6, 4), (12, 6)])
def test_triangle_rules_exact(n, deg):
    p, w = gauss_points_triangle(n)
    assert abs(w.sum() - 1.0) < 1e-12
    tol = 1e-12 if n != 6 else 1e-12
    for a in range(deg + 1):
        for b in range(deg + 1 - a):
            exact = 2.0 * math.factorial(a) * math.factorial(b) / math.factorial(a + b + 2)
            got = float(np.sum(w * p[:, 0] ** a * p[:, 1] ** b))
            assert abs(got - exact) < tol * 10 + 1e-13, (a, b, got, exact)


def test_reference_four_point_rule_weights_sum_to_half():
    _, w = gauss_points_triangle(4)  # gauss_point.rs:64-69 as tabulated there
    assert abs(w.sum() - 0.5) < 1e-15


@pytest.mark.parametrize("n", [2, 3, 4, 5])
def test_interval_rules_exact(n):
    x, w = gauss_points_interval(n)
    for k in range(2 * n):
        exact = 0.0 if k % 2 else 2.0 / (k + 1)
        assert abs(float(np.sum(w * x ** k)) - exact) < 1e-14


@pytest.mark.parametrize("order", [1, 2, 3])
def test_dubiner_mass_matrix_diagonal(order):
    nq, ng = {1: (3, 2), 2: (6, 3), 3: (12, 4)}[order]
    g = GaussPoints(nq, ng)
    b = DubinerBasis(order, g)
    M = (b.phis_cell_gps * g.cell_weights[:, None]).T @ b.phis_cell_gps
    off = M - np.diag(np.diag(M))
    assert np.abs(off).max() < 1e-12 * np.abs(np.diag(M)).max()
    assert np.allclose(np.diag(M), b.mass_mat_diag, rtol=1e-14)
    # closed form of the Dubiner norm (mean of phi^2 over the triangle): 4^k / ((2k+1)(k+l+1))
    for m in range(b.dof):
        l, k = mode_lk(m)
        assert abs(b.mass_mat_diag[m] - 4.0 ** k / ((2 * k + 1) * (k + l + 1))) < 1e-11


@pytest.mark.parametrize("order", [2, 3])
def test_derivative_tables_match_finite_differences(order):
    nq, ng = {2: (6, 3), 3: (12, 4)}[order]
    g = GaussPoints(nq, ng)
    b = DubinerBasis(order, g)
    h = 1e-5
    for q in range(nq):
        xi, eta = g.cell_points[q]
        for m in range(b.dof):
            l, k = mode_lk(m)
            f = lambda x, y: dubiner_basis(l, k, x, y)
            dx = (f(xi + h, eta) - f(xi - h, eta)) / (2 * h)
            dy = (f(xi, eta + h) - f(xi, eta - h)) / (2 * h)
            dxx = (f(xi + h, eta) - 2 * f(xi, eta) + f(xi - h, eta)) / h ** 2
            dyy = (f(xi, eta + h) - 2 * f(xi, eta) + f(xi, eta - h)) / h ** 2
            dxy = (f(xi + h, eta + h) - f(xi + h, eta - h) - f(xi - h, eta + h) + f(xi - h, eta - h)) / (4 * h * h)
            got = b.dphis_cell_gps[q, m]
            scale = 1.0 + np.abs(got).max()
            assert abs(got[0] - dx) < 1e-6 * scale and abs(got[1] - dy) < 1e-6 * scale
            assert abs(got[2] - dxx) < 1e-3 * scale and abs(got[3] - dxy) < 1e-3 * scale
            assert abs(got[4] - dyy) < 1e-3 * scale


def test_reference_cfl_formula():
    assert abs(reference_cfl(2) - 0.16) < 1e-15  # initialization.rs:29-33


def test_hllc_consistency_and_rotation():
    rng = np.random.default_rng(1)
    for _ in range(50):
        rho = rng.uniform(0.5, 2.0)
        u, v = rng.uniform(-1, 1, 2)
        p = rng.uniform(0.3, 2.0)
        q = np.array([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)])
        th = rng.uniform(0, 2 * np.pi)
        nx, ny = math.cos(th), math.sin(th)
        st, fl = orc.hllc(q, q, nx, ny)
        f, g = orc.euler_flux(q)
        assert st == 0
        assert np.allclose(fl, f * nx + g * ny, rtol=1e-12, atol=1e-12)
    qn = np.array([-1.0, 0, 0, 1.0])
    assert orc.hllc(qn, qn, 1.0, 0.0)[0] == 1  # "Negative density found in HLLC!"
    qp = np.array([1.0, 0, 0, -1.0])
    assert orc.hllc(qp, qp, 1.0, 0.0)[0] == 2  # "Negative pressure found in HLLC!"


def test_eigenmatrix_inverse_pair():
    rng = np.random.default_rng(2)
    for _ in range(20):
        rho, p = rng.uniform(0.5, 2), rng.uniform(0.3, 2)
        u, v = rng.uniform(-1, 1, 2)
        q = np.array([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)])
        th = rng.uniform(0, 2 * np.pi)
        L, R = orc.eigenmatrix(q, math.cos(th), math.sin(th))
        assert np.allclose(L @ R, np.eye(4), atol=1e-12)


def test_freestream_preserved_on_farfield_box():
    raw = square_mesh(6)
    o = orc.Oracle(raw=raw, order=2, freestream=FS)
    U = o.initial_solution()
    R = o.new_state()
    o.compute_residuals(R, U)
    assert np.abs(R).max() < 1e-11
    assert o.apply_limiter(U.copy()) == 0


def test_initial_projection_is_the_uniform_state():
    o = orc.Oracle(raw=naca0012_ogrid(16, 8), order=2, freestream=FS)
    U = o.initial_solution()
    q = freestream_quantity(FS[1], FS[0], FS[2], FS[3], 1.4)
    cons = np.array([q[0], q[0] * q[1], q[0] * q[2], q[3] / 0.4 + 0.5 * q[0] * (q[1] ** 2 + q[2] ** 2)])
    assert np.allclose(U[:, :, 0], cons[None, :], rtol=1e-13)
    assert np.abs(U[:, :, 1:]).max() < 1e-12


def test_conservation_wall_box():
    """Sum over elements of the mode-0 residual (times its mass) equals minus the boundary flux;
    in a wall-bounded box mass and energy are conserved and the momentum change is -int p n."""
    raw = square_mesh(5, name="Wall")
    o = orc.Oracle(raw=raw, order=2, freestream=FS)
    U = o.initial_solution()
    rng = np.random.default_rng(3)
    U[:, :, 1:] += 0.01 * rng.standard_normal(U[:, :, 1:].shape) * np.abs(U[:, :, :1])
    R = o.new_state()
    o.compute_residuals(R, U)
    J = o.get("elem_jacob_det")
    m0 = o.get("mass")[0]
    tot = (R[:, :, 0] * (m0 * 0.5 * J)[:, None]).sum(0)
    assert abs(tot[0]) < 1e-12 and abs(tot[3]) < 1e-10
    # momentum: - sum over wall edges of int p n (outward), from the element traces
    ev, ee, ic, jd, nrm = (o.get("edge_vertices"), o.get("edge_elements"), o.get("edge_in_cell"),
                           o.get("edge_jacob_det"), o.get("edge_normal"))
    ivs = o.get("elem_vertices")
    phi_e, w = o.get("phi_edge"), o.get("edge_weights")
    mom = np.zeros(2)
    for d in np.nonzero(ee[:, 1] == -1)[0]:
        e, k = ee[d, 0], ic[d, 0]
        n = nrm[d] if ivs[e, k] == ev[d, 0] else -nrm[d]
        for g in range(len(w)):
            qv = U[e] @ phi_e[k, g]
            p = 0.4 * (qv[3] - 0.5 * (qv[1] ** 2 + qv[2] ** 2) / qv[0])
            mom += w[g] * p * n * 0.5 * jd[d]
    assert np.allclose(tot[1:3], -mom, rtol=1e-10, atol=1e-12)


def test_limiter_preserves_cell_means():
    o = orc.Oracle(raw=naca0012_ogrid(32, 16), order=2, freestream=FS)
    U = o.initial_solution()
    rng = np.random.default_rng(4)
    U[:, :, 1:] += 0.1 * rng.standard_normal(U[:, :, 1:].shape) * np.abs(U[:, :, :1])
    V = U.copy()
    n = o.apply_limiter(V)
    assert n > 0
    assert np.allclose(V[:, :, 0], U[:, :, 0], rtol=1e-12, atol=1e-13)
    changed = np.abs(V - U).max(axis=(1, 2)) > 0
    assert changed.sum() == n


def test_limiter_sequential_order_matters():
    """The reference limits in element order in place (weno.rs:90,263): its result differs from
    limiting every troubled cell from the unlimited state (Jacobi) when troubled cells touch."""
    raw = naca0012_ogrid(32, 16, order="quad")
    o = orc.Oracle(raw=raw, order=2, freestream=FS)
    U = o.initial_solution()
    rng = np.random.default_rng(5)
    U[:, :, 1:] += 0.2 * rng.standard_normal(U[:, :, 1:].shape) * np.abs(U[:, :, :1])
    flags = o.troubled_flags(U)
    seq = U.copy()
    o.apply_limiter(seq)
    nbr = o.get("elem_neighbours")
    touching = [(e, n) for e in np.nonzero(flags)[0] for n in nbr[e] if n >= 0 and flags[n]]
    assert touching, "test state should have neighbouring troubled cells"
    # a cell whose lower-index neighbour was limited sees limited values
    assert np.isfinite(seq).all()


def test_oracle_threads_agree():
    raw = naca0012_ogrid(32, 16)
    a = orc.Oracle(raw=raw, order=2, freestream=FS, threads=1)
    b = orc.Oracle(raw=raw, order=2, freestream=FS, threads=4)
    U = a.initial_solution()
    rng = np.random.default_rng(6)
    U[:, :, 1:] += 0.02 * rng.standard_normal(U[:, :, 1:].shape) * np.abs(U[:, :, :1])
    Ra, Rb = a.new_state(), b.new_state()
    a.compute_residuals(Ra, U)
    b.compute_residuals(Rb, U)
    assert rel_l2(Rb, Ra) < 1e-14
    Ra2 = a.new_state()
    a.compute_residuals(Ra2, U)
    assert np.array_equal(Ra, Ra2)  # deterministic with one thread


def test_negative_pressure_raises_like_reference():
    o = orc.Oracle(raw=naca0012_ogrid(16, 8), order=2, freestream=FS)
    U = o.initial_solution()
    U[5, 3, :] *= -1.0
    with pytest.raises(orc.OracleError) as ei:
        o.compute_residuals(o.new_state(), U)
    assert ei.value.status in (1, 2)


def test_time_march_clamps_to_final_time():
    raw = naca0012_ogrid(16, 8)
    o = orc.Oracle(raw=raw, order=2, freestream=FS, final_time=2.5e-4, final_step=1000)
    U = o.initial_solution()
    R = o.new_state()
    t, s = o.time_march(R, U)
    assert t == 2.5e-4 and 0 < s < 1000


def test_viscous_residual_freestream_only_at_the_wall():
    """The Navier-Stokes residual (the reference's disabled NS functions) of the uniform free
    stream: zero jumps and gradients everywhere except the no-slip wall, so it equals the Euler
    residual bit for bit on every element that does not touch the wall, and differs on those that
    do (the wall's momentum jumps feed their lifts)."""
    raw = naca0012_ogrid(16, 8)
    o = orc.Oracle(raw=raw, order=2, freestream=FS)
    U = o.initial_solution()
    U[:, :, 0] = U[0, :, 0]  # exactly uniform: the projection's mode 0 and the higher modes
    U[:, :, 1:] = 0.0        # carry element-to-element round-off
    Re, Rn = o.new_state(), o.new_state()
    o.compute_residuals(Re, U)
    o.set_viscous(True, 0.72, 1e-3)
    o.compute_residuals(Rn, U)
    differs = np.nonzero(np.abs(Rn - Re).max(axis=(1, 2)) > 0.0)[0]
    m = process_mesh(raw, freestream_quantity(FS[1], FS[0], FS[2], FS[3], 1.4), 1.4)
    wall = [m.edge_elements[d, 0] for d in range(m.n_edges)
            if m.edge_elements[d, 1] == -1 and m.patch_type[m.edge_patch[d]] == 0]
    assert len(wall) == 16 and set(differs.tolist()) == set(int(e) for e in wall)
    assert np.isfinite(Rn).all()
