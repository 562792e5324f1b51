"""Quadrature and Dubiner-basis tables (host side, built once).

Mirrors ``GaussPoints`` (src/gauss_point.rs:4-95) and ``DubinerBasis``
(src/basis_function.rs:6-203) of DGM_in_rust.  The tables are uploaded to the device by
:class:`dgm_in_rust_b200.solver.SpatialDisc`; the CUDA kernels never rebuild them.

The reference supports only p = 2 (six modes, 6-point triangle rule, 3/4/5-point edge
rules).  Orders 1 and 3 are extensions: the same Dubiner recursion, a 3-point / 12-point
triangle rule and a 2-point / 4-point edge rule, and derivatives the reference does not
tabulate taken from an exact polynomial expansion of each mode.
"""
from __future__ import annotations

import math

import numpy as np

__all__ = [
    "GaussPoints",
    "DubinerBasis",
    "gauss_points_interval",
    "gauss_points_triangle",
    "jacobi_poly",
    "dubiner_basis",
    "mode_lk",
    "key_index",
    "n_keys",
    "default_rules",
]

# Supported (order -> (number of cell points, number of edge points)).
_DEFAULT_RULES = {1: (3, 2), 2: (6, 3), 3: (12, 4)}


def default_rules(order: int) -> tuple[int, int]:
    """Cell/edge rule sizes used for a polynomial order (p=2 is the reference's 6/3)."""
    return _DEFAULT_RULES[order]


def gauss_points_interval(n: int) -> tuple[np.ndarray, np.ndarray]:
    """Gauss-Legendre nodes/weights on [-1, 1] (gauss_point.rs:39-61; n=2 is an extension)."""
    if n == 2:
        x = [-0.5773502691896257, 0.5773502691896257]
        w = [1.0, 1.0]
    elif n == 3:
        x = [-0.7745966692414834, 0.0, 0.7745966692414834]
        w = [0.5555555555555556, 0.8888888888888889, 0.5555555555555556]
    elif n == 4:
        x = [-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526]
        w = [0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538]
    elif n == 5:
        x = [-0.9061798459386640, -0.5384693101056831, 0.0, 0.5384693101056831, 0.9061798459386640]
        w = [0.2369268850561891, 0.4786286704993665, 0.5688888888888889, 0.4786286704993665,
             0.2369268850561891]
    else:
        raise ValueError("Number of points not supported")
    return np.array(x, dtype=np.float64), np.array(w, dtype=np.float64)


def gauss_points_triangle(n: int) -> tuple[np.ndarray, np.ndarray]:
    """Triangle rules on the reference triangle (gauss_point.rs:62-95; 3 and 12 are extensions).

    Weights sum to 1 (integral = 0.5 * J * sum w f), except the reference's 4-point rule whose
    weights sum to 0.5 as tabulated there.
    """
    if n == 3:
        p = [[1.0 / 6.0, 1.0 / 6.0], [2.0 / 3.0, 1.0 / 6.0], [1.0 / 6.0, 2.0 / 3.0]]
        w = [1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0]
    elif n == 4:
        p = [[1.0 / 3.0, 1.0 / 3.0], [2.0 / 15.0, 11.0 / 15.0], [2.0 / 15.0, 2.0 / 15.0],
             [11.0 / 15.0, 2.0 / 15.0]]
        w = [-27.0 / 96.0, 25.0 / 96.0, 25.0 / 96.0, 25.0 / 96.0]
    elif n == 6:
        a, b = 0.44594849091597, 0.10810301816807
        c, d = 0.09157621350977, 0.81684757298046
        p = [[a, a], [a, b], [b, a], [c, c], [c, d], [d, c]]
        w = [0.22338158967801] * 3 + [0.10995174365532] * 3
    elif n == 12:
        a, wa = 0.063089014491502, 0.050844906370207
        b, wb = 0.249286745170910, 0.116786275726379
        c, d, wc = 0.053145049844817, 0.310352451033784, 0.082851075618374
        e = 1.0 - c - d
        p = [[a, a], [1.0 - 2.0 * a, a], [a, 1.0 - 2.0 * a],
             [b, b], [1.0 - 2.0 * b, b], [b, 1.0 - 2.0 * b],
             [c, d], [d, c], [c, e], [e, c], [d, e], [e, d]]
        w = [wa] * 3 + [wb] * 3 + [wc] * 6
    else:
        raise ValueError("Number of points not supported")
    return np.array(p, dtype=np.float64), np.array(w, dtype=np.float64)


def _powi(a: float, b: int) -> float:
    """Rust f64::powi (compiler-rt square-and-multiply)."""
    r = 1.0
    while True:
        if b & 1:
            r *= a
        b //= 2
        if b == 0:
            break
        a *= a
    return r


def jacobi_poly(n: int, alpha: float, beta: float, x: float) -> float:
    """Jacobi polynomial P_n^(alpha,beta)(x) by the recursion of basis_function.rs:56-74."""
    if n == 0:
        return 1.0
    if n == 1:
        return (alpha + 1.0) + (alpha + beta + 2.0) * (x - 1.0) / 2.0
    nn = float(n)
    a1 = 2.0 * nn * (nn + alpha + beta) * (2.0 * nn + alpha + beta - 2.0)
    a2 = 2.0 * nn + alpha + beta - 1.0
    a3 = (2.0 * nn + alpha + beta) * (2.0 * nn + alpha + beta - 2.0) * x + alpha * alpha - beta * beta
    a4 = 2.0 * (nn + alpha - 1.0) * (nn + beta - 1.0) * (2.0 * nn + alpha + beta)
    pn_1 = jacobi_poly(n - 1, alpha, beta, x)
    pn_2 = jacobi_poly(n - 2, alpha, beta, x)
    return (a2 * a3 * pn_1 - a4 * pn_2) / a1


def dubiner_basis(l: int, k: int, xi: float, eta: float) -> float:
    """Dubiner mode (l, k) at (xi, eta), basis_function.rs:75-79."""
    legendre = jacobi_poly(k, 0.0, 0.0, 2.0 * xi / (1.0 - eta) - 1.0)
    jacobi = jacobi_poly(l, 2.0 * float(k) + 1.0, 0.0, 2.0 * eta - 1.0)
    return _powi(2.0, k) * legendre * _powi(1.0 - eta, k) * jacobi


def mode_lk(b: int) -> tuple[int, int]:
    """(l, k) of mode b in the order of compute_phi_cell (basis_function.rs:86-93)."""
    d, start = 0, 0
    while start + d + 1 <= b:
        start += d + 1
        d += 1
    l = b - start
    return l, d - l


def key_index(a: int, b: int) -> int:
    """Index of derivative key (a, b) = d^a/dx^a d^b/dy^b: (1,0),(0,1),(2,0),(1,1),(0,2),..."""
    o = a + b
    return o * (o + 1) // 2 - 1 + b


def n_keys(max_order: int) -> int:
    return (max_order + 1) * (max_order + 2) // 2 - 1


# ---- exact polynomial form of a mode (only for derivatives the reference does not tabulate) --
def _pmul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    r = np.zeros((4, 4))
    for i in range(4):
        for j in range(4):
            if a[i, j] != 0.0:
                for k in range(4 - i):
                    for m in range(4 - j):
                        r[i + k, j + m] += a[i, j] * b[k, m]
    return r


def _pconst(v: float) -> np.ndarray:
    r = np.zeros((4, 4))
    r[0, 0] = v
    return r


def _jacobi_eta(n: int, alpha: float) -> np.ndarray:
    y = np.zeros((4, 4))
    y[0, 0], y[0, 1] = -1.0, 2.0
    p0 = _pconst(1.0)
    if n == 0:
        return p0
    p1 = _pconst(alpha + 1.0) + (alpha + 2.0) / 2.0 * (y + _pconst(-1.0))
    if n == 1:
        return p1
    pm2, pm1 = p0, p1
    for m in range(2, n + 1):
        nn, beta = float(m), 0.0
        a1 = 2.0 * nn * (nn + alpha + beta) * (2.0 * nn + alpha + beta - 2.0)
        a2 = 2.0 * nn + alpha + beta - 1.0
        a3s = (2.0 * nn + alpha + beta) * (2.0 * nn + alpha + beta - 2.0)
        a3 = a3s * y + _pconst(alpha * alpha - beta * beta)
        cur = (a2 / a1) * _pmul(a3, pm1) + (-a4_(nn, alpha, beta) / a1) * pm2
        pm2, pm1 = pm1, cur
    return pm1


def a4_(nn: float, alpha: float, beta: float) -> float:
    return 2.0 * (nn + alpha - 1.0) * (nn + beta - 1.0) * (2.0 * nn + alpha + beta)


_LEGENDRE = [[1.0, 0, 0, 0], [0, 1.0, 0, 0], [-0.5, 0, 1.5, 0], [0, -1.5, 0, 2.5]]


def _dubiner_poly(l: int, k: int) -> np.ndarray:
    s = np.zeros((4, 4))
    s[0, 0], s[1, 0], s[0, 1] = -1.0, 2.0, 1.0
    om = np.zeros((4, 4))
    om[0, 0], om[0, 1] = 1.0, -1.0
    q = np.zeros((4, 4))
    for m in range(k + 1):
        if _LEGENDRE[k][m] == 0.0:
            continue
        t = _pconst(_LEGENDRE[k][m])
        for _ in range(m):
            t = _pmul(t, s)
        for _ in range(k - m):
            t = _pmul(t, om)
        q = q + t
    return _pmul(q, _jacobi_eta(l, 2.0 * k + 1.0)) * _powi(2.0, k)


def _poly_deriv_eval(p: np.ndarray, da: int, db: int, xi: float, eta: float) -> float:
    total = 0.0
    for i in range(da, 4):
        for j in range(db, 4):
            c = p[i, j]
            if c == 0.0:
                continue
            f = c
            for t in range(da):
                f *= float(i - t)
            for t in range(db):
                f *= float(j - t)
            total += f * _powi(xi, i - da) * _powi(eta, j - db)
    return total


def _ref_deriv(b: int, a: int, c: int, xi: float, eta: float) -> float:
    """d^a/dxi^a d^c/deta^c of mode b; modes 0..5 up to second order are the closed forms of
    basis_function.rs:114-151."""
    order = a + c
    if b < 6 and order <= 2:
        if b == 0:
            return 0.0
        if b == 1:
            return 4.0 if (a, c) == (1, 0) else (2.0 if (a, c) == (0, 1) else 0.0)
        if b == 2:
            return 3.0 if (a, c) == (0, 1) else 0.0
        if b == 3:
            if (a, c) == (1, 0):
                return 48.0 * xi + 24.0 * eta - 24.0
            if (a, c) == (0, 1):
                return 24.0 * xi + 8.0 * eta - 8.0
            return {(2, 0): 48.0, (1, 1): 24.0, (0, 2): 8.0}[(a, c)]
        if b == 4:
            if (a, c) == (1, 0):
                return 20.0 * eta - 4.0
            if (a, c) == (0, 1):
                return 20.0 * xi + 20.0 * eta - 12.0
            return {(2, 0): 0.0, (1, 1): 20.0, (0, 2): 20.0}[(a, c)]
        if b == 5:
            if (a, c) == (1, 0):
                return 0.0
            if (a, c) == (0, 1):
                return 20.0 * eta - 8.0
            return {(2, 0): 0.0, (1, 1): 0.0, (0, 2): 20.0}[(a, c)]
    l, k = mode_lk(b)
    if l + k < order:
        return 0.0
    return _poly_deriv_eval(_dubiner_poly(l, k), a, c, xi, eta)


class GaussPoints:
    """GaussPoints (gauss_point.rs:4-37): cell and edge quadrature on the reference triangle.

    edge_points[e][g] maps interval point g onto reference edge e: edge 0 ((x+1)/2, 0), edge 1
    ((1-x)/2, (1+x)/2), edge 2 (0, (x_rev+1)/2) with the interval points reversed, so all three
    edges run counter-clockwise.
    """

    def __init__(self, cell_gp: int, edge_gp: int):
        self.cell_gp_number = cell_gp
        self.edge_gp_number = edge_gp
        self.cell_points, self.cell_weights = gauss_points_triangle(cell_gp)
        x, self.edge_weights = gauss_points_interval(edge_gp)
        ep = np.zeros((3, edge_gp, 2))
        for i in range(edge_gp):
            ep[0, i] = ((x[i] + 1.0) / 2.0, 0.0)
            ep[1, i] = ((1.0 - x[i]) / 2.0, (1.0 + x[i]) / 2.0)
            ep[2, i] = (0.0, (x[edge_gp - 1 - i] + 1.0) / 2.0)
        self.edge_points = ep


class DubinerBasis:
    """DubinerBasis (basis_function.rs:6-203) for polynomial order ``order``.

    ``dphis_cell_gps[q, b, key]`` holds the reference-space derivatives of the modes at the
    cell points for keys (1,0),(0,1),(2,0),(1,1),(0,2)[,(3,0),(2,1),(1,2),(0,3)], the HashMap
    entries of the reference (basis_function.rs:114-151) laid out densely.
    """

    def __init__(self, order: int, gauss_points: GaussPoints):
        if order not in (1, 2, 3):
            raise ValueError("order must be 1, 2 or 3")
        self.order = order
        self.dof = (order + 1) * (order + 2) // 2
        self.max_order = max(order, 2)
        self.nkeys = n_keys(self.max_order)
        g = gauss_points
        nb, nq, ng = self.dof, g.cell_gp_number, g.edge_gp_number
        self.phis_cell_gps = np.zeros((nq, nb))
        self.phis_edge_gps = np.zeros((3, ng, nb))
        self.dphis_cell_gps = np.zeros((nq, nb, self.nkeys))
        self.mass_mat_diag = np.zeros(nb)
        for i in range(nq):
            xi, eta = float(g.cell_points[i, 0]), float(g.cell_points[i, 1])
            for b in range(nb):
                l, k = mode_lk(b)
                self.phis_cell_gps[i, b] = dubiner_basis(l, k, xi, eta)
        for e in range(3):
            for i in range(ng):
                xi, eta = float(g.edge_points[e, i, 0]), float(g.edge_points[e, i, 1])
                for b in range(nb):
                    l, k = mode_lk(b)
                    self.phis_edge_gps[e, i, b] = dubiner_basis(l, k, xi, eta)
        for i in range(nq):
            xi, eta = float(g.cell_points[i, 0]), float(g.cell_points[i, 1])
            for b in range(nb):
                for o in range(1, self.max_order + 1):
                    for c in range(o + 1):
                        a = o - c
                        self.dphis_cell_gps[i, b, key_index(a, c)] = _ref_deriv(b, a, c, xi, eta)
        # compute_dphi_edge, basis_function.rs:152-193: the first derivatives (d/dxi, d/deta)
        self.dphis_edge_gps = np.zeros((3, ng, nb, 2))
        for e in range(3):
            for i in range(ng):
                xi, eta = float(g.edge_points[e, i, 0]), float(g.edge_points[e, i, 1])
                for b in range(nb):
                    self.dphis_edge_gps[e, i, b, 0] = _ref_deriv(b, 1, 0, xi, eta)
                    self.dphis_edge_gps[e, i, b, 1] = _ref_deriv(b, 0, 1, xi, eta)
        # compute_mass_mat, basis_function.rs:194-203
        for b in range(nb):
            acc = 0.0
            for i in range(nq):
                ph = float(self.phis_cell_gps[i, b])
                acc += float(g.cell_weights[i]) * (ph * ph)
            self.mass_mat_diag[b] = acc
