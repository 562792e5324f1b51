"""The allocation-free time step (dgm_compute_time_step_noalloc) against the context entry point.

It exists for callers that cannot call cudaMalloc (a host whose device memory belongs to another
allocator, code running during stream capture, real-time loops): they pass device buffers they
already own and the library uses a fixed scratch array in its image.  The buffers here are made
by torch only to play that caller.  This file is collected last on purpose: if it fails, a run
that stops at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from dgm_in_rust_b200 import (InitialSolution, build_solver, freestream_quantity, initial_state,
                              naca0012_ogrid, process_mesh)

pytestmark = pytest.mark.gpu

DGM_BAD_ARG = 7
MAX_ELEMENTS = 4096 * 2048
TOL = 1e-14


def _entry():
    from dgm_in_rust_b200 import _native
    L = _native.lib()
    f = L.dgm_compute_time_step_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_double,
                  ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int32
    return f


def _call(f, dU, dh, ne, nb, out, cfl=0.1, hcr=1.4):
    import torch
    stream = torch.cuda.current_stream(out.device)
    st = f(dU.data_ptr(), dh.data_ptr(), ne, nb, cfl, hcr, out.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    return st, float(out.item())


def _numpy_time_step(U, h, cfl=0.1, hcr=1.4):
    """compute_time_step (temporal_disc.rs:58-88) in numpy: modal sums taken in basis order."""
    s = [U[:, v, 0].copy() for v in range(4)]
    for v in range(4):
        for b in range(1, U.shape[2]):
            s[v] = s[v] + U[:, v, b]
    rho = s[0]
    with np.errstate(invalid="ignore", divide="ignore"):
        vx, vy = s[1] / rho, s[2] / rho
        p = (hcr - 1.0) * (s[3] - 0.5 * rho * (vx * vx + vy * vy))
        c = np.sqrt(hcr * p / rho)
        dt = cfl * h / (np.sqrt(vx * vx + vy * vy) + c)
    ok = dt < 1.0e10
    return float(dt[ok].min()) if ok.any() else 1.0e10


@pytest.mark.parametrize("order", [1, 2, 3])
def test_time_step_noalloc_matches_context_entry(built, order):
    """Two calls in a row on different states, each equal to dgm_compute_time_step."""
    import torch
    fs = (1.25, 0.8, 1.0, 1.0 / 1.4)
    mesh = process_mesh(naca0012_ogrid(64, 32), freestream_quantity(fs[1], fs[0], fs[2], fs[3], 1.4), 1.4)
    solver = build_solver(mesh, order, 1.4, 0.1, 1.0e30, 10)
    U0 = initial_state(mesh, solver.basis, solver.gauss_points, 1.4, InitialSolution(fs[2], fs[0], fs[1], fs[3]))
    nb = U0.shape[2]
    rng = np.random.default_rng(11 + order)
    f = _entry()
    dev = torch.device("cuda:0")
    h = torch.from_numpy(np.ascontiguousarray(mesh.elem_minimum_height)).to(dev)
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    for amp in (0.0, 0.05):
        U = U0.copy()
        U[:, :, 1:] += amp * rng.standard_normal(U[:, :, 1:].shape) * np.abs(U[:, :, :1])
        expected = solver.temporal_disc.compute_time_step(U)
        st, got = _call(f, torch.from_numpy(U).to(dev), h, mesh.n_elements, nb, out)
        assert st == 0
        assert abs(got - expected) <= TOL * abs(expected), (got, expected)
    # sizes beyond the fixed scratch are refused before anything is launched
    dU = torch.from_numpy(U0).to(dev)
    out.fill_(-1.0)
    st = f(dU.data_ptr(), h.data_ptr(), MAX_ELEMENTS + 1, nb, 0.1, 1.4, out.data_ptr(), 0)
    assert st == DGM_BAD_ARG
    # a non-positive or NaN CFL number is refused (the minimum is taken over non-negative steps)
    for cfl in (0.0, -0.1, float("nan")):
        assert f(dU.data_ptr(), h.data_ptr(), mesh.n_elements, nb, cfl, 1.4, out.data_ptr(), 0) == DGM_BAD_ARG
    torch.cuda.synchronize()
    assert float(out.item()) == -1.0  # nothing was launched
    solver.close()


def test_time_step_noalloc_many_partials_against_numpy(built):
    """600,000 elements (293 partial minima: the final reduction's strided loop runs), seeded random
    positive densities, heights and pressures, two calls in a row; against a numpy restatement."""
    import torch
    rng = np.random.default_rng(5)
    ne, nb = 600_000, 6
    dev = torch.device("cuda:0")
    f = _entry()
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    for call in range(2):
        U = np.zeros((ne, 4, nb))
        U[:, 0, 0] = rng.uniform(0.5, 2.0, ne)
        U[:, 1, 0] = U[:, 0, 0] * rng.uniform(-1.0, 1.0, ne)
        U[:, 2, 0] = U[:, 0, 0] * rng.uniform(-1.0, 1.0, ne)
        U[:, 3, 0] = rng.uniform(3.0, 6.0, ne)
        U[:, :, 1:] = 1e-3 * rng.standard_normal((ne, 4, nb - 1))
        h = rng.uniform(1e-6, 1e-2, ne)
        expected = _numpy_time_step(U, h)
        st, got = _call(f, torch.from_numpy(U).to(dev), torch.from_numpy(h).to(dev), ne, nb, out)
        assert st == 0
        assert abs(got - expected) <= TOL * abs(expected), (call, got, expected)


def test_time_step_noalloc_without_a_valid_step(built):
    """No element gives a finite step below the reference's start value: the result is 1e10, both
    for NaN states and for steps of 1e10 or more (the scratch holds the previous call's minima)."""
    import torch
    dev = torch.device("cuda:0")
    f = _entry()
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    ne, nb = 5000, 3
    U = np.zeros((ne, 4, nb))
    U[:, 0, 0], U[:, 3, 0] = 1.0, 2.5
    h = np.full(ne, 1e-3)
    st, got = _call(f, torch.from_numpy(U).to(dev), torch.from_numpy(h).to(dev), ne, nb, out)
    expected = _numpy_time_step(U, h)
    assert st == 0 and expected < 1e10 and abs(got - expected) <= TOL * expected
    st, got = _call(f, torch.full((ne, 4, nb), float("nan"), dtype=torch.float64, device=dev),
                    torch.from_numpy(h).to(dev), ne, nb, out)
    assert st == 0 and got == 1.0e10
    st, got = _call(f, torch.from_numpy(U).to(dev), torch.full((ne,), 1e12, dtype=torch.float64, device=dev),
                    ne, nb, out)
    assert st == 0 and got == 1.0e10
