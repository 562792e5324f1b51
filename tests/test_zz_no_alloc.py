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


def _entry():
    from dgm_in_rust_b200 import _native
    L = _native.lib()
    f = L.dgm_compute_time_step_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_double,
                  ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int32
    return f


def test_time_step_noalloc_matches_context_entry(built):
    import torch
    fs = (1.25, 0.8, 1.0, 1.0 / 1.4)
    mesh = process_mesh(naca0012_ogrid(64, 32), freestream_quantity(fs[1], fs[0], fs[2], fs[3], 1.4), 1.4)
    solver = build_solver(mesh, 2, 1.4, 0.1, 1.0e30, 10)
    U0 = initial_state(mesh, solver.basis, solver.gauss_points, 1.4, InitialSolution(fs[2], fs[0], fs[1], fs[3]))
    rng = np.random.default_rng(11)
    states = []
    for amp in (0.0, 0.05):  # two calls in a row on different states
        U = U0.copy()
        U[:, :, 1:] += amp * rng.standard_normal(U[:, :, 1:].shape) * np.abs(U[:, :, :1])
        states.append(U)
    f = _entry()
    dev = torch.device("cuda:0")
    h = torch.from_numpy(np.ascontiguousarray(mesh.elem_minimum_height)).to(dev)
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    for U in states:
        expected = solver.temporal_disc.compute_time_step(U)
        dU = torch.from_numpy(U).to(dev)
        st = f(dU.data_ptr(), h.data_ptr(), mesh.n_elements, 6, 0.1, 1.4, out.data_ptr(), stream.cuda_stream)
        assert st == 0
        torch.cuda.synchronize()
        got = float(out.item())
        assert abs(got - expected) <= 1e-14 * abs(expected), (got, expected)
    # sizes beyond the fixed scratch are refused before anything is launched
    st = f(dU.data_ptr(), h.data_ptr(), MAX_ELEMENTS + 1, 6, 0.1, 1.4, out.data_ptr(), stream.cuda_stream)
    assert st == DGM_BAD_ARG
    solver.close()
