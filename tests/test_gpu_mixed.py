"""Mixed batches (dgm_create_mixed): meshes of orders 1, 2 and 3 advanced by the same launches.

* Every instance of a mixed batch produces exactly (bit for bit) what its mesh produces alone:
  state, clock and FP64 diagnostics, for {1, 2} and {1, 2, 3}, in FP64, FP32 and FP32 arithmetic on
  an FP64 state, with instances stopping at different steps.
* Slots of a mixed batch: a finished instance's slot takes a new mesh of its order while the
  others keep running, and the new solve is again bitwise its solo run.
* The per-order calls (launch configuration, single-mesh entry points) are refused.
"""
import numpy as np
import pytest

from dgm_in_rust_b200 import (Batch, DgmError, InitialSolution, build_solver, freestream_quantity, initial_state,
                              naca0012_ogrid, process_mesh, slot_capacity)

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _lib(built):
    return built


def _case(ni, nj, mach, aoa, rho=1.0, p=1.0 / 1.4):
    mesh = process_mesh(naca0012_ogrid(ni, nj), freestream_quantity(mach, aoa, rho, p, 1.4), 1.4)
    return mesh, InitialSolution(rho, aoa, mach, p)


def _solo(mesh, init, order, steps, precision):
    s = build_solver(mesh, order, 1.4, 0.1, 1.0e30, steps, precision=precision)
    U = initial_state(mesh, s.basis, s.gauss_points, 1.4, init)
    R = np.zeros_like(U)
    s.temporal_disc.time_march(s.spatial_disc, R, U)
    out = (U, s.temporal_disc.current_time, s.temporal_disc.current_step, s.spatial_disc.diagnostics())
    s.close()
    return out


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32_compute"])
@pytest.mark.parametrize("orders", [(1, 2, 2, 1), (3, 1, 2, 3)])
def test_mixed_instances_match_solo(precision, orders):
    shapes = [(32, 16, 0.5, 2.0), (48, 24, 0.8, 1.25), (40, 20, 0.7, -1.0), (24, 12, 0.6, 3.0)]
    cases = [_case(*sh) for sh in shapes]
    steps = [5, 9, 7, 8]
    b = Batch([m for m, _ in cases], list(orders), 1.4, [0.1] * 4, [1.0e30] * 4, steps, precision=precision)
    assert b.mixed
    for i, (m, init) in enumerate(cases):
        b.set_initial(i, init)
    b.advance(10)
    assert b.synchronize() == 0
    d = b.diagnostics()
    for i, (m, init) in enumerate(cases):
        U, t, st, ds = _solo(m, init, orders[i], steps[i], precision)
        bt, bs, bstat, _ = b.state(i)
        assert bstat == 0 and bs == st == steps[i] and bt == t, i
        assert np.array_equal(b.download(i), U), i
        assert np.array_equal(d[i, :6], ds[:6]) and d[i, 7] == m.n_elements, i
    b.close()


def test_mixed_slot_replacement_matches_solo():
    cases = [_case(32, 16, 0.5, 2.0), _case(40, 20, 0.8, 1.25), _case(24, 12, 0.6, 0.0)]
    orders = [1, 2, 1]
    new_mesh, new_init = _case(44, 22, 0.7, 2.5)
    caps = [slot_capacity(new_mesh), slot_capacity(cases[1][0]), slot_capacity(cases[2][0])]
    b = Batch([m for m, _ in cases], orders, 1.4, [0.1] * 3, [1.0e30] * 3, [3, 12, 12], capacities=caps)
    for i, (m, init) in enumerate(cases):
        b.set_initial(i, init)
    b.advance(3)
    assert b.synchronize() == 0 and b.state(0)[1] == 3
    b.replace(0, new_mesh, 0.1, 1.0e30, 8)
    b.set_initial(0, new_init)
    b.advance(9)
    assert b.synchronize() == 0
    Un, tn, sn, _ = _solo(new_mesh, new_init, 1, 8, "fp64")
    assert b.state(0)[1] == sn == 8 and b.state(0)[0] == tn
    assert np.array_equal(b.download(0), Un)
    for i in (1, 2):
        U, t, st, _ = _solo(cases[i][0], cases[i][1], orders[i], 12, "fp64")
        assert b.state(i)[1] == st == 12 and b.state(i)[0] == t
        assert np.array_equal(b.download(i), U)
    b.close()


def test_mixed_refuses_per_order_calls():
    cases = [_case(16, 8, 0.5, 2.0), _case(16, 8, 0.5, 2.0)]
    b = Batch([m for m, _ in cases], [1, 2], 1.4, [0.1] * 2, [1.0e30] * 2, [2, 2])
    assert b.autotune() == {}
    assert b._lib.dgm_set_launch_config(b.ctx, 128, 0, 128) == 7
    assert b._lib.dgm_set_limiter_schedule(b.ctx, 1) == 7
    with pytest.raises(DgmError):
        b.set_initial(5, cases[0][1])
    b.close()
