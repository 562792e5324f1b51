"""Batch slots (dgm_create_batch_slots / dgm_instance_replace): instances with room for larger
meshes, and a finished slot taking a new mesh while the others keep running.

* Every instance of a padded batch produces exactly (bit for bit) what its mesh produces alone:
  state, clock and FP64 diagnostics.
* A slot that takes a new mesh mid-run computes it exactly as alone, and the instance that keeps
  running beside it is not disturbed (bitwise against its own solo run).
* A mesh larger than the slot is refused with DGM_BAD_ARG and changes nothing.
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


def _solo(mesh, init, steps, precision, order=2):
    s = build_solver(mesh, order, 1.4, 0.1, 1.0e30, steps, precision=precision)
    U = initial_state(mesh, s.basis, s.gauss_points, 1.4, init)
    R = np.zeros_like(U)
    s.temporal_disc.time_march(s.spatial_disc, R, U)
    out = (U, s.temporal_disc.current_time, s.temporal_disc.current_step, s.spatial_disc.diagnostics())
    s.close()
    return out


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_padded_slots_match_solo(precision):
    cases = [_case(32, 16, 0.5, 2.0), _case(48, 24, 0.8, 1.25), _case(40, 20, 0.7, -1.0)]
    big = slot_capacity(_case(64, 32, 0.5, 0.0)[0])
    caps = [big, big, slot_capacity(cases[2][0])]  # the last slot exact: padding before and after it
    steps = [6, 9, 7]
    b = Batch([m for m, _ in cases], 2, 1.4, [0.1] * 3, [1.0e30] * 3, steps, precision=precision, capacities=caps)
    assert [b.capacity(i) for i in range(3)] == [tuple(c) for c in caps]
    for i, (m, init) in enumerate(cases):
        b.upload(i, initial_state(m, b.basis, b.gauss_points, 1.4, init))
    b.advance(12)
    assert b.synchronize() == 0
    d = b.diagnostics()
    for i, (m, init) in enumerate(cases):
        U, t, st, ds = _solo(m, init, steps[i], precision)
        bt, bs, bstat, _ = b.state(i)
        assert bstat == 0 and bs == st == steps[i] and bt == t
        assert np.array_equal(b.download(i), U)
        assert np.array_equal(d[i, :6], ds[:6]) and d[i, 7] == m.n_elements
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_replaced_slot_matches_solo_and_leaves_neighbour_alone(precision):
    cases = [_case(32, 16, 0.5, 2.0), _case(48, 24, 0.8, 1.25)]
    new_mesh, new_init = _case(56, 28, 0.6, 3.0)
    caps = [slot_capacity(new_mesh), slot_capacity(cases[1][0])]
    b = Batch([m for m, _ in cases], 2, 1.4, [0.1] * 2, [1.0e30] * 2, [4, 20], precision=precision, capacities=caps)
    for i, (m, init) in enumerate(cases):
        b.set_initial(i, init)
    b.advance(4)  # instance 0 finishes, instance 1 is at step 4 of 20
    assert b.synchronize() == 0 and b.state(0)[1] == 4 and b.state(1)[1] == 4
    U0, t0, _, _ = _solo(cases[0][0], cases[0][1], 4, precision)
    assert np.array_equal(b.download(0), U0) and b.state(0)[0] == t0
    # slot 0 takes a larger mesh and runs 11 steps while instance 1 goes on
    b.replace(0, new_mesh, 0.1, 1.0e30, 11)
    b.set_initial(0, new_init)
    assert b.state(0)[1] == 0
    b.advance(16)
    assert b.synchronize() == 0
    Un, tn, sn, dn = _solo(new_mesh, new_init, 11, precision)
    assert b.state(0)[1] == sn == 11 and b.state(0)[0] == tn
    assert np.array_equal(b.download(0), Un)
    assert np.array_equal(b.diagnostics()[0, :6], dn[:6])
    U1, t1, s1, _ = _solo(cases[1][0], cases[1][1], 20, precision)
    assert b.state(1)[1] == s1 == 20 and b.state(1)[0] == t1
    assert np.array_equal(b.download(1), U1)
    b.close()


def test_replace_refuses_a_mesh_larger_than_the_slot():
    small, init = _case(32, 16, 0.5, 2.0)
    b = Batch([small], 2, 1.4, [0.1], [1.0e30], [3], capacities=[slot_capacity(small)])
    b.set_initial(0, init)
    big, _ = _case(40, 20, 0.5, 2.0)
    with pytest.raises(DgmError) as ei:
        b.replace(0, big, 0.1, 1.0e30, 3)
    assert ei.value.status == 7
    b.advance(3)
    assert b.synchronize() == 0
    U, t, st, _ = _solo(small, init, 3, "fp64")
    assert np.array_equal(b.download(0), U) and b.state(0)[1] == 3
    b.close()
