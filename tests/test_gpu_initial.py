"""Solver::set_initial_solution on the device (dgm_set_initial_solution / dgm_instance_set_initial)
against the host restatement and the oracle.  Tolerance: bitwise."""
import numpy as np
import pytest

from dgm_in_rust_b200 import Batch, InitialSolution, build_solver, initial_state
from dgm_in_rust_b200.workloads import Instance, instance_mesh


@pytest.mark.gpu
@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_device_projection_matches_host(built, order, precision):
    mesh, _ = instance_mesh(Instance(24, 12, 0.7, 2.0, order))
    init = InitialSolution(density=1.3, angle_of_attack=-3.25, mach_number=0.72, pressure=0.9)
    s = build_solver(mesh, order, 1.4, 0.1, 1.0, 10, precision=precision)
    try:
        host = initial_state(mesh, s.basis, s.gauss_points, 1.4, init)
        s.temporal_disc.set_initial_on_device(init)
        dev = s.spatial_disc.new_state()
        s.temporal_disc.download(dev)
        want = host if precision == "fp64" else host.astype(np.float32).astype(np.float64)
        assert np.array_equal(dev, want)
    finally:
        s.close()


@pytest.mark.gpu
def test_device_projection_matches_oracle(built):
    from oracle.oracle import Oracle
    from dgm_in_rust_b200 import freestream_quantity, naca0012_ogrid, process_mesh
    aoa, mach, rho, p = 2.0, 0.5, 1.0, 1.0 / 1.4
    raw = naca0012_ogrid(16, 8)
    mesh = process_mesh(raw, freestream_quantity(mach, aoa, rho, p, 1.4), 1.4)
    s = build_solver(mesh, 2, 1.4, 0.1, 1.0, 10)
    try:
        s.temporal_disc.set_initial_on_device(InitialSolution(rho, aoa, mach, p))
        dev = s.spatial_disc.new_state()
        s.temporal_disc.download(dev)
    finally:
        s.close()
    o = Oracle(raw=raw, order=2, freestream=(aoa, mach, rho, p), initial=(aoa, mach, rho, p))
    try:
        assert np.array_equal(dev, o.initial_solution())
    finally:
        o.close()


@pytest.mark.gpu
def test_batch_instances_projected_separately(built):
    insts = [Instance(16, 8, 0.5, 2.0, 2), Instance(24, 12, 0.8, -1.0, 2)]
    built_ = [instance_mesh(i) for i in insts]
    b = Batch([m for m, _ in built_], 2, 1.4, [0.1] * 2, [1.0] * 2, [10] * 2)
    try:
        for i, (_, init) in enumerate(built_):
            b.set_initial(i, init)
        for i, (m, init) in enumerate(built_):
            assert np.array_equal(b.download(i), initial_state(m, b.basis, b.gauss_points, 1.4, init))
    finally:
        b.close()
