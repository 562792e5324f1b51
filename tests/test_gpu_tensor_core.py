"""The element pass on the tensor cores (precision modes tf32 and tf32x3: tcgen05.mma kind::tf32,
FP32 accumulation in tensor memory) against the oracle, the FP32 FMA path and FP64.

Tolerances: tf32x3 (split operands) behaves like FP32: residual of a given state within 1e-5
relative L2 of the oracle, and after 200 steps of the 64 x 32 O-grid relative L2 density error
<= 1e-5 and |dC_L|, |dC_D| <= 1e-4 against FP64.  tf32 (single TF32 operands, about 1e-3
relative per product): residual within 2e-2 of the oracle, density after 200 steps within 1e-3.
"""
import numpy as np
import pytest

from conftest import rel_l2
from dgm_in_rust_b200 import (Batch, InitialSolution, build_solver, default_rules, forces_to_coefficients,
                              freestream_quantity, initial_state, naca0012_ogrid, process_mesh)
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

TOL_RES = {"tf32x3": 1e-5, "tf32": 2e-2}
TOL_RHO = {"tf32x3": 1e-5, "tf32": 1e-3}


@pytest.fixture(autouse=True)
def _lib(built):
    return built


def _case(raw, mach, aoa):
    mesh = process_mesh(raw, freestream_quantity(mach, aoa, 1.0, 1.0 / 1.4, 1.4), 1.4)
    return mesh, InitialSolution(1.0, aoa, mach, 1.0 / 1.4)


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("precision", ["tf32x3", "tf32"])
def test_tensor_core_residual_vs_oracle(order, precision):
    raw = naca0012_ogrid(64, 32)
    mesh, init = _case(raw, 0.8, 1.25)
    s = build_solver(mesh, order, 1.4, 0.1, 1.0e30, 1, precision=precision)
    U = initial_state(mesh, s.basis, s.gauss_points, 1.4, init)
    rng = np.random.default_rng(order)
    U[:, :, 1:] += 0.02 * rng.standard_normal(U[:, :, 1:].shape) * np.abs(U[:, :, :1])
    Rg = np.zeros_like(U)
    s.spatial_disc.compute_residuals(Rg, U.copy())
    nq, ng = default_rules(order)
    o = Oracle(raw=raw, order=order, ncell_gp=nq, nedge_gp=ng, freestream=(1.25, 0.8, 1.0, 1.0 / 1.4))
    Ro = o.new_state()
    o.compute_residuals(Ro, U)
    err = rel_l2(Rg, Ro)
    print(f"{precision} p={order}: residual rel L2 vs oracle {err:.3e}")
    assert err < TOL_RES[precision]
    s.close()


@pytest.mark.parametrize("precision", ["tf32x3", "tf32"])
def test_tensor_core_accuracy_vs_fp64(precision):
    mesh, init = _case(naca0012_ogrid(64, 32), 0.5, 2.0)
    out = {}
    for prec in ("fp64", precision):
        s = build_solver(mesh, 2, 1.4, 0.1, 1.0e30, 200, precision=prec)
        td = s.temporal_disc
        td.set_initial_on_device(init)
        td.advance(200)
        td.synchronize()
        V = s.spatial_disc.new_state()
        td.download(V)
        d = s.spatial_disc.diagnostics()
        out[prec] = (V, forces_to_coefficients(d[4], d[5], 2.0, 1.0, 0.5))
        s.close()
    (V, (cl, cd)), (V64, (cl64, cd64)) = out[precision], out["fp64"]
    err = rel_l2(V[:, 0], V64[:, 0])
    print(f"{precision}: density rel L2 {err:.3e}, dCL {abs(cl - cl64):.2e}, dCD {abs(cd - cd64):.2e}")
    assert err <= TOL_RHO[precision]
    if precision == "tf32x3":
        assert abs(cl - cl64) <= 1e-4 and abs(cd - cd64) <= 1e-4


def test_tensor_core_batch_matches_solo():
    """Tiles of 32 elements straddle instances in a batch; each accumulator row depends on its own
    row only, so every instance still matches its solo run bit for bit."""
    cases = [_case(naca0012_ogrid(32, 16), 0.5, 2.0), _case(naca0012_ogrid(40, 20), 0.8, 1.25)]
    steps = [5, 7]
    b = Batch([m for m, _ in cases], 2, 1.4, [0.1] * 2, [1.0e30] * 2, steps, precision="tf32x3")
    for i, (m, init) in enumerate(cases):
        b.set_initial(i, init)
    b.advance(8)
    assert b.synchronize() == 0
    for i, (m, init) in enumerate(cases):
        s = build_solver(m, 2, 1.4, 0.1, 1.0e30, steps[i], precision="tf32x3")
        s.temporal_disc.set_initial_on_device(init)
        s.temporal_disc.advance(steps[i])
        s.temporal_disc.synchronize()
        U = s.spatial_disc.new_state()
        s.temporal_disc.download(U)
        s.close()
        assert np.array_equal(b.download(i), U)
    b.close()
