"""The oracle against the committed golden fixtures (regression pins; see
tests/golden/make_golden.py).  No GPU."""
import os

import numpy as np

from conftest import GOLDEN, airfoil_raw, rel_l2
from dgm_in_rust_b200 import naca0012_ogrid
from oracle.oracle import Oracle

FS = (1.25, 0.8, 1.0, 1.0 / 1.4)
REF_FS = (1.5, 0.8, 1.0, 100000.0)


def test_airfoil_fixture_shape():
    raw = airfoil_raw()
    assert raw.vertices.shape == (1961, 2)
    assert sum(len(t) for t in raw.element_blocks) == 3738
    assert sum(len(b.node_pairs) for b in raw.edge_blocks) == 184
    names = {b.physical_name for b in raw.edge_blocks}
    assert names == {"Wall", "Farfield"}


def test_airfoil_reference_run_golden():
    z = np.load(os.path.join(GOLDEN, "airfoil_run.npz"))
    o = Oracle(raw=airfoil_raw(), order=2, ncell_gp=6, nedge_gp=3, hcr=1.4, cfl=-1.0, final_time=5.0,
               final_step=20, freestream=REF_FS)
    assert abs(o.cfl - 0.16) < 1e-15
    U = o.initial_solution()
    R = o.new_state()
    t, s = o.time_march(R, U)
    assert s == int(z["steps"]) == 20
    assert abs(t - float(z["t20"])) <= 1e-15 * abs(t)
    assert rel_l2(U, z["U20"]) < 1e-13


def test_ogrid_golden():
    z = np.load(os.path.join(GOLDEN, "ogrid16x8.npz"))
    o = Oracle(raw=naca0012_ogrid(16, 8), order=2, cfl=0.1, final_time=1.0e30, final_step=3, freestream=FS)
    U0 = o.initial_solution()
    assert np.array_equal(U0, z["U0"])
    R0 = o.new_state()
    o.compute_residuals(R0, U0)
    assert rel_l2(R0, z["R0"]) < 1e-14
    Rp = o.new_state()
    o.compute_residuals(Rp, z["Up"].copy())
    assert rel_l2(Rp, z["Rp"]) < 1e-14
    Ul = z["Ut"].copy()
    assert o.apply_limiter(Ul) == int(z["troubled"])
    assert rel_l2(Ul, z["Ul"]) < 1e-14
    R3 = o.new_state()
    t, s = o.time_march(R3, U0)
    assert s == 3 and abs(t - float(z["t3"])) < 1e-18
    assert rel_l2(U0, z["U3"]) < 1e-14
