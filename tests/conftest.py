import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity of the CUDA path vs the oracle")


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


@pytest.fixture(scope="session", autouse=True)
def built():
    """Compile the CUDA library (nvcc cross-compiles without a GPU; it also holds the native
    mesh preprocessing every test uses) and the oracle."""
    from dgm_in_rust_b200.build import build
    from oracle.oracle import build as build_oracle
    build()
    build_oracle()
    return True


def airfoil_raw():
    """The reference's airfoil.msh fixture as a RawMesh."""
    from dgm_in_rust_b200.mesh import EdgeBlock, RawMesh
    z = np.load(os.path.join(GOLDEN, "airfoil_mesh.npz"))
    names = [str(n) for n in z["edge_block_names"]]
    eb = [EdgeBlock(z[f"edge_block_{k}"], names[k]) for k in range(len(names))]
    tb = [z[k] for k in sorted(z.files) if k.startswith("tri_block_")]
    return RawMesh(vertices=z["vertices"], edge_blocks=eb, element_blocks=tb)
