"""Regenerate the golden fixtures in this folder.

  python tests/golden/make_golden.py <DGM_in_rust checkout>

* reference_airfoil.msh.gz, reference_mesh.vtk.gz -- the reference's own input fixture
  (inputfiles/airfoil.msh) and its own output file (outputfiles/mesh.vtk, written by its
  write_to_vtk), copied gzipped: the VTK bytes pin the gmsh reader, the element/vertex order and
  the writer to an output the reference produced.
* airfoil_mesh.npz -- the reference's own mesh fixture (inputfiles/airfoil.msh of
  DGM_in_rust: 1961 nodes, 3738 triangles, Wall/Farfield lines), parsed with the package's
  GmshParser and checked against the oracle's parser; stored as arrays so the tests do not need
  the reference tree.
* airfoil_run.npz -- the reference's configured run on that mesh (its parameters.json /
  freestream.json / initial_solution.json: p = 2, 6/3-point rules, gamma 1.4, M 0.8,
  AoA 1.5 deg, rho 1, p 1e5, CFL from the formula of initialization.rs:29-33, 20 steps),
  computed by the oracle.
* ogrid16x8.npz -- a 16 x 8 O-grid (p = 2): initial state, its residual, a seeded perturbed
  state with its residual and limited state, and 3 time-march steps.
* c2_run.npz -- the transonic limiter configuration (256 x 128 O-grid, 65,536 triangles, p = 2,
  M 0.8, AoA 1.25 deg, free-stream start, CFL 0.1, limiter on) marched by the oracle for its
  configured 2000 steps, with checkpoints after 200 and 2000 steps: clock, per-(variable, mode)
  sums and sums of squares over all elements, and the full records of a sample of elements (every
  128th element and every boundary element); the same for the oracle's twin run started from the
  initial state perturbed by 1e-15 (relative, seeded), whose distance from the first run is the
  spread that round-off alone produces in this chaotic start.  About an hour on 8 host threads.

  python tests/golden/make_golden.py --c2-run

The oracle is the C++ restatement under oracle/ (parity with the Rust reference unpinned).
"""
import gzip
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from dgm_in_rust_b200 import GmshParser, naca0012_ogrid  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

AIRFOIL = None  # <checkout>/inputfiles/airfoil.msh, set from the command line
REF_FS = (1.5, 0.8, 1.0, 100000.0)  # aoa, mach, rho, p of freestream.json / initial_solution.json


def airfoil():
    raw = GmshParser.parse(AIRFOIL)
    o = Oracle(msh_path=AIRFOIL, order=2, ncell_gp=6, nedge_gp=3, freestream=REF_FS)
    assert np.array_equal(o.get("xy"), raw.vertices.reshape(-1, 2))
    arrays = {"vertices": raw.vertices}
    for k, b in enumerate(raw.edge_blocks):
        arrays[f"edge_block_{k}"] = b.node_pairs
    for k, t in enumerate(raw.element_blocks):
        arrays[f"tri_block_{k}"] = t
    arrays["edge_block_names"] = np.array([b.physical_name for b in raw.edge_blocks])
    np.savez_compressed(os.path.join(HERE, "airfoil_mesh.npz"), **arrays)
    # the reference's configured run: cfl <= 0 selects the formula
    o = Oracle(raw=raw, order=2, ncell_gp=6, nedge_gp=3, hcr=1.4, cfl=-1.0, final_time=5.0, final_step=20,
               freestream=REF_FS)
    U = o.initial_solution()
    R = o.new_state()
    t, s = o.time_march(R, U)
    np.savez_compressed(os.path.join(HERE, "airfoil_run.npz"), U20=U, t20=np.array(t), steps=np.array(s),
                        cfl=np.array(o.cfl))
    print("airfoil:", o.ne, "elements, t after 20 steps", t)


def ogrid():
    raw = naca0012_ogrid(16, 8)
    fs = (1.25, 0.8, 1.0, 1.0 / 1.4)
    o = Oracle(raw=raw, order=2, ncell_gp=6, nedge_gp=3, cfl=0.1, final_time=1.0e30, final_step=3, freestream=fs)
    U0 = o.initial_solution()
    R0 = o.new_state()
    o.compute_residuals(R0, U0)
    rng = np.random.default_rng(2024)
    noise = rng.standard_normal(U0[:, :, 1:].shape) * np.abs(U0[:, :, :1])
    Up = U0.copy()
    Up[:, :, 1:] += 0.03 * noise  # mild: residual well defined
    Rp = o.new_state()
    o.compute_residuals(Rp, Up)
    Ut = U0.copy()
    Ut[:, :, 1:] += 0.1 * noise  # strong: limiter active
    Ul = Ut.copy()
    n = o.apply_limiter(Ul)
    assert np.isfinite(Ul).all() and n > 0
    U3 = U0.copy()
    R3 = o.new_state()
    t, s = o.time_march(R3, U3)
    np.savez_compressed(os.path.join(HERE, "ogrid16x8.npz"), U0=U0, R0=R0, Up=Up, Rp=Rp, Ut=Ut, Ul=Ul,
                        troubled=np.array(n), U3=U3, R3=R3, t3=np.array(t), dt0=np.array(o.compute_time_step(U0)))
    print("ogrid16x8: troubled", n, "t3", t)


C2_CHECKPOINTS = (200, 2000)


def c2_sample(ne, boundary_elements):
    return np.union1d(np.arange(0, ne, 128), boundary_elements).astype(np.int64)


C2_PERTURBATION = 1e-15  # relative, seeded normal: the round-off-sized twin run


def _c2_march(o, U, R, sample, prefix, out):
    done, t = 0, 0.0
    for n in C2_CHECKPOINTS:
        while done < n:
            dt = o.compute_time_step(U)
            o.rk3(R, U, dt)
            t += dt
            done += 1
        out[f"{prefix}t{n}"] = np.array(t)
        out[f"{prefix}sum{n}"] = U.sum(axis=0)
        out[f"{prefix}sumsq{n}"] = (U * U).sum(axis=0)
        out[f"{prefix}U{n}"] = U[sample]
        out[f"{prefix}troubled{n}"] = np.array(int(o.troubled_flags(U).sum()))
        print(f"c2 {prefix or 'oracle'}: {n} steps, t = {t}", flush=True)


def c2_run(threads=8, only_twin=False):
    """The oracle's run, and its twin from the initial state times (1 + 1e-15 N(0,1)) (seed 5): the
    spread between the two measures how far round-off alone carries this impulsive start."""
    from dgm_in_rust_b200 import freestream_quantity, process_mesh
    raw = naca0012_ogrid(256, 128)
    fs = (1.25, 0.8, 1.0, 1.0 / 1.4)
    mesh = process_mesh(raw, freestream_quantity(fs[1], fs[0], fs[2], fs[3], 1.4), 1.4)
    o = Oracle(raw=raw, order=2, ncell_gp=6, nedge_gp=3, cfl=0.1, final_time=1.0e30, final_step=0,
               limiter=True, threads=threads, freestream=fs)
    sample = c2_sample(o.ne, mesh.boundary_element_indices)
    path = os.path.join(HERE, "c2_run.npz")
    out = dict(np.load(path)) if only_twin else {"sample": sample}
    if not only_twin:
        _c2_march(o, o.initial_solution(), o.new_state(), sample, "", out)
    U = o.initial_solution()
    U *= 1.0 + C2_PERTURBATION * np.random.default_rng(5).standard_normal(U.shape)
    _c2_march(o, U, o.new_state(), sample, "twin_", out)
    np.savez_compressed(path, **out)


def reference_files(checkout):
    for src, dst in (("inputfiles/airfoil.msh", "reference_airfoil.msh.gz"),
                     ("outputfiles/mesh.vtk", "reference_mesh.vtk.gz")):
        with open(os.path.join(checkout, src), "rb") as f:
            data = f.read()
        with open(os.path.join(HERE, dst), "wb") as f:
            f.write(gzip.compress(data, compresslevel=9, mtime=0))


if __name__ == "__main__":
    if len(sys.argv) == 2 and sys.argv[1] == "--c2-run":
        c2_run()
        raise SystemExit(0)
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_golden.py <path of a DGM_in_rust checkout> | --c2-run")
    AIRFOIL = os.path.join(sys.argv[1], "inputfiles", "airfoil.msh")
    reference_files(sys.argv[1])
    airfoil()
    ogrid()
