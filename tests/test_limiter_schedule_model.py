"""A host model of the limiter's scheduling, no GPU.

The reference limits element by element in index order, in place (src/spatial_disc/limiter/weno.rs:90,
write at :263): the detector and the reconstruction of element e read neighbours that may already
have been rewritten.  The device limiter settles elements in waves and comes in two schedules:
a grid barrier between a wave's scan and its reconstructions, or a queue that lets reconstructions
run while other elements of the same wave are still being scanned.  This model runs the same
settling rules on real mesh adjacency, with a stand-in detector and reconstruction that read the
element and its neighbours, and checks that both schedules -- the queue one under random
interleavings of scans and reconstructions -- end in exactly the sequential loop's state.
"""
import numpy as np
import pytest

from conftest import airfoil_raw
from dgm_in_rust_b200 import freestream_quantity, naca0012_ogrid, process_mesh


def _neighbours(raw):
    mesh = process_mesh(raw, freestream_quantity(0.8, 1.25, 1.0, 1.0 / 1.4, 1.4), 1.4)
    return [[int(n) for n in row if n >= 0] for row in mesh.elem_neighbours]


def _flag(v, e, nbrs, thr):
    """Stand-in for modified_kxrcf: reads the element and its neighbours."""
    return abs(v[e] - sum(v[n] for n in nbrs[e]) / len(nbrs[e])) > thr


def _recon(v, e, nbrs):
    """Stand-in for the WENO reconstruction: a new value from the element and its neighbours."""
    return 0.25 * v[e] + 0.75 * sum(v[n] for n in nbrs[e]) / len(nbrs[e]) + 0.01


def _sequential(v, nbrs, thr):
    v = list(v)
    for e in range(len(v)):
        if _flag(v, e, nbrs, thr):
            v[e] = _recon(v, e, nbrs)
    return v


def _waves(v, nbrs, thr, rng=None):
    """The device's settling rules.  rng None: barrier schedule (every scan of a wave before any
    reconstruction).  Otherwise queue schedule: scans and reconstructions of a wave interleave in a
    random order, a reconstruction any time after its element was enlisted."""
    v = list(v)
    ne = len(v)
    status = [0] * ne            # (wave << 2) | kind, kind 1 clean, 2 limited; 0 pending
    t0 = [False] * ne
    wave = 0
    while True:
        wave += 1
        pending = [e for e in range(ne) if (status[e] & 3) == 0]
        if not pending:
            return v, wave - 1
        order = list(pending) if rng is None else list(rng.permutation(pending))
        tasks = [("scan", e) for e in order]
        queue = []
        while tasks or queue:
            take_recon = queue and (not tasks or (rng is not None and rng.random() < 0.5))
            if take_recon:
                e = queue.pop(0 if rng is None else int(rng.integers(len(queue))))
                v[e] = _recon(v, e, nbrs)
                status[e] = (wave << 2) | 2
                continue
            _, e = tasks.pop(0)
            lower = [n for n in nbrs[e] if n < e]
            if wave == 1:
                t0[e] = _flag(v, e, nbrs, thr)   # may read neighbours rewritten in this wave
                ready = not lower
                any_mod = False
            else:
                ready = all((status[n] & 3) != 0 and (status[n] >> 2) < wave for n in lower)
                any_mod = any((status[n] & 3) == 2 and (status[n] >> 2) < wave for n in lower)
            if not ready:
                continue
            # wave 1: the flag just computed; later: recomputed only when a lower neighbour was
            # rewritten, else the wave-1 flag stands
            trouble = _flag(v, e, nbrs, thr) if any_mod else t0[e]
            if trouble:
                queue.append(e)
            else:
                status[e] = (wave << 2) | 1
        if rng is None:
            assert not queue


MESHES = {
    "ogrid_colored": lambda: naca0012_ogrid(24, 12),
    "ogrid_quad": lambda: naca0012_ogrid(24, 12, order="quad"),
    "airfoil": airfoil_raw,
}


@pytest.mark.parametrize("mesh", sorted(MESHES))
@pytest.mark.parametrize("thr", [0.05, 0.2])
def test_wave_schedules_match_sequential_loop(mesh, thr):
    nbrs = _neighbours(MESHES[mesh]())
    rng = np.random.default_rng(5)
    v0 = list(rng.standard_normal(len(nbrs)) * 0.3)
    ref = _sequential(v0, nbrs, thr)
    assert sum(a != b for a, b in zip(ref, v0)) > 0
    got, waves = _waves(v0, nbrs, thr)
    assert got == ref
    if mesh == "ogrid_colored":
        assert waves <= 2  # 2-colour numbering: chains of increasing-index neighbours are short
    for seed in range(3):
        got_q, waves_q = _waves(v0, nbrs, thr, np.random.default_rng(100 + seed))
        assert got_q == ref and waves_q == waves
