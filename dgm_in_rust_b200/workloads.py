"""Synthetic workloads: seeded sets of NACA 0012 O-grid solves.

The reference solves one configured mesh per run; these generators produce the many-instance
and request-stream inputs used to measure batching and serving.  All meshes are synthetic
(no dataset is involved): NACA 0012 O-grids from :func:`dgm_in_rust_b200.mesh.naca0012_ogrid`,
uniform free-stream starts with rho = 1, p = 1/gamma (sound speed 1).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .mesh import freestream_quantity, naca0012_ogrid, process_mesh

__all__ = ["Instance", "batch_instances", "request_stream", "instance_mesh"]

HCR = 1.4
RHO_INF = 1.0
P_INF = 1.0 / HCR


@dataclasses.dataclass
class Instance:
    ni: int
    nj: int
    mach: float
    aoa: float
    order: int

    @property
    def elements(self) -> int:
        return 2 * self.ni * self.nj

    @property
    def dofs(self) -> int:
        nb = (self.order + 1) * (self.order + 2) // 2
        return self.elements * 4 * nb


def batch_instances(n: int = 256, seed: int = 2024, orders=(1, 2)) -> list:
    """Ni uniform on {32, 64, ..., 256}, Nj = Ni / 2, Mach ~ U[0.3, 0.85], AoA ~ U[-4, 6] deg,
    order drawn uniformly from ``orders`` (numpy default_rng(seed))."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        ni = int(rng.integers(1, 9)) * 32
        out.append(Instance(ni=ni, nj=ni // 2, mach=float(rng.uniform(0.3, 0.85)),
                            aoa=float(rng.uniform(-4.0, 6.0)), order=int(orders[int(rng.integers(0, len(orders)))])))
    return out


def request_stream(n: int, rate: float, seed: int = 7, e_min: float = 2.0e3, e_max: float = 5.0e5,
                   orders=(1, 2, 3)) -> list:
    """Poisson arrivals at ``rate`` requests/s; triangle count log-uniform in [e_min, e_max] with an
    O-grid of aspect 2:1 (Ni = even(sqrt(E)), Nj = Ni / 2); Mach ~ U[0.3, 0.85], AoA ~ U[-4, 6] deg,
    order uniform on ``orders``.  Returns [(arrival_time_s, Instance)]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(n):
        t += float(rng.exponential(1.0 / rate))
        e = math.exp(rng.uniform(math.log(e_min), math.log(e_max)))
        ni = max(8, int(round(math.sqrt(e) / 2.0)) * 2)
        out.append((t, Instance(ni=ni, nj=ni // 2, mach=float(rng.uniform(0.3, 0.85)),
                                aoa=float(rng.uniform(-4.0, 6.0)), order=int(orders[int(rng.integers(0, len(orders)))]))))
    return out


def instance_mesh(inst: Instance):
    """Processed mesh and free-stream initial condition of an instance."""
    from .solver import InitialSolution
    raw = naca0012_ogrid(inst.ni, inst.nj)
    mesh = process_mesh(raw, freestream_quantity(inst.mach, inst.aoa, RHO_INF, P_INF, HCR), HCR)
    return mesh, InitialSolution(RHO_INF, inst.aoa, inst.mach, P_INF)
