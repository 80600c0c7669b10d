"""Synthetic pressure systems of the benchmark configurations.

Every case is generated from a fixed seed (20261203 + config index by default) by the library's
C++ generators (``include/cfdb_synth.h``); none is a public dataset.

* cavity   -- uniform n^3 hex box, rAU = 1 (face coefficient A_f/|d|), flux u_f . S_f with
              u_f ~ U(-1,1)^3, source = -div(flux), zero mean; reference cell 0 pinned.
* graded   -- n^3 hex box graded two-sided (ratio r between neighbouring cells, smallest at all
              walls), rAU_c = V_c X_c with X_c ~ LogNormal(0, sigma), flux u_f . S_f, source =
              N(0,1) - div(flux), zero mean; reference cell 0 pinned.
* tet      -- n^3 box cells split into 6 tets, interior nodes jittered by U(-j h, j h),
              over-relaxed delta coefficients, otherwise as graded.
Walls are pure Neumann (wall flux 0), as in the lid-driven cavity's pressure equation.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

SEED_BASE = 20261203


@dataclass
class PressureCase:
    name: str
    mesh: object
    n: int
    n_faces: int
    owner: np.ndarray      # internal faces
    neighbour: np.ndarray
    flux: np.ndarray       # phiHbyA on internal faces
    gamma: np.ndarray      # rAU_f
    delta: np.ndarray      # over-relaxed delta coefficients
    source0: np.ndarray    # cell source before the divergence term
    ref_cell: int = 0
    ref_value: float = 0.0

    def finalize(self, upper, lower, diag, div):
        """flow_solver.cpp:768-770 and 794-796: source -= div; set_reference(ref, value).
        Returns (diag, source) as new arrays (the LDU coefficients are final after this)."""
        d = np.array(diag, dtype=np.float64, copy=True)
        s = self.source0 - np.asarray(div)
        c = self.ref_cell
        s[c] += d[c] * self.ref_value
        d[c] += d[c]
        return d, s


def _case(name, mesh, sigma, unit_rau, rhs_kind, seed) -> PressureCase:
    gamma, flux, src = mesh.pressure_inputs(sigma=sigma, unit_rau=unit_rau, flux_kind=0,
                                            rhs_kind=rhs_kind, seed=seed)
    nif = mesh.n_internal_faces
    return PressureCase(name, mesh, mesh.n_cells, nif, mesh.owner[:nif].copy(),
                        mesh.neighbour.copy(), flux, gamma, mesh.delta.copy(), src)


def cavity(n=32, seed=SEED_BASE + 0) -> PressureCase:
    from . import Mesh
    m = Mesh.box(n, n, n)
    return _case(f"cavity{n}", m, sigma=0.0, unit_rau=True, rhs_kind=0, seed=seed)


def graded(n=128, ratio=1.05, sigma=0.5, seed=SEED_BASE + 1) -> PressureCase:
    from . import Mesh, positions_two_sided
    xs = positions_two_sided(n, ratio)
    m = Mesh.box(n, n, n, xs, xs, xs)
    return _case(f"graded{n}", m, sigma=sigma, unit_rau=False, rhs_kind=1, seed=seed)


def tet(n=95, jitter=0.2, sigma=1.0, seed=SEED_BASE + 2) -> PressureCase:
    from . import Mesh
    m = Mesh.tet(n, n, n, jitter=jitter, seed=seed)
    return _case(f"tet{n}", m, sigma=sigma, unit_rau=False, rhs_kind=1, seed=seed + 1000)


def box_edges(count=256, lo=8, hi=64, seed=SEED_BASE + 3):
    """Edge lengths of the batched configuration: round(exp(U(ln lo, ln hi)))."""
    rng = np.random.default_rng(seed)
    return [int(round(float(np.exp(rng.uniform(np.log(lo), np.log(hi)))))) for _ in range(count)]


def batch_box(edge, sigma=0.5, seed=0) -> PressureCase:
    from . import Mesh
    m = Mesh.box(edge, edge, edge)
    return _case(f"box{edge}", m, sigma=sigma, unit_rau=False, rhs_kind=1, seed=seed)


# serving mix: box meshes with edge log-uniform in [16, 128] and jittered-tet meshes of 0.1-2M
# cells, one tet request in four. The pool holds log-spaced sizes of each kind; a request picks
# its kind, then a pool size uniformly (log-uniform in size).
SERVE_BOX_EDGES = (16, 23, 32, 45, 64, 91, 128)
SERVE_TET_EDGES = (26, 35, 46, 55, 69)  # 6 n^3 cells: 0.105M, 0.257M, 0.584M, 0.998M, 1.97M


def serve_pool(seed=SEED_BASE + 4, box_edges=SERVE_BOX_EDGES, tet_edges=SERVE_TET_EDGES):
    """Pressure cases of the serving pool, each with its finalized LDU coefficients:
    [(kind, case, diag, upper, lower, source)]."""
    from . import assemble_convection_diffusion
    out = []
    for i, e in enumerate(box_edges):
        out.append(("box", graded_box(e, seed=seed + i)))
    for i, e in enumerate(tet_edges):
        out.append(("tet", tet(e, seed=seed + 100 + i)))
    res = []
    for kind, c in out:
        up, lo = np.zeros(c.n_faces), np.zeros(c.n_faces)
        dg, dv = np.zeros(c.n), np.zeros(c.n)
        assemble_convection_diffusion(c.n, c.n_faces, c.owner, c.neighbour, c.flux, c.gamma,
                                      c.delta, 0.0, up, lo, dg, dv)  # on the device
        d, s = c.finalize(up, lo, dg, dv)
        res.append((kind, c, d, up, lo, s))
    return res


def graded_box(edge, sigma=0.5, seed=0) -> PressureCase:
    """Uniform box of the serving mix (rAU log-normal, random zero-mean source)."""
    return batch_box(edge, sigma=sigma, seed=seed)
