"""The reference's FlowSolver pressure correction and its restatement, side by side -- TEST
INFRASTRUCTURE ONLY.

``reference_step`` runs one SIMPLE iteration of the reference's own ``FlowSolver`` (compiled
unchanged against the Eigen stand-in, ``oracle/ref_flow_shim.cpp``) step by step on a small box
or tet mesh: ``assemble_momentum``, ``solve_momentum``, then ``pressure_correction``
(flow_solver.cpp:673-847), and records every input and output of the pressure correction.

``restated_step`` recomputes the same pressure correction from those inputs with the oracle's
face-by-face restatement (``oracle.pressure_step_parts``, ``pressure_gradient``,
``non_orth_source``, ``correct_flux_all``, ``relax``, ``correct_velocity``); its pressure solves
go through the reference's own ``LduMatrix::solve`` with a fresh ``AmgCache``, as the
FlowSolver's do. Equal fields bit for bit mean that every face and cell loop of the restatement
(which the device step is checked against) is the reference's.
"""
from __future__ import annotations

import types

import numpy as np

import oracle as O

from . import reference as RX

# inlet at x = 0, outlet at x = 1 (p = 0.25), walls at y = 0 and z = 1, a moving wall at y = 1,
# symmetry at z = 0 (patch p = 2 * direction + side, as box_tag_quads / tet_tags tag them)
PATCHES = [("VelocityInlet", (1.0, 0.0, 0.0), 0.0), ("PressureOutlet", (0.0, 0.0, 0.0), 0.25),
           ("Wall", (0.0, 0.0, 0.0), 0.0), ("Wall", (0.3, 0.0, 0.0), 0.0),
           ("Symmetry", (0.0, 0.0, 0.0), 0.0), ("Wall", (0.0, 0.0, 0.0), 0.0)]
BOX_XS = np.array([0.0, 0.08, 0.2, 0.35, 0.52, 0.7, 0.86, 1.0])
TET_N, TET_JITTER, TET_SEED = (5, 4, 4), 0.2, 3


def mesh(kind: str) -> "RX.RefMesh":
    """Graded 7 x 5 x 4 hex box, or the jittered 5 x 4 x 4 x 6 tet box, built by the reference."""
    if kind == "box":
        return RX.RefMesh.hex_box(BOX_XS, np.linspace(0.0, 1.0, 6), np.linspace(0.0, 1.0, 5))
    nx, ny, nz = TET_N
    pts = RX.jittered_lattice(nx, ny, nz, np.linspace(0.0, 1.0, nx + 1), np.linspace(0.0, 1.0, ny + 1),
                              np.linspace(0.0, 1.0, nz + 1), TET_JITTER, TET_SEED)
    return RX.RefMesh.tet_box(nx, ny, nz, pts)


def reference_step(kind: str, n_corr: int, relax_p=True, majumdar=True, alpha_u=0.7, alpha_p=0.3,
                   p_solver=("GpuCg", 1e-10, 0.01, 500), seed=5) -> dict:
    """One SIMPLE iteration of the reference FlowSolver from a seeded state, step by step."""
    m = mesh(kind)
    delta, weights, _ = m.fv()
    fl = RX.RefFlow(m, PATCHES, alpha_u=alpha_u, alpha_p=alpha_p, n_non_orth=n_corr, p_solver=p_solver)
    n, nf = m.n_cells, m.n_faces
    rng = np.random.default_rng(seed)
    fl.set_state(rng.standard_normal((n, 3)) * 0.3 + np.array([1.0, 0.0, 0.0]), 0.1 * rng.standard_normal(n),
                 0.01 * rng.standard_normal(nf))
    u_prev, _, phi_prev = fl.state()
    mom = fl.momentum(0.0, True)
    fl.solve_momentum()
    u, p, phi = fl.state()
    kinds, pout, ufix = fl.boundary()
    initial = fl.pressure_correction(relax_p, u_prev if majumdar else None, phi_prev if majumdar else None)
    u_out, p_out, phi_out = fl.state()
    fl.close()
    return dict(mesh=m, delta=delta, weights=weights, kinds=kinds, outlet_pressure=pout, fixed_velocity=ufix,
                mom_diag=mom[0], mom_upper=mom[1], mom_lower=mom[2], mom_source=mom[3], u=u, p=p, phi=phi,
                u_prev=u_prev if majumdar else None, phi_prev=phi_prev if majumdar else None,
                n_corr=n_corr, relax_p=relax_p, alpha_u=alpha_u, alpha_p=alpha_p, p_solver=p_solver,
                initial=initial, u_out=u_out, p_out=p_out, phi_out=phi_out)


def mesh_view(step: dict):
    """The attributes of the reference mesh that the oracle's restatement reads."""
    m = step["mesh"]
    return types.SimpleNamespace(n_cells=m.n_cells, n_faces=m.n_faces, n_internal_faces=m.n_internal_faces,
                                 owner=m.owner, neighbour=m.neighbour, weights=step["weights"],
                                 face_areas=m.face_areas, face_centres=m.face_centres,
                                 cell_centres=m.cell_centres, cell_volumes=m.cell_volumes)


def restated_step(step: dict) -> dict:
    """The pressure correction of ``step`` by the oracle's restatement, its solves by the
    reference's LduMatrix::solve (GpuCg with a persistent AmgCache, as FlowSolver's p_amg_)."""
    m, v = step["mesh"], mesh_view(step)
    ni = m.n_internal_faces
    parts = O.pressure_step_parts(v, step["kinds"], step["outlet_pressure"], step["mom_diag"], step["mom_upper"],
                                  step["mom_lower"], step["mom_source"], step["u"], step["fixed_velocity"],
                                  step["u_prev"], step["phi_prev"], alpha_u=step["alpha_u"])
    grad_args = (m.n_cells, ni, m.owner, m.neighbour, step["weights"], m.face_areas, m.face_centres,
                 m.cell_centres, m.cell_volumes, step["kinds"], step["outlet_pressure"])
    ldu = RX.RefLdu(m)
    p_new = np.array(step["p"], np.float64)
    solves = []
    non_orth = np.zeros(ni)
    for corr in range(step["n_corr"] + 1):
        non_orth, source = np.zeros(ni), parts["source"]
        if corr > 0 or step["n_corr"] > 0:
            g = O.pressure_gradient(*grad_args, p_new)
            non_orth, source = O.non_orth_source(v, g, parts["rau_f"], parts["source"])
        ldu.set(parts["diag"], parts["upper"], parts["lower"], source)
        name, tol, rel, maxit = step["p_solver"]
        r = ldu.solve(p_new, name, tol, rel, maxit, max_age=20)
        solves.append(dict(r, source=np.array(source), p=p_new.copy()))
    ldu.close()
    phi = O.correct_flux_all(v, step["kinds"], step["outlet_pressure"], parts["phi_hbya"], parts["rau_f"],
                             parts["delta"], non_orth, p_new)
    p = O.relax(step["p"], p_new, step["alpha_p"]) if step["relax_p"] else p_new
    u = O.correct_velocity(parts["hbya"], parts["rau"], O.pressure_gradient(*grad_args, p))
    return dict(parts=parts, solves=solves, non_orth=non_orth, p_new=p_new, initial=solves[0]["initial_residual"],
                u_out=u, p_out=p, phi_out=phi)
