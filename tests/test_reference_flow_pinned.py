"""FlowSolver::pressure_correction (flow_solver.cpp:673-847), the reference's own code compiled
unchanged against the Eigen stand-in, against the oracle's face-by-face restatement, on the CPU.

The reference runs one SIMPLE iteration step by step (assemble_momentum, solve_momentum,
pressure_correction) from a seeded state on a graded hex box and a jittered tet box with an
inlet, an outlet, walls (one moving) and a symmetry plane. The restatement recomputes the
pressure correction from the same momentum system and velocity with its own loops (HbyA and
rAU, predicted face flux with the boundary conditions and the relaxation-independent term,
pressure matrix with the boundary terms, non-orthogonal correctors with the two-pass Gauss
gradient, conservative flux, relaxation, velocity correction); its pressure solves go through
the reference's own LduMatrix::solve. Velocity, pressure and face flux come out equal bit for
bit, so every loop of the restatement is the reference's (the device step is checked against
the same restatement in test_gpu_pressure_step.py and test_gpu_flow_step.py).
"""
import numpy as np
import pytest

RX = pytest.importorskip("oracle.reference")
if not RX.available() or not hasattr(RX.lib(), "refx_flow_create"):
    pytest.skip("reference build with FlowSolver not available", allow_module_level=True)

from oracle import flowref as F  # noqa: E402


@pytest.mark.parametrize("kind,n_corr,relax_p,majumdar", [
    ("box", 0, True, True), ("box", 1, False, False), ("tet", 1, True, True), ("tet", 2, True, False),
])
def test_pressure_correction_equals_the_reference_flow_solver(kind, n_corr, relax_p, majumdar):
    step = F.reference_step(kind, n_corr, relax_p=relax_p, majumdar=majumdar)
    got = F.restated_step(step)
    assert got["initial"] == step["initial"]
    assert np.array_equal(got["p_out"], step["p_out"])
    assert np.array_equal(got["phi_out"], step["phi_out"])
    assert np.array_equal(got["u_out"], step["u_out"])
    # the correctors changed the pressure and the step did real work
    assert len(got["solves"]) == n_corr + 1
    assert not np.array_equal(step["p_out"], step["p"])


def test_delta_coefficients_and_boundary_of_the_flow_solver():
    """The FlowSolver's geometry and boundary conditions, as the restatement reads them:
    FvGeometry's delta coefficients equal the oracle's, and every patch got its condition."""
    import oracle as O
    step = F.reference_step("tet", 0)
    v = F.mesh_view(step)
    delta, _ = O.fv_delta_corrections(v.n_internal_faces, v.owner, v.neighbour, v.face_areas, v.face_centres,
                                      v.cell_centres)
    assert np.array_equal(delta, step["delta"])
    ni = v.n_internal_faces
    fc = v.face_centres[ni:]
    kinds = step["kinds"]
    assert np.all(kinds[np.isclose(fc[:, 0], 0.0)] == 0)   # inlet
    assert np.all(kinds[np.isclose(fc[:, 0], 1.0)] == 2)   # outlet
    assert np.all(step["outlet_pressure"][kinds == 2] == 0.25)
    moving = np.isclose(fc[:, 1], 1.0) & ~np.isclose(fc[:, 0], 0.0) & ~np.isclose(fc[:, 0], 1.0)
    assert np.all(step["fixed_velocity"][moving] == [0.3, 0.0, 0.0])
    assert set(np.unique(kinds)) == {0, 1, 2, 3}


@pytest.mark.parametrize("kind", ["box", "tet"])
def test_product_mesh_equals_the_flow_solver_mesh(kind):
    """The product's host mesh generator gives the reference's mesh for these cases (the device
    step of test_gpu_flow_step.py runs on it)."""
    import cfd_b200 as cb
    r = F.mesh(kind)
    _, weights, _ = r.fv()
    if kind == "box":
        m = cb.Mesh.box(len(F.BOX_XS) - 1, 5, 4, xs=F.BOX_XS)
    else:
        m = cb.Mesh.tet(*F.TET_N, jitter=F.TET_JITTER, seed=F.TET_SEED)
    assert (m.n_cells, m.n_faces, m.n_internal_faces) == (r.n_cells, r.n_faces, r.n_internal_faces)
    assert np.array_equal(m.owner, r.owner) and np.array_equal(m.neighbour, r.neighbour)
    for a in ("face_areas", "face_centres", "cell_centres", "cell_volumes"):
        assert np.array_equal(getattr(m, a), getattr(r, a)), a
    assert np.array_equal(m.weights, weights)
