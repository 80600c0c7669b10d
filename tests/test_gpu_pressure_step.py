"""FlowSolver::pressure_correction with every array on the device (cfd_b200.pressure): each step
against the oracle's face-by-face restatement of flow_solver.cpp:673-847, bit for bit: HbyA,
rAU, predicted face flux (with the relaxation-independent term), pressure matrix with boundary
terms, non-orthogonal corrector sources, conservative flux, relaxed pressure and corrected
velocity; the pressure solves themselves meet their tolerance."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _setup(cb, kind):
    m = cb.Mesh.box(7, 5, 4, xs=np.array([0.0, 0.08, 0.2, 0.35, 0.52, 0.7, 0.86, 1.0])) if kind == "box" \
        else cb.Mesh.tet(5, 4, 4, jitter=0.2, seed=3)
    ni = m.n_internal_faces
    fc_b = m.face_centres[ni:]
    kinds = np.full(m.n_faces - ni, int(cb.BoundaryKind.Wall), np.int32)
    kinds[np.isclose(fc_b[:, 0], 0.0)] = int(cb.BoundaryKind.VelocityInlet)
    kinds[np.isclose(fc_b[:, 0], 1.0)] = int(cb.BoundaryKind.PressureOutlet)
    kinds[np.isclose(fc_b[:, 2], 0.0)] = int(cb.BoundaryKind.Symmetry)
    pout = np.where(kinds == int(cb.BoundaryKind.PressureOutlet), 0.25, 0.0)
    ufix = np.zeros((m.n_faces - ni, 3))
    ufix[kinds == int(cb.BoundaryKind.VelocityInlet)] = [1.0, 0.0, 0.0]
    rng = np.random.default_rng(17)
    n = m.n_cells
    mom = dict(mom_diag=rng.uniform(2.0, 4.0, (n, 3)), mom_upper=-rng.uniform(0.1, 0.5, ni),
               mom_lower=-rng.uniform(0.1, 0.5, ni), mom_source=rng.standard_normal((n, 3)))
    u = rng.standard_normal((n, 3))
    u_prev = u + 0.1 * rng.standard_normal((n, 3))
    phi_prev = rng.standard_normal(m.n_faces)
    p = 0.1 * rng.standard_normal(n)
    return m, kinds, pout, ufix, mom, u, u_prev, phi_prev, p


@pytest.mark.parametrize("kind,n_corr,majumdar", [("box", 0, False), ("tet", 1, True)])
def test_pressure_correction_step_bitwise(gpu, kind, n_corr, majumdar):
    import torch
    cb = gpu
    from cfd_b200 import pressure as P
    m, kinds, pout, ufix, mom, u0, u_prev, phi_prev, p0 = _setup(cb, kind)
    ni = m.n_internal_faces
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")  # noqa: E731
    ds = cb.DeviceSolver(mesh=(m.n_cells, m.owner[:ni], m.neighbour))
    fv = cb.FvGeometry(m, kinds, pout)
    u, p = T(u0), T(p0)
    s = P.PressureSettings(alpha_u=0.7, alpha_p=0.3, n_non_orth_correctors=n_corr, ref_cell=-1,
                           p_solver=cb.LduSettings(tolerance=1e-13, rel_tolerance=1e-10, max_iterations=2000))
    keep = {}
    init = P.pressure_correction(ds, fv, T(mom["mom_diag"]), T(mom["mom_upper"]), T(mom["mom_lower"]),
                                 T(mom["mom_source"]), u, p, T(ufix), s, relax_p=True,
                                 u_prev=T(u_prev) if majumdar else None,
                                 phi_prev=T(phi_prev) if majumdar else None, keep=keep)
    torch.cuda.synchronize()
    h = lambda t: t.cpu().numpy()  # noqa: E731
    want = O.pressure_step_parts(m, kinds, pout, mom["mom_diag"], mom["mom_upper"], mom["mom_lower"],
                                 mom["mom_source"], u0, ufix, u_prev if majumdar else None,
                                 phi_prev if majumdar else None, alpha_u=0.7)
    for k in ("hbya", "rau", "phi_hbya", "rau_f", "upper", "lower", "diag"):
        assert np.array_equal(h(keep[k]), want[k]), k
    assert np.array_equal(h(keep["base_source"]), want["source"])
    # the corrector sources use the gradient of the pressure before each solve
    grad_args = (m.n_cells, ni, m.owner, m.neighbour, m.weights, m.face_areas, m.face_centres,
                 m.cell_centres, m.cell_volumes, kinds, pout)
    p_before = p0
    non_orth = np.zeros(ni)
    for k, (res, p_after, src) in enumerate(keep["solves"]):
        if n_corr > 0:
            g = O.pressure_gradient(*grad_args, p_before)
            non_orth, want_src = O.non_orth_source(m, g, want["rau_f"], want["source"])
            assert np.array_equal(h(src), want_src), f"corrector source {k}"
        else:
            assert np.array_equal(h(src), want["source"])
        a = O.ldu_to_csr(O.build_pattern(m.n_cells, m.owner[:ni], m.neighbour), want["diag"],
                         want["upper"], want["lower"])
        x = h(p_after)
        assert np.linalg.norm(h(src) - a.matvec(x)) <= 1e-8 * np.linalg.norm(h(src))
        p_before = x
    assert init == keep["solves"][0][0].initial_residual
    if n_corr > 0:
        assert np.array_equal(h(keep["non_orth"])[:ni], non_orth)
    p_new = h(keep["p_new"])
    assert np.array_equal(h(keep["phi"]), O.correct_flux_all(m, kinds, pout, want["phi_hbya"], want["rau_f"],
                                                             want["delta"], non_orth, p_new))
    p_want = O.relax(p0, p_new, 0.3)
    assert np.array_equal(h(p), p_want)
    assert np.array_equal(h(u), O.correct_velocity(want["hbya"], want["rau"], O.pressure_gradient(*grad_args, p_want)))
    fv.close()
