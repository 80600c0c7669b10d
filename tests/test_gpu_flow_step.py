"""The device pressure correction (cfdb_pressure_correction_device through cfd_b200.pressure) on
the state of the reference's own FlowSolver (flow_solver.cpp:673-847, compiled unchanged against
the Eigen stand-in): its momentum system after assemble_momentum, its velocity after
solve_momentum, its pressure and face flux.

* Every array before the first solve (HbyA, rAU, predicted face flux and face rAU, pressure
  matrix with the boundary terms) equals, bit for bit, the restatement that
  test_reference_flow_pinned.py shows equal to the reference's FlowSolver.
* Both sides solve the pressure equation tightly (normalised residual 1e-12; the reference's
  fields move by < 5e-13 relative between that and 1e-14): the corrected velocity, pressure and
  face flux then agree with the reference's FlowSolver to 1e-9 relative (the solvers'
  arithmetic differs, so not bitwise); the first solve's initial normalised residual agrees to
  1e-12.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RX = pytest.importorskip("oracle.reference")
if not RX.available() or not hasattr(RX.lib(), "refx_flow_create"):
    pytest.skip("reference build with FlowSolver not available", allow_module_level=True)

from oracle import flowref as F  # noqa: E402


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.mark.parametrize("kind,n_corr,majumdar", [("box", 1, True), ("tet", 2, True), ("tet", 0, False)])
def test_device_step_on_the_reference_flow_solver_state(gpu, kind, n_corr, majumdar):
    import torch
    cb = gpu
    from cfd_b200 import pressure as P
    tight = ("GpuCg", 1e-12, 0.0, 2000)
    step = F.reference_step(kind, n_corr, majumdar=majumdar, p_solver=tight)
    want = F.restated_step(step)
    assert np.array_equal(want["p_out"], step["p_out"]) and np.array_equal(want["u_out"], step["u_out"])
    r = step["mesh"]
    if kind == "box":
        m = cb.Mesh.box(len(F.BOX_XS) - 1, 5, 4, xs=F.BOX_XS)
    else:
        m = cb.Mesh.tet(*F.TET_N, jitter=F.TET_JITTER, seed=F.TET_SEED)
    assert np.array_equal(m.owner, r.owner) and np.array_equal(m.face_areas, r.face_areas)
    n, nf, ni = m.n_cells, m.n_faces, m.n_internal_faces
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")  # noqa: E731
    ds = cb.DeviceSolver(mesh=(n, m.owner[:ni], m.neighbour))
    fv = cb.FvGeometry(m, step["kinds"], step["outlet_pressure"])
    s = P.PressureSettings(alpha_u=step["alpha_u"], alpha_p=step["alpha_p"], n_non_orth_correctors=n_corr,
                           ref_cell=-1, p_solver=cb.LduSettings(tolerance=1e-12, rel_tolerance=0.0,
                                                                max_iterations=2000))
    u, p, phi = T(step["u"]), T(step["p"]), torch.empty(nf, dtype=torch.float64, device="cuda")
    keep = {}
    init = P.pressure_correction(ds, fv, T(step["mom_diag"]), T(step["mom_upper"]), T(step["mom_lower"]),
                                 T(step["mom_source"]), u, p, T(step["fixed_velocity"]), s, relax_p=True,
                                 u_prev=None if step["u_prev"] is None else T(step["u_prev"]),
                                 phi_prev=None if step["phi_prev"] is None else T(step["phi_prev"]),
                                 phi=phi, keep=keep)
    torch.cuda.synchronize()
    h = lambda t: t.cpu().numpy()  # noqa: E731
    parts = want["parts"]
    for k in ("hbya", "rau", "phi_hbya", "rau_f", "diag"):
        assert np.array_equal(h(keep[k]), parts[k]), k
    assert np.array_equal(h(keep["upper"])[:ni], parts["upper"]) and np.array_equal(h(keep["lower"])[:ni],
                                                                                     parts["lower"])
    assert np.array_equal(h(keep["base_source"]), parts["source"])
    assert abs(init - step["initial"]) <= 1e-12 * abs(step["initial"])
    assert all(res.final_residual <= 1e-11 for res, _, _ in keep["solves"])
    assert _rel(h(p), step["p_out"]) <= 1e-9
    assert _rel(h(phi), step["phi_out"]) <= 1e-9
    assert _rel(h(u), step["u_out"]) <= 1e-9
