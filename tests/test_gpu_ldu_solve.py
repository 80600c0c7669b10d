"""The persistent LDU solve (cfdb_system_solve_ldu) against the reference's LduMatrix::solve
semantics (ldu_matrix.cpp:111-131, 287-366): the normalised residuals before and after (the
oracle's restatement of ldu_matrix.cpp:65-103), the early return below the tolerance, the
absolute CG target, the AmgCache rebuild every max_age CG solves, and BiCGStab without a
hierarchy."""
import numpy as np
import pytest

import oracle as O
from cfd_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _system(case):
    up, lo, dg, dv = O.assemble(case.n, case.owner, case.neighbour, case.flux, case.gamma,
                                case.delta, 0.0)
    diag, src = case.finalize(up, lo, dg, dv)
    return up, lo, diag, src


@pytest.fixture(scope="module")
def graded(gpu):
    cb = gpu
    case = W.graded(16)
    up, lo, diag, src = _system(case)
    nf = len(up)
    return cb, case, up, lo, diag, src, case.owner[:nf], case.neighbour


def _norm(own, nei, diag, up, lo, src, x):
    return O.normalised_residual(own, nei, diag, up, lo, src, x)


def test_residuals_and_target_follow_the_reference(graded):
    cb, case, up, lo, diag, src, own, nei = graded
    ds = cb.DeviceSolver(cb.build_csr_pattern(case.n, case.owner, case.neighbour))
    settings = cb.LduSettings(tolerance=1e-12, rel_tolerance=1e-6)
    amg = cb.AmgSettings(strength_threshold=0.04)
    rng = np.random.default_rng(3)
    x0 = rng.standard_normal(case.n)
    x = x0.copy()
    r = ds.solve_ldu(diag, up, lo, src, x, settings, amg)
    assert r.amg_rebuilt and r.iterations > 0
    init = _norm(own, nei, diag, up, lo, src, x0)
    assert r.initial_residual == pytest.approx(init, rel=1e-12)
    assert r.final_residual == pytest.approx(_norm(own, nei, diag, up, lo, src, x), rel=1e-6)
    # the same solve through DeviceSolver.solve with the reference's absolute target
    a = O.ldu_to_csr(O.build_pattern(case.n, case.owner, case.neighbour), diag, up, lo)
    r0 = np.linalg.norm(src - a.matvec(x0))
    target = max(settings.rel_tolerance, settings.tolerance / max(init, 1e-20)) * r0
    ds2 = cb.DeviceSolver(cb.build_csr_pattern(case.n, case.owner, case.neighbour))
    ds2.setup_amg(diag, up, lo, amg)
    x2 = x0.copy()
    st = ds2.solve(diag, up, lo, src, x2, cb.Method.Cg, True, cb.SolveControl(target, 1000))
    assert st.iterations == r.iterations
    assert np.allclose(x, x2, rtol=0, atol=1e-9 * np.abs(x2).max())


def test_below_tolerance_returns_without_solving(graded):
    cb, case, up, lo, diag, src, own, nei = graded
    ds = cb.DeviceSolver(cb.build_csr_pattern(case.n, case.owner, case.neighbour))
    x = np.zeros(case.n)
    r = ds.solve_ldu(diag, up, lo, src, x, cb.LduSettings(tolerance=1e-13, rel_tolerance=0.0))
    x_conv = x.copy()
    r2 = ds.solve_ldu(diag, up, lo, src, x, cb.LduSettings(tolerance=2.0 * r.final_residual))
    assert r2.iterations == 0 and not r2.amg_rebuilt
    assert r2.final_residual == r2.initial_residual and np.array_equal(x, x_conv)


def test_hierarchy_rebuilt_every_max_age_cg_solves(graded):
    cb, case, up, lo, diag, src, own, nei = graded
    ds = cb.DeviceSolver(cb.build_csr_pattern(case.n, case.owner, case.neighbour))
    s = cb.LduSettings(tolerance=1e-14, rel_tolerance=1e-8, max_age=3)
    rebuilt = []
    for k in range(7):
        x = np.zeros(case.n)
        scale = 1.0 + 0.01 * k  # a new matrix every call
        r = ds.solve_ldu(diag * scale, up * scale, lo * scale, src, x, s)
        rebuilt.append(r.amg_rebuilt)
        assert r.final_residual < r.initial_residual
    assert rebuilt == [True, False, False, True, False, False, True]


def test_bicgstab_and_device_arrays(graded):
    import torch
    cb, case, up, lo, diag, src, own, nei = graded
    s = cb.LduSettings(method=int(cb.Method.BiCgStab), tolerance=1e-14, rel_tolerance=1e-8)
    ds = cb.DeviceSolver(cb.build_csr_pattern(case.n, case.owner, case.neighbour))
    x = np.zeros(case.n)
    r = ds.solve_ldu(diag, up, lo, src, x, s)
    assert not r.amg_rebuilt and r.final_residual < 1e-6 * r.initial_residual
    t = lambda v: torch.as_tensor(v, dtype=torch.float64, device="cuda")  # noqa: E731
    ds2 = cb.DeviceSolver(cb.build_csr_pattern(case.n, case.owner, case.neighbour))
    xd = t(np.zeros(case.n))
    r2 = ds2.solve_ldu(t(diag), t(up), t(lo), t(src), xd, s)
    torch.cuda.synchronize()
    assert r2.iterations == r.iterations and r2.final_residual == r.final_residual
    assert np.array_equal(xd.cpu().numpy(), x)


@pytest.mark.parametrize("name", ["cavity12", "tet8", "graded10", "cavity32"])
def test_solve_ldu_matches_the_reference_ldu_matrix(gpu, name):
    """cfdb_system_solve_ldu against the reference's own LduMatrix::solve -> solve_persistent
    (ldu_matrix.cpp:111-131, 287-366, compiled unchanged into oracle/_ref with the Eigen
    stand-in, on the reference's host DeviceSolver and its own AmgPreconditioner::setup at the
    default strength threshold 0.08): the same normalised residual before, the same AmgCache
    rebuild sequence over repeated solves of changing matrices, iterations within 1, and both
    final residuals below the translated target."""
    RX = pytest.importorskip("oracle.reference")
    if not RX.available():
        pytest.skip("reference build with the Eigen stand-in not available")
    cb = gpu
    rc = {"cavity12": lambda: RX.cavity(12), "tet8": lambda: RX.tet(8), "graded10": lambda: RX.graded(10),
          "cavity32": lambda: RX.cavity(32)}[name]()
    up, lo, dg, dv = O.ref_assemble(rc.n, rc.owner, rc.neighbour, rc.flux, rc.gamma, rc.delta, 0.0)
    src = rc.source0 - dv
    diag = dg.copy()
    O.set_reference(diag, src, rc.ref_cell, rc.ref_value)
    ldu = RX.RefLdu(rc.mesh)
    ds = cb.DeviceSolver(cb.build_csr_pattern(rc.n, rc.owner, rc.neighbour))
    settings = dict(tolerance=1e-11, rel_tolerance=1e-6, max_age=2)
    rng = np.random.default_rng(12)
    for k in range(5):
        s = 1.0 + 0.05 * k  # a new matrix every call
        d_k, u_k, l_k = diag * s, up * s, lo * s
        x0 = 0.1 * rng.standard_normal(rc.n)
        ldu.set(d_k, u_k, l_k, src)
        x_ref = x0.copy()
        r_ref = ldu.solve(x_ref, "GpuCg", max_iterations=500, **settings)
        x = x0.copy()
        r = ds.solve_ldu(d_k, u_k, l_k, src, x, cb.LduSettings(max_iterations=500, **settings))
        assert r.initial_residual == pytest.approx(r_ref["initial_residual"], rel=1e-12)
        assert r.amg_rebuilt == (r_ref["amg_age"] == 1)
        assert abs(r.iterations - r_ref["iterations"]) <= 1
        target = max(settings["rel_tolerance"], settings["tolerance"] / r.initial_residual)
        # the CG target is on the 2-norm; the normalised residual tracks it within a small factor
        assert r.final_residual <= 5.0 * target * r.initial_residual
        assert r_ref["final_residual"] <= 5.0 * target * r_ref["initial_residual"]
        assert np.linalg.norm(x - x_ref) <= 1e-4 * np.linalg.norm(x_ref)
