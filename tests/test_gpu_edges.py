"""Edge cases of the solver entry points, with the reference's semantics (test_gpu.cpp,
ldu_matrix.cpp): zero right-hand sides, already-converged guesses, iteration caps,
non-convergence reported in the stats rather than as an error, single cells, systems without
faces, and ragged batches."""
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
    ds = cb.DeviceSolver(cb.build_csr_pattern(case.n, case.owner, case.neighbour))
    ds.setup_amg(diag, up, lo)
    return cb, case, ds, up, lo, diag, src


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_zero_rhs_returns_zero_without_iterating(graded, precision):
    cb, case, ds, up, lo, diag, src = graded
    ds.set_precision(getattr(cb.Precision, precision))
    x = np.zeros(case.n)
    st = ds.solve(diag, up, lo, np.zeros(case.n), x, cb.Method.Cg, True, cb.SolveControl(1e-12, 100))
    assert st.converged and st.iterations == 0 and not x.any()


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_converged_guess_returns_at_once(graded, precision):
    """test_gpu.cpp:93-109: an input that already meets the tolerance returns 0 iterations and
    leaves x unchanged."""
    cb, case, ds, up, lo, diag, src = graded
    ds.set_precision(getattr(cb.Precision, precision))
    tol = 1e-8 * np.linalg.norm(src)
    x = np.zeros(case.n)
    assert ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, cb.SolveControl(tol, 500)).converged
    x0 = x.copy()
    st = ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, cb.SolveControl(2.0 * tol, 500))
    assert st.converged and st.iterations == 0 and np.array_equal(x, x0)


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_iteration_cap_is_reported_not_raised(graded, precision):
    cb, case, ds, up, lo, diag, src = graded
    ds.set_precision(getattr(cb.Precision, precision))
    x = np.zeros(case.n)
    st = ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, cb.SolveControl(1e-300, 3))
    assert not st.converged and st.iterations == 3
    assert st.residual > 0 and np.isfinite(x).all()
    x = np.zeros(case.n)
    st = ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, cb.SolveControl(1e-300, 0))
    assert not st.converged and st.iterations == 0 and not x.any()


def test_single_cell_without_faces(gpu):
    cb = gpu
    ds = cb.DeviceSolver(cb.build_csr_pattern(1, np.zeros(0, np.int32), np.zeros(0, np.int32)))
    x = np.zeros(1)
    st = ds.solve([4.0], [], [], [2.0], x, cb.Method.Cg, False, cb.SolveControl(1e-14, 10))
    assert st.converged and st.iterations == 1 and x[0] == 0.5


def test_disconnected_cells(gpu):
    """Cells with no faces next to a connected block: rows with only a diagonal."""
    cb = gpu
    owner = np.array([0, 1, 2], np.int32)
    neighbour = np.array([1, 2, 3], np.int32)
    n = 6  # cells 4 and 5 have no faces
    up = lo = -np.ones(3)
    diag = np.array([2.0, 3.0, 3.0, 2.0, 5.0, 7.0])
    b = np.arange(1.0, 7.0)
    ds = cb.DeviceSolver(cb.build_csr_pattern(n, owner, neighbour))
    x = np.zeros(n)
    st = ds.solve(diag, up, lo, b, x, cb.Method.Cg, False, cb.SolveControl(1e-13, 50))
    a = O.ldu_to_csr(O.build_pattern(n, owner, neighbour), diag, up, lo)
    assert st.converged and np.linalg.norm(b - a.matvec(x)) <= 1e-13
    assert x[4] == pytest.approx(1.0, rel=1e-12) and x[5] == pytest.approx(6.0 / 7.0, rel=1e-12)


def test_ragged_batch_with_converged_and_tiny_systems(gpu):
    """A batch mixing a multi-level system, a single-cell-edge box, a zero right-hand side and
    an iteration-capped system: each system keeps its own stopping rule."""
    import torch
    cb = gpu
    cases = [W.batch_box(14, seed=3), W.batch_box(2, seed=4), W.batch_box(9, seed=5),
             W.batch_box(11, seed=6)]
    nc = [c.n for c in cases]
    nf = [c.n_faces for c in cases]
    cat = lambda k: np.concatenate([getattr(c, k) for c in cases])  # noqa: E731
    b = cb.Batch(nc, nf, cat("owner"), cat("neighbour"))
    sysd = [_system(c) for c in cases]
    up = np.concatenate([s[0] for s in sysd])
    lo = np.concatenate([s[1] for s in sysd])
    dg = np.concatenate([s[2] for s in sysd])
    src = [s[3].copy() for s in sysd]
    src[2][:] = 0.0  # zero right-hand side
    rhs = np.concatenate(src)
    b.setup_amg(dg, up, lo)
    dev = torch.device("cuda")
    T = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev)  # noqa: E731
    x = torch.zeros(len(rhs), dtype=torch.float64, device=dev)
    ctl = [cb.SolveControl(1e-8 * max(np.linalg.norm(s), 1e-300), 500) for s in src]
    ctl[3] = cb.SolveControl(1e-300, 2)  # capped
    stats = b.solve_device(T(dg), T(up), T(lo), T(rhs), x, ctl)
    xs = x.cpu().numpy()
    assert stats[0].converged and stats[1].converged
    assert stats[2].converged and stats[2].iterations == 0
    assert not stats[3].converged and stats[3].iterations == 2
    off = np.concatenate([[0], np.cumsum(nc)])
    assert not xs[off[2]:off[3]].any()
    for i in (0, 1):
        c = cases[i]
        a = O.ldu_to_csr(O.build_pattern(c.n, c.owner, c.neighbour), sysd[i][2], sysd[i][0], sysd[i][1])
        assert np.linalg.norm(src[i] - a.matvec(xs[off[i]:off[i + 1]])) <= 1.05e-8 * np.linalg.norm(src[i])


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
@pytest.mark.parametrize("knobs", [{"tail_rows": 0}, {"tail_rows": 10 ** 6}, {"krylov_stage": 3}],
                         ids=["coarse-staging-wait", "tail-grid-barrier", "krylov-staging-wait"])
def test_expired_device_wait_reports_timeout_and_recovers(gpu, knobs, precision):
    """Every device-side wait is bounded. With the poll limit set to give up at once
    (Tuning.wait_polls < 0) the waits expire -- the coarse kernel's wait for its bulk copy
    (which it still drains before it exits), the persistent tail's grid barrier, or the staged
    Krylov SpMV's wait for a chunk (the CTA drains its copies in flight and still joins the
    block reduction) -- and the solve reports CFDB_ERR_TIMEOUT. With the default limit restored,
    the next solve is bit-identical to one that never timed out (error flag and barrier and
    reduction counters reset)."""
    cb = gpu
    case = W.graded(20)
    up, lo, diag, src = _system(case)
    ds = cb.DeviceSolver(cb.build_csr_pattern(case.n, case.owner, case.neighbour))
    ds.set_precision(getattr(cb.Precision, precision))
    ds.setup_amg(diag, up, lo, cb.AmgSettings(strength_threshold=0.04))
    ctl = cb.SolveControl(1e-8 * np.linalg.norm(src), 200)
    ds.set_tuning(cb.Tuning(**knobs))
    x_ref = np.zeros(case.n)
    st_ref = ds.solve(diag, up, lo, src, x_ref, cb.Method.Cg, True, ctl)
    assert st_ref.converged
    ds.set_tuning(cb.Tuning(**knobs, wait_polls=-1))
    with pytest.raises(cb.Timeout, match="bounded device wait expired"):
        ds.solve(diag, up, lo, src, np.zeros(case.n), cb.Method.Cg, True, ctl)
    ds.set_tuning(cb.Tuning(**knobs))
    for _ in range(2):
        x = np.zeros(case.n)
        st = ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, ctl)
        assert st.converged and st.iterations == st_ref.iterations
        assert np.array_equal(x, x_ref)
    ds.close()
