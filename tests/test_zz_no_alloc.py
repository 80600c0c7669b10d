"""The allocation-free Jacobi-CG entry point (cfdb_solve_device_noalloc).

It serves callers that cannot call cudaMalloc (an application that owns all device memory
through its own pool, or a loop that must not stall on the allocator): all arrays are the
caller's device memory and the work vectors live in the library's static device array. This
file is collected last so that a failure here cannot hide the results of the other tests.
"""
import numpy as np
import pytest

import oracle as O
from cfd_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _system():
    case = W.cavity(16)  # 4096 cells
    up, lo, dg, dv = O.assemble(case.n, case.owner, case.neighbour, case.flux, case.gamma,
                                case.delta, 0.0)
    diag, src = case.finalize(up, lo, dg, dv)
    pat = O.build_pattern(case.n, case.owner, case.neighbour)
    return O.ldu_to_csr(pat, diag, up, lo), src


def test_noalloc_matches_allocating_solve(gpu):
    import torch
    cb = gpu
    a, b = _system()
    n = a.n_rows
    tol = 1e-10 * np.linalg.norm(b)
    ctl = cb.SolveControl(tol, 5000)
    x_ref = np.zeros(n)
    st_ref = cb.solve(cb.CsrView(n, a.rp, a.ci, a.va), b, x_ref, cb.Method.Cg, ctl)
    assert st_ref.converged
    dev = torch.device("cuda")
    d_rp = torch.as_tensor(a.rp, dtype=torch.int32, device=dev)
    d_ci = torch.as_tensor(a.ci, dtype=torch.int32, device=dev)
    d_va = torch.as_tensor(a.va, device=dev)
    d_b = torch.as_tensor(b, device=dev)
    # the oracle's Jacobi-CG (krylov_kernels.inc:44-95, pinned to the reference's host path)
    x_orc, st_orc = O.krylov(a, b, method=0, abs_tol=tol, max_iterations=5000)
    assert st_orc["converged"]
    for call in range(2):  # two calls in a row share the static scratch
        d_x = torch.zeros(n, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        st = cb.solve_device_noalloc(n, a.nnz, d_rp, d_ci, d_va, d_b, d_x, cb.Method.Cg, ctl)
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        if call == 1:
            # the first call may load the kernels' code; the second must leave free memory as is
            assert free_after == free_before
        x = d_x.cpu().numpy()
        assert st.converged
        assert abs(st.iterations - st_ref.iterations) <= 2
        assert abs(st.iterations - st_orc["iterations"]) <= 2
        assert np.linalg.norm(b - a.matvec(x)) <= 1.05 * tol
        assert abs(st.true_residual - np.linalg.norm(b - a.matvec(x))) <= 1e-6 * tol
        assert np.linalg.norm(x - x_ref) <= 1e-6 * np.linalg.norm(x_ref)
        assert np.linalg.norm(x - x_orc) <= 1e-6 * np.linalg.norm(x_orc)


def test_noalloc_rejects_malformed_csr(gpu):
    """Row offsets and column indices are checked on the device before any kernel reads through
    them; a bad structure is refused and the next good call still solves."""
    import torch
    cb = gpu
    a, b = _system()
    n = a.n_rows
    dev = torch.device("cuda")
    T = lambda v, dt: torch.as_tensor(np.ascontiguousarray(v), dtype=dt, device=dev)  # noqa: E731
    bad_col = a.ci.copy()
    bad_col[17] = n  # outside [0, n)
    bad_rp = a.rp.copy()
    bad_rp[5], bad_rp[6] = bad_rp[6], bad_rp[5]  # decreasing
    ctl = cb.SolveControl(1e-10 * np.linalg.norm(b), 5000)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    with pytest.raises(cb.InvalidArgument, match="column index"):
        cb.solve_device_noalloc(n, a.nnz, T(a.rp, torch.int32), T(bad_col, torch.int32), T(a.va, torch.float64),
                                T(b, torch.float64), x, cb.Method.Cg, ctl)
    with pytest.raises(cb.InvalidArgument, match="row_ptr"):
        cb.solve_device_noalloc(n, a.nnz, T(bad_rp, torch.int32), T(a.ci, torch.int32), T(a.va, torch.float64),
                                T(b, torch.float64), x, cb.Method.Cg, ctl)
    st = cb.solve_device_noalloc(n, a.nnz, T(a.rp, torch.int32), T(a.ci, torch.int32), T(a.va, torch.float64),
                                 T(b, torch.float64), x, cb.Method.Cg, ctl)
    assert st.converged


def test_noalloc_rejects_oversize(gpu):
    import torch
    cb = gpu
    dev = torch.device("cuda")
    rp = torch.zeros(2, dtype=torch.int32, device=dev)
    ci = torch.zeros(1, dtype=torch.int32, device=dev)
    va = torch.ones(1, dtype=torch.float64, device=dev)
    b = torch.ones(1, dtype=torch.float64, device=dev)
    x = torch.zeros(1, dtype=torch.float64, device=dev)
    # raw device pointers: the C entry point itself refuses the size (tensors would already be
    # refused by the wrapper's length checks)
    with pytest.raises(cb.InvalidArgument, match="maximum of 65536 rows"):
        cb.solve_device_noalloc(65537, 1, rp.data_ptr(), ci.data_ptr(), va.data_ptr(), b.data_ptr(),
                                x.data_ptr(), cb.Method.Cg, cb.SolveControl())
