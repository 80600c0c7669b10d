"""GPU parity of the CUDA path against the CPU oracle (restated reference algorithms, pinned to
the reference's own compiled host path) on seeded inputs.

Bars: integer / index work bit-exact; assembly bit-exact (same accumulation order as the
reference's serial loop); one FP64 V-cycle bit-exact (same operation order, no FMA); AMG-PCG
iteration counts equal to the oracle's within 1 and true relative residual <= the target.
"""
import numpy as np
import pytest

import oracle as O
from cfd_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _assembled(case):
    up, lo, dg, dv = O.assemble(case.n, case.owner, case.neighbour, case.flux, case.gamma,
                                case.delta, 0.0)
    diag, src = case.finalize(up, lo, dg, dv)
    return up, lo, diag, src


def _hierarchy(case, up, lo, diag):
    pat = O.build_pattern(case.n, case.owner, case.neighbour)
    a = O.ldu_to_csr(pat, diag, up, lo)
    return pat, a, O.Hierarchy(a)


def _view(cb, h):
    lv = []
    for l in range(h.levels):
        A = cb.CsrView(h.a[l].n_rows, h.a[l].rp, h.a[l].ci, h.a[l].va)
        P = R = None
        if l + 1 < h.levels:
            P = cb.CsrView(h.p[l].n_rows, h.p[l].rp, h.p[l].ci, h.p[l].va)
            R = cb.CsrView(h.r[l].n_rows, h.r[l].rp, h.r[l].ci, h.r[l].va)
        lv.append(cb.AmgLevelView(A, P, R))
    return cb.AmgView(lv, h.coarse_inverse, 2, 0.7)


def _pattern(cb, pat):
    return cb.LduPattern(pat.n, pat.n_faces, pat.row_ptr, pat.col, pat.diag_pos, pat.upper_pos,
                         pat.lower_pos)


CASES = [lambda: W.cavity(12), lambda: W.graded(16), lambda: W.tet(8)]


@pytest.mark.parametrize("make", CASES, ids=["cavity12", "graded16", "tet8"])
def test_assembly_bitwise(gpu, make):
    case = make()
    cb = gpu
    nf = case.n_faces
    for conv in (0.0, 1.0):
        up, lo = np.zeros(nf), np.zeros(nf)
        dg, dv = np.full(case.n, 0.25), np.zeros(case.n)
        cb.assemble_convection_diffusion(case.n, nf, case.owner, case.neighbour, case.flux,
                                         case.gamma, case.delta, conv, up, lo, dg, dv)
        u2, l2, d2, v2 = O.assemble(case.n, case.owner, case.neighbour, case.flux, case.gamma,
                                    case.delta, conv, diag=np.full(case.n, 0.25))
        assert np.array_equal(up, u2) and np.array_equal(lo, l2)
        assert np.array_equal(dg, d2) and np.array_equal(dv, v2)


@pytest.mark.parametrize("size,permute", [(12, False), (100, False), (82, True)],
                         ids=["graded12-one-slice", "graded100-three-slices", "graded82-faces-shuffled"])
def test_system_assembly_host_arrays_bitwise(gpu, size, permute):
    """DeviceSolver.assemble on host arrays (the call the e2e sequence makes): the copies are
    pipelined over cell slices once a mesh has 2^19 cells or more; diag and div accumulate.
    With the faces shuffled (no owner order) each slice needs a long face prefix, which must
    stay correct."""
    cb = gpu
    case = W.graded(size)
    own, nei = np.asarray(case.owner), np.asarray(case.neighbour)
    flux, gamma, delta = case.flux, case.gamma, case.delta
    nf = case.n_faces
    if permute:
        p = np.random.default_rng(7).permutation(nf)
        own, nei, flux, gamma, delta = own[p], nei[p], flux[p], gamma[p], delta[p]
    ds = cb.DeviceSolver(mesh=(case.n, own, nei))
    try:
        for conv, d0 in ((0.0, 0.0), (1.0, 0.25), (0.0, 0.0)):
            up, lo = np.zeros(nf), np.zeros(nf)
            dg, dv = np.full(case.n, d0), np.full(case.n, -d0)
            ds.assemble(flux, gamma, delta, conv, up, lo, dg, dv)
            u2, l2, d2, v2 = O.assemble(case.n, own, nei, flux, gamma, delta, conv,
                                        diag=np.full(case.n, d0), div=np.full(case.n, -d0))
            assert np.array_equal(up, u2) and np.array_equal(lo, l2)
            assert np.array_equal(dg, d2) and np.array_equal(dv, v2)
    finally:
        ds.close()


def test_assembly_matches_reference_kat(gpu):
    """test_gpu.cpp:274-309 (AssemblyMatchesCpu): 7x5x3 box, convection 1."""
    cb = gpu
    m = cb.Mesh.box(7, 5, 3)
    nif, nc = m.n_internal_faces, m.n_cells
    f = np.arange(nif, dtype=np.float64)
    flux = np.sin(1.3 * f)
    gamma = 0.1 + 0.01 * (np.arange(nif) % 7)
    dc = 2.0 + 0.1 * (np.arange(nif) % 3)
    up, lo, diag, div = np.zeros(nif), np.zeros(nif), np.ones(nc), np.zeros(nc)
    cb.assemble_convection_diffusion(nc, nif, m.owner, m.neighbour, flux, gamma, dc, 1.0, up, lo,
                                     diag, div)
    g = gamma * dc
    assert np.array_equal(up, np.minimum(flux, 0.0) - g)
    assert np.array_equal(lo, -np.maximum(flux, 0.0) - g)
    dref, vref = np.ones(nc), np.zeros(nc)
    for k in range(nif):
        p, n = m.owner[k], m.neighbour[k]
        dref[p] += max(flux[k], 0.0) + g[k]
        dref[n] += -min(flux[k], 0.0) + g[k]
        vref[p] += flux[k]
        vref[n] -= flux[k]
    assert np.allclose(diag, dref, atol=1e-12, rtol=0) and np.allclose(div, vref, atol=1e-12, rtol=0)


@pytest.mark.parametrize("make", CASES, ids=["cavity12", "graded16", "tet8"])
def test_vcycle_bitwise(gpu, make):
    """One FP64 V-cycle (Jacobi 2+2, dense coarse) equals the oracle bit for bit."""
    cb = gpu
    case = make()
    up, lo, diag, src = _assembled(case)
    pat, a, h = _hierarchy(case, up, lo, diag)
    ds = cb.DeviceSolver(_pattern(cb, pat))
    ds.set_ordered(True)
    ds.set_amg(_view(cb, h))
    x = np.zeros(case.n)
    ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, cb.SolveControl(1e300, 1))  # installs A
    rng = np.random.default_rng(7)
    r = rng.standard_normal(case.n)
    z = ds.apply_amg(r)
    zr = O.vcycle_apply(h.a, h.p, h.r, h.coarse_inverse, r, 2, 0.7)
    assert np.array_equal(z, zr)


@pytest.mark.parametrize("make", CASES, ids=["cavity12", "graded16", "tet8"])
def test_amg_pcg_matches_oracle(gpu, make):
    cb = gpu
    case = make()
    up, lo, diag, src = _assembled(case)
    pat, a, h = _hierarchy(case, up, lo, diag)
    tol = 1e-8 * np.linalg.norm(src)
    xo, so = O.amg_cg(h.a, h.p, h.r, h.coarse_inverse, src, abs_tol=tol, max_iterations=500)
    ds = cb.DeviceSolver(_pattern(cb, pat))
    ds.set_amg(_view(cb, h))
    x = np.zeros(case.n)
    st = ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, cb.SolveControl(tol, 500))
    assert st.converged and st.on_device
    assert abs(st.iterations - so["iterations"]) <= 1
    tr = np.linalg.norm(src - a.matvec(x))
    assert tr <= 1.05 * tol and abs(tr - st.true_residual) <= 1e-6 * tol
    # solutions agree to the solver tolerance (relative to the solution scale)
    assert np.linalg.norm(x - xo) <= 1e-5 * np.linalg.norm(xo)


@pytest.mark.parametrize("make", CASES, ids=["cavity12", "graded16", "tet8"])
def test_vcycle_fast_mode_close(gpu, make):
    """Default (warp-per-row sums on wide coarse levels): V-cycle agrees to FP64 round-off."""
    cb = gpu
    case = make()
    up, lo, diag, src = _assembled(case)
    pat, a, h = _hierarchy(case, up, lo, diag)
    ds = cb.DeviceSolver(_pattern(cb, pat))
    ds.set_amg(_view(cb, h))
    x = np.zeros(case.n)
    ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, cb.SolveControl(1e300, 1))
    r = np.random.default_rng(8).standard_normal(case.n)
    z = ds.apply_amg(r)
    zr = O.vcycle_apply(h.a, h.p, h.r, h.coarse_inverse, r, 2, 0.7)
    assert np.linalg.norm(z - zr) <= 1e-12 * np.linalg.norm(zr)


def test_solve_amg_cg_oneshot(gpu):
    cb = gpu
    case = W.graded(12)
    up, lo, diag, src = _assembled(case)
    pat, a, h = _hierarchy(case, up, lo, diag)
    tol = 1e-10 * np.linalg.norm(src)
    x = np.zeros(case.n)
    st = cb.solve_amg_cg(_view(cb, h), src, x, cb.SolveControl(tol, 500))
    xo, so = O.amg_cg(h.a, h.p, h.r, h.coarse_inverse, src, abs_tol=tol, max_iterations=500)
    assert st.converged and abs(st.iterations - so["iterations"]) <= 1
    assert np.linalg.norm(src - a.matvec(x)) <= 1.05 * tol


def test_jacobi_cg_matches_oracle(gpu):
    cb = gpu
    case = W.cavity(8)
    up, lo, diag, src = _assembled(case)
    pat = O.build_pattern(case.n, case.owner, case.neighbour)
    a = O.ldu_to_csr(pat, diag, up, lo)
    tol = 1e-10 * np.linalg.norm(src)
    xo, so = O.krylov(a, src, method=0, abs_tol=tol, max_iterations=5000)
    x = np.zeros(case.n)
    st = cb.solve(cb.CsrView(a.n_rows, a.rp, a.ci, a.va), src, x, cb.Method.Cg,
                  cb.SolveControl(tol, 5000))
    assert st.converged and abs(st.iterations - so["iterations"]) <= 2
    assert np.linalg.norm(src - a.matvec(x)) <= 1.05 * tol


@pytest.mark.parametrize("make", CASES, ids=["cavity12", "graded16", "tet8"])
def test_mixed_precision_reaches_target(gpu, make):
    """FP32 V-cycle inside FP64 flexible CG: true FP64 relative residual <= 1e-8."""
    cb = gpu
    case = make()
    up, lo, diag, src = _assembled(case)
    pat, a, h = _hierarchy(case, up, lo, diag)
    tol = 1e-8 * np.linalg.norm(src)
    ds = cb.DeviceSolver(_pattern(cb, pat))
    ds.set_precision(cb.Precision.MIXED)
    ds.set_amg(_view(cb, h))
    x = np.zeros(case.n)
    st = ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, cb.SolveControl(tol, 500))
    assert st.converged
    assert np.linalg.norm(src - a.matvec(x)) <= tol
    xo, so = O.amg_cg(h.a, h.p, h.r, h.coarse_inverse, src, abs_tol=tol, max_iterations=500)
    assert np.linalg.norm(x - xo) <= 1e-5 * np.linalg.norm(xo)


@pytest.mark.parametrize("precision,schedule,cluster", [
    ("FP64", (0, 0.0), 0), ("MIXED", (0, 0.0), 0), ("MIXED", (1, 0.85), 0), ("MIXED", (3, 0.85), 0),
    ("FP64", (0, 0.0), 16), ("MIXED", (1, 0.85), 8), ("MIXED", (1, 0.85), 16)],
    ids=["FP64", "MIXED", "MIXED-1sweep", "MIXED-3sweeps", "FP64-cluster16", "MIXED-1sweep-cluster8",
         "MIXED-1sweep-cluster16"])
def test_persistent_tail_matches_separate_kernels(gpu, precision, schedule, cluster):
    """The persistent tail kernel (small coarse levels + coarse solve in one launch: a
    cooperative grid, or one thread-block cluster) computes every row exactly as the separate
    per-level kernels do, under the hierarchy's smoother schedule and under the mixed path's
    tuned ones."""
    cb = gpu
    case = W.graded(24)
    up, lo, diag, src = _assembled(case)
    ds = cb.DeviceSolver(cb.build_csr_pattern(case.n, case.owner, case.neighbour))
    ds.set_precision(getattr(cb.Precision, precision))
    ds.setup_amg(diag, up, lo, cb.AmgSettings(strength_threshold=0.04))
    tol = 1e-10 * np.linalg.norm(src)
    out = []
    for tail in (0, 10**6):
        ds.set_tuning(cb.Tuning(tail_rows=tail, mixed_sweeps=schedule[0], mixed_weight=schedule[1],
                                tail_cluster=cluster if tail else 0))
        x = np.zeros(case.n)
        st = ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, cb.SolveControl(tol, 500))
        z = ds.apply_amg(np.random.default_rng(3).standard_normal(case.n))
        assert st.converged
        out.append((x, st.iterations, z))
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][2], out[1][2])


@pytest.mark.parametrize("make", [lambda: W.cavity(8), lambda: W.tet(5)], ids=["cavity8", "tet5"])
def test_bicgstab_matches_oracle(gpu, make):
    """Jacobi-preconditioned BiCGStab (krylov_kernels.inc:97-169): one-shot on a CSR matrix and
    through the persistent system, iterations within 2 of the oracle, tolerance met."""
    cb = gpu
    case = make()
    up, lo, diag, src = _assembled(case)
    pat = O.build_pattern(case.n, case.owner, case.neighbour)
    a = O.ldu_to_csr(pat, diag, up, lo)
    tol = 1e-10 * np.linalg.norm(src)
    xo, so = O.krylov(a, src, method=1, abs_tol=tol, max_iterations=5000)
    assert so["converged"]
    x = np.zeros(case.n)
    st = cb.solve(cb.CsrView(a.n_rows, a.rp, a.ci, a.va), src, x, cb.Method.BiCgStab,
                  cb.SolveControl(tol, 5000))
    assert st.converged and abs(st.iterations - so["iterations"]) <= 2
    assert np.linalg.norm(src - a.matvec(x)) <= 1.05 * tol
    ds = cb.DeviceSolver(_pattern(cb, pat))
    x2 = np.zeros(case.n)
    st2 = ds.solve(diag, up, lo, src, x2, cb.Method.BiCgStab, False, cb.SolveControl(tol, 5000))
    assert st2.converged and abs(st2.iterations - so["iterations"]) <= 2
    assert np.linalg.norm(src - a.matvec(x2)) <= 1.05 * tol


def test_flux_correction_and_relaxation_bitwise(gpu):
    """The steps after the pressure solve on the device (flow_solver.cpp:821-840): face flux
    correction with and without a non-orthogonal term, relaxed and unrelaxed pressure, against
    the oracle's restatement, bit for bit."""
    import torch
    cb = gpu
    case = W.tet(6)
    nf = case.n_faces
    rng = np.random.default_rng(11)
    p_new = rng.standard_normal(case.n)
    p_prev = rng.standard_normal(case.n)
    non_orth = 1e-3 * rng.standard_normal(nf)
    ds = cb.DeviceSolver(mesh=(case.n, case.owner, case.neighbour))
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")  # noqa: E731
    own, nei = case.owner[:nf], case.neighbour
    for no, prev, alpha in ((None, None, 1.0), (non_orth, p_prev, 0.3)):
        phi = torch.empty(nf, dtype=torch.float64, device="cuda")
        p = torch.empty(case.n, dtype=torch.float64, device="cuda")
        ds.correct_pressure_device(T(case.flux), T(case.gamma), T(case.delta), T(p_new), phi, p,
                                   p_prev=None if prev is None else T(prev), alpha=alpha,
                                   non_orth=None if no is None else T(no))
        torch.cuda.synchronize()
        want_phi = O.correct_flux(own, nei, case.flux, case.gamma, case.delta, p_new, no)
        want_p = p_new if prev is None else O.relax(prev, p_new, alpha)
        assert np.array_equal(phi.cpu().numpy(), want_phi)
        assert np.array_equal(p.cpu().numpy(), want_p)


@pytest.mark.parametrize("kind", ["box", "tet"])
def test_pressure_gradient_and_velocity_correction_bitwise(gpu, kind):
    """Gauss pressure gradient with the two-pass tangential boundary extrapolation and the
    velocity correction on the device (flow_solver.cpp:339-372, 843-846), against the oracle's
    face-by-face restatement, bit for bit; one wall is a pressure outlet."""
    import torch
    cb = gpu
    m = cb.Mesh.box(6, 5, 4, xs=np.array([0.0, 0.1, 0.25, 0.45, 0.7, 0.85, 1.0])) if kind == "box" \
        else cb.Mesh.tet(4, 3, 3, jitter=0.2, seed=9)
    nb = m.n_faces - m.n_internal_faces
    fc_b = m.face_centres[m.n_internal_faces:]
    kinds = np.where(np.isclose(fc_b[:, 0], 1.0), int(cb.BoundaryKind.PressureOutlet),
                     int(cb.BoundaryKind.Wall)).astype(np.int32)
    kinds[np.isclose(fc_b[:, 0], 0.0)] = int(cb.BoundaryKind.VelocityInlet)
    pout = np.where(kinds == int(cb.BoundaryKind.PressureOutlet), 0.25, 0.0)
    rng = np.random.default_rng(5)
    p = rng.standard_normal(m.n_cells)
    hbya = rng.standard_normal((m.n_cells, 3))
    rau = rng.uniform(0.5, 2.0, m.n_cells)
    fv = cb.FvGeometry(m, kinds, pout)
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")  # noqa: E731
    grad = torch.empty((m.n_cells, 3), dtype=torch.float64, device="cuda")
    u = torch.empty((m.n_cells, 3), dtype=torch.float64, device="cuda")
    fv.pressure_gradient_device(T(p), grad)
    fv.correct_velocity_device(T(hbya), T(rau), grad, u)
    want = O.pressure_gradient(m.n_cells, m.n_internal_faces, m.owner, m.neighbour, m.weights,
                               m.face_areas, m.face_centres, m.cell_centres, m.cell_volumes, kinds,
                               pout, p)
    assert nb > 0 and np.array_equal(grad.cpu().numpy(), want)
    assert np.array_equal(u.cpu().numpy(), O.correct_velocity(hbya, rau, want))
    fv.close()


@pytest.mark.parametrize("make", [lambda: W.graded(20), lambda: W.tet(10)], ids=["graded20", "tet10"])
def test_mixed_smoother_schedule(gpu, make):
    """Tuning.mixed_sweeps / mixed_weight change the mixed-precision V-cycle only: every
    schedule still reaches the FP64 true residual 1e-8 (flexible CG), and the FP64 path solves
    bit-identically with or without the knobs set (it keeps the hierarchy's schedule)."""
    cb = gpu
    case = make()
    up, lo, diag, src = _assembled(case)
    pat, a, h = _hierarchy(case, up, lo, diag)
    tol = 1e-8 * np.linalg.norm(src)
    for sweeps, weight in ((1, 0.85), (2, 0.85), (3, 0.6)):
        ds = cb.DeviceSolver(_pattern(cb, pat))
        ds.set_precision(cb.Precision.MIXED)
        ds.set_amg(_view(cb, h))
        ds.set_tuning(cb.Tuning(mixed_sweeps=sweeps, mixed_weight=weight))
        x = np.zeros(case.n)
        st = ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, cb.SolveControl(tol, 500))
        assert st.converged and np.linalg.norm(src - a.matvec(x)) <= tol
        ds.close()
    out = []
    for t in (cb.Tuning(), cb.Tuning(mixed_sweeps=1, mixed_weight=0.85)):
        ds = cb.DeviceSolver(_pattern(cb, pat))
        ds.set_amg(_view(cb, h))
        ds.set_tuning(t)
        x = np.zeros(case.n)
        st = ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, cb.SolveControl(tol, 500))
        out.append((st.iterations, x))
        ds.close()
    assert out[0][0] == out[1][0] and np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_two_row_vcycle_kernels_match_one_row(gpu, precision):
    """The V-cycle kernels of SELL operators with two rows per thread per pass (vcycle_pair)
    sum every row in the same order as the one-row kernels: solves and preconditioner
    applications are bit-identical."""
    cb = gpu
    case = W.tet(12)
    up, lo, diag, src = _assembled(case)
    ds = cb.DeviceSolver(cb.build_csr_pattern(case.n, case.owner, case.neighbour))
    ds.set_precision(getattr(cb.Precision, precision))
    ds.setup_amg(diag, up, lo, cb.AmgSettings(strength_threshold=0.04))
    tol = 1e-10 * np.linalg.norm(src)
    out = []
    for pair in (0, 1):
        ds.set_tuning(cb.Tuning(vcycle_pair=pair, sell_rows=512, wide_row=64))
        x = np.zeros(case.n)
        st = ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, cb.SolveControl(tol, 500))
        z = ds.apply_amg(np.random.default_rng(5).standard_normal(case.n))
        assert st.converged
        out.append((x, st.iterations, z))
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][2], out[1][2])


def _mixed_stencil(nx, ny, nz, wide_x):
    """LDU system on an nx x ny x nz lattice: 6-neighbour couplings everywhere, and the 26
    neighbours of the cells with x < wide_x (rows of 27 entries: their SELL chunks hold more
    slots than a staging buffer, so the staged kernel sums them from global memory).
    Symmetric, diagonally dominant."""
    idx = np.arange(nx * ny * nz).reshape(nz, ny, nx)
    pairs = []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if (dz, dy, dx) <= (0, 0, 0):
                    continue
                a = idx[max(0, -dz):nz - max(0, dz), max(0, -dy):ny - max(0, dy), max(0, -dx):nx - max(0, dx)]
                b = idx[max(0, dz):nz - max(0, -dz) or None, max(0, dy):ny - max(0, -dy) or None,
                        max(0, dx):nx - max(0, -dx) or None]
                a, b = a.ravel(), b.ravel()
                axis = abs(dz) + abs(dy) + abs(dx) == 1
                keep = axis | ((a % nx < wide_x) & (b % nx < wide_x))
                pairs.append(np.stack([np.minimum(a, b)[keep], np.maximum(a, b)[keep]], 1))
    p = np.concatenate(pairs)
    p = p[np.lexsort((p[:, 1], p[:, 0]))]
    owner, neighbour = p[:, 0].astype(np.int32), p[:, 1].astype(np.int32)
    n = nx * ny * nz
    rng = np.random.default_rng(21)
    w = rng.uniform(0.5, 1.5, len(owner))
    diag = np.bincount(owner, w, n) + np.bincount(neighbour, w, n) + 0.05
    src = rng.standard_normal(n)
    return n, owner, neighbour, -w, -w.copy(), diag, src


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
@pytest.mark.parametrize("mesh", ["tet", "mixed-stencil"])
def test_staged_krylov_spmv_matches_thread_loads(gpu, precision, mesh):
    """The level-0 Krylov SpMV with the operator streamed through shared memory by bulk copies
    (krylov_stage 2..4 buffers) visits and sums every row as the thread-load kernels do: solves
    are bit-identical (iterations and x). Few tiles, so that each CTA pipelines many chunks
    through its buffers; on the mixed stencil the wide chunks take the unstaged path."""
    cb = gpu
    if mesh == "tet":
        case = W.tet(14)
        up, lo, diag, src = _assembled(case)
        n, owner, neighbour = case.n, case.owner, case.neighbour
    else:
        n, owner, neighbour, up, lo, diag, src = _mixed_stencil(40, 30, 24, 9)
    ds = cb.DeviceSolver(cb.build_csr_pattern(n, owner, neighbour))
    ds.set_precision(getattr(cb.Precision, precision))
    ds.setup_amg(diag, up, lo, cb.AmgSettings(strength_threshold=0.04))
    ctl = cb.SolveControl(1e-10 * np.linalg.norm(src), 500)
    out = []
    for pair, stage in ((1, 0), (0, 0), (1, 2), (1, 3), (1, 4)):
        ds.set_tuning(cb.Tuning(krylov_pair=pair, krylov_stage=stage, target_tiles=3))
        x = np.zeros(n)
        st = ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, ctl)
        assert st.converged
        out.append((st.iterations, x))
    for it, x in out[1:]:
        assert it == out[0][0] and np.array_equal(x, out[0][1])
    ds.close()


@pytest.mark.parametrize("make", [lambda: W.graded(24), lambda: W.tet(12)], ids=["graded24", "tet12"])
def test_col16_columns_match_int32_columns(gpu, make):
    """FP32 operators with 16-bit column offsets from a per-slice / per-row base (Tuning.col16,
    used where every slice or row spans fewer than 65,536 columns) decode to the same columns:
    mixed-precision solves and preconditioner applications are bit-identical to the int32
    layout."""
    cb = gpu
    case = make()
    up, lo, diag, src = _assembled(case)
    ds = cb.DeviceSolver(cb.build_csr_pattern(case.n, case.owner, case.neighbour))
    ds.set_precision(cb.Precision.MIXED)
    ds.setup_amg(diag, up, lo, cb.AmgSettings(strength_threshold=0.04))
    ctl = cb.SolveControl(1e-10 * np.linalg.norm(src), 500)
    r = np.random.default_rng(9).standard_normal(case.n)
    out = []
    for col16 in (0, 1):
        ds.set_tuning(cb.Tuning(col16=col16, wide_row=24))
        x = np.zeros(case.n)
        st = ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, ctl)
        assert st.converged
        out.append((st.iterations, x, ds.apply_amg(r)))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])
    ds.close()
