"""Batched solves: many uneven systems in one device plan give each system the same answer as
solving it alone (iterations within 1, solutions to the solver tolerance), in FP64 and mixed
precision, with per-system reference cells and convergence."""
import numpy as np
import pytest

import oracle as O
from cfd_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _cases():
    # the 18^3 box has more than 4096 rows: its host setup, inside the batch's parallel loop
    # over systems, transposes in a nested OpenMP region
    return [W.batch_box(e, seed=100 + i) for i, e in enumerate([6, 9, 4, 12, 7, 18])] + [W.tet(4, seed=7)]


def _concat(cases):
    cat = lambda k: np.concatenate([getattr(c, k) for c in cases])  # noqa: E731
    return ([c.n for c in cases], [c.n_faces for c in cases], cat("owner"), cat("neighbour"),
            cat("flux"), cat("gamma"), cat("delta"), cat("source0"))


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_batch_matches_single_solves(gpu, precision):
    import torch
    cb = gpu
    cases = _cases()
    nc, nf, own, nei, flux, gamma, delta, src0 = _concat(cases)
    b = cb.Batch(nc, nf, own, nei)
    dev = torch.device("cuda")
    T = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev)  # noqa: E731
    d_up, d_lo = torch.empty(b.total_faces, dtype=torch.float64, device=dev), torch.empty(b.total_faces, dtype=torch.float64, device=dev)
    d_dg, d_src = torch.empty(b.total_cells, dtype=torch.float64, device=dev), torch.empty(b.total_cells, dtype=torch.float64, device=dev)
    b.assemble_pressure_device(T(flux), T(gamma), T(delta), T(src0), d_up, d_lo, d_dg, d_src,
                               ref_cells=[0] * len(cases))
    torch.cuda.synchronize()
    up, lo, dg, src = d_up.cpu().numpy(), d_lo.cpu().numpy(), d_dg.cpu().numpy(), d_src.cpu().numpy()
    # the batched assembly equals the oracle's per-system assembly + finalize, bit for bit
    co, fo = 0, 0
    for c in cases:
        u, l, d, v = O.assemble(c.n, c.owner, c.neighbour, c.flux, c.gamma, c.delta, 0.0)
        d2, s2 = c.finalize(u, l, d, v)
        assert np.array_equal(up[fo:fo + c.n_faces], u) and np.array_equal(lo[fo:fo + c.n_faces], l)
        assert np.array_equal(dg[co:co + c.n], d2) and np.array_equal(src[co:co + c.n], s2)
        co += c.n
        fo += c.n_faces
    b.setup_amg(dg, up, lo)
    b.set_precision(getattr(cb.Precision, precision))
    x = torch.zeros(b.total_cells, dtype=torch.float64, device=dev)
    tols = []
    co = 0
    for c in cases:
        tols.append(1e-8 * np.linalg.norm(src[co:co + c.n]))
        co += c.n
    stats = b.solve_device(d_dg, d_up, d_lo, d_src, x, [cb.SolveControl(t, 300) for t in tols])
    xb = x.cpu().numpy()
    co, fo = 0, 0
    for i, c in enumerate(cases):
        ds = cb.DeviceSolver(cb.build_csr_pattern(c.n, c.owner, c.neighbour))
        ds.set_precision(getattr(cb.Precision, precision))
        u, l, d = up[fo:fo + c.n_faces], lo[fo:fo + c.n_faces], dg[co:co + c.n]
        ds.setup_amg(d, u, l)
        xs = np.zeros(c.n)
        st = ds.solve(d, u, l, src[co:co + c.n], xs, cb.Method.Cg, True, cb.SolveControl(tols[i], 300))
        assert stats[i].converged and st.converged
        assert abs(stats[i].iterations - st.iterations) <= 1
        pat = O.build_pattern(c.n, c.owner, c.neighbour)
        a = O.ldu_to_csr(pat, d, u, l)
        xi = xb[co:co + c.n]
        assert np.linalg.norm(src[co:co + c.n] - a.matvec(xi)) <= 1.05 * tols[i]
        assert np.linalg.norm(xi - xs) <= 1e-5 * np.linalg.norm(xs)
        co += c.n
        fo += c.n_faces


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_batch_device_setup_equals_host_setup(gpu, precision):
    """Batch hierarchies built on the device (cfdb_batch_setup_amg_device, several systems at a
    time) equal the host build: the batched solves that follow are bit-identical."""
    import torch
    cb = gpu
    cases = _cases()
    nc, nf, own, nei, flux, gamma, delta, src0 = _concat(cases)
    dev = torch.device("cuda")
    T = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev)  # noqa: E731
    out = []
    for how in ("host", "device", "device1"):
        b = cb.Batch(nc, nf, own, nei)
        d_up, d_lo = torch.empty(b.total_faces, dtype=torch.float64, device=dev), torch.empty(b.total_faces, dtype=torch.float64, device=dev)
        d_dg, d_src = torch.empty(b.total_cells, dtype=torch.float64, device=dev), torch.empty(b.total_cells, dtype=torch.float64, device=dev)
        b.assemble_pressure_device(T(flux), T(gamma), T(delta), T(src0), d_up, d_lo, d_dg, d_src,
                                   ref_cells=[0] * len(cases))
        torch.cuda.synchronize()
        s = cb.AmgSettings(strength_threshold=0.04)
        if how == "host":
            b.setup_amg(d_dg.cpu().numpy(), d_up.cpu().numpy(), d_lo.cpu().numpy(), s)
        else:
            b.setup_amg(d_dg, d_up, d_lo, s, device=True, concurrency=1 if how == "device1" else 0)
        b.set_precision(getattr(cb.Precision, precision))
        src = d_src.cpu().numpy()
        co, tols = 0, []
        for c in cases:
            tols.append(1e-8 * np.linalg.norm(src[co:co + c.n]))
            co += c.n
        x = torch.zeros(b.total_cells, dtype=torch.float64, device=dev)
        stats = b.solve_device(d_dg, d_up, d_lo, d_src, x, [cb.SolveControl(t, 300) for t in tols])
        torch.cuda.synchronize()
        out.append(([st.iterations for st in stats], x.cpu().numpy()))
        b.close()
    for its, x in out[1:]:
        assert its == out[0][0] and np.array_equal(x, out[0][1])


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_batch_staged_krylov_spmv_matches_thread_loads(gpu, precision):
    """In a batch the level-0 Krylov tiles hold one system each, starting on the system's
    32-row-aligned offset: the staged SpMV (krylov_stage, operator chunks through shared
    memory) gives every system the same iterations and solution bit for bit as the
    thread-load kernels, with tiles of many chunks (target_tiles 4) and of one."""
    import torch
    cb = gpu
    cases = _cases()
    nc, nf, own, nei, flux, gamma, delta, src0 = _concat(cases)
    dev = torch.device("cuda")
    T = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev)  # noqa: E731
    b = cb.Batch(nc, nf, own, nei)
    d_up, d_lo = torch.empty(b.total_faces, dtype=torch.float64, device=dev), torch.empty(b.total_faces, dtype=torch.float64, device=dev)
    d_dg, d_src = torch.empty(b.total_cells, dtype=torch.float64, device=dev), torch.empty(b.total_cells, dtype=torch.float64, device=dev)
    b.assemble_pressure_device(T(flux), T(gamma), T(delta), T(src0), d_up, d_lo, d_dg, d_src,
                               ref_cells=[0] * len(cases))
    b.setup_amg(d_dg, d_up, d_lo, cb.AmgSettings(strength_threshold=0.04), device=True)
    b.set_precision(getattr(cb.Precision, precision))
    src = d_src.cpu().numpy()
    co, tols = 0, []
    for c in cases:
        tols.append(1e-8 * np.linalg.norm(src[co:co + c.n]))
        co += c.n
    out = []
    for stage, tiles in ((0, 4), (3, 4), (2, 0), (4, 0)):
        b.set_tuning(cb.Tuning(krylov_stage=stage, target_tiles=tiles))
        x = torch.zeros(b.total_cells, dtype=torch.float64, device=dev)
        stats = b.solve_device(d_dg, d_up, d_lo, d_src, x, [cb.SolveControl(t, 300) for t in tols])
        torch.cuda.synchronize()
        assert all(st.converged for st in stats)
        out.append(([st.iterations for st in stats], x.cpu().numpy()))
    # target_tiles changes the reduction tiles (the dot products' partial sums), so compare
    # within each tiling: staged against thread loads with the same tiles
    b.set_tuning(cb.Tuning(krylov_stage=0, target_tiles=0))
    x = torch.zeros(b.total_cells, dtype=torch.float64, device=dev)
    stats = b.solve_device(d_dg, d_up, d_lo, d_src, x, [cb.SolveControl(t, 300) for t in tols])
    ref0 = ([st.iterations for st in stats], x.cpu().numpy())
    assert out[0][0] == out[1][0] and np.array_equal(out[0][1], out[1][1])
    for it, xs in out[2:]:
        assert it == ref0[0] and np.array_equal(xs, ref0[1])
