"""The hierarchy built on the device (cfdb_amg_setup_device, cfdb_system_setup_amg_device)
against the oracle's restated setup (amg.cpp:12-240) and the host build: aggregates, P, R,
Galerkin operators and coarse inverse bit-identical, and solves after a device setup
bit-identical to solves after a host setup."""
import numpy as np
import pytest

import oracle as O
from cfd_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _pressure(case):
    up, lo, dg, dv = O.assemble(case.n, case.owner, case.neighbour, case.flux, case.gamma,
                                case.delta, 0.0)
    diag, src = case.finalize(up, lo, dg, dv)
    return up, lo, diag, src


def _same(h, o):
    """h: cfd_b200.AmgHierarchy; o: oracle Hierarchy (or an AmgHierarchy of the host build)."""
    if isinstance(o, O.Hierarchy):
        levels, A, Pm, Rm = o.levels, o.a, o.p, o.r
        agg_of = lambda l: (o.aggregates[l], o.a[l + 1].n_rows)  # noqa: E731
        inv = o.coarse_inverse
        csr = lambda m: (m.rp, m.ci, m.va)  # noqa: E731
    else:
        levels = o.levels()
        A = [o.level_matrix(l) for l in range(levels)]
        Pm = [o.level_prolongation(l) for l in range(levels - 1)]
        Rm = [o.level_restriction(l) for l in range(levels - 1)]
        agg_of = o.aggregates
        inv = o.coarse_inverse()
        csr = lambda m: (m.row_ptr, m.col, m.val)  # noqa: E731
    assert h.levels() == levels
    for l in range(levels):
        got = h.level_matrix(l)
        for x, y in zip((got.row_ptr, got.col, got.val), csr(A[l])):
            assert np.array_equal(x, y), f"A[{l}]"
        if l + 1 < levels:
            agg, n_agg = h.aggregates(l)
            want_agg, want_n = agg_of(l)
            assert np.array_equal(agg, want_agg) and n_agg == want_n, f"aggregates[{l}]"
            for name, g, w in (("P", h.level_prolongation(l), Pm[l]), ("R", h.level_restriction(l), Rm[l])):
                for x, y in zip((g.row_ptr, g.col, g.val), csr(w)):
                    assert np.array_equal(x, y), f"{name}[{l}]"
    assert np.array_equal(h.coarse_inverse(), inv)


CASES = {"cavity10": lambda: W.cavity(10), "graded12": lambda: W.graded(12),
         "tet6": lambda: W.tet(6), "tet7_sigma": lambda: W.tet(7, sigma=1.5, seed=5)}


@pytest.mark.parametrize("theta", [0.08, 0.04, 0.0])
@pytest.mark.parametrize("name", list(CASES))
def test_device_setup_matches_oracle(gpu, name, theta):
    cb = gpu
    case = CASES[name]()
    up, lo, diag, _ = _pressure(case)
    a = O.ldu_to_csr(O.build_pattern(case.n, case.owner, case.neighbour), diag, up, lo)
    h = cb.AmgHierarchy(cb.CsrView(a.n_rows, a.rp, a.ci, a.va),
                        cb.AmgSettings(strength_threshold=theta), device=True)
    _same(h, O.Hierarchy(a, theta=theta))


@pytest.mark.parametrize("make,theta", [(lambda: W.graded(80), 0.04), (lambda: W.tet(18), 0.04),
                                        (lambda: W.tet(14), 0.0)], ids=["graded80", "tet18", "tet14_theta0"])
def test_device_setup_matches_host_build(gpu, make, theta):
    """Larger meshes (coarse rows of hundreds to thousands of entries: warp and CTA tables)."""
    cb = gpu
    case = make()
    up, lo, diag, _ = _pressure(case)
    p = cb.build_csr_pattern(case.n, case.owner, case.neighbour)
    a = O.ldu_to_csr(O.build_pattern(case.n, case.owner, case.neighbour), diag, up, lo)
    s = cb.AmgSettings(strength_threshold=theta)
    view = cb.CsrView(a.n_rows, a.rp, a.ci, a.va)
    assert np.array_equal(p.row_ptr, a.rp)
    _same(cb.AmgHierarchy(view, s, device=True), cb.AmgHierarchy(view, s))


@pytest.mark.parametrize("size,every", [(36, 300), (36, 250)], ids=["pass3-device", "pass3-host"])
def test_device_setup_with_rows_left_for_pass3(gpu, size, every):
    """The fine level of tet 36 (279,936 rows, sparse) is aggregated on the device. Rows whose
    every off-diagonal is weak have no strong connection: passes 1 and 2 leave them for pass 3
    (amg.cpp:66-76), which one device thread runs when at most 1024 rows are left (every 300th
    row: 934) and the host runs from the strength graph read back when more are (every 250th:
    1,120). The hierarchy equals the oracle's either way."""
    import dataclasses
    theta = 0.04
    cb = gpu
    case = W.tet(size)
    up, lo, diag, _ = _pressure(case)
    a = O.ldu_to_csr(O.build_pattern(case.n, case.owner, case.neighbour), diag, up, lo)
    rows = np.repeat(np.arange(a.n_rows), np.diff(a.rp))
    iso = np.arange(a.n_rows) % every == 5
    weak = (a.ci != rows) & (iso[rows] | iso[a.ci])
    va = a.va.copy()
    va[weak] *= 1e-6
    a = dataclasses.replace(a, va=va)
    d = np.zeros(a.n_rows)
    d[rows[a.ci == rows]] = va[a.ci == rows]
    strong = (a.ci != rows) & (np.abs(va) > theta * np.sqrt(np.abs(d[rows] * d[a.ci])))
    assert not strong[iso[rows]].any() and strong.any()  # isolated rows exist at level 0
    h = cb.AmgHierarchy(cb.CsrView(a.n_rows, a.rp, a.ci, a.va), cb.AmgSettings(strength_threshold=theta),
                        device=True)
    _same(h, O.Hierarchy(a, theta=theta))


@pytest.mark.parametrize("limit", [24, 200])
@pytest.mark.parametrize("name,theta", [("tet7_sigma", 0.0), ("graded12", 0.04)])
def test_device_memory_tables_match_oracle(gpu, name, theta, limit):
    """device_table_limit moves every row longer than `limit` out of the shared-memory tables
    (symbolic overflow, device-memory tables, device-memory sorts of the transpose): the result
    must not change."""
    cb = gpu
    case = CASES[name]()
    up, lo, diag, _ = _pressure(case)
    a = O.ldu_to_csr(O.build_pattern(case.n, case.owner, case.neighbour), diag, up, lo)
    h = cb.AmgHierarchy(cb.CsrView(a.n_rows, a.rp, a.ci, a.va),
                        cb.AmgSettings(strength_threshold=theta, device_table_limit=limit), device=True)
    _same(h, O.Hierarchy(a, theta=theta))


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_solve_after_device_setup_is_identical(gpu, precision):
    """cfdb_system_setup_amg_device installs the same hierarchy as the host build, so the solve
    that follows is bit-identical; the device variant takes CUDA tensors."""
    import torch
    cb = gpu
    case = W.graded(20)
    up, lo, diag, src = _pressure(case)
    ctl = cb.SolveControl(1e-8 * np.linalg.norm(src), 200)
    out = []
    for how in ("host", "device", "device_tensors"):
        ds = cb.DeviceSolver(cb.build_csr_pattern(case.n, case.owner, case.neighbour))
        ds.set_precision(getattr(cb.Precision, precision))
        s = cb.AmgSettings(strength_threshold=0.04)
        if how == "host":
            ds.setup_amg(diag, up, lo, s, device=False)
        elif how == "device":
            ds.setup_amg(diag, up, lo, s, device=True)
        else:
            t = lambda v: torch.as_tensor(v, dtype=torch.float64, device="cuda")  # noqa: E731
            ds.setup_amg(t(diag), t(up), t(lo), s, device=True)
        x = np.zeros(case.n)
        st = ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, ctl)
        assert st.converged
        out.append((st.iterations, x))
    for it, x in out[1:]:
        assert it == out[0][0] and np.array_equal(x, out[0][1])


def test_plan_rebuild_from_device_levels(gpu):
    """A device setup keeps its levels on the device: changing the precision or the tuning
    afterwards rebuilds the plan from them, and the solves match plans built from a host setup."""
    cb = gpu
    case = W.graded(20)
    up, lo, diag, src = _pressure(case)
    ctl = cb.SolveControl(1e-8 * np.linalg.norm(src), 200)
    s = cb.AmgSettings(strength_threshold=0.04)

    def run(device, tuning=None):
        ds = cb.DeviceSolver(cb.build_csr_pattern(case.n, case.owner, case.neighbour))
        ds.setup_amg(diag, up, lo, s, device=device)
        ds.set_precision(cb.Precision.MIXED)  # rebuild after the setup
        if tuning is not None:
            ds.set_tuning(tuning)
        x = np.zeros(case.n)
        st = ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, ctl)
        assert st.converged
        return st.iterations, x

    for tuning in (None, cb.Tuning(wide_row=24, sell_rows=512, krylov_pair=0)):
        it_h, x_h = run(False, tuning)
        it_d, x_d = run(True, tuning)
        assert it_h == it_d and np.array_equal(x_h, x_d)


def test_dropped_levels_refuse_replan(gpu):
    """Without kept levels, a plan change after a device setup is refused until the next setup
    (it cannot rebuild the operators), and a new setup restores it."""
    cb = gpu
    case = W.graded(10)
    up, lo, diag, src = _pressure(case)
    ds = cb.DeviceSolver(cb.build_csr_pattern(case.n, case.owner, case.neighbour))
    ds.set_keep_levels(False)
    ds.setup_amg(diag, up, lo)
    x = np.zeros(case.n)
    assert ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, cb.SolveControl(1e-9, 100)).converged
    with pytest.raises(cb.CfdbError):
        ds.set_precision(cb.Precision.MIXED)
    ds.setup_amg(diag, up, lo)
    x[:] = 0.0
    assert ds.solve(diag, up, lo, src, x, cb.Method.Cg, True, cb.SolveControl(1e-9, 100)).converged
