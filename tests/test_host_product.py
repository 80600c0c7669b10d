"""Host-side product code against the oracle: the CSR pattern, the smoothed-aggregation setup
(bit-exact: aggregates, P, R, Galerkin operators, coarse inverse) and the synthetic mesh
generators (face / cell indexing bit-exact, geometry bit-exact against the restatement)."""
import numpy as np
import pytest

import oracle as O
from cfd_b200 import workloads as W
from oracle import meshref as M


def _pressure(case):
    up, lo, dg, dv = O.assemble(case.n, case.owner, case.neighbour, case.flux, case.gamma,
                                case.delta, 0.0)
    diag, src = case.finalize(up, lo, dg, dv)
    return up, lo, diag, src


CASES = {"cavity10": lambda: W.cavity(10), "graded12": lambda: W.graded(12),
         "tet6": lambda: W.tet(6), "tet7_sigma": lambda: W.tet(7, sigma=1.5, seed=5)}


@pytest.mark.parametrize("name", list(CASES))
def test_pattern_bitwise(cb, name):
    case = CASES[name]()
    p = cb.build_csr_pattern(case.n, case.owner, case.neighbour)
    o = O.build_pattern(case.n, case.owner, case.neighbour)
    for a, b in (("row_ptr", "row_ptr"), ("col", "col"), ("diag_pos", "diag_pos"),
                 ("upper_pos", "upper_pos"), ("lower_pos", "lower_pos")):
        assert np.array_equal(getattr(p, a), getattr(o, b)), a


@pytest.mark.parametrize("theta", [0.08, 0.04, 0.0])
@pytest.mark.parametrize("name", list(CASES))
def test_amg_setup_bitwise(cb, name, theta):
    case = CASES[name]()
    up, lo, diag, _ = _pressure(case)
    pat = O.build_pattern(case.n, case.owner, case.neighbour)
    a = O.ldu_to_csr(pat, diag, up, lo)
    o = O.Hierarchy(a, theta=theta)
    h = cb.AmgHierarchy(cb.CsrView(a.n_rows, a.rp, a.ci, a.va),
                        cb.AmgSettings(strength_threshold=theta))
    assert h.levels() == o.levels
    for l in range(o.levels):
        m = h.level_matrix(l)
        assert np.array_equal(m.row_ptr, o.a[l].rp) and np.array_equal(m.col, o.a[l].ci)
        assert np.array_equal(m.val, o.a[l].va)
        if l + 1 < o.levels:
            agg, n_agg = h.aggregates(l)
            assert np.array_equal(agg, o.aggregates[l]) and n_agg == o.a[l + 1].n_rows
            for got, want in ((h.level_prolongation(l), o.p[l]), (h.level_restriction(l), o.r[l])):
                assert np.array_equal(got.row_ptr, want.rp) and np.array_equal(got.col, want.ci)
                assert np.array_equal(got.val, want.va)
    assert np.array_equal(h.coarse_inverse(), o.coarse_inverse)


def test_aggregation_handles_isolated_and_weak_rows(cb):
    """Rows without strong connections become singleton aggregates (amg.cpp pass 3); a
    diagonal matrix therefore does not coarsen and the hierarchy has one level."""
    n = 50
    rp = np.arange(n + 1, dtype=np.int32)
    ci = np.arange(n, dtype=np.int32)
    va = np.linspace(1.0, 2.0, n)
    o = O.Hierarchy(O.Csr(n, n, rp, ci, va), coarse_size=10)
    h = cb.AmgHierarchy(cb.CsrView(n, rp, ci, va), cb.AmgSettings(coarse_size=10))
    assert o.levels == 1 and h.levels() == 1
    agg, n_agg = O.aggregate(O.Csr(n, n, rp, ci, va), va)
    assert n_agg == n and np.array_equal(agg, np.arange(n))


def test_setup_rejects_bad_input(cb):
    with pytest.raises(cb.InvalidArgument):
        cb.AmgHierarchy(cb.CsrView(3, [0, 1, 2, 4], [0, 1, 2, 7], [1.0, 1.0, 1.0, 1.0]))
    with pytest.raises(cb.InvalidArgument):
        cb.build_csr_pattern(4, [0, 1], [1, 9])


def test_box_mesh_matches_restatement(cb):
    xs = M.two_sided_positions(5, 1.3)
    assert np.array_equal(cb.positions_two_sided(5, 1.3), np.array(xs))
    assert np.array_equal(cb.positions_graded(6, 3.0), np.array(M.graded_positions(6, 3.0)))
    ys = M.graded_positions(3, 2.0)
    zs = M.graded_positions(2, 1.0)
    m = cb.Mesh.box(5, 3, 2, xs, ys, zs)
    r = M.hex_box(5, 3, 2, xs, ys, zs)
    assert np.array_equal(m.owner, r.owner) and np.array_equal(m.neighbour, r.neighbour)
    assert np.array_equal(m.face_nodes, np.concatenate([np.array(f) for f in r.faces]))
    for got, want in ((m.face_centres, r.face_centres), (m.face_areas, r.face_areas),
                      (m.cell_centres, r.cell_centres), (m.cell_volumes, r.cell_volumes)):
        assert np.array_equal(got, want)
    d, w = r.fv_geometry()
    assert np.array_equal(m.delta, d) and np.array_equal(m.weights, w)
    assert abs(m.cell_volumes.sum() - 1.0) < 1e-12


def test_tet_mesh_matches_restatement(cb):
    m = cb.Mesh.tet(3, 3, 2, jitter=0.2, seed=3)
    r = M.tet_box(3, 3, 2, [tuple(p) for p in m.points])
    assert np.array_equal(m.owner, r.owner) and np.array_equal(m.neighbour, r.neighbour)
    assert np.array_equal(m.cell_volumes, r.cell_volumes)
    assert np.array_equal(m.cell_centres, r.cell_centres)
    d, w = r.fv_geometry()
    assert np.array_equal(m.delta, d) and np.array_equal(m.weights, w)
    assert (m.cell_volumes > 0).all() and abs(m.cell_volumes.sum() - 1.0) < 1e-12
    # the jitter moved interior nodes and kept boundary coordinates on the walls
    p = m.points
    assert ((p >= 0.0) & (p <= 1.0)).all()


def test_face_ordering_contract(cb):
    """mesh.hpp:53-55: internal faces sorted by (owner, neighbour) with owner < neighbour."""
    for m in (cb.Mesh.box(6, 5, 4), cb.Mesh.tet(4, 3, 3, jitter=0.15, seed=1)):
        own = m.owner[:m.n_internal_faces]
        nei = m.neighbour
        assert (own < nei).all()
        key = own.astype(np.int64) * m.n_cells + nei
        assert (np.diff(key) > 0).all()


def test_workload_sizes(cb):
    c = W.cavity(32)
    assert c.n == 32768 and c.n_faces == 95232  # configs: 32^3 box
    t = W.tet(5)
    # 6 tets per box cell; internal faces = (4 * 6 n^3 - 12 n^2) / 2 (12 n^2 boundary triangles)
    assert t.n == 6 * 125 and t.n_faces == 12 * 125 - 6 * 25
    assert abs(c.source0).max() == 0.0  # cavity: divergence-only right-hand side
    g = W.graded(8)
    assert abs(g.source0.mean()) < 1e-14
    edges = W.box_edges()
    assert len(edges) == 256 and min(edges) >= 8 and max(edges) <= 64
