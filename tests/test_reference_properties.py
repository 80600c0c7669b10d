"""Ports of the reference's own hot-path tests (tests/test_amg.cpp, tests/test_ldu_matrix.cpp)
run against the CPU oracle (the CPU AmgCg with Gauss-Seidel V-cycle, LduMatrix operations)
and against the product's host hierarchy setup. These properties are what the reference pins
for the parts whose Eigen arithmetic cannot be compiled here."""
import numpy as np
import pytest

import oracle as O
from oracle import meshref as M


def box(nx, ny, nz):
    return M.hex_box(nx, ny, nz, M.graded_positions(nx, 1.0), M.graded_positions(ny, 1.0),
                     M.graded_positions(nz, 1.0))


def build_poisson(m, dirichlet_xmin):
    """test_amg.cpp:44-72: A/|d| internal coefficients, xmin patch Dirichlet A/|Cf - C_P|."""
    nif = m.n_internal_faces
    n = m.n_cells
    up, lo, dg = np.zeros(nif), np.zeros(nif), np.zeros(n)
    for f in range(nif):
        s = m.face_areas[f]
        c = np.sqrt(s @ s) / np.linalg.norm(m.cell_centres[m.neighbour[f]] - m.cell_centres[m.owner[f]])
        up[f] = lo[f] = -c
        dg[m.owner[f]] += c
        dg[m.neighbour[f]] += c
    if dirichlet_xmin:
        start, count = m.patches[0]
        for f in range(start, start + count):
            s = m.face_areas[f]
            dg[m.owner[f]] += np.sqrt(s @ s) / np.linalg.norm(m.face_centres[f] - m.cell_centres[m.owner[f]])
    return up, lo, dg


def csr_of(m, up, lo, dg):
    pat = O.build_pattern(m.n_cells, m.owner, m.neighbour)
    return pat, O.ldu_to_csr(pat, dg, up, lo)


def manufactured(n, s):
    return np.sin(s * np.arange(n)) + 1.0


def test_hierarchy_is_built():
    """test_amg.cpp:155-170."""
    m = box(64, 64, 1)
    _, a = csr_of(m, *build_poisson(m, True))
    h = O.Hierarchy(a)
    assert h.levels >= 3
    for l in range(1, h.levels):
        assert h.a[l].n_rows < h.a[l - 1].n_rows
    assert h.a[-1].n_rows <= 400
    assert 1.0 <= h.operator_complexity <= 3.0


def test_pcg_converges_fast_and_independent_of_size():
    """test_amg.cpp:172-196 (CPU AmgCg: Gauss-Seidel V-cycle, LDLT coarse)."""
    iters = []
    for k in (32, 64, 128):
        m = box(k, k, 1)
        _, a = csr_of(m, *build_poisson(m, True))
        xe = manufactured(a.n_rows, 0.01)
        b = a.matvec(xe)
        tol = 1e-8 * np.linalg.norm(b)
        h = O.Hierarchy(a)
        x, it, res = h.pcg_gs(b, tol=tol, max_iterations=200)
        assert res <= tol and it < 30 and np.abs(x - xe).max() < 1e-5
        iters.append(it)
    assert iters[2] <= iters[0] + 10


def test_poisson_3d():
    """test_amg.cpp:198-202."""
    m = box(16, 16, 16)
    _, a = csr_of(m, *build_poisson(m, True))
    xe = manufactured(a.n_rows, 0.01)
    b = a.matvec(xe)
    tol = 1e-8 * np.linalg.norm(b)
    x, it, res = O.Hierarchy(a).pcg_gs(b, tol=tol, max_iterations=200)
    assert res <= tol and it < 30 and np.abs(x - xe).max() < 1e-5


def test_singular_neumann_with_reference():
    """test_amg.cpp:254-265: pure Neumann + set_reference(0, 3) gives x == 3."""
    m = box(40, 40, 1)
    up, lo, dg = build_poisson(m, False)
    src = np.zeros(m.n_cells)
    O.set_reference(dg, src, 0, 3.0)
    _, a = csr_of(m, up, lo, dg)
    # LduMatrix::solve tolerance translation (ldu_matrix.cpp:160-171) with tol 1e-12, rel 0
    x, it, res = O.Hierarchy(a).pcg_gs(src, tol=1e-12 * 1e3, max_iterations=200)
    assert np.abs(x - 3.0).max() < 1e-6


def chain():
    """test_ldu_matrix.cpp:26-56: 10-cell chain, Laplacian + Dirichlet ends."""
    m = box(10, 1, 1)
    nif = m.n_internal_faces
    up, lo = -np.ones(nif), -np.ones(nif)
    dg = np.zeros(10)
    for f in range(nif):
        dg[m.owner[f]] += 1.0
        dg[m.neighbour[f]] += 1.0
    return m, up, lo, dg


def test_ldu_multiply_matches_dense():
    """test_ldu_matrix.cpp:94-127."""
    m, up, lo, dg = chain()
    dg = dg.copy()
    dg[0] += 1.0
    dg[9] += 1.0
    dense = np.diag(dg)
    for f in range(m.n_internal_faces):
        dense[m.owner[f], m.neighbour[f]] += up[f]
        dense[m.neighbour[f], m.owner[f]] += lo[f]
    x = np.arange(1, 11, dtype=float)
    y = O.ldu_multiply(m.owner, m.neighbour, dg, up, lo, x)
    assert np.allclose(y, dense @ x, atol=1e-12, rtol=0)
    _, a = csr_of(m, up, lo, dg)
    assert np.array_equal(a.matvec(x), dense @ x)


def test_normalised_residual_zero_at_solution():
    """test_ldu_matrix.cpp:171-182."""
    m, up, lo, dg = chain()
    dg[0] += 1.0
    dg[9] += 1.0
    xe = np.sin(0.3 * np.arange(10))
    src = O.ldu_multiply(m.owner, m.neighbour, dg, up, lo, xe)
    assert O.normalised_residual(m.owner, m.neighbour, dg, up, lo, src, xe) < 1e-12


def test_set_reference_fixes_value():
    """test_ldu_matrix.cpp:184-197 through the accelerator-path Jacobi CG."""
    m, up, lo, dg = chain()
    src = np.zeros(10)
    O.set_reference(dg, src, 0, 2.0)
    _, a = csr_of(m, up, lo, dg)
    x, st = O.krylov(a, src, method=0, abs_tol=1e-12, max_iterations=1000)
    assert np.abs(x - 2.0).max() < 1e-6


@pytest.mark.parametrize("theta", [0.08, 0.04])
def test_product_setup_keeps_reference_properties(theta, cb):
    """The product's host setup on the same problems: identical to the oracle, same bounds."""
    m = box(64, 64, 1)
    _, a = csr_of(m, *build_poisson(m, True))
    h = cb.AmgHierarchy(cb.CsrView(a.n_rows, a.rp, a.ci, a.va), cb.AmgSettings(strength_threshold=theta))
    o = O.Hierarchy(a, theta=theta)
    assert h.levels() == o.levels >= 3
    assert abs(h.operator_complexity() - o.operator_complexity) == 0.0
    assert h.level_size(h.levels() - 1) <= 400
