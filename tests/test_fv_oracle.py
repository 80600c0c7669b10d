"""The finite-volume cell-kernel oracle (oracle/fvcells.py) pinned against the reference's own
DeviceFv host path (src/gpu/src/fv_openmp.cpp + fv_device.cpp, compiled unchanged into
oracle/_ref): bit-identical gradients (Gauss, least squares, skewness-corrected Gauss), vector
gradients, scalar corrections and momentum corrections in every flag combination; the
reference test's properties (test_gpu.cpp:370-450: corrected Gauss exact for linear fields on
a skewed mesh, scalar corrections equal to the face loop); the product's FvMeshView builder
against the oracle's."""
import itertools

import numpy as np
import pytest

import oracle.fvcells as F
from oracle import meshref as M


def _field(x):
    return np.sin(2.0 * x[:, 0]) + x[:, 1] * x[:, 1] + x[:, 0] * x[:, 2]


def _skewed_tet(nx=6, ny=5, nz=4):
    xs, ys, zs = [list(np.linspace(0.0, 1.0, n + 1)) for n in (nx, ny, nz)]
    pts = [(x + 0.03 * np.sin(7 * y + 3 * z), y + 0.03 * np.cos(5 * x + 2 * z), z + 0.02 * np.sin(4 * x + 6 * y))
           for (x, y, z) in M.lattice(nx, ny, nz, xs, ys, zs)]
    return M.tet_box(nx, ny, nz, pts)


def _skewed_hex(nx=6, ny=5, nz=4):
    xs, ys, zs = [list(np.linspace(0.0, 1.0, n + 1)) for n in (nx, ny, nz)]
    pts = [(x + 0.15 * y / ny * (1.0 - x), y + 0.02 * np.sin(5 * x), z + 0.1 * x * y)
           for (x, y, z) in M.lattice(nx, ny, nz, xs, ys, zs)]
    P = lambda i, j, k: M.pid(nx, ny, i, j, k)  # noqa: E731
    cells = [("hex", (P(i, j, k), P(i + 1, j, k), P(i + 1, j + 1, k), P(i, j + 1, k), P(i, j, k + 1),
                      P(i + 1, j, k + 1), P(i + 1, j + 1, k + 1), P(i, j + 1, k + 1)))
             for k in range(nz) for j in range(ny) for i in range(nx)]
    return M.build_mesh(pts, cells, M.box_tags(nx, ny, nz), 6)


def _graded_hex():
    return M.hex_box(5, 4, 3, M.graded_positions(5, 4.0), M.graded_positions(4, 0.5), M.graded_positions(3, 2.0))


MESHES = {"skewed_tet": _skewed_tet, "skewed_hex": _skewed_hex, "graded_hex": _graded_hex}


@pytest.fixture(scope="module", params=list(MESHES))
def case(request):
    mesh = MESHES[request.param]()
    mesh.weights = mesh.fv_geometry()[1]
    v = F.view_of(mesh)
    ref = F.RefFv(v) if F._ref_lib() is not None else None
    return request.param, mesh, v, ref


def _fields(v):
    bc = v.cf[v.nif:]
    u = np.stack([_field(v.cc), np.cos(3.0 * v.cc[:, 1]), v.cc[:, 0] * v.cc[:, 2] - v.cc[:, 1]], axis=1)
    ub = np.stack([_field(bc), np.cos(3.0 * bc[:, 1]), bc[:, 0] * bc[:, 2] - bc[:, 1]], axis=1)
    flux = np.sin(0.7 * np.arange(v.nf))
    gamma = 0.05 + 0.01 * (np.arange(v.nf) % 5)
    nu = 0.01 * (1.0 + 0.5 * np.cos(np.arange(v.nif)))
    return _field(v.cc), _field(bc), u, ub, flux, gamma, nu


def _need_ref(ref):
    if ref is None:
        pytest.skip("the reference's host path is not built here (oracle/_ref)")


@pytest.mark.parametrize("scheme", [0, 1, 2])
def test_gradients_bit_identical_to_reference(case, scheme):
    _, _, v, ref = case
    _need_ref(ref)
    phi, bv, u, ub, *_ = _fields(v)
    assert np.array_equal(F.gradient(v, phi, bv, scheme), ref.gradient(phi, bv, scheme))
    assert np.array_equal(F.vector_gradient(v, u, ub, scheme), ref.vector_gradient(u, ub, scheme))


@pytest.mark.parametrize("scheme,linear_upwind", list(itertools.product([0, 1, 2], [False, True])))
def test_scalar_corrections_bit_identical_to_reference(case, scheme, linear_upwind):
    _, _, v, ref = case
    _need_ref(ref)
    phi, bv, _, _, flux, gamma, _ = _fields(v)
    src = np.full(v.nc, 0.5)
    a = F.scalar_corrections(v, phi, bv, scheme, flux, gamma, linear_upwind, src)
    b = ref.scalar_corrections(phi, bv, scheme, flux, gamma, linear_upwind, src)
    assert np.array_equal(a, b)


def test_momentum_corrections_bit_identical_to_reference(case):
    _, _, v, ref = case
    _need_ref(ref)
    _, _, u, ub, flux, _, nu = _fields(v)
    eps2 = (1e-3, 2e-3, 3e-3)
    for scheme in (1, 2):
        g = ref.vector_gradient(u, ub, scheme)
        for lu, lim, venkat, central, tr in itertools.product([0, 1], [0, 1], [0, 1], [0.0, 0.75], [0, 1]):
            src = np.full((v.nc, 3), 0.25)
            a = F.momentum_corrections(v, u, ub, g, flux[: v.nif], nu, lu, lim, venkat, eps2, central, tr, src)
            b = ref.momentum_corrections(flux[: v.nif], nu, lu, lim, venkat, eps2, central, tr, src)
            assert np.array_equal(a, b), (scheme, lu, lim, venkat, central, tr)


def test_reference_momentum_needs_a_vector_gradient():
    mesh = _graded_hex()
    mesh.weights = mesh.fv_geometry()[1]
    v = F.view_of(mesh)
    if F._ref_lib() is None:
        pytest.skip("reference not built")
    ref = F.RefFv(v)
    with pytest.raises(RuntimeError):  # fv_openmp.cpp:205-207: std::logic_error
        ref.momentum_corrections(np.zeros(v.nif), np.zeros(v.nif), True, False, False, None, 0.0, False,
                                 np.zeros((v.nc, 3)))


def test_corrected_gauss_exact_for_linear_fields(case):
    """test_gpu.cpp:397-417: exact on a skewed mesh, where plain Gauss is not."""
    name, _, v, _ = case
    a = np.array([0.7, -1.3, 2.1])
    lin, lin_b = v.cc @ a + 0.4, v.cf[v.nif:] @ a + 0.4
    err_c = np.abs(F.gradient(v, lin, lin_b, 2) - a).max()
    err_l = np.abs(F.gradient(v, lin, lin_b, 1) - a).max()
    assert err_c < 1e-10 and err_l < 1e-10
    if name != "graded_hex":
        assert np.abs(F.gradient(v, lin, lin_b, 0) - a).max() > 1e-3


def test_scalar_corrections_equal_the_face_loop(case):
    """test_gpu.cpp:419-449: the face loop -F (g_up . (x_f - x_up)) + gamma k . g_f."""
    _, _, v, _ = case
    phi, bv, _, _, flux, gamma, _ = _fields(v)
    g = F.gradient(v, phi, bv, 1)
    ref = np.full(v.nc, 0.5)
    for f in range(v.nif):
        p, n = v.own[f], v.nei[f]
        up = p if flux[f] >= 0.0 else n
        w = v.w[f]
        e = -flux[f] * g[up] @ (v.cf[f] - v.cc[up]) + gamma[f] * v.kv[f] @ (w * g[p] + (1.0 - w) * g[n])
        ref[p] += e
        ref[n] -= e
    out = F.scalar_corrections(v, phi, bv, 1, flux, gamma, True, np.full(v.nc, 0.5))
    assert np.allclose(out, ref, rtol=0, atol=1e-12)


def test_product_mesh_view_matches_the_oracle(case):
    from cfd_b200 import fv_device as D
    _, mesh, v, _ = case
    pv = D.mesh_view(mesh.n_cells, mesh.owner, mesh.neighbour, mesh.face_areas, mesh.face_centres,
                     mesh.cell_centres, mesh.cell_volumes, mesh.weights)
    assert np.array_equal(pv.cell_offsets, v.start) and np.array_equal(pv.cell_faces, v.faces)
    for a, b in ((pv.correction, v.kv), (pv.lsq_d, v.lsq_d), (pv.lsq_inverse, v.lsq)):
        assert np.allclose(a, b, rtol=1e-12, atol=1e-12 * np.abs(b).max())


def test_scalar_restatement_conserves_and_holds_constants():
    """oracle/scalar.py (the restatement of solve_scalar's assembly): with no flux and
    zero-gradient walls the rows sum to zero; with fixed-value walls at c and no sources the
    constant field c satisfies A c = b exactly up to rounding."""
    import oracle.scalar as OS
    mesh = _skewed_tet(4, 3, 3)
    mesh.weights = mesh.fv_geometry()[1]
    v = F.view_of(mesh)
    nb = v.nf - v.nif
    area = np.sqrt((v.sf ** 2).sum(axis=1))
    un = v.sf / area[:, None]
    d = np.concatenate([v.cc[v.nei] - v.cc[v.own[: v.nif]], v.cf[v.nif:] - v.cc[v.own[v.nif:]]])
    dc = area * area / np.maximum((v.sf * d).sum(axis=1), 0.05 * area * np.sqrt((d * d).sum(axis=1)))
    eq = {"gamma_face": np.full(v.nf, 0.1), "su": np.zeros(v.nc), "sp": np.zeros(v.nc),
          "bc_kind": np.full(nb, OS.ZERO_GRADIENT, np.int32), "bc_value": np.zeros(nb),
          "bc_coefficient": np.zeros(nb), "linear_upwind": False, "gradient": 0}
    field = np.zeros(v.nc)
    up, lo, dg, src, _ = OS.scalar_system(v, dc, un, area, eq, np.zeros(v.nf), field)
    rows = dg.copy()
    np.add.at(rows, v.own[: v.nif], up)
    np.add.at(rows, v.nei, lo)
    assert np.abs(rows).max() < 1e-12 * np.abs(dg).max()
    eq["bc_kind"] = np.full(nb, OS.FIXED_VALUE, np.int32)
    eq["bc_value"] = np.full(nb, 2.5)
    up, lo, dg, src, _ = OS.scalar_system(v, dc, un, area, eq, np.zeros(v.nf), np.full(v.nc, 2.5))
    ax = 2.5 * dg
    np.add.at(ax, v.own[: v.nif], 2.5 * up)
    np.add.at(ax, v.nei, 2.5 * lo)
    assert np.allclose(ax, src, rtol=0, atol=1e-12 * np.abs(src).max())


@pytest.mark.parametrize("seed", [0, 1])
def test_ragged_random_view_bit_identical_to_reference(seed):
    """Random addressing: cells with no faces, only boundary faces, or up to ~20 faces."""
    v = F.random_view(150, 700, 120, seed)
    deg = np.diff(v.start)
    assert deg.min() <= 3 and deg.max() > 8
    if F._ref_lib() is None:
        pytest.skip("reference not built")
    ref = F.RefFv(v)
    rng = np.random.default_rng(seed)
    phi, bv = rng.standard_normal(v.nc), rng.standard_normal(v.nf - v.nif)
    u, ub = rng.standard_normal((v.nc, 3)), rng.standard_normal((v.nf - v.nif, 3))
    flux, gamma, nu = rng.standard_normal(v.nf), rng.random(v.nf), rng.random(v.nif)
    for scheme in (0, 1, 2):
        assert np.array_equal(F.gradient(v, phi, bv, scheme), ref.gradient(phi, bv, scheme))
        g = ref.vector_gradient(u, ub, scheme)
        assert np.array_equal(F.vector_gradient(v, u, ub, scheme), g)
        src = np.full(v.nc, 0.5)
        assert np.array_equal(F.scalar_corrections(v, phi, bv, scheme, flux, gamma, True, src),
                              ref.scalar_corrections(phi, bv, scheme, flux, gamma, True, src))
        for venkat in (0, 1):
            m0 = np.full((v.nc, 3), 0.25)
            assert np.array_equal(F.momentum_corrections(v, u, ub, g, flux[: v.nif], nu, 1, 1, venkat, (1e-3,) * 3,
                                                         0.75, 1, m0),
                                  ref.momentum_corrections(flux[: v.nif], nu, 1, 1, venkat, (1e-3,) * 3, 0.75, 1, m0))
