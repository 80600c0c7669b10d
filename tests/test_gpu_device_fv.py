"""DeviceFv on the device (cfdb_device_fv_*) against the oracle's restatement of fv_cell.inc /
fv_openmp.cpp and, where it was built, the reference's own host path: bit-identical gradients,
vector gradients, scalar and momentum corrections (every flag combination), host-array and
device-array entry points alike, and the reference's error behaviour."""
import itertools

import numpy as np
import pytest

import oracle.fvcells as F

pytestmark = pytest.mark.gpu


def _field(x):
    return np.sin(2.0 * x[:, 0]) + x[:, 1] * x[:, 1] + x[:, 0] * x[:, 2]


def _oracle_view(pv):
    return F.FvView(pv.n_cells, pv.owner, pv.neighbour, pv.cell_offsets, pv.cell_faces, pv.weight, pv.sf,
                    pv.face_centre, pv.cell_centre, pv.volume, pv.correction, pv.lsq_d, pv.lsq_inverse)


def _fields(v, seed=0):
    rng = np.random.default_rng(seed)
    bc = v.cf[v.nif:]
    u = np.stack([_field(v.cc), np.cos(3.0 * v.cc[:, 1]), v.cc[:, 0] * v.cc[:, 2] - v.cc[:, 1]], axis=1)
    ub = np.stack([_field(bc), np.cos(3.0 * bc[:, 1]), bc[:, 0] * bc[:, 2] - bc[:, 1]], axis=1)
    flux = rng.standard_normal(v.nif)
    gamma = 0.05 + 0.01 * (np.arange(v.nif) % 5)
    nu = 0.01 * (1.0 + 0.5 * np.cos(np.arange(v.nif)))
    return _field(v.cc), _field(bc), u, ub, flux, gamma, nu


def _meshes(cb):
    return {
        "tet_jitter": cb.Mesh.tet(6, 5, 4, jitter=0.22, seed=3),
        "graded_box": cb.Mesh.box(7, 5, 4, xs=cb.positions_graded(7, 5.0), zs=cb.positions_graded(4, 0.3)),
    }


@pytest.fixture(scope="module", params=["tet_jitter", "graded_box"])
def case(request, gpu):
    from cfd_b200 import fv_device as D
    mesh = _meshes(gpu)[request.param]
    pv = D.mesh_view_of(mesh)
    return D, D.DeviceFv(pv), _oracle_view(pv)


@pytest.mark.parametrize("scheme", [0, 1, 2])
def test_gradients_bit_identical(case, scheme):
    D, fv, v = case
    phi, bv, u, ub, *_ = _fields(v)
    assert fv.on_device()
    assert np.array_equal(fv.gradient(phi, bv, scheme), F.gradient(v, phi, bv, scheme))
    assert np.array_equal(fv.vector_gradient(u, ub, scheme), F.vector_gradient(v, u, ub, scheme))


@pytest.mark.parametrize("scheme,linear_upwind", list(itertools.product([0, 1, 2], [False, True])))
def test_scalar_corrections_bit_identical(case, scheme, linear_upwind):
    D, fv, v = case
    phi, bv, _, _, flux, gamma, _ = _fields(v, seed=scheme)
    src = np.linspace(-1.0, 1.0, v.nc)
    want = F.scalar_corrections(v, phi, bv, scheme, flux, gamma, linear_upwind, src)
    fv.scalar_corrections(phi, bv, scheme, flux, gamma, linear_upwind, src)
    assert np.array_equal(src, want)


@pytest.mark.parametrize("scheme", [1, 2])
def test_momentum_corrections_bit_identical(case, scheme):
    D, fv, v = case
    _, _, u, ub, flux, _, nu = _fields(v, seed=10 + scheme)
    eps2 = np.array([1e-3, 2e-3, 3e-3])
    g = fv.vector_gradient(u, ub, scheme)
    assert np.array_equal(g, F.vector_gradient(v, u, ub, scheme))
    for lu, lim, venkat, central, tr in itertools.product([0, 1], [0, 1], [0, 1], [0.0, 0.75], [0, 1]):
        src = np.full((v.nc, 3), 0.25)
        want = F.momentum_corrections(v, u, ub, g, flux, nu, lu, lim, venkat, eps2, central, tr, src)
        fv.momentum_corrections(flux, nu, lu, lim, venkat, eps2, central, tr, src)
        assert np.array_equal(src, want), (lu, lim, venkat, central, tr)


def test_device_arrays_equal_host_arrays(case):
    import torch
    D, fv, v = case
    phi, bv, u, ub, flux, gamma, nu = _fields(v, seed=5)
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")  # noqa: E731
    for scheme in (0, 1, 2):
        g = torch.empty((v.nc, 3), dtype=torch.float64, device="cuda")
        fv.gradient_device(T(phi), T(bv), scheme, g)
        assert np.array_equal(g.cpu().numpy(), fv.gradient(phi, bv, scheme))
        vg = torch.empty((v.nc, 9), dtype=torch.float64, device="cuda")
        fv.vector_gradient_device(T(u), T(ub), scheme, vg)
        host_g = fv.vector_gradient(u, ub, scheme)
        assert np.array_equal(vg.cpu().numpy(), host_g)
        s = T(np.full(v.nc, 0.5))
        fv.scalar_corrections_device(T(phi), T(bv), scheme, T(flux), T(gamma), True, s)
        s_host = np.full(v.nc, 0.5)
        fv.scalar_corrections(phi, bv, scheme, flux, gamma, True, s_host)
        assert np.array_equal(s.cpu().numpy(), s_host)
        m = T(np.full((v.nc, 3), 0.25))
        fv.momentum_corrections_device(T(u), T(ub), vg, T(flux), T(nu), True, True, True, [1e-3, 2e-3, 3e-3],
                                       0.75, True, m)
        m_host = np.full((v.nc, 3), 0.25)
        fv.momentum_corrections(flux, nu, True, True, True, [1e-3, 2e-3, 3e-3], 0.75, True, m_host)
        assert np.array_equal(m.cpu().numpy(), m_host)


def test_device_equals_the_reference_host_path(gpu):
    """Against the reference's own fv_openmp.cpp (compiled into oracle/_ref) where present."""
    from cfd_b200 import fv_device as D
    if F._ref_lib() is None:
        pytest.skip("the reference's host path is not built (oracle/_ref)")
    pv = D.mesh_view_of(gpu.Mesh.tet(5, 4, 4, jitter=0.24, seed=11))
    v = _oracle_view(pv)
    ref, fv = F.RefFv(v), D.DeviceFv(pv)
    phi, bv, u, ub, flux, gamma, nu = _fields(v, seed=7)
    for scheme in (0, 1, 2):
        assert np.array_equal(fv.gradient(phi, bv, scheme), ref.gradient(phi, bv, scheme))
        assert np.array_equal(fv.vector_gradient(u, ub, scheme), ref.vector_gradient(u, ub, scheme))
        a, b = np.full(v.nc, 0.5), np.full(v.nc, 0.5)
        fv.scalar_corrections(phi, bv, scheme, flux, gamma, True, a)
        assert np.array_equal(a, ref.scalar_corrections(phi, bv, scheme, flux, gamma, True, b))
        m = np.full((v.nc, 3), 0.25)
        fv.momentum_corrections(flux, nu, True, True, scheme == 2, [1e-3, 1e-3, 1e-3], 0.75, True, m)
        want = ref.momentum_corrections(flux, nu, True, True, scheme == 2, [1e-3, 1e-3, 1e-3], 0.75, True,
                                        np.full((v.nc, 3), 0.25))
        assert np.array_equal(m, want)


def test_larger_tet_mesh_bit_identical(gpu):
    from cfd_b200 import fv_device as D
    pv = D.mesh_view_of(gpu.Mesh.tet(20, 20, 20, jitter=0.2, seed=1))  # 48,000 cells
    v = _oracle_view(pv)
    fv = D.DeviceFv(pv)
    _, _, u, ub, flux, _, nu = _fields(v, seed=2)
    g = fv.vector_gradient(u, ub, 2)
    assert np.array_equal(g, F.vector_gradient(v, u, ub, 2))
    src = np.zeros((v.nc, 3))
    fv.momentum_corrections(flux, nu, True, True, False, None, 0.0, True, src)
    assert np.array_equal(src, F.momentum_corrections(v, u, ub, g, flux, nu, True, True, False, None, 0.0, True,
                                                      np.zeros((v.nc, 3))))


def test_errors_follow_the_reference(gpu):
    from cfd_b200 import fv_device as D
    pv = D.mesh_view_of(gpu.Mesh.box(3, 3, 2))
    fv = D.DeviceFv(pv)
    with pytest.raises(gpu.NotReady):  # fv_openmp.cpp:205-207
        fv.momentum_corrections(np.zeros(pv.n_internal_faces), np.zeros(pv.n_internal_faces), True, False, False,
                                None, 0.0, False, np.zeros((pv.n_cells, 3)))
    with pytest.raises(gpu.InvalidArgument):
        fv.gradient(np.zeros(pv.n_cells), np.zeros(pv.n_boundary_faces), 3)
    bad = D.MeshView(pv.n_cells, pv.owner, pv.neighbour, pv.cell_offsets, pv.cell_faces.copy(), pv.weight, pv.sf,
                     pv.face_centre, pv.cell_centre, pv.volume, pv.correction, pv.lsq_d, pv.lsq_inverse)
    bad.cell_faces[3] = pv.n_faces  # out of range: rejected on the host, never reaches a kernel
    with pytest.raises(gpu.InvalidArgument):
        D.DeviceFv(bad)
    bad2 = D.MeshView(0, pv.owner, pv.neighbour, pv.cell_offsets[:1], pv.cell_faces, pv.weight, pv.sf,
                      pv.face_centre, pv.cell_centre, pv.volume, pv.correction, pv.lsq_d, pv.lsq_inverse)
    with pytest.raises(gpu.InvalidArgument):  # fv_device.cpp:25-27
        D.DeviceFv(bad2)


@pytest.mark.parametrize("sizes,seed", [((150, 700, 120), 0), ((300, 350, 100), 0), ((400, 380, 120), 1)])
def test_ragged_views_bit_identical(gpu, sizes, seed):
    """Random addressing with cells of 0 to ~20 faces: the face sums take their generic loop
    (more than 8 faces) or the 8-face batch, and every call still equals the oracle."""
    from cfd_b200 import fv_device as D
    v = F.random_view(*sizes, seed)
    pv = D.MeshView(v.nc, v.own, v.nei, v.start, v.faces, v.w, v.sf, v.cf, v.cc, v.vol, v.kv, v.lsq_d, v.lsq)
    fv = D.DeviceFv(pv)
    rng = np.random.default_rng(seed + 100)
    nb = v.nf - v.nif
    phi, bv = rng.standard_normal(v.nc), rng.standard_normal(nb)
    u, ub = rng.standard_normal((v.nc, 3)), rng.standard_normal((nb, 3))
    flux, gamma, nu = rng.standard_normal(v.nf), rng.random(v.nf), rng.random(v.nif)
    for scheme in (0, 1, 2):
        assert np.array_equal(fv.gradient(phi, bv, scheme), F.gradient(v, phi, bv, scheme))
        g = fv.vector_gradient(u, ub, scheme)
        assert np.array_equal(g, F.vector_gradient(v, u, ub, scheme))
        src = np.linspace(-1.0, 1.0, v.nc)
        want = F.scalar_corrections(v, phi, bv, scheme, flux, gamma, True, src)
        fv.scalar_corrections(phi, bv, scheme, flux, gamma, True, src)
        assert np.array_equal(src, want)
        for venkat in (False, True):
            m = np.full((v.nc, 3), 0.25)
            want = F.momentum_corrections(v, u, ub, g, flux[: v.nif], nu, True, True, venkat, [1e-3] * 3, 0.75,
                                          True, m)
            fv.momentum_corrections(flux, nu, True, True, venkat, [1e-3] * 3, 0.75, True, m)
            assert np.array_equal(m, want)


def test_single_cell_mesh(gpu):
    """No internal faces (the reference pads its empty neighbour array, fv_device.cpp:45-49)."""
    from cfd_b200 import fv_device as D
    pv = D.mesh_view_of(gpu.Mesh.box(1, 1, 1))
    assert pv.n_internal_faces == 0 and pv.n_faces == 6
    v = _oracle_view(pv)
    fv = D.DeviceFv(pv)
    bv = pv.face_centre[:, 0] * 2.0 - pv.face_centre[:, 1]
    for scheme in (0, 1, 2):
        assert np.array_equal(fv.gradient(np.array([0.3]), bv, scheme), F.gradient(v, [0.3], bv, scheme))
    u, ub = np.array([[1.0, 2.0, 3.0]]), np.stack([bv, -bv, 2 * bv], axis=1)
    g = fv.vector_gradient(u, ub, 1)
    m = np.zeros((1, 3))
    fv.momentum_corrections(np.zeros(0), np.zeros(0), True, True, True, [1e-3] * 3, 0.0, True, m)
    assert np.array_equal(m, F.momentum_corrections(v, u, ub, g, np.zeros(0), np.zeros(0), True, True, True,
                                                    [1e-3] * 3, 0.0, True, np.zeros((1, 3))))
