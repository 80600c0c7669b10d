"""solve_scalar's GPU path on the device (cfdb_device_fv_scalar_system_device + the persistent
LDU solve) against the face-by-face restatement of scalar_transport.cpp:10-177 (oracle/scalar.py):
the assembled system and the fixed-cell field bit for bit, for every boundary-condition kind,
gradient scheme, with and without linear upwind, time term, under-relaxation and fixed cells;
the solve through cfd_b200.scalar.solve_scalar equals solve_ldu on the oracle's system."""
import numpy as np
import pytest

import oracle as O
import oracle.fvcells as F
import oracle.scalar as OS

pytestmark = pytest.mark.gpu


def _oracle_view(pv):
    return F.FvView(pv.n_cells, *pv.arrays())


def _equation(pv, seed, fixed=True, transient=True, relaxation=0.8, linear_upwind=True, gradient=1):
    rng = np.random.default_rng(seed)
    nc, nf, nif = pv.n_cells, pv.n_faces, pv.n_internal_faces
    nb = nf - nif
    eq = {
        "gamma_face": 0.01 + 0.05 * rng.random(nf),
        "su": rng.standard_normal(nc),
        "sp": np.where(rng.random(nc) < 0.8, -rng.random(nc), 0.3 * rng.random(nc)),
        "bc_kind": (np.arange(nb) % 4).astype(np.int32),
        "bc_value": rng.standard_normal(nb),
        "bc_coefficient": 0.5 + rng.random(nb),
        "relaxation": relaxation,
        "dt": 0.05 if transient else 0.0,
        "old_value": rng.standard_normal(nc) if transient else None,
        "capacity": 1.0 + rng.random(nc) if transient else None,
        "linear_upwind": linear_upwind,
        "gradient": gradient,
    }
    if fixed:
        fc = np.zeros(nc, np.uint8)
        fc[rng.choice(nc, size=max(1, nc // 50), replace=False)] = 1
        eq["fixed_cell"] = fc
        eq["fixed_value"] = rng.standard_normal(nc)
    flux = 0.1 * rng.standard_normal(nf)
    field = rng.standard_normal(nc)
    return eq, flux, field


def _device_eq(S, eq, T):
    return S.ScalarEquation(
        gamma_face=T(eq["gamma_face"]), su=T(eq["su"]), sp=T(eq["sp"]), bc_kind=T(eq["bc_kind"], "int32"),
        bc_value=T(eq["bc_value"]), bc_coefficient=T(eq["bc_coefficient"]),
        fixed_cell=T(eq["fixed_cell"], "uint8") if "fixed_cell" in eq else None,
        fixed_value=T(eq["fixed_value"]) if "fixed_value" in eq else None, relaxation=eq["relaxation"],
        dt=eq["dt"], old_value=T(eq["old_value"]) if eq["old_value"] is not None else None,
        capacity=T(eq["capacity"]) if eq["capacity"] is not None else None,
        linear_upwind=eq["linear_upwind"], gradient=eq["gradient"])


@pytest.fixture(scope="module", params=["tet", "graded_box"])
def mesh(request, gpu):
    from cfd_b200 import fv_device as D
    m = (gpu.Mesh.tet(5, 4, 4, jitter=0.2, seed=9) if request.param == "tet"
         else gpu.Mesh.box(6, 5, 4, xs=gpu.positions_graded(6, 3.0)))
    pv = D.mesh_view_of(m)
    fv = D.DeviceFv(pv)
    fv.set_face_geometry()
    return gpu, pv, fv


CASES = [dict(), dict(fixed=False), dict(transient=False, relaxation=1.0), dict(linear_upwind=False, gradient=0),
         dict(gradient=2), dict(relaxation=0.7, transient=False, fixed=False, gradient=2)]


@pytest.mark.parametrize("k", range(len(CASES)))
def test_scalar_system_bit_identical(mesh, k):
    import torch
    from cfd_b200 import scalar as S
    cb, pv, fv = mesh
    eq, flux, field = _equation(pv, seed=k, **CASES[k])
    v = _oracle_view(pv)
    want = OS.scalar_system(v, pv.delta_coeffs, pv.unit_normals, pv.face_areas, eq, flux, field)
    T = lambda a, dt="float64": torch.as_tensor(np.ascontiguousarray(a), dtype=getattr(torch, dt),  # noqa: E731
                                                device="cuda")
    nc, nif = pv.n_cells, pv.n_internal_faces
    up, lo = T(np.zeros(nif)), T(np.zeros(nif))
    dg, src, fd = T(np.zeros(nc)), T(np.zeros(nc)), T(field)
    S.scalar_system_device(fv, _device_eq(S, eq, T), T(flux), fd, up, lo, dg, src)
    torch.cuda.synchronize()
    got = [up.cpu().numpy(), lo.cpu().numpy(), dg.cpu().numpy(), src.cpu().numpy(), fd.cpu().numpy()]
    for name, a, b in zip(["upper", "lower", "diag", "source", "field"], got, want):
        assert np.array_equal(a, b), name


def test_solve_scalar_equals_solve_ldu_on_the_oracle_system(mesh):
    import torch
    from cfd_b200 import scalar as S
    cb, pv, fv = mesh
    eq, flux, field = _equation(pv, seed=42)
    v = _oracle_view(pv)
    up, lo, dg, src, fld = OS.scalar_system(v, pv.delta_coeffs, pv.unit_normals, pv.face_areas, eq, flux, field)
    nif = pv.n_internal_faces
    pat = cb.build_csr_pattern(pv.n_cells, pv.owner[:nif], pv.neighbour)
    settings = cb.LduSettings(method=int(cb.Method.BiCgStab), tolerance=1e-12, rel_tolerance=1e-9)
    ds_ref = cb.DeviceSolver(pat)
    x_ref = fld.copy()
    r_ref = ds_ref.solve_ldu(dg, up, lo, src, x_ref, settings)
    T = lambda a, dt="float64": torch.as_tensor(np.ascontiguousarray(a), dtype=getattr(torch, dt),  # noqa: E731
                                                device="cuda")
    ds = cb.DeviceSolver(pat)
    x = T(field)
    r = S.solve_scalar(ds, fv, _device_eq(S, eq, T), T(flux), x, settings)
    torch.cuda.synchronize()
    assert r.iterations == r_ref.iterations and r.iterations > 0
    assert r.initial_residual == r_ref.initial_residual and r.final_residual == r_ref.final_residual
    assert np.array_equal(x.cpu().numpy(), x_ref)
    a = O.ldu_to_csr(O.build_pattern(pv.n_cells, pv.owner[:nif], pv.neighbour), dg, up, lo)
    assert np.linalg.norm(src - a.matvec(x_ref)) < 1e-6 * np.linalg.norm(src)


def test_scalar_system_errors(mesh):
    import torch
    from cfd_b200 import fv_device as D
    from cfd_b200 import scalar as S
    cb, pv, fv = mesh
    eq, flux, field = _equation(pv, seed=3)
    T = lambda a, dt="float64": torch.as_tensor(np.ascontiguousarray(a), dtype=getattr(torch, dt),  # noqa: E731
                                                device="cuda")
    nc, nif = pv.n_cells, pv.n_internal_faces
    bufs = [T(np.zeros(nif)), T(np.zeros(nif)), T(np.zeros(nc)), T(np.zeros(nc))]
    fresh = D.DeviceFv(pv)  # no face geometry yet
    with pytest.raises(cb.NotReady):
        S.scalar_system_device(fresh, _device_eq(S, eq, T), T(flux), T(field), *bufs)
    bad = _device_eq(S, eq, T)
    bad.relaxation = 0.0
    with pytest.raises(cb.InvalidArgument):
        S.scalar_system_device(fv, bad, T(flux), T(field), *bufs)
    bad = _device_eq(S, eq, T)
    bad.fixed_value = None
    with pytest.raises(cb.InvalidArgument):
        S.scalar_system_device(fv, bad, T(flux), T(field), *bufs)
