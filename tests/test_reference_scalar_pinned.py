"""solve_scalar's GPU path (scalar_transport.cpp:49-183), the reference's own code compiled
unchanged against the Eigen stand-in, against the face-by-face restatement that the device
assembly is checked against (oracle/scalar.py, test_gpu_scalar_step.py), on the CPU.

The reference assembles and solves the equation with GpuBiCgStab on its own host path (its
DeviceFv corrections in fv_openmp.cpp, its assemble_convection_diffusion, its LduMatrix::solve
without an AmgCache). The restatement assembles the system from the same inputs and solves it
with the reference's own LduMatrix::solve, also without a cache. The solutions and the solve
records come out equal bit for bit, so the restated assembly is the reference's: every boundary
condition kind, gradient scheme, with and without linear upwind, time term, under-relaxation
and fixed cells, on a graded hex box and a jittered tet box."""
import numpy as np
import pytest

RX = pytest.importorskip("oracle.reference")
if not RX.available() or not hasattr(RX.lib(), "refx_scalar_solve"):
    pytest.skip("reference build with the scalar transport step not available", allow_module_level=True)

import oracle.fvcells as F  # noqa: E402
import oracle.scalar as OS  # noqa: E402
from oracle import flowref  # noqa: E402

SOLVER = ("GpuBiCgStab", 1e-12, 1e-9, 1000)


@pytest.fixture(scope="module", autouse=True)
def one_openmp_thread():
    """The reference's host path reduces with OpenMP; one thread fixes its summation order, so
    that two solves of the same system agree bit for bit."""
    import ctypes
    try:
        gomp = ctypes.CDLL("libgomp.so.1")
    except OSError:
        pytest.skip("libgomp not found")
    before = gomp.omp_get_max_threads()
    gomp.omp_set_num_threads(1)
    yield
    gomp.omp_set_num_threads(before)


def _equation(nc, nf, nb, seed, fixed=True, transient=True, relaxation=0.8, linear_upwind=True, gradient=1):
    rng = np.random.default_rng(seed)
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
    return eq, 0.1 * rng.standard_normal(nf), rng.standard_normal(nc)


CASES = [dict(), dict(fixed=False), dict(transient=False, relaxation=1.0), dict(linear_upwind=False, gradient=0),
         dict(gradient=2), dict(relaxation=0.7, transient=False, fixed=False, gradient=2)]


@pytest.fixture(scope="module", params=["box", "tet"])
def meshes(request):
    import cfd_b200 as cb
    from cfd_b200 import fv_device as D
    ref = flowref.mesh(request.param)
    prod = (cb.Mesh.box(len(flowref.BOX_XS) - 1, 5, 4, xs=flowref.BOX_XS) if request.param == "box"
            else cb.Mesh.tet(*flowref.TET_N, jitter=flowref.TET_JITTER, seed=flowref.TET_SEED))
    assert np.array_equal(prod.owner, ref.owner) and np.array_equal(prod.face_areas, ref.face_areas)
    return ref, D.mesh_view_of(prod)


@pytest.mark.parametrize("k", range(len(CASES)))
def test_scalar_step_equals_the_reference_solve_scalar(meshes, k):
    ref, pv = meshes
    nc, nf, nif = pv.n_cells, pv.n_faces, pv.n_internal_faces
    eq, flux, field = _equation(nc, nf, nf - nif, seed=k, **CASES[k])
    x_ref, r_ref = RX.scalar_solve(ref, flux, eq, field, SOLVER)
    v = F.FvView(pv.n_cells, *pv.arrays())
    up, lo, dg, src, fld = OS.scalar_system(v, pv.delta_coeffs, pv.unit_normals, pv.face_areas, eq, flux, field)
    ldu = RX.RefLdu(ref)
    ldu.set(dg, up, lo, src)
    x = np.array(fld)
    r = ldu.solve(x, SOLVER[0], SOLVER[1], SOLVER[2], SOLVER[3], with_cache=False)
    ldu.close()
    assert r["iterations"] == r_ref["iterations"] and r["iterations"] > 0
    assert r["initial_residual"] == r_ref["initial_residual"] and r["final_residual"] == r_ref["final_residual"]
    assert np.array_equal(x, x_ref)
