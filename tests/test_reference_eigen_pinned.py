"""The reference's own Eigen-dependent sources, compiled unchanged against the Eigen stand-in
(oracle/eigen_standin, oracle/ref_eigen_shim.cpp), against the oracle's restatements and the
product's host code, on the CPU.

What each comparison pins:
* mesh pipeline (mesh_builder.cpp:51-233, mesh.cpp:100-212, box_mesher.cpp:30-143) and
  FvGeometry (fv_geometry.cpp:17-69): face ordering, owner / neighbour and face nodes are
  integer results of the reference's own code (bit-exact); geometry, delta coefficients and
  weights are bitwise equal as far as the stand-in's Vec3 arithmetic follows Eigen's;
* build_csr_pattern (ldu_matrix.cpp:572-612): integer, bit-exact;
* amg_aggregate (amg.cpp:12-78) on level 0: integer, bit-exact, independent of the stand-in;
  AmgPreconditioner::setup (amg.cpp:122-190): P, R, Galerkin operators and coarse-level
  aggregates bitwise equal as far as the stand-in follows Eigen's published sparse-product
  order; the coarse inverse (amg.cpp:227-240) is the stand-in's natural-order LDL^T (Eigen
  orders with AMD first), so it pins the oracle only to that factorisation;
* LduMatrix::multiply / residual_norms / set_reference (ldu_matrix.cpp:39-109): bit-exact
  (plain loops, no Eigen arithmetic);
* the CPU AmgCg (pcg with the Gauss-Seidel V-cycle, amg.cpp:192-285): the oracle's restatement
  takes the same iterations and reaches the same residual (dot products follow Eigen's
  reduction order in the stand-in and a plain loop in the oracle).
"""
import numpy as np
import pytest

import oracle as O
from cfd_b200 import workloads as W

RX = pytest.importorskip("oracle.reference")
if not RX.available():
    pytest.skip("reference build with the Eigen stand-in not available", allow_module_level=True)


def _pressure(case):
    up, lo, dg, dv = O.ref_assemble(case.n, case.owner, case.neighbour, case.flux, case.gamma,
                                    case.delta, 0.0)
    src = case.source0 - dv
    diag = dg.copy()
    O.set_reference(diag, src, case.ref_cell, case.ref_value)
    return up, lo, diag, src


MESHES = {
    "cavity8": (lambda: RX.cavity(8), lambda: W.cavity(8)),
    "cavity32": (lambda: RX.cavity(32), lambda: W.cavity(32)),
    "graded12": (lambda: RX.graded(12), lambda: W.graded(12)),
    "tet7": (lambda: RX.tet(7), lambda: W.tet(7)),
    "tet7_sigma": (lambda: RX.tet(7, sigma=1.5, seed=5), lambda: W.tet(7, sigma=1.5, seed=5)),
}


@pytest.mark.parametrize("name", list(MESHES))
def test_generated_workload_equals_the_reference_mesh_pipeline(name):
    """The product's generator (cfdb_mesh_box / cfdb_mesh_tet, cfdb_synth_pressure_inputs) and
    the reference's MeshBuilder / make_box_mesh + FvGeometry give the same system."""
    make_ref, make_prod = MESHES[name]
    r, p = make_ref(), make_prod()
    m = p.mesh
    assert (r.n, r.n_faces) == (p.n, p.n_faces)
    for f in ("owner", "neighbour", "delta", "gamma", "flux", "source0"):
        assert np.array_equal(getattr(r, f), getattr(p, f)), f
    rm = r.mesh
    assert np.array_equal(rm.owner, m.owner) and np.array_equal(rm.neighbour, m.neighbour)
    assert np.array_equal(rm.face_offsets, m.face_offsets) and np.array_equal(rm.face_nodes, m.face_nodes)
    for f in ("face_centres", "face_areas", "cell_centres", "cell_volumes"):
        assert np.array_equal(getattr(rm, f), getattr(m, f)), f


def test_box_mesher_equals_builder_on_lattice():
    """make_box_mesh (uniform and one-sided graded) equals MeshBuilder fed with the lattice
    cells and tags this project generates: the vectorised lattice follows box_mesher.cpp."""
    for grading in ((1.0, 1.0, 1.0), (3.0, 0.5, 1.7)):
        a = RX.RefMesh.box(5, 4, 3, grading)
        b = RX.RefMesh.build(_box_points(5, 4, 3, grading), RX.hex_cells(5, 4, 3), *RX.box_tag_quads(5, 4, 3))
        for f in ("owner", "neighbour", "face_offsets", "face_nodes"):
            assert np.array_equal(getattr(a, f), getattr(b, f)), f
        for f in ("face_centres", "face_areas", "cell_centres", "cell_volumes"):
            assert np.allclose(getattr(a, f), getattr(b, f), rtol=0, atol=1e-15), f


def _box_points(nx, ny, nz, grading):
    out = []
    for n, g in zip((nx, ny, nz), grading):
        r = g ** (1.0 / (n - 1)) if n > 1 else 1.0
        out.append([i / n if abs(r - 1.0) < 1e-12 else (r ** i - 1.0) / (r ** n - 1.0) for i in range(n + 1)])
    return RX.lattice_points(*out)


@pytest.mark.parametrize("name", ["cavity8", "graded12", "tet7"])
def test_pattern_equals_reference(cb, name):
    r = MESHES[name][0]()
    o = O.build_pattern(r.n, r.owner, r.neighbour)
    p = cb.build_csr_pattern(r.n, r.owner, r.neighbour)
    ldu = RX.RefLdu(r.mesh)
    for got in (r.pattern, ldu.pattern()):
        for f in ("row_ptr", "col", "diag_pos", "upper_pos", "lower_pos"):
            assert np.array_equal(getattr(got, f), getattr(o, f)), f
            assert np.array_equal(getattr(got, f), getattr(p, f)), f


@pytest.mark.parametrize("theta", [0.08, 0.04, 0.0])
@pytest.mark.parametrize("name", ["cavity8", "graded12", "tet7", "tet7_sigma"])
def test_amg_setup_equals_reference(cb, name, theta):
    r = MESHES[name][0]()
    up, lo, diag, _ = _pressure(r)
    a = O.ldu_to_csr(r.pattern, diag, up, lo)
    ref = RX.RefAmg(a, theta=theta)
    orc = O.Hierarchy(a, theta=theta)
    prod = cb.AmgHierarchy(cb.CsrView(a.n_rows, a.rp, a.ci, a.va), cb.AmgSettings(strength_threshold=theta))
    assert ref.levels == orc.levels == prod.levels()
    # level-0 aggregation is integer work on the assembled matrix: bit-exact without any Eigen
    agg0, n0 = RX.aggregate(a, RX.last_diagonal(a), theta)
    assert np.array_equal(agg0, orc.aggregates[0]) if ref.levels > 1 else True
    for l in range(ref.levels):
        for x, y in zip((ref.a[l].rp, ref.a[l].ci, ref.a[l].va), (orc.a[l].rp, orc.a[l].ci, orc.a[l].va)):
            assert np.array_equal(x, y), f"A[{l}]"
        if l + 1 < ref.levels:
            agg, n_agg = ref.aggregates(l, theta)
            assert np.array_equal(agg, orc.aggregates[l]) and n_agg == orc.a[l + 1].n_rows
            pa, pn = prod.aggregates(l)
            assert np.array_equal(pa, agg) and pn == n_agg
            for nm, x, y in (("P", ref.p[l], orc.p[l]), ("R", ref.r[l], orc.r[l])):
                for u, v in zip((x.rp, x.ci, x.va), (y.rp, y.ci, y.va)):
                    assert np.array_equal(u, v), f"{nm}[{l}]"
    assert np.array_equal(ref.coarse_inverse, np.asarray(orc.coarse_inverse).reshape(ref.coarse_inverse.shape))
    assert ref.operator_complexity == orc.operator_complexity


def test_amg_setup_equals_reference_at_cavity32():
    """The lid-driven cavity configuration (32^3, 32,768 cells) at the reference default
    strength threshold 0.08 and at 0.04."""
    r = RX.cavity(32)
    up, lo, diag, _ = _pressure(r)
    a = O.ldu_to_csr(r.pattern, diag, up, lo)
    for theta in (0.08, 0.04):
        ref, orc = RX.RefAmg(a, theta=theta), O.Hierarchy(a, theta=theta)
        assert ref.levels == orc.levels
        for l in range(ref.levels - 1):
            agg, _ = ref.aggregates(l, theta)
            assert np.array_equal(agg, orc.aggregates[l])
            assert np.array_equal(ref.p[l].va, orc.p[l].va) and np.array_equal(ref.a[l + 1].va, orc.a[l + 1].va)


@pytest.mark.parametrize("name", ["cavity8", "tet7"])
def test_ldu_matrix_operations_equal_reference(name):
    r = MESHES[name][0]()
    up, lo, dg, dv = O.ref_assemble(r.n, r.owner, r.neighbour, r.flux, r.gamma, r.delta, 0.0)
    src = r.source0 - dv
    ldu = RX.RefLdu(r.mesh)
    ldu.set(dg, up, lo, src)
    ldu.set_reference(3, 0.25)
    d_ref, s_ref = ldu.get()
    d, s = dg.copy(), src.copy()
    O.set_reference(d, s, 3, 0.25)
    assert np.array_equal(d_ref, d) and np.array_equal(s_ref, s)
    x = np.random.default_rng(4).standard_normal(r.n)
    assert np.array_equal(ldu.multiply(x), O.ldu_multiply(r.owner, r.neighbour, d, up, lo, x))
    assert ldu.residual_norms(x) == O.ldu_residual_norms(r.owner, r.neighbour, d, up, lo, s, x)


@pytest.mark.parametrize("name", ["cavity8", "graded12", "tet7"])
def test_cpu_amg_cg_equals_reference(name):
    """The CPU AmgCg (pcg + Gauss-Seidel V-cycle + LDL^T coarse solve) of the oracle against the
    reference's pcg on the reference's hierarchy: same iterations, solutions to round-off."""
    r = MESHES[name][0]()
    up, lo, diag, src = _pressure(r)
    a = O.ldu_to_csr(r.pattern, diag, up, lo)
    ref, orc = RX.RefAmg(a, theta=0.08), O.Hierarchy(a, theta=0.08)
    tol = 1e-10 * np.linalg.norm(src)
    x_ref, st = ref.pcg(a, src, tol=tol, max_iterations=200)
    x_orc, it, res = orc.pcg_gs(src, tol=tol, max_iterations=200)
    assert st["iterations"] == it
    assert np.linalg.norm(x_ref - x_orc) <= 1e-9 * np.linalg.norm(x_ref)
    z_ref = ref.apply(src)
    assert np.linalg.norm(src - a.matvec(x_ref)) <= tol * 1.0000001
    assert np.isfinite(z_ref).all()


@pytest.mark.parametrize("name", ["cavity8", "tet7"])
def test_persistent_gpu_cg_path_of_the_reference_runs(name):
    """LduMatrix::solve with GpuCg through solve_persistent (ldu_matrix.cpp:287-366) on the
    reference's host DeviceSolver, with the AmgCache rebuild every max_age CG solves: the
    rebuild sequence and the residual target the GPU path reproduces."""
    r = MESHES[name][0]()
    up, lo, diag, src = _pressure(r)
    ldu = RX.RefLdu(r.mesh)
    ldu.set(diag, up, lo, src)
    ages = []
    for _ in range(5):
        x = np.zeros(r.n)
        res = ldu.solve(x, "GpuCg", tolerance=0.0, rel_tolerance=1e-8, max_iterations=500, max_age=2)
        ages.append(res["amg_age"])
        assert res["initial_residual"] == 1.0 and res["final_residual"] < 1e-7
        a = O.ldu_to_csr(r.pattern, diag, up, lo)
        assert np.linalg.norm(src - a.matvec(x)) <= 1.05e-8 * np.linalg.norm(src)
    assert ages == [1, 2, 1, 2, 1]


@pytest.mark.parametrize("name", ["cavity8", "graded8", "tet5"])
def test_golden_hierarchies_equal_the_reference_setup(name):
    """The committed golden hierarchies (made by the oracle's setup) equal the reference's own
    AmgPreconditioner::setup on the golden matrix."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", f"{name}.npz"))
    n = int(g["n"])
    pat = O.Pattern(n, len(g["neighbour"]), g["pat_rp"], g["pat_col"], g["pat_diag"], g["pat_upper"],
                    g["pat_lower"])
    a = O.ldu_to_csr(pat, g["ldu_diag"], g["ldu_upper"], g["ldu_lower"])
    ref = RX.RefAmg(a)
    assert ref.levels == int(g["h_levels"])
    for l in range(ref.levels):
        for nm, m in (("a", ref.a[l]), ("p", ref.p[l] if l + 1 < ref.levels else None),
                      ("r", ref.r[l] if l + 1 < ref.levels else None)):
            if m is None:
                continue
            for f, v in (("rp", m.rp), ("ci", m.ci), ("va", m.va)):
                assert np.array_equal(v, g[f"h_{nm}{l}_{f}"]), f"{nm}{l}_{f}"
        if l + 1 < ref.levels:
            assert np.array_equal(ref.aggregates(l, 0.08)[0], g[f"h_agg{l}"])
    assert np.array_equal(ref.coarse_inverse.ravel(), np.asarray(g["h_coarse_inverse"]).ravel())
