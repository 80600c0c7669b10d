"""Python front end of the reference's Eigen-dependent host sources -- TEST INFRASTRUCTURE ONLY.

``oracle/_ref/libcfdref.so`` holds the reference's unchanged mesh pipeline (``mesh.cpp``,
``mesh_builder.cpp``, ``box_mesher.cpp``), ``fv_geometry.cpp``, ``ldu_matrix.cpp``, ``amg.cpp``
and ``flow_solver.cpp``, compiled against the Eigen stand-in in ``oracle/eigen_standin`` (see
``oracle/ref_eigen_shim.cpp`` and ``oracle/ref_flow_shim.cpp``). Integer results (face ordering, CSR pattern, aggregates) are the
reference's own; floating-point results follow Eigen as far as the stand-in does.

The lattice helpers (cells and boundary tags of box meshes, the 6-tet split, the jittered nodes)
and ``pressure_inputs`` restate this project's synthetic workload definitions (the same
definitions ``oracle/meshref.py`` restates for small meshes), vectorised with numpy so that the
benchmark configurations can be built at full size without the product library.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import Csr, Pattern, ref

_i, _d, _u64 = C.c_int, C.c_double, C.c_uint64
_pi, _pd = C.POINTER(C.c_int), C.POINTER(C.c_double)
_vp = C.c_void_p

_declared = False


def lib():
    """The reference build with the Eigen-dependent sources, or None if it was never built."""
    global _declared
    R = ref()
    if R is None or not hasattr(R, "refx_mesh_build"):
        return None
    if not _declared:
        R.refx_box_mesh.argtypes = [_i, _i, _i, _d, _d, _d]
        R.refx_box_mesh.restype = _vp
        R.refx_mesh_build.argtypes = [_i, _pd, _i, _i, _pi, _i, _pi, _pi, _i]
        R.refx_mesh_build.restype = _vp
        R.refx_mesh_destroy.argtypes = [_vp]
        R.refx_mesh_sizes.argtypes = [_vp, _pi, _pi, _pi, _pi, _pi]
        R.refx_mesh_topology.argtypes = [_vp, _pi, _pi, _pi, _pi]
        R.refx_mesh_geometry.argtypes = [_vp, _pd, _pd, _pd, _pd]
        R.refx_fv_geometry.argtypes = [_vp, _pd, _pd, _pi, _pi, _pi, _pi, _pi]
        R.refx_fv_geometry.restype = _i
        R.refx_amg_setup.argtypes = [_i, _pi, _pi, _pd, _d, _i, _i]
        R.refx_amg_setup.restype = _vp
        R.refx_amg_destroy.argtypes = [_vp]
        R.refx_amg_levels.argtypes = [_vp]
        R.refx_amg_levels.restype = _i
        R.refx_amg_operator_complexity.argtypes = [_vp]
        R.refx_amg_operator_complexity.restype = _d
        R.refx_amg_level.argtypes = [_vp, _i, _i, _pi, _pi, _pi, C.POINTER(_pi), C.POINTER(_pi),
                                     C.POINTER(_pd)]
        R.refx_amg_level.restype = _i
        R.refx_amg_coarse_inverse.argtypes = [_vp, _pd]
        R.refx_amg_coarse_inverse.restype = _i
        R.refx_amg_apply.argtypes = [_vp, _i, _pd, _pd]
        R.refx_amg_apply.restype = _i
        R.refx_amg_aggregate.argtypes = [_i, _pi, _pi, _pd, _pd, _d, _pi]
        R.refx_amg_aggregate.restype = _i
        R.refx_pcg.argtypes = [_vp, _i, _pi, _pi, _pd, _pd, _pd, _d, _i, _pi, _pd]
        R.refx_pcg.restype = _i
        R.refx_ldu_create.argtypes = [_vp]
        R.refx_ldu_create.restype = _vp
        R.refx_ldu_destroy.argtypes = [_vp]
        R.refx_ldu_set.argtypes = [_vp, _pd, _pd, _pd, _pd]
        R.refx_ldu_get.argtypes = [_vp, _pd, _pd]
        R.refx_ldu_set_reference.argtypes = [_vp, _i, _d]
        R.refx_ldu_multiply.argtypes = [_vp, _pd, _pd]
        R.refx_ldu_residual_norms.argtypes = [_vp, _pd, _pd, _pd]
        R.refx_ldu_pattern.argtypes = [_vp, _pi, _pi, _pi, _pi, _pi]
        R.refx_ldu_solve.argtypes = [_vp, _i, _d, _d, _i, _i, _i, _i, _pd, _pd, _pd, _pi, _pi, _pi]
        R.refx_ldu_solve.restype = _i
        R.refx_jittered_lattice.argtypes = [_i, _i, _i, _pd, _pd, _pd, _d, _u64, _pd]
        R.refx_pressure_inputs.argtypes = [_i, _i, _pi, _pi, _pd, _pd, _pd, _d, _i, _i, _i, _u64, _pd,
                                           _pd, _pd]
        if hasattr(R, "refx_flow_create"):
            R.refx_flow_create.argtypes = [_vp, _i, _pi, _pd, _pd, _pd, _pi]
            R.refx_flow_create.restype = _vp
            R.refx_flow_destroy.argtypes = [_vp]
            for name, args in (("refx_flow_set_state", [_vp, _pd, _pd, _pd]),
                               ("refx_flow_get_state", [_vp, _pd, _pd, _pd]),
                               ("refx_flow_boundary", [_vp, _pi, _pd, _pd]),
                               ("refx_flow_momentum", [_vp, _d, _i]),
                               ("refx_flow_momentum_arrays", [_vp, _pd, _pd, _pd, _pd]),
                               ("refx_flow_solve_momentum", [_vp, _pd]),
                               ("refx_flow_pressure_correction", [_vp, _i, _pd, _pd, _pd]),
                               ("refx_flow_simple_iteration", [_vp, _pd]),
                               ("refx_scalar_solve", [_vp, _pd, _pd, _pd, _pd, _pi, _pd, _pd, C.c_void_p,
                                                      _pd, _pd, _pd, _pi, _pd, _pd, _pd])):
                getattr(R, name).argtypes = args
                getattr(R, name).restype = _i
        _declared = True
    return R


def available() -> bool:
    return lib() is not None


def _ip(a):
    return a.ctypes.data_as(_pi)


def _dp(a):
    return a.ctypes.data_as(_pd)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ---------------------------------------------------------------------------------------------
# lattice workloads (this project's definitions, vectorised)
# ---------------------------------------------------------------------------------------------

def lattice_ids(nx, ny, nz):
    """Node id i + (nx+1)(j + (ny+1)k) of every lattice node, shape (nz+1, ny+1, nx+1)."""
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    return (i + (nx + 1) * (j + (ny + 1) * k)).astype(np.int32)


def lattice_points(xs, ys, zs):
    """Nodes k outer, then j, then i (box_mesher.cpp:48-69), shape (n, 3)."""
    zz, yy, xx = np.meshgrid(np.asarray(zs, float), np.asarray(ys, float), np.asarray(xs, float),
                             indexing="ij")
    return np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)


def hex_cells(nx, ny, nz):
    """Hex cells k outer, i inner, nodes in the order of box_mesher.cpp:71-92."""
    P = lattice_ids(nx, ny, nz)
    s = np.s_
    c = [P[s[:-1, :-1, :-1]], P[s[:-1, :-1, 1:]], P[s[:-1, 1:, 1:]], P[s[:-1, 1:, :-1]],
         P[s[1:, :-1, :-1]], P[s[1:, :-1, 1:]], P[s[1:, 1:, 1:]], P[s[1:, 1:, :-1]]]
    return np.stack([a.ravel() for a in c], axis=1).astype(np.int32)


KUHN_PERMS = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]


def tet_cells(nx, ny, nz):
    """Six tets per box cell sharing the main diagonal, (v000, +e_a, +e_a+e_b, v111) over the
    axis permutations, nodes 1 and 2 swapped for odd permutations; box cells k outer."""
    P = lattice_ids(nx, ny, nz)
    base = P[:-1, :-1, :-1].ravel().astype(np.int64)
    step = [1, nx + 1, (nx + 1) * (ny + 1)]
    out = np.empty((base.size, 6, 4), np.int64)
    for q, perm in enumerate(KUHN_PERMS):
        v0 = base
        v1 = v0 + step[perm[0]]
        v2 = v1 + step[perm[1]]
        v3 = v2 + step[perm[2]]
        par = sum(1 for a in range(3) for b in range(a + 1, 3) if perm[a] > perm[b]) & 1
        if par:
            v1, v2 = v2, v1
        out[:, q, 0], out[:, q, 1], out[:, q, 2], out[:, q, 3] = v0, v1, v2, v3
    return out.reshape(-1, 4).astype(np.int32)


def box_tag_quads(nx, ny, nz):
    """Boundary quads and patches in the order of box_mesher.cpp:94-140 (patch = 2 * axis + side)."""
    P = lattice_ids(nx, ny, nz)  # [k, j, i]
    quads, patches = [], []
    for side, i in enumerate((0, nx)):
        a = P[:-1, :-1, i]
        b = P[:-1, 1:, i]
        c = P[1:, 1:, i]
        d = P[1:, :-1, i]
        quads.append(np.stack([a.ravel(), b.ravel(), c.ravel(), d.ravel()], 1))
        patches.append(np.full(a.size, side))
    for side, j in enumerate((0, ny)):
        a = P[:-1, j, :-1]
        b = P[:-1, j, 1:]
        c = P[1:, j, 1:]
        d = P[1:, j, :-1]
        quads.append(np.stack([a.ravel(), b.ravel(), c.ravel(), d.ravel()], 1))
        patches.append(np.full(a.size, 2 + side))
    for side, k in enumerate((0, nz)):
        a = P[k, :-1, :-1]
        b = P[k, :-1, 1:]
        c = P[k, 1:, 1:]
        d = P[k, 1:, :-1]
        quads.append(np.stack([a.ravel(), b.ravel(), c.ravel(), d.ravel()], 1))
        patches.append(np.full(a.size, 4 + side))
    return np.concatenate(quads).astype(np.int32), np.concatenate(patches).astype(np.int32)


def tet_tags(nx, ny, nz):
    """Every boundary quad split by its diagonal through corners a and c: (a, b, c), (a, c, d)."""
    q, p = box_tag_quads(nx, ny, nz)
    tri = np.empty((2 * len(q), 4), np.int32)
    tri[0::2, :3] = q[:, [0, 1, 2]]
    tri[1::2, :3] = q[:, [0, 2, 3]]
    tri[:, 3] = -1
    return tri, np.repeat(p, 2).astype(np.int32)


def jittered_lattice(nx, ny, nz, xs, ys, zs, jitter, seed):
    R = lib()
    pts = np.empty(((nx + 1) * (ny + 1) * (nz + 1), 3))
    R.refx_jittered_lattice(nx, ny, nz, _dp(_f64(xs)), _dp(_f64(ys)), _dp(_f64(zs)), float(jitter),
                            int(seed), _dp(pts))
    return pts


# ---------------------------------------------------------------------------------------------
# the reference's mesh pipeline
# ---------------------------------------------------------------------------------------------

class RefMesh:
    """cfd::mesh::Mesh built by the reference's own MeshBuilder / make_box_mesh."""

    def __init__(self, handle):
        if not handle:
            raise ValueError("reference mesh build failed")
        R = lib()
        self._h = handle
        nc, nf, ni, npt, nfn = _i(), _i(), _i(), _i(), _i()
        R.refx_mesh_sizes(handle, C.byref(nc), C.byref(nf), C.byref(ni), C.byref(npt), C.byref(nfn))
        self.n_cells, self.n_faces, self.n_internal_faces = nc.value, nf.value, ni.value
        self.owner = np.empty(self.n_faces, np.int32)
        self.neighbour = np.empty(self.n_internal_faces, np.int32)
        self.face_offsets = np.empty(self.n_faces + 1, np.int32)
        self.face_nodes = np.empty(nfn.value, np.int32)
        R.refx_mesh_topology(handle, _ip(self.owner), _ip(self.neighbour), _ip(self.face_offsets),
                             _ip(self.face_nodes))
        self.face_centres = np.empty((self.n_faces, 3))
        self.face_areas = np.empty((self.n_faces, 3))
        self.cell_centres = np.empty((self.n_cells, 3))
        self.cell_volumes = np.empty(self.n_cells)
        R.refx_mesh_geometry(handle, _dp(self.face_centres), _dp(self.face_areas),
                             _dp(self.cell_centres), _dp(self.cell_volumes))

    @classmethod
    def box(cls, nx, ny, nz, grading=(1.0, 1.0, 1.0)):
        """make_box_mesh on the unit cube (box_mesher.cpp:30-143)."""
        return cls(lib().refx_box_mesh(nx, ny, nz, *map(float, grading)))

    @classmethod
    def build(cls, points, cells, tag_nodes, tag_patch, n_patches=6):
        """MeshBuilder::build (mesh_builder.cpp:51-233) of one cell shape."""
        points, cells = _f64(points), _i32(cells)
        tag_nodes, tag_patch = _i32(tag_nodes), _i32(tag_patch)
        return cls(lib().refx_mesh_build(len(points), _dp(points), len(cells), cells.shape[1], _ip(cells),
                                         len(tag_nodes), _ip(tag_nodes), _ip(tag_patch), n_patches))

    @classmethod
    def hex_box(cls, xs, ys, zs):
        nx, ny, nz = len(xs) - 1, len(ys) - 1, len(zs) - 1
        q, p = box_tag_quads(nx, ny, nz)
        return cls.build(lattice_points(xs, ys, zs), hex_cells(nx, ny, nz), q, p)

    @classmethod
    def tet_box(cls, nx, ny, nz, points):
        t, p = tet_tags(nx, ny, nz)
        return cls.build(points, tet_cells(nx, ny, nz), t, p)

    def fv(self):
        """FvGeometry (fv_geometry.cpp:17-69): (delta[n_faces], weights[n_internal], Pattern)."""
        R = lib()
        n, nif = self.n_cells, self.n_internal_faces
        nnz = n + 2 * nif
        delta, weights = np.empty(self.n_faces), np.empty(nif)
        rp, col = np.empty(n + 1, np.int32), np.empty(nnz, np.int32)
        dpos, upos, lpos = np.empty(n, np.int32), np.empty(nif, np.int32), np.empty(nif, np.int32)
        rc = R.refx_fv_geometry(self._h, _dp(delta), _dp(weights), _ip(rp), _ip(col), _ip(dpos), _ip(upos),
                                _ip(lpos))
        if rc != 0:
            raise ValueError("FvGeometry failed")
        return delta, weights, Pattern(n, nif, rp, col, dpos, upos, lpos)

    def close(self):
        if self._h:
            lib().refx_mesh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pressure_inputs(mesh: RefMesh, weights, sigma, unit_rau, flux_kind, rhs_kind, seed):
    """(gamma, flux, source0) of the synthetic pressure configurations."""
    R = lib()
    n, nif = mesh.n_cells, mesh.n_internal_faces
    gamma, flux, src = np.empty(nif), np.empty(nif), np.empty(n)
    R.refx_pressure_inputs(n, nif, _ip(mesh.owner), _ip(mesh.neighbour), _dp(_f64(weights)),
                           _dp(mesh.cell_volumes), _dp(_f64(mesh.face_areas)), float(sigma), int(unit_rau),
                           int(flux_kind), int(rhs_kind), int(seed), _dp(gamma), _dp(flux), _dp(src))
    return gamma, flux, src


@dataclass
class RefCase:
    """A synthetic pressure configuration built through the reference's mesh pipeline."""
    name: str
    mesh: RefMesh
    n: int
    n_faces: int
    owner: np.ndarray
    neighbour: np.ndarray
    flux: np.ndarray
    gamma: np.ndarray
    delta: np.ndarray
    source0: np.ndarray
    pattern: Pattern
    ref_cell: int = 0
    ref_value: float = 0.0


def _case(name, mesh, sigma, unit_rau, rhs_kind, seed):
    delta, weights, pat = mesh.fv()
    gamma, flux, src = pressure_inputs(mesh, weights, sigma, unit_rau, 0, rhs_kind, seed)
    nif = mesh.n_internal_faces
    return RefCase(name, mesh, mesh.n_cells, nif, mesh.owner[:nif].copy(), mesh.neighbour.copy(), flux,
                   gamma, delta[:nif].copy(), src, pat)


SEED_BASE = 20261203


def cavity(n=32, seed=SEED_BASE + 0):
    """Uniform n^3 box from make_box_mesh, rAU = 1, seeded face flux, zero source."""
    return _case(f"cavity{n}", RefMesh.box(n, n, n), 0.0, True, 0, seed)


def two_sided_positions(n, ratio):
    """Nodes in [0, 1], cells growing by `ratio` from both walls to the centre."""
    sizes = np.array([ratio ** min(i, n - 1 - i) for i in range(n)])
    total = 0.0
    for s in sizes:
        total += s
    acc, pos = 0.0, [0.0]
    for s in sizes:
        acc += s
        pos.append(acc / total)
    pos[n] = 1.0
    return np.array(pos)


def graded(n=128, ratio=1.05, sigma=0.5, seed=SEED_BASE + 1):
    xs = two_sided_positions(n, ratio)
    return _case(f"graded{n}", RefMesh.hex_box(xs, xs, xs), sigma, False, 1, seed)


def tet(n=95, jitter=0.2, sigma=1.0, seed=SEED_BASE + 2):
    xs = np.linspace(0.0, 1.0, n + 1)
    pts = jittered_lattice(n, n, n, xs, xs, xs, jitter, seed)
    return _case(f"tet{n}", RefMesh.tet_box(n, n, n, pts), sigma, False, 1, seed + 1000)


# ---------------------------------------------------------------------------------------------
# AMG (amg.cpp)
# ---------------------------------------------------------------------------------------------

class RefAmg:
    """AmgPreconditioner::setup (amg.cpp:122-190) of the reference, arrays copied out."""

    def __init__(self, a: Csr, theta=0.08, max_levels=25, coarse_size=400):
        R = lib()
        self._h = R.refx_amg_setup(a.n_rows, _ip(a.rp), _ip(a.ci), _dp(a.va), float(theta), int(max_levels),
                                   int(coarse_size))
        if not self._h:
            raise ValueError("reference AMG setup failed")
        self.levels = R.refx_amg_levels(self._h)
        self.operator_complexity = R.refx_amg_operator_complexity(self._h)
        self.a, self.p, self.r = [], [], []
        for l in range(self.levels):
            for which, dst in ((0, self.a), (1, self.p), (2, self.r)):
                if which > 0 and l + 1 >= self.levels:
                    continue
                rows, cols, nnz = _i(), _i(), _i()
                rp, ci, va = _pi(), _pi(), _pd()
                assert R.refx_amg_level(self._h, l, which, C.byref(rows), C.byref(cols), C.byref(nnz),
                                        C.byref(rp), C.byref(ci), C.byref(va)) == 0
                dst.append(Csr(rows.value, cols.value,
                               np.ctypeslib.as_array(rp, (rows.value + 1,)).copy(),
                               np.ctypeslib.as_array(ci, (max(nnz.value, 1),))[:nnz.value].copy(),
                               np.ctypeslib.as_array(va, (max(nnz.value, 1),))[:nnz.value].copy()))
        nc = self.a[-1].n_rows
        self.coarse_inverse = np.empty((nc, nc))
        assert R.refx_amg_coarse_inverse(self._h, _dp(self.coarse_inverse)) == 0

    def aggregates(self, level, theta):
        """amg_aggregate of a level's operator with its last diagonal entries (amg.cpp:82-92)."""
        a = self.a[level]
        return aggregate(a, last_diagonal(a), theta)

    def apply(self, r):
        """One Gauss-Seidel V-cycle (amg.cpp:192-225)."""
        r = _f64(r)
        z = np.empty_like(r)
        assert lib().refx_amg_apply(self._h, len(r), _dp(r), _dp(z)) == 0
        return z

    def pcg(self, a: Csr, b, x=None, tol=1e-10, max_iterations=500):
        """cfd::fv::pcg (amg.cpp:253-285), the CPU AmgCg."""
        b = _f64(b)
        x = np.zeros_like(b) if x is None else _f64(x).copy()
        it, res = _i(), _d()
        assert lib().refx_pcg(self._h, a.n_rows, _ip(a.rp), _ip(a.ci), _dp(a.va), _dp(b), _dp(x), float(tol),
                              int(max_iterations), C.byref(it), C.byref(res)) == 0
        return x, {"iterations": it.value, "residual": res.value}

    def close(self):
        if self._h:
            lib().refx_amg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def last_diagonal(a: Csr):
    """The last stored diagonal entry of every row (zero if none)."""
    d = np.zeros(a.n_rows)
    rows = np.repeat(np.arange(a.n_rows), np.diff(a.rp))
    on = a.ci == rows
    d[rows[on]] = a.va[on]  # later entries overwrite earlier ones
    return d


def aggregate(a: Csr, diag, theta=0.08):
    """cfd::fv::amg_aggregate (amg.cpp:12-78): (aggregate per row, number of aggregates)."""
    agg = np.empty(a.n_rows, np.int32)
    n = lib().refx_amg_aggregate(a.n_rows, _ip(a.rp), _ip(a.ci), _dp(a.va), _dp(_f64(diag)), float(theta),
                                 _ip(agg))
    if n < 0:
        raise ValueError("amg_aggregate failed")
    return agg, n


# ---------------------------------------------------------------------------------------------
# LduMatrix (ldu_matrix.cpp)
# ---------------------------------------------------------------------------------------------

LINEAR_SOLVER = {"ConjugateGradient": 0, "BiCgStab": 1, "AmgCg": 2, "GpuCg": 3, "GpuBiCgStab": 4}


class RefLdu:
    """cfd::fv::LduMatrix on a reference mesh with its CSR pattern and a persistent AmgCache."""

    def __init__(self, mesh: RefMesh):
        R = lib()
        self.mesh = mesh
        self._h = R.refx_ldu_create(mesh._h)
        if not self._h:
            raise ValueError("LduMatrix creation failed")

    def set(self, diag, upper, lower, source):
        lib().refx_ldu_set(self._h, _dp(_f64(diag)), _dp(_f64(upper)), _dp(_f64(lower)), _dp(_f64(source)))

    def get(self):
        d, s = np.empty(self.mesh.n_cells), np.empty(self.mesh.n_cells)
        lib().refx_ldu_get(self._h, _dp(d), _dp(s))
        return d, s

    def set_reference(self, cell, value):
        lib().refx_ldu_set_reference(self._h, int(cell), float(value))

    def multiply(self, x):
        y = np.empty(self.mesh.n_cells)
        lib().refx_ldu_multiply(self._h, _dp(_f64(x)), _dp(y))
        return y

    def residual_norms(self, x):
        r, n = _d(), _d()
        lib().refx_ldu_residual_norms(self._h, _dp(_f64(x)), C.byref(r), C.byref(n))
        return r.value, n.value

    def pattern(self):
        n, nif = self.mesh.n_cells, self.mesh.n_internal_faces
        rp, col = np.empty(n + 1, np.int32), np.empty(n + 2 * nif, np.int32)
        d, u, lo = np.empty(n, np.int32), np.empty(nif, np.int32), np.empty(nif, np.int32)
        lib().refx_ldu_pattern(self._h, _ip(rp), _ip(col), _ip(d), _ip(u), _ip(lo))
        return Pattern(n, nif, rp, col, d, u, lo)

    def solve(self, x, solver="GpuCg", tolerance=1e-10, rel_tolerance=0.01, max_iterations=1000,
              max_age=20, with_pattern=True, with_cache=True):
        """LduMatrix::solve (ldu_matrix.cpp:111-282) in place on x, with the handle's AmgCache
        or (with_cache False) none; returns the result record."""
        x_ = _f64(x)
        if x_ is not x:
            raise ValueError("x must be a contiguous float64 array (solved in place)")
        ini, fin = _d(), _d()
        it, age, lv = _i(), _i(), _i()
        rc = lib().refx_ldu_solve(self._h, LINEAR_SOLVER[solver], float(tolerance), float(rel_tolerance),
                                  int(max_iterations), int(max_age), 1 if with_pattern else 0,
                                  1 if with_cache else 0, _dp(x),
                                  C.byref(ini), C.byref(fin), C.byref(it), C.byref(age), C.byref(lv))
        if rc != 0:
            raise ValueError("LduMatrix::solve failed")
        return {"initial_residual": ini.value, "final_residual": fin.value, "iterations": it.value,
                "amg_age": age.value, "amg_levels": lv.value}

    def close(self):
        if self._h:
            lib().refx_ldu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# FlowBoundary, LinearSolverType, ConvectionScheme and GradientScheme as the reference numbers
# them (flow_solver.hpp:15, ldu_matrix.hpp:21, flow_solver.hpp:40, fv_geometry.hpp:32)
FLOW_BOUNDARY = {"VelocityInlet": 0, "Wall": 1, "PressureOutlet": 2, "Symmetry": 3, "Empty": 4}
CONVECTION = {"Upwind": 0, "LinearUpwind": 1, "LimitedLinearUpwind": 2, "Lust": 3, "LimitedLust": 4}
GRADIENT = {"Gauss": 0, "LeastSquares": 1, "GaussCorrected": 2}


class RefFlow:
    """cfd::fv::FlowSolver on a reference mesh (one condition per patch, in the mesh's patch
    order), driven one SIMPLE step at a time (oracle/ref_flow_shim.cpp)."""

    def __init__(self, mesh: RefMesh, patches, nu=1e-3, alpha_u=0.7, alpha_p=0.3, n_non_orth=0,
                 p_solver=("GpuCg", 1e-10, 0.01, 500), u_solver=("GpuBiCgStab", 1e-10, 0.1, 1000),
                 convection="LinearUpwind", gradient="Gauss"):
        """patches: one (kind, velocity (3), pressure) per patch, kind a FLOW_BOUNDARY name."""
        R = lib()
        if R is None or not hasattr(R, "refx_flow_create"):
            raise RuntimeError("the reference build has no FlowSolver")
        self.mesh = mesh
        kinds = _i32([FLOW_BOUNDARY[k] for k, _, _ in patches])
        vel = _f64([v for _, v, _ in patches]).reshape(-1, 3)
        pre = _f64([p for _, _, p in patches])
        real = _f64([nu, alpha_u, alpha_p, p_solver[1], p_solver[2], u_solver[1], u_solver[2]])
        ints = _i32([n_non_orth, LINEAR_SOLVER[p_solver[0]], p_solver[3], LINEAR_SOLVER[u_solver[0]],
                     u_solver[3], CONVECTION[convection], GRADIENT[gradient]])
        self._h = R.refx_flow_create(mesh._h, len(patches), _ip(kinds), _dp(vel), _dp(pre), _dp(real), _ip(ints))
        if not self._h:
            raise ValueError("FlowSolver construction failed")

    def _call(self, name, *args):
        if getattr(lib(), name)(self._h, *args) != 0:
            raise ValueError(f"{name} failed")

    def set_state(self, u, p, phi=None):
        u, p = _f64(u), _f64(p)
        self._call("refx_flow_set_state", _dp(u), _dp(p), None if phi is None else _dp(_f64(phi)))

    def state(self):
        m = self.mesh
        u, p, phi = np.empty((m.n_cells, 3)), np.empty(m.n_cells), np.empty(m.n_faces)
        self._call("refx_flow_get_state", _dp(u), _dp(p), _dp(phi))
        return u, p, phi

    def boundary(self):
        """Per boundary face: (FlowBoundary kind, outlet pressure, fixed velocity)."""
        nb = self.mesh.n_faces - self.mesh.n_internal_faces
        k, p, v = np.empty(nb, np.int32), np.empty(nb), np.empty((nb, 3))
        self._call("refx_flow_boundary", _ip(k), _dp(p), _dp(v))
        return k, p, v

    def momentum(self, dt=0.0, relax=True):
        """assemble_momentum into the solver's momentum system; returns (diag (n, 3), upper,
        lower, source (n, 3))."""
        self._call("refx_flow_momentum", float(dt), 1 if relax else 0)
        m = self.mesh
        d, s = np.empty((m.n_cells, 3)), np.empty((m.n_cells, 3))
        up, lo = np.empty(m.n_internal_faces), np.empty(m.n_internal_faces)
        self._call("refx_flow_momentum_arrays", _dp(d), _dp(up), _dp(lo), _dp(s))
        return d, up, lo, s

    def solve_momentum(self):
        r = np.empty(3)
        self._call("refx_flow_solve_momentum", _dp(r))
        return r

    def simple_iteration(self):
        """FlowSolver::simple_iteration; returns (u residuals (3), p residual, continuity)."""
        r = np.empty(5)
        self._call("refx_flow_simple_iteration", _dp(r))
        return r[:3].copy(), float(r[3]), float(r[4])

    def pressure_correction(self, relax_p=True, u_prev=None, phi_prev=None):
        """FlowSolver::pressure_correction on the momentum system; returns the initial residual."""
        ini = _d()
        self._call("refx_flow_pressure_correction", 1 if relax_p else 0,
                   None if u_prev is None else _dp(_f64(u_prev)),
                   None if phi_prev is None else _dp(_f64(phi_prev)), C.byref(ini))
        return ini.value

    def close(self):
        if self._h:
            lib().refx_flow_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def scalar_solve(mesh: RefMesh, face_flux, eq: dict, field, solver=("GpuBiCgStab", 1e-12, 1e-9, 1000)):
    """The reference's solve_scalar (scalar_transport.cpp:49-183) on `mesh` with its own
    FvGeometry; eq as oracle.scalar.scalar_system takes it. Returns (field after the solve,
    {initial_residual, final_residual, iterations})."""
    R = lib()
    fx = eq.get("fixed_cell")
    fixed = None if fx is None else np.ascontiguousarray(fx, np.uint8)
    opt = lambda k: None if eq.get(k) is None else _dp(_f64(eq[k]))  # noqa: E731
    keep = [_f64(face_flux), _f64(eq["gamma_face"]), _f64(eq["su"]), _f64(eq["sp"]), _i32(eq["bc_kind"]),
            _f64(eq["bc_value"]), _f64(eq["bc_coefficient"])]
    flags = _i32([LINEAR_SOLVER[solver[0]], solver[3], 1 if eq.get("linear_upwind", True) else 0,
                  int(eq.get("gradient", 0))])
    real = _f64([eq.get("relaxation", 1.0), eq.get("dt", 0.0), solver[1], solver[2]])
    x = np.array(field, np.float64)
    res = np.empty(3)
    rc = R.refx_scalar_solve(mesh._h, _dp(keep[0]), _dp(keep[1]), _dp(keep[2]), _dp(keep[3]), _ip(keep[4]),
                             _dp(keep[5]), _dp(keep[6]), None if fixed is None else fixed.ctypes.data,
                             opt("fixed_value") if fixed is not None else None, opt("old_value"), opt("capacity"),
                             _ip(flags), _dp(real), _dp(x), _dp(res))
    if rc != 0:
        raise ValueError("solve_scalar failed")
    return x, {"initial_residual": float(res[0]), "final_residual": float(res[1]), "iterations": int(res[2])}
