"""CPU restatement of the reference's finite-volume cell kernels (TEST INFRASTRUCTURE ONLY).

Restates src/gpu/src/fv_cell.inc (cell_gradient :24-74, cell_gradient_corrected :76-121,
cell_limiter :123-163, cell_scalar_corrections :165-196, cell_momentum_corrections :198-259)
and the call sequence of src/gpu/src/fv_openmp.cpp (gradient :158-163, vector_gradient
:165-173, scalar_corrections :175-202, momentum_corrections :204-248, gradient_loop
:250-297). Every cell gathers over its faces in ascending face order; here the cells advance
together one face slot at a time (slot j = the j-th face of every cell that has one), so each
cell sees the same operations in the same order as the reference's per-cell loop, and numpy's
element-wise float64 arithmetic rounds each of them the same way (no FMA). The results are
therefore bit-identical to the reference's host build (pinned by tests/test_fv_oracle.py
against oracle/_ref, the reference's own fv_openmp.cpp compiled here).

Vectors are (n, 3) arrays; the vector gradient is (n_cells, 9) with g[c, 3 i + j] = du_i/dx_j.
"""
from __future__ import annotations

import numpy as np


class FvView:
    """An FvMeshView (fv_device.hpp:15-31) as numpy arrays."""

    def __init__(self, n_cells, owner, neighbour, cell_offsets, cell_faces, weight, sf,
                 face_centre, cell_centre, volume, correction, lsq_d, lsq_inverse):
        self.nc = int(n_cells)
        self.own = np.ascontiguousarray(owner, np.int32)
        self.nei = np.ascontiguousarray(neighbour, np.int32)
        self.nif = len(self.nei)
        self.nf = len(self.own)
        self.start = np.ascontiguousarray(cell_offsets, np.int32)
        self.faces = np.ascontiguousarray(cell_faces, np.int32)
        self.w = np.ascontiguousarray(weight, np.float64)
        self.sf = np.ascontiguousarray(sf, np.float64).reshape(-1, 3)
        self.cf = np.ascontiguousarray(face_centre, np.float64).reshape(-1, 3)
        self.cc = np.ascontiguousarray(cell_centre, np.float64).reshape(-1, 3)
        self.vol = np.ascontiguousarray(volume, np.float64)
        self.kv = np.ascontiguousarray(correction, np.float64).reshape(-1, 3)
        self.lsq_d = np.ascontiguousarray(lsq_d, np.float64).reshape(-1, 3)
        self.lsq = np.ascontiguousarray(lsq_inverse, np.float64).reshape(-1, 9)
        deg = np.diff(self.start)
        self.slots = []  # per slot j: (cells with a j-th face, that face)
        for j in range(int(deg.max()) if len(deg) else 0):
            cells = np.nonzero(deg > j)[0]
            self.slots.append((cells, self.faces[self.start[cells] + j]))


def view_of(mesh) -> FvView:
    """The FvMeshView that FvGeometry::device() builds (fv_geometry.cpp:209-260) for a mesh with
    owner, neighbour, face_areas, face_centres, cell_centres, cell_volumes and interpolation
    weights (a meshref.Mesh, or any object with those attributes): corrections
    S - d |S|^2 / max(S.d, 0.05 |S||d|) (fv_geometry.cpp:33-50), d / |d|^2 and the inverse of
    sum d d^T / |d|^2 accumulated face by face (fv_geometry.cpp:71-92), cell -> face lists in
    ascending face order. These arrays are inputs: every implementation under test receives
    the same ones."""
    own = np.asarray(mesh.owner, np.int64)
    nei = np.asarray(mesh.neighbour, np.int64)
    nc, nf, nif = int(mesh.n_cells), len(own), len(nei)
    sf = np.asarray(mesh.face_areas, np.float64).reshape(-1, 3)
    cf = np.asarray(mesh.face_centres, np.float64).reshape(-1, 3)
    cc = np.asarray(mesh.cell_centres, np.float64).reshape(-1, 3)
    w = mesh.weights if hasattr(mesh, "weights") else mesh.fv_geometry()[1]
    kv = np.zeros((nf, 3))
    lsq_d = np.zeros((nf, 3))
    mat = np.zeros((nc, 3, 3))
    lists = [[] for _ in range(nc)]
    for f in range(nf):
        p = own[f]
        d = (cc[nei[f]] if f < nif else cf[f]) - cc[p]
        s = sf[f]
        area = np.sqrt(s @ s)
        s_dot_d = max(s @ d, 0.05 * area * np.sqrt(d @ d))
        kv[f] = s - d * (area * area / s_dot_d)
        lsq_d[f] = d / (d @ d)
        dd = np.outer(d, d) / (d @ d)
        mat[p] += dd
        lists[p].append(f)
        if f < nif:
            mat[nei[f]] += dd
            lists[nei[f]].append(f)
    start = np.zeros(nc + 1, np.int32)
    start[1:] = np.cumsum([len(x) for x in lists])
    faces = np.array([f for x in lists for f in sorted(x)], np.int32)
    inv = np.linalg.inv(mat)
    return FvView(nc, own, nei, start, faces, w, sf, cf, cc, mesh.cell_volumes, kv, lsq_d,
                  inv.transpose(0, 2, 1).reshape(-1, 9))


def _gradient_component(v: FvView, phi, bv, lsq: bool):
    """cell_gradient (fv_cell.inc:24-74) for one component: phi (n_cells), bv (n_boundary)."""
    g = np.zeros((v.nc, 3))
    for cells, f in v.slots:
        internal = f < v.nif
        fi, ci = f[internal], cells[internal]
        fb, cb = f[~internal], cells[~internal]
        if lsq:
            dv = phi[v.nei[fi]] - phi[v.own[fi]]
            g[ci] = g[ci] + v.lsq_d[fi] * dv[:, None]
            dvb = bv[fb - v.nif] - phi[cb]
            g[cb] = g[cb] + v.lsq_d[fb] * dvb[:, None]
        else:
            wf = v.w[fi]
            pf = wf * phi[v.own[fi]] + (1.0 - wf) * phi[v.nei[fi]]
            t = v.sf[fi] * pf[:, None]
            mine = (v.own[fi] == ci)[:, None]
            g[ci] = np.where(mine, g[ci] + t, g[ci] - t)
            g[cb] = g[cb] + v.sf[fb] * bv[fb - v.nif][:, None]
    if lsq:
        a = v.lsq
        return np.stack([a[:, 0] * g[:, 0] + a[:, 3] * g[:, 1] + a[:, 6] * g[:, 2],
                         a[:, 1] * g[:, 0] + a[:, 4] * g[:, 1] + a[:, 7] * g[:, 2],
                         a[:, 2] * g[:, 0] + a[:, 5] * g[:, 1] + a[:, 8] * g[:, 2]], axis=1)
    return g / v.vol[:, None]


def _corrected_component(v: FvView, phi, bv, gl):
    """cell_gradient_corrected (fv_cell.inc:76-121) with the least-squares gradient gl."""
    g = np.zeros((v.nc, 3))
    for cells, f in v.slots:
        internal = f < v.nif
        fi, ci = f[internal], cells[internal]
        fb, cb = f[~internal], cells[~internal]
        p, n = v.own[fi], v.nei[fi]
        wf = v.w[fi]
        pf = wf * phi[p] + (1.0 - wf) * phi[n]
        dot = None
        for j in range(3):
            xip = wf * v.cc[p, j] + (1.0 - wf) * v.cc[n, j]
            gf = wf * gl[p, j] + (1.0 - wf) * gl[n, j]
            dot = gf * (v.cf[fi, j] - xip) if j == 0 else dot + gf * (v.cf[fi, j] - xip)
        pf = pf + dot
        t = v.sf[fi] * pf[:, None]
        mine = (p == ci)[:, None]
        g[ci] = np.where(mine, g[ci] + t, g[ci] - t)
        g[cb] = g[cb] + v.sf[fb] * bv[fb - v.nif][:, None]
    return g / v.vol[:, None]


def _scheme_component(v: FvView, phi, bv, scheme: int):
    """gradient_loop (fv_openmp.cpp:250-297) for one component."""
    if scheme == 2:
        return _corrected_component(v, phi, bv, _gradient_component(v, phi, bv, True))
    return _gradient_component(v, phi, bv, scheme == 1)


def gradient(v: FvView, phi, bv, scheme: int):
    """DeviceFv::gradient: (n_cells, 3)."""
    return _scheme_component(v, np.asarray(phi, np.float64), np.asarray(bv, np.float64), scheme)


def vector_gradient(v: FvView, u, ub, scheme: int):
    """DeviceFv::vector_gradient: (n_cells, 9), g[c, 3 i + j] = du_i / dx_j."""
    u = np.asarray(u, np.float64).reshape(-1, 3)
    ub = np.asarray(ub, np.float64).reshape(-1, 3)
    return np.concatenate([_scheme_component(v, u[:, i].copy(), ub[:, i].copy(), scheme)
                           for i in range(3)], axis=1)


def limiter(v: FvView, u, ub, g, venkat: bool, eps2=(0.0, 0.0, 0.0)):
    """cell_limiter (fv_cell.inc:123-163): (n_cells, 3)."""
    u = np.asarray(u, np.float64).reshape(-1, 3)
    ub = np.asarray(ub, np.float64).reshape(-1, 3)
    lo, hi = u.copy(), u.copy()
    for cells, f in v.slots:
        internal = f < v.nif
        fi, ci = f[internal], cells[internal]
        val = np.empty((len(f), 3))
        val[internal] = u[np.where(v.own[fi] == ci, v.nei[fi], v.own[fi])]
        val[~internal] = ub[f[~internal] - v.nif]
        lo[cells] = np.where(val < lo[cells], val, lo[cells])
        hi[cells] = np.where(val > hi[cells], val, hi[cells])
    lim = np.ones((v.nc, 3))
    for cells, f in v.slots:
        r = v.cf[f] - v.cc[cells]
        gc = g[cells]
        for i in range(3):
            d = gc[:, 3 * i] * r[:, 0] + gc[:, 3 * i + 1] * r[:, 1] + gc[:, 3 * i + 2] * r[:, 2]
            skip = (d < 1e-300) & (d > -1e-300)
            uc = u[cells, i]
            bound = np.where(d > 0.0, hi[cells, i] - uc, lo[cells, i] - uc)
            with np.errstate(divide="ignore", invalid="ignore"):
                if venkat:
                    e = eps2[i]
                    q = (bound * bound + e + 2.0 * d * bound) / (bound * bound + 2.0 * d * d + d * bound + e)
                else:
                    ratio = bound / d
                    q = np.where(ratio > 0.0, ratio, 0.0)
            cur = lim[cells, i]
            lim[cells, i] = np.where(skip, cur, np.where(q < cur, q, cur))
    return lim


def _internal_slots(v: FvView):
    """Slots of the per-cell loops that stop at the cell's first boundary face
    (fv_cell.inc:172-174)."""
    alive = np.ones(v.nc, bool)
    for cells, f in v.slots:
        alive[cells] &= f < v.nif
        keep = alive[cells]
        yield cells[keep], f[keep]


def scalar_corrections(v: FvView, phi, bv, scheme: int, flux, gamma, linear_upwind: bool, source):
    """DeviceFv::scalar_corrections: returns the updated source (n_cells)."""
    g = gradient(v, phi, bv, scheme)
    flux = np.asarray(flux, np.float64)
    gamma = np.asarray(gamma, np.float64)
    s = np.zeros(v.nc)
    for cells, f in _internal_slots(v):
        p, n = v.own[f], v.nei[f]
        fl = flux[f]
        e = np.zeros(len(f))
        if linear_upwind:
            up = np.where(fl >= 0.0, p, n)
            r = v.cf[f] - v.cc[up]
            e = e - fl * (g[up, 0] * r[:, 0] + g[up, 1] * r[:, 1] + g[up, 2] * r[:, 2])
        wf = v.w[f]
        gf = wf[:, None] * g[p] + (1.0 - wf)[:, None] * g[n]
        e = e + gamma[f] * (v.kv[f, 0] * gf[:, 0] + v.kv[f, 1] * gf[:, 1] + v.kv[f, 2] * gf[:, 2])
        s[cells] = np.where(p == cells, s[cells] + e, s[cells] - e)
    return np.asarray(source, np.float64) + s


def momentum_corrections(v: FvView, u, ub, g, flux, nu_face, linear_upwind: bool, limited: bool,
                         venkat: bool, eps2, central: float, transpose_term: bool, source):
    """DeviceFv::momentum_corrections with the field u, its boundary values ub and its vector
    gradient g of the last vector_gradient call: returns the updated source (n_cells, 3)."""
    u = np.asarray(u, np.float64).reshape(-1, 3)
    flux = np.asarray(flux, np.float64)
    nu_face = np.asarray(nu_face, np.float64)
    use_lim = limited and linear_upwind
    e2 = tuple(eps2) if venkat else (0.0, 0.0, 0.0)
    lim = limiter(v, u, ub, g, venkat, e2) if use_lim else None
    s = np.zeros((v.nc, 3))
    for cells, f in _internal_slots(v):
        p, n = v.own[f], v.nei[f]
        fl = flux[f]
        wf = v.w[f]
        e = np.zeros((len(f), 3))
        if linear_upwind:
            up = np.where(fl >= 0.0, p, n)
            r = v.cf[f] - v.cc[up]
            gu = g[up]
            for i in range(3):
                d = gu[:, 3 * i] * r[:, 0] + gu[:, 3 * i + 1] * r[:, 1] + gu[:, 3 * i + 2] * r[:, 2]
                if central > 0.0:
                    uf = wf * u[p, i] + (1.0 - wf) * u[n, i]
                    d = (1.0 - central) * d + central * (uf - u[up, i])
                if use_lim:
                    d = lim[up, i] * d
                e[:, i] = e[:, i] - fl * d
        gf = wf[:, None] * g[p] + (1.0 - wf)[:, None] * g[n]
        nu = nu_face[f]
        k = v.kv[f]
        for i in range(3):
            e[:, i] = e[:, i] + nu * (gf[:, 3 * i] * k[:, 0] + gf[:, 3 * i + 1] * k[:, 1] + gf[:, 3 * i + 2] * k[:, 2])
        if transpose_term:
            a = v.sf[f]
            for i in range(3):
                e[:, i] = e[:, i] + nu * (gf[:, i] * a[:, 0] + gf[:, i + 3] * a[:, 1] + gf[:, i + 6] * a[:, 2])
        mine = (p == cells)[:, None]
        s[cells] = np.where(mine, s[cells] + e, s[cells] - e)
    return np.asarray(source, np.float64).reshape(-1, 3) + s


# -------------------------------------------------------------------------------------------
# The reference's own DeviceFv host path (oracle/_ref: fv_openmp.cpp + fv_device.cpp)
# -------------------------------------------------------------------------------------------

def _ref_lib():
    import ctypes as C

    from . import ref
    R = ref()
    if R is None:
        return None
    if not getattr(R, "_fv_declared", False):
        i, d, vp = C.c_int, C.c_double, C.c_void_p
        pi, pd = C.POINTER(C.c_int), C.POINTER(C.c_double)
        R.ref_fv_create.argtypes = [i, i, i, pi, pi, pi, pi, pd, pd, pd, pd, pd, pd, pd, pd]
        R.ref_fv_create.restype = vp
        R.ref_fv_destroy.argtypes = [vp]
        R.ref_fv_destroy.restype = None
        R.ref_fv_gradient.argtypes = [vp, pd, pd, i, pd]
        R.ref_fv_vector_gradient.argtypes = [vp, pd, pd, i, pd]
        R.ref_fv_scalar_corrections.argtypes = [vp, pd, pd, i, pd, pd, i, pd]
        R.ref_fv_momentum_corrections.argtypes = [vp, pd, pd, i, i, i, pd, d, i, pd]
        for f in (R.ref_fv_gradient, R.ref_fv_vector_gradient, R.ref_fv_scalar_corrections,
                  R.ref_fv_momentum_corrections):
            f.restype = i
        R._fv_declared = True
    return R


class RefFv:
    """cfd::gpu::DeviceFv of the reference, running its per-cell kernels on host threads."""

    def __init__(self, v: FvView):
        import ctypes as C
        self._C = C
        self.R = _ref_lib()
        if self.R is None:
            raise RuntimeError("the reference's host path was not built (oracle/_ref)")
        self.v = v
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))  # noqa: E731
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        self._keep = [v.own, v.nei, v.start, v.faces, v.w, v.sf, v.cf, v.cc, v.vol, v.kv, v.lsq_d, v.lsq]
        self.h = self.R.ref_fv_create(v.nc, v.nif, v.nf, ip(v.own), ip(v.nei), ip(v.start), ip(v.faces),
                                      dp(v.w), dp(v.sf), dp(v.cf), dp(v.cc), dp(v.vol), dp(v.kv),
                                      dp(v.lsq_d), dp(v.lsq))
        if not self.h:
            raise ValueError("ref_fv_create failed")

    def _dp(self, a):
        return a.ctypes.data_as(self._C.POINTER(self._C.c_double))

    def gradient(self, phi, bv, scheme):
        phi, bv = np.ascontiguousarray(phi, np.float64), np.ascontiguousarray(bv, np.float64)
        g = np.empty((self.v.nc, 3))
        assert self.R.ref_fv_gradient(self.h, self._dp(phi), self._dp(bv), int(scheme), self._dp(g)) == 0
        return g

    def vector_gradient(self, u, ub, scheme):
        u, ub = np.ascontiguousarray(u, np.float64), np.ascontiguousarray(ub, np.float64)
        g = np.empty((self.v.nc, 9))
        assert self.R.ref_fv_vector_gradient(self.h, self._dp(u), self._dp(ub), int(scheme), self._dp(g)) == 0
        return g

    def scalar_corrections(self, phi, bv, scheme, flux, gamma, linear_upwind, source):
        phi, bv = np.ascontiguousarray(phi, np.float64), np.ascontiguousarray(bv, np.float64)
        flux, gamma = np.ascontiguousarray(flux, np.float64), np.ascontiguousarray(gamma, np.float64)
        s = np.array(source, np.float64)
        assert self.R.ref_fv_scalar_corrections(self.h, self._dp(phi), self._dp(bv), int(scheme),
                                                self._dp(flux), self._dp(gamma), int(bool(linear_upwind)),
                                                self._dp(s)) == 0
        return s

    def momentum_corrections(self, flux, nu_face, linear_upwind, limited, venkat, eps2, central,
                             transpose_term, source):
        flux, nu = np.ascontiguousarray(flux, np.float64), np.ascontiguousarray(nu_face, np.float64)
        e = np.ascontiguousarray(eps2 if eps2 is not None else np.zeros(3), np.float64)
        s = np.array(source, np.float64).reshape(-1, 3).copy()
        rc = self.R.ref_fv_momentum_corrections(self.h, self._dp(flux), self._dp(nu), int(bool(linear_upwind)),
                                                int(bool(limited)), int(bool(venkat)), self._dp(e),
                                                float(central), int(bool(transpose_term)), self._dp(s))
        if rc != 0:
            raise RuntimeError("ref_fv_momentum_corrections failed")
        return s

    def close(self):
        if getattr(self, "h", None):
            self.R.ref_fv_destroy(self.h)
            self.h = None

    __del__ = close


def random_view(n_cells: int, n_internal: int, n_boundary: int, seed: int = 0) -> FvView:
    """A consistent FvMeshView with random addressing and data (no geometry behind it): cells
    with anything from no faces to many, to exercise ragged face counts. Internal faces are
    ordered by (owner, neighbour) with owner < neighbour, boundary faces follow."""
    rng = np.random.default_rng(seed)
    pairs = set()
    inner = max(2, (4 * n_cells) // 5)  # the last fifth of the cells get no internal faces
    while len(pairs) < n_internal:
        a, b = rng.integers(0, inner, 2)
        if a != b:
            pairs.add((min(a, b), max(a, b)))
    pairs = sorted(pairs)
    own = np.array([p[0] for p in pairs] + list(rng.integers(0, n_cells, n_boundary)), np.int32)
    nei = np.array([p[1] for p in pairs], np.int32)
    nf = len(own)
    lists = [[] for _ in range(n_cells)]
    for f in range(nf):
        lists[own[f]].append(f)
        if f < n_internal:
            lists[nei[f]].append(f)
    start = np.zeros(n_cells + 1, np.int32)
    start[1:] = np.cumsum([len(x) for x in lists])
    faces = np.array([f for x in lists for f in sorted(x)], np.int32)
    return FvView(n_cells, own, nei, start, faces, rng.uniform(0.05, 0.95, n_internal),
                  rng.standard_normal((nf, 3)), rng.standard_normal((nf, 3)), rng.standard_normal((n_cells, 3)),
                  rng.uniform(0.5, 2.0, n_cells), rng.standard_normal((nf, 3)), rng.standard_normal((nf, 3)),
                  rng.standard_normal((n_cells, 9)))
