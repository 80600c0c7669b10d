"""cfd::gpu::DeviceFv (fv_device.hpp:33-72) on the B200: cell gradients and explicit face
corrections with the mesh resident in HBM.

:func:`mesh_view` builds the FvMeshView the reference's FvGeometry::device() hands to the
DeviceFv constructor (fv_geometry.cpp:209-260): cell -> face lists in ascending face order, the
non-orthogonal correction vectors of every face (fv_geometry.cpp:33-50), d / |d|^2 and the
inverse least-squares matrices (fv_geometry.cpp:71-92). :class:`DeviceFv` takes that view and
runs the four calls on the device; the host-array methods keep the reference's semantics
(momentum_corrections reuses the field and gradient of the last vector_gradient call), the
``*_device`` methods take CUDA tensors and copy nothing.
"""
from __future__ import annotations

import ctypes as C
import enum

import numpy as np

from . import (InvalidArgument, _check, _devptr, _dp, _f64, _i32, _ip, _lib, _proto, _stream_ordered)

_i, _d, _vp, _sz = C.c_int, C.c_double, C.c_void_p, C.c_size_t
_pi, _pd = C.POINTER(C.c_int), C.POINTER(C.c_double)


class GradientScheme(enum.IntEnum):
    """fv_geometry.hpp:31."""
    Gauss = 0
    LeastSquares = 1
    GaussCorrected = 2


class FvMeshViewStruct(C.Structure):
    _fields_ = [("n_cells", _i), ("n_internal_faces", _i), ("n_faces", _i), ("owner", _pi),
                ("neighbour", _pi), ("cell_offsets", _pi), ("cell_faces", _pi), ("weight", _pd),
                ("sf", _pd), ("face_centre", _pd), ("cell_centre", _pd), ("volume", _pd),
                ("correction", _pd), ("lsq_d", _pd), ("lsq_inverse", _pd)]


_proto("cfdb_device_fv_create", [C.POINTER(FvMeshViewStruct), C.POINTER(_vp)])
_proto("cfdb_device_fv_destroy", [_vp])
_proto("cfdb_device_fv_on_device", [_vp])
_proto("cfdb_device_fv_device_bytes", [_vp, C.POINTER(_sz)])
_proto("cfdb_device_fv_stream", [_vp, C.POINTER(_vp)])
_proto("cfdb_device_fv_gradient", [_vp, _pd, _pd, _i, _pd])
_proto("cfdb_device_fv_vector_gradient", [_vp, _pd, _pd, _i, _pd])
_proto("cfdb_device_fv_scalar_corrections", [_vp, _pd, _pd, _i, _pd, _pd, _i, _pd])
_proto("cfdb_device_fv_momentum_corrections", [_vp, _pd, _pd, _i, _i, _i, _pd, _d, _i, _pd])
_proto("cfdb_device_fv_gradient_device", [_vp, _vp, _vp, _i, _vp])
_proto("cfdb_device_fv_vector_gradient_device", [_vp, _vp, _vp, _i, _vp])
_proto("cfdb_device_fv_scalar_corrections_device", [_vp, _vp, _vp, _i, _vp, _vp, _i, _vp])
_proto("cfdb_device_fv_momentum_corrections_device",
       [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _pd, _d, _i, _vp])
_proto("cfdb_device_fv_set_face_geometry", [_vp, _pd, _pd, _pd])


class MeshView:
    """Host arrays of an FvMeshView (fv_device.hpp:15-31); vectors are (n, 3), the inverse
    least-squares matrices (n_cells, 9) column-major."""

    def __init__(self, n_cells, owner, neighbour, cell_offsets, cell_faces, weight, sf,
                 face_centre, cell_centre, volume, correction, lsq_d, lsq_inverse):
        self.n_cells = int(n_cells)
        self.owner, self.neighbour = _i32(owner), _i32(neighbour)
        self.n_faces, self.n_internal_faces = len(self.owner), len(self.neighbour)
        self.cell_offsets, self.cell_faces = _i32(cell_offsets), _i32(cell_faces)
        self.weight = _f64(weight)
        self.sf = _f64(sf).reshape(-1, 3)
        self.face_centre = _f64(face_centre).reshape(-1, 3)
        self.cell_centre = _f64(cell_centre).reshape(-1, 3)
        self.volume = _f64(volume)
        self.correction = _f64(correction).reshape(-1, 3)
        self.lsq_d = _f64(lsq_d).reshape(-1, 3)
        self.lsq_inverse = _f64(lsq_inverse).reshape(-1, 9)

    @property
    def n_boundary_faces(self) -> int:
        return self.n_faces - self.n_internal_faces

    def arrays(self):
        """The 13 arrays in FvMeshView order (after n_cells)."""
        return (self.owner, self.neighbour, self.cell_offsets, self.cell_faces, self.weight, self.sf,
                self.face_centre, self.cell_centre, self.volume, self.correction, self.lsq_d,
                self.lsq_inverse)

    def check(self) -> None:
        """Array lengths against the sizes (the C entry point then checks the contents)."""
        nc, nf, nif = self.n_cells, self.n_faces, self.n_internal_faces
        want = {"cell_offsets": (self.cell_offsets, nc + 1), "weight": (self.weight, nif),
                "sf": (self.sf, nf), "face_centre": (self.face_centre, nf),
                "cell_centre": (self.cell_centre, nc), "volume": (self.volume, nc),
                "correction": (self.correction, nf), "lsq_d": (self.lsq_d, nf),
                "lsq_inverse": (self.lsq_inverse, nc)}
        for name, (a, n) in want.items():
            if len(a) != n:
                raise InvalidArgument(f"FvMeshView.{name}: {len(a)} entries, expected {n}")
        if len(self.cell_offsets) and len(self.cell_faces) != int(self.cell_offsets[-1]):
            raise InvalidArgument("FvMeshView.cell_faces: length differs from cell_offsets[n_cells]")

    def _c(self):
        return FvMeshViewStruct(self.n_cells, self.n_internal_faces, self.n_faces, _ip(self.owner),
                                _ip(self.neighbour), _ip(self.cell_offsets), _ip(self.cell_faces),
                                _dp(self.weight), _dp(self.sf), _dp(self.face_centre),
                                _dp(self.cell_centre), _dp(self.volume), _dp(self.correction),
                                _dp(self.lsq_d), _dp(self.lsq_inverse))


def cell_face_lists(n_cells, owner, neighbour):
    """Faces of each cell in ascending face order (CSR): the Mesh::cell_faces the view needs."""
    own, nei = _i32(owner), _i32(neighbour)
    cells = np.concatenate([own, nei])
    faces = np.concatenate([np.arange(len(own), dtype=np.int32), np.arange(len(nei), dtype=np.int32)])
    order = np.lexsort((faces, cells))
    offsets = np.zeros(int(n_cells) + 1, np.int64)
    np.cumsum(np.bincount(cells, minlength=int(n_cells)), out=offsets[1:])
    return offsets.astype(np.int32), faces[order].astype(np.int32)


def _face_sums(n_cells, own, nei, per_face):
    """Per cell, the sum of per_face[f] over its faces in ascending face order, as the face loop
    of FvGeometry::build_least_squares (fv_geometry.cpp:78-87) adds them (each face to its
    owner, then to its neighbour): the k-th contribution of every cell is added in round k."""
    nf, nif = len(own), len(nei)
    cell_of = np.concatenate([np.stack([own[:nif], nei], axis=1).ravel(), own[nif:]]).astype(np.int64)
    face_of = np.concatenate([np.repeat(np.arange(nif), 2), np.arange(nif, nf)])
    order = np.argsort(cell_of, kind="stable")  # by cell; each cell's faces stay in face order
    c_sorted = cell_of[order]
    rank = np.arange(len(order)) - np.searchsorted(c_sorted, np.arange(n_cells))[c_sorted]
    out = np.zeros((n_cells,) + per_face.shape[1:])
    for k in range(int(rank.max()) + 1 if len(rank) else 0):
        e = order[rank == k]
        out[cell_of[e]] += per_face[face_of[e]]
    return out


def _inverse3(m):
    """Inverses of 3x3 matrices by cofactors, in the operation order of Eigen's fixed-size 3x3
    inverse that FvGeometry calls (Matrix3d::inverse): the cofactors of column 0 give the
    determinant (c00 m00 + c10 m10) + c20 m20, and entry (i, j) is cofactor (j, i) times 1 / det."""
    def cof(i, j):
        i1, i2, j1, j2 = (i + 1) % 3, (i + 2) % 3, (j + 1) % 3, (j + 2) % 3
        return m[:, i1, j1] * m[:, i2, j2] - m[:, i1, j2] * m[:, i2, j1]
    det = (cof(0, 0) * m[:, 0, 0] + cof(1, 0) * m[:, 1, 0]) + cof(2, 0) * m[:, 2, 0]
    invdet = 1.0 / det
    out = np.empty_like(m)
    for i in range(3):
        for j in range(3):
            out[:, i, j] = cof(j, i) * invdet
    return out


def mesh_view(n_cells, owner, neighbour, face_areas, face_centres, cell_centres, cell_volumes,
              weights) -> MeshView:
    """The FvMeshView of FvGeometry::device() (fv_geometry.cpp:209-260) from a mesh's
    addressing and geometry: d = C_N - C_P (boundary: C_f - C_P), delta = |S|^2 / max(S.d,
    0.05 |S||d|), correction = S - d delta, lsq_d = d / |d|^2, lsq_inverse = (sum d d^T /
    |d|^2)^-1 over each cell's faces (column-major), each in the reference's operation order
    (FvGeometry::build_least_squares, fv_geometry.cpp:70-92)."""
    own, nei = _i32(owner), _i32(neighbour)
    nf, nif = len(own), len(nei)
    sf = _f64(face_areas).reshape(-1, 3)
    cf = _f64(face_centres).reshape(-1, 3)
    cc = _f64(cell_centres).reshape(-1, 3)
    if len(sf) != nf or len(cf) != nf or len(cc) != int(n_cells):
        raise InvalidArgument("mesh_view: array sizes do not match the addressing")
    to = np.concatenate([cc[nei], cf[nif:]])
    d = to - cc[own]
    area = np.sqrt((sf * sf).sum(axis=1))
    s_dot_d = np.maximum((sf * d).sum(axis=1), 0.05 * area * np.sqrt((d * d).sum(axis=1)))
    if np.any(area <= 0.0) or np.any(s_dot_d <= 0.0):
        raise InvalidArgument("mesh_view: zero-area face or degenerate cell-to-face distance")
    delta = area * area / s_dot_d
    correction = sf - d * delta[:, None]
    s2 = (d * d).sum(axis=1)  # |d|^2, x + y first, then z
    q = d / s2[:, None]
    dd = (d[:, :, None] * d[:, None, :]) / s2[:, None, None]  # d d^T / |d|^2 (fv_geometry.cpp:82)
    mat = _face_sums(int(n_cells), own, nei, dd)
    inv = _inverse3(mat)
    offsets, faces = cell_face_lists(n_cells, own, nei)
    view = MeshView(n_cells, own, nei, offsets, faces, weights, sf, cf, cc, cell_volumes, correction,
                    q, inv.transpose(0, 2, 1).reshape(-1, 9))
    # FvGeometry's other face factors (fv_geometry.cpp:36-50), for the scalar equation
    view.delta_coeffs = delta
    view.face_areas = area
    view.unit_normals = sf / area[:, None]
    return view


def mesh_view_of(mesh) -> MeshView:
    """mesh_view of a :class:`cfd_b200.Mesh`."""
    return mesh_view(mesh.n_cells, mesh.owner, mesh.neighbour, mesh.face_areas, mesh.face_centres,
                     mesh.cell_centres, mesh.cell_volumes, mesh.weights)


def _host_in(a, n, name, prefix=False):
    """float64 host array of n values (prefix: at least n, the first n are used, like the
    reference's per-face inputs that may cover all faces)."""
    a = _f64(a).ravel()
    if len(a) < n or (len(a) != n and not prefix):
        raise InvalidArgument(f"{name}: expected {n} values, got {len(a)}")
    return a


class DeviceFv:
    """cfd::gpu::DeviceFv: the mesh of a :class:`MeshView` resident on the current device."""

    def __init__(self, view: MeshView):
        self.view = view
        self.n_cells, self.n_faces = view.n_cells, view.n_faces
        self.n_internal_faces, self.n_boundary_faces = view.n_internal_faces, view.n_boundary_faces
        view.check()
        h = _vp()
        s = view._c()
        _check(_lib.cfdb_device_fv_create(C.byref(s), C.byref(h)))
        self._h = h

    def on_device(self) -> bool:
        return bool(_lib.cfdb_device_fv_on_device(self._h))

    def device_bytes(self) -> int:
        b = _sz()
        _check(_lib.cfdb_device_fv_device_bytes(self._h, C.byref(b)))
        return int(b.value)

    def stream(self) -> int:
        s = _vp()
        _check(_lib.cfdb_device_fv_stream(self._h, C.byref(s)))
        return int(s.value or 0)

    # -- host arrays (the reference's signatures) --------------------------------------------
    def gradient(self, phi, bv, scheme) -> np.ndarray:
        """(n_cells, 3) gradient of phi with boundary face values bv."""
        p = _host_in(phi, self.n_cells, "phi")
        b = _host_in(bv, self.n_boundary_faces, "bv")
        g = np.empty((self.n_cells, 3))
        _check(_lib.cfdb_device_fv_gradient(self._h, _dp(p), _dp(b), int(scheme), _dp(g)))
        return g

    def vector_gradient(self, u, ub, scheme) -> np.ndarray:
        """(n_cells, 9) gradient of u, g[c, 3 i + j] = du_i / dx_j; u, ub and the gradient stay
        on the device for :meth:`momentum_corrections`."""
        uu = _host_in(u, 3 * self.n_cells, "u")
        b = _host_in(ub, 3 * self.n_boundary_faces, "ub")
        g = np.empty((self.n_cells, 9))
        _check(_lib.cfdb_device_fv_vector_gradient(self._h, _dp(uu), _dp(b), int(scheme), _dp(g)))
        return g

    def scalar_corrections(self, phi, bv, scheme, flux, gamma, linear_upwind, source) -> None:
        """Accumulates the explicit internal-face fluxes into source (float64, in place)."""
        p = _host_in(phi, self.n_cells, "phi")
        b = _host_in(bv, self.n_boundary_faces, "bv")
        fl = _host_in(flux, self.n_internal_faces, "flux", prefix=True)
        ga = _host_in(gamma, self.n_internal_faces, "gamma", prefix=True)
        src = self._inplace(source, self.n_cells)
        _check(_lib.cfdb_device_fv_scalar_corrections(self._h, _dp(p), _dp(b), int(scheme), _dp(fl),
                                                      _dp(ga), 1 if linear_upwind else 0, _dp(src)))

    def momentum_corrections(self, flux, nu_face, linear_upwind, limited, venkat, eps2, central,
                             transpose_term, source) -> None:
        """Accumulates the explicit momentum fluxes into source (n_cells x 3 float64, in place)."""
        fl = _host_in(flux, self.n_internal_faces, "flux", prefix=True)
        nu = _host_in(nu_face, self.n_internal_faces, "nu_face", prefix=True)
        e = _f64(eps2 if eps2 is not None else np.zeros(3))
        src = self._inplace(source, 3 * self.n_cells)
        _check(_lib.cfdb_device_fv_momentum_corrections(
            self._h, _dp(fl), _dp(nu), 1 if linear_upwind else 0, 1 if limited else 0,
            1 if venkat else 0, _dp(e), float(central), 1 if transpose_term else 0, _dp(src)))

    @staticmethod
    def _inplace(a, n):
        if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous and a.size == n):
            raise InvalidArgument(f"source must be a C-contiguous float64 numpy array of {n} values")
        return a

    # -- device arrays (CUDA tensors, no copies) ----------------------------------------------
    @_stream_ordered
    def gradient_device(self, phi, bv, scheme, grad) -> None:
        _check(_lib.cfdb_device_fv_gradient_device(self._h, _devptr(phi), _devptr(bv) if bv is not None else None,
                                                   int(scheme), _devptr(grad)))

    @_stream_ordered
    def vector_gradient_device(self, u, ub, scheme, grad) -> None:
        _check(_lib.cfdb_device_fv_vector_gradient_device(
            self._h, _devptr(u), _devptr(ub) if ub is not None else None, int(scheme), _devptr(grad)))

    @_stream_ordered
    def scalar_corrections_device(self, phi, bv, scheme, flux, gamma, linear_upwind, source) -> None:
        _check(_lib.cfdb_device_fv_scalar_corrections_device(
            self._h, _devptr(phi), _devptr(bv) if bv is not None else None, int(scheme), _devptr(flux),
            _devptr(gamma), 1 if linear_upwind else 0, _devptr(source)))

    @_stream_ordered
    def momentum_corrections_device(self, u, ub, grad, flux, nu_face, linear_upwind, limited, venkat,
                                    eps2, central, transpose_term, source) -> None:
        e = _f64(eps2 if eps2 is not None else np.zeros(3))
        _check(_lib.cfdb_device_fv_momentum_corrections_device(
            self._h, _devptr(u), _devptr(ub) if ub is not None else None, _devptr(grad), _devptr(flux),
            _devptr(nu_face), 1 if linear_upwind else 0, 1 if limited else 0, 1 if venkat else 0, _dp(e),
            float(central), 1 if transpose_term else 0, _devptr(source)))

    def set_face_geometry(self, delta_coeffs=None, unit_normals=None, face_areas=None) -> None:
        """FvGeometry's delta coefficients, unit normals and face areas (all faces) for the
        scalar equation; by default those :func:`mesh_view` computed."""
        dc = _host_in(self.view.delta_coeffs if delta_coeffs is None else delta_coeffs, self.n_faces, "delta_coeffs")
        un = _host_in(self.view.unit_normals if unit_normals is None else unit_normals, 3 * self.n_faces,
                      "unit_normals")
        ar = _host_in(self.view.face_areas if face_areas is None else face_areas, self.n_faces, "face_areas")
        _check(_lib.cfdb_device_fv_set_face_geometry(self._h, _dp(dc), _dp(un), _dp(ar)))

    def close(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:  # the library may be gone at interpreter exit
            _lib.cfdb_device_fv_destroy(h)
            self._h = None

    __del__ = close
