"""CPU oracle for the pressure-correction hot path -- TEST INFRASTRUCTURE ONLY.

Python (ctypes + numpy) front end of ``oracle/oracle.c`` (a serial C restatement of the
reference algorithms) and of ``oracle/_ref`` (the reference's own host sources compiled
unchanged). Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference legs may import this package, and only as the checker or the timed CPU baseline.
The product package ``cfd_b200`` never imports it.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import numpy as np

from . import build as _build

_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        path = _build.build_oracle()
        _lib = C.CDLL(path)
        _declare(_lib)
    return _lib


def ref():
    """The reference's compiled host path, or None when it was never built here."""
    global _ref
    if _ref is None:
        path = _build.build_ref()
        if path is None or not os.path.exists(path):
            return None
        _ref = C.CDLL(path)
        _declare_ref(_ref)
    return _ref


_i = C.c_int
_d = C.c_double
_pi = C.POINTER(C.c_int)
_pd = C.POINTER(C.c_double)


class CsrView(C.Structure):
    _fields_ = [("n", _i), ("rp", _pi), ("ci", _pi), ("va", _pd)]


class RefCsr(C.Structure):
    _fields_ = [("n", _i), ("nnz", _i), ("rp", _pi), ("ci", _pi), ("va", _pd)]


class Stats(C.Structure):
    _fields_ = [("iterations", _i), ("residual", _d), ("converged", _i)]


def _declare(L):
    L.orc_build_pattern.argtypes = [_i, _i, _pi, _pi, _pi, _pi, _pi, _pi, _pi]
    L.orc_build_pattern.restype = _i
    L.orc_assemble.argtypes = [_i, _i, _pi, _pi, _pd, _pd, _pd, _d, _pd, _pd, _pd, _pd]
    L.orc_assemble.restype = None
    L.orc_ldu_multiply.argtypes = [_i, _i, _pi, _pi, _pd, _pd, _pd, _pd, _pd]
    L.orc_ldu_residual_norms.argtypes = [_i, _i, _pi, _pi, _pd, _pd, _pd, _pd, _pd, _pd]
    L.orc_set_reference.argtypes = [_pd, _pd, _i, _d]
    L.orc_ldu_to_csr.argtypes = [_i, _i, _pi, _pi, _pi, _pd, _pd, _pd, _pd]
    L.orc_csr_spmv.argtypes = [_i, _pi, _pi, _pd, _pd, _pd]
    L.orc_aggregate.argtypes = [_i, _pi, _pi, _pd, _pd, _d, _pi]
    L.orc_aggregate.restype = _i
    L.orc_amg_setup.argtypes = [_i, _pi, _pi, _pd, _d, _i, _i]
    L.orc_amg_setup.restype = C.c_void_p
    L.orc_amg_free.argtypes = [C.c_void_p]
    L.orc_amg_levels.argtypes = [C.c_void_p]
    L.orc_amg_levels.restype = _i
    L.orc_amg_level_csr.argtypes = [C.c_void_p, _i, _i, _pi, _pi, _pi, C.POINTER(_pi),
                                    C.POINTER(_pi), C.POINTER(_pd)]
    L.orc_amg_level_csr.restype = _i
    L.orc_amg_aggregates.argtypes = [C.c_void_p, _i, _pi]
    L.orc_amg_aggregates.restype = _pi
    L.orc_amg_coarse_inverse.argtypes = [C.c_void_p, _pi, _pi]
    L.orc_amg_coarse_inverse.restype = _pd
    L.orc_amg_operator_complexity.argtypes = [C.c_void_p]
    L.orc_amg_operator_complexity.restype = _d
    L.orc_pcg_gs.argtypes = [C.c_void_p, _pd, _pd, _d, _i, _pd]
    L.orc_pcg_gs.restype = _i
    L.orc_amg_cg.argtypes = [_i, C.POINTER(CsrView), C.POINTER(CsrView), C.POINTER(CsrView),
                             _pd, _i, _d, _pd, _pd, _d, _i]
    L.orc_amg_cg.restype = Stats
    L.orc_vcycle_apply.argtypes = [_i, C.POINTER(CsrView), C.POINTER(CsrView),
                                   C.POINTER(CsrView), _pd, _i, _d, _pd, _pd]
    L.orc_krylov.argtypes = [C.POINTER(CsrView), _pd, _pd, _i, _d, _i]
    L.orc_krylov.restype = Stats


def _declare_ref(R):
    R.ref_assemble.argtypes = [_i, _i, _pi, _pi, _pd, _pd, _pd, _d, _pd, _pd, _pd, _pd]
    R.ref_assemble.restype = _i
    R.ref_solve_host.argtypes = [C.POINTER(RefCsr), _pd, _pd, _i, _d, _i, _pi, _pd, _pi]
    R.ref_solve_host.restype = _i
    R.ref_solve_amg_cg_host.argtypes = [_i, C.POINTER(RefCsr), C.POINTER(RefCsr),
                                        C.POINTER(RefCsr), _pd, _i, _d, _pd, _pd, _d, _i, _pi,
                                        _pd, _pi]
    R.ref_solve_amg_cg_host.restype = _i
    R.ref_device_solver_solve.argtypes = [_i, _i, _i, _pi, _pi, _pi, _pi, _pi, _i,
                                          C.POINTER(RefCsr), C.POINTER(RefCsr),
                                          C.POINTER(RefCsr), _pd, _pd, _pd, _pd, _pd, _pd, _i,
                                          _i, _d, _i, _pi, _pd, _pi]
    R.ref_device_solver_solve.restype = _i
    R.ref_backend_is_host.restype = _i


def _ip(a):
    return a.ctypes.data_as(_pi)


def _dp(a):
    return a.ctypes.data_as(_pd)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


@dataclass
class Csr:
    """Square or rectangular CSR matrix (int32 indices, float64 values)."""
    n_rows: int
    n_cols: int
    rp: np.ndarray
    ci: np.ndarray
    va: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.rp[-1])

    def view(self) -> CsrView:
        return CsrView(self.n_rows, _ip(self.rp), _ip(self.ci), _dp(self.va))

    def ref_view(self) -> RefCsr:
        return RefCsr(self.n_rows, self.nnz, _ip(self.rp), _ip(self.ci), _dp(self.va))

    def matvec(self, x: np.ndarray) -> np.ndarray:
        y = np.zeros(self.n_rows)
        x = _f64(x)
        lib().orc_csr_spmv(self.n_rows, _ip(self.rp), _ip(self.ci), _dp(self.va), _dp(x), _dp(y))
        return y

    def dense(self) -> np.ndarray:
        d = np.zeros((self.n_rows, self.n_cols))
        for i in range(self.n_rows):
            for k in range(self.rp[i], self.rp[i + 1]):
                d[i, self.ci[k]] += self.va[k]
        return d


# ---------------------------------------------------------------------------------------
# LDU matrix
# ---------------------------------------------------------------------------------------

@dataclass
class Pattern:
    n: int
    n_faces: int
    row_ptr: np.ndarray
    col: np.ndarray
    diag_pos: np.ndarray
    upper_pos: np.ndarray
    lower_pos: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])


def build_pattern(n: int, owner, neighbour) -> Pattern:
    """build_csr_pattern (ldu_matrix.cpp:572-612)."""
    nei = _i32(neighbour)
    nf = len(nei)
    own = _i32(owner[:nf])
    rp = np.zeros(n + 1, np.int32)
    col = np.zeros(n + 2 * nf, np.int32)
    dp, up, lp = np.zeros(n, np.int32), np.zeros(nf, np.int32), np.zeros(nf, np.int32)
    nnz = lib().orc_build_pattern(n, nf, _ip(own), _ip(nei), _ip(rp), _ip(col), _ip(dp),
                                  _ip(up), _ip(lp))
    if nnz < 0:
        raise ValueError("build_pattern: face index out of range")
    return Pattern(n, nf, rp, col[:nnz].copy(), dp, up, lp)


def assemble(n_cells, owner, neighbour, flux, gamma, delta, convection=0.0, diag=None,
             div=None):
    """Serial assemble_openmp face loop; returns (upper, lower, diag, div)."""
    nei = _i32(neighbour)
    nf = len(nei)
    own = _i32(owner[:nf])
    flux, gamma, delta = _f64(flux), _f64(gamma), _f64(delta)
    up, lo = np.zeros(nf), np.zeros(nf)
    dg = np.zeros(n_cells) if diag is None else _f64(diag).copy()
    dv = np.zeros(n_cells) if div is None else _f64(div).copy()
    lib().orc_assemble(n_cells, nf, _ip(own), _ip(nei), _dp(flux), _dp(gamma), _dp(delta),
                       float(convection), _dp(up), _dp(lo), _dp(dg), _dp(dv))
    return up, lo, dg, dv


def ldu_multiply(owner, neighbour, diag, upper, lower, x):
    nei = _i32(neighbour)
    own = _i32(owner[:len(nei)])
    diag, upper, lower, x = _f64(diag), _f64(upper), _f64(lower), _f64(x)
    y = np.zeros(len(diag))
    lib().orc_ldu_multiply(len(diag), len(own), _ip(own), _ip(nei), _dp(diag), _dp(upper),
                           _dp(lower), _dp(x), _dp(y))
    return y


def ldu_residual_norms(owner, neighbour, diag, upper, lower, source, x):
    nei = _i32(neighbour)
    own = _i32(owner[:len(nei)])
    args = [_f64(a) for a in (diag, upper, lower, source, x)]
    out = np.zeros(2)
    lib().orc_ldu_residual_norms(len(args[0]), len(own), _ip(own), _ip(nei),
                                 *[_dp(a) for a in args], _dp(out))
    return float(out[0]), float(out[1])


def normalised_residual(owner, neighbour, diag, upper, lower, source, x):
    """LduMatrix::normalised_residual (ldu_matrix.cpp:65-67)."""
    res, norm = ldu_residual_norms(owner, neighbour, diag, upper, lower, source, x)
    return res / (norm + 1e-20)


def correct_flux(owner, neighbour, flux, gamma, delta, p, non_orth=None):
    """Conservative internal-face flux of FlowSolver::pressure_correction
    (flow_solver.cpp:821-826): phi_hbya - rau_f * dc * (p[N] - p[P]) - non_orth, elementwise in
    that rounding order (numpy float64 rounds each operation; no fused multiply-add)."""
    own, nei = np.asarray(owner), np.asarray(neighbour)
    no = np.zeros(len(nei)) if non_orth is None else np.asarray(non_orth, np.float64)
    return (np.asarray(flux, np.float64) - (np.asarray(gamma, np.float64) * np.asarray(delta, np.float64))
            * (np.asarray(p)[nei] - np.asarray(p)[own])) - no


def pressure_gradient(n_cells, n_internal, owner, neighbour, weights, face_areas, face_centres,
                      cell_centres, cell_volumes, kinds, outlet_pressure, p):
    """FlowSolver::pressure_gradient, Gauss branch (flow_solver.cpp:339-372), face by face in the
    reference's order: internal faces add S_f (w p_P + (1 - w) p_N) to the owner and subtract
    it from the neighbour; two passes over the boundary faces add S_f p_b (p_b = outlet
    pressure, else p_P; the second pass adds the tangential extrapolation prev_P . (d - (d.n) n)
    to every non-outlet face); the sums are divided by the cell volume. Every product and sum
    is rounded separately (Python floats). Small meshes only: plain loops. kinds: 2 = outlet."""
    nf = len(owner)
    internal = [[0.0, 0.0, 0.0] for _ in range(n_cells)]
    for f in range(n_internal):
        o, n = int(owner[f]), int(neighbour[f])
        w = float(weights[f])
        s = w * float(p[o]) + (1.0 - w) * float(p[n])
        for i in range(3):
            fl = float(face_areas[f][i]) * s
            internal[o][i] = internal[o][i] + fl
            internal[n][i] = internal[n][i] - fl
    prev = None
    for pas in range(2):
        grad = [list(g) for g in internal]
        for f in range(n_internal, nf):
            c = int(owner[f])
            b = f - n_internal
            outlet = int(kinds[b]) == 2
            pb = float(outlet_pressure[b]) if outlet else float(p[c])
            sf = [float(v) for v in face_areas[f]]
            if pas > 0 and not outlet:
                area = math.sqrt((sf[0] * sf[0] + sf[1] * sf[1]) + sf[2] * sf[2])
                nrm = [v / area for v in sf]
                d = [float(face_centres[f][i]) - float(cell_centres[c][i]) for i in range(3)]
                dn = (d[0] * nrm[0] + d[1] * nrm[1]) + d[2] * nrm[2]
                t = [d[i] - dn * nrm[i] for i in range(3)]
                pb = pb + ((prev[c][0] * t[0] + prev[c][1] * t[1]) + prev[c][2] * t[2])
            for i in range(3):
                grad[c][i] = grad[c][i] + sf[i] * pb
        for c in range(n_cells):
            v = float(cell_volumes[c])
            grad[c] = [g / v for g in grad[c]]
        prev = grad
    return np.array(grad)


def fv_delta_corrections(n_internal, owner, neighbour, face_areas, face_centres, cell_centres):
    """Delta coefficients of every face and non-orthogonal corrections of the internal faces
    (fv_geometry.cpp:34-50): delta = |S|^2 / max(S.d, 0.05 |S||d|), k = S - d delta."""
    nf = len(owner)
    delta = np.zeros(nf)
    corr = np.zeros((n_internal, 3))
    dot = lambda a, b: (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]  # noqa: E731
    for f in range(nf):
        s = [float(v) for v in face_areas[f]]
        cp = [float(v) for v in cell_centres[int(owner[f])]]
        to = cell_centres[int(neighbour[f])] if f < n_internal else face_centres[f]
        d = [float(to[i]) - cp[i] for i in range(3)]
        area = math.sqrt(dot(s, s))
        sd = max(dot(s, d), 0.05 * area * math.sqrt(dot(d, d)))
        delta[f] = area * area / sd
        if f < n_internal:
            corr[f] = [s[i] - d[i] * delta[f] for i in range(3)]
    return delta, corr


def pressure_step_parts(m, kinds, outlet_pressure, mom_diag, mom_upper, mom_lower, mom_source, u,
                        fixed_velocity, u_prev=None, phi_prev=None, alpha_u=1.0, ref_cell=-1,
                        ref_value=0.0):
    """FlowSolver::pressure_correction up to the solve, face by face in the reference's order
    (flow_solver.cpp:688-796, GpuCg branch): HbyA, rAU, predicted flux phi_hbya and rau_f on
    every face (with the relaxation-independent term when u_prev / phi_prev are given and
    alpha_u < 1), the pressure matrix (internal assembly as krylov_openmp.cpp:289-300, then
    source = -divergence) with the boundary terms and set_reference. Returns a dict."""
    n, nf, ni = m.n_cells, m.n_faces, m.n_internal_faces
    own, nei, w, sf = m.owner, m.neighbour, m.weights, m.face_areas
    delta, _ = fv_delta_corrections(ni, own, nei, sf, m.face_centres, m.cell_centres)
    dot = lambda a, b: (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]  # noqa: E731
    hbya = np.zeros((n, 3))
    for i in range(3):
        off = [0.0] * n
        for f in range(ni):
            p, q = int(own[f]), int(nei[f])
            off[p] = off[p] + float(mom_upper[f]) * float(u[q][i])
            off[q] = off[q] + float(mom_lower[f]) * float(u[p][i])
        for c in range(n):
            hbya[c][i] = (float(mom_source[c][i]) - off[c]) / float(mom_diag[c][i])
    rau = np.array([float(m.cell_volumes[c]) / (((float(mom_diag[c][0]) + float(mom_diag[c][1]))
                    + float(mom_diag[c][2])) / 3.0) for c in range(n)])
    phi = np.zeros(nf)
    rau_f = np.zeros(nf)
    for f in range(ni):
        p, q = int(own[f]), int(nei[f])
        wf = float(w[f])
        v = [wf * hbya[p][i] + (1.0 - wf) * hbya[q][i] for i in range(3)]
        phi[f] = dot(v, sf[f])
        rau_f[f] = wf * rau[p] + (1.0 - wf) * rau[q]
    for f in range(ni, nf):
        p, b = int(own[f]), f - ni
        rau_f[f] = rau[p]
        k = int(kinds[b])
        phi[f] = dot(fixed_velocity[b], sf[f]) if k in (0, 1) else (dot(hbya[p], sf[f]) if k == 2 else 0.0)
    if u_prev is not None and phi_prev is not None and alpha_u < 1.0:
        beta = 1.0 - alpha_u
        for f in range(ni):
            p, q = int(own[f]), int(nei[f])
            wf = float(w[f])
            uf = [wf * float(u_prev[p][i]) + (1.0 - wf) * float(u_prev[q][i]) for i in range(3)]
            phi[f] = phi[f] + beta * (float(phi_prev[f]) - dot(uf, sf[f]))
        for f in range(ni, nf):
            if int(kinds[f - ni]) == 2:
                p = int(own[f])
                phi[f] = phi[f] + beta * (float(phi_prev[f]) - dot(u_prev[p], sf[f]))
    up, lo, dg, dv = assemble(n, own[:ni], nei, phi[:ni], rau_f[:ni], delta[:ni], 0.0)
    source = 0.0 - dv
    for f in range(ni, nf):
        p, b = int(own[f]), f - ni
        source[p] = source[p] - phi[f]
        if int(kinds[b]) == 2:
            coeff = rau_f[f] * delta[f]
            dg[p] = dg[p] + coeff
            source[p] = source[p] + coeff * float(outlet_pressure[b])
    if ref_cell >= 0:
        source[ref_cell] = source[ref_cell] + dg[ref_cell] * ref_value
        dg[ref_cell] = dg[ref_cell] + dg[ref_cell]
    return dict(hbya=hbya, rau=rau, phi_hbya=phi, rau_f=rau_f, upper=up, lower=lo, diag=dg,
                source=source, delta=delta)


def non_orth_source(m, grad, rau_f, base_source):
    """Non-orthogonal corrector terms (flow_solver.cpp:805-816): (non_orth, source)."""
    ni = m.n_internal_faces
    _, corr = fv_delta_corrections(ni, m.owner, m.neighbour, m.face_areas, m.face_centres,
                                   m.cell_centres)
    non_orth = np.zeros(ni)
    source = np.array(base_source, np.float64)
    for f in range(ni):
        p, q = int(m.owner[f]), int(m.neighbour[f])
        wf = float(m.weights[f])
        v = [wf * float(grad[p][i]) + (1.0 - wf) * float(grad[q][i]) for i in range(3)]
        non_orth[f] = float(rau_f[f]) * ((corr[f][0] * v[0] + corr[f][1] * v[1]) + corr[f][2] * v[2])
        source[p] = source[p] + non_orth[f]
        source[q] = source[q] - non_orth[f]
    return non_orth, source


def correct_flux_all(m, kinds, outlet_pressure, phi_hbya, rau_f, delta, non_orth, p_new):
    """Conservative flux on every face (flow_solver.cpp:818-833)."""
    ni = m.n_internal_faces
    phi = np.zeros(m.n_faces)
    for f in range(m.n_faces):
        p = int(m.owner[f])
        coeff = float(rau_f[f]) * float(delta[f])
        if f < ni:
            q = int(m.neighbour[f])
            phi[f] = (float(phi_hbya[f]) - coeff * (float(p_new[q]) - float(p_new[p]))) - float(non_orth[f])
        else:
            phi[f] = float(phi_hbya[f])
            if int(kinds[f - ni]) == 2:
                phi[f] = phi[f] - coeff * (float(outlet_pressure[f - ni]) - float(p_new[p]))
    return phi


def correct_velocity(hbya, rau, grad):
    """u = HbyA - rAU grad p (flow_solver.cpp:843-846)."""
    return np.asarray(hbya, np.float64) - np.asarray(rau, np.float64)[:, None] * np.asarray(grad, np.float64)


def relax(p_prev, p_new, alpha):
    """Pressure under-relaxation of FlowSolver::pressure_correction (flow_solver.cpp:837-840)."""
    p_prev, p_new = np.asarray(p_prev, np.float64), np.asarray(p_new, np.float64)
    return p_prev + alpha * (p_new - p_prev)


def set_reference(diag, source, cell, value):
    """In place, like LduMatrix::set_reference."""
    assert diag.dtype == np.float64 and source.dtype == np.float64
    lib().orc_set_reference(_dp(diag), _dp(source), int(cell), float(value))


def ldu_to_csr(pattern: Pattern, diag, upper, lower) -> Csr:
    val = np.zeros(pattern.nnz)
    lib().orc_ldu_to_csr(pattern.n, pattern.n_faces, _ip(pattern.diag_pos),
                         _ip(pattern.upper_pos), _ip(pattern.lower_pos), _dp(_f64(diag)),
                         _dp(_f64(upper)), _dp(_f64(lower)), _dp(val))
    return Csr(pattern.n, pattern.n, pattern.row_ptr, pattern.col, val)


# ---------------------------------------------------------------------------------------
# AMG
# ---------------------------------------------------------------------------------------

def aggregate(a: Csr, diag, theta=0.08):
    agg = np.zeros(a.n_rows, np.int32)
    n_agg = lib().orc_aggregate(a.n_rows, _ip(a.rp), _ip(a.ci), _dp(a.va), _dp(_f64(diag)),
                                float(theta), _ip(agg))
    return agg, int(n_agg)


class Hierarchy:
    """AmgPreconditioner::setup (amg.cpp:122-190) restated in C; arrays are copied out."""

    def __init__(self, a: Csr, theta=0.08, max_levels=25, coarse_size=400):
        L = lib()
        h = L.orc_amg_setup(a.n_rows, _ip(a.rp), _ip(a.ci), _dp(a.va), float(theta),
                            int(max_levels), int(coarse_size))
        if not h:
            raise ValueError("amg setup failed")
        self._h = h
        self.a, self.p, self.r, self.aggregates = [], [], [], []
        nl = L.orc_amg_levels(h)
        for l in range(nl):
            row = []
            for which in range(3):
                nr, nc, nz = _i(), _i(), _i()
                rp, ci, va = _pi(), _pi(), _pd()
                ok = L.orc_amg_level_csr(h, l, which, C.byref(nr), C.byref(nc), C.byref(nz),
                                         C.byref(rp), C.byref(ci), C.byref(va))
                if not ok:
                    row.append(None)
                    continue
                row.append(Csr(nr.value, nc.value,
                               np.ctypeslib.as_array(rp, (nr.value + 1,)).copy(),
                               np.ctypeslib.as_array(ci, (max(nz.value, 1),))[:nz.value].copy(),
                               np.ctypeslib.as_array(va, (max(nz.value, 1),))[:nz.value].copy()))
            self.a.append(row[0])
            self.p.append(row[1])
            self.r.append(row[2])
            if l + 1 < nl:
                na = _i()
                ptr = L.orc_amg_aggregates(h, l, C.byref(na))
                self.aggregates.append(np.ctypeslib.as_array(ptr, (self.a[l].n_rows,)).copy())
        nc, ok = _i(), _i()
        ptr = L.orc_amg_coarse_inverse(h, C.byref(nc), C.byref(ok))
        self.coarse_inverse = np.ctypeslib.as_array(ptr, (nc.value * nc.value,)).copy()
        self.coarse_ldlt_ok = bool(ok.value)
        self.operator_complexity = float(L.orc_amg_operator_complexity(h))

    @property
    def levels(self) -> int:
        return len(self.a)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_amg_free(h)
            self._h = None

    def pcg_gs(self, b, x=None, tol=1e-10, max_iterations=500):
        """CPU AmgCg: pcg with the Gauss-Seidel V-cycle (amg.cpp:253-285)."""
        b = _f64(b)
        x = np.zeros_like(b) if x is None else _f64(x).copy()
        res = _d()
        it = lib().orc_pcg_gs(self._h, _dp(b), _dp(x), float(tol), int(max_iterations),
                              C.byref(res))
        return x, int(it), float(res.value)


def _level_arrays(a_levels, p_levels, r_levels):
    nl = len(a_levels)
    empty = CsrView(0, None, None, None)
    A = (CsrView * nl)(*[m.view() for m in a_levels])
    P = (CsrView * nl)(*[(p_levels[l].view() if l + 1 < nl else empty) for l in range(nl)])
    R = (CsrView * nl)(*[(r_levels[l].view() if l + 1 < nl else empty) for l in range(nl)])
    return nl, A, P, R


def amg_cg(a_levels, p_levels, r_levels, coarse_inverse, b, x=None, abs_tol=1e-10,
           max_iterations=1000, sweeps=2, weight=0.7):
    """GPU-path AMG-PCG (krylov_kernels.inc:240-301) restated serially; returns (x, stats)."""
    nl, A, P, R = _level_arrays(a_levels, p_levels, r_levels)
    b = _f64(b)
    x = np.zeros_like(b) if x is None else _f64(x).copy()
    ci = _f64(coarse_inverse)
    st = lib().orc_amg_cg(nl, A, P, R, _dp(ci), int(sweeps), float(weight), _dp(b), _dp(x),
                          float(abs_tol), int(max_iterations))
    return x, {"iterations": st.iterations, "residual": st.residual,
               "converged": bool(st.converged)}


def vcycle_apply(a_levels, p_levels, r_levels, coarse_inverse, rhs, sweeps=2, weight=0.7):
    nl, A, P, R = _level_arrays(a_levels, p_levels, r_levels)
    rhs = _f64(rhs)
    z = np.zeros_like(rhs)
    lib().orc_vcycle_apply(nl, A, P, R, _dp(_f64(coarse_inverse)), int(sweeps), float(weight),
                           _dp(rhs), _dp(z))
    return z


def krylov(a: Csr, b, x=None, method=0, abs_tol=1e-10, max_iterations=1000):
    """Jacobi-preconditioned CG (method 0) / BiCGStab (method 1), krylov_kernels.inc:44-169."""
    b = _f64(b)
    x = np.zeros_like(b) if x is None else _f64(x).copy()
    v = a.view()
    st = lib().orc_krylov(C.byref(v), _dp(b), _dp(x), int(method), float(abs_tol),
                          int(max_iterations))
    return x, {"iterations": st.iterations, "residual": st.residual,
               "converged": bool(st.converged)}


# ---------------------------------------------------------------------------------------
# The reference's compiled host path (oracle/_ref)
# ---------------------------------------------------------------------------------------

def ref_assemble(n_cells, owner, neighbour, flux, gamma, delta, convection=0.0, diag=None,
                 div=None):
    R = ref()
    nei = _i32(neighbour)
    nf = len(nei)
    own = _i32(owner[:nf])
    up, lo = np.zeros(nf), np.zeros(nf)
    dg = np.zeros(n_cells) if diag is None else _f64(diag).copy()
    dv = np.zeros(n_cells) if div is None else _f64(div).copy()
    rc = R.ref_assemble(n_cells, nf, _ip(own), _ip(nei), _dp(_f64(flux)), _dp(_f64(gamma)),
                        _dp(_f64(delta)), float(convection), _dp(up), _dp(lo), _dp(dg), _dp(dv))
    assert rc == 0
    return up, lo, dg, dv


def _ref_levels(a_levels, p_levels, r_levels):
    nl = len(a_levels)
    empty = RefCsr(0, 0, None, None, None)
    A = (RefCsr * nl)(*[(m.ref_view() if m is not None else empty) for m in a_levels])
    P = (RefCsr * nl)(*[(p_levels[l].ref_view() if l + 1 < nl else empty) for l in range(nl)])
    R = (RefCsr * nl)(*[(r_levels[l].ref_view() if l + 1 < nl else empty) for l in range(nl)])
    return nl, A, P, R


def ref_amg_cg(a_levels, p_levels, r_levels, coarse_inverse, b, x=None, abs_tol=1e-10,
               max_iterations=1000, sweeps=2, weight=0.7):
    R = ref()
    nl, A, P, RR = _ref_levels(a_levels, p_levels, r_levels)
    b = _f64(b)
    x = np.zeros_like(b) if x is None else _f64(x).copy()
    it, res, conv = _i(), _d(), _i()
    rc = R.ref_solve_amg_cg_host(nl, A, P, RR, _dp(_f64(coarse_inverse)), int(sweeps),
                                 float(weight), _dp(b), _dp(x), float(abs_tol),
                                 int(max_iterations), C.byref(it), C.byref(res), C.byref(conv))
    assert rc == 0
    return x, {"iterations": it.value, "residual": res.value, "converged": bool(conv.value)}


def ref_krylov(a: Csr, b, x=None, method=0, abs_tol=1e-10, max_iterations=1000):
    R = ref()
    b = _f64(b)
    x = np.zeros_like(b) if x is None else _f64(x).copy()
    v = a.ref_view()
    it, res, conv = _i(), _d(), _i()
    rc = R.ref_solve_host(C.byref(v), _dp(b), _dp(x), int(method), float(abs_tol),
                          int(max_iterations), C.byref(it), C.byref(res), C.byref(conv))
    assert rc == 0
    return x, {"iterations": it.value, "residual": res.value, "converged": bool(conv.value)}


def ref_device_solver(pattern: Pattern, hierarchy, diag, upper, lower, b, x=None, method=0,
                      use_amg=True, abs_tol=1e-10, max_iterations=1000):
    """cfd::gpu::DeviceSolver host path: LDU scatter + AMG-PCG / Jacobi Krylov."""
    R = ref()
    if hierarchy is not None:
        nl, A, P, RR = _ref_levels([None] + list(hierarchy.a[1:]), hierarchy.p, hierarchy.r)
        ci = _f64(hierarchy.coarse_inverse)
        cip = _dp(ci)
    else:
        nl, A, P, RR, cip = 0, None, None, None, None
    b = _f64(b)
    x = np.zeros_like(b) if x is None else _f64(x).copy()
    it, res, conv = _i(), _d(), _i()
    rc = R.ref_device_solver_solve(
        pattern.n, pattern.n_faces, pattern.nnz, _ip(pattern.row_ptr), _ip(pattern.col),
        _ip(pattern.diag_pos), _ip(pattern.upper_pos), _ip(pattern.lower_pos), nl, A, P, RR,
        cip, _dp(_f64(diag)), _dp(_f64(upper)), _dp(_f64(lower)), _dp(b), _dp(x), int(method),
        1 if use_amg else 0, float(abs_tol), int(max_iterations), C.byref(it), C.byref(res),
        C.byref(conv))
    assert rc == 0
    return x, {"iterations": it.value, "residual": res.value, "converged": bool(conv.value)}
