"""Face-by-face restatement of solve_scalar's assembly on the GPU path (TEST INFRASTRUCTURE ONLY).

Follows src/fv/src/scalar_transport.cpp with `device` and `device_fv` true:
  * boundary_values            :10-40   (fixed value, zero / fixed gradient, mixed);
  * DeviceFv::scalar_corrections :81-83 (oracle/fvcells.py, pinned to the compiled reference);
  * assemble_convection_diffusion(convection = 1) :85-90 (the C oracle's serial face loop,
    pinned to the compiled reference);
  * the boundary-face loop     :127-148;
  * the cell loop              :150-161 (bounded convection form, sources, time term,
    under-relaxation);
  * fixed cells                :162-177.
Plain Python loops over faces and cells in the reference's order with float64 arithmetic, so
the result is what the reference computes, operation for operation. Small meshes only. The
reference's solve_scalar itself is not compiled here (it needs Eigen and the fv library).
"""
from __future__ import annotations

import numpy as np

from . import assemble as _assemble
from . import fvcells as F

FIXED_VALUE, ZERO_GRADIENT, FIXED_GRADIENT, MIXED = 0, 1, 2, 3


def _dn(v, un, f, p):
    d = v.cf[f] - v.cc[p]
    return abs(d[0] * un[f, 0] + d[1] * un[f, 1] + d[2] * un[f, 2])


def _min(a, b):  # std::min
    return b if b < a else a


def _max(a, b):  # std::max
    return b if a < b else a


def boundary_values(v, un, kind, value, coef, field):
    """scalar_transport.cpp:10-40."""
    nb = v.nf - v.nif
    out = np.zeros(nb)
    for b in range(nb):
        f = v.nif + b
        p = v.own[f]
        k = kind[b]
        if k == FIXED_VALUE:
            out[b] = value[b]
        elif k == ZERO_GRADIENT:
            out[b] = field[p]
        elif k == FIXED_GRADIENT:
            out[b] = field[p] + value[b] * _dn(v, un, f, p)
        else:
            rd = coef[b] * _dn(v, un, f, p)
            out[b] = (field[p] + rd * value[b]) / (1.0 + rd)
    return out


def scalar_system(v, dc, un, area, eq: dict, face_flux, field):
    """(upper, lower, diag, source, field) of solve_scalar's GPU path before a.solve; eq holds
    numpy arrays gamma_face, su, sp, bc_kind, bc_value, bc_coefficient and optional fixed_cell,
    fixed_value, old_value, capacity, plus relaxation, dt, linear_upwind, gradient."""
    nc, nif, nf = v.nc, v.nif, v.nf
    field = np.array(field, np.float64)
    flux = np.asarray(face_flux, np.float64)
    gamma = np.asarray(eq["gamma_face"], np.float64)
    un = np.asarray(un, np.float64).reshape(-1, 3)
    bv = boundary_values(v, un, eq["bc_kind"], eq["bc_value"], eq["bc_coefficient"], field)
    source = F.scalar_corrections(v, field, bv, eq.get("gradient", 0), flux, gamma,
                                  eq.get("linear_upwind", True), np.zeros(nc))
    upper, lower, diag, div = _assemble(nc, v.own[:nif], v.nei, flux[:nif], gamma[:nif], dc[:nif], 1.0)
    kind, value, coef = eq["bc_kind"], eq["bc_value"], eq["bc_coefficient"]
    for f in range(nif, nf):
        p = v.own[f]
        fl = flux[f]
        b = f - nif
        div[p] += fl
        if kind[b] == FIXED_VALUE:
            diff = gamma[f] * dc[f]
            diag[p] += diff + _max(fl, 0.0)
            source[p] += (diff - _min(fl, 0.0)) * value[b]
        elif kind[b] == MIXED:
            dn = _dn(v, un, f, p)
            rd = coef[b] * dn
            cm = gamma[f] * dc[f] * rd / (1.0 + rd)
            diag[p] += cm + fl
            source[p] += cm * value[b]
        else:
            diag[p] += fl
            if kind[b] == FIXED_GRADIENT:
                dn = _dn(v, un, f, p)
                source[p] += gamma[f] * value[b] * area[f] - fl * value[b] * dn
    su, sp, vol = eq["su"], eq["sp"], v.vol
    dt, relax = eq.get("dt", 0.0), eq.get("relaxation", 1.0)
    old, cap = eq.get("old_value"), eq.get("capacity")
    for c in range(nc):
        diag[c] -= div[c]
        diag[c] -= _min(sp[c], 0.0) * vol[c]
        source[c] += su[c] * vol[c] + _max(sp[c], 0.0) * field[c] * vol[c]
        if dt > 0.0:
            ddt = vol[c] / dt * (cap[c] if cap is not None else 1.0)
            diag[c] += ddt
            source[c] += ddt * (old[c] if old is not None else field[c])
        if relax < 1.0:
            d1 = diag[c] / relax
            source[c] += (d1 - diag[c]) * field[c]
            diag[c] = d1
    fixed = eq.get("fixed_cell")
    if fixed is not None:
        for f in range(nif):
            if fixed[v.own[f]] != 0:
                upper[f] = 0.0
            if fixed[v.nei[f]] != 0:
                lower[f] = 0.0
        for c in range(nc):
            if fixed[c] != 0:
                diag[c] = 1.0
                source[c] = eq["fixed_value"][c]
                field[c] = eq["fixed_value"][c]
    return upper, lower, diag, source, field
