"""FlowSolver::pressure_correction (flow_solver.cpp:673-847) with every array in device memory,
through one C-ABI call (cfdb_pressure_correction_device, composed in C++ in
cfd_b200/csrc/pressure_step.cu): HbyA and rAU from the momentum system, the predicted face
flux, the pressure equation (internal faces, boundary terms, reference cell), the
non-orthogonal correctors, the persistent LDU solve with its AMG cache, the conservative flux,
pressure relaxation, the pressure gradient and the velocity correction. The steps run in the
reference's order; the face and cell loops are the library's device kernels (bit-identical to
the reference's serial loops) and the solve is cfdb_system_solve_ldu."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import (AmgSettings, AmgSettingsStruct, DeviceSolver, FvGeometry, LduResult, LduResultStruct, LduSettings,
               LduSettingsStruct, _check, _devptr, _lib, _stream_ordered)


@dataclass
class PressureSettings:
    """The FlowSolver settings the step reads (flow_solver.hpp): under-relaxation factors,
    non-orthogonal correctors, the pressure solver and the reference cell (-1: none, for a
    case with a pressure outlet)."""
    alpha_u: float = 0.7
    alpha_p: float = 0.3
    n_non_orth_correctors: int = 0
    p_solver: LduSettings = None
    amg: AmgSettings = None
    ref_cell: int = 0
    ref_value: float = 0.0


class PressureSettingsStruct(C.Structure):
    _fields_ = [("alpha_u", C.c_double), ("alpha_p", C.c_double), ("n_non_orth_correctors", C.c_int),
                ("ref_cell", C.c_int), ("ref_value", C.c_double), ("relax_p", C.c_int),
                ("p_solver", LduSettingsStruct), ("amg", AmgSettingsStruct)]


class PressureWorkspaceStruct(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("hbya", "rau", "phi_hbya", "rau_f", "upper", "lower", "diag",
                                          "source", "base_source", "p_prev", "p_new", "non_orth", "grad",
                                          "phi", "solve_p", "solve_source")]


_lib.cfdb_pressure_correction_device.argtypes = [C.c_void_p] * 11 + [
    C.POINTER(PressureSettingsStruct), C.POINTER(PressureWorkspaceStruct), C.POINTER(LduResultStruct),
    C.POINTER(C.c_double)]
_lib.cfdb_pressure_correction_device.restype = C.c_int


@_stream_ordered
def pressure_correction(ds: DeviceSolver, fv: FvGeometry, mom_diag, mom_upper, mom_lower, mom_source,
                        u, p, fixed_velocity, settings: PressureSettings | None = None, relax_p=True,
                        u_prev=None, phi_prev=None, phi=None, keep=None, results=None):
    """One pressure correction on CUDA float64 tensors: u (n_cells x 3) and p (n_cells) are
    updated in place, phi (n_faces, optional) receives the conservative face flux. Returns the
    initial normalised residual of the first pressure solve. keep: a dict that receives the
    workspace arrays and, under "solves", (result, p after, right-hand side) of every solve.
    results: a list that receives the LduResult of every solve."""
    import torch
    s = settings or PressureSettings()
    n, nf, ni = fv.n_cells, fv.n_faces, fv.n_internal_faces
    dev, f64 = p.device, torch.float64
    e = lambda *shape: torch.empty(*shape, dtype=f64, device=dev)  # noqa: E731
    n_solves = s.n_non_orth_correctors + 1
    ws = dict(hbya=e(n, 3), rau=e(n), phi_hbya=e(nf), rau_f=e(nf), upper=e(max(ni, 1)), lower=e(max(ni, 1)),
              diag=e(n), source=e(n), base_source=e(n), p_prev=e(n), p_new=e(n), non_orth=e(max(ni, 1)),
              grad=e(n, 3), phi=phi if phi is not None else e(nf))
    if keep is not None:
        ws["solve_p"], ws["solve_source"] = e(n_solves, n), e(n_solves, n)
    wst = PressureWorkspaceStruct(**{k: _devptr(v) for k, v in ws.items()})
    cs = PressureSettingsStruct(float(s.alpha_u), float(s.alpha_p), int(s.n_non_orth_correctors), int(s.ref_cell),
                                float(s.ref_value), 1 if relax_p else 0, (s.p_solver or LduSettings())._c(),
                                (s.amg or AmgSettings())._c())
    res = (LduResultStruct * n_solves)()
    initial = C.c_double()
    ptr = lambda t: None if t is None else _devptr(t)  # noqa: E731
    _check(_lib.cfdb_pressure_correction_device(
        ds._h, fv._h, _devptr(mom_diag), _devptr(mom_upper), _devptr(mom_lower), _devptr(mom_source),
        _devptr(u), _devptr(p), ptr(fixed_velocity), ptr(u_prev), ptr(phi_prev), C.byref(cs), C.byref(wst),
        res, C.byref(initial)))
    out = [LduResult(r.initial_residual, r.final_residual, r.iterations, bool(r.amg_rebuilt)) for r in res]
    if results is not None:
        results.extend(out)
    if keep is not None:
        keep.update({k: v for k, v in ws.items() if k not in ("solve_p", "solve_source")})
        keep["solves"] = [(r, ws["solve_p"][k], ws["solve_source"][k]) for k, r in enumerate(out)]
    return initial.value
