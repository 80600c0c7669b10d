"""solve_scalar (scalar_transport.cpp:50-177) on the GPU path with every array in HBM.

The reference assembles the scalar transport equation with host face loops around two
accelerator calls (DeviceFv::scalar_corrections and assemble_convection_diffusion with
convection = 1), then solves it with LduMatrix::solve. Here the whole assembly is one call
(:meth:`DeviceFv.scalar_system_device`: boundary values, explicit corrections, coefficients,
boundary-face terms, sources, time term, under-relaxation, fixed cells) and the solve is the
persistent LDU solve of :class:`cfd_b200.DeviceSolver` (``solve_ldu``, the AmgCache rule
included). Results are bit-identical to the reference's loops; the solve matches its
LinearSolveResult semantics.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass

from . import InvalidArgument, LduResult, LduSettings, _check, _devptr, _lib, _proto, _stream_ordered
from .fv_device import DeviceFv


class ScalarBoundaryKind(enum.IntEnum):
    """scalar_transport.hpp:14."""
    FixedValue = 0
    ZeroGradient = 1
    FixedGradient = 2
    Mixed = 3


class ScalarEquationStruct(C.Structure):
    _fields_ = [("gamma_face", C.c_void_p), ("su", C.c_void_p), ("sp", C.c_void_p),
                ("bc_kind", C.c_void_p), ("bc_value", C.c_void_p), ("bc_coefficient", C.c_void_p),
                ("fixed_cell", C.c_void_p), ("fixed_value", C.c_void_p), ("relaxation", C.c_double),
                ("dt", C.c_double), ("old_value", C.c_void_p), ("capacity", C.c_void_p),
                ("linear_upwind", C.c_int), ("gradient", C.c_int)]


_proto("cfdb_device_fv_scalar_system_device",
       [C.c_void_p, C.POINTER(ScalarEquationStruct), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
        C.c_void_p, C.c_void_p])


@dataclass
class ScalarEquation:
    """ScalarEquation (scalar_transport.hpp:24-37) with CUDA float64 tensors (bc_kind int32,
    fixed_cell uint8); per boundary face kind / value / coefficient."""
    gamma_face: object
    su: object
    sp: object
    bc_kind: object
    bc_value: object
    bc_coefficient: object
    fixed_cell: object = None
    fixed_value: object = None
    relaxation: float = 1.0
    dt: float = 0.0
    old_value: object = None
    capacity: object = None
    linear_upwind: bool = True
    gradient: int = 0  # GradientScheme.Gauss

    def _c(self):
        p = lambda t: _devptr(t) if t is not None else None  # noqa: E731
        return ScalarEquationStruct(p(self.gamma_face), p(self.su), p(self.sp), p(self.bc_kind),
                                    p(self.bc_value), p(self.bc_coefficient), p(self.fixed_cell),
                                    p(self.fixed_value), float(self.relaxation), float(self.dt),
                                    p(self.old_value), p(self.capacity), 1 if self.linear_upwind else 0,
                                    int(self.gradient))


@_stream_ordered
def scalar_system_device(fv: DeviceFv, eq: ScalarEquation, face_flux, field, upper, lower, diag,
                         source) -> None:
    """The LDU system of solve_scalar into device arrays (field takes fixed values)."""
    s = eq._c()
    _check(_lib.cfdb_device_fv_scalar_system_device(fv._h, C.byref(s), _devptr(face_flux), _devptr(field),
                                                    _devptr(upper), _devptr(lower), _devptr(diag),
                                                    _devptr(source)))


def solve_scalar(ds, fv: DeviceFv, eq: ScalarEquation, face_flux, field,
                 settings: LduSettings | None = None, keep: dict | None = None) -> LduResult:
    """solve_scalar on the GPU path: assemble on the device, then LduMatrix::solve through the
    persistent solver ``ds`` (a :class:`cfd_b200.DeviceSolver` on the mesh's pattern). field is a
    CUDA float64 tensor, updated in place. ``keep`` (optional dict) receives the assembled
    upper / lower / diag / source tensors."""
    import torch
    if not (hasattr(field, "is_cuda") and field.is_cuda):
        raise InvalidArgument("solve_scalar: field must be a CUDA tensor")
    dev = field.device
    nif, nc = fv.n_internal_faces, fv.n_cells
    z = lambda n: torch.empty(n, dtype=torch.float64, device=dev)  # noqa: E731
    upper, lower, diag, source = z(max(nif, 1)), z(max(nif, 1)), z(nc), z(nc)
    torch.cuda.current_stream(dev).synchronize()
    scalar_system_device(fv, eq, face_flux, field, upper, lower, diag, source)
    if keep is not None:
        keep.update(upper=upper, lower=lower, diag=diag, source=source)
    return ds.solve_ldu(diag, upper[:nif], lower[:nif], source, field,
                        settings or LduSettings(method=1, tolerance=1e-8, rel_tolerance=0.01))
