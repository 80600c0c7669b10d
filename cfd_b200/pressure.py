"""FlowSolver::pressure_correction (flow_solver.cpp:673-847) with every array in device memory:
HbyA and rAU from the momentum system, the predicted face flux, the pressure equation
(internal faces, boundary terms, reference cell), the non-orthogonal correctors, the
persistent LDU solve with its AMG cache, the conservative flux, pressure relaxation, the
pressure gradient and the velocity correction. The steps run in the reference's order; the
face and cell loops are the library's device kernels (bit-identical to the reference's serial
loops) and the solve is cfdb_system_solve_ldu."""
from __future__ import annotations

from dataclasses import dataclass

from . import AmgSettings, DeviceSolver, FvGeometry, LduSettings


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


def pressure_correction(ds: DeviceSolver, fv: FvGeometry, mom_diag, mom_upper, mom_lower, mom_source,
                        u, p, fixed_velocity, settings: PressureSettings | None = None, relax_p=True,
                        u_prev=None, phi_prev=None, phi=None, keep=None):
    """One pressure correction on CUDA float64 tensors: u (n_cells x 3) and p (n_cells) are
    updated in place, phi (n_faces, optional) receives the conservative face flux. Returns the
    initial normalised residual of the first pressure solve. keep: a dict that receives the
    intermediate arrays (for checking)."""
    import torch
    s = settings or PressureSettings()
    n, nf, ni = fv.n_cells, fv.n_faces, fv.n_internal_faces
    dev, f64 = p.device, torch.float64
    z = lambda *shape: torch.zeros(*shape, dtype=f64, device=dev)  # noqa: E731
    torch.cuda.current_stream().synchronize()
    e = lambda *shape: torch.empty(*shape, dtype=f64, device=dev)  # noqa: E731  (fully written)
    hbya, rau = e(n, 3), e(n)
    fv.hbya_rau_device(mom_diag, mom_upper, mom_lower, mom_source, u, hbya, rau)
    phi_hbya, rau_f = e(nf), e(nf)
    majumdar = u_prev is not None and phi_prev is not None and s.alpha_u < 1.0
    fv.face_flux_device(hbya, rau, fixed_velocity, phi_hbya, rau_f,
                        u_prev if majumdar else None, phi_prev if majumdar else None,
                        1.0 - s.alpha_u if majumdar else 0.0)
    upper, lower, diag, source = z(ni), z(ni), z(n), z(n)
    delta = fv.delta_device()
    ds.assemble_pressure_device(phi_hbya, rau_f, delta, z(n), upper, lower, diag, source,
                                ref_cell=-1)
    torch.cuda.synchronize()
    fv.pressure_boundary_device(phi_hbya, rau_f, diag, source, s.ref_cell, s.ref_value)
    base_source = source.clone()
    p_prev = p.clone()
    p_new = p.clone()
    non_orth = z(max(ni, 1))
    grad = z(n, 3)
    initial = 0.0
    for corr in range(s.n_non_orth_correctors + 1):
        non_orth.zero_()
        source.copy_(base_source)
        if corr > 0 or s.n_non_orth_correctors > 0:
            torch.cuda.synchronize()
            fv.pressure_gradient_device(p_new, grad)
            fv.non_orth_device(grad, rau_f, base_source, non_orth, source)
        torch.cuda.synchronize()
        r = ds.solve_ldu(diag, upper, lower, source, p_new, s.p_solver or LduSettings(), s.amg or AmgSettings())
        if corr == 0:
            initial = r.initial_residual
        if keep is not None:
            keep.setdefault("solves", []).append((r, p_new.clone(), source.clone()))
    phi_out = phi if phi is not None else z(nf)
    fv.correct_flux_device(phi_hbya, rau_f, p_new, phi_out, non_orth)
    if relax_p:
        fv.relax_device(p_prev, p_new, s.alpha_p, p)
    else:
        p.copy_(p_new)
    fv.pressure_gradient_device(p, grad)
    fv.correct_velocity_device(hbya, rau, grad, u)
    if keep is not None:
        keep.update(hbya=hbya, rau=rau, phi_hbya=phi_hbya, rau_f=rau_f, upper=upper, lower=lower,
                    diag=diag, base_source=base_source, p_new=p_new, non_orth=non_orth, phi=phi_out,
                    grad=grad)
    return initial
