"""Generates the golden fixtures of the hot path from the reference's own host implementation.

Run from the repository root in a container that has the reference checkout:
    python tests/golden/make_golden.py
It compiles (oracle/build.py) and calls the reference's unchanged host sources
(src/gpu/src/krylov_openmp.cpp, krylov_kernels.inc, device_solver.cpp, dispatch.cpp) through
oracle/ref_shim.cpp, with one OpenMP thread so every reduction is the serial loop, and stores
inputs and outputs as .npz files beside this script. The hierarchies handed to the reference
solver come from the C restatement of AmgPreconditioner::setup (amg.cpp needs Eigen, which is
not available); meshes come from the product's synthetic generator.
"""
from __future__ import annotations

import os
import sys

os.environ["OMP_NUM_THREADS"] = "1"
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

import oracle as O  # noqa: E402
from cfd_b200 import workloads as W  # noqa: E402


def hier_arrays(prefix, h):
    out = {f"{prefix}levels": np.array(h.levels)}
    for l in range(h.levels):
        for nm, m in (("a", h.a[l]), ("p", h.p[l] if l + 1 < h.levels else None),
                      ("r", h.r[l] if l + 1 < h.levels else None)):
            if m is None:
                continue
            out[f"{prefix}{nm}{l}_shape"] = np.array([m.n_rows, m.n_cols])
            out[f"{prefix}{nm}{l}_rp"] = m.rp
            out[f"{prefix}{nm}{l}_ci"] = m.ci
            out[f"{prefix}{nm}{l}_va"] = m.va
        if l + 1 < h.levels:
            out[f"{prefix}agg{l}"] = h.aggregates[l]
    out[f"{prefix}coarse_inverse"] = h.coarse_inverse
    return out


def main():
    assert O.ref() is not None, "reference host library not available"
    assert O.ref().ref_backend_is_host() == 1
    cases = {"cavity8": W.cavity(8), "graded8": W.graded(8), "tet5": W.tet(5)}
    for name, case in cases.items():
        d = {"n": np.array(case.n), "owner": case.owner, "neighbour": case.neighbour,
             "flux": case.flux, "gamma": case.gamma, "delta": case.delta,
             "source0": case.source0}
        # assembly (reference assemble_convection_diffusion host loop), convection 0 and 1
        for conv in (0.0, 1.0):
            up, lo, dg, dv = O.ref_assemble(case.n, case.owner, case.neighbour, case.flux,
                                            case.gamma, case.delta, conv,
                                            diag=np.full(case.n, 0.5), div=np.zeros(case.n))
            tag = f"c{int(conv)}"
            d[f"asm_{tag}_upper"], d[f"asm_{tag}_lower"] = up, lo
            d[f"asm_{tag}_diag"], d[f"asm_{tag}_div"] = dg, dv
        up, lo, dg, dv = O.ref_assemble(case.n, case.owner, case.neighbour, case.flux, case.gamma,
                                        case.delta, 0.0)
        diag, src = case.finalize(up, lo, dg, dv)
        pat = O.build_pattern(case.n, case.owner, case.neighbour)
        d.update({"pat_rp": pat.row_ptr, "pat_col": pat.col, "pat_diag": pat.diag_pos,
                  "pat_upper": pat.upper_pos, "pat_lower": pat.lower_pos,
                  "ldu_diag": diag, "ldu_upper": up, "ldu_lower": lo, "rhs": src})
        a = O.ldu_to_csr(pat, diag, up, lo)
        h = O.Hierarchy(a)
        d.update(hier_arrays("h_", h))
        tol = 1e-10 * np.linalg.norm(src)
        x, st = O.ref_amg_cg(h.a, h.p, h.r, h.coarse_inverse, src, abs_tol=tol,
                             max_iterations=500)
        d["amgcg_x"], d["amgcg_iters"], d["amgcg_res"] = x, np.array(st["iterations"]), np.array(st["residual"])
        # The reference exposes no V-cycle entry: its V-cycle is pinned through the whole
        # AMG-PCG trajectory above (every iterate depends on every preconditioner application).
        assert h.levels > 1  # the reference solver needs a coarse level (ldu_matrix.cpp:358)
        x, st = O.ref_device_solver(pat, h, diag, up, lo, src, abs_tol=tol, max_iterations=500)
        d["ds_x"], d["ds_iters"] = x, np.array(st["iterations"])
        for meth in (0, 1):
            x, st = O.ref_krylov(a, src, method=meth, abs_tol=tol, max_iterations=5000)
            d[f"kry{meth}_x"], d[f"kry{meth}_iters"] = x, np.array(st["iterations"])
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **d)
        print(name, case.n, "levels", h.levels, "amg-cg iters", int(d["amgcg_iters"]))


if __name__ == "__main__":
    main()
