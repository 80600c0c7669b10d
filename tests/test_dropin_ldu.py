"""The reference's own callers of cfd::gpu (LduMatrix::solve -> solve_persistent, the one-shot
AMG-CG branch, the host BiCGStab path, FlowSolver's assembly call), compiled unchanged against
include/cfd_gpu_krylov.hpp + include/cfd_gpu_fv.hpp and linked with libcfdb.so and the
reference's own krylov_openmp.cpp (tests/cpp/test_dropin_ldu.cpp, built by oracle/build.py
into oracle/_ref/dropin_ldu). This is the INTEGRATION.md option A build, linked and run."""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "dropin_ldu")

pytestmark = pytest.mark.skipif(not os.path.exists(EXE), reason="drop-in program not built (needs the reference)")


def _run(n):
    r = subprocess.run([EXE, str(n)], capture_output=True, text=True, timeout=600)
    return r.returncode, [json.loads(line) for line in r.stdout.splitlines() if line.startswith("{")]


def test_links_against_the_product_library():
    out = subprocess.run(["ldd", EXE], capture_output=True, text=True).stdout
    line = next(ln for ln in out.splitlines() if "libcfdb.so" in ln)
    assert os.path.realpath(os.path.join(ROOT, "cfd_b200", "libcfdb.so")) in os.path.realpath(
        line.split("=>")[1].split("(")[0].strip())
    # the reference's callers bind the product's DeviceSolver and its host path binds solve_host
    und = subprocess.run(["nm", "-C", "--undefined-only", EXE], capture_output=True, text=True).stdout
    for sym in ("cfd::gpu::DeviceSolver::DeviceSolver", "cfd::gpu::DeviceSolver::set_amg",
                "cfd::gpu::DeviceSolver::solve", "cfd::gpu::solve_amg_cg", "cfd::gpu::assemble_convection_diffusion",
                "cfd::gpu::backend_name"):
        assert sym in und, sym
    defined = subprocess.run(["nm", "-C", "--defined-only", EXE], capture_output=True, text=True).stdout
    assert "cfd::gpu::solve_host" in defined and "cfd::gpu::detail::solve_amg_openmp" in defined


def test_fails_loudly_without_a_device(cb):
    if cb.device_available():
        pytest.skip("a CUDA device is present")
    rc, lines = _run(4)
    assert rc == 2 and "no host fallback" in lines[-1]["error"]


@pytest.mark.gpu
def test_reference_callers_run_the_gpu_path(gpu):
    RX = pytest.importorskip("oracle.reference")
    n = 16
    rc, lines = _run(n)
    assert rc == 0, lines
    head, runs = lines[0], {}
    for ln in lines[1:]:
        runs.setdefault(ln["path"], []).append(ln)
    assert head["backend"] == "cuda" and head["device_available"] and head["cells"] == n ** 3
    gpu_cg = runs["GpuCg"]
    assert [r["amg_age"] for r in gpu_cg] == [1, 2, 1]
    for r in gpu_cg + runs["GpuCg_one_shot"] + runs["GpuBiCgStab"] + runs["BiCgStab_host"]:
        assert r["true_rel_residual"] <= 1.05e-8, r
    # the same system through the reference's own host DeviceSolver (oracle/_ref)
    if not RX.available():
        pytest.skip("reference build with the Eigen stand-in not available")
    mesh = RX.RefMesh.box(n, n, n)
    delta, _, _ = mesh.fv()
    nif = mesh.n_internal_faces
    f = np.arange(nif, dtype=np.int64)
    flux = ((f * 7919) % 1000).astype(np.float64) / 500.0 - 1.0
    gamma = 1.0 + 0.125 * (f % 7).astype(np.float64)
    up, lo, dg, dv = O.ref_assemble(mesh.n_cells, mesh.owner, mesh.neighbour, flux, gamma, delta[:nif], 0.0)
    ldu = RX.RefLdu(mesh)
    ldu.set(dg, up, lo, 0.0 - dv)
    ldu.set_reference(0, 0.0)
    x = np.zeros(mesh.n_cells)
    ref = ldu.solve(x, "GpuCg", tolerance=0.0, rel_tolerance=1e-8, max_iterations=500, max_age=2)
    assert abs(gpu_cg[0]["iterations"] - ref["iterations"]) <= 1
    assert gpu_cg[0]["initial"] == pytest.approx(ref["initial_residual"], rel=1e-12)
    assert gpu_cg[0]["x_sum"] == pytest.approx(float(x.sum()), rel=1e-6, abs=1e-6 * np.abs(x).sum())
