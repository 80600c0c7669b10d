"""The reference's own FlowSolver (flow_solver.cpp, unchanged) compiled against
include/cfd_gpu_krylov.hpp + include/cfd_gpu_fv.hpp and linked with libcfdb.so
(tests/cpp/test_dropin_flow.cpp, built by oracle/build.py into oracle/_ref/dropin_flow): SIMPLE
iterations with "solver": {"device": "gpu"}, every accelerator call in the product. On the GPU
its residual history and final fields are compared with the same FlowSolver built against the
reference's own host path (oracle/_ref, FlowSolver with the same settings): both solve every
linear system to a normalised residual of 1e-12, so they agree to solver precision, not bit for
bit (the GPU reductions sum in another order)."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "dropin_flow")

pytestmark = pytest.mark.skipif(not os.path.exists(EXE), reason="drop-in program not built (needs the reference)")

BOX = (12, 10, 8, 1.5)  # cells per direction, grading along x
ITERATIONS = 5


def _run(tmp_path, box=BOX, iterations=ITERATIONS):
    out = tmp_path / "fields.bin"
    r = subprocess.run([EXE, *map(str, box), str(iterations), str(out)], capture_output=True, text=True, timeout=600)
    return r.returncode, [json.loads(line) for line in r.stdout.splitlines() if line.startswith("{")], out


def test_links_the_flow_solver_to_the_product_library():
    out = subprocess.run(["ldd", EXE], capture_output=True, text=True).stdout
    line = next(ln for ln in out.splitlines() if "libcfdb.so" in ln)
    assert os.path.realpath(os.path.join(ROOT, "cfd_b200", "libcfdb.so")) in os.path.realpath(
        line.split("=>")[1].split("(")[0].strip())
    und = subprocess.run(["nm", "-C", "--undefined-only", EXE], capture_output=True, text=True).stdout
    for sym in ("cfd::gpu::DeviceSolver::solve", "cfd::gpu::assemble_convection_diffusion",
                "cfd::gpu::DeviceFv::DeviceFv", "cfd::gpu::DeviceFv::gradient", "cfd::gpu::DeviceFv::vector_gradient",
                "cfd::gpu::DeviceFv::momentum_corrections"):
        assert sym in und, sym
    defined = subprocess.run(["nm", "-C", "--defined-only", EXE], capture_output=True, text=True).stdout
    assert "cfd::fv::FlowSolver::simple_iteration" in defined


def test_flow_solver_fails_loudly_without_a_device(cb, tmp_path):
    if cb.device_available():
        pytest.skip("a CUDA device is present")
    rc, lines, _ = _run(tmp_path, (4, 3, 2, 1.0), 1)
    assert rc == 2 and "no host fallback" in lines[-1]["error"]


@pytest.mark.gpu
def test_reference_flow_solver_on_the_gpu_path(gpu, tmp_path):
    RX = pytest.importorskip("oracle.reference")
    if not RX.available() or not hasattr(RX.lib(), "refx_flow_simple_iteration"):
        pytest.skip("reference build with FlowSolver not available")
    rc, lines, out = _run(tmp_path)
    assert rc == 0, lines
    head, hist = lines[0], lines[1:]
    nx, ny, nz, gx = BOX
    assert head["backend"] == "cuda" and head["device_available"] and head["cells"] == nx * ny * nz
    assert len(hist) == ITERATIONS
    # the same FlowSolver on the reference's own host path
    mesh = RX.RefMesh.box(nx, ny, nz, (gx, 1.0, 1.0))
    patches = [("VelocityInlet", (1.0, 0.0, 0.0), 0.0), ("PressureOutlet", (0.0, 0.0, 0.0), 0.25),
               ("Wall", (0.0, 0.0, 0.0), 0.0), ("Wall", (0.3, 0.0, 0.0), 0.0),
               ("Symmetry", (0.0, 0.0, 0.0), 0.0), ("Wall", (0.0, 0.0, 0.0), 0.0)]
    fl = RX.RefFlow(mesh, patches, nu=0.01, p_solver=("GpuCg", 1e-12, 0.0, 2000),
                    u_solver=("GpuBiCgStab", 1e-12, 0.0, 2000))
    for h in hist:
        ru, rp, rc_ = fl.simple_iteration()
        assert np.allclose(h["u"], ru, rtol=1e-6, atol=1e-10)
        assert abs(h["p"] - rp) <= 1e-6 * abs(rp)
        # mass is conserved to the pressure solve's tolerance on both paths
        assert h["continuity"] <= 1e-9 and rc_ <= 1e-9
    u, p, phi = fl.state()
    n, nf = mesh.n_cells, mesh.n_faces
    got = np.fromfile(out, dtype=np.float64)
    assert got.size == 3 * n + n + nf
    gu, gp, gphi = got[:3 * n].reshape(n, 3), got[3 * n:4 * n], got[4 * n:]
    rel = lambda a, b: np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b))  # noqa: E731
    assert rel(gu, u) <= 1e-8 and rel(gp, p) <= 1e-8 and rel(gphi, phi) <= 1e-8
    fl.close()
