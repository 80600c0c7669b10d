"""Host-side argument checks of the allocation-free entry point (cfdb_solve_device_noalloc):
the pointer rule of the C library (compiled and run as a host program) and the Python
wrapper's dtype / layout / length checks, which reject a bad array before any launch."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_pointer_rule(tmp_path):
    exe = str(tmp_path / "test_pointer_rule")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "cfd_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "test_pointer_rule.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    assert r.stdout.strip() == "ok"


def test_wrapper_rejects_wrong_dtypes_before_any_launch(cb):
    import torch
    n = 4
    rp64 = torch.as_tensor(np.arange(n + 1, dtype=np.int64))  # int64: the kernels read int32
    ci = torch.zeros(n, dtype=torch.int32)
    va = torch.ones(n, dtype=torch.float64)
    b = torch.ones(n, dtype=torch.float64)
    x = torch.zeros(n, dtype=torch.float64)
    with pytest.raises(cb.InvalidArgument, match="row_ptr must be torch.int32"):
        cb.solve_device_noalloc(n, n, rp64, ci, va, b, x, cb.Method.Cg, cb.SolveControl())
    rp = rp64.to(torch.int32)
    with pytest.raises(cb.InvalidArgument, match="val must be torch.float64"):
        cb.solve_device_noalloc(n, n, rp, ci, va.float(), b, x, cb.Method.Cg, cb.SolveControl())
    with pytest.raises(cb.InvalidArgument, match="contiguous"):
        cb.solve_device_noalloc(n, n, rp, ci, va, torch.ones(2 * n, dtype=torch.float64)[::2], x,
                                cb.Method.Cg, cb.SolveControl())
    with pytest.raises(cb.InvalidArgument, match="current CUDA device"):
        cb.solve_device_noalloc(n, n, rp, ci, va, b, x, cb.Method.Cg, cb.SolveControl())
