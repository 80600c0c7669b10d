"""The C ABI library: loads without a GPU, exports every entry point declared in include/*.h,
reports its backend, and fails loudly (no CPU fallback) when no device is present."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(cfdb_\w+)\s*\(", text))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared_symbols()
    assert "cfdb_system_solve" in names and "cfdb_assemble" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol(cb):
    lib = ctypes.CDLL(cb.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_backend_queries(cb):
    assert cb.backend_name() == "cuda"
    assert cb.device_description().startswith("cuda")


@pytest.mark.skipif(__import__("cfd_b200").device_available(), reason="a GPU is present")
def test_no_device_fails_loudly(cb):
    n = 4
    own, nei = np.array([0, 1, 2], np.int32), np.array([1, 2, 3], np.int32)
    up, lo, dg, dv = np.zeros(3), np.zeros(3), np.zeros(n), np.zeros(n)
    with pytest.raises(cb.NoDevice):
        cb.assemble_convection_diffusion(n, 3, own, nei, np.zeros(3), np.ones(3), np.ones(3), 0.0,
                                         up, lo, dg, dv)
    pat = cb.build_csr_pattern(n, own, nei)  # host-side work needs no device
    assert pat.nnz == n + 6
    with pytest.raises(cb.NoDevice):
        cb.DeviceSolver(pat)


def test_argument_errors_before_device_work(cb):
    with pytest.raises(cb.InvalidArgument):
        cb.assemble_convection_diffusion(4, 3, [0, 1, 2], [1, 2, 3], np.zeros(3), np.ones(3),
                                         np.ones(3), 0.0, [0.0] * 3, np.zeros(3), np.zeros(4),
                                         np.zeros(4))


def test_device_array_wrappers_wait_for_torch_first(cb):
    """The library's kernels run on its own streams, so every Python entry point that takes CUDA
    tensors first drains torch's current stream (zero fills and copies queued there must not
    land on a buffer the library is writing)."""
    from cfd_b200 import fv_device, scalar
    owners = [cb.DeviceSolver, cb.Batch, cb.FvGeometry, fv_device.DeviceFv]
    getters = {"delta_device", "device_bytes", "on_device"}
    checked = []
    for cls in owners:
        for name, fn in vars(cls).items():
            if name.endswith("_device") and name not in getters and callable(fn):
                assert hasattr(fn, "__wrapped__"), f"{cls.__name__}.{name} is not stream-ordered"
                checked.append(name)
    for fn in (cb.assemble_convection_diffusion_device, cb.solve_device_noalloc, scalar.scalar_system_device):
        assert hasattr(fn, "__wrapped__"), fn.__name__
    assert len(checked) >= 18
