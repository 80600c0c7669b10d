"""The cfd::gpu C++ front end (include/cfd_gpu_krylov.hpp over libcfdb.so), driven by a C++
program written like the reference's accelerator tests (tests/cpp/test_cfd_gpu_api.cpp)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    import cfd_b200  # noqa: F401  (builds / loads libcfdb.so)
    exe = str(tmp_path / "test_cfd_gpu_api")
    lib = os.path.join(ROOT, "cfd_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "test_cfd_gpu_api.cpp"), "-L", lib, "-lcfdb",
                    f"-Wl,-rpath,{lib}", "-o", exe], check=True, capture_output=True, text=True)
    return exe


def test_cxx_front_end_without_device(tmp_path):
    import cfd_b200 as cb
    if cb.device_available():
        pytest.skip("a GPU is present: the device checks run in the gpu test")
    r = subprocess.run([_build(tmp_path), "--no-device"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_cxx_front_end_on_device(tmp_path):
    r = subprocess.run([_build(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all checks passed" in r.stdout
