"""Builds the cfdb shared library in-tree (``cfd_b200/libcfdb.so``) for sm_100a only.

CUDA sources are compiled with ``-gencode arch=compute_100a,code=sm_100a`` and without FMA
contraction (``--fmad=false``): the FP64 kernels round every product and sum separately, as the
reference's host path does; FP32 kernels request fused multiply-adds explicitly (fmaf).
Run ``python -m cfd_b200.build`` or call :func:`build`.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcfdb.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-fopenmp",
              "-I", os.path.join(ROOT, "include"), "-I", CSRC]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off",
             "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-I", "/usr/local/cuda/include"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu"))), sorted(glob.glob(os.path.join(CSRC, "*.cpp")))


def _deps():
    return (glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
            + glob.glob(os.path.join(ROOT, "include", "*.hpp")) + [os.path.abspath(__file__)])


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r


def build(force: bool = False, verbose: bool = False) -> str:
    cu, cpp = _sources()
    if not force and not _stale(LIB, _deps()):
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    objs = []
    hdr = [d for d in _deps() if d.endswith((".h", ".hpp", ".cuh"))]
    for src in cu:
        o = os.path.join(OBJ, os.path.basename(src) + ".o")
        if force or _stale(o, [src] + hdr):
            cmd = [NVCC, *ARCH, *NVCC_FLAGS]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            cmd += ["-c", src, "-o", o]
            r = _run(cmd)
            if verbose:
                sys.stderr.write(r.stderr)
        objs.append(o)
    for src in cpp:
        o = os.path.join(OBJ, os.path.basename(src) + ".o")
        if force or _stale(o, [src] + hdr):
            _run(["g++", *CXX_FLAGS, "-c", src, "-o", o])
        objs.append(o)
    tmp = LIB + f".tmp{os.getpid()}"
    _run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-Xcompiler", "-fopenmp", "-lgomp"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
