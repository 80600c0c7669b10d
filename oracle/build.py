"""Build recipe for the CPU oracle (test infrastructure only).

* ``oracle/_build/liboracle.so``: the C restatement in ``oracle/oracle.c`` (gcc, no FMA
  contraction so roundings match the reference's x86-64 host build).
* ``oracle/_ref/libcfdref.so``: the reference's own host sources, compiled unchanged where
  they lie under the reference checkout (the Eigen-dependent ones against
  ``oracle/eigen_standin``), plus the shims ``oracle/ref_shim.cpp``,
  ``oracle/ref_eigen_shim.cpp`` and ``oracle/ref_flow_shim.cpp``. Only built when the
  reference checkout is present; the built library is git-ignored and travels with the tree.

Run ``python -m oracle.build`` (or call :func:`build_all`).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
REF_DIR = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(BUILD_DIR, "liboracle.so")
REF_SO = os.path.join(REF_DIR, "libcfdref.so")

# The reference checkout: CFD_REFERENCE_ROOT, else a directory named "reference" beside the
# repository (read-only; only this recipe reads it).
REFERENCE_ROOT = os.environ.get(
    "CFD_REFERENCE_ROOT", os.path.normpath(os.path.join(HERE, os.pardir, os.pardir, "reference")))
REF_SOURCES = [
    "src/gpu/src/krylov_openmp.cpp",
    "src/gpu/src/device_solver.cpp",
    "src/gpu/src/dispatch.cpp",
    "src/gpu/src/fv_openmp.cpp",
    "src/gpu/src/fv_device.cpp",
]
# Eigen-dependent sources, compiled unchanged against the Eigen stand-in (oracle/eigen_standin).
REF_EIGEN_SOURCES = [
    "src/mesh/src/mesh.cpp",
    "src/mesh/src/mesh_builder.cpp",
    "src/mesh/src/box_mesher.cpp",
    "src/fv/src/fv_geometry.cpp",
    "src/fv/src/ldu_matrix.cpp",
    "src/fv/src/amg.cpp",
    "src/fv/src/parallel_amg.cpp",
    "src/parallel/src/comm.cpp",
]
# FlowSolver (the callers of the pressure path) and the scalar transport step, in the
# reference build only (the drop-in program links flow_solver.cpp alone)
REF_FLOW_SOURCES = ["src/fv/src/flow_solver.cpp", "src/fv/src/scalar_transport.cpp"]
REF_INCLUDES = ["src/gpu/include", "src/core/include", "src/mesh/include", "src/fv/include",
                "src/parallel/include"]


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "oracle.c")
    hdr = os.path.join(HERE, "oracle.h")
    if force or _stale(ORACLE_SO, [src, hdr]):
        os.makedirs(BUILD_DIR, exist_ok=True)
        tmp = ORACLE_SO + f".tmp{os.getpid()}"
        cmd = ["gcc", "-std=c11", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
               "-shared", src, "-o", tmp, "-lm"]
        subprocess.run(cmd, check=True)
        os.replace(tmp, ORACLE_SO)
    return ORACLE_SO


def reference_available() -> bool:
    return all(os.path.exists(os.path.join(REFERENCE_ROOT, s))
               for s in REF_SOURCES + REF_EIGEN_SOURCES + REF_FLOW_SOURCES)


def build_ref(force: bool = False) -> str | None:
    """Compile the reference's host path (unchanged sources) + our shim into oracle/_ref."""
    if not reference_available():
        return REF_SO if os.path.exists(REF_SO) else None
    srcs = [os.path.join(REFERENCE_ROOT, s) for s in REF_SOURCES + REF_EIGEN_SOURCES + REF_FLOW_SOURCES]
    shims = [os.path.join(HERE, "ref_shim.cpp"), os.path.join(HERE, "ref_eigen_shim.cpp"),
             os.path.join(HERE, "ref_flow_shim.cpp")]
    standin = os.path.join(HERE, "eigen_standin")
    deps = srcs + shims + [os.path.join(REFERENCE_ROOT, "src/gpu/src/krylov_kernels.inc"),
                           os.path.join(REFERENCE_ROOT, "src/gpu/src/fv_cell.inc"),
                           os.path.join(REFERENCE_ROOT, "src/gpu/src/fv_impl.hpp")]
    for inc in REF_INCLUDES:
        for dirpath, _, files in os.walk(os.path.join(REFERENCE_ROOT, inc)):
            deps += [os.path.join(dirpath, f) for f in files]
    deps += [os.path.join(standin, "Eigen", f) for f in os.listdir(os.path.join(standin, "Eigen"))]
    if force or _stale(REF_SO, deps):
        if shutil.which("g++") is None:
            return None
        os.makedirs(REF_DIR, exist_ok=True)
        objdir = os.path.join(REF_DIR, "obj")
        os.makedirs(objdir, exist_ok=True)
        # No -march: plain x86-64 (SSE2, no FMA), so the host path rounds every product and sum
        # separately, as a default build of the reference does.
        flags = ["g++", "-std=c++20", "-O3", "-fopenmp", "-fPIC", "-I", standin]
        for inc in REF_INCLUDES:
            flags += ["-I", os.path.join(REFERENCE_ROOT, inc)]
        from concurrent.futures import ThreadPoolExecutor
        objs = [os.path.join(objdir, f"{i:02d}_{os.path.basename(src)}.o") for i, src in enumerate(srcs + shims)]

        def compile_one(pair):
            src, obj = pair
            subprocess.run(flags + ["-c", src, "-o", obj], check=True)

        with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
            list(ex.map(compile_one, zip(srcs + shims, objs)))
        tmp = REF_SO + f".tmp{os.getpid()}"
        subprocess.run(["g++", "-shared", "-fopenmp", *objs, "-o", tmp], check=True)
        os.replace(tmp, REF_SO)
    return REF_SO


DROPIN_EXE = os.path.join(REF_DIR, "dropin_ldu")
DROPIN_FLOW_EXE = os.path.join(REF_DIR, "dropin_flow")
DROPIN_SOURCES = [s for s in REF_EIGEN_SOURCES] + ["src/gpu/src/krylov_openmp.cpp"]


def build_dropin(force: bool = False) -> str | None:
    """The drop-in programs: tests/cpp/test_dropin_ldu.cpp with the reference's unchanged
    LduMatrix / AMG / mesh / FvGeometry sources and its host path (krylov_openmp.cpp), and
    tests/cpp/test_dropin_flow.cpp with the same sources plus its unchanged flow_solver.cpp,
    compiled against this project's C++ front end (include/cfd_gpu_krylov.hpp and
    include/cfd_gpu_fv.hpp in place of the reference's cfd/gpu headers) and linked with
    libcfdb.so: the reference's callers driving the product. Built where the reference checkout
    and the product library are present; the binaries travel with the tree (rpath to
    cfd_b200/). Returns the LDU program's path."""
    root = os.path.dirname(HERE)
    lib = os.path.join(root, "cfd_b200", "libcfdb.so")
    if not reference_available() or not os.path.exists(lib):
        return DROPIN_EXE if os.path.exists(DROPIN_EXE) else None
    srcs = [os.path.join(REFERENCE_ROOT, s) for s in DROPIN_SOURCES]
    flow_src = os.path.join(REFERENCE_ROOT, REF_FLOW_SOURCES[0])
    tests = {DROPIN_EXE: os.path.join(root, "tests", "cpp", "test_dropin_ldu.cpp"),
             DROPIN_FLOW_EXE: os.path.join(root, "tests", "cpp", "test_dropin_flow.cpp")}
    ours = {"krylov.hpp": os.path.join(root, "include", "cfd_gpu_krylov.hpp"),
            "fv_device.hpp": os.path.join(root, "include", "cfd_gpu_fv.hpp")}
    standin = os.path.join(HERE, "eigen_standin")
    deps = srcs + [flow_src, lib, os.path.join(REFERENCE_ROOT, "src/gpu/src/krylov_kernels.inc")] + list(ours.values())
    deps += list(tests.values())
    deps += [os.path.join(standin, "Eigen", f) for f in os.listdir(os.path.join(standin, "Eigen"))]
    if not (force or any(_stale(exe, deps) for exe in tests)):
        return DROPIN_EXE
    # <cfd/gpu/...> resolves to this project's headers; the other reference headers as they are
    shadow = os.path.join(REF_DIR, "dropin_include", "cfd", "gpu")
    os.makedirs(shadow, exist_ok=True)
    for name, path in ours.items():
        shutil.copyfile(path, os.path.join(shadow, name))
    flags = ["g++", "-std=c++20", "-O2", "-fopenmp", "-fPIC", "-I", os.path.join(REF_DIR, "dropin_include"),
             "-I", standin]
    for inc in REF_INCLUDES:
        if inc != "src/gpu/include":
            flags += ["-I", os.path.join(REFERENCE_ROOT, inc)]
    objdir = os.path.join(REF_DIR, "dropin_obj")
    os.makedirs(objdir, exist_ok=True)
    from concurrent.futures import ThreadPoolExecutor
    units = srcs + [flow_src] + list(tests.values())
    objs = [os.path.join(objdir, f"{i:02d}_{os.path.basename(u)}.o") for i, u in enumerate(units)]

    def compile_one(pair):
        subprocess.run(flags + ["-c", pair[0], "-o", pair[1]], check=True)

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(compile_one, zip(units, objs)))
    common = objs[:len(srcs)]
    flow_obj = objs[len(srcs)]
    test_objs = dict(zip(tests, objs[len(srcs) + 1:]))
    for exe, extra in ((DROPIN_EXE, []), (DROPIN_FLOW_EXE, [flow_obj])):
        tmp = exe + f".tmp{os.getpid()}"
        subprocess.run(["g++", "-fopenmp", *common, *extra, test_objs[exe], "-L", os.path.dirname(lib), "-lcfdb",
                        "-Wl,-rpath,$ORIGIN/../../cfd_b200", "-o", tmp], check=True)
        os.replace(tmp, exe)
    return DROPIN_EXE


def build_all(force: bool = False) -> None:
    build_oracle(force)
    build_ref(force)
    build_dropin(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print(ORACLE_SO)
    print(REF_SO if os.path.exists(REF_SO) else "(reference not built)")
