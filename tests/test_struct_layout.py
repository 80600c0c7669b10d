"""Every ctypes mirror of a C-ABI struct has the C compiler's layout: a small C program built
against include/ prints sizeof and every field's offset, and the Python structs must agree
(a mismatch would pass wrong values through the library's entry points silently)."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

import cfd_b200 as cb
from cfd_b200 import fv_device, pressure, scalar, serving

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

MIRRORS = [
    ("cfdb_csr", cb.CsrStruct), ("cfdb_amg_level", cb.AmgLevelStruct), ("cfdb_amg_view", cb.AmgViewStruct),
    ("cfdb_control", cb.ControlStruct), ("cfdb_stats", cb.StatsStruct), ("cfdb_ldu_pattern", cb.PatternStruct),
    ("cfdb_kernel_record", cb.KernelRecordStruct), ("cfdb_ldu_settings", cb.LduSettingsStruct),
    ("cfdb_ldu_result", cb.LduResultStruct), ("cfdb_amg_settings", cb.AmgSettingsStruct),
    ("cfdb_tuning", cb.TuningStruct), ("cfdb_fv_mesh_view", fv_device.FvMeshViewStruct),
    ("cfdb_pressure_settings", pressure.PressureSettingsStruct),
    ("cfdb_pressure_workspace", pressure.PressureWorkspaceStruct),
    ("cfdb_scalar_equation", scalar.ScalarEquationStruct),
    ("cfdb_server_config", serving.ServerConfigStruct), ("cfdb_server_info_t", serving.ServerInfoStruct),
]


def _c_layout(tmp_path):
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "cfdb.h"', '#include "cfdb_serve.h"',
             "int main(void) {"]
    for cname, py in MIRRORS:
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'    printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, timeout=120)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True, timeout=60).stdout
    layout = {}
    for line in out.splitlines():
        cname, key, value = line.split()
        layout[(cname, key)] = int(value)
    return layout


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_ctypes_mirrors_match_the_c_layout(tmp_path):
    layout = _c_layout(tmp_path)
    for cname, py in MIRRORS:
        assert C.sizeof(py) == layout[(cname, "size")], cname
        for fname, _ in py._fields_:
            assert getattr(py, fname).offset == layout[(cname, fname)], f"{cname}.{fname}"
