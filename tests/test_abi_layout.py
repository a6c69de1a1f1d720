"""The Python mirror's ctypes structures have the C-ABI's layout: the size of each struct of
include/neon_b200.h and the offset of every field, read from a small C program compiled with
the host compiler against the header (no GPU)."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from neon_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# C struct name -> ctypes mirror
MIRRORS = {
    "nb2_mesh_desc": api.MeshDesc,
    "nb2_material": api.MaterialDesc,
    "nb2_dof_table": api.DofTableDesc,
    "nb2_solver_options": api.SolverOptions,
    "nb2_solve_report": api.SolveReport,
    "nb2_newton_log": api.NewtonLog,
}


def _c_layout(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "neon_b200.h"',
             "int main(void) {"]
    for name, mirror in MIRRORS.items():
        lines.append(f'    printf("{name} size %zu\\n", sizeof({name}));')
        for field, _ in mirror._fields_:
            lines.append(f'    printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    layout = {}
    for line in out.splitlines():
        struct, key, value = line.split()
        layout[(struct, key)] = int(value)
    return layout


def test_ctypes_structs_match_the_header(tmp_path):
    layout = _c_layout(tmp_path)
    for name, mirror in MIRRORS.items():
        assert C.sizeof(mirror) == layout[(name, "size")], name
        for field, _ in mirror._fields_:
            assert getattr(mirror, field).offset == layout[(name, field)], (name, field)
