"""The C-ABI library loads and exports every entry point the header declares."""
import ctypes
import os
import subprocess
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu

HEADER = os.path.join(ROOT, "include", "lbfs_b200.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^int\s+(lbfs_\w+)\s*\(", src, re.M)))


def test_header_declares_the_entry_points():
    names = declared()
    assert "lbfs_create" in names and "lbfs_step" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    from lbfs_b200 import _abi
    lib = ctypes.CDLL(_abi.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(declared()) == set(_abi.EXPORTED)


def test_structs_match_header_sizes():
    # sizes of the descriptors as a C compiler lays them out (64-bit)
    from lbfs_b200 import _abi
    assert ctypes.sizeof(_abi.MeshDesc) == 8 * 4 + 14 * 8 + 8 * 8 + 8 + 8 + 3 * 8 + 8  # ... periodic_node
    assert ctypes.sizeof(_abi.GridDesc) == 8 + 8 * 8
    assert ctypes.sizeof(_abi.Params) == 4 * 8 + 3 * 8 + 4 * 8 + 4 * 4 + 8 + 8 + 8  # time stepping, gamma, precond.
    assert ctypes.sizeof(_abi.RbcDesc) == 16 + 4 * 8 + 13 * 8 + 8 + 8  # ... instance, periodic


def test_struct_layout_matches_c_compiler(tmp_path):
    # every field offset of the ctypes mirrors equals the C compiler's offsetof
    from lbfs_b200 import _abi
    structs = {"lbfs_mesh_desc": _abi.MeshDesc, "lbfs_grid_desc": _abi.GridDesc, "lbfs_params": _abi.Params,
               "lbfs_rbc_desc": _abi.RbcDesc, "lbfs_launch_shape": _abi.LaunchShape}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "lbfs_b200.h"', 'int main(void) {']
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            lines.append(f'printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {(a, b): int(c) for a, b, c in (l.split() for l in out if l)}
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for f in py._fields_:
            assert got[(cname, f[0])] == getattr(py, f[0]).offset, (cname, f[0])


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU error path")
def test_create_fails_loudly_without_gpu():
    from lbfs_b200 import GpuSolver, LbfsError, StepParams, build_uniform_mesh
    m = build_uniform_mesh(8.0, 8.0, 8.0, 1.0)
    m.set_boundaries({p: (2, 2, 1.0, 0.0, 0.0, 0.0) for p in ("left", "right", "bottom", "top", "back", "front")})
    with pytest.raises(LbfsError) as e:
        GpuSolver(m, StepParams(visc=0.1))
    assert e.value.code == 2  # LBFS_ERR_CUDA: there is no CPU path


def test_argument_errors_are_status_codes():
    from lbfs_b200 import _abi
    out = (ctypes.c_int32 * 8)()
    assert _abi.lib().lbfs_mesh_uniform_counts(-1.0, 8.0, 8.0, 1.0, out) == _abi.LBFS_ERR_ARG
    tris = np.array([[0, 1, 2]], np.int32)
    spr = np.zeros((3, 4), np.int32)
    n = ctypes.c_int32()
    rc = _abi.lib().lbfs_rbc_build_springs(3, 1, _abi.iptr(tris), 3, _abi.iptr(spr), ctypes.byref(n))
    assert rc == _abi.LBFS_ERR_ARG  # an open triangle is not a closed membrane
