"""The drop-in C++ shim (gpu_solver::General_Purpose_Solver_mk_i over the C ABI)
compiles against the reference's own headers, where those are present."""
import os
import subprocess

import pytest

from conftest import ROOT

# the reference sources (read-only); LBFS_REFERENCE_DIR overrides the default location
REF = os.environ.get("LBFS_REFERENCE_DIR", "/root/reference")


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "Solver_gpu.h")),
                    reason=f"reference headers absent at {REF} (set LBFS_REFERENCE_DIR)")
def test_drop_in_shim_compiles_against_reference_headers():
    src = os.path.join(ROOT, "lbfs-ibm-ade-sp_b200", "integration", "Solver_gpu_lbfs.cpp")
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-fpermissive", "-w", "-I", os.path.join(ROOT, "oracle", "ref_stub"),
           "-I", REF, "-I", os.path.join(ROOT, "include"), src]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_header_compiles_as_c():
    r = subprocess.run(["gcc", "-std=c99", "-fsyntax-only", "-Wall", "-Werror", "-x", "c", "-I",
                        os.path.join(ROOT, "include"), "-"], input="#include \"lbfs_b200.h\"\n", capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
