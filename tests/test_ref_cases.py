"""The reference arm's workload (oracle/ref_cases.py, built from the reference's
own generator and numpy only) is the benchmark workload: the same mesh,
boundary tables, initial state and red cell as lbfs_b200.cases.shear_rbc with
the reference's 2-point stencil, so both arms step the same inputs."""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN
from lbfs_b200 import _abi, cases

sys.path.insert(0, GOLDEN)
import ref_lbfs as R  # noqa: E402

pytestmark = pytest.mark.skipif(not R.available(), reason="oracle/_ref/libref_lbfs.so not built")


def test_reference_arm_inputs_equal_the_workload():
    import ref_cases
    from make_golden import ref_case
    n = 24
    rc, n_cells, n_nodes = ref_cases.shear_rbc(n=n, radius_cells=4.0)
    c = cases.shear_rbc(n=n, radius_cells=4.0, ibm_stencil=_abi.LBFS_IBM_HAT2)
    assert n_cells == c.mesh.n_cells and n_nodes == c.membranes[0].n_nodes
    # boundary tables
    mesh = R.RefMesh(c.mesh.X, c.mesh.Y, c.mesh.Z, c.mesh.dt, c.mesh.origin, c.params.visc)
    rt, vt, vals = ref_cases.boundary_tables(mesh.arrays(), mesh.n_interior, c.bcs)
    assert np.array_equal(rt, c.mesh.bc_rho_type) and np.array_equal(vt, c.mesh.bc_vel_type)
    assert np.array_equal(vals, c.mesh.bc_values)
    # red cell
    # red cell of the 64^3 workload (radius 8 cells = 16 length units, at the centre)
    tris, springs, sphere, initial = ref_cases.red_cell_l3(16.0, (64.0, 64.0, 64.0))
    m3 = cases.shear_rbc(n=64, ibm_stencil=_abi.LBFS_IBM_HAT2).membranes[0]
    assert np.array_equal(tris, m3.tris) and np.array_equal(springs, m3.springs)
    assert np.array_equal(sphere, m3.xyz_stress_free) and np.array_equal(initial, m3.xyz_initial)
    # the whole case: same states after stepping both
    ref = ref_case(c)
    rc.step(3)
    ref.step(3)
    for a, b in zip(rc.state(), ref.state()):
        assert np.array_equal(a, b)
    assert np.array_equal(rc.get(R.REF_NODE_X), ref.get(R.REF_NODE_X))
    rc.close()
    ref.close()
