"""Uniform meshes: the coded least-squares weights and the per-axis face geometry.

On the generator's uniform meshes every cell's least-squares weight vectors are six axis vectors
in a per-cell order, and every interior face of an axis has the same geometry.  The library checks
both bit for bit at create and then reads 3-bit codes into a parameter table (gradients, adjoint)
and the per-axis geometry from the kernel parameters (interior faces, their adjoint) instead of the
per-cell and per-face arrays.  With LBFS_GENERIC_GEOMETRY set it reads the arrays: the results must
agree bit for bit.
"""
import numpy as np
import pytest


def _run(c, steps, monkeypatch, generic, adjoint=False):
    from lbfs_b200 import GpuSolver
    if generic:
        monkeypatch.setenv("LBFS_GENERIC_GEOMETRY", "1")
    else:
        monkeypatch.delenv("LBFS_GENERIC_GEOMETRY", raising=False)
    with GpuSolver(c.mesh, c.params, c.membranes) as s:
        s.set_state(c.rho, c.u, c.v, c.w)
        if adjoint:
            J, g, _ = s.adjoint(steps, 4, membrane=0)
            return J, g
        s.step(steps, graph=True)
        return s.state(), s.nodes(), s.residuals(), s.status()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_coded_geometry_equals_generic(precision, monkeypatch):
    from lbfs_b200 import cases
    c = cases.shear_rbc(n=16, level=2, radius_cells=3.0, precision=precision)
    coded = _run(c, 6, monkeypatch, False)
    generic = _run(c, 6, monkeypatch, True)
    for a, b in zip(coded[0], generic[0]):
        assert np.array_equal(a, b)
    assert np.array_equal(coded[1], generic[1])
    assert np.array_equal(coded[2], generic[2])
    assert coded[3] == 0 and generic[3] == 0


@pytest.mark.gpu
def test_coded_geometry_adjoint_equals_generic(monkeypatch):
    import dataclasses
    from lbfs_b200 import cases
    c = cases.shear_rbc(n=16, level=2, radius_cells=3.0)
    c.membranes = [dataclasses.replace(m, internal_viscosity_ratio=1.0) for m in c.membranes]
    assert _run(c, 12, monkeypatch, False, adjoint=True) == _run(c, 12, monkeypatch, True, adjoint=True)


def test_generator_mesh_is_uniform():
    """CPU: the bench's byte counts assume the coded forms on the uniform generator's mesh and not
    on a jittered one (the same checks as the library's)."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from lbfs_b200 import cases
    c = cases.shear_rbc(n=12, level=1, radius_cells=2.0)
    assert bench.axis_geometry_uniform(c.mesh) and bench.ls_weights_coded(c.mesh)
    j = cases.jittered_channel(n=8)
    assert not bench.axis_geometry_uniform(j.mesh) and not bench.ls_weights_coded(j.mesh)


def test_cell_update_closed_form_faces():
    """CPU: the bench counts K3's face list only where the library reads it.  The uniform
    generator's mesh matches the closed-form face list entry for entry; a jittered mesh (not axis
    aligned) and a uniform mesh whose table no longer matches (one interior face with owner and
    neighbour swapped) do not, and then the 24 B per cell of the list are counted."""
    import copy
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from lbfs_b200 import cases
    c = cases.shear_rbc(n=12, level=1, radius_cells=2.0)
    faces, _ = bench.cell_update_closed_forms(c.mesh)
    assert faces
    nc = c.mesh.n_cells
    full = bench.algorithmic_bytes(c.mesh, "update")
    assert full == nc * (8 + 64 + 32) + c.mesh.n_faces * 32 or full == nc * (64 + 32) + c.mesh.n_faces * 32
    j = cases.jittered_channel(n=8)
    assert not bench.cell_update_closed_forms(j.mesh)[0]
    m = copy.copy(c.mesh)
    m.owner, m.neighbour = np.array(c.mesh.owner, copy=True), np.array(c.mesh.neighbour, copy=True)
    f = c.mesh.n_face_x // 2
    m.owner[f], m.neighbour[f] = c.mesh.neighbour[f], c.mesh.owner[f]
    assert not bench.cell_update_closed_forms(m)[0]
    assert bench.algorithmic_bytes(m, "update") == full + 24 * nc
