"""Jittered hex meshes (the general-normal path of imported meshes).

Interior vertices move by a seeded offset of up to 10 % of the spacing; the
geometry formulas are the uniform builder's (bit-exact against the reference
for zero jitter), the step takes the general-normal flux on every face.
"""
import numpy as np
import pytest

from helpers import FP64_RTOL, rel_err


def _mesh(jitter, seed=5, n=(8, 6, 5)):
    from lbfs_b200 import build_uniform_mesh
    return build_uniform_mesh(2.0 * n[0], 2.0 * n[1], 2.0 * n[2], 1.0, jitter=jitter, seed=seed)


def test_jittered_geometry_is_consistent():
    m, u = _mesh(0.1), _mesh(0.0)
    nc = m.n_cells
    assert not m.axis_aligned and u.axis_aligned
    vol = m.cell_volume[:nc]
    assert np.all(vol > 0)
    # moving interior vertices keeps the box: the cell volumes still sum to it (float vertices)
    assert abs(vol.sum() - 16.0 * 12.0 * 10.0) <= 1e-5 * 16.0 * 12.0 * 10.0
    assert np.allclose(np.linalg.norm(m.face_normal, axis=1), 1.0, atol=1e-12)
    interior = m.face_normal[:m.n_interior]
    assert np.max(np.abs(interior - np.round(interior))) > 1e-3  # normals are general
    # face and cell centroids move by no more than the vertices do (10 % of the 2-unit spacing)
    assert np.max(np.abs(m.face_centroid - u.face_centroid)) <= 0.2 + 1e-6
    assert np.max(np.abs(m.cell_centroid[:nc] - u.cell_centroid[:nc])) <= 0.2 + 1e-6
    # boundary faces stay on the box
    assert np.array_equal(m.face_normal[m.n_interior:], u.face_normal[u.n_interior:])
    # same connectivity and stencils as the uniform mesh; different seeds differ
    assert np.array_equal(m.owner, u.owner) and np.array_equal(m.gradient_stencil, u.gradient_stencil)
    assert not np.array_equal(m.cell_centroid, _mesh(0.1, seed=6).cell_centroid)
    assert np.array_equal(m.cell_centroid, _mesh(0.1, seed=5).cell_centroid)


@pytest.mark.gpu
def test_jittered_duct_matches_oracle():
    from lbfs_b200 import GpuSolver, cases
    from oracle_lbfs import OracleSolver
    c = cases.poiseuille(n=8, ny=6, nz=5)
    m = _mesh(0.1)
    m.set_boundaries(c.bcs)
    steps = 20
    with GpuSolver(m, c.params) as s:
        s.set_state(c.rho, c.u, c.v, c.w)
        s.step(steps)
        got = s.state()
    o = OracleSolver(m, c.params, [])
    o.set_state(c.rho, c.u, c.v, c.w)
    o.step(steps)
    want = o.state()
    for a, b in zip(got, want):
        assert rel_err(a, b) <= FP64_RTOL


@pytest.mark.gpu
def test_jittered_channel_with_red_cell_matches_oracle():
    from lbfs_b200 import GpuSolver, cases
    from oracle_lbfs import OracleSolver
    c = cases.jittered_channel(n=16, n_rbc=1, level=2, radius_cells=2.0)
    steps = 8
    with GpuSolver(c.mesh, c.params, c.membranes) as s:
        s.set_state(c.rho, c.u, c.v, c.w)
        s.step(steps)
        got, nodes = s.state(), s.nodes()
    o = OracleSolver(c.mesh, c.params, c.membranes)
    o.set_state(c.rho, c.u, c.v, c.w)
    o.step(steps)
    for a, b in zip(got, o.state()):
        assert rel_err(a, b) <= FP64_RTOL
    assert rel_err(nodes, o.nodes()) <= FP64_RTOL


def test_jittered_box_at_rest_stays_at_rest():
    """With the faces' vector areas closing around every cell, a fluid at rest
    in a closed jittered box feels no net pressure force (oracle, CPU)."""
    from lbfs_b200 import StepParams
    from oracle_lbfs import OracleSolver
    m = _mesh(0.1, n=(6, 5, 4))
    m.set_boundaries({p: (2, 1, 1.0, 0.0, 0.0, 0.0) for p in ("left", "right", "bottom", "top", "back", "front")})
    p = StepParams(visc=0.1, delta_t=0.5, testcase=2, viscosity_period=0)
    o = OracleSolver(m, p, [])
    n = m.n_cells
    o.set_state(np.ones(n), np.zeros(n), np.zeros(n), np.zeros(n))
    o.step(50)
    rho, u, v, w = o.state()
    assert np.max(np.abs(rho - 1.0)) < 1e-12
    assert max(np.max(np.abs(u)), np.max(np.abs(v)), np.max(np.abs(w))) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["local", "min"])
def test_jittered_time_stepping_matches_oracle(mode):
    """Per-cell CFL steps vary across a jittered mesh (volumes and face areas
    differ per cell): local and minimum time stepping against the oracle, with
    a red cell moving by the minimum step."""
    from dataclasses import replace
    from lbfs_b200 import GpuSolver, _abi, cases
    from oracle_lbfs import OracleSolver
    ts = {"local": _abi.LBFS_DT_LOCAL, "min": _abi.LBFS_DT_MIN}[mode]
    c = cases.jittered_channel(n=16, n_rbc=1, level=2, radius_cells=2.0)
    c.params = replace(c.params, time_stepping=ts)
    steps = 8
    with GpuSolver(c.mesh, c.params, c.membranes) as s:
        s.set_state(c.rho, c.u, c.v, c.w)
        s.step(steps, graph=True)
        got, nodes, dtl, dt = s.state(), s.nodes(), s.field(_abi.LBFS_FIELD_DT_LOCAL), s.time_step()
        assert s.status() == 0
    o = OracleSolver(c.mesh, c.params, c.membranes)
    o.set_state(c.rho, c.u, c.v, c.w)
    o.step(steps)
    for a, b in zip(got, o.state()):
        assert rel_err(a, b) <= FP64_RTOL
    assert rel_err(nodes, o.nodes()) <= FP64_RTOL
    want = o.field(_abi.LBFS_FIELD_DT_LOCAL)
    assert rel_err(dtl, want) <= FP64_RTOL and rel_err(dt, o.time_step()) <= FP64_RTOL
    if mode == "local":
        assert np.ptp(want) > 1e-3 * np.mean(want)  # the steps do vary from cell to cell


@pytest.mark.gpu
def test_jittered_preconditioning_matches_oracle():
    """Preconditioning (gamma = 2) where every face takes the general-normal
    flux: the lattice equilibria of all faces carry 1/gamma."""
    from dataclasses import replace
    from lbfs_b200 import GpuSolver, cases
    from oracle_lbfs import OracleSolver
    c = cases.poiseuille(n=8, ny=6, nz=5)
    c.params = replace(c.params, gamma_inv=0.5, preconditioning=1)
    m = _mesh(0.1)
    m.set_boundaries(c.bcs)
    with GpuSolver(m, c.params) as s:
        s.set_state(c.rho, c.u, c.v, c.w)
        s.step(10)
        got = s.state()
    o = OracleSolver(m, c.params, [])
    o.set_state(c.rho, c.u, c.v, c.w)
    o.step(10)
    for a, b in zip(got, o.state()):
        assert rel_err(a, b) <= FP64_RTOL
