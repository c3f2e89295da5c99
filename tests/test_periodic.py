"""Periodic boundaries (type 3) on the host side: the partner search and the oracle.

The reference's GPU kernels implement no periodic type (LBFS.cu:1872-1918);
its CPU solver does: a type-3 ghost takes the state (Solution::
update_unstructured_bcs, Solution.cpp:777-803) and the gradients (gradients::
Get_LS_Gradients, gradients.cpp:428-440) of its partner cell, the interior
cell nearest to the ghost moved by the periodic translation (Boundary_
Conditions.cpp:417-432, whose search point is an uninitialised index there).
The partner search is checked against the all-cell search it replaces; the
oracle's periodic step against the symmetry of an x-invariant duct.
"""
import numpy as np
import pytest

from lbfs_b200 import _abi, build_uniform_mesh, cases
from lbfs_b200.mesh import find_periodic_nodes
from oracle_lbfs import OracleSolver

PATCHES = ("left", "right", "bottom", "top", "back", "front")


def all_cell_search(mesh, translation):
    """Boundary_Conditions.cpp:417-432 with the ghost's own centroid as the point, over +-translation:
    the first cell (ascending index) with the smallest |c_i - p|."""
    nc = mesh.n_cells
    cen = mesh.cell_centroid.reshape(-1, 3)
    out = np.zeros(mesh.n_bc, np.int32)
    t = np.asarray(translation, np.float64)
    for b in range(mesh.n_bc):
        if mesh.bc_rho_type[b] != 3 and mesh.bc_vel_type[b] != 3:
            continue
        best, best_i = np.inf, -1
        for p in (cen[nc + b] + t, cen[nc + b] - t):
            d = cen[:nc] - p
            dist = np.sqrt(d[:, 0] ** 2 + d[:, 1] ** 2 + d[:, 2] ** 2)
            i = int(np.argmin(dist))  # first index of the minimum
            if dist[i] < best or (dist[i] == best and i < best_i):
                best, best_i = dist[i], i
        out[b] = best_i
    return out


def periodic_mesh(n, ny, nz, axis, jitter=0.0, seed=3):
    m = build_uniform_mesh(2.0 * n, 2.0 * ny, 2.0 * nz, 1.0, jitter=jitter, seed=seed)
    pair = [("left", "right"), ("bottom", "top"), ("back", "front")][axis]
    spec = {p: (3, 3, 1.0, 0.0, 0.0, 0.0) if p in pair else (2, 1, 1.0, 0.0, 0.0, 0.0) for p in PATCHES}
    t = [0.0, 0.0, 0.0]
    t[axis] = (2.0 * n, 2.0 * ny, 2.0 * nz)[axis]
    m.set_boundaries(spec, periodic_translation=t)
    return m, t


@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("jitter", [0.0, 0.15])
def test_partners_equal_all_cell_search(axis, jitter):
    m, t = periodic_mesh(9, 7, 5, axis, jitter)
    assert np.count_nonzero(m.bc_rho_type == 3) > 0
    np.testing.assert_array_equal(m.periodic_node, all_cell_search(m, t))


def test_partners_of_a_uniform_mesh_are_the_opposite_cells():
    m, _ = periodic_mesh(8, 6, 5, 0)
    nx, ny, nz = m.shape
    for b in np.flatnonzero(m.bc_rho_type == 3):
        o = m.owner[m.n_interior + b]
        p = m.periodic_node[b]
        assert p // nx == o // nx and p % nx == nx - 1 - o % nx


def test_partner_ties_take_the_lower_cell():
    # a translation of half the box puts every search point on a plane between two cell rows:
    # equal distances, and the search keeps the lower index as the reference's strict < does
    m = build_uniform_mesh(8.0, 6.0, 4.0, 1.0)
    spec = {p: (3, 3, 1.0, 0.0, 0.0, 0.0) if p in ("left", "right") else (2, 2, 1.0, 0.0, 0.0, 0.0) for p in PATCHES}
    m.set_boundaries(spec, periodic_translation=(3.0, 0.0, 0.0))
    np.testing.assert_array_equal(m.periodic_node, all_cell_search(m, (3.0, 0.0, 0.0)))


def test_periodic_needs_a_translation():
    m = build_uniform_mesh(8.0, 6.0, 4.0, 1.0)
    with pytest.raises(ValueError):
        m.set_boundaries({p: (3, 3, 1.0, 0.0, 0.0, 0.0) for p in PATCHES})


def test_non_periodic_ghosts_get_zero():
    m, t = periodic_mesh(6, 5, 4, 1)
    assert np.all(m.periodic_node[(m.bc_rho_type != 3) & (m.bc_vel_type != 3)] == 0)
    assert np.all(find_periodic_nodes(m, t) == m.periodic_node)


def x_invariant_state(mesh, seed=3):
    nx, ny, nz = mesh.shape
    rng = np.random.default_rng(seed)
    row = lambda a: np.ascontiguousarray(np.repeat(a.reshape(nz, ny, 1), nx, axis=2).ravel())
    return (row(1.0 + 1e-4 * rng.standard_normal(ny * nz)), row(1e-3 * rng.standard_normal(ny * nz)),
            row(1e-4 * rng.standard_normal(ny * nz)), row(1e-4 * rng.standard_normal(ny * nz)))


def test_oracle_periodic_duct_stays_x_invariant():
    # periodic in x, walls in y and z, a state independent of x: every x column evolves alike
    c = cases.poiseuille(n=8, ny=6, nz=5, periodic_x=True)
    nx, ny, nz = c.mesh.shape
    o = OracleSolver(c.mesh, c.params, c.membranes)
    o.set_state(*x_invariant_state(c.mesh))
    o.step(30)
    for a in o.state():
        A = a.reshape(nz, ny, nx)
        assert np.abs(A - A[:, :, :1]).max() <= 1e-10 * np.abs(A).max()
    o.close()


def test_oracle_periodic_ghosts_take_the_partner_values():
    c = cases.poiseuille(n=6, ny=5, nz=4, periodic_x=True)
    m = c.mesh
    o = OracleSolver(m, c.params, c.membranes)
    o.set_state(c.rho, c.u, c.v, c.w)
    o.step(3)
    # fields of the last step: ghosts formed from the state the step started from
    ghost = o.field(_abi.LBFS_FIELD_GHOST).reshape(-1, 4)
    grad = o.field(_abi.LBFS_FIELD_GRADIENTS).reshape(-1, 12)
    o2 = OracleSolver(m, c.params, c.membranes)
    o2.set_state(c.rho, c.u, c.v, c.w)
    o2.step(2)
    r, u, v, w = o2.state()
    per = np.flatnonzero(m.bc_rho_type == 3)
    assert len(per) == 2 * 5 * 4
    pn = m.periodic_node[per]
    np.testing.assert_array_equal(ghost[per], np.stack([u[pn], v[pn], w[pn], r[pn]], 1))
    np.testing.assert_array_equal(grad[m.n_cells + per], grad[pn])
    o.close()
    o2.close()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["own", "all"])
def test_periodic_objects_wrap_modes_vs_oracle(mode):
    """Two periodic red cells, one high in z (0.8 Z) and one lower (0.4 Z): with LBFS_WRAP_OWN only the
    high one moves down by Z / 2 at t = 1 (its own mean is above 0.75 Z); with LBFS_WRAP_ALL on
    membrane 0 -- the reference's check_periodic_object over all objects' nodes -- the joint mean is
    below the bound and neither moves.  CUDA path and oracle agree to 1e-10."""
    from helpers import FP64_RTOL, rel_err
    from lbfs_b200 import GpuSolver, _abi, cases, red_cell
    from oracle_lbfs import OracleSolver
    c = cases.shear_rbc(n=16, level=1, radius_cells=2.0, ibm_stencil=_abi.LBFS_IBM_HAT2)
    first = c.membranes[0]
    moduli = {k: getattr(first, k) for k in ("volume_modulus", "local_area_modulus", "global_area_modulus",
                                             "shear_modulus", "global_bending_modulus", "wlc_ratio",
                                             "internal_viscosity_ratio")}
    X = c.mesh.X
    flag = _abi.LBFS_WRAP_OWN if mode == "own" else _abi.LBFS_WRAP_ALL
    c.membranes = [red_cell(1, 4.0, (0.3 * X, 0.5 * X, 0.8 * X), **moduli),
                   red_cell(1, 4.0, (0.7 * X, 0.5 * X, 0.4 * X), **moduli)]
    for m in c.membranes:
        m.periodic = flag
    s = GpuSolver(c.mesh, c.params, c.membranes)
    o = OracleSolver(c.mesh, c.params, c.membranes)
    z_before = []
    for h in (s, o):
        h.set_state(c.rho, c.u, c.v, c.w)
    z_before = s.nodes()[:, 2].copy()
    s.step(2)  # the wrap follows the fluid update of step t = 1
    o.step(2)
    z_gpu, z_ora = s.nodes()[:, 2], o.nodes()[:, 2]
    assert rel_err(s.nodes(), o.nodes()) < FP64_RTOL
    n0 = c.membranes[0].n_nodes
    moved = z_before - z_gpu > 0.25 * X  # moved by Z / 2 (the advection moves nodes far less)
    if mode == "own":
        assert moved[:n0].all() and not moved[n0:].any()
    else:
        assert not moved.any()
    for a, b in zip(s.state(), o.state()):
        assert rel_err(a, b) < FP64_RTOL
    s.close()
    o.close()


@pytest.mark.parametrize("mode", ["own", "all"])
def test_oracle_periodic_object_wrap_modes(mode):
    """The oracle's check_periodic_object: LBFS_WRAP_OWN moves each membrane by its own mean,
    LBFS_WRAP_ALL (membrane 0) moves all membranes by the mean over all their nodes."""
    from lbfs_b200 import red_cell
    c = cases.shear_rbc(n=16, level=1, radius_cells=2.0, ibm_stencil=_abi.LBFS_IBM_HAT2)
    first = c.membranes[0]
    moduli = {k: getattr(first, k) for k in ("volume_modulus", "local_area_modulus", "global_area_modulus",
                                             "shear_modulus", "global_bending_modulus", "wlc_ratio",
                                             "internal_viscosity_ratio")}
    X = c.mesh.X
    flag = _abi.LBFS_WRAP_OWN if mode == "own" else _abi.LBFS_WRAP_ALL
    for zs, expect in (((0.8, 0.4), {"own": (True, False), "all": (False, False)}),
                       ((0.8, 0.78), {"own": (True, True), "all": (True, True)})):
        c.membranes = [red_cell(1, 4.0, (x * X, 0.5 * X, z * X), **moduli) for x, z in zip((0.3, 0.7), zs)]
        for m in c.membranes:
            m.periodic = flag
        o = OracleSolver(c.mesh, c.params, c.membranes)
        o.set_state(c.rho, c.u, c.v, c.w)
        z0 = o.nodes()[:, 2].copy()
        o.step(2)  # the wrap follows the fluid update of step t = 1
        moved = z0 - o.nodes()[:, 2] > 0.25 * X
        n0 = c.membranes[0].n_nodes
        assert (bool(moved[:n0].all()), bool(moved[n0:].all())) == expect[mode], (zs, mode)
        assert moved[:n0].all() or not moved[:n0].any()
        o.close()
