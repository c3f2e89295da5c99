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
