"""Mesh, gradient geometry and spring connectivity are bit-exact against the
reference's own host code (golden fixtures from tests/golden/make_golden.py)."""
import numpy as np
import pytest

from lbfs_b200 import build_springs, build_uniform_mesh, icosphere, uniform_counts


@pytest.mark.parametrize("name", ["mesh_4x3x5.npz", "mesh_6x6x6_hybrid.npz", "mesh_plateau_10x8x6.npz",
                                  "mesh_cosine5_8x6x5.npz", "mesh_cosine7_8x6x5.npz"])
def test_uniform_mesh_bit_exact(golden, name):
    g = golden(name)
    X, Y, Z, hybrid = float(g["X"]), float(g["Y"]), float(g["Z"]), int(g["hybrid"])
    mesh_type, plateau = int(g["mesh_type"]), tuple(float(x) for x in g["plateau_params"])
    assert uniform_counts(X, Y, Z, 1.0) == list(g["counts"])
    m = build_uniform_mesh(X, Y, Z, 1.0, visc=0.1, gradient="hybrid" if hybrid else "LS", mesh_type=mesh_type,
                           plateau_width=plateau[0], plateau_slope=plateau[1])
    if mesh_type == 4:
        # the plateau arrays the 4x4x4 IBM stencil searches (plateau_x, _y, _z)
        assert np.array_equal(np.concatenate(m.grid), g["plateau"])
    mine = dict(owner=m.owner, neighbour=m.neighbour, face_area=m.face_area, face_normal=m.face_normal,
                face_centroid=m.face_centroid, streaming_dt=m.streaming_dt, cell_volume=m.cell_volume,
                cell_centroid=m.cell_centroid, gradient_stencil=m.gradient_stencil, lhs_inverse=m.lhs_inverse,
                rhs=m.rhs)
    for key, arr in mine.items():
        assert np.array_equal(arr, g[key]), key  # integers and doubles bit for bit
    assert m.delta_h == float(g["delta_h"])


def test_face_order_and_ghost_numbering(golden):
    g = golden("mesh_4x3x5.npz")
    nc, nf, ni, nb = (int(x) for x in g["counts"][:4])
    neighbour = g["neighbour"]
    assert np.array_equal(neighbour[ni:], nc + np.arange(nb))  # ghost of bc face i is cell nc + i
    assert (g["owner"][:ni] < neighbour[:ni]).all()             # owner is the west/south/back cell


@pytest.mark.parametrize("level", [1, 2, 3])
def test_springs_bit_exact(golden, level):
    g = golden(f"springs_L{level}.npz")
    unit, tris = icosphere(level, 1.0)
    assert np.array_equal(tris, g["tris"]) and np.array_equal(g["ref_tris"], tris)
    spr = build_springs(len(unit), tris)
    assert np.array_equal(spr, g["ref_springs"])
    assert len(spr) == 3 * len(tris) // 2


def test_springs_cover_every_edge_once():
    unit, tris = icosphere(2, 1.0)
    spr = build_springs(len(unit), tris)
    edges = {tuple(sorted((int(a), int(c)))) for a, _, c, _ in spr}
    tri_edges = {tuple(sorted((int(t[i]), int(t[(i + 1) % 3])))) for t in tris for i in range(3)}
    assert edges == tri_edges
