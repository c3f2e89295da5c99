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


FOAM = "polymesh_jitter_8x6x5"


@pytest.mark.parametrize("hybrid", [False, True], ids=["LS", "hybrid"])
def test_openfoam_import_bit_exact(golden, hybrid):
    """The importer reads the committed polyMesh exactly as the reference's importer did
    (import_openfoam_mesh + generate_internal_mesh + pre_fill_LHS_and_RHS_matrix)."""
    import os
    from conftest import ROOT
    from lbfs_b200 import import_openfoam
    g = golden(f"mesh_foam_jitter_8x6x5{'_hybrid' if hybrid else ''}.npz")
    m = import_openfoam(os.path.join(ROOT, "tests", "golden", FOAM), gradient="hybrid" if hybrid else "LS")
    assert [m.n_cells, m.n_faces, m.n_interior, m.n_bc] == list(g["counts"])
    for key in ("owner", "neighbour", "face_area", "face_normal", "face_centroid", "streaming_dt", "cell_volume",
                "cell_centroid", "gradient_stencil", "lhs_inverse", "rhs"):
        assert np.array_equal(getattr(m, key), g[key]), key
    assert m.patch_names == ("left", "right", "bottom", "top", "back", "front") and not m.axis_aligned


def test_openfoam_writer_and_round_trip(tmp_path):
    """The writer reproduces the committed polyMesh byte for byte, and reading it back gives the
    generator's mesh with the reference's face areas (lbfs_mesh_build_jittered, closed_faces=0)."""
    import os
    from conftest import ROOT
    from lbfs_b200 import import_openfoam, write_openfoam
    write_openfoam(tmp_path, 16.0, 12.0, 10.0, 1.0, jitter=0.1, seed=5)
    for name in ("points", "faces", "owner", "neighbour", "boundary"):
        with open(os.path.join(ROOT, "tests", "golden", FOAM, name)) as a, open(tmp_path / name) as b:
            assert a.read() == b.read(), name
    m = import_openfoam(tmp_path)
    g = build_uniform_mesh(16.0, 12.0, 10.0, 1.0, visc=0.1, jitter=0.1, seed=5, closed_faces=False)
    for key in ("owner", "neighbour", "face_area", "face_normal", "face_centroid", "streaming_dt", "cell_volume",
                "cell_centroid", "gradient_stencil", "lhs_inverse", "rhs", "bc_patch"):
        assert np.array_equal(getattr(m, key), getattr(g, key)), key
    # the closed-face variant changes only the areas of warped faces (and what depends on them)
    c = build_uniform_mesh(16.0, 12.0, 10.0, 1.0, visc=0.1, jitter=0.1, seed=5)
    assert np.array_equal(c.face_normal, g.face_normal) and not np.array_equal(c.face_area, g.face_area)
    assert np.allclose(c.face_area, g.face_area, rtol=5e-2)  # warped faces: up to about 2 % apart


def test_openfoam_import_rejects_bad_headers(tmp_path):
    from lbfs_b200 import LbfsError, import_openfoam, write_openfoam
    write_openfoam(tmp_path, 8.0, 6.0, 10.0, 1.0)
    lines = (tmp_path / "owner").read_text().split("\n")
    lines[12] = "    note        \"no counts here\";"
    (tmp_path / "owner").write_text("\n".join(lines))
    with pytest.raises(LbfsError):
        import_openfoam(tmp_path)


@pytest.mark.parametrize("defect", ["cell_with_7_faces", "owner_is_neighbour"])
def test_openfoam_gpu_import_rejects_bad_topology(tmp_path, defect):
    """The GPU geometry's topology checks run on the host before any device work."""
    from lbfs_b200 import LbfsError, import_openfoam, write_openfoam
    write_openfoam(tmp_path, 8.0, 6.0, 10.0, 1.0)
    name = "owner" if defect == "cell_with_7_faces" else "neighbour"
    lines = (tmp_path / name).read_text().split("\n")
    start = lines.index("(") + 1
    if defect == "cell_with_7_faces":  # the last (boundary) face handed to cell 0
        end = lines.index(")")
        lines[end - 1] = "0"
    else:  # face 0's neighbour set to its owner
        own = (tmp_path / "owner").read_text().split("\n")
        lines[start] = own[own.index("(") + 1]
    (tmp_path / name).write_text("\n".join(lines))
    with pytest.raises(LbfsError, match="6 stencil entries|owner as neighbour"):
        import_openfoam(tmp_path, device=0)
