"""The generator's meshes built on the GPU (lbfs_mesh_build_gpu) and imported
polyMesh files whose geometry is formed on the GPU (lbfs_mesh_import_openfoam_gpu)
against the host builder and importer, whose arrays are pinned bit for bit on the
reference's own generator and importer (tests/test_setup_golden.py): every
array equal, bit for bit."""
import os
import time

import numpy as np
import pytest

from conftest import ROOT
from lbfs_b200 import build_uniform_mesh, import_openfoam, write_openfoam

pytestmark = pytest.mark.gpu

FIELDS = ("owner", "neighbour", "face_area", "face_normal", "face_centroid", "streaming_dt", "cell_volume",
          "cell_centroid", "gradient_stencil", "lhs_inverse", "rhs", "bc_patch")


def same(a, b):
    for f in FIELDS:
        x, y = getattr(a, f), getattr(b, f)
        assert x.shape == y.shape and x.dtype == y.dtype, f
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), (f, np.flatnonzero(x != y)[:5])
    assert a.delta_h == b.delta_h
    if a.grid is not None or b.grid is not None:
        for x, y in zip(a.grid, b.grid):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("kw", [
    dict(),
    dict(gradient="hybrid", visc=0.07, fneq_min=0.05),
    dict(jitter=0.15, seed=7),
    dict(jitter=0.2, seed=11, closed_faces=False, gradient="hybrid"),
    dict(mesh_type=7),
    dict(mesh_type=5, gradient="hybrid"),
    dict(mesh_type=4, plateau_width=5.0, plateau_slope=0.3),
], ids=["uniform", "hybrid", "jitter", "jitter_open_hybrid", "cosine7", "cosine5", "plateau"])
def test_gpu_mesh_equals_host_mesh(kw):
    args = (26.0, 18.0, 14.0, 1.0)
    same(build_uniform_mesh(*args, origin=(0.5, -1.0, 2.0), device=0, **kw),
         build_uniform_mesh(*args, origin=(0.5, -1.0, 2.0), **kw))


def test_gpu_mesh_128_jittered():
    # the precision study's mesh: 128^3 cells, jitter 0.1, seed 1313, closed faces
    t0 = time.perf_counter()
    g = build_uniform_mesh(256.0, 256.0, 256.0, 1.0, jitter=0.1, seed=1313, device=0)
    t1 = time.perf_counter()
    h = build_uniform_mesh(256.0, 256.0, 256.0, 1.0, jitter=0.1, seed=1313)
    t2 = time.perf_counter()
    same(g, h)
    print(f"128^3 jittered mesh: GPU build {t1 - t0:.3f} s, host build {t2 - t1:.3f} s")


@pytest.mark.parametrize("kw", [dict(), dict(gradient="hybrid", visc=0.07, fneq_min=0.05), dict(closed_faces=True)],
                         ids=["LS", "hybrid", "closed"])
def test_gpu_import_equals_host_import(kw):
    d = os.path.join(ROOT, "tests", "golden", "polymesh_jitter_8x6x5")
    g = import_openfoam(d, device=0, **kw)
    h = import_openfoam(d, **kw)
    same(g, h)
    assert g.patch_names == h.patch_names


@pytest.mark.parametrize("kw", [dict(jitter=0.15, seed=3), dict(mesh_type=7)], ids=["jitter", "cosine7"])
def test_gpu_import_written_meshes(tmp_path, kw):
    write_openfoam(tmp_path, 40.0, 30.0, 24.0, 1.0, origin=(1.0, 0.0, -2.0), **kw)
    for hybrid in (False, True):
        grad = "hybrid" if hybrid else "LS"
        same(import_openfoam(tmp_path, gradient=grad, device=0), import_openfoam(tmp_path, gradient=grad))


def test_gpu_import_64_jittered(tmp_path):
    # 64^3 cells, jitter 0.1: the file read is shared, the geometry differs in where it runs
    write_openfoam(tmp_path, 128.0, 128.0, 128.0, 1.0, jitter=0.1, seed=1313)
    t0 = time.perf_counter()
    g = import_openfoam(tmp_path, device=0)
    t1 = time.perf_counter()
    h = import_openfoam(tmp_path)
    t2 = time.perf_counter()
    same(g, h)
    print(f"64^3 jittered polyMesh: import with GPU geometry {t1 - t0:.3f} s, host geometry {t2 - t1:.3f} s")
