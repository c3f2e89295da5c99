"""Slab decomposition of one mesh (lbfs_b200.slabs): the host side.

The local meshes (owned planes plus halos) carry, for every owned cell and each
of its faces, the whole mesh's geometry and least-squares arrays bit for bit;
windows, halo ranges and membrane placement; the halo exchange over
torch.distributed with two gloo ranks (CPU buffers standing in for the handles).
The GPU side (owned cells equal to the one-mesh step bit for bit) is in
tests/test_slabs_gpu.py."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT
from lbfs_b200 import build_uniform_mesh, red_cell
from lbfs_b200.slabs import HALO, assign_membranes, build_slab_mesh, slab_bounds

DOM = (16.0, 12.0, 40.0, 1.0)  # 8 x 6 x 20 cells of spacing 2


def test_slab_bounds():
    assert slab_bounds(20, 3) == [(0, 7), (7, 14), (14, 20)]
    assert slab_bounds(20, 2, planes=[14, 6]) == [(0, 14), (14, 20)]
    with pytest.raises(ValueError):
        slab_bounds(20, 2, planes=[19, 1])
    with pytest.raises(ValueError):
        slab_bounds(20, 2, planes=[10, 9])


def _face_key(m, f, off):
    # (owner, neighbour) in the whole mesh's cell numbers; boundary faces by (owner, outward normal)
    o = int(m.owner[f]) + off
    if f < m.n_interior:
        return (o, int(m.neighbour[f]) + off)
    return (o, tuple(np.round(m.face_normal[f], 6)))


@pytest.mark.parametrize("world", [2, 3])
def test_local_meshes_carry_the_whole_mesh_geometry(world):
    full = build_uniform_mesh(*DOM, visc=0.1)
    fkeys = {_face_key(full, f, 0): f for f in range(full.n_faces)}
    bounds = slab_bounds(20, world)
    for r in range(world):
        s = build_slab_mesh(*DOM, bounds, r, visc=0.1)
        m, off = s.mesh, s.lo * s.plane_cells
        assert s.plane_cells == 48 and m.n_cells == (s.hi - s.lo) * 48
        own = s.owned
        g = slice(own.start + off, own.stop + off)
        for name in ("cell_volume", "lhs_inverse", "rhs", "cell_centroid"):
            a, b = getattr(m, name), getattr(full, name)
            if name == "cell_centroid":
                a, b = a.reshape(-1, 3), b.reshape(-1, 3)
            assert np.array_equal(a[own], b[g]), name
        st = m.gradient_stencil.reshape(-1, 6)[own]
        gst = full.gradient_stencil.reshape(-1, 6)[g]
        interior = st < m.n_cells
        assert np.array_equal(st[interior] + off, gst[interior])
        assert np.all(gst[~interior] >= full.n_cells)
        # every face of an owned cell: the same area, normal, centroid and streaming dt
        owned_cells = set(range(own.start, own.stop))
        n_checked = 0
        for f in range(m.n_faces):
            if int(m.owner[f]) in owned_cells or (f < m.n_interior and int(m.neighbour[f]) in owned_cells):
                k = fkeys[_face_key(m, f, off)]
                assert m.face_area[f] == full.face_area[k] and m.streaming_dt[f] == full.streaming_dt[k]
                assert np.array_equal(m.face_normal[f], full.face_normal[k])
                assert np.array_equal(m.face_centroid[f], full.face_centroid[k])
                n_checked += 1
        assert n_checked > 0


def test_windows_and_halo_ranges():
    b = slab_bounds(20, 3)
    s0, s1, s2 = (build_slab_mesh(*DOM, b, r, visc=0.1) for r in range(3))
    assert (s0.lo, s0.hi, s1.lo, s1.hi, s2.lo, s2.hi) == (0, 9, 5, 16, 12, 20)
    assert s0.window == (0, 5) and s1.window == (4, 7) and s2.window == (4, 8)
    P = 48
    assert s1.sends() == [(-1, 2 * P, HALO * P), (1, 7 * P, HALO * P)]
    assert s1.recvs() == [(-1, 0, HALO * P), (1, 9 * P, HALO * P)]
    assert s0.sends() == [(1, 5 * P, HALO * P)] and s2.recvs() == [(-1, 0, HALO * P)]


def test_inexact_slab_origin_is_rejected():
    with pytest.raises(ValueError, match="exact in binary"):
        build_slab_mesh(5.6, 5.6, 28.0, 0.7, slab_bounds(20, 2), 1, origin=(0.0, 0.0, 0.1))


def test_z_periodic_and_periodic_objects_are_rejected():
    spec = {p: (2, 2, 1.0, 0.0, 0.0, 0.0) for p in ("left", "right", "bottom", "top", "back", "front")}
    spec["back"] = spec["front"] = (3, 3, 1.0, 0.0, 0.0, 0.0)
    with pytest.raises(ValueError, match="periodic"):
        build_slab_mesh(*DOM, slab_bounds(20, 2), 0, bcs=spec, periodic_translation=(0.0, 0.0, 40.0), visc=0.1)
    c = red_cell(1, 3.0, (8.0, 6.0, 10.0))
    c.periodic = 1
    with pytest.raises(ValueError, match="periodic"):
        assign_membranes([c], slab_bounds(20, 2), 20, 0.0, 2.0, 4)


def test_membranes_go_to_the_slab_whose_window_holds_them():
    b = slab_bounds(40, 2)  # (0, 20), (20, 40); windows [0, 18) and [22, 40)
    low = red_cell(1, 4.0, (8.0, 6.0, 16.0))   # z cells 6 .. 9 (+ stencil)
    high = red_cell(1, 4.0, (8.0, 6.0, 64.0))  # z cells 30 .. 33
    assert assign_membranes([low, high], b, 40, 0.0, 2.0, 4) == [0, 1]
    across = red_cell(1, 4.0, (8.0, 6.0, 40.0))
    with pytest.raises(ValueError, match="crosses"):
        assign_membranes([across], b, 40, 0.0, 2.0, 4)


# --- the exchange over torch.distributed (gloo), handles replaced by host arrays ---------------

class _HostSlab:
    """A stand-in slab solver: each cell one row of a host array, packed to and unpacked from CPU buffers."""

    def __init__(self, slab, values):
        import torch
        self.slab, self.cells, self._bufs = slab, values, {}
        self.row = values.shape[1] * values.itemsize
        self.torch = torch

    def _buf(self, key, n):
        if key not in self._bufs:
            self._bufs[key] = self.torch.empty(n * self.row, dtype=self.torch.uint8)
        return self._bufs[key]

    def pack(self, device):
        out = {}
        for peer, first, n in self.slab.sends():
            b = self._buf(("send", peer), n)
            b.numpy()[:] = self.cells[first:first + n].view(np.uint8).ravel()
            out[peer] = b
        return out

    def recv_buffers(self, device):
        return {peer: self._buf(("recv", peer), n) for peer, _, n in self.slab.recvs()}

    def unpack(self, bufs):
        for peer, first, n in self.slab.recvs():
            self.cells[first:first + n] = bufs[peer].numpy().view(self.cells.dtype).reshape(n, -1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _exchange_worker(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "lbfs-ibm-ade-sp_b200"))
    import torch.distributed as dist
    from lbfs_b200.slabs import TorchExchange, build_slab_mesh, slab_bounds
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    b = slab_bounds(20, world)
    s = build_slab_mesh(*DOM, b, rank, visc=0.1)
    # every local cell holds (global cell index, rank that wrote it); halo rows start as -1
    vals = np.full((s.mesh.n_cells, 2), -1.0)
    own = s.owned
    vals[own, 0] = np.arange(own.start, own.stop) + s.lo * s.plane_cells
    vals[own, 1] = rank
    ex = TorchExchange(_HostSlab(s, vals), "cpu")
    ex()
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, s.lo, s.plane_cells, vals))


def test_two_and_three_rank_halo_exchange_over_gloo():
    for world in (2, 3):
        ctx = mp.get_context("spawn")
        q = ctx.Queue()
        port = _free_port()
        procs = [ctx.Process(target=_exchange_worker, args=(r, world, port, q)) for r in range(world)]
        for p in procs:
            p.start()
        got = {}
        while len(got) < world:  # stop waiting as soon as a rank has failed
            try:
                r, lo, pc, v = q.get(timeout=5)
                got[r] = (lo, pc, v)
            except Exception:
                assert all(p.exitcode in (None, 0) for p in procs), [p.exitcode for p in procs]
        for p in procs:
            p.join(timeout=60)
            assert p.exitcode == 0
        bounds = slab_bounds(20, world)
        for r, (lo, pc, v) in got.items():
            # every local cell now holds its own global index, written by the rank that owns it
            gidx = np.arange(v.shape[0]) + lo * pc
            assert np.array_equal(v[:, 0], gidx), r
            owner = np.searchsorted([z1 for _, z1 in bounds], gidx // pc, side="right")
            assert np.array_equal(v[:, 1], owner), r
