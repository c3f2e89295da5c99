"""Slab decomposition on the GPU (lbfs_b200.slabs): after every step and halo
exchange, the owned cells of each slab hold the one-mesh step's state bit for
bit, and the membrane's nodes are the one-mesh run's.  Two slabs in one process
(device copies), and two gloo ranks each holding a slab as a GPU handle (host
copies; both on the one GPU of this run, their kernels never wait on each
other's).  The IBM window raises LBFS_FLAG_IBM_RANGE when a patch leaves it."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT
from lbfs_b200 import GpuSolver, _abi, cases
from lbfs_b200.slabs import SlabSolver, assign_membranes, build_slab_mesh, slab_bounds, step_local

pytestmark = pytest.mark.gpu

N, NZ, PLANES, STEPS = 32, 48, [30, 18], 25


def _case(precision, zc=0.3):
    # shear + a level-2 red cell of radius 5 cells at height zc of the box (IBM reach at 0.3: z cells ~10 .. 20,
    # in the lower of slabs [30, 18]; at 0.5: ~19 .. 29, in the middle of slabs [16, 16, 16])
    return cases.shear_rbc(n=N, n_cells_z=NZ, level=2, radius_cells=5.0, centre=(0.5, 0.5, zc), precision=precision)


def _slab_solvers(c, bounds, ranks=None):
    dom = (2.0 * N, 2.0 * N, 2.0 * NZ, 1.0)
    owner = assign_membranes(c.membranes, bounds, NZ, 0.0, 2.0, c.params.ibm_stencil)
    out = []
    for r in (ranks if ranks is not None else range(len(bounds))):
        slab = build_slab_mesh(*dom, bounds, r, bcs=c.bcs, visc=c.params.visc)
        s = SlabSolver(slab, c.params, [m for m, o in zip(c.membranes, owner) if o == r])
        s.set_state(c.rho, c.u, c.v, c.w)
        out.append(s)
    return out


def _one_mesh(c, steps):
    with GpuSolver(c.mesh, c.params, c.membranes) as s:
        s.set_state(c.rho, c.u, c.v, c.w)
        s.step(steps, graph=True)
        return s.state(), s.nodes(), s.status()


@pytest.mark.parametrize("precision,planes,zc", [(_abi.LBFS_FP64, PLANES, 0.3), (_abi.LBFS_FP32_BULK, PLANES, 0.3),
                                                 (_abi.LBFS_FP64, [16, 16, 16], 0.5)],
                         ids=["fp64_2slabs", "fp32_2slabs", "fp64_3slabs"])
def test_slabs_in_one_process_equal_the_one_mesh_step(precision, planes, zc):
    c = _case(precision, zc)
    bounds = slab_bounds(NZ, len(planes), planes)
    ref_state, ref_nodes, ref_status = _one_mesh(c, STEPS)
    slabs = _slab_solvers(c, bounds)
    try:
        step_local(slabs, STEPS, "cuda:0")
        P = slabs[0].slab.plane_cells
        for s, (z0, z1) in zip(slabs, bounds):
            got = s.owned_state()
            for a, b in zip(got, ref_state):
                assert np.array_equal(a, b[z0 * P:z1 * P]), (z0, np.flatnonzero(a != b[z0 * P:z1 * P])[:5])
            assert s.solver.status() == 0
        (holder,) = [s for s in slabs if s.membranes]
        assert np.array_equal(holder.solver.nodes(), ref_nodes)
        assert ref_status == 0
    finally:
        for s in slabs:
            s.solver.close()


def test_ibm_window_flags_a_patch_outside_it():
    c = cases.shear_rbc(n=16, level=1, radius_cells=3.0)
    with GpuSolver(c.mesh, c.params, c.membranes) as s:
        s.set_state(c.rho, c.u, c.v, c.w)
        s.step(1)
        assert s.status() == 0
        s.set_ibm_window(0, 3)  # the cell sits at the centre: its patch spans z cells ~5 .. 11
        s.step(1)
        assert s.status() & _abi.LBFS_FLAG_IBM_RANGE


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _slab_worker(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "lbfs-ibm-ade-sp_b200"))
    import torch.distributed as dist
    from lbfs_b200.slabs import TorchExchange
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    c = _case(_abi.LBFS_FP64)
    bounds = slab_bounds(NZ, world, PLANES)
    (s,) = _slab_solvers(c, bounds, ranks=[rank])
    TorchExchange(s, "cuda:0").step(STEPS)
    got = (s.owned_state(), s.solver.nodes(), s.solver.status())
    s.solver.close()
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got))


def test_two_gloo_ranks_each_with_a_slab_equal_the_one_mesh_step():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    while len(got) < 2:  # stop waiting as soon as a rank has failed
        try:
            r, res = q.get(timeout=5)
            got[r] = res
        except Exception:
            assert all(p.exitcode in (None, 0) for p in procs), [p.exitcode for p in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    c = _case(_abi.LBFS_FP64)
    ref_state, ref_nodes, _ = _one_mesh(c, STEPS)
    bounds = slab_bounds(NZ, 2, PLANES)
    P = N * N
    for r, (z0, z1) in enumerate(bounds):
        state, nodes, status = got[r]
        for a, b in zip(state, ref_state):
            assert np.array_equal(a, b[z0 * P:z1 * P]), r
        assert status == 0
    assert np.array_equal(got[0][1], ref_nodes)
