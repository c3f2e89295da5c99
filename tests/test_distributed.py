"""The multi-process path on CPU: two gloo ranks, each stepping its shard of
independent instances (the C restatement stands in for the GPU), agree on the
max-over-ranks time and gather per-instance results identical to one process."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _instances():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "lbfs-ibm-ade-sp_b200"))
    from lbfs_b200 import cases
    return [cases.poiseuille(n=n, ny=5, nz=4, seed=10 + n) for n in (4, 6, 5, 7, 4)]


def _run_instance(c, steps=3):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle_lbfs import OracleSolver
    o = OracleSolver(c.mesh, c.params, c.membranes)
    o.set_state(c.rho, c.u, c.v, c.w)
    o.step(steps)
    rho, u, v, w = o.state()
    o.close()
    return float(np.sum(rho)), float(np.sum(u))


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "lbfs-ibm-ade-sp_b200"))
    import torch.distributed as dist
    from datetime import timedelta
    from lbfs_b200.parallel import gather_objects, max_over_ranks, shard_instances
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    inst = _instances()
    shards = shard_instances([c.mesh.n_cells for c in inst], world)
    mine = {i: _run_instance(inst[i]) for i in shards[rank]}
    t = max_over_ranks(1.0 + rank)
    gathered = gather_objects(mine)
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        q.put((t, shards, gathered))


def test_two_rank_gloo_replicas_match_single_process():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_lbfs
    oracle_lbfs.lib()  # build the oracle here, not in both ranks at once
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    t, shards, gathered = q.get(timeout=240)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert t == 2.0
    assert sorted(shards[0] + shards[1]) == list(range(5))
    merged = {}
    for part in gathered:
        merged.update(part)
    inst = _instances()
    for i, c in enumerate(inst):
        assert merged[i] == _run_instance(c)  # same instance, same numbers, whichever rank ran it


def test_shard_instances_balances_and_is_deterministic():
    from lbfs_b200.parallel import shard_instances
    costs = [16 ** 3, 48 ** 3, 20 ** 3, 40 ** 3, 33 ** 3, 17 ** 3, 48 ** 3, 30 ** 3]
    a = shard_instances(costs, 3)
    assert a == shard_instances(costs, 3)
    assert sorted(sum(a, [])) == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in a]
    assert max(loads) <= 1.34 * (sum(costs) / 3)


_ENS = dict(n_instances=6, seed=31, n_range=(8, 12), rbc_range=(1, 2), levels=(1, 2))


def _ensemble_worker(rank, world, port, q):
    """One rank of the sharded batched workload: its instances by cost (cells + red-cell nodes),
    its own ensemble layout of just those, and each of its instances stepped (the oracle standing in
    for the GPU), gathered by instance number."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "lbfs-ibm-ade-sp_b200"))
    import torch.distributed as dist
    from datetime import timedelta
    from lbfs_b200 import cases
    from lbfs_b200.parallel import gather_objects, shard_instances
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    specs = cases.ensemble_specs(**_ENS)
    shard = shard_instances([s["cost"] for s in specs], world)[rank]
    part = cases.ensemble(**_ENS, subset=shard)
    layout = {k: (part.mesh.split(part.u)[j].copy(), m.membranes[0].xyz_initial.copy())
              for j, (k, m) in enumerate(zip(part.info["indices"], part.info["members"]))}
    stepped = {k: _run_instance(m, steps=2) for k, m in zip(part.info["indices"], part.info["members"])}
    gathered = gather_objects((shard, layout, stepped))
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        q.put(gathered)


def test_two_rank_sharded_ensemble_equals_single_process():
    """Sharding the batched workload over 2 gloo ranks: the shards cover every instance once, each
    rank's ensemble holds exactly its instances' meshes, states and red cells as the one-process
    ensemble does, and stepping them gives the one-process numbers."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_lbfs
    from lbfs_b200 import cases
    oracle_lbfs.lib()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ensemble_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=240)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    shards = [g[0] for g in gathered]
    assert sorted(shards[0] + shards[1]) == list(range(_ENS["n_instances"]))
    full = cases.ensemble(**_ENS)
    u = full.mesh.split(full.u)
    for shard, layout, stepped in gathered:
        for k in shard:
            assert np.array_equal(layout[k][0], u[k])
            assert np.array_equal(layout[k][1], full.info["members"][k].membranes[0].xyz_initial)
            assert stepped[k] == _run_instance(full.info["members"][k], steps=2)


_ENS_GPU = dict(n_instances=6, seed=17, n_range=(10, 14), rbc_range=(1, 2), levels=(1, 2), radius_cells=1.5)


def _gpu_ensemble_worker(rank, world, port, q):
    """One rank of the sharded batched workload on the GPU: its shard of instances as one ensemble
    handle, stepped in a graph; the ranks share nothing on the data path (gloo carries only the
    max-over-ranks time and the gathered results), so none of their kernels waits on another's."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "lbfs-ibm-ade-sp_b200"))
    import torch.distributed as dist
    from datetime import timedelta
    from lbfs_b200 import GpuSolver, cases
    from lbfs_b200.parallel import gather_objects, max_over_ranks, shard_instances
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    specs = cases.ensemble_specs(**_ENS_GPU)
    shard = shard_instances([s["cost"] for s in specs], world)[rank]
    part = cases.ensemble(**_ENS_GPU, subset=shard)
    with GpuSolver(part.mesh, part.params, part.membranes, device=0) as s:
        s.set_state(part.rho, part.u, part.v, part.w)
        s.step(8, graph=True)
        state = s.state()
        status = s.status()
    per = {k: [part.mesh.split(a)[j].copy() for a in state] for j, k in enumerate(part.info["indices"])}
    t = max_over_ranks(10.0 + rank)
    gathered = gather_objects((shard, per, status))
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        q.put((t, gathered))


@pytest.mark.gpu
def test_two_rank_sharded_ensemble_on_gpu_equals_single_process():
    """The sharded batched path with real GPU handles: two gloo ranks (both on the one GPU of this
    run) each step their shard; every instance's state equals, bit for bit, the same instance in the
    one-process ensemble handle."""
    from lbfs_b200 import GpuSolver, cases
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gpu_ensemble_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    t, gathered = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert t == 11.0
    shards = [g[0] for g in gathered]
    assert sorted(shards[0] + shards[1]) == list(range(_ENS_GPU["n_instances"]))
    assert all(g[2] == 0 for g in gathered)
    full = cases.ensemble(**_ENS_GPU)
    with GpuSolver(full.mesh, full.params, full.membranes) as s:
        s.set_state(full.rho, full.u, full.v, full.w)
        s.step(8, graph=True)
        ref = [full.mesh.split(a) for a in s.state()]
    for shard, per, _ in gathered:
        for k in shard:
            for c in range(4):
                assert np.array_equal(per[k][c], ref[c][k]), (k, c)
