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
