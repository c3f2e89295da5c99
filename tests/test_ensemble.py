"""Batched ensembles and launch shapes.

An ensemble handle steps K independent cases at once; each instance must evolve
bit for bit as it does in a handle of its own.  Launch shapes (block sizes,
grid caps, what the autotuner picks) must not change any field.
"""
import numpy as np
import pytest

from conftest import has_gpu
from helpers import FP32_RTOL, rel_err


def _small_ensemble(precision):
    from lbfs_b200 import _abi, cases
    return cases.ensemble(n_instances=3, seed=7, n_range=(12, 16), rbc_range=(2, 3), levels=(1, 2),
                          precision=precision, ibm_stencil=_abi.LBFS_IBM_PESKIN4, radius_cells=1.0)


def test_concatenated_layout():
    """Connectivity of the concatenated mesh: every face stays inside its
    instance, boundary faces own their ghosts, and each cell meets its faces in
    the same relative order as in its own mesh."""
    from lbfs_b200 import build_uniform_mesh
    from lbfs_b200.ensemble import concatenate
    bcs = {p: (2, 1, 1.0, 0.0, 0.0, 0.0) for p in ("left", "right", "bottom", "top", "back", "front")}
    meshes = [build_uniform_mesh(2.0 * a, 2.0 * b, 2.0 * c, 1.0).set_boundaries(bcs)
              for a, b, c in ((4, 3, 5), (6, 6, 6), (3, 4, 2))]
    e = concatenate(meshes)
    assert e.n_cells == sum(m.n_cells for m in meshes) and e.n_faces == sum(m.n_faces for m in meshes)
    inst = np.concatenate([np.full(m.n_cells, k) for k, m in enumerate(meshes)] +
                          [np.full(m.n_bc, k) for k, m in enumerate(meshes)])
    assert np.array_equal(inst[e.owner], inst[e.neighbour])
    b = np.arange(e.n_bc)
    assert np.array_equal(e.neighbour[e.n_interior + b], e.n_cells + b)
    assert np.all(e.gradient_stencil >= 0) and np.all(inst[e.gradient_stencil] == inst[:e.n_cells, None])
    # per instance: the global face order of each cell's faces follows the local order
    glob = [[] for _ in range(e.n_cells)]
    for f in range(e.n_faces):
        glob[e.owner[f]].append(("o", f))
        if f < e.n_interior:
            glob[e.neighbour[f]].append(("n", f))
    for k, m in enumerate(meshes):
        loc = [[] for _ in range(m.n_cells)]
        for f in range(m.n_faces):
            loc[m.owner[f]].append(("o", f))
            if f < m.n_interior:
                loc[m.neighbour[f]].append(("n", f))
        for i in range(m.n_cells):
            g = glob[e.cell0[k] + i]
            assert [s for s, _ in g] == [s for s, _ in loc[i]]
            assert np.allclose([e.face_area[f] for _, f in g], [m.face_area[f] for _, f in loc[i]])
    assert np.array_equal(e.split(np.arange(e.n_cells))[1], np.arange(e.cell0[1], e.cell0[1] + meshes[1].n_cells))


@pytest.mark.gpu
@pytest.mark.parametrize("precision,membrane_cluster", [(0, 0), (1, 0), (0, 8), (1, 16)],
                         ids=["fp64", "fp32", "fp64_cluster8", "fp32_cluster16"])
def test_ensemble_matches_separate_handles(precision, membrane_cluster):
    from lbfs_b200 import GpuSolver
    c = _small_ensemble(precision)
    steps = 12  # crosses the interior-viscosity update at t = 1
    with GpuSolver(c.mesh, c.params, c.membranes) as s:
        s.set_launch_shape(membrane_cluster=membrane_cluster)
        s.set_state(c.rho, c.u, c.v, c.w)
        s.step(steps, graph=True)
        state = s.state()
        nodes = s.nodes()
        visc = s.field(5)
        assert s.status() == 0
    node0 = 0
    for k, m in enumerate(c.info["members"]):
        with GpuSolver(m.mesh, m.params, m.membranes) as t:
            t.set_launch_shape(membrane_cluster=membrane_cluster)
            t.set_state(m.rho, m.u, m.v, m.w)
            t.step(steps, graph=True)
            own = t.state()
            for a, b in zip(state, own):
                assert np.array_equal(c.mesh.split(a)[k], b), f"instance {k}"
            assert np.array_equal(c.mesh.split(visc)[k], t.field(5))
            n = t.nodes()
            assert np.array_equal(nodes[node0:node0 + len(n)], n), f"instance {k} nodes"
            node0 += len(n)
    assert node0 == len(nodes)


@pytest.mark.gpu
def test_launch_shapes_do_not_change_fields():
    from lbfs_b200 import GpuSolver, cases
    c = cases.shear_rbc(n=16, level=2, radius_cells=3.0)
    shapes = [dict(), dict(gradient_threads=128, flux_threads=64, general_flux_threads=256, update_threads=512,
                           update_blocks=296, spread_blocks=148),
              dict(gradient_threads=512, flux_threads=256, general_flux_threads=64, update_threads=128,
                   update_blocks=2368, spread_blocks=2368),
              dict(flux_chunks=2), dict(flux_chunks=8, gradient_threads=128),
              dict(membrane_cluster=0), dict(membrane_cluster=8), dict(membrane_cluster=16, flux_chunks=4)]
    out = []
    for sh in shapes:
        with GpuSolver(c.mesh, c.params, c.membranes) as s:
            s.set_launch_shape(**sh)
            s.set_state(c.rho, c.u, c.v, c.w)
            s.step(6, graph=True)
            out.append((s.state(), s.nodes(), s.residuals(), s.launch_shape()["membrane_cluster"]))
    for st, nd, res, mcl in out[1:]:
        if mcl == out[0][3]:
            for a, b in zip(st, out[0][0]):
                assert np.array_equal(a, b)
            assert np.array_equal(nd, out[0][1])
        else:  # the membrane's V, A and MAD are summed in another order: rounding-level differences
            for a, b in zip(st, out[0][0]):
                assert rel_err(a, b) < 1e-12
            assert rel_err(nd, out[0][1]) < 1e-12
        assert rel_err(res, out[0][2]) < 1e-9  # block partials follow the update grid


@pytest.mark.gpu
def test_autotune_keeps_state_and_results():
    from lbfs_b200 import GpuSolver, cases
    c = cases.shear_rbc(n=16, level=2, radius_cells=3.0)
    with GpuSolver(c.mesh, c.params, c.membranes) as s, GpuSolver(c.mesh, c.params, c.membranes) as ref:
        for h in (s, ref):
            h.set_state(c.rho, c.u, c.v, c.w)
            h.step(2, graph=True)
        before = s.state()
        chosen = s.autotune(reps=3)
        assert chosen["step_us"] > 0
        for a, b in zip(s.state(), before):
            assert np.array_equal(a, b)
        assert s.launch_shape()["update_blocks"] == chosen["update_blocks"]
        # the reference handle takes the chosen shape too (membrane_cluster changes rounding)
        ref.set_launch_shape(**{k: v for k, v in s.launch_shape().items() if k != "step_us"})
        s.step(4, graph=True)
        ref.step(4, graph=True)
        for a, b in zip(s.state(), ref.state()):
            assert np.array_equal(a, b)
        assert np.array_equal(s.nodes(), ref.nodes())


@pytest.mark.skipif(has_gpu(), reason="checks argument validation without a device")
def test_launch_shape_struct_roundtrip():
    from lbfs_b200 import _abi
    sh = _abi.LaunchShape()
    sh.update_blocks = _abi.LBFS_MAX_UPDATE_BLOCKS
    assert sh.update_blocks == 148 * 16


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_checkpoint_restart_is_lossless(precision):
    """Snapshot, run on, restore (into the same and into a fresh handle), run
    the same steps again: bit-identical states, nodes and residuals."""
    from lbfs_b200 import GpuSolver, cases
    c = cases.shear_rbc(n=16, level=2, radius_cells=3.0, precision=precision)
    with GpuSolver(c.mesh, c.params, c.membranes) as s:
        s.set_state(c.rho, c.u, c.v, c.w)
        s.step(3, graph=True)
        blob = s.checkpoint()
        s.step(5, graph=True)
        ref = (s.state(), s.nodes(), s.residuals())
        s.restore(blob)
        s.step(5, graph=True)
        again = (s.state(), s.nodes(), s.residuals())
    with GpuSolver(c.mesh, c.params, c.membranes) as t:
        t.restore(blob)
        t.step(5)
        fresh = (t.state(), t.nodes(), t.residuals())
    for other in (again, fresh):
        for a, b in zip(other[0], ref[0]):
            assert np.array_equal(a, b)
        assert np.array_equal(other[1], ref[1])
        assert np.array_equal(other[2], ref[2])


def test_checkpoint_rejects_foreign_blob():
    from lbfs_b200 import _abi
    import ctypes
    buf = ctypes.create_string_buffer(b"not a checkpoint" * 8)
    # argument checks run before any device work: a null handle is an argument error
    assert _abi.lib().lbfs_checkpoint_load(None, buf, len(buf)) == _abi.LBFS_ERR_ARG


@pytest.mark.gpu
def test_batched_fp32_bulk_within_bound_of_fp64():
    """The batched workload itself (64 shear channels of 16^3-48^3 cells, 1-8 red cells each, FP32 bulk)
    against the same ensemble in FP64 after 205 steps.  The velocity field within FP32_RTOL (1e-6):
    max over cells of |u32 - u64| relative to the largest |u64|.  Each component relative to its own
    largest magnitude within 5e-6: the cross-stream components are ~50x smaller than the stream
    velocity, whose FP32 storage (rounding ~6e-11 at |u| ~ 1e-3, renewed every step from the FP64
    accumulator) seeds noise of that absolute size in every component.  The density deviation from
    rho0 within 1e-4 of its largest; red-cell nodes within 1e-9."""
    import dataclasses

    from lbfs_b200 import GpuSolver, _abi, cases
    ce = cases.ensemble(n_instances=64, precision=_abi.LBFS_FP32_BULK)
    p64 = dataclasses.replace(ce.params, precision=_abi.LBFS_FP64)
    a = GpuSolver(ce.mesh, p64, ce.membranes)
    b = GpuSolver(ce.mesh, ce.params, ce.membranes)
    for s in (a, b):
        s.set_state(ce.rho, ce.u, ce.v, ce.w)
        s.step(205, graph=True)
    sa, sb = a.state(), b.state()
    mag = np.sqrt(sa[1] ** 2 + sa[2] ** 2 + sa[3] ** 2)
    diff = np.sqrt((sb[1] - sa[1]) ** 2 + (sb[2] - sa[2]) ** 2 + (sb[3] - sa[3]) ** 2)
    assert np.max(diff) / np.max(mag) < FP32_RTOL, np.max(diff) / np.max(mag)
    errs = {k: rel_err(sb[i], sa[i]) for i, k in ((1, "u"), (2, "v"), (3, "w"))}
    assert max(errs.values()) < 5e-6, errs
    assert rel_err(sb[0] - 1.0, sa[0] - 1.0) < 1e-4
    assert rel_err(b.nodes(), a.nodes()) < 1e-9
    assert a.status() == 0 and b.status() == 0
    a.close()
    b.close()
