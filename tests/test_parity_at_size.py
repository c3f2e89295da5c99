"""Parity at the benchmark configurations' own sizes.

The fixture tests pin the CUDA path on small meshes; these run the configured
workloads themselves and compare with the reference's own code (its kernel
bodies compiled for the host, oracle/_ref, driven in the order of
Solver_gpu.cu:749-1021) or, where the reference has no such kernel (the 4-point
Peskin delta), with the C restatement oracle:

* shear + one L3 red cell on 64^3 cells (262,144 cells, 642 nodes) with the
  reference's 2-point hat IBM, 5 steps, against the reference: every
  intermediate field of step 1 and the state, nodes, forces and totals after 5;
* the same workload with the 4-point Peskin delta (the benchmark's stencil),
  5 steps, against the oracle;
* the 32^3 body-force duct with zero-gradient x ends (velocity type 2), 20
  steps, against the reference;
* 48^3 shear with one rotated L4 red cell (2,562 nodes), 3 steps (the interior
  viscosity update runs in step 1), against the oracle.

Tolerance: FP64_RTOL (1e-10) relative to each field's largest magnitude.
"""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN
from helpers import FP64_RTOL, rel_err
from lbfs_b200 import GpuSolver, _abi, cases
from oracle_lbfs import OracleSolver

sys.path.insert(0, GOLDEN)

import ref_lbfs as R  # noqa: E402

needs_ref = pytest.mark.skipif(not R.available(), reason="oracle/_ref/libref_lbfs.so not built "
                                                         "(oracle/build_ref.sh needs the reference sources)")


def _ref(c):
    from make_golden import ref_case
    return ref_case(c)


def _gpu(c):
    s = GpuSolver(c.mesh, c.params, c.membranes)
    s.set_state(c.rho, c.u, c.v, c.w)
    return s


def _oracle(c):
    o = OracleSolver(c.mesh, c.params, c.membranes)
    o.set_state(c.rho, c.u, c.v, c.w)
    return o


def _check(pairs):
    bad = {k: rel_err(a, b) for k, (a, b) in pairs.items() if not rel_err(a, b) < FP64_RTOL}
    assert not bad, bad


def _step1_fields_vs_ref(s, rc, membranes):
    pairs = {
        "grad": (s.field(_abi.LBFS_FIELD_GRADIENTS), rc.get(R.REF_GRAD)),
        "flux": (s.field(_abi.LBFS_FIELD_FACE_FLUX), rc.get(R.REF_RES_FACE)),
        "res": (s.field(_abi.LBFS_FIELD_RESIDUAL), rc.get(R.REF_RES)),
        "force": (s.field(_abi.LBFS_FIELD_FORCE), rc.get(R.REF_FORCE)),
        "ghost": (s.field(_abi.LBFS_FIELD_GHOST), rc.get(R.REF_GHOST)),
        "t1": (s.field(_abi.LBFS_FIELD_T1), rc.get(R.REF_T1)),
        "resid": (s.residuals(), rc.get(R.REF_RESID)),
    }
    for k, (a, b) in enumerate(zip(s.state(), rc.state())):
        pairs[f"state{k}"] = (a, b)
    if membranes:
        pairs.update({
            "nodes_x": (s.nodes(_abi.LBFS_NODES_POSITION).ravel(), rc.get(R.REF_NODE_X)),
            "nodes_v": (s.nodes(_abi.LBFS_NODES_VELOCITY).ravel(), rc.get(R.REF_NODE_V)),
            "nodes_f": (s.nodes(_abi.LBFS_NODES_FORCE).ravel(), rc.get(R.REF_NODE_F)),
            "totals": (s.totals()[0], rc.get(R.REF_TOTALS)),
            "visc": (s.field(_abi.LBFS_FIELD_VISC), rc.get(R.REF_VISC)),
            "spring": (s.field(_abi.LBFS_FIELD_SPRING), rc.get(R.REF_SPRING)),
        })
    _check(pairs)


def _final_vs_ref(s, rc, membranes):
    pairs = {f"state{k}": (a, b) for k, (a, b) in enumerate(zip(s.state(), rc.state()))}
    pairs["resid"] = (s.residuals(), rc.get(R.REF_RESID))
    if membranes:
        pairs.update({
            "nodes_x": (s.nodes().ravel(), rc.get(R.REF_NODE_X)),
            "nodes_f": (s.nodes(_abi.LBFS_NODES_FORCE).ravel(), rc.get(R.REF_NODE_F)),
            "totals": (s.totals()[0], rc.get(R.REF_TOTALS)),
            "visc": (s.field(_abi.LBFS_FIELD_VISC), rc.get(R.REF_VISC)),
        })
    _check(pairs)


def _final_vs_oracle(s, o, membranes):
    pairs = {f"state{k}": (a, b) for k, (a, b) in enumerate(zip(s.state(), o.state()))}
    if membranes:
        pairs.update({
            "nodes_x": (s.nodes(), o.nodes()),
            "nodes_f": (s.nodes(_abi.LBFS_NODES_FORCE), o.nodes(_abi.LBFS_NODES_FORCE)),
            "totals": (s.totals(), o.totals()),
            "visc": (s.field(_abi.LBFS_FIELD_VISC), o.field(_abi.LBFS_FIELD_VISC)),
        })
    _check(pairs)


@needs_ref
def test_oracle_matches_reference_shear_rbc64_hat2():
    """CPU only: the oracle and the reference agree at the benchmark size (5 steps)."""
    c = cases.shear_rbc(n=64, ibm_stencil=_abi.LBFS_IBM_HAT2)
    rc, o = _ref(c), _oracle(c)
    rc.step(5)
    o.step(5)
    _check({f"state{k}": (a, b) for k, (a, b) in enumerate(zip(o.state(), rc.state()))})
    _check({"nodes_x": (o.nodes().ravel(), rc.get(R.REF_NODE_X)), "totals": (o.totals()[0], rc.get(R.REF_TOTALS))})
    rc.close()
    o.close()


@pytest.mark.gpu
@needs_ref
def test_shear_rbc64_hat2_vs_reference():
    c = cases.shear_rbc(n=64, ibm_stencil=_abi.LBFS_IBM_HAT2)
    s, rc = _gpu(c), _ref(c)
    s.keep_residuals(True)
    _check({"init_totals": (s.totals()[0], rc.get(R.REF_TOTALS)),
            "init_spring": (s.field(_abi.LBFS_FIELD_SPRING), rc.get(R.REF_SPRING))})
    s.step(1)
    rc.step(1)
    _step1_fields_vs_ref(s, rc, True)
    s.step(4, graph=True)
    rc.step(4)
    _final_vs_ref(s, rc, True)
    assert s.status() == 0
    s.close()
    rc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("membrane_cluster", [0, 8, 16])
def test_shear_rbc64_peskin4_vs_oracle(membrane_cluster):
    """membrane_cluster 0: the membrane step as separate kernels; 8 / 16: as one thread-block
    cluster of that many CTAs per membrane (k_mem_step)."""
    c = cases.shear_rbc(n=64)  # the benchmark workload: 4-point Peskin delta
    s, o = _gpu(c), _oracle(c)
    s.set_launch_shape(membrane_cluster=membrane_cluster)
    s.step(1)
    o.step(1)
    _check({name: (s.field(w), o.field(w)) for name, w in (
        ("grad", _abi.LBFS_FIELD_GRADIENTS), ("flux", _abi.LBFS_FIELD_FACE_FLUX), ("force", _abi.LBFS_FIELD_FORCE),
        ("visc", _abi.LBFS_FIELD_VISC), ("t1", _abi.LBFS_FIELD_T1))})
    s.step(4, graph=True)
    o.step(4)
    _final_vs_oracle(s, o, True)
    assert rel_err(s.residuals(), o.residuals()) < 1e-8
    assert s.status() == 0
    s.close()
    o.close()


@pytest.mark.gpu
@needs_ref
def test_poiseuille32_neumann_ends_vs_reference():
    c = cases.poiseuille(n=32)  # velocity type 2 at the x ends, no-slip y/z walls
    assert set(np.unique(c.mesh.bc_vel_type)) == {1, 2}
    s, rc = _gpu(c), _ref(c)
    s.keep_residuals(True)
    s.step(1)
    rc.step(1)
    _step1_fields_vs_ref(s, rc, False)
    s.step(19, graph=True)
    rc.step(19)
    _final_vs_ref(s, rc, False)
    assert s.status() == 0
    s.close()
    rc.close()


@pytest.mark.gpu
def test_shear48_l4_vs_oracle():
    c = cases.shear_rbc(n=48, level=4, radius_cells=8.0, rotate=True)
    s, o = _gpu(c), _oracle(c)
    s.step(3, graph=True)
    o.step(3)
    _final_vs_oracle(s, o, True)
    assert np.count_nonzero(o.field(_abi.LBFS_FIELD_VISC) != 1.0) > 0  # the interior viscosity update ran
    assert s.status() == 0
    s.close()
    o.close()


@pytest.mark.gpu
@needs_ref
def test_zero_initial_visc_factor_vs_reference():
    """The reference reads visc_factor before its first interior-viscosity update (zero-filled managed
    memory in an RBC run, what the C++ drop-in passes), and that update first sets every cell to 1
    (update_viscosities, Solver_gpu.cu:2194): cells outside the membrane's box must end at 1, not at
    the initial value.  16^3 shear + L2 cell, 10 steps across the update at t = 1."""
    import dataclasses
    c = cases.shear_rbc(n=16, level=2, radius_cells=3.0, ibm_stencil=_abi.LBFS_IBM_HAT2)
    c.params = dataclasses.replace(c.params, visc_factor_initial=0.0)
    s, rc = _gpu(c), _ref(c)
    s.step(10, graph=True)
    rc.step(10)
    _final_vs_ref(s, rc, True)
    assert np.count_nonzero(s.field(_abi.LBFS_FIELD_VISC) == 1.0) > c.mesh.n_cells // 2
    s.close()
    rc.close()
