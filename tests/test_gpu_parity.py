"""Parity of the CUDA path (called through the C ABI) with the reference and the oracle.

* against the golden fixtures written by the reference itself;
* against the C restatement oracle on seeded inputs, including the paths the
  fixtures do not reach (general-normal faces, 4-point Peskin IBM, several
  membranes);
* size-independent properties at the full benchmark size (64^3 + one L3 red
  cell): exactness of uniform states, run-to-run determinism, graph replay
  identical to eager launches;
* the FP32-bulk form against the FP64 path within FP32_RTOL.
"""
import tempfile
from dataclasses import replace

import numpy as np
import pytest

from helpers import FP32_RTOL, FP64_RTOL, rel_err
from lbfs_b200 import GpuSolver, _abi, cases, red_cell
from oracle_lbfs import OracleSolver

pytestmark = pytest.mark.gpu


def make(c, cls=GpuSolver):
    s = cls(c.mesh, c.params, c.membranes)
    s.set_state(c.rho, c.u, c.v, c.w)
    return s


def fixture_case(golden, name):
    g = golden(name)
    if "foam_duct" in name:  # the imported jittered mesh (general-normal fluxes everywhere)
        c = cases.imported(cases.poiseuille(n=8, ny=6, nz=5), tempfile.mkdtemp(prefix="polymesh"))
    elif "foam_shear" in name:
        c = cases.imported(cases.shear_rbc(n=16, level=2, radius_cells=3.0, ibm_stencil=_abi.LBFS_IBM_HAT2),
                           tempfile.mkdtemp(prefix="polymesh"))
        c.params = replace(c.params, viscosity_period=0)  # as the fixture (the reference's delta_h is unset)
        mb = c.membranes[0]
        mb.xyz_stress_free, mb.xyz_initial = g["xyz_stress_free"], g["xyz_initial"]
    elif "poiseuille" in name:
        c = cases.poiseuille(n=6, ny=5, nz=4)
    elif "plateau" in name:
        c = cases.shear_rbc(n=16, level=2, radius_cells=3.0, ibm_stencil=_abi.LBFS_IBM_VANDERMONDE4, mesh_type=4,
                            plateau=(5.0, 0.3))
        mb = c.membranes[0]
        mb.xyz_stress_free, mb.xyz_initial = g["xyz_stress_free"], g["xyz_initial"]
    else:
        c = cases.shear_rbc(n=16, level=2, radius_cells=3.0, ibm_stencil=_abi.LBFS_IBM_HAT2)
        mb = c.membranes[0]
        mb.xyz_stress_free, mb.xyz_initial = g["xyz_stress_free"], g["xyz_initial"]
    if "wrap" in name:  # a periodic object: check_periodic_object moves it at t = 1
        c.membranes[0].periodic = True
    c.rho, c.u, c.v, c.w = g["rho0"], g["u0"], g["v0"], g["w0"]
    if "time_stepping" in g.files:
        c.params = replace(c.params, time_stepping=int(g["time_stepping"]), gamma_inv=float(g["gamma_inv"]),
                           preconditioning=int(g["preconditioning"]))
    return c, g


FIXTURES = ["step_poiseuille_6x5x4.npz", "step_shear_rbc_16.npz", "step_poiseuille_6x5x4_local.npz",
            "step_poiseuille_6x5x4_talts.npz", "step_shear_rbc_16_min.npz", "step_plateau_rbc_16.npz",
            "step_poiseuille_6x5x4_precond.npz", "step_foam_duct_8x6x5.npz", "step_foam_shear_rbc_16.npz",
            "step_shear_rbc_16_wrap.npz"]


@pytest.mark.parametrize("name", FIXTURES)
def test_gpu_matches_reference_fixture(golden, name):
    c, g = fixture_case(golden, name)
    s = make(c)
    s.keep_residuals(True)
    if c.membranes:
        assert rel_err(s.totals()[0], g["init_totals"]) < FP64_RTOL
        assert rel_err(s.field(_abi.LBFS_FIELD_SPRING), g["init_spring"]) < FP64_RTOL
    s.step(1)
    checks = {
        "grad": (s.field(_abi.LBFS_FIELD_GRADIENTS), g["s1_grad"]),
        "flux": (s.field(_abi.LBFS_FIELD_FACE_FLUX), g["s1_flux"]),
        "res": (s.field(_abi.LBFS_FIELD_RESIDUAL), g["s1_res"]),
        "force": (s.field(_abi.LBFS_FIELD_FORCE), g["s1_force"]),
        "ghost": (s.field(_abi.LBFS_FIELD_GHOST), g["s1_ghost"]),
        "t1": (s.field(_abi.LBFS_FIELD_T1), g["s1_t1"]),
        "resid": (s.residuals(), g["s1_resid"]),
        "dt_local": (s.field(_abi.LBFS_FIELD_DT_LOCAL), g["s1_dtl"]),
        "dt": (np.array([s.time_step()]), np.array([g["s1_dt"]])),
    }
    for k, arr in enumerate(s.state()):
        checks[f"state{k}"] = (arr, g["s1_state"][k])
    if c.membranes:
        checks["nodes_x"] = (s.nodes(_abi.LBFS_NODES_POSITION).ravel(), g["s1_nodes_x"])
        checks["nodes_v"] = (s.nodes(_abi.LBFS_NODES_VELOCITY).ravel(), g["s1_nodes_v"])
        checks["nodes_f"] = (s.nodes(_abi.LBFS_NODES_FORCE).ravel(), g["s1_nodes_f"])
        checks["totals"] = (s.totals()[0], g["s1_totals"])
        checks["visc"] = (s.field(_abi.LBFS_FIELD_VISC), g["s1_visc"])
        checks["spring"] = (s.field(_abi.LBFS_FIELD_SPRING), g["s1_spring"])
        checks["energy"] = (s.energies()[0], g["s1_energy"])
    for key, (a, b) in checks.items():
        assert rel_err(a, b) < FP64_RTOL, (key, rel_err(a, b))
    s.step(int(g["steps"]) - 1, graph=True)
    for k, arr in enumerate(s.state()):
        assert rel_err(arr, g["sN_state"][k]) < FP64_RTOL, (k, rel_err(arr, g["sN_state"][k]))
    assert rel_err(s.field(_abi.LBFS_FIELD_DT_LOCAL), g["sN_dtl"]) < FP64_RTOL
    assert rel_err(s.time_step(), g["sN_dt"]) < FP64_RTOL
    if c.membranes:
        assert rel_err(s.nodes().ravel(), g["sN_nodes_x"]) < FP64_RTOL
        assert rel_err(s.nodes(_abi.LBFS_NODES_FORCE).ravel(), g["sN_nodes_f"]) < FP64_RTOL
        assert rel_err(s.totals()[0], g["sN_totals"]) < FP64_RTOL
        assert rel_err(s.field(_abi.LBFS_FIELD_VISC), g["sN_visc"]) < FP64_RTOL
        assert rel_err(s.energies()[0], g["sN_energy"]) < FP64_RTOL
    assert s.status() == 0
    s.close()


def compare_with_oracle(c, steps, fields=True):
    s, o = make(c), make(c, OracleSolver)
    s.step(1)
    o.step(1)
    if fields:
        for which in (_abi.LBFS_FIELD_GRADIENTS, _abi.LBFS_FIELD_FACE_FLUX, _abi.LBFS_FIELD_FORCE,
                      _abi.LBFS_FIELD_VISC, _abi.LBFS_FIELD_GHOST, _abi.LBFS_FIELD_T1):
            assert rel_err(s.field(which), o.field(which)) < FP64_RTOL, which
    s.step(steps - 1, graph=True)
    o.step(steps - 1)
    for k, (a, b) in enumerate(zip(s.state(), o.state())):
        assert rel_err(a, b) < FP64_RTOL, (k, rel_err(a, b))
    assert rel_err(s.residuals(), o.residuals()) < 1e-8
    if c.membranes:
        assert rel_err(s.nodes(), o.nodes()) < FP64_RTOL
        assert rel_err(s.nodes(_abi.LBFS_NODES_FORCE), o.nodes(_abi.LBFS_NODES_FORCE)) < FP64_RTOL
        assert rel_err(s.totals(), o.totals()) < FP64_RTOL
    assert s.status() == 0
    s.close()
    o.close()


def test_interior_viscosity_l4_vs_oracle():
    # the binned interior-viscosity test (triangles binned by their y-z boxes) against the oracle's
    # test of every triangle: a rotated L4 cell (5120 triangles over many bins), 805 cells inside;
    # the update runs in the second step (t % period == 1)
    c = cases.shear_rbc(n=32, level=4, radius_cells=8.0, rotate=True)
    s, o = make(c), make(c, OracleSolver)
    s.step(2)
    o.step(2)
    a, b = s.field(_abi.LBFS_FIELD_VISC), o.field(_abi.LBFS_FIELD_VISC)
    assert np.count_nonzero(b != 1.0) > 500
    assert rel_err(a, b) < FP64_RTOL
    for x, y in zip(s.state(), o.state()):
        assert rel_err(x, y) < FP64_RTOL
    assert s.status() == 0
    s.close()
    o.close()


def test_axis_faces_vs_oracle_non_cubic():
    compare_with_oracle(cases.poiseuille(n=12, ny=8, nz=10), 25)


def test_general_normal_faces_vs_oracle():
    # the mesh_type 3 path (calc_face_flux with sign-switch upwinding) on the same mesh
    c = cases.poiseuille(n=10, ny=8, nz=6)
    desc = c.mesh.desc
    c.mesh.desc = lambda: _set_general(desc())
    compare_with_oracle(c, 15)


def _set_general(d):
    d.axis_aligned = 0
    return d


def test_periodic_duct_vs_oracle():
    # type-3 ends: ghosts take the partner cell's state (K1) and gradients (boundary-face flux kernel)
    compare_with_oracle(cases.poiseuille(n=10, ny=8, nz=6, periodic_x=True), 20)


def test_periodic_jittered_duct_vs_oracle():
    # general-normal faces everywhere, partners found on the moved centroids
    compare_with_oracle(cases.poiseuille(n=10, ny=8, nz=6, periodic_x=True, jitter=0.15), 12)


def test_periodic_channel_32_vs_oracle():
    # the 32^3 body-force duct with periodic x and seeded +-1e-4 velocity perturbations
    compare_with_oracle(cases.poiseuille(n=32, periodic_x=True), 6, fields=False)


def test_periodic_duct_fp32_bulk_against_fp64():
    a = make(cases.poiseuille(n=16, periodic_x=True))
    b = make(cases.poiseuille(n=16, periodic_x=True, precision=_abi.LBFS_FP32_BULK))
    a.step(40, graph=True)
    b.step(40, graph=True)
    sa, sb = a.state(), b.state()
    assert rel_err(sb[0] - 1.0, sa[0] - 1.0) < 1e-3
    for k in (1, 2, 3):
        assert rel_err(sb[k], sa[k]) < FP32_RTOL, (k, rel_err(sb[k], sa[k]))
    a.close()
    b.close()


def test_periodic_needs_partners_and_no_adjoint():
    c = cases.poiseuille(n=6, ny=5, nz=4, periodic_x=True)
    keep = c.mesh.periodic_node
    c.mesh.periodic_node = None
    with pytest.raises(_abi.LbfsError) as e:
        make(c)
    assert e.value.code == _abi.LBFS_ERR_ARG
    c.mesh.periodic_node = keep.copy()
    c.mesh.periodic_node[np.flatnonzero(c.mesh.bc_rho_type == 3)[0]] = c.mesh.n_cells  # not an interior cell
    with pytest.raises(_abi.LbfsError):
        make(c)
    c.mesh.periodic_node = keep
    s = make(c)
    with pytest.raises(_abi.LbfsError) as e:
        s.adjoint(2, weights=np.ones((c.mesh.n_cells, 3)))
    assert e.value.code == _abi.LBFS_ERR_UNSUPPORTED
    s.close()


def test_peskin4_ibm_vs_oracle():
    compare_with_oracle(cases.shear_rbc(n=20, level=2, radius_cells=3.0, ibm_stencil=_abi.LBFS_IBM_PESKIN4), 8)


def test_hat2_ibm_rotated_cell_vs_oracle():
    compare_with_oracle(cases.shear_rbc(n=20, level=2, radius_cells=3.5, ibm_stencil=_abi.LBFS_IBM_HAT2,
                                        rotate=True), 8)


def test_two_membranes_vs_oracle():
    c = cases.shear_rbc(n=24, level=2, radius_cells=3.0, ibm_stencil=_abi.LBFS_IBM_HAT2)
    first = c.membranes[0]
    moduli = {k: getattr(first, k) for k in ("volume_modulus", "local_area_modulus", "global_area_modulus",
                                             "shear_modulus", "global_bending_modulus", "wlc_ratio",
                                             "internal_viscosity_ratio")}
    X = c.mesh.X
    c.membranes = [red_cell(2, 6.0, (0.3 * X, 0.5 * X, 0.5 * X), **moduli),
                   red_cell(1, 5.0, (0.7 * X, 0.45 * X, 0.55 * X), **moduli)]
    compare_with_oracle(c, 6)


def test_uniform_states_stay_exact_at_full_size():
    c = cases.shear_rbc(n=64)  # the benchmark size
    c.params.body_force = (0.0, 0.0, 0.0)
    c.mesh.set_boundaries({p: (2, 2, 1.0, 0.0, 0.0, 0.0) for p in ("left", "right", "bottom", "top", "back", "front")})
    c.membranes = []
    n = c.mesh.n_cells
    # at rest every face sees the same equilibria: the state stays at rest to rounding
    c.rho, c.u, c.v, c.w = np.full(n, 1.0), np.zeros(n), np.zeros(n), np.zeros(n)
    s = make(c)
    s.step(5, graph=True)
    rho, u, v, w = s.state()
    dev = [float(np.max(np.abs(rho - 1.0))), float(np.max(np.abs(u))), float(np.max(np.abs(v))),
           float(np.max(np.abs(w)))]
    assert dev[0] == 0.0 and max(dev) < 1e-16, dev
    s.close()
    # a uniform stream stays uniform to rounding (tangential wall fluxes cancel only to rounding)
    c.u = np.full(n, 0.013)
    s = make(c)
    s.step(5, graph=True)
    rho, u, v, w = s.state()
    dev = [float(np.max(np.abs(rho - 1.0))), float(np.max(np.abs(u - 0.013))), float(np.max(np.abs(v))),
           float(np.max(np.abs(w)))]
    assert max(dev) < 1e-14, dev
    s.close()


def test_full_size_deterministic_and_graph_equals_eager():
    c = cases.shear_rbc(n=64)  # 64^3 cells, one L3 red cell, 4-point Peskin
    a, b = make(c), make(c)
    a.step(6)
    b.step(6, graph=True)
    for x, y in zip(a.state(), b.state()):
        assert np.array_equal(x, y)
    assert np.array_equal(a.nodes(), b.nodes())
    assert np.array_equal(a.totals(), b.totals())
    assert all(np.isfinite(x).all() for x in a.state())
    a.close()
    b.close()


@pytest.mark.parametrize("builder", ["poiseuille", "shear_rbc", "imported_channel"])
def test_fp32_bulk_against_fp64(builder):
    if builder == "poiseuille":
        c64 = cases.poiseuille(n=16)
        c32 = cases.poiseuille(n=16, precision=_abi.LBFS_FP32_BULK)
    elif builder == "imported_channel":
        # the reference importer's geometry of a jittered mesh: cell faces do not close, so the
        # FP32 form needs its per-cell closure term to stay with the FP64 path
        c64 = cases.jittered_channel(n=16, n_rbc=1, level=2, radius_cells=2.0, closed_faces=False)
        c32 = cases.jittered_channel(n=16, n_rbc=1, level=2, radius_cells=2.0, closed_faces=False,
                                     precision=_abi.LBFS_FP32_BULK)
    else:
        c64 = cases.shear_rbc(n=24, level=2, radius_cells=4.0)
        c32 = cases.shear_rbc(n=24, level=2, radius_cells=4.0, precision=_abi.LBFS_FP32_BULK)
    a, b = make(c64), make(c32)
    a.step(40, graph=True)
    b.step(40, graph=True)
    sa, sb = a.state(), b.state()
    assert rel_err(sb[0] - 1.0, sa[0] - 1.0) < 1e-3  # density deviation from rho0
    for k in (1, 2, 3):
        assert rel_err(sb[k], sa[k]) < FP32_RTOL, (k, rel_err(sb[k], sa[k]))
    if c64.membranes:
        assert rel_err(b.nodes(), a.nodes()) < 1e-9
    a.close()
    b.close()


def test_pipelined_gradients_and_fluxes_are_bit_identical():
    """K1 -> K2 pipelined in chunks of cells on two streams (launch shape flux_chunks) gives the
    same fields and residual norms as the sequential step, bit for bit, at the benchmark size."""
    c = cases.shear_rbc(n=64, level=3, radius_cells=8.0)
    out = []
    for k in (1, 4, 8):
        s = make(c)
        s.set_launch_shape(flux_chunks=k)
        assert s.launch_shape()["flux_chunks"] == k
        s.keep_residuals(True)
        s.step(5, graph=True)
        out.append((s.state(), s.nodes(), s.field(_abi.LBFS_FIELD_FACE_FLUX), s.field(_abi.LBFS_FIELD_RESIDUAL),
                    s.residuals()))
        assert s.status() == 0
        s.close()
    for o in out[1:]:
        for a, b in zip(out[0][0], o[0]):
            assert np.array_equal(a, b)
        for x, y in zip(out[0][1:4], o[1:4]):
            assert np.array_equal(x, y)
        assert np.array_equal(o[4], out[0][4])


@pytest.mark.parametrize("precision,cluster,chunks", [(0, 0, 1), (1, 0, 1), (0, 8, 1), (0, 0, 4)],
                         ids=["fp64", "fp32", "fp64_cluster8", "fp64_chunks4"])
def test_membranes_behind_the_gradient_launch_are_bit_identical(precision, cluster, chunks):
    """Launch shape membrane_after_k1: in a captured step the membrane kernels start behind the
    gradient kernel's launch completion instead of beside it from the step's start; the order changes,
    the results do not (graph steps, several per graph, and eager steps in between)."""
    c = cases.shear_rbc(n=32, level=2, radius_cells=5.0, precision=precision)
    out = []
    for after in (0, 1):
        s = make(c)
        s.set_launch_shape(membrane_after_k1=after, membrane_cluster=cluster, flux_chunks=chunks)
        assert s.launch_shape()["membrane_after_k1"] == after
        s.step(3, graph=True)
        s.step(1)
        s.step(4, graph=True)
        out.append((s.state(), s.nodes(), s.residuals()))
        assert s.status() == 0
        s.close()
    for a, b in zip(out[0][0], out[1][0]):
        assert np.array_equal(a, b)
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])


@pytest.mark.parametrize("precision,shape,period", [(0, {}, 10000), (1, {}, 10000),
                                                   (0, {"membrane_cluster": 8, "membrane_after_k1": 1}, 10000),
                                                   (0, {}, 7)],
                         ids=["fp64", "fp32", "fp64_cluster8_after_k1", "fp64_viscosity_every_7"])
def test_step_until_matches_the_host_loop(precision, shape, period):
    """lbfs_step_until runs the reference's convergence test on the device (a CUDA graph while node
    repeating the step and a check kernel): it stops at the same step as a host loop of single graph
    steps reading the residual norms after each, with the same state and norms, bit for bit; with no
    tolerance it runs every step; a non-finite state stops it after one step."""
    c = cases.shear_rbc(n=32, level=2, radius_cells=5.0, precision=precision)
    c.params.viscosity_period = period  # 7: an interior-viscosity step (one at a time) between every six

    def make_shaped(case):
        h = make(case)
        if shape:
            h.set_launch_shape(**shape)
        return h

    s = make_shaped(c)
    errs = []
    for _ in range(40):
        s.step(1, graph=True)
        errs.append(float(np.max(s.residuals())))
    s.close()
    tol = errs[24] * (1.0 + 1e-12)
    expected = next(i for i, e in enumerate(errs) if e < tol) + 1
    a, b = make_shaped(c), make_shaped(c)
    n, res = a.step_until(40, tol)
    assert n == expected
    for _ in range(expected):
        b.step(1, graph=True)
    assert np.array_equal(res, b.residuals())
    for x, y in zip(a.state(), b.state()):
        assert np.array_equal(x, y)
    assert np.array_equal(a.nodes(), b.nodes())
    n2, _ = a.step_until(7, 0.0)  # no tolerance: all seven
    b.step(7, graph=True)
    assert n2 == 7
    for x, y in zip(a.state(), b.state()):
        assert np.array_equal(x, y)
    a.close()
    b.close()
    d = make_shaped(c)
    d.step(2, graph=True)
    rho, u, v, w = d.state()
    u = u.copy()
    u[123] = np.nan
    d.set_state(rho, u, v, w)
    n3, _ = d.step_until(10, 1e-30)
    assert n3 == 1 and d.status() & _abi.LBFS_FLAG_NONFINITE
    d.close()


def test_nonfinite_state_sets_status_flag():
    c = cases.poiseuille(n=8)
    c.u = c.u.copy()
    c.u[17] = np.nan
    s = make(c)
    s.step(1)
    assert s.status() & _abi.LBFS_FLAG_NONFINITE
    c2 = cases.poiseuille(n=8)
    s2 = make(c2)  # the device context stays usable for a new handle
    s2.step(2)
    assert s2.status() == 0
    s.close()
    s2.close()
