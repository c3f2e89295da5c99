"""The C restatement oracle reproduces the reference's own kernels (golden
fixtures produced by the reference sources compiled for the host)."""
import tempfile
from dataclasses import replace

import numpy as np
import pytest

from helpers import FP64_RTOL, rel_err
from lbfs_b200 import _abi, cases
from oracle_lbfs import OracleSolver


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
        assert np.array_equal(mb.tris, g["tris"]) and np.array_equal(mb.springs, g["springs"])
        mb.xyz_stress_free = g["xyz_stress_free"]
        mb.xyz_initial = g["xyz_initial"]
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
def test_oracle_matches_reference(golden, name):
    c, g = fixture_case(golden, name)
    o = OracleSolver(c.mesh, c.params, c.membranes)
    o.set_state(c.rho, c.u, c.v, c.w)
    if c.membranes:
        assert rel_err(o.totals()[0], g["init_totals"]) < FP64_RTOL
        assert rel_err(o.field(_abi.LBFS_FIELD_SPRING), g["init_spring"]) < FP64_RTOL
    o.step(1)
    checks = {
        "grad": (o.field(_abi.LBFS_FIELD_GRADIENTS), g["s1_grad"]),
        "flux": (o.field(_abi.LBFS_FIELD_FACE_FLUX), g["s1_flux"]),
        "res": (o.field(_abi.LBFS_FIELD_RESIDUAL), g["s1_res"]),
        "force": (o.field(_abi.LBFS_FIELD_FORCE), g["s1_force"]),
        "ghost": (o.field(_abi.LBFS_FIELD_GHOST), g["s1_ghost"]),
        "t1": (o.field(_abi.LBFS_FIELD_T1), g["s1_t1"]),
        "resid": (o.residuals(), g["s1_resid"]),
        "dt_local": (o.field(_abi.LBFS_FIELD_DT_LOCAL), g["s1_dtl"]),
        "dt": (np.array([o.time_step()]), np.array([g["s1_dt"]])),
    }
    for k, arr in enumerate(o.state()):
        checks[f"state{k}"] = (arr, g["s1_state"][k])
    if c.membranes:
        checks["nodes_x"] = (o.nodes(_abi.LBFS_NODES_POSITION).ravel(), g["s1_nodes_x"])
        checks["nodes_v"] = (o.nodes(_abi.LBFS_NODES_VELOCITY).ravel(), g["s1_nodes_v"])
        checks["nodes_f"] = (o.nodes(_abi.LBFS_NODES_FORCE).ravel(), g["s1_nodes_f"])
        checks["totals"] = (o.totals()[0], g["s1_totals"])
        checks["visc"] = (o.field(_abi.LBFS_FIELD_VISC), g["s1_visc"])
        checks["spring"] = (o.field(_abi.LBFS_FIELD_SPRING), g["s1_spring"])
        checks["energy"] = (o.energies()[0], g["s1_energy"])
    for key, (a, b) in checks.items():
        assert rel_err(a, b) < FP64_RTOL, (key, rel_err(a, b))
    o.step(int(g["steps"]) - 1)
    for k, arr in enumerate(o.state()):
        assert rel_err(arr, g["sN_state"][k]) < FP64_RTOL, (k, rel_err(arr, g["sN_state"][k]))
    assert rel_err(o.field(_abi.LBFS_FIELD_DT_LOCAL), g["sN_dtl"]) < FP64_RTOL
    assert rel_err(o.time_step(), g["sN_dt"]) < FP64_RTOL
    if c.membranes:
        assert rel_err(o.nodes(_abi.LBFS_NODES_POSITION).ravel(), g["sN_nodes_x"]) < FP64_RTOL
        assert rel_err(o.nodes(_abi.LBFS_NODES_FORCE).ravel(), g["sN_nodes_f"]) < FP64_RTOL
        assert rel_err(o.totals()[0], g["sN_totals"]) < FP64_RTOL
        assert rel_err(o.field(_abi.LBFS_FIELD_VISC), g["sN_visc"]) < FP64_RTOL
        assert rel_err(o.energies()[0], g["sN_energy"]) < FP64_RTOL
