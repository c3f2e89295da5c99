"""Writes the golden fixtures of tests/golden/ by running the REFERENCE itself.

The reference's own sources (unstructured_mesh.cpp, gradients.cpp,
lagrangian_object.cpp and the kernel bodies of LBFS.cu,
immersed_boundary_method.cu, spring_network.cu, common_kernels.cu) are
compiled for the host by oracle/build_ref.sh into oracle/_ref/libref_lbfs.so
and driven by oracle/ref_driver.cpp in the order of the GPU time loop
(Solver_gpu.cu:749-1046).  Run here, where the reference sources exist:

    oracle/build_ref.sh && python tests/golden/make_golden.py

Each fixture stores its inputs as well as the reference's outputs, so the
tests replay them without the reference.
"""
import os
import subprocess
import sys
import tempfile
from dataclasses import replace

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "lbfs-ibm-ade-sp_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import ref_lbfs as R  # noqa: E402
from lbfs_b200 import _abi, cases, icosphere, write_openfoam  # noqa: E402


def ref_case(c):
    m = c.mesh
    rm = R.RefMesh(m.X, m.Y, m.Z, m.dt, m.origin, c.params.visc, mesh_type=m.mesh_type, plateau_width=m.plateau[0],
                   plateau_slope=m.plateau[1], import_dir=m.source)
    p = R.RefParams()
    sp = c.params
    p.visc, p.delta_t, p.gamma_inv, p.channel_diameter = sp.visc, sp.delta_t, sp.gamma_inv, sp.channel_diameter
    p.force[:] = sp.body_force
    p.ref_rho, p.max_velocity, p.testcase = sp.ref_rho, sp.max_velocity, sp.testcase
    p.visc_factor_initial, p.viscosity_period = sp.visc_factor_initial, sp.viscosity_period
    p.time_stepping, p.pre_conditioned_gamma = sp.time_stepping, sp.pre_conditioned_gamma
    p.preconditioning = sp.preconditioning
    p.has_rbc = 1 if c.membranes else 0
    if c.membranes:
        mb = c.membranes[0]
        for k in ("volume_modulus", "local_area_modulus", "global_area_modulus", "shear_modulus",
                  "global_bending_modulus", "local_bending_modulus", "membrane_thickness", "viscosity", "wlc_ratio",
                  "curvature_ratio", "volume_ratio", "internal_viscosity_ratio", "reference_length"):
            setattr(p, k, float(getattr(mb, k)))
        p.pivkin_length, p.sphere_reference = int(mb.pivkin_length), int(mb.sphere_reference)
        p.object_periodic = int(bool(mb.periodic))
    rc = R.RefCase(rm, p, m.bc_rho_type, m.bc_vel_type, m.bc_values)
    rc.set_state(c.rho, c.u, c.v, c.w)
    if c.membranes:
        mb = c.membranes[0]
        rc.set_rbc(mb.tris, mb.springs, mb.xyz_stress_free, mb.xyz_initial)
    return rc


def mesh_fixture(name, X, Y, Z, hybrid=False, mesh_type=6, plateau=(0.0, 0.0)):
    rm = R.RefMesh(X, Y, Z, 1.0, (0.0, 0.0, 0.0), 0.1, hybrid, mesh_type, *plateau)
    arrays = rm.arrays()
    if mesh_type != 4:
        arrays.pop("plateau")
    np.savez_compressed(os.path.join(HERE, name), X=X, Y=Y, Z=Z, hybrid=int(hybrid), mesh_type=mesh_type,
                        plateau_params=np.array(plateau),
                        counts=np.array([rm.n_cells, rm.n_faces, rm.n_interior, rm.n_bc, rm.n_face_x, rm.n_face_y,
                                         rm.n_face_z, rm.total_cells]), **arrays)


def spring_fixture(name, level):
    unit, tris = icosphere(level, 1.0)
    nodes = unit * 8.0
    spr, tri, xyz = R.ref_springs(nodes, tris, (10.0, 20.0, 30.0))
    np.savez_compressed(os.path.join(HERE, name), nodes=nodes, tris=tris, ref_springs=spr, ref_tris=tri, ref_xyz=xyz)


def icosphere_fixture():
    """Unit level-2 and level-3 icospheres (nodes, outward triangles): the red
    cells of the reference arm's workload and of the reference's own decks
    (oracle/ref_cases.py, oracle/ref_deck.py), which load no code of this
    repository."""
    for level in (2, 3):
        unit, tris = icosphere(level, 1.0)
        np.savez_compressed(os.path.join(HERE, f"icosphere_L{level}.npz"), unit_nodes=unit, tris=tris)


def plateau_case():
    return cases.shear_rbc(n=16, level=2, radius_cells=3.0, ibm_stencil=_abi.LBFS_IBM_VANDERMONDE4, mesh_type=4,
                           plateau=(5.0, 0.3))


def step_fixture(name, case, steps):
    rc = ref_case(case)
    out = dict(rho0=case.rho, u0=case.u, v0=case.v, w0=case.w)
    if case.membranes:
        mb = case.membranes[0]
        out.update(tris=mb.tris, springs=mb.springs, xyz_stress_free=mb.xyz_stress_free, xyz_initial=mb.xyz_initial,
                   init_totals=rc.get(R.REF_TOTALS), init_spring=rc.get(R.REF_SPRING))
    rc.step(1)
    out.update(s1_grad=rc.get(R.REF_GRAD), s1_flux=rc.get(R.REF_RES_FACE), s1_res=rc.get(R.REF_RES),
               s1_force=rc.get(R.REF_FORCE), s1_ghost=rc.get(R.REF_GHOST), s1_t1=rc.get(R.REF_T1),
               s1_state=np.stack(rc.state()), s1_resid=rc.get(R.REF_RESID), time_stepping=case.params.time_stepping,
               s1_dtl=rc.get(R.REF_DT_LOCAL), s1_dt=rc.get(R.REF_DELTA_T)[0], gamma_inv=case.params.gamma_inv,
               preconditioning=case.params.preconditioning)
    if case.membranes:
        out.update(s1_nodes_x=rc.get(R.REF_NODE_X), s1_nodes_v=rc.get(R.REF_NODE_V), s1_nodes_f=rc.get(R.REF_NODE_F),
                   s1_totals=rc.get(R.REF_TOTALS), s1_visc=rc.get(R.REF_VISC), s1_spring=rc.get(R.REF_SPRING),
                   s1_energy=rc.get(R.REF_ENERGY))
    rc.step(steps - 1)
    out.update(sN_state=np.stack(rc.state()), sN_resid=rc.get(R.REF_RESID), steps=steps,
               sN_dtl=rc.get(R.REF_DT_LOCAL), sN_dt=rc.get(R.REF_DELTA_T)[0])
    if case.membranes:
        out.update(sN_nodes_x=rc.get(R.REF_NODE_X), sN_nodes_f=rc.get(R.REF_NODE_F), sN_totals=rc.get(R.REF_TOTALS),
                   sN_visc=rc.get(R.REF_VISC), sN_energy=rc.get(R.REF_ENERGY))
    np.savez_compressed(os.path.join(HERE, name), **out)


def main():
    if not R.available():
        sys.exit("oracle/_ref/libref_lbfs.so is missing: run oracle/build_ref.sh first")
    mesh_fixture("mesh_4x3x5.npz", 8.0, 6.0, 10.0)
    mesh_fixture("mesh_6x6x6_hybrid.npz", 12.0, 12.0, 12.0, hybrid=True)
    # the generator's other rectilinear meshes: cosine in x, y, z (5), cosine in x, y (7); the plateau
    # mesh (4) in a process of its own, below
    mesh_fixture("mesh_cosine5_8x6x5.npz", 16.0, 12.0, 10.0, mesh_type=5)
    mesh_fixture("mesh_cosine7_8x6x5.npz", 16.0, 12.0, 10.0, mesh_type=7)
    spring_fixture("springs_L1.npz", 1)
    spring_fixture("springs_L2.npz", 2)
    spring_fixture("springs_L3.npz", 3)
    icosphere_fixture()
    step_fixture("step_poiseuille_6x5x4.npz", cases.poiseuille(n=6, ny=5, nz=4), 20)
    step_fixture("step_shear_rbc_16.npz",
                 cases.shear_rbc(n=16, level=2, radius_cells=3.0, ibm_stencil=_abi.LBFS_IBM_HAT2), 10)
    # time stepping other than constant (get_cfl_device + min, Solver_gpu.cu:767-787)
    for name, mode in (("local", _abi.LBFS_DT_LOCAL), ("talts", _abi.LBFS_DT_TALTS)):
        c = cases.poiseuille(n=6, ny=5, nz=4)
        c.params = replace(c.params, time_stepping=mode)
        step_fixture(f"step_poiseuille_6x5x4_{name}.npz", c, 20)
    c = cases.shear_rbc(n=16, level=2, radius_cells=3.0, ibm_stencil=_abi.LBFS_IBM_HAT2)
    c.params = replace(c.params, time_stepping=_abi.LBFS_DT_MIN)
    step_fixture("step_shear_rbc_16_min.npz", c, 10)
    # a periodic object above 0.75 Z: check_periodic_object moves it down by Z / 2 after step t = 1
    step_fixture("step_shear_rbc_16_wrap.npz",
                 cases.shear_rbc(n=16, level=2, radius_cells=3.0, ibm_stencil=_abi.LBFS_IBM_HAT2,
                                 centre=(0.5, 0.5, 0.8), periodic_object=True), 4)
    # preconditioning: gamma = 2 in the relaxation, the interface and the
    # boundary faces' lattice equilibria, with local time stepping
    c = cases.poiseuille(n=6, ny=5, nz=4)
    c.params = replace(c.params, gamma_inv=0.5, preconditioning=1, time_stepping=_abi.LBFS_DT_LOCAL)
    step_fixture("step_poiseuille_6x5x4_precond.npz", c, 20)
    # OpenFOAM polyMesh: a jittered mesh written by lbfs_mesh_write_openfoam (kept as a fixture) and
    # read by the reference's importer; steps on imported meshes take the general-normal flux
    foam = os.path.join(HERE, "polymesh_jitter_8x6x5")
    os.makedirs(foam, exist_ok=True)
    write_openfoam(foam, 16.0, 12.0, 10.0, 1.0, jitter=0.1, seed=5)
    for hybrid in (False, True):
        rm = R.RefMesh(16.0, 12.0, 10.0, 1.0, (0.0, 0.0, 0.0), 0.1, hybrid, 3, 0.0, 0.0, foam)
        np.savez_compressed(os.path.join(HERE, f"mesh_foam_jitter_8x6x5{'_hybrid' if hybrid else ''}.npz"),
                            hybrid=int(hybrid), counts=np.array([rm.n_cells, rm.n_faces, rm.n_interior, rm.n_bc]),
                            **rm.arrays())
    with tempfile.TemporaryDirectory() as d:
        step_fixture("step_foam_duct_8x6x5.npz", cases.imported(cases.poiseuille(n=8, ny=6, nz=5), d), 20)
    with tempfile.TemporaryDirectory() as d:
        # no interior-viscosity update: on imported meshes the reference reads an
        # uninitialised delta_h there (unstructured_mesh.h:61 is set only by the generator)
        c = cases.shear_rbc(n=16, level=2, radius_cells=3.0, ibm_stencil=_abi.LBFS_IBM_HAT2)
        c.params = replace(c.params, viscosity_period=0)
        step_fixture("step_foam_shear_rbc_16.npz", cases.imported(c, d), 10)
    subprocess.run([sys.executable, os.path.abspath(__file__), "--plateau"], check=True)
    print("golden fixtures written to", HERE)


def plateau_fixtures():
    """The plateau mesh (mesh_type 4) and a step on it with the 4x4x4 Vandermonde IBM.

    create_uniform_openfoam_mesh initialises plateau_sum_x but not plateau_sum_y
    and plateau_sum_z (unstructured_mesh.cpp:296-317), so the reference's y and z
    plateau arrays depend on what those reads return.  This runs in a fresh
    process (where they read 0, the value plateau_sum_x starts from) and checks
    that every plateau array ends at the domain length before writing."""
    rm = R.RefMesh(20.0, 16.0, 12.0, 1.0, (0.0, 0.0, 0.0), 0.1, False, 4, 2.0, 0.6)
    pl = rm.arrays()["plateau"]
    ends = np.cumsum([11, 9, 7]) - 1
    if not np.allclose(pl[ends], (20.0, 16.0, 12.0), rtol=0, atol=1e-9):
        sys.exit("the reference's plateau sums were not zero-initialised in this process; not writing fixtures")
    mesh_fixture("mesh_plateau_10x8x6.npz", 20.0, 16.0, 12.0, mesh_type=4, plateau=(2.0, 0.6))
    c = plateau_case()
    g = R.RefMesh(c.mesh.X, c.mesh.Y, c.mesh.Z, 1.0, (0.0, 0.0, 0.0), c.params.visc, False, 4, *c.mesh.plateau)
    if not np.array_equal(g.arrays()["plateau"], np.concatenate(c.mesh.grid)):
        sys.exit("plateau arrays of the step case differ from the builder's; not writing fixtures")
    step_fixture("step_plateau_rbc_16.npz", c, 10)


if __name__ == "__main__":
    if "--plateau" in sys.argv:
        plateau_fixtures()
    else:
        main()
