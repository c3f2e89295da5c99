"""The benchmark workloads built for the reference alone (test and bench
infrastructure).

bench.py's reference arm times the reference's own code (oracle/_ref) and must
not load this repository's library, so the inputs are formed here from the
reference's own builders and numpy only:

* the mesh from the reference's generator (unstructured_mesh, mesh_type 6,
  through ref_lbfs.RefMesh);
* the boundary tables from the patch of every boundary face (the sign of its
  unit normal: left/right = -x/+x, bottom/top = -y/+y, back/front = -z/+z), as
  Boundary_Conditions::assign_boundary_conditions fills them per patch;
* the red cell from the committed level-3 icosphere (tests/golden/icosphere_L3.npz:
  unit-sphere nodes and outward triangles), its Evans-Fung biconcave map, and
  the spring table from the reference's lagrangian_object (ref_lbfs.ref_springs);
* the seeded initial state (numpy default_rng, the same draws as the
  workload's own set-up).

tests/test_ref_cases.py checks that these inputs equal the ones the CUDA path's
workload builder forms, array for array.
"""
import os

import numpy as np

import ref_lbfs as R

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(os.path.dirname(HERE), "tests", "golden")
EVANS_FUNG = (0.2072, 2.0026, -1.1228)
PATCHES = ("left", "right", "bottom", "top", "back", "front")


def boundary_tables(arrays, n_interior, spec):
    """bc_rho_type, bc_vel_type, bc_values (u, v, w, rho) per boundary face from the
    patch spec {patch: (rho_type, vel_type, rho, u, v, w)}."""
    n = arrays["face_normal"][n_interior:]
    axis = np.argmax(np.abs(n), axis=1)
    patch = 2 * axis + (n[np.arange(len(n)), axis] > 0)
    rt = np.zeros(len(n), np.int32)
    vt = np.zeros(len(n), np.int32)
    vals = np.zeros((len(n), 4))
    for p, name in enumerate(PATCHES):
        rho_type, vel_type, rho, u, v, w = spec[name]
        sel = patch == p
        rt[sel], vt[sel], vals[sel] = rho_type, vel_type, (u, v, w, rho)
    return rt, vt, vals


def initial_state(n_cells, seed, amplitude=1e-4, u0=None):
    rng = np.random.default_rng(seed)
    rho = np.full(n_cells, 1.0)
    u = rng.uniform(-amplitude, amplitude, n_cells)
    v = rng.uniform(-amplitude, amplitude, n_cells)
    w = rng.uniform(-amplitude, amplitude, n_cells)
    if u0 is not None:
        u = u + u0
    return rho, u, v, w


def red_cell_l3(radius, centre):
    """Stress-free sphere and biconcave initial shape of the level-3 red cell, its
    triangles, and sprIdx from the reference's lagrangian_object."""
    g = np.load(os.path.join(GOLDEN, "icosphere_L3.npz"))
    unit, tris = g["unit_nodes"], g["tris"]
    c0, c1, c2 = EVANS_FUNG
    x, y, z = unit[:, 0], unit[:, 1], unit[:, 2]
    r2 = np.clip(x * x + y * y, 0.0, 1.0)
    zz = np.sign(z) * 0.5 * radius * np.sqrt(1.0 - r2) * (c0 + c1 * r2 + c2 * r2 * r2)
    disc = np.stack([radius * x, radius * y, zz], axis=1)
    c = np.asarray(centre, np.float64)
    sphere = unit * radius + c
    initial = disc + c
    springs, _, _ = R.ref_springs(unit * radius, tris)
    return np.ascontiguousarray(tris), springs, np.ascontiguousarray(sphere), np.ascontiguousarray(initial)


def shear_rbc(n=64, radius_cells=8.0, capillary=0.1, u_wall=0.02, seed=4321, tau=0.8, delta_t=0.5):
    """Wall-driven shear on n^3 cells with one L3 red cell at the centre (the
    reference's 2-point hat IBM: its uniform-mesh kernels have no other stencil).
    Returns (RefCase, n_cells, n_nodes)."""
    dt = 1.0
    visc = (tau - 0.5) / 3.0 * dt
    L = 2.0 * n
    mesh = R.RefMesh(L, L, L, dt, (0.0, 0.0, 0.0), visc)
    A = mesh.arrays()
    gamma = u_wall / L
    spec = {"left": (2, 2, 1.0, 0.0, 0.0, 0.0), "right": (2, 2, 1.0, 0.0, 0.0, 0.0),
            "bottom": (2, 10, 1.0, gamma, 0.0, 0.0), "top": (2, 10, 1.0, gamma, 0.0, 0.0),
            "back": (2, 2, 1.0, 0.0, 0.0, 0.0), "front": (2, 2, 1.0, 0.0, 0.0, 0.0)}
    rt, vt, vals = boundary_tables(A, mesh.n_interior, spec)
    Rr = radius_cells * 2.0 * dt
    gs = visc * gamma * Rr / capillary
    p = R.RefParams()
    p.visc, p.delta_t, p.gamma_inv, p.channel_diameter = visc, delta_t, 1.0, L
    p.force[:] = (0.0, 0.0, 0.0)
    p.ref_rho, p.max_velocity, p.testcase = 1.0, u_wall, 5
    p.visc_factor_initial, p.viscosity_period = 1.0, 10000
    p.time_stepping, p.pre_conditioned_gamma, p.preconditioning = 2, 0.0, 0  # 2: constant
    p.has_rbc = 1
    moduli = dict(volume_modulus=500.0 * gs, local_area_modulus=10.0 * gs, global_area_modulus=500.0 * gs,
                  shear_modulus=gs, global_bending_modulus=0.05 * gs * Rr * Rr, local_bending_modulus=0.0,
                  membrane_thickness=1.0, viscosity=0.0, wlc_ratio=2.2, curvature_ratio=0.0, volume_ratio=1.0,
                  internal_viscosity_ratio=5.0, reference_length=0.0)
    for k, v in moduli.items():
        setattr(p, k, float(v))
    p.pivkin_length, p.sphere_reference, p.object_periodic = 0, 1, 0
    rc = R.RefCase(mesh, p, rt, vt, vals)
    y = A["cell_centroid"][: mesh.n_cells, 1]
    rc.set_state(*initial_state(mesh.n_cells, seed, u0=gamma * y))
    tris, springs, sphere, initial = red_cell_l3(Rr, (0.5 * L, 0.5 * L, 0.5 * L))
    rc.set_rbc(tris, springs, sphere, initial)
    return rc, mesh.n_cells, len(sphere)
