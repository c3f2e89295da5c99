"""XML decks in the reference's own input format (test and bench infrastructure).

The reference reads its whole configuration from one XML file through
preprocessor::initialise_program_variables (preprocessor.cpp:27-51): global
variables, geometry, initial conditions, the structured and unstructured
boundary conditions and the lagrangian objects, every key that preprocessor.cpp
reads (no <?xml ?> declaration).  Velocities in the deck are in units of the
Mach number (mach_number_factor, preprocessor.cpp:53-84, multiplies the
unstructured boundary values by mach_no / scale), and the viscosity follows
from nu = mach_no * ref_length / reynolds_no (global_variables::initialise).

shear_rbc_deck writes the wall-driven shear workload with one red cell:
n^3 cells of width 2 (streaming_dt 1), walls at y = 0 and y = Y moving with
u = y * gamma_dot (velocity type "shear"), zero-gradient elsewhere, the red
cell's stress-free sphere and initial biconcave shape as Osay files
(lagrangian_object::osay_mesh_read / read_initial_mesh: "n_nodes n_tris", node
coordinates relative to the centre, 1-based triangles), and the seeded initial
state as a binary file for oracle/ref_program.cpp (rho, u, v, w planes).
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(os.path.dirname(HERE), "tests", "golden")
EVANS_FUNG = (0.2072, 2.0026, -1.1228)


def _icosphere(level):
    g = np.load(os.path.join(GOLDEN, f"icosphere_L{level}.npz"))
    return g["unit_nodes"], g["tris"]


def _osay(path, nodes, tris):
    with open(path, "w") as f:
        f.write(f"{len(nodes)} {len(tris)}\n")
        for p in nodes:
            f.write(f"{p[0]:.17g} {p[1]:.17g} {p[2]:.17g}\n")
        for t in tris:
            f.write(f"{t[0] + 1} {t[1] + 1} {t[2] + 1}\n")


def _bc(name, vel_type, rho_type, u=0.0, v=0.0, w=0.0, rho=1.0):
    return (f"<bc><name>{name}</name><rho>{rho!r}</rho><u>{u!r}</u><v>{v!r}</v><w>{w!r}</w>"
            f"<vel_type>{vel_type}</vel_type><rho_type>{rho_type}</rho_type></bc>")


def _seeded_state(n, seed, u0_of_y=None, dt=1.0):
    """rho0 = 1, velocities U(-1e-4, 1e-4) (+ u0(y) in u) on the lexicographic grid's cell centroids
    (cell i + n j + n^2 k at ((i + 1/2) 2 dt, ...)), as rho, u, v, w planes."""
    rng = np.random.default_rng(seed)
    nc = n ** 3
    u = rng.uniform(-1e-4, 1e-4, nc)
    v = rng.uniform(-1e-4, 1e-4, nc)
    w = rng.uniform(-1e-4, 1e-4, nc)
    if u0_of_y is not None:
        u = u + u0_of_y((np.arange(nc) // n % n + 0.5) * 2.0 * dt)
    return np.concatenate([np.full(nc, 1.0), u, v, w])


def poiseuille_deck(directory, n=32, steps=20, u_centre=0.01, seed=1234, tau=0.8, delta_t=0.5, cpu_solver=False,
                    tolerance=0.0):
    """The body-force-driven square duct on n^3 cells without a red cell (testcase 2): no-slip walls in y
    and z (velocity type dirichlet), zero-gradient x ends, force along x for a centreline speed u_centre
    (series solution of the square duct); the seeded +-1e-4 velocity perturbation.  cpu_solver selects
    the reference's CPU Solver (gpu_solver 0).  The deck still names a spring-network object (program
    set-up initialises object 0 whatever the test case)."""
    os.makedirs(directory, exist_ok=True)
    dt = 1.0
    L = 2.0 * n
    visc = (tau - 0.5) / 3.0 * dt
    a = 0.5 * L
    force = u_centre * visc / (0.2947 * a * a)
    unit, tris = _icosphere(2)
    sf_path = os.path.join(directory, "stress_free.dat")
    _osay(sf_path, unit * 2.0, tris)
    state_path = os.path.join(directory, "state0.bin")
    _seeded_state(n, seed, dt=dt).astype(np.float64).tofile(state_path)
    bcs = "".join([_bc("left", "neumann", "neumann"), _bc("right", "neumann", "neumann")] +
                  [_bc(p, "dirichlet", "neumann") for p in ("bottom", "top", "back", "front")])
    deck = _deck(directory, L, dt, steps, delta_t, mach=u_centre, visc=visc, testcase=2, force=force, bcs=bcs,
                 tolerance=tolerance,
                 obj=(f"<name>dummy</name><num_nodes>{len(unit)}</num_nodes><radius>2.0</radius><depth>0.0</depth>"
                      f"<stiffness>0.0</stiffness><centre_x>{0.5 * L!r}</centre_x><centre_y>{0.5 * L!r}</centre_y>"
                      f"<centre_z>{0.5 * L!r}</centre_z><type>spring_network</type><mesh_file>{sf_path}</mesh_file>"
                      "<local_area_modulus>0.0</local_area_modulus><global_area_modulus>0.0</global_area_modulus>"
                      "<volume_modulus>0.0</volume_modulus><shear_modulus>0.0</shear_modulus>"
                      "<local_bending_modulus>0.0</local_bending_modulus><global_bending_modulus>0.0</global_bending_modulus>"
                      "<viscosity>0.0</viscosity><wlc_ratio>2.2</wlc_ratio><curvature_ratio>0.0</curvature_ratio>"
                      f"<stress_free_mesh>{sf_path}</stress_free_mesh><curvature_mesh>{sf_path}</curvature_mesh>"),
                 gpu_solver=0 if cpu_solver else 1)
    deck_path = os.path.join(directory, "deck.xml")
    with open(deck_path, "w") as f:
        f.write(deck)
    return deck_path, state_path, {"n_cells": n ** 3, "steps": steps, "visc": visc, "force": force}


def _deck(directory, L, dt, steps, delta_t, mach, visc, testcase, force, bcs, obj, gpu_solver=1, output_step=None,
          tolerance=0.0):
    zero3 = "<x>0.0</x><y>0.0</y><z>0.0</z>"
    quad = "".join(f"<{side}><rho>1.0</rho><u>0.0</u><v>0.0</v><vel_type>dirichlet</vel_type>"
                   f"<rho_type>neumann</rho_type></{side}>" for side in ("west", "east", "north", "south"))
    reynolds = mach * L / visc  # nu = mach * ref_length / Re
    return (
        "<lbfs>"
        "<global_variables>"
        f"<tolerance>{tolerance!r}</tolerance><pre_condition_gamma>1.0</pre_condition_gamma>"
        f"<simulation_length>{steps}</simulation_length><time_marching_step>{delta_t!r}</time_marching_step>"
        f"<reynolds_no>{reynolds!r}</reynolds_no><mach_no>{mach!r}</mach_no>"
        f"<simulation_name>case</simulation_name><output_directory>{os.path.join(directory, 'out')}/</output_directory>"
        "<max_multi_grid_levels>0</max_multi_grid_levels><FMG_levels>0</FMG_levels><FMG_tolerance>0.0</FMG_tolerance>"
        "<dissipation_kappa_2>0.0</dissipation_kappa_2><dissipation_kappa_4>0.0</dissipation_kappa_4>"
        f"<martinelli_exponent>0.0</martinelli_exponent><testcase>{testcase}</testcase><mesh_type>6</mesh_type>"
        f"<scale>1.0</scale><womersley_no>0.0</womersley_no><output_step>{output_step or steps + 10}</output_step>"
        "<import_file>none</import_file><import_format>openfoam</import_format><gradient_calc>LS</gradient_calc>"
        "<restart_analysis>false</restart_analysis><time_stepping>constant</time_stepping>"
        f"<preconditioning>false</preconditioning><gpu_solver>{gpu_solver}</gpu_solver><fneq_min>0.0</fneq_min>"
        "<gpu_device>0</gpu_device>"
        "</global_variables>"
        "<geometry>"
        f"<x>{L!r}</x><y>{L!r}</y><z>{L!r}</z><dx>2.0</dx><dy>2.0</dy><dz>2.0</dz><streaming_dt>{dt!r}</streaming_dt>"
        f"<origin_x>0.0</origin_x><origin_y>0.0</origin_y><origin_z>0.0</origin_z><ref_length>{L!r}</ref_length>"
        "<plateau_slope>0.0</plateau_slope><plateau_width>0.0</plateau_width><IBM_face>none</IBM_face>"
        "</geometry>"
        "<initial_conditions>"
        f"<average_rho>1.0</average_rho><pressure_gradient>{force!r}</pressure_gradient>"
        "<pressure_direction>x</pressure_direction>"
        f"<rho><gradient>{zero3}</gradient><origin_magnitude>{zero3}</origin_magnitude></rho>"
        f"<origin_location>{zero3}</origin_location>"
        f"<vel><gradient>{zero3}</gradient><origin_magnitude>{zero3}</origin_magnitude></vel>"
        "<u>0.0</u><v>0.0</v><w>0.0</w>"
        "</initial_conditions>"
        f"<boundary_conditions>{quad}</boundary_conditions>"
        f"<uns_boundary_conditions>{bcs}<periodic_translation>{zero3}</periodic_translation></uns_boundary_conditions>"
        f"<lagrangian_objects><object>{obj}<sphere_reference>false</sphere_reference><mz_importer>false</mz_importer>"
        "</object></lagrangian_objects>"
        "</lbfs>\n")


def shear_rbc_deck(directory, n=16, steps=10, level=3, radius_cells=3.0, capillary=0.1, u_wall=0.02, seed=4321,
                   tau=0.8, delta_t=0.5, output_step=None):
    """Deck, membrane files and initial state of the shear + red-cell workload on n^3 cells
    (the parameters of the CUDA path's cases.shear_rbc with the reference's 2-point IBM).
    Returns the paths (deck, state) and a dict of the workload's numbers."""
    os.makedirs(directory, exist_ok=True)
    dt = 1.0
    L = 2.0 * n
    visc = (tau - 0.5) / 3.0 * dt
    gamma = u_wall / L
    R = radius_cells * 2.0 * dt
    gs = visc * gamma * R / capillary
    mach = u_wall                    # the velocity scale: deck velocities are multiples of it
    unit, tris = _icosphere(level)
    sphere = unit * R
    c0, c1, c2 = EVANS_FUNG
    x, y, z = unit[:, 0], unit[:, 1], unit[:, 2]
    r2 = np.clip(x * x + y * y, 0.0, 1.0)
    disc = np.stack([R * x, R * y, np.sign(z) * 0.5 * R * np.sqrt(1.0 - r2) * (c0 + c1 * r2 + c2 * r2 * r2)], axis=1)
    sf_path, init_path = os.path.join(directory, "stress_free.dat"), os.path.join(directory, "initial.dat")
    _osay(sf_path, sphere, tris)
    _osay(init_path, disc, tris)
    state_path = os.path.join(directory, "state0.bin")
    _seeded_state(n, seed, u0_of_y=lambda y: gamma * y, dt=dt).astype(np.float64).tofile(state_path)
    nc = n ** 3
    shear = gamma / mach  # wall velocity per unit y, in Mach units
    bcs = "".join([_bc("left", "neumann", "neumann"), _bc("right", "neumann", "neumann"),
                   _bc("bottom", "shear", "neumann", u=shear), _bc("top", "shear", "neumann", u=shear),
                   _bc("back", "neumann", "neumann"), _bc("front", "neumann", "neumann")])
    moduli = dict(volume_modulus=500.0 * gs, local_area_modulus=10.0 * gs, global_area_modulus=500.0 * gs,
                  shear_modulus=gs, global_bending_modulus=0.05 * gs * R * R, local_bending_modulus=0.0,
                  membrane_thickness=1.0, viscosity=0.0, wlc_ratio=2.2, internal_viscosity_ratio=5.0,
                  volume_ratio=1.0, curvature_ratio=0.0)
    obj = (f"<name>rbc</name><num_nodes>{len(unit)}</num_nodes><radius>{R!r}</radius><depth>0.0</depth>"
           f"<stiffness>0.0</stiffness><centre_x>{0.5 * L!r}</centre_x><centre_y>{0.5 * L!r}</centre_y>"
           f"<centre_z>{0.5 * L!r}</centre_z><type>spring_network</type><mesh_file>{init_path}</mesh_file>"
           + "".join(f"<{k}>{v!r}</{k}>" for k, v in moduli.items())
           + f"<stress_free_mesh>{sf_path}</stress_free_mesh><curvature_mesh>{sf_path}</curvature_mesh>")
    deck = _deck(directory, L, dt, steps, delta_t, mach=mach, visc=visc, testcase=5, force=0.0, bcs=bcs, obj=obj,
                 output_step=output_step)
    deck_path = os.path.join(directory, "deck.xml")
    with open(deck_path, "w") as f:
        f.write(deck)
    return deck_path, state_path, {"n_cells": nc, "n_nodes": len(unit), "steps": steps, "visc": visc,
                                   "gamma_dot": gamma, "shear_modulus": gs}
