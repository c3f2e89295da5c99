"""Seeded synthetic workloads (the reference ships no input decks or meshes).

poiseuille : 3D square-duct channel driven by a body force along x; no-slip
             walls in y and z (bc velocity type 1), zero-gradient (type 2) at
             the x ends, which matches an x-periodic duct once developed.
shear_rbc  : wall-driven simple shear (bc velocity type 10, u = y * gamma_dot
             on the y walls) with one red cell: a level-L icosphere of radius R
             cells as the stress-free shape and its Evans-Fung biconcave map as
             the initial shape, at the domain centre.

Lengths are in the reference's units: a cell is 2 * dt wide (dt = streaming
step = 1), so a domain of n cells per axis has X = 2 n.
"""
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .mesh import build_uniform_mesh, import_openfoam, write_openfoam
from .rbc import red_cell, rotation_matrix
from .solver import StepParams


@dataclass
class Case:
    name: str
    mesh: object
    params: StepParams
    membranes: list
    rho: np.ndarray
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    bcs: dict
    info: dict = field(default_factory=dict)


def _initial_state(n_cells, seed, amplitude=1e-4, rho0=1.0, u0=None):
    rng = np.random.default_rng(seed)
    rho = np.full(n_cells, rho0)
    u = rng.uniform(-amplitude, amplitude, n_cells)
    v = rng.uniform(-amplitude, amplitude, n_cells)
    w = rng.uniform(-amplitude, amplitude, n_cells)
    if u0 is not None:
        u = u + u0
    return rho, u, v, w


def poiseuille(n=32, seed=1234, tau=0.8, u_centre=0.01, delta_t=0.5, precision=_abi.LBFS_FP64, ny=None, nz=None,
               periodic_x=False, jitter=0.0, mesh_seed=1):
    """Body-force-driven square duct, n x ny x nz cells (default cube).  The x ends are
    Neumann (type 2), or periodic (type 3, translation X along x) with periodic_x; jitter > 0
    moves the interior vertices (general-normal fluxes, closed faces)."""
    ny = ny or n
    nz = nz or n
    dt = 1.0
    visc = (tau - 0.5) / 3.0 * dt
    mesh = build_uniform_mesh(2.0 * n, 2.0 * ny, 2.0 * nz, dt, visc=visc, jitter=jitter, seed=mesh_seed)
    end = (3, 3, 1.0, 0.0, 0.0, 0.0) if periodic_x else (2, 2, 1.0, 0.0, 0.0, 0.0)
    bcs = {"left": end, "right": end,
           "bottom": (2, 1, 1.0, 0.0, 0.0, 0.0), "top": (2, 1, 1.0, 0.0, 0.0, 0.0),
           "back": (2, 1, 1.0, 0.0, 0.0, 0.0), "front": (2, 1, 1.0, 0.0, 0.0, 0.0)}
    mesh.set_boundaries(bcs, periodic_translation=(2.0 * n, 0.0, 0.0) if periodic_x else None)
    # square duct of half-width a: u_max = 0.2947 f a^2 / (rho nu)  (series solution)
    a = 0.5 * 2.0 * min(ny, nz)
    force = u_centre * visc / (0.2947 * a * a)
    params = StepParams(visc=visc, delta_t=delta_t, channel_diameter=2.0 * ny, body_force=(force, 0.0, 0.0),
                        ref_rho=1.0, max_velocity=u_centre, rho0=1.0, visc_factor_initial=1.0, testcase=2,
                        precision=precision, viscosity_period=0)
    rho, u, v, w = _initial_state(mesh.n_cells, seed)
    return Case("poiseuille", mesh, params, [], rho, u, v, w, bcs,
                {"n": (n, ny, nz), "tau": tau, "force": force, "u_centre": u_centre})


def shear_rbc(n=64, level=3, radius_cells=8.0, capillary=0.1, u_wall=0.02, seed=4321, tau=0.8, delta_t=0.5,
              precision=_abi.LBFS_FP64, ibm_stencil=_abi.LBFS_IBM_PESKIN4, n_cells_y=None, n_cells_z=None,
              rotate=False, mesh_type=6, plateau=(0.0, 0.0), centre=None, periodic_object=False):
    """Simple shear with one red cell of radius `radius_cells` cells at the centre (or at `centre`,
    as fractions of the box).  mesh_type 4 with plateau = (width, slope) is the reference's plateau
    mesh (uniform cells in the middle, coarser towards the walls), whose IBM is
    LBFS_IBM_VANDERMONDE4.  periodic_object sets the membrane's periodic flag (its z wrap)."""
    ny = n_cells_y or n
    nz = n_cells_z or n
    dt = 1.0
    visc = (tau - 0.5) / 3.0 * dt
    X, Y, Z = 2.0 * n, 2.0 * ny, 2.0 * nz
    mesh = build_uniform_mesh(X, Y, Z, dt, visc=visc, mesh_type=mesh_type, plateau_width=plateau[0],
                              plateau_slope=plateau[1])
    gamma = u_wall / Y
    bcs = {"left": (2, 2, 1.0, 0.0, 0.0, 0.0), "right": (2, 2, 1.0, 0.0, 0.0, 0.0),
           "bottom": (2, 10, 1.0, gamma, 0.0, 0.0), "top": (2, 10, 1.0, gamma, 0.0, 0.0),
           "back": (2, 2, 1.0, 0.0, 0.0, 0.0), "front": (2, 2, 1.0, 0.0, 0.0, 0.0)}
    mesh.set_boundaries(bcs)
    R = radius_cells * 2.0 * dt
    shear_modulus = visc * gamma * R / capillary
    moduli = dict(volume_modulus=500.0 * shear_modulus, local_area_modulus=10.0 * shear_modulus,
                  global_area_modulus=500.0 * shear_modulus, shear_modulus=shear_modulus,
                  global_bending_modulus=0.05 * shear_modulus * R * R, local_bending_modulus=0.0,
                  viscosity=0.0, wlc_ratio=2.2, curvature_ratio=0.0, volume_ratio=1.0,
                  internal_viscosity_ratio=5.0)
    rng = np.random.default_rng(seed)
    rot = rotation_matrix(rng) if rotate else None
    fx, fy, fz = centre or (0.5, 0.5, 0.5)
    cell = red_cell(level, R, (fx * X, fy * Y, fz * Z), rot, **moduli)
    cell.periodic = periodic_object
    params = StepParams(visc=visc, delta_t=delta_t, channel_diameter=Y, ref_rho=1.0, max_velocity=u_wall, rho0=1.0,
                        visc_factor_initial=1.0, testcase=5, precision=precision, ibm_stencil=ibm_stencil,
                        viscosity_period=10000)
    y = mesh.cell_centroid[: mesh.n_cells, 1]
    rho, u, v, w = _initial_state(mesh.n_cells, seed, u0=gamma * y)
    return Case("shear_rbc", mesh, params, [cell], rho, u, v, w, bcs,
                {"n": (n, ny, nz), "level": level, "radius_cells": radius_cells, "capillary": capillary,
                 "gamma_dot": gamma, "shear_modulus": shear_modulus})


def _rbc_moduli(shear_modulus, R):
    return dict(volume_modulus=500.0 * shear_modulus, local_area_modulus=10.0 * shear_modulus,
                global_area_modulus=500.0 * shear_modulus, shear_modulus=shear_modulus,
                global_bending_modulus=0.05 * shear_modulus * R * R, local_bending_modulus=0.0,
                viscosity=0.0, wlc_ratio=2.2, curvature_ratio=0.0, volume_ratio=1.0,
                internal_viscosity_ratio=5.0)


def shear_channel(n, n_rbc=1, level=2, radius_cells=3.0, shear_modulus=1e-5, capillary=0.1, seed=99, tau=0.8,
                  delta_t=0.5, precision=_abi.LBFS_FP64, ibm_stencil=_abi.LBFS_IBM_PESKIN4):
    """Wall-driven shear in an n^3 channel with up to n_rbc red cells of radius
    `radius_cells`, randomly oriented at distinct points of a lattice of spacing
    2 R + 2 cells, at least R + 3 cells from the walls (fewer cells when fewer
    points fit).  The wall speed follows from the capillary number
    Ca = mu gamma_dot R / G_s with mu = rho nu, rho = 1."""
    dt = 1.0
    visc = (tau - 0.5) / 3.0 * dt
    L = 2.0 * n
    mesh = build_uniform_mesh(L, L, L, dt, visc=visc)
    R = radius_cells * 2.0 * dt
    gamma = capillary * shear_modulus / (visc * R)
    bcs = {"left": (2, 2, 1.0, 0.0, 0.0, 0.0), "right": (2, 2, 1.0, 0.0, 0.0, 0.0),
           "bottom": (2, 10, 1.0, gamma, 0.0, 0.0), "top": (2, 10, 1.0, gamma, 0.0, 0.0),
           "back": (2, 2, 1.0, 0.0, 0.0, 0.0), "front": (2, 2, 1.0, 0.0, 0.0, 0.0)}
    mesh.set_boundaries(bcs)
    rng = np.random.default_rng(seed)
    margin = R + 3 * 2.0 * dt
    axis = np.arange(margin, L - margin + 1e-9, 2 * R + 2 * 2.0 * dt)
    if len(axis) == 0:
        axis = np.array([0.5 * L])
    points = np.array([(x, y, z) for z in axis for y in axis for x in axis])
    chosen = rng.permutation(len(points))[:n_rbc]
    moduli = _rbc_moduli(shear_modulus, R)
    cells = [red_cell(level, R, tuple(points[i]), rotation_matrix(rng), **moduli) for i in sorted(chosen)]
    params = StepParams(visc=visc, delta_t=delta_t, channel_diameter=L, ref_rho=1.0, max_velocity=max(gamma * L, 1e-3),
                        rho0=1.0, visc_factor_initial=1.0, testcase=5, precision=precision, ibm_stencil=ibm_stencil,
                        viscosity_period=10000)
    y = mesh.cell_centroid[: mesh.n_cells, 1]
    rho, u, v, w = _initial_state(mesh.n_cells, seed, amplitude=1e-5, u0=gamma * y)
    return Case("shear_channel", mesh, params, cells, rho, u, v, w, bcs,
                {"n": n, "level": level, "radius_cells": radius_cells, "capillary": capillary,
                 "shear_modulus": shear_modulus, "gamma_dot": gamma, "n_rbc": len(cells)})


def ensemble_specs(n_instances=64, seed=2024, n_range=(16, 48), rbc_range=(1, 8), levels=(2, 3),
                   shear_modulus_range=(2e-6, 2e-5), capillary_range=(0.05, 0.5), radius_cells=None):
    """The seeded draws of the batched workload, one dict per instance (n, n_rbc, level, shear
    modulus, capillary number, radius, seed) and its cost for sharding (cells + red-cell nodes,
    n_rbc taken as drawn)."""
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(n_instances):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        n_rbc = int(rng.integers(rbc_range[0], rbc_range[1] + 1))
        level = int(rng.choice(levels))
        gs = float(np.exp(rng.uniform(np.log(shear_modulus_range[0]), np.log(shear_modulus_range[1]))))
        ca = float(rng.uniform(*capillary_range))
        r = radius_cells if radius_cells is not None else max(1.5, n / 12.0)
        specs.append(dict(n=n, n_rbc=n_rbc, level=level, shear_modulus=gs, capillary=ca, radius_cells=r,
                          seed=seed * 1000 + k, cost=n ** 3 + n_rbc * (10 * 4 ** level + 2)))
    return specs


def ensemble(n_instances=64, seed=2024, n_range=(16, 48), rbc_range=(1, 8), levels=(2, 3),
             shear_modulus_range=(2e-6, 2e-5), capillary_range=(0.05, 0.5), precision=_abi.LBFS_FP32_BULK,
             ibm_stencil=_abi.LBFS_IBM_PESKIN4, tau=0.8, delta_t=0.5, radius_cells=None, subset=None):
    """Batched ensemble of independent shear channels: per instance a cube of n
    cells per axis (n uniform in n_range), 1-8 red cells of a level drawn from
    `levels`, shear modulus log-uniform and capillary number uniform in their
    ranges.  Red-cell radius: n / 12 cells, at least 1.5 (unless given).
    subset: the indices of the instances to build (a rank's shard; every
    instance is the same whatever the subset).  Returns a Case whose mesh is an
    EnsembleMesh and whose info['members'] holds the stand-alone Case of every
    built instance (info['indices'] their instance numbers)."""
    from dataclasses import replace
    from .ensemble import concatenate
    specs = ensemble_specs(n_instances, seed, n_range, rbc_range, levels, shear_modulus_range, capillary_range,
                           radius_cells)
    indices = list(range(n_instances)) if subset is None else sorted(int(k) for k in subset)
    members = []
    for k in indices:
        sp = specs[k]
        members.append(shear_channel(sp["n"], sp["n_rbc"], sp["level"], sp["radius_cells"], sp["shear_modulus"],
                                     sp["capillary"], seed=sp["seed"], tau=tau, delta_t=delta_t,
                                     precision=precision, ibm_stencil=ibm_stencil))
    mesh = concatenate([c.mesh for c in members])
    membranes = [replace(m, instance=k) for k, c in enumerate(members) for m in c.membranes]
    p = members[0].params
    params = replace(p, max_velocity=max(c.params.max_velocity for c in members))
    cat = lambda name: np.ascontiguousarray(np.concatenate([getattr(c, name) for c in members]))
    return Case("ensemble", mesh, params, membranes, cat("rho"), cat("u"), cat("v"), cat("w"), None,
                {"members": members, "indices": indices, "n_instances": n_instances, "cells": int(mesh.n_cells),
                 "membranes": len(membranes), "nodes": int(sum(m.n_nodes for m in membranes))})


def jittered_channel(n=128, n_rbc=16, jitter=0.1, level=3, radius_cells=6.0, capillary=0.1, u_centre=0.01,
                     seed=1313, tau=0.8, delta_t=0.5, precision=_abi.LBFS_FP64, ibm_stencil=_abi.LBFS_IBM_PESKIN4,
                     closed_faces=True):
    """Body-force-driven square duct on a jittered n^3 hex mesh (every interior
    vertex moved by a seeded offset of up to `jitter` x spacing per axis;
    general-normal fluxes) with up to n_rbc red cells of radius `radius_cells`,
    randomly oriented at distinct points of a lattice of spacing 2 R + 2 cells,
    at least R + 3 cells from the walls.  The shear modulus follows from
    Ca = mu gamma R / G_s with gamma = 4 u_centre / (duct width), the wall shear
    rate of the duct."""
    dt = 1.0
    visc = (tau - 0.5) / 3.0 * dt
    L = 2.0 * n
    # closed_faces=False: the geometry the reference's importer forms from this mesh as a polyMesh
    mesh = build_uniform_mesh(L, L, L, dt, visc=visc, jitter=jitter, seed=seed, closed_faces=closed_faces)
    bcs = {"left": (2, 2, 1.0, 0.0, 0.0, 0.0), "right": (2, 2, 1.0, 0.0, 0.0, 0.0),
           "bottom": (2, 1, 1.0, 0.0, 0.0, 0.0), "top": (2, 1, 1.0, 0.0, 0.0, 0.0),
           "back": (2, 1, 1.0, 0.0, 0.0, 0.0), "front": (2, 1, 1.0, 0.0, 0.0, 0.0)}
    mesh.set_boundaries(bcs)
    a = 0.5 * L
    force = u_centre * visc / (0.2947 * a * a)
    R = radius_cells * 2.0 * dt
    gamma = 4.0 * u_centre / L
    shear_modulus = visc * gamma * R / capillary
    rng = np.random.default_rng(seed)
    margin = R + 3 * 2.0 * dt
    axis = np.arange(margin, L - margin + 1e-9, 2 * R + 2 * 2.0 * dt)
    points = np.array([(x, y, z) for z in axis for y in axis for x in axis])
    chosen = rng.permutation(len(points))[:n_rbc]
    moduli = _rbc_moduli(shear_modulus, R)
    cells = [red_cell(level, R, tuple(points[i]), rotation_matrix(rng), **moduli) for i in sorted(chosen)]
    params = StepParams(visc=visc, delta_t=delta_t, channel_diameter=L, body_force=(force, 0.0, 0.0), ref_rho=1.0,
                        max_velocity=u_centre, rho0=1.0, visc_factor_initial=1.0, testcase=5, precision=precision,
                        ibm_stencil=ibm_stencil, viscosity_period=10000)
    rho, u, v, w = _initial_state(mesh.n_cells, seed)
    return Case("jittered_channel", mesh, params, cells, rho, u, v, w, bcs,
                {"n": n, "jitter": jitter, "level": level, "radius_cells": radius_cells, "n_rbc": len(cells),
                 "shear_modulus": shear_modulus, "force": force})


def imported(case, directory, jitter=0.1, seed=5):
    """The case on its box meshed as a jittered hex mesh written as an OpenFOAM polyMesh in
    `directory` and read back through the importer (mesh_type 3: the reference importer's
    geometry, general-normal fluxes on every face)."""
    from dataclasses import replace
    m = case.mesh
    write_openfoam(directory, m.X, m.Y, m.Z, m.dt, m.origin, jitter=jitter, seed=seed)
    mesh = import_openfoam(directory, dt=m.dt, visc=case.params.visc)
    mesh.source = str(directory)
    mesh.set_boundaries(case.bcs)
    return replace(case, mesh=mesh, info=dict(case.info, jitter=jitter, seed=seed, polymesh=str(directory)))
