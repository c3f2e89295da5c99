"""Uniform OpenFOAM-layout hex meshes and boundary tables.

The mesh arrays come from lbfs_mesh_build_uniform, which reproduces
unstructured_mesh::create_uniform_openfoam_mesh + generate_internal_mesh and
gradients::pre_fill_LHS_and_RHS_matrix (unstructured_mesh.cpp:239-666,
1592-1692; gradients.cpp:214-315): same face order (interior x, y, z faces,
then the boundary patches left, right, bottom, top, back, front), same ghost
numbering, same gradient stencil order.
"""
import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _abi

PATCHES = ("left", "right", "bottom", "top", "back", "front")


@dataclass
class UniformMesh:
    X: float
    Y: float
    Z: float
    dt: float
    origin: tuple
    n_cells: int
    n_faces: int
    n_interior: int
    n_bc: int
    n_face_x: int
    n_face_y: int
    n_face_z: int
    owner: np.ndarray
    neighbour: np.ndarray
    face_area: np.ndarray
    face_normal: np.ndarray
    face_centroid: np.ndarray
    streaming_dt: np.ndarray
    cell_volume: np.ndarray
    cell_centroid: np.ndarray
    gradient_stencil: np.ndarray
    lhs_inverse: np.ndarray
    rhs: np.ndarray
    bc_patch: np.ndarray
    delta_h: float
    bc_rho_type: np.ndarray = field(default=None)
    bc_vel_type: np.ndarray = field(default=None)
    bc_values: np.ndarray = field(default=None)
    axis_aligned: bool = True  # False for jittered meshes: every face takes the general-normal flux
    mesh_type: int = 6         # 6 uniform, 7 / 5 cosine-clustered, 4 plateau (rectilinear), 3 jittered
    grid: tuple = None         # vertex coordinates per axis (rectilinear meshes)
    plateau: tuple = (0.0, 0.0)  # plateau width and slope (mesh_type 4)
    patch_names: tuple = PATCHES  # boundary patches in bc_patch order
    source: str = None            # polyMesh directory of an imported mesh
    periodic_node: np.ndarray = field(default=None)  # partner cell of each type-3 ghost

    @property
    def shape(self):
        """Cells per axis (nx, ny, nz); cell index = i + nx (j + ny k)."""
        d = 2 * self.dt
        return int(round(self.X / d)), int(round(self.Y / d)), int(round(self.Z / d))

    @property
    def delta_x(self):
        return 2 * self.dt

    def set_boundaries(self, spec, periodic_translation=None):
        """spec: {patch: (rho_type, vel_type, rho, u, v, w)} for the six patches,
        values already scaled as after preprocessor::mach_number_factor
        (Boundary_Conditions::assign_boundary_conditions, Boundary_Conditions.cpp:377-441).
        Type 3 is periodic: each such ghost takes the state and gradients of the interior
        cell nearest to its centroid moved by +-periodic_translation (the XML's
        periodic_translation, one vector for every periodic patch)."""
        rt = np.zeros(self.n_bc, np.int32)
        vt = np.zeros(self.n_bc, np.int32)
        vals = np.zeros((self.n_bc, 4), np.float64)
        for p, name in enumerate(self.patch_names):
            rho_type, vel_type, rho, u, v, w = spec[name]
            sel = self.bc_patch == p
            rt[sel] = rho_type
            vt[sel] = vel_type
            vals[sel] = (u, v, w, rho)
        self.bc_rho_type, self.bc_vel_type, self.bc_values = rt, vt, np.ascontiguousarray(vals)
        self.periodic_node = None
        if np.any(rt == 3) or np.any(vt == 3):
            if periodic_translation is None:
                raise ValueError("periodic boundaries (type 3) need periodic_translation")
            self.periodic_node = find_periodic_nodes(self, periodic_translation)
        return self

    def desc(self):
        """MeshDesc pointing into this object's arrays (keep the mesh alive while it is used)."""
        if self.bc_rho_type is None:
            raise ValueError("set_boundaries() first")
        d = _abi.MeshDesc()
        d.n_cells, d.n_faces, d.n_interior, d.n_bc = self.n_cells, self.n_faces, self.n_interior, self.n_bc
        d.n_face_x, d.n_face_y, d.n_face_z = self.n_face_x, self.n_face_y, self.n_face_z
        d.axis_aligned = 1 if self.axis_aligned else 0
        d.owner, d.neighbour = _abi.iptr(self.owner), _abi.iptr(self.neighbour)
        d.face_area, d.face_normal = _abi.ptr(self.face_area), _abi.ptr(self.face_normal)
        d.face_centroid, d.streaming_dt = _abi.ptr(self.face_centroid), _abi.ptr(self.streaming_dt)
        d.cell_volume, d.cell_centroid = _abi.ptr(self.cell_volume), _abi.ptr(self.cell_centroid)
        d.gradient_stencil = _abi.iptr(self.gradient_stencil)
        d.lhs_inverse, d.rhs = _abi.ptr(self.lhs_inverse), _abi.ptr(self.rhs)
        d.bc_rho_type, d.bc_vel_type = _abi.iptr(self.bc_rho_type), _abi.iptr(self.bc_vel_type)
        d.bc_values = _abi.ptr(self.bc_values)
        d.origin[:] = self.origin
        d.length[:] = (self.X, self.Y, self.Z)
        d.delta_x = self.delta_x
        d.delta_h = self.delta_h
        if self.grid is not None:
            d.grid_x, d.grid_y, d.grid_z = (_abi.ptr(g) for g in self.grid)
        if self.periodic_node is not None:
            d.periodic_node = _abi.iptr(self.periodic_node)
        return d


def find_periodic_nodes(mesh, translation):
    """Partner cell of every type-3 ghost: the interior cell nearest to the ghost's centroid
    moved by +translation or -translation (lbfs_mesh_find_periodic_nodes); 0 elsewhere."""
    out = np.zeros(mesh.n_bc, np.int32)
    keep = mesh.periodic_node
    mesh.periodic_node = None  # the search reads sizes, centroids and types only
    try:
        d = mesh.desc()
    finally:
        mesh.periodic_node = keep
    t = np.ascontiguousarray(translation, dtype=np.float64)
    _abi.check(_abi.lib().lbfs_mesh_find_periodic_nodes(ctypes.byref(d), _abi.ptr(t), _abi.iptr(out)))
    return out


def uniform_counts(X, Y, Z, dt):
    out = (ctypes.c_int32 * 8)()
    _abi.check(_abi.lib().lbfs_mesh_uniform_counts(X, Y, Z, dt, out))
    return list(out)


def build_uniform_mesh(X, Y, Z, dt=1.0, origin=(0.0, 0.0, 0.0), visc=0.1, fneq_min=0.0, gradient="LS", jitter=0.0,
                       seed=0, mesh_type=6, plateau_width=0.0, plateau_slope=0.0, closed_faces=True, device=None):
    """Mesh of ceil(X/(2 dt)) x ceil(Y/(2 dt)) x ceil(Z/(2 dt)) cells.  mesh_type 6 (uniform),
    7 / 5 (cosine-clustered in x, y / in x, y, z) and 4 (the plateau mesh of plateau_width,
    plateau_slope) are the reference generator's rectilinear meshes; with jitter > 0 every
    interior vertex of the uniform mesh moves by a seeded uniform offset of up to jitter x spacing
    per axis and the mesh is stepped through the general-normal flux (mesh_type 3); closed_faces=False
    gives the reference importer's geometry of that mesh (lbfs_mesh_build_jittered).  device = a
    CUDA device index builds the same arrays on that GPU (lbfs_mesh_build_gpu)."""
    nc, nf, ni, nb, nfx, nfy, nfz, nt = uniform_counts(X, Y, Z, dt)
    owner = np.zeros(nf, np.int32)
    neighbour = np.zeros(nf, np.int32)
    area = np.zeros(nf)
    normal = np.zeros((nf, 3))
    fcen = np.zeros((nf, 3))
    sdt = np.zeros(nf)
    vol = np.zeros(nt)
    ccen = np.zeros((nt, 3))
    stencil = np.zeros((nc, 6), np.int32)
    lhs = np.zeros((nc, 9))
    rhs = np.zeros((nc, 6, 3))
    patch = np.zeros(nb, np.int32)
    dh = ctypes.c_double()
    org = np.asarray(origin, np.float64)
    outs = (_abi.iptr(owner), _abi.iptr(neighbour), _abi.ptr(area), _abi.ptr(normal), _abi.ptr(fcen), _abi.ptr(sdt),
            _abi.ptr(vol), _abi.ptr(ccen), _abi.iptr(stencil), _abi.ptr(lhs), _abi.ptr(rhs), _abi.iptr(patch),
            ctypes.byref(dh))
    hybrid = 1 if gradient == "hybrid" else 0
    grid = None
    if mesh_type != 6 and jitter > 0:
        raise ValueError("jitter applies to the uniform mesh only")
    if device is not None:
        nx, ny, nz = (int(np.ceil(L / dt * 0.5)) for L in (X, Y, Z))
        g = np.zeros(nx + ny + nz + 3)
        _abi.check(_abi.lib().lbfs_mesh_build_gpu(X, Y, Z, dt, _abi.ptr(org), visc, fneq_min, hybrid, int(mesh_type),
                                                  float(plateau_width), float(plateau_slope), float(jitter), int(seed),
                                                  1 if closed_faces else 0, int(device), *outs, _abi.ptr(g)))
        if mesh_type != 6:
            grid = (g[:nx + 1].copy(), g[nx + 1:nx + ny + 2].copy(), g[nx + ny + 2:].copy())
    elif mesh_type != 6:
        nx, ny, nz = (int(np.ceil(L / dt * 0.5)) for L in (X, Y, Z))
        g = np.zeros(nx + ny + nz + 3)
        _abi.check(_abi.lib().lbfs_mesh_build_rectilinear(X, Y, Z, dt, _abi.ptr(org), visc, fneq_min, hybrid,
                                                          int(mesh_type), float(plateau_width),
                                                          float(plateau_slope), *outs, _abi.ptr(g)))
        grid = (g[:nx + 1].copy(), g[nx + 1:nx + ny + 2].copy(), g[nx + ny + 2:].copy())
    elif jitter > 0:
        _abi.check(_abi.lib().lbfs_mesh_build_jittered(X, Y, Z, dt, _abi.ptr(org), visc, fneq_min, hybrid,
                                                       float(jitter), int(seed), 1 if closed_faces else 0, *outs))
    else:
        _abi.check(_abi.lib().lbfs_mesh_build_uniform(X, Y, Z, dt, _abi.ptr(org), visc, fneq_min, hybrid, *outs))
    return UniformMesh(X, Y, Z, dt, tuple(origin), nc, nf, ni, nb, nfx, nfy, nfz, owner, neighbour, area, normal,
                       fcen, sdt, vol, ccen, stencil, lhs, rhs, patch, dh.value, axis_aligned=not jitter > 0,
                       mesh_type=3 if jitter > 0 else int(mesh_type), grid=grid,
                       plateau=(float(plateau_width), float(plateau_slope)))


def write_openfoam(directory, X, Y, Z, dt=1.0, origin=(0.0, 0.0, 0.0), mesh_type=6, plateau_width=0.0,
                   plateau_slope=0.0, jitter=0.0, seed=0):
    """Write the generator's mesh as an ASCII OpenFOAM polyMesh in `directory` (points, faces,
    owner, neighbour, boundary; patches left, right, bottom, top, back, front)."""
    org = np.asarray(origin, np.float64)
    _abi.check(_abi.lib().lbfs_mesh_write_openfoam(str(directory).encode(), X, Y, Z, dt, _abi.ptr(org),
                                                   int(mesh_type), float(plateau_width), float(plateau_slope),
                                                   float(jitter), int(seed)))


def import_openfoam(directory, dt=1.0, visc=0.1, fneq_min=0.0, gradient="LS", closed_faces=False, delta_h=None,
                    device=None):
    """Read an OpenFOAM polyMesh of hexahedra as the reference's importer does (mesh_type 3: every face
    takes the general-normal flux).  The IBM grid is the mesh's bounding box with cells of 2 dt
    (cell order must be lexicographic for the IBM, as in the reference); delta_h defaults to
    min(0.1, dt).  device = a CUDA device index forms the geometry and least-squares arrays on that
    GPU (lbfs_mesh_import_openfoam_gpu; the same arrays bit for bit)."""
    d = str(directory).encode()
    c = (ctypes.c_int32 * 6)()
    _abi.check(_abi.lib().lbfs_mesh_openfoam_counts(d, c))
    n_points, nc, nf, ni, nb, n_patches = list(c)
    nt = nc + nb
    owner = np.zeros(nf, np.int32)
    neighbour = np.zeros(nf, np.int32)
    area = np.zeros(nf)
    normal = np.zeros((nf, 3))
    fcen = np.zeros((nf, 3))
    sdt = np.zeros(nf)
    vol = np.zeros(nt)
    ccen = np.zeros((nt, 3))
    stencil = np.zeros((nc, 6), np.int32)
    lhs = np.zeros((nc, 9))
    rhs = np.zeros((nc, 6, 3))
    patch = np.zeros(nb, np.int32)
    names = ctypes.create_string_buffer(64 * (n_patches + 1) + 64)
    head = (d, visc, fneq_min, 1 if gradient == "hybrid" else 0, 1 if closed_faces else 0)
    outs = (_abi.iptr(owner), _abi.iptr(neighbour), _abi.ptr(area), _abi.ptr(normal), _abi.ptr(fcen), _abi.ptr(sdt),
            _abi.ptr(vol), _abi.ptr(ccen), _abi.iptr(stencil), _abi.ptr(lhs), _abi.ptr(rhs), _abi.iptr(patch), names,
            len(names))
    if device is None:
        _abi.check(_abi.lib().lbfs_mesh_import_openfoam(*head, *outs))
    else:
        _abi.check(_abi.lib().lbfs_mesh_import_openfoam_gpu(*head, int(device), *outs))
    patch_names = tuple(names.value.decode().split())
    # bounding box of the boundary face centroids: the box the IBM grid covers
    bf = fcen[ni:]
    lo, hi = bf.min(axis=0), bf.max(axis=0)
    m = UniformMesh(float(hi[0] - lo[0]), float(hi[1] - lo[1]), float(hi[2] - lo[2]), dt, tuple(lo), nc, nf, ni, nb,
                    0, 0, 0, owner, neighbour, area, normal, fcen, sdt, vol, ccen, stencil, lhs, rhs, patch,
                    float(min(0.1, dt)) if delta_h is None else float(delta_h), axis_aligned=False, mesh_type=3)
    m.patch_names = patch_names
    return m
