"""Batched ensembles: many independent cases stepped by one solver handle.

The reference runs one case per process (program::run, program.cpp:113-115).
Here K independent cases (meshes of different sizes, each with its own red
cells, moduli and wall speed) are concatenated into one unstructured mesh with
an instance table, so every phase of the step is ONE launch over all instances
and the whole step is one CUDA graph.  The fluid kernels only follow the
face/cell connectivity, which never links two instances, and the concatenation
keeps each cell's faces in their original relative order, so every instance
evolves bit for bit as it would in a handle of its own.  Each membrane carries
the IBM grid of its instance.

Layout of the concatenated mesh (what lbfs_mesh_desc.instances describes):
  cells   : interior cells of instance 0, 1, ..., then the ghost cells of
            instance 0, 1, ... (ghost b of the whole mesh belongs to face ni + b)
  faces   : x-normal interior faces of every instance, then y-normal, then
            z-normal, then the boundary faces, each block instance by instance.
The residual norms of an ensemble handle are taken over all instances; the
per-instance norms follow from the residual field (LBFS_FIELD_RESIDUAL).
"""
import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _abi


@dataclass
class EnsembleMesh:
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
    bc_rho_type: np.ndarray
    bc_vel_type: np.ndarray
    bc_values: np.ndarray
    cell0: np.ndarray            # first interior cell of each instance
    cells: np.ndarray            # interior cells of each instance
    members: list = field(default_factory=list, repr=False)
    _grids: object = field(default=None, repr=False)
    periodic_node: np.ndarray = field(default=None)  # partner cells of type-3 ghosts (whole-mesh indices)

    @property
    def n_instances(self):
        return len(self.cells)

    def split(self, values):
        """Per-instance views of a per-interior-cell array (first axis = cell)."""
        return [values[c0:c0 + n] for c0, n in zip(self.cell0, self.cells)]

    def desc(self):
        d = _abi.MeshDesc()
        d.n_cells, d.n_faces, d.n_interior, d.n_bc = self.n_cells, self.n_faces, self.n_interior, self.n_bc
        d.n_face_x, d.n_face_y, d.n_face_z = self.n_face_x, self.n_face_y, self.n_face_z
        d.axis_aligned = 1
        d.owner, d.neighbour = _abi.iptr(self.owner), _abi.iptr(self.neighbour)
        d.face_area, d.face_normal = _abi.ptr(self.face_area), _abi.ptr(self.face_normal)
        d.face_centroid, d.streaming_dt = _abi.ptr(self.face_centroid), _abi.ptr(self.streaming_dt)
        d.cell_volume, d.cell_centroid = _abi.ptr(self.cell_volume), _abi.ptr(self.cell_centroid)
        d.gradient_stencil = _abi.iptr(self.gradient_stencil)
        d.lhs_inverse, d.rhs = _abi.ptr(self.lhs_inverse), _abi.ptr(self.rhs)
        d.bc_rho_type, d.bc_vel_type = _abi.iptr(self.bc_rho_type), _abi.iptr(self.bc_vel_type)
        d.bc_values = _abi.ptr(self.bc_values)
        if self.periodic_node is not None:
            d.periodic_node = _abi.iptr(self.periodic_node)
        grids = (_abi.GridDesc * self.n_instances)()
        for k, m in enumerate(self.members):
            g = grids[k]
            g.cell0, g.n_cells = int(self.cell0[k]), int(self.cells[k])
            g.origin[:] = m.origin
            g.length[:] = (m.X, m.Y, m.Z)
            g.delta_x, g.delta_h = m.delta_x, m.delta_h
        self._grids = grids  # the descriptor points into it
        d.n_instances = self.n_instances
        d.instances = ctypes.cast(grids, ctypes.POINTER(_abi.GridDesc))
        # the single-grid fields describe instance 0 (used by no kernel of an ensemble)
        m0 = self.members[0]
        d.origin[:] = m0.origin
        d.length[:] = (m0.X, m0.Y, m0.Z)
        d.delta_x, d.delta_h = m0.delta_x, m0.delta_h
        return d


def concatenate(meshes):
    """One EnsembleMesh holding the axis-aligned meshes `meshes` (boundaries set)."""
    meshes = list(meshes)
    if not meshes:
        raise ValueError("an ensemble needs at least one instance")
    for m in meshes:
        if m.bc_rho_type is None:
            raise ValueError("set_boundaries() on every instance first")
    nc = np.array([m.n_cells for m in meshes])
    nb = np.array([m.n_bc for m in meshes])
    C = np.concatenate([[0], np.cumsum(nc)[:-1]])
    G = np.concatenate([[0], np.cumsum(nb)[:-1]])
    NC, NB = int(nc.sum()), int(nb.sum())

    def remap(k, idx):
        m = meshes[k]
        idx = np.asarray(idx, np.int64)
        return np.where(idx < m.n_cells, C[k] + idx, NC + G[k] + (idx - m.n_cells)).astype(np.int32)

    # face permutation: (instance, local face) per category
    cats = []
    for lo_hi in (lambda m: (0, m.n_face_x), lambda m: (m.n_face_x, m.n_face_x + m.n_face_y),
                  lambda m: (m.n_face_x + m.n_face_y, m.n_interior), lambda m: (m.n_interior, m.n_faces)):
        cats.append([(k, *lo_hi(m)) for k, m in enumerate(meshes)])
    owner, neigh, area, normal, fcen, sdt = [], [], [], [], [], []
    for cat in cats:
        for k, lo, hi in cat:
            m = meshes[k]
            owner.append(remap(k, m.owner[lo:hi]))
            neigh.append(remap(k, m.neighbour[lo:hi]))
            area.append(m.face_area[lo:hi])
            normal.append(m.face_normal[lo:hi])
            fcen.append(m.face_centroid[lo:hi])
            sdt.append(m.streaming_dt[lo:hi])
    vol = [m.cell_volume[:m.n_cells] for m in meshes] + [m.cell_volume[m.n_cells:] for m in meshes]
    cen = [m.cell_centroid[:m.n_cells] for m in meshes] + [m.cell_centroid[m.n_cells:] for m in meshes]
    cat = lambda xs, dt=None: np.ascontiguousarray(np.concatenate(xs), dt)
    return EnsembleMesh(
        n_cells=NC, n_faces=sum(m.n_faces for m in meshes), n_interior=sum(m.n_interior for m in meshes), n_bc=NB,
        n_face_x=sum(m.n_face_x for m in meshes), n_face_y=sum(m.n_face_y for m in meshes),
        n_face_z=sum(m.n_face_z for m in meshes),
        owner=cat(owner, np.int32), neighbour=cat(neigh, np.int32), face_area=cat(area, np.float64),
        face_normal=cat(normal, np.float64), face_centroid=cat(fcen, np.float64), streaming_dt=cat(sdt, np.float64),
        cell_volume=cat(vol, np.float64), cell_centroid=cat(cen, np.float64),
        gradient_stencil=cat([remap(k, m.gradient_stencil) for k, m in enumerate(meshes)], np.int32),
        lhs_inverse=cat([m.lhs_inverse for m in meshes], np.float64),
        rhs=cat([m.rhs for m in meshes], np.float64),
        bc_rho_type=cat([m.bc_rho_type for m in meshes], np.int32),
        bc_vel_type=cat([m.bc_vel_type for m in meshes], np.int32),
        bc_values=cat([m.bc_values for m in meshes], np.float64),
        cell0=C.astype(np.int64), cells=nc.astype(np.int64), members=meshes,
        periodic_node=(cat([C[k] + (m.periodic_node if m.periodic_node is not None else np.zeros(m.n_bc, np.int64))
                            for k, m in enumerate(meshes)], np.int32)
                       if any(m.periodic_node is not None for m in meshes) else None))
