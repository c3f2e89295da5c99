"""Spring-network membranes: synthetic meshes and the descriptor of the C ABI.

Synthetic inputs (the reference ships no membrane meshes): a subdivided
icosahedron (level L has 10 * 4**L + 2 nodes) as the stress-free sphere, and
the Evans-Fung biconcave shape obtained by mapping the same nodes.  Files use
the reference's Osay mesh format (lagrangian_object::osay_mesh_read,
lagrangian_object.cpp:238-297: "n_nodes n_tris", node coordinates relative to
the centre, 1-based triangle indices).
"""
import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _abi

# Evans & Fung (1972) biconcave profile coefficients.
EVANS_FUNG = (0.2072, 2.0026, -1.1228)


def icosphere(level, radius=1.0):
    """Nodes (N, 3) and outward-oriented triangles (T, 3) of a subdivided icosahedron."""
    t = (1.0 + 5 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    nodes = np.array(verts) * radius
    tris = np.array(faces, np.int32)
    # orient every triangle outward
    for k, (a, b, c) in enumerate(tris):
        n = np.cross(nodes[b] - nodes[a], nodes[c] - nodes[a])
        if np.dot(n, nodes[a] + nodes[b] + nodes[c]) < 0:
            tris[k] = (a, c, b)
    return np.ascontiguousarray(nodes), np.ascontiguousarray(tris)


def biconcave(unit_nodes, radius):
    """Map unit-sphere nodes to the Evans-Fung biconcave disc of the given radius (axis z)."""
    c0, c1, c2 = EVANS_FUNG
    x, y, z = unit_nodes[:, 0], unit_nodes[:, 1], unit_nodes[:, 2]
    r2 = np.clip(x * x + y * y, 0.0, 1.0)
    zz = np.sign(z) * 0.5 * radius * np.sqrt(1.0 - r2) * (c0 + c1 * r2 + c2 * r2 * r2)
    return np.ascontiguousarray(np.stack([radius * x, radius * y, zz], axis=1))


def rotation_matrix(rng):
    """Uniform random rotation (QR of a Gaussian matrix with sign fix)."""
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q @ np.diag(np.sign(np.diag(r)))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def write_osay(path, nodes, tris):
    with open(path, "w") as f:
        f.write(f"{len(nodes)} {len(tris)}\n")
        for p in nodes:
            f.write(f"{p[0]:.17g} {p[1]:.17g} {p[2]:.17g}\n")
        for t in tris:
            f.write(f"{t[0] + 1} {t[1] + 1} {t[2] + 1}\n")


def build_springs(n_nodes, tris):
    """sprIdx quadruples (a, b, c, d) in the reference's order (lbfs_rbc_build_springs)."""
    tris = np.ascontiguousarray(tris, np.int32)
    cap = 3 * len(tris)
    out = np.zeros((cap, 4), np.int32)
    n = ctypes.c_int32()
    _abi.check(_abi.lib().lbfs_rbc_build_springs(n_nodes, len(tris), _abi.iptr(tris), cap, _abi.iptr(out),
                                                 ctypes.byref(n)))
    return np.ascontiguousarray(out[: n.value])


@dataclass
class Membrane:
    """One lagrangian_object of type 2 (spring network)."""
    tris: np.ndarray
    springs: np.ndarray
    xyz_stress_free: np.ndarray
    xyz_initial: np.ndarray
    volume_modulus: float = 0.0
    local_area_modulus: float = 0.0
    global_area_modulus: float = 0.0
    shear_modulus: float = 0.0
    global_bending_modulus: float = 0.0
    local_bending_modulus: float = 0.0
    membrane_thickness: float = 1.0
    viscosity: float = 0.0
    wlc_ratio: float = 2.2
    curvature_ratio: float = 0.0
    volume_ratio: float = 1.0
    internal_viscosity_ratio: float = 5.0
    reference_length: float = 0.0
    pivkin_length: bool = False
    sphere_reference: bool = True
    instance: int = 0  # ensemble instance the membrane lives in
    periodic: int = 0  # lagrangian_object::periodic, the z wrap every 5000 steps: 0, LBFS_WRAP_OWN or LBFS_WRAP_ALL
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n_nodes(self):
        return len(self.xyz_initial)

    def desc(self):
        d = _abi.RbcDesc()
        self._keep = [np.ascontiguousarray(self.tris, np.int32), np.ascontiguousarray(self.springs, np.int32),
                      np.ascontiguousarray(self.xyz_stress_free, np.float64),
                      np.ascontiguousarray(self.xyz_initial, np.float64)]
        tri, spr, sf, ini = self._keep
        d.n_nodes, d.n_tris, d.n_springs = len(ini), len(tri), len(spr)
        d.tri, d.spring, d.xyz_stress_free, d.xyz_initial = _abi.iptr(tri), _abi.iptr(spr), _abi.ptr(sf), _abi.ptr(ini)
        for name in ("volume_modulus", "local_area_modulus", "global_area_modulus", "shear_modulus",
                     "global_bending_modulus", "local_bending_modulus", "membrane_thickness", "viscosity",
                     "wlc_ratio", "curvature_ratio", "volume_ratio", "internal_viscosity_ratio", "reference_length"):
            setattr(d, name, float(getattr(self, name)))
        d.pivkin_length = int(bool(self.pivkin_length))
        d.sphere_reference = int(bool(self.sphere_reference))
        d.instance = int(self.instance)
        d.periodic = int(self.periodic)
        return d


def red_cell(level, radius, centre, rotation=None, **moduli):
    """A red cell: icosphere of `radius` (stress free) and its biconcave map
    (initial shape), optionally rotated, centred at `centre`."""
    unit, tris = icosphere(level, 1.0)
    sphere = unit * radius
    disc = biconcave(unit, radius)
    if rotation is not None:
        sphere = sphere @ rotation.T
        disc = disc @ rotation.T
    c = np.asarray(centre, np.float64)
    springs = build_springs(len(unit), tris)
    return Membrane(tris=tris, springs=springs, xyz_stress_free=np.ascontiguousarray(sphere + c),
                    xyz_initial=np.ascontiguousarray(disc + c), **moduli)
