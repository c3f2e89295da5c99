"""ctypes front end of oracle/_ref/libref_lbfs.so: the reference's own sources
compiled for the host (oracle/build_ref.sh) and driven by oracle/ref_driver.cpp.

Test infrastructure only: tests/golden/make_golden.py uses it to write the
golden fixtures, and bench.py's reference arm times it.  The product never
imports it.
"""
import ctypes
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libref_lbfs.so")

REF_RHO, REF_U, REF_V, REF_W = 0, 1, 2, 3
REF_T1, REF_GRAD, REF_RES_FACE, REF_RES, REF_FORCE = 4, 5, 6, 7, 8
REF_NODE_X, REF_NODE_V, REF_NODE_F, REF_TOTALS, REF_VISC, REF_SPRING, REF_RESID, REF_GHOST = range(9, 17)
REF_DT_LOCAL, REF_DELTA_T, REF_ENERGY = 17, 18, 19


class RefParams(ctypes.Structure):
    _fields_ = [
        ("visc", ctypes.c_double), ("delta_t", ctypes.c_double), ("gamma_inv", ctypes.c_double),
        ("channel_diameter", ctypes.c_double), ("force", ctypes.c_double * 3), ("ref_rho", ctypes.c_double),
        ("max_velocity", ctypes.c_double), ("testcase", ctypes.c_int), ("visc_factor_initial", ctypes.c_double),
        ("has_rbc", ctypes.c_int),
        ("volume_modulus", ctypes.c_double), ("local_area_modulus", ctypes.c_double),
        ("global_area_modulus", ctypes.c_double), ("shear_modulus", ctypes.c_double),
        ("global_bending_modulus", ctypes.c_double), ("local_bending_modulus", ctypes.c_double),
        ("membrane_thickness", ctypes.c_double), ("viscosity", ctypes.c_double), ("wlc_ratio", ctypes.c_double),
        ("curvature_ratio", ctypes.c_double), ("volume_ratio", ctypes.c_double),
        ("internal_viscosity_ratio", ctypes.c_double), ("reference_length", ctypes.c_double),
        ("pivkin_length", ctypes.c_int), ("sphere_reference", ctypes.c_int), ("viscosity_period", ctypes.c_int),
        ("time_stepping", ctypes.c_int), ("pre_conditioned_gamma", ctypes.c_double),
        ("preconditioning", ctypes.c_int), ("object_periodic", ctypes.c_int),
    ]


_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.ref_mesh_create.restype = vp
        L.ref_mesh_create.argtypes = [ctypes.c_double] * 8 + [ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                                               ctypes.c_double, ctypes.c_double, ctypes.c_char_p]
        L.ref_mesh_plateau.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        L.ref_mesh_counts.argtypes = [vp, ctypes.c_void_p]
        L.ref_mesh_dump.argtypes = [vp] + [ctypes.c_void_p] * 12
        L.ref_mesh_free.argtypes = [vp]
        L.ref_rbc_create.restype = vp
        L.ref_rbc_create.argtypes = [ctypes.c_char_p] + [ctypes.c_double] * 3
        L.ref_rbc_counts.argtypes = [vp, ctypes.c_void_p]
        L.ref_rbc_dump.argtypes = [vp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.ref_rbc_free.argtypes = [vp]
        L.ref_case_create.restype = vp
        L.ref_case_create.argtypes = [vp, ctypes.POINTER(RefParams), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.ref_case_set_state.argtypes = [vp] + [ctypes.c_void_p] * 4
        L.ref_case_set_rbc.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 4
        L.ref_case_step.argtypes = [vp, ctypes.c_int]
        L.ref_case_get.argtypes = [vp, ctypes.c_int, ctypes.c_void_p]
        L.ref_case_free.argtypes = [vp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class RefMesh:
    """unstructured_mesh (generated: mesh_type 6, 7, 5 or 4) + gradients built by the reference code."""

    def __init__(self, X, Y, Z, dt=1.0, origin=(0.0, 0.0, 0.0), visc=0.1, hybrid=False, mesh_type=6,
                 plateau_width=0.0, plateau_slope=0.0, import_dir=None):
        self._dir = tempfile.mkdtemp(prefix="refmesh")
        self.dims = tuple(int(np.ceil(L / dt * 0.5)) for L in (X, Y, Z))
        self.mesh_type = mesh_type
        self.h = lib().ref_mesh_create(X, Y, Z, dt, origin[0], origin[1], origin[2], visc, int(hybrid),
                                       self._dir.encode(), int(mesh_type), float(plateau_width),
                                       float(plateau_slope), None if import_dir is None else str(import_dir).encode())
        c = (ctypes.c_int * 8)()
        lib().ref_mesh_counts(self.h, c)
        (self.n_cells, self.n_faces, self.n_interior, self.n_bc, self.n_face_x, self.n_face_y, self.n_face_z,
         self.total_cells) = list(c)

    def arrays(self):
        nc, nf, nt = self.n_cells, self.n_faces, self.total_cells
        A = dict(owner=np.zeros(nf, np.int32), neighbour=np.zeros(nf, np.int32), face_area=np.zeros(nf),
                 face_normal=np.zeros((nf, 3)), face_centroid=np.zeros((nf, 3)), streaming_dt=np.zeros(nf),
                 cell_volume=np.zeros(nt), cell_centroid=np.zeros((nt, 3)),
                 gradient_stencil=np.zeros((nc, 6), np.int32), lhs_inverse=np.zeros((nc, 9)),
                 rhs=np.zeros((nc, 6, 3)))
        dh = ctypes.c_double()
        lib().ref_mesh_dump(self.h, *[_p(a) for a in A.values()], ctypes.byref(dh))
        A["delta_h"] = dh.value
        if self.mesh_type != 3:  # the importer allocates no plateau arrays
            nx, ny, nz = self.dims
            g = np.zeros(nx + ny + nz + 3)
            lib().ref_mesh_plateau(self.h, nx, ny, nz, _p(g))
            A["plateau"] = g
        return A


def ref_springs(nodes, tris, centre=(0.0, 0.0, 0.0)):
    """sprIdx / sorted_triIdx / coordinates from lagrangian_object::initialise on an Osay file."""
    d = tempfile.mkdtemp(prefix="refrbc")
    path = os.path.join(d, "stress_free.dat")
    with open(path, "w") as f:
        f.write(f"{len(nodes)} {len(tris)}\n")
        for p in nodes:
            f.write(f"{p[0]:.17g} {p[1]:.17g} {p[2]:.17g}\n")
        for t in tris:
            f.write(f"{t[0] + 1} {t[1] + 1} {t[2] + 1}\n")
    h = lib().ref_rbc_create(path.encode(), *centre)
    c = (ctypes.c_int * 4)()
    lib().ref_rbc_counts(h, c)
    nn, nt, ns, _ = list(c)
    spr = np.zeros((ns, 4), np.int32)
    tri = np.zeros((nt, 3), np.int32)
    xyz = np.zeros((nn, 3))
    lib().ref_rbc_dump(h, _p(spr), _p(tri), _p(xyz))
    lib().ref_rbc_free(h)
    return spr, tri, xyz


class RefCase:
    """The reference GPU time loop (kernel bodies run serially on the host)."""

    def __init__(self, mesh: RefMesh, params: RefParams, rho_type, vel_type, bc_values):
        self.mesh = mesh
        self._keep = [np.ascontiguousarray(rho_type, np.int32), np.ascontiguousarray(vel_type, np.int32),
                      np.ascontiguousarray(bc_values, np.float64)]
        self.params = params
        self.h = lib().ref_case_create(mesh.h, ctypes.byref(params), *[_p(a) for a in self._keep])
        self.n_nodes = 0
        self.n_springs = 0

    def set_state(self, rho, u, v, w):
        arrs = [np.ascontiguousarray(a, np.float64) for a in (rho, u, v, w)]
        lib().ref_case_set_state(self.h, *[_p(a) for a in arrs])

    def set_rbc(self, tris, springs, xyz_stress_free, xyz_initial):
        keep = [np.ascontiguousarray(tris, np.int32), np.ascontiguousarray(springs, np.int32),
                np.ascontiguousarray(xyz_stress_free, np.float64), np.ascontiguousarray(xyz_initial, np.float64)]
        self.n_nodes, self.n_springs = len(keep[2]), len(keep[1])
        lib().ref_case_set_rbc(self.h, len(keep[2]), len(keep[0]), len(keep[1]), *[_p(a) for a in keep])

    def step(self, n=1):
        lib().ref_case_step(self.h, int(n))

    def get(self, which):
        m = self.mesh
        size = {REF_RHO: m.n_cells, REF_U: m.n_cells, REF_V: m.n_cells, REF_W: m.n_cells, REF_T1: 4 * m.n_cells,
                REF_GRAD: 12 * m.total_cells, REF_RES_FACE: 4 * m.n_faces, REF_RES: 4 * m.n_cells,
                REF_FORCE: 3 * m.n_cells, REF_NODE_X: 3 * self.n_nodes, REF_NODE_V: 3 * self.n_nodes,
                REF_NODE_F: 3 * self.n_nodes, REF_TOTALS: 6, REF_VISC: m.n_cells, REF_SPRING: 9 * self.n_springs,
                REF_RESID: 4, REF_GHOST: 4 * m.n_bc, REF_DT_LOCAL: m.n_cells, REF_DELTA_T: 1, REF_ENERGY: 7}[which]
        out = np.zeros(max(size, 1))
        lib().ref_case_get(self.h, which, _p(out))
        return out[:size]

    def state(self):
        return tuple(self.get(k) for k in (REF_RHO, REF_U, REF_V, REF_W))

    def close(self):
        if self.h:
            lib().ref_case_free(self.h)
            self.h = None
