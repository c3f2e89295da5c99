"""ctypes binding of include/lbfs_b200.h (the library's C ABI).

The structures mirror the header field for field.  The library is the in-tree
build lbfs_b200/_lib/liblbfs_b200.so; importing this module does not need a
GPU, but every solver entry point fails with LBFS_ERR_CUDA when no CUDA device
is present -- there is no CPU path.
"""
import ctypes
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "liblbfs_b200.so")

LBFS_OK = 0
LBFS_ERR_ARG = 1
LBFS_ERR_CUDA = 2
LBFS_ERR_NOMEM = 3
LBFS_ERR_STATE = 4
LBFS_ERR_UNSUPPORTED = 5
LBFS_ERR_LIMIT = 6

LBFS_FLAG_NONFINITE = 1
LBFS_FLAG_RHO_RANGE = 2
LBFS_FLAG_IBM_RANGE = 4

LBFS_FP64 = 0
LBFS_FP32_BULK = 1
LBFS_IBM_HAT2 = 2
LBFS_IBM_PESKIN4 = 4
LBFS_IBM_VANDERMONDE4 = 5

LBFS_NODES_POSITION = 0
LBFS_NODES_VELOCITY = 1
LBFS_NODES_FORCE = 2

LBFS_FIELD_GRADIENTS = 0
LBFS_FIELD_FACE_FLUX = 1
LBFS_FIELD_RESIDUAL = 2
LBFS_FIELD_FORCE = 3
LBFS_FIELD_T1 = 4
LBFS_FIELD_VISC = 5
LBFS_FIELD_GHOST = 6
LBFS_FIELD_SPRING = 7
LBFS_FIELD_DT_LOCAL = 8

LBFS_DT_LOCAL = 1
LBFS_DT_CONSTANT = 2
LBFS_DT_MIN = 3
LBFS_DT_TALTS = 4
LBFS_WRAP_OWN = 1
LBFS_WRAP_ALL = 2

LBFS_NOALLOC_MAX_BLOCKS = 65536
LBFS_NOALLOC_MAX_CELLS = LBFS_NOALLOC_MAX_BLOCKS * 256

_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.POINTER(ctypes.c_double)


class GridDesc(ctypes.Structure):
    _fields_ = [
        ("cell0", ctypes.c_int32), ("n_cells", ctypes.c_int32),
        ("origin", ctypes.c_double * 3), ("length", ctypes.c_double * 3),
        ("delta_x", ctypes.c_double), ("delta_h", ctypes.c_double),
    ]


class MeshDesc(ctypes.Structure):
    _fields_ = [
        ("n_cells", ctypes.c_int32), ("n_faces", ctypes.c_int32), ("n_interior", ctypes.c_int32),
        ("n_bc", ctypes.c_int32), ("n_face_x", ctypes.c_int32), ("n_face_y", ctypes.c_int32),
        ("n_face_z", ctypes.c_int32), ("axis_aligned", ctypes.c_int32),
        ("owner", _i32p), ("neighbour", _i32p), ("face_area", _f64p), ("face_normal", _f64p),
        ("face_centroid", _f64p), ("streaming_dt", _f64p), ("cell_volume", _f64p), ("cell_centroid", _f64p),
        ("gradient_stencil", _i32p), ("lhs_inverse", _f64p), ("rhs", _f64p),
        ("bc_rho_type", _i32p), ("bc_vel_type", _i32p), ("bc_values", _f64p),
        ("origin", ctypes.c_double * 3), ("length", ctypes.c_double * 3),
        ("delta_x", ctypes.c_double), ("delta_h", ctypes.c_double),
        ("n_instances", ctypes.c_int32), ("instances", ctypes.POINTER(GridDesc)),
        ("grid_x", _f64p), ("grid_y", _f64p), ("grid_z", _f64p),
        ("periodic_node", _i32p),
    ]


class Params(ctypes.Structure):
    _fields_ = [
        ("visc", ctypes.c_double), ("delta_t", ctypes.c_double), ("gamma_inv", ctypes.c_double),
        ("channel_diameter", ctypes.c_double), ("body_force", ctypes.c_double * 3),
        ("ref_rho", ctypes.c_double), ("max_velocity", ctypes.c_double), ("rho0", ctypes.c_double),
        ("visc_factor_initial", ctypes.c_double),
        ("testcase", ctypes.c_int32), ("precision", ctypes.c_int32), ("ibm_stencil", ctypes.c_int32),
        ("viscosity_period", ctypes.c_int32),
        ("time_stepping", ctypes.c_int32), ("pre_conditioned_gamma", ctypes.c_double),
        ("preconditioning", ctypes.c_int32),
    ]


class RbcDesc(ctypes.Structure):
    _fields_ = [
        ("n_nodes", ctypes.c_int32), ("n_tris", ctypes.c_int32), ("n_springs", ctypes.c_int32),
        ("tri", _i32p), ("spring", _i32p), ("xyz_stress_free", _f64p), ("xyz_initial", _f64p),
        ("volume_modulus", ctypes.c_double), ("local_area_modulus", ctypes.c_double),
        ("global_area_modulus", ctypes.c_double), ("shear_modulus", ctypes.c_double),
        ("global_bending_modulus", ctypes.c_double), ("local_bending_modulus", ctypes.c_double),
        ("membrane_thickness", ctypes.c_double), ("viscosity", ctypes.c_double),
        ("wlc_ratio", ctypes.c_double), ("curvature_ratio", ctypes.c_double), ("volume_ratio", ctypes.c_double),
        ("internal_viscosity_ratio", ctypes.c_double), ("reference_length", ctypes.c_double),
        ("pivkin_length", ctypes.c_int32), ("sphere_reference", ctypes.c_int32),
        ("instance", ctypes.c_int32), ("periodic", ctypes.c_int32),
    ]


class LaunchShape(ctypes.Structure):
    _fields_ = [
        ("gradient_threads", ctypes.c_int32), ("flux_threads", ctypes.c_int32),
        ("general_flux_threads", ctypes.c_int32), ("update_threads", ctypes.c_int32),
        ("update_blocks", ctypes.c_int32), ("spread_blocks", ctypes.c_int32), ("flux_chunks", ctypes.c_int32), ("membrane_cluster", ctypes.c_int32),
        ("membrane_after_k1", ctypes.c_int32), ("time_us", ctypes.c_double * 5),
    ]


class Objective(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("membrane", ctypes.c_int32), ("cell_weights", _f64p)]


LBFS_OBJ_VELOCITY = 0
LBFS_OBJ_TAYLOR = 1

LBFS_MAX_UPDATE_BLOCKS = 148 * 16
LBFS_MAX_SPREAD_BLOCKS = 148 * 16

_lib = None


def lib():
    """Load the shared library once; raise loudly when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with python lbfs-ibm-ade-sp_b200/build_lib.py")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        sig = {
            "lbfs_create": [ctypes.POINTER(MeshDesc), ctypes.POINTER(Params), ctypes.POINTER(RbcDesc), ctypes.c_int32,
                            ctypes.c_int32, ctypes.POINTER(vp)],
            "lbfs_destroy": [vp],
            "lbfs_set_state": [vp, _f64p, _f64p, _f64p, _f64p],
            "lbfs_get_state": [vp, _f64p, _f64p, _f64p, _f64p],
            "lbfs_step": [vp, ctypes.c_int32],
            "lbfs_step_graph": [vp, ctypes.c_int32],
            "lbfs_synchronize": [vp],
            "lbfs_set_stream": [vp, vp],
            "lbfs_get_nodes": [vp, ctypes.c_int32, _f64p],
            "lbfs_set_nodes": [vp, _f64p],
            "lbfs_get_totals": [vp, _f64p],
            "lbfs_get_residuals": [vp, _f64p],
            "lbfs_get_energies": [vp, _f64p],
            "lbfs_get_time_step": [vp, ctypes.POINTER(ctypes.c_double)],
            "lbfs_get_field": [vp, ctypes.c_int32, _f64p],
            "lbfs_keep_residuals": [vp, ctypes.c_int32],
            "lbfs_status": [vp, ctypes.POINTER(ctypes.c_uint32)],
            "lbfs_launches_per_step": [vp, _i32p],
            "lbfs_set_profiling": [vp, ctypes.c_int32],
            "lbfs_get_phase_times": [vp, _f64p],
            "lbfs_last_error": [ctypes.c_char_p, ctypes.c_int32],
            "lbfs_mesh_uniform_counts": [ctypes.c_double] * 4 + [_i32p],
            "lbfs_mesh_build_uniform": [ctypes.c_double] * 4 + [_f64p, ctypes.c_double, ctypes.c_double,
                                                                  ctypes.c_int32, _i32p, _i32p, _f64p, _f64p, _f64p,
                                                                  _f64p, _f64p, _f64p, _i32p, _f64p, _f64p, _i32p,
                                                                  _f64p],
            "lbfs_mesh_build_jittered": [ctypes.c_double] * 4 + [_f64p, ctypes.c_double, ctypes.c_double,
                                                                   ctypes.c_int32, ctypes.c_double, ctypes.c_uint64,
                                                                   ctypes.c_int32, _i32p, _i32p, _f64p, _f64p, _f64p,
                                                                   _f64p, _f64p, _f64p, _i32p, _f64p, _f64p, _i32p,
                                                                   _f64p],
            "lbfs_mesh_write_openfoam": [ctypes.c_char_p] + [ctypes.c_double] * 4 + [_f64p, ctypes.c_int32,
                                                                                       ctypes.c_double, ctypes.c_double,
                                                                                       ctypes.c_double, ctypes.c_uint64],
            "lbfs_mesh_openfoam_counts": [ctypes.c_char_p, _i32p],
            "lbfs_mesh_find_periodic_nodes": [ctypes.POINTER(MeshDesc), _f64p, _i32p],
            "lbfs_mesh_build_gpu": [ctypes.c_double] * 4 + [_f64p, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                                              ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                                              ctypes.c_double, ctypes.c_uint64, ctypes.c_int32,
                                                              ctypes.c_int32, _i32p, _i32p, _f64p, _f64p, _f64p,
                                                              _f64p, _f64p, _f64p, _i32p, _f64p, _f64p, _i32p,
                                                              _f64p, _f64p],
            "lbfs_mesh_import_openfoam": [ctypes.c_char_p, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                          ctypes.c_int32, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p,
                                          _i32p, _f64p, _f64p, _i32p, ctypes.c_char_p, ctypes.c_int32],
            "lbfs_mesh_import_openfoam_gpu": [ctypes.c_char_p, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                              ctypes.c_int32, ctypes.c_int32, _i32p, _i32p, _f64p, _f64p, _f64p,
                                              _f64p, _f64p, _f64p, _i32p, _f64p, _f64p, _i32p, ctypes.c_char_p,
                                              ctypes.c_int32],
            "lbfs_mesh_build_rectilinear": [ctypes.c_double] * 4 + [_f64p, ctypes.c_double, ctypes.c_double,
                                                                      ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                                                      ctypes.c_double, _i32p, _i32p, _f64p, _f64p,
                                                                      _f64p, _f64p, _f64p, _f64p, _i32p, _f64p,
                                                                      _f64p, _i32p, _f64p, _f64p],
            "lbfs_rbc_build_springs": [ctypes.c_int32, ctypes.c_int32, _i32p, ctypes.c_int32, _i32p, _i32p],
            "lbfs_residual_rms_noalloc": [vp, ctypes.c_int32, ctypes.c_double, ctypes.c_double, vp, vp],
            "lbfs_step_until": [vp, ctypes.c_int32, ctypes.c_double, ctypes.POINTER(ctypes.c_int32), _f64p],
            "lbfs_halo_bytes": [vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64)],
            "lbfs_halo_pack": [vp, ctypes.c_int32, ctypes.c_int32, vp],
            "lbfs_halo_unpack": [vp, ctypes.c_int32, ctypes.c_int32, vp],
            "lbfs_set_ibm_window": [vp, ctypes.c_int32, ctypes.c_int32],
            "lbfs_get_launch_shape": [vp, ctypes.POINTER(LaunchShape)],
            "lbfs_set_launch_shape": [vp, ctypes.POINTER(LaunchShape)],
            "lbfs_autotune": [vp, ctypes.c_int32, ctypes.POINTER(LaunchShape)],
            "lbfs_adjoint": [vp, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(Objective), _f64p, _f64p, _f64p],
            "lbfs_checkpoint_size": [vp, ctypes.POINTER(ctypes.c_uint64)],
            "lbfs_checkpoint_save": [vp, vp, ctypes.c_uint64],
            "lbfs_checkpoint_load": [vp, vp, ctypes.c_uint64],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        _lib = L
    return _lib


class LbfsError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"lbfs error {code}: {message}")
        self.code = code


def check(rc):
    if rc != LBFS_OK:
        buf = ctypes.create_string_buffer(512)
        lib().lbfs_last_error(buf, 512)
        raise LbfsError(rc, buf.value.decode(errors="replace"))


def ptr(a, ctype=ctypes.c_double):
    """Pointer to a C-contiguous numpy array (kept alive by the caller)."""
    assert a.flags["C_CONTIGUOUS"], "array must be C contiguous"
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def iptr(a):
    assert a.dtype == np.int32
    return ptr(a, ctypes.c_int32)


EXPORTED = [
    "lbfs_create", "lbfs_destroy", "lbfs_set_state", "lbfs_get_state", "lbfs_step", "lbfs_step_graph",
    "lbfs_synchronize", "lbfs_set_stream", "lbfs_get_nodes", "lbfs_set_nodes", "lbfs_get_totals",
    "lbfs_get_residuals", "lbfs_get_time_step", "lbfs_get_energies", "lbfs_get_field", "lbfs_keep_residuals", "lbfs_status", "lbfs_launches_per_step",
    "lbfs_set_profiling", "lbfs_get_phase_times",
    "lbfs_last_error", "lbfs_mesh_uniform_counts", "lbfs_mesh_build_uniform", "lbfs_rbc_build_springs",
    "lbfs_residual_rms_noalloc", "lbfs_get_launch_shape", "lbfs_set_launch_shape", "lbfs_autotune",
    "lbfs_adjoint", "lbfs_checkpoint_size", "lbfs_checkpoint_save", "lbfs_checkpoint_load",
    "lbfs_mesh_build_jittered", "lbfs_mesh_build_rectilinear", "lbfs_mesh_write_openfoam", "lbfs_mesh_openfoam_counts",
    "lbfs_mesh_import_openfoam", "lbfs_mesh_find_periodic_nodes", "lbfs_mesh_build_gpu",
    "lbfs_mesh_import_openfoam_gpu", "lbfs_step_until", "lbfs_halo_bytes", "lbfs_halo_pack", "lbfs_halo_unpack", "lbfs_set_ibm_window",
]
