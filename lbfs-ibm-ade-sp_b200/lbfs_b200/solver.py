"""Host-side mirror of the reference's GPU solver entry point.

GpuSolver is the time loop of gpu_solver::General_Purpose_Solver_mk_i
(Solver_gpu.cu:178-1275) over the C ABI: construction uploads the mesh and the
membranes and runs the membrane set-up (Solver_gpu.cu:659-735), step() advances
the time loop (one iteration = Solver_gpu.cu:749-1046), state() is the
write-back into Solution.  Errors surface as LbfsError, never as exit().
"""
import ctypes
from dataclasses import dataclass

import numpy as np

from . import _abi


@dataclass
class StepParams:
    """Scalars of global_variables / initial_conditions the step uses (values as
    after preprocessor::mach_number_factor and global_variables::initialise)."""
    visc: float
    delta_t: float = 1.0
    gamma_inv: float = 1.0
    channel_diameter: float = 1.0
    body_force: tuple = (0.0, 0.0, 0.0)
    ref_rho: float = 1.0
    max_velocity: float = 0.01
    rho0: float = 1.0
    visc_factor_initial: float = 1.0
    testcase: int = 1
    precision: int = _abi.LBFS_FP64
    ibm_stencil: int = _abi.LBFS_IBM_HAT2
    viscosity_period: int = 10000
    time_stepping: int = _abi.LBFS_DT_CONSTANT
    pre_conditioned_gamma: float = 0.0  # 0: 1 / gamma_inv
    preconditioning: int = 0             # globals.preconditioning_active

    def to_c(self):
        p = _abi.Params()
        p.visc, p.delta_t, p.gamma_inv = self.visc, self.delta_t, self.gamma_inv
        p.channel_diameter = self.channel_diameter
        p.body_force[:] = self.body_force
        p.ref_rho, p.max_velocity, p.rho0 = self.ref_rho, self.max_velocity, self.rho0
        p.visc_factor_initial = self.visc_factor_initial
        p.testcase, p.precision, p.ibm_stencil = self.testcase, self.precision, self.ibm_stencil
        p.viscosity_period = self.viscosity_period
        p.time_stepping, p.pre_conditioned_gamma = self.time_stepping, self.pre_conditioned_gamma
        p.preconditioning = self.preconditioning
        return p


def _shape_dict(sh):
    d = {name: getattr(sh, name) for name, _ in _abi.LaunchShape._fields_ if name != "time_us"}
    d["step_us"] = float(sh.time_us[0])
    return d


class GpuSolver:
    def __init__(self, mesh, params, membranes=(), device=0):
        self.mesh = mesh
        self.params = params
        self.membranes = list(membranes)
        self._mdesc = mesh.desc()
        self._pdesc = params.to_c()
        descs = [m.desc() for m in self.membranes]
        self._rdesc = (_abi.RbcDesc * max(1, len(descs)))(*descs) if descs else None
        h = ctypes.c_void_p()
        _abi.check(_abi.lib().lbfs_create(ctypes.byref(self._mdesc), ctypes.byref(self._pdesc),
                                          self._rdesc if self._rdesc is not None else None, len(descs), device,
                                          ctypes.byref(h)))
        self._h = h
        self.n_cells = mesh.n_cells
        self.total_nodes = sum(m.n_nodes for m in self.membranes)
        self.total_springs = sum(len(m.springs) for m in self.membranes)

    # -- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _abi.lib().lbfs_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state ----------------------------------------------------------------
    def set_state(self, rho, u, v, w):
        arrs = [np.ascontiguousarray(a, np.float64) for a in (rho, u, v, w)]
        for a in arrs:
            if a.shape != (self.n_cells,):
                raise ValueError("state arrays must have n_cells entries")
        _abi.check(_abi.lib().lbfs_set_state(self._h, *[_abi.ptr(a) for a in arrs]))

    def state(self):
        out = [np.empty(self.n_cells) for _ in range(4)]
        _abi.check(_abi.lib().lbfs_get_state(self._h, *[_abi.ptr(a) for a in out]))
        return tuple(out)

    def step(self, n=1, graph=False):
        fn = _abi.lib().lbfs_step_graph if graph else _abi.lib().lbfs_step
        _abi.check(fn(self._h, int(n)))

    def synchronize(self):
        _abi.check(_abi.lib().lbfs_synchronize(self._h))

    def step_until(self, max_steps, tolerance):
        """Up to max_steps steps, stopping after the first whose largest residual norm is below
        tolerance (or once the state diverged), the tests on the device.  Returns (steps, residuals)."""
        n = ctypes.c_int32()
        res = np.zeros(4)
        _abi.check(_abi.lib().lbfs_step_until(self._h, int(max_steps), float(tolerance), ctypes.byref(n), _abi.ptr(res)))
        return n.value, res

    # -- diagnostics ----------------------------------------------------------
    def nodes(self, which=_abi.LBFS_NODES_POSITION):
        out = np.zeros((self.total_nodes, 3))
        if self.total_nodes:
            _abi.check(_abi.lib().lbfs_get_nodes(self._h, which, _abi.ptr(out)))
        return out

    def set_nodes(self, xyz):
        a = np.ascontiguousarray(xyz, np.float64)
        _abi.check(_abi.lib().lbfs_set_nodes(self._h, _abi.ptr(a)))

    def totals(self):
        """(n_membranes, 6): V, V0, A, A0, MAD, MAD0."""
        out = np.zeros((max(1, len(self.membranes)), 6))
        if self.membranes:
            _abi.check(_abi.lib().lbfs_get_totals(self._h, _abi.ptr(out)))
        return out[: len(self.membranes)]

    def energies(self):
        """Per membrane: volume, global area, local area, local bending, ADE, spring, total energy."""
        out = np.zeros((max(1, len(self.membranes)), 7))
        if self.membranes:
            _abi.check(_abi.lib().lbfs_get_energies(self._h, _abi.ptr(out)))
        return out[: len(self.membranes)]

    def residuals(self):
        out = np.zeros(4)
        _abi.check(_abi.lib().lbfs_get_residuals(self._h, _abi.ptr(out)))
        return out

    def keep_residuals(self, on=True):
        _abi.check(_abi.lib().lbfs_keep_residuals(self._h, 1 if on else 0))

    def field(self, which):
        m = self.mesh
        nt = m.n_cells + m.n_bc
        size = {
            _abi.LBFS_FIELD_GRADIENTS: 12 * nt, _abi.LBFS_FIELD_FACE_FLUX: 4 * m.n_faces,
            _abi.LBFS_FIELD_RESIDUAL: 4 * m.n_cells, _abi.LBFS_FIELD_FORCE: 3 * m.n_cells,
            _abi.LBFS_FIELD_T1: 4 * m.n_cells, _abi.LBFS_FIELD_VISC: m.n_cells, _abi.LBFS_FIELD_GHOST: 4 * m.n_bc,
            _abi.LBFS_FIELD_SPRING: 9 * self.total_springs, _abi.LBFS_FIELD_DT_LOCAL: m.n_cells,
        }[which]
        out = np.zeros(max(size, 1))
        _abi.check(_abi.lib().lbfs_get_field(self._h, which, _abi.ptr(out)))
        return out[:size]

    def time_step(self):
        """The delta_t of the last step (the minimum per-cell step unless constant)."""
        dt = ctypes.c_double()
        _abi.check(_abi.lib().lbfs_get_time_step(self._h, ctypes.byref(dt)))
        return dt.value

    def status(self):
        f = ctypes.c_uint32()
        _abi.check(_abi.lib().lbfs_status(self._h, ctypes.byref(f)))
        return f.value

    def set_profiling(self, level=2):
        """0 off, 1 whole-step events, 2 whole-step and per-kernel events."""
        _abi.check(_abi.lib().lbfs_set_profiling(self._h, int(level)))

    def phase_times(self):
        """Durations (ms) of the last step: membrane, gradients, flux, update, viscosity kernels, whole step."""
        out = np.zeros(6)
        _abi.check(_abi.lib().lbfs_get_phase_times(self._h, _abi.ptr(out)))
        return out

    def set_stream(self, stream_ptr):
        _abi.check(_abi.lib().lbfs_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    # -- slab decomposition -----------------------------------------------------
    def halo_bytes(self, n_cells):
        """Bytes of a halo buffer for n_cells cells (state records, then FP64 accumulators)."""
        b = ctypes.c_uint64()
        _abi.check(_abi.lib().lbfs_halo_bytes(self._h, int(n_cells), ctypes.byref(b)))
        return b.value

    def halo_pack(self, first_cell, n_cells, device_ptr):
        """Copy cells [first_cell, first_cell + n_cells) into a device buffer (on the handle's stream)."""
        _abi.check(_abi.lib().lbfs_halo_pack(self._h, int(first_cell), int(n_cells), ctypes.c_void_p(device_ptr)))

    def halo_unpack(self, first_cell, n_cells, device_ptr):
        """Overwrite cells [first_cell, first_cell + n_cells) from a device buffer (on the handle's stream)."""
        _abi.check(_abi.lib().lbfs_halo_unpack(self._h, int(first_cell), int(n_cells), ctypes.c_void_p(device_ptr)))

    def set_ibm_window(self, z_lo, z_hi):
        """Confine the membranes' IBM patches to z cells [z_lo, z_hi) of the grid (else LBFS_FLAG_IBM_RANGE)."""
        _abi.check(_abi.lib().lbfs_set_ibm_window(self._h, int(z_lo), int(z_hi)))

    def launch_shape(self):
        """Current launch shape as a dict (block sizes, grid caps)."""
        sh = _abi.LaunchShape()
        _abi.check(_abi.lib().lbfs_get_launch_shape(self._h, ctypes.byref(sh)))
        return _shape_dict(sh)

    def set_launch_shape(self, **kw):
        """Change some fields of the launch shape (the rest stay)."""
        sh = _abi.LaunchShape()
        _abi.check(_abi.lib().lbfs_get_launch_shape(self._h, ctypes.byref(sh)))
        for k, v in kw.items():
            if k in ("time_us", "step_us") or not hasattr(sh, k):
                raise KeyError(k)
            setattr(sh, k, int(v))
        _abi.check(_abi.lib().lbfs_set_launch_shape(self._h, ctypes.byref(sh)))

    def autotune(self, reps=20):
        """Search the launch shape by timing whole steps from this handle's state
        (which it puts back); returns the choice and its step time (us)."""
        sh = _abi.LaunchShape()
        _abi.check(_abi.lib().lbfs_autotune(self._h, int(reps), ctypes.byref(sh)))
        return _shape_dict(sh)

    def adjoint(self, n_steps, checkpoint_every=25, weights=None, membrane=None):
        """Discrete adjoint over n_steps from the current state.  Objective: the
        Taylor deformation of `membrane` (x-y plane) when given, else
        sum_c weights[c] . (u, v, w)_c at the final step.  Returns
        (J, {"shear_modulus", "bending_modulus", "velocity_scale"}, times_ms);
        the handle ends on the final forward state."""
        obj = _abi.Objective()
        keep = None
        if membrane is not None:
            obj.kind, obj.membrane = _abi.LBFS_OBJ_TAYLOR, int(membrane)
        else:
            keep = np.ascontiguousarray(weights, np.float64).reshape(-1)
            if keep.size != 3 * self.n_cells:
                raise ValueError("weights: 3 per interior cell")
            obj.kind, obj.cell_weights = _abi.LBFS_OBJ_VELOCITY, _abi.ptr(keep)
        J = ctypes.c_double()
        g = np.zeros(3)
        t = np.zeros(2)
        _abi.check(_abi.lib().lbfs_adjoint(self._h, int(n_steps), int(checkpoint_every), ctypes.byref(obj),
                                           ctypes.byref(J), _abi.ptr(g), _abi.ptr(t)))
        return J.value, dict(zip(("shear_modulus", "bending_modulus", "velocity_scale"), g.tolist())), t.tolist()

    def checkpoint(self):
        """Lossless snapshot of the handle's state (bytes)."""
        n = ctypes.c_uint64()
        _abi.check(_abi.lib().lbfs_checkpoint_size(self._h, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        _abi.check(_abi.lib().lbfs_checkpoint_save(self._h, buf, n.value))
        return buf.raw

    def restore(self, blob):
        """Resume from a snapshot taken by checkpoint() on a handle of the same case."""
        buf = ctypes.create_string_buffer(blob, len(blob))
        _abi.check(_abi.lib().lbfs_checkpoint_load(self._h, buf, len(blob)))

    def launches_per_step(self):
        n = ctypes.c_int32()
        _abi.check(_abi.lib().lbfs_launches_per_step(self._h, ctypes.byref(n)))
        return n.value
