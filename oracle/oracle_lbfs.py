"""ctypes front end of the C restatement oracle (oracle/lbfs_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline as the CPU checker.  Same interface as
lbfs_b200.GpuSolver so parity tests read symmetrically.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "liblbfs_oracle.so")

FIELD_SIZES = None
_lib = None


def build():
    subprocess.run(["bash", os.path.join(HERE, "build_oracle.sh")], check=True, capture_output=True)


def lib():
    global _lib
    if _lib is None:
        srcs = [os.path.join(HERE, "lbfs_oracle.c"), os.path.join(HERE, "..", "include", "lbfs_b200.h")]
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(os.path.getmtime(f) for f in srcs):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [vp, vp, vp, ctypes.c_int]
        L.oracle_free.argtypes = [vp]
        L.oracle_set_state.argtypes = [vp] + [vp] * 4
        L.oracle_get_state.argtypes = [vp] + [vp] * 4
        L.oracle_step.argtypes = [vp, ctypes.c_int]
        L.oracle_get_field.argtypes = [vp, ctypes.c_int, vp]
        L.oracle_get_nodes.argtypes = [vp, ctypes.c_int, vp]
        L.oracle_get_totals.argtypes = [vp, vp]
        L.oracle_get_residuals.argtypes = [vp, vp]
        L.oracle_get_energies.argtypes = [vp, vp]
        L.oracle_time_step.argtypes = [vp]
        L.oracle_time_step.restype = ctypes.c_double
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class OracleSolver:
    """CPU oracle with GpuSolver's interface (mesh, StepParams, Membrane list)."""

    def __init__(self, mesh, params, membranes=()):
        self.mesh = mesh
        self.membranes = list(membranes)
        self._mdesc = mesh.desc()
        self._pdesc = params.to_c()
        descs = [m.desc() for m in self.membranes]
        self._rdesc = None
        if descs:
            T = type(descs[0]) * len(descs)
            self._rdesc = T(*descs)
        self.h = lib().oracle_create(ctypes.addressof(self._mdesc), ctypes.addressof(self._pdesc),
                                     ctypes.addressof(self._rdesc) if self._rdesc is not None else None, len(descs))
        if not self.h:
            raise ValueError("the oracle runs one case at a time (no ensemble instance table)")
        self.n_cells = mesh.n_cells
        self.total_nodes = sum(m.n_nodes for m in self.membranes)
        self.total_springs = sum(len(m.springs) for m in self.membranes)

    def close(self):
        if self.h:
            lib().oracle_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, rho, u, v, w):
        arrs = [np.ascontiguousarray(a, np.float64) for a in (rho, u, v, w)]
        lib().oracle_set_state(self.h, *[_p(a) for a in arrs])

    def state(self):
        out = [np.empty(self.n_cells) for _ in range(4)]
        lib().oracle_get_state(self.h, *[_p(a) for a in out])
        return tuple(out)

    def step(self, n=1, graph=False):
        lib().oracle_step(self.h, int(n))

    def synchronize(self):
        pass

    def nodes(self, which=0):
        out = np.zeros((self.total_nodes, 3))
        if self.total_nodes:
            lib().oracle_get_nodes(self.h, which, _p(out))
        return out

    def totals(self):
        out = np.zeros((max(1, len(self.membranes)), 6))
        if self.membranes:
            lib().oracle_get_totals(self.h, _p(out))
        return out[: len(self.membranes)]

    def residuals(self):
        out = np.zeros(4)
        lib().oracle_get_residuals(self.h, _p(out))
        return out

    def field(self, which):
        m = self.mesh
        nt = m.n_cells + m.n_bc
        size = {0: 12 * nt, 1: 4 * m.n_faces, 2: 4 * m.n_cells, 3: 3 * m.n_cells, 4: 4 * m.n_cells, 5: m.n_cells,
                6: 4 * m.n_bc, 7: 9 * self.total_springs, 8: m.n_cells}[which]
        out = np.zeros(max(size, 1))
        lib().oracle_get_field(self.h, which, _p(out))
        return out[:size]

    def time_step(self):
        return lib().oracle_time_step(self.h)

    def energies(self):
        out = np.zeros((max(1, len(self.membranes)), 7))
        if self.membranes:
            lib().oracle_get_energies(self.h, _p(out))
        return out[: len(self.membranes)]
