"""Discrete adjoint: gradients against central finite differences.

The objective is evaluated after N forward steps; the adjoint sweeps back over
checkpointed segments.  Finite differences use h = 1e-6 relative, as the
adjoint configuration prescribes, and must agree to 1e-5 relative.
"""
import numpy as np
import pytest

FD_H = 1e-6
FD_RTOL = 1e-5


def _shear(n=10, general=False):
    from lbfs_b200 import cases
    c = cases.shear_channel(n, n_rbc=0, shear_modulus=1e-5, capillary=0.2)
    if general:
        desc = c.mesh.desc

        def general_desc():
            d = desc()
            d.axis_aligned = 0
            return d
        c.mesh.desc = general_desc
    return c


def _objective(c, sigma, steps, weights):
    from lbfs_b200 import GpuSolver
    bcv = c.mesh.bc_values
    keep = bcv.copy()
    bcv[:, :3] *= sigma
    try:
        with GpuSolver(c.mesh, c.params, c.membranes) as s:
            s.set_state(c.rho, c.u, c.v, c.w)
            s.step(steps)
            _, u, v, w = s.state()
    finally:
        bcv[:] = keep
    return float(np.sum(weights[:, 0] * u + weights[:, 1] * v + weights[:, 2] * w))


@pytest.mark.gpu
@pytest.mark.parametrize("general", [False, True], ids=["axis", "general"])
def test_fluid_adjoint_matches_finite_differences(general):
    from lbfs_b200 import GpuSolver
    c = _shear(general=general)
    steps, K = 30, 7
    rng = np.random.default_rng(11)
    weights = rng.uniform(-1, 1, (c.mesh.n_cells, 3))
    with GpuSolver(c.mesh, c.params, c.membranes) as s:
        s.set_state(c.rho, c.u, c.v, c.w)
        J, g, _ = s.adjoint(steps, K, weights=weights)
    J0 = _objective(c, 1.0, steps, weights)
    assert abs(J - J0) <= 1e-12 * max(1.0, abs(J0))
    fd = (_objective(c, 1 + FD_H, steps, weights) - _objective(c, 1 - FD_H, steps, weights)) / (2 * FD_H)
    assert abs(g["velocity_scale"] - fd) <= FD_RTOL * abs(fd), (g, fd)
