"""Discrete adjoint: gradients against central finite differences.

The objective is evaluated after N forward steps; the adjoint sweeps back over
checkpointed segments.  Fluid sensitivities: h = 1e-6 relative, agreement to
1e-5 relative.  Membrane moduli: over the few steps a test can afford, the
Taylor deformation moves by ~1e-12 of itself for a 1e-6 change of G_s or k_b,
which is the rounding noise of the forward runs, so the central differences
use h = 1e-4 (converged: 1e-5, 1e-4 and 1e-3 agree to 1e-7) and must agree to
1e-5 relative.
"""
import numpy as np
import pytest

FD_H = 1e-6
FD_H_MODULI = 1e-4
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


def _rbc_case(level=2):
    from dataclasses import replace
    from lbfs_b200 import cases
    c = cases.shear_channel(16, n_rbc=1, level=level, radius_cells=3.0, shear_modulus=2e-4, capillary=0.3, seed=5)
    # interior viscosity ratio 1: the viscosity update at t = 1 leaves the field unchanged
    c.membranes = [replace(m, internal_viscosity_ratio=1.0) for m in c.membranes]
    return c


def _taylor(c, steps, membranes=None, sigma=1.0):
    from lbfs_b200 import GpuSolver
    bcv = c.mesh.bc_values
    keep = bcv.copy()
    bcv[:, :3] *= sigma
    try:
        with GpuSolver(c.mesh, c.params, membranes if membranes is not None else c.membranes) as s:
            s.set_state(c.rho, c.u, c.v, c.w)
            s.step(steps)
            xyz = s.nodes().reshape(-1, 3)
            assert s.status() == 0
    finally:
        bcv[:] = keep
    x, y = xyz[:, 0], xyz[:, 1]
    dx, dy = x - x.mean(), y - y.mean()
    Ixx, Iyy, Ixy = np.sum(dx * dx), np.sum(dy * dy), np.sum(dx * dy)
    T, D = 0.5 * (Ixx + Iyy), 0.5 * (Ixx - Iyy)
    R = np.sqrt(D * D + Ixy * Ixy)
    L, B = np.sqrt(T + R), np.sqrt(T - R)
    return (L - B) / (L + B)


@pytest.mark.gpu
def test_membrane_adjoint_matches_finite_differences():
    from dataclasses import replace
    from lbfs_b200 import GpuSolver
    c = _rbc_case()
    steps, K = 24, 5
    with GpuSolver(c.mesh, c.params, c.membranes) as s:
        s.set_state(c.rho, c.u, c.v, c.w)
        J, g, _ = s.adjoint(steps, K, membrane=0)
    J0 = _taylor(c, steps)
    assert abs(J - J0) <= 1e-12 * abs(J0)
    m = c.membranes[0]
    h = FD_H_MODULI
    fd_gs = (_taylor(c, steps, [replace(m, shear_modulus=m.shear_modulus * (1 + h))]) -
             _taylor(c, steps, [replace(m, shear_modulus=m.shear_modulus * (1 - h))])) / (2 * h * m.shear_modulus)
    kb = m.global_bending_modulus
    fd_kb = (_taylor(c, steps, [replace(m, global_bending_modulus=kb * (1 + h))]) -
             _taylor(c, steps, [replace(m, global_bending_modulus=kb * (1 - h))])) / (2 * h * kb)
    for name, fd in (("shear_modulus", fd_gs), ("bending_modulus", fd_kb)):
        assert abs(g[name] - fd) <= FD_RTOL * abs(fd), (name, g[name], fd)


@pytest.mark.gpu
@pytest.mark.parametrize("objective", ["taylor", "velocity"])
def test_stored_trajectory_equals_segment_reruns(objective, monkeypatch):
    """The adjoint keeps every segment's intermediates from the forward sweep when they fit
    (the default here), or re-runs each segment from its checkpoint (LBFS_ADJOINT_MEMORY_MB=0):
    the same kernels on the same inputs, so J and the gradients agree bit for bit, and the
    handle ends in the same state."""
    from lbfs_b200 import GpuSolver
    c = _rbc_case()
    steps, K = 20, 6
    weights = np.random.default_rng(5).uniform(-1, 1, (c.mesh.n_cells, 3))
    out = []
    for budget in (None, "0"):
        if budget is None:
            monkeypatch.delenv("LBFS_ADJOINT_MEMORY_MB", raising=False)
        else:
            monkeypatch.setenv("LBFS_ADJOINT_MEMORY_MB", budget)
        with GpuSolver(c.mesh, c.params, c.membranes) as s:
            s.set_state(c.rho, c.u, c.v, c.w)
            if objective == "taylor":
                J, g, _ = s.adjoint(steps, K, membrane=0)
            else:
                J, g, _ = s.adjoint(steps, K, weights=weights)
            out.append((J, g, s.state(), s.nodes()))
    (Ja, ga, sa, na), (Jb, gb, sb, nb) = out
    assert Ja == Jb
    assert ga == gb
    for x, y in zip(sa, sb):
        assert np.array_equal(x, y)
    assert np.array_equal(na, nb)


@pytest.mark.gpu
def test_coupled_adjoint_velocity_objective():
    """Velocity objective with a red cell in the flow: the fluid adjoint runs
    through the IBM coupling (spread and interpolation transposes, springs)."""
    from dataclasses import replace
    from lbfs_b200 import GpuSolver
    c = _rbc_case()
    steps, K = 20, 6
    rng = np.random.default_rng(3)
    weights = rng.uniform(-1, 1, (c.mesh.n_cells, 3))
    with GpuSolver(c.mesh, c.params, c.membranes) as s:
        s.set_state(c.rho, c.u, c.v, c.w)
        J, g, _ = s.adjoint(steps, K, weights=weights)
    assert abs(J - _objective(c, 1.0, steps, weights)) <= 1e-12 * max(1.0, abs(J))
    fd = (_objective(c, 1 + FD_H, steps, weights) - _objective(c, 1 - FD_H, steps, weights)) / (2 * FD_H)
    assert abs(g["velocity_scale"] - fd) <= FD_RTOL * abs(fd), (g, fd)
    m = c.membranes[0]
    h = FD_H_MODULI

    def with_gs(f):
        cc = replace(c, membranes=[replace(m, shear_modulus=m.shear_modulus * f)])
        return _objective(cc, 1.0, steps, weights)
    fd_gs = (with_gs(1 + h) - with_gs(1 - h)) / (2 * h * m.shear_modulus)
    assert abs(g["shear_modulus"] - fd_gs) <= FD_RTOL * abs(fd_gs), (g, fd_gs)


@pytest.mark.gpu
def test_torch_gradcheck_through_the_adjoint():
    """torch.autograd.gradcheck of the Taylor deformation in the multipliers of
    (shear modulus, bending modulus, boundary velocity), central differences."""
    import torch
    from lbfs_b200.autograd import deformation
    c = _rbc_case()
    theta = torch.ones(3, dtype=torch.float64, requires_grad=True)
    f = lambda t: deformation(t, c, 16, 5)
    assert torch.autograd.gradcheck(f, (theta,), eps=FD_H_MODULI, atol=1e-9, rtol=FD_RTOL, fast_mode=False)
