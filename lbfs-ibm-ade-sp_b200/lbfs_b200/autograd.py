"""torch.autograd bridge to the discrete adjoint (lbfs_adjoint).

`deformation(theta, case, n_steps, checkpoint_every, membrane)` returns the
Taylor deformation of one red cell after n_steps as a differentiable function
of theta = (s_G, s_b, s_U), multipliers of every membrane's shear modulus, of
every membrane's global bending modulus and of every boundary velocity value
(theta = 1 is the case as given).  The forward pass runs the solver and the
adjoint sweep once; backward returns the stored gradient, so
torch.autograd.gradcheck compares the adjoint against central differences of
the same solver.  `flow_functional` is the same for J = sum_c w_c . u_c.
"""
from dataclasses import replace

import numpy as np
import torch

from .solver import GpuSolver

__all__ = ["deformation", "flow_functional", "AdjointFunction"]


def _run(case, theta, n_steps, checkpoint_every, membrane, weights, device):
    sg, sb, su = (float(t) for t in theta)
    mems = [replace(m, shear_modulus=m.shear_modulus * sg, global_bending_modulus=m.global_bending_modulus * sb)
            for m in case.membranes]
    bcv = case.mesh.bc_values
    keep = bcv.copy()
    bcv[:, :3] *= su
    try:
        with GpuSolver(case.mesh, case.params, mems, device=device) as s:
            s.set_state(case.rho, case.u, case.v, case.w)
            J, g, _ = s.adjoint(n_steps, checkpoint_every, weights=weights, membrane=membrane)
    finally:
        bcv[:] = keep
    # chain rule to the multipliers
    G0 = case.membranes[0].shear_modulus if case.membranes else 0.0
    B0 = case.membranes[0].global_bending_modulus if case.membranes else 0.0
    if case.membranes and any(m.shear_modulus != G0 or m.global_bending_modulus != B0 for m in case.membranes):
        raise ValueError("the multipliers assume one shear and one bending modulus for every membrane")
    return J, np.array([g["shear_modulus"] * G0, g["bending_modulus"] * B0, g["velocity_scale"]])


class AdjointFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, case, n_steps, checkpoint_every, membrane, weights, device):
        J, grad = _run(case, theta.detach().cpu().numpy(), n_steps, checkpoint_every, membrane, weights, device)
        ctx.save_for_backward(torch.as_tensor(grad, dtype=theta.dtype, device=theta.device))
        return torch.as_tensor(J, dtype=theta.dtype, device=theta.device)

    @staticmethod
    def backward(ctx, gJ):
        (grad,) = ctx.saved_tensors
        return gJ * grad, None, None, None, None, None, None


def deformation(theta, case, n_steps, checkpoint_every=25, membrane=0, device=0):
    return AdjointFunction.apply(theta, case, n_steps, checkpoint_every, membrane, None, device)


def flow_functional(theta, case, weights, n_steps, checkpoint_every=25, device=0):
    return AdjointFunction.apply(theta, case, n_steps, checkpoint_every, None, weights, device)
