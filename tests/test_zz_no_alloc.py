"""lbfs_residual_rms_noalloc: the residual norms without any device allocation.

It serves callers that cannot call cudaMalloc (a host loop running inside a
CUDA-graph capture or a stream callback, or an integration whose device memory
belongs entirely to its own pool).  The test calls it through the C ABI on a
residual field produced by the solver, twice in a row (the second call reuses
the shared scratch array left by the first), and checks both results against
the solver's own residual norms (lbfs_get_residuals) within the FP64 tolerance
of the other parity tests.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from helpers import FP64_RTOL, rel_err
from lbfs_b200 import GpuSolver, _abi, cases

pytestmark = pytest.mark.gpu


def test_residual_rms_noalloc_matches_solver_twice():
    import torch

    c = cases.poiseuille(n=12, ny=10, nz=8)
    s = GpuSolver(c.mesh, c.params, c.membranes)
    s.set_state(c.rho, c.u, c.v, c.w)
    s.keep_residuals(True)
    lib = _abi.lib()
    for step in range(2):
        s.step(1)
        expected = s.residuals()
        res = torch.from_numpy(s.field(_abi.LBFS_FIELD_RESIDUAL)).cuda()  # the caller owns its buffers
        out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.lbfs_residual_rms_noalloc(ctypes.c_void_p(res.data_ptr()), c.mesh.n_cells, c.params.ref_rho,
                                           c.params.max_velocity, ctypes.c_void_p(out.data_ptr()), None)
        _abi.check(rc)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_err(got, expected) < FP64_RTOL, (step, got, expected)
    s.close()


def test_residual_rms_noalloc_multi_wave_grid_twice():
    """About 1e6 cells of synthetic residuals in a caller-owned tensor (3907 blocks, many waves
    on 148 SMs, so the last-block ticket and the strided gather of the partial sums both matter),
    against a torch FP64 reduction, called twice back to back on one stream."""
    import torch

    n = 1_000_003
    g = torch.Generator(device="cpu").manual_seed(7)
    res = (torch.rand((n, 4), generator=g, dtype=torch.float64) - 0.5).mul_(1e-3).cuda()
    ref_rho, max_velocity = 1.0, 0.01
    expected = torch.sqrt((res * res).sum(dim=0) / n).cpu().numpy()
    expected[1:] /= ref_rho * max_velocity
    expected[0] /= ref_rho
    outs = [torch.full((4,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
    stream = torch.cuda.Stream()
    lib = _abi.lib()
    torch.cuda.synchronize()
    for out in outs:
        rc = lib.lbfs_residual_rms_noalloc(ctypes.c_void_p(res.data_ptr()), n, ref_rho, max_velocity,
                                           ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        _abi.check(rc)
    stream.synchronize()
    for out in outs:
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_err(got, expected) < FP64_RTOL, (got, expected)


def test_residual_rms_noalloc_rejects_oversize():
    lib = _abi.lib()
    rc = lib.lbfs_residual_rms_noalloc(ctypes.c_void_p(16), _abi.LBFS_NOALLOC_MAX_CELLS + 1, 1.0, 0.01,
                                       ctypes.c_void_p(16), None)
    assert rc == _abi.LBFS_ERR_LIMIT
