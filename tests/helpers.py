"""Shared helpers of the parity tests."""
import numpy as np


def rel_err(a, b):
    """max |a - b| / max |b| (0 when both are zero)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = np.max(np.abs(b)) if b.size else 0.0
    diff = np.max(np.abs(a - b)) if a.size else 0.0
    return 0.0 if diff == 0.0 else diff / max(scale, 1e-300)


# Tolerances, relative to the largest magnitude of the compared field.
FP64_RTOL = 1e-10   # FP64 path vs the reference / the oracle (stated in the north-star contract)
FP32_RTOL = 1e-6    # FP32-bulk path vs the FP64 path: every velocity component, relative to its own largest magnitude
