"""Device arithmetic that the fused forms build themselves, checked against correctly rounded values.

The Kurganov-Petrova flux divides by a+ - a- through the hardware reciprocal refined by one
Newton-Raphson step (rcp_newton in fused.cu).  Without the step the reciprocal carries a small
systematic bias, and the compensated form's water volume drifted from the FP64 oracle through the
fluxes at open boundaries.  Here the refined values are compared with IEEE single-precision 1/x
(numpy rounds float32 division correctly) over the range the denominators take (wave speeds of
1e-3 .. 1e3 m/s) and beyond: within one unit in the last place everywhere, equal to the correctly
rounded value almost everywhere, and without a bias in either direction.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_flux_reciprocal_is_within_one_ulp_and_unbiased(celeris):
    rng = np.random.default_rng(11)
    x = np.concatenate([np.logspace(-6, 6, 200_001), rng.uniform(1e-3, 1e3, 200_000),
                        rng.uniform(0.5, 1.0, 100_000)]).astype(np.float32)
    out = np.zeros_like(x)
    fp = C.POINTER(C.c_float)
    st = celeris.lib().cel_selftest_reciprocal(x.ctypes.data_as(fp), out.ctypes.data_as(fp), len(x))
    assert st == 0, celeris.lib().cel_last_error().decode()
    exact = np.float32(1.0) / x
    ulp = np.abs(out.view(np.int32).astype(np.int64) - exact.view(np.int32).astype(np.int64))
    assert ulp.max() <= 1
    assert (ulp == 0).mean() > 0.99
    signed = (out.astype(np.float64) - exact.astype(np.float64)) / exact.astype(np.float64)
    assert abs(signed.mean()) < 1e-10
