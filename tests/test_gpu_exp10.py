"""The FP64 10^x of the Newton solves (cl_exp10: Cody-Waite reduction, a
degree-13 Taylor polynomial in Horner's form) against CUDA's exp10 and
against numpy's 10**x on the host, over the range the clamped logs reach and
the rest of its domain |x| < 300.

Bound: relative error <= 6e-16 (three units in the last place) against
both, on every point (Newton needs its species to ~1e-12: the tolerance is a
1e-10 relative residual).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_exp10_accuracy(gpu_lib, pkg):
    rng = np.random.default_rng(10)
    x = np.concatenate([rng.uniform(-31.0, 2.0, 200000), rng.uniform(-299.0, 299.0, 50000),
                        np.linspace(-30.0, 1.0, 3101), np.arange(-30, 23, dtype=np.float64)])
    ours = pkg.math_exp10(x, 0)
    cuda = pkg.math_exp10(x, 1)
    host = np.power(10.0, x)
    assert np.max(np.abs(ours - cuda) / cuda) <= 6e-16
    assert np.max(np.abs(ours - host) / host) <= 6e-16


def test_exp10_nan(gpu_lib, pkg):
    assert np.isnan(pkg.math_exp10(np.array([np.nan]), 0)[0])
