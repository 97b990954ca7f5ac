"""Surrogate rate network on the GPU: the shipped network (golden fixture from
the reference's defineSurrogateModel) through the FP32 CUDA-core kernel, and
the BF16 tensor-core kernel against the FP32 kernel.

Tolerances: FP32 kernel vs FP64 reference 1e-5 relative; BF16 tensor-core
kernel vs the FP32 kernel and vs the FP64 oracle 2e-2 of the output span
2/y_gain (BF16 operands, FP32 accumulate).
"""
import numpy as np
import pytest

from oracle import oracle as o
from test_golden import shipped_net

pytestmark = pytest.mark.gpu


def test_shipped_network_fp32(gpu_lib, pkg):
    net, z = shipped_net(pkg)
    y = pkg.surrogate_batch(net, z["fin"].astype(np.float32), mode=pkg.SRG_FP32)[:, 0].astype(np.float64)
    yo = o.surrogate_forward(net, z["fin"].astype(np.float32).astype(np.float64))[:, 0]
    np.testing.assert_allclose(y, yo, rtol=1e-4, atol=2e-6)
    ref = z["bior"]
    big = ref > 1e-3
    np.testing.assert_allclose(y[big], ref[big], rtol=1e-3)


def c4_net(pkg, seed=0):
    rng = np.random.default_rng(seed)
    widths = [3, 20, 20, 4]
    W = [rng.normal(0, 0.3, (widths[l + 1], widths[l])) for l in range(3)]
    b = [rng.normal(0, 0.3, widths[l + 1]) for l in range(3)]
    lo = np.array([1e-4, 1e-5, 1.0]); hi = np.array([1e-1, 5e-2, 100.0])
    gain = 2.0 / (hi - lo)
    return pkg.make_surrogate_net(widths, W, b, lo, gain, [0.0] * 4, [20.0, 40.0, 40.0, 40.0], x_lo=lo, x_hi=hi)


@pytest.mark.parametrize("n", [1, 15, 16, 1000, 100003])
def test_tensor_core_matches_fp32(gpu_lib, pkg, n):
    net = c4_net(pkg)
    rng = np.random.default_rng(n)
    x = np.stack([rng.uniform(0, 0.12, n), rng.uniform(0, 0.06, n), rng.uniform(0, 120, n)], 1).astype(np.float32)
    y32 = pkg.surrogate_batch(net, x, mode=pkg.SRG_FP32)
    ytc = pkg.surrogate_batch(net, x, mode=pkg.SRG_TENSOR)
    yo = o.surrogate_forward(net, x.astype(np.float64))
    # the network's output span: mapminmax maps [-1, 1] onto 2 / y_gain
    span = np.array([2.0 / net.y_gain[o] for o in range(4)])
    assert np.max(np.abs(y32 - yo) / span) < 1e-5
    assert np.max(np.abs(ytc - y32) / span) < 2e-2
    assert np.max(np.abs(ytc - yo) / span) < 2e-2       # the tensor path against FP64 directly
    # the tcgen05 path: the same BF16 operands and activations as the warp
    # MMA path, only the order of the FP32 sums differs
    y5 = pkg.surrogate_batch(net, x, mode=pkg.SRG_TCGEN05)
    assert np.isfinite(y5).all()
    assert np.max(np.abs(y5 - ytc) / span) < 5e-3
    assert np.max(np.abs(y5 - yo) / span) < 2e-2
