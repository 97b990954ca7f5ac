"""cl_eq_solve_noalloc: the batch speciation entry point that allocates
nothing, for callers that may not allocate device memory (a framework's
caching allocator owns the GPU's memory, or a cudaMalloc/cudaFree between
stream-ordered kernels would synchronise the device).  Its scratch is a fixed
array inside the library.

Checked through the C ABI against the existing entry point
(cl_eq_solve_device) on the same inputs, on two calls in a row, within the
tolerance the other speciation tests use (1e-8 in log10 free concentration;
statuses and iteration counts equal), and the converged solutions checked
against the FP64 oracle's relative mass-balance residual (<= 1e-10).
Collected last so that a run stopping at the first failure has already run
every other test."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as o

pytestmark = pytest.mark.gpu


def _bind(lib):
    vp = ctypes.c_void_p
    lib.cl_eq_solve_noalloc.restype = ctypes.c_int
    lib.cl_eq_solve_noalloc.argtypes = [vp, vp, vp, vp, vp, vp, ctypes.c_int64, ctypes.c_int32, vp]
    return lib


def test_noalloc_matches_existing_entry_point(gpu_lib, pkg, wl):
    import torch
    lib = _bind(gpu_lib)
    S, logk, cs = wl.tableau(5, 9, seed=4)
    sys_ = pkg.EqSystem()
    pkg.set_eq_system(sys_, S, logk, cs, max_iter=200, tol=1e-10, warm_iter=4)
    n = 20000
    T, xs, _, _ = wl.speciation_batch(S, logk, n, seed=909)
    rng = np.random.default_rng(1)
    x0 = xs + rng.normal(0, 0.8, xs.shape)          # a rough warm start: some voxels fall back
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    dev = dict(device="cuda")
    dT = torch.tensor(T, dtype=torch.float64, **dev)
    dC = torch.tensor(wl.cold_species(S, T, cs), dtype=torch.float64, **dev)

    def run_existing():
        eq = pkg.EqSolver(sys_, stream=stream.cuda_stream)
        X = torch.tensor(x0, dtype=torch.float64, **dev)
        I = torch.zeros(n, dtype=torch.int32, **dev)
        St = torch.zeros(n, dtype=torch.uint8, **dev)
        eq.solve_device(dT.data_ptr(), dC.data_ptr(), X.data_ptr(), I.data_ptr(), St.data_ptr(), n,
                        pkg.EQ_START_GIVEN)
        torch.cuda.synchronize()
        eq.close()
        return X.cpu().numpy(), I.cpu().numpy(), St.cpu().numpy()

    def run_noalloc():
        X = torch.tensor(x0, dtype=torch.float64, **dev)
        I = torch.zeros(n, dtype=torch.int32, **dev)
        St = torch.full((n,), 255, dtype=torch.uint8, **dev)
        st = lib.cl_eq_solve_noalloc(ctypes.byref(sys_), dT.data_ptr(), dC.data_ptr(), X.data_ptr(), I.data_ptr(),
                                     St.data_ptr(), n, pkg.EQ_START_GIVEN, stream.cuda_stream)
        assert st == pkg.OK, lib.cl_last_error()
        torch.cuda.synchronize()
        return X.cpu().numpy(), I.cpu().numpy(), St.cpu().numpy()

    xr, ir, sr = run_existing()
    assert (sr == 1).sum() > 0, "the warm start should leave some voxels to the cold fallback"
    for _ in range(2):                                # two calls in a row share the fixed scratch
        xn, inn, sn = run_noalloc()
        np.testing.assert_array_equal(sn, sr)
        np.testing.assert_array_equal(inn, ir)
        ok = sr <= 1
        np.testing.assert_allclose(xn[ok], xr[ok], rtol=0, atol=1e-8)
        sample = np.nonzero(ok)[0][::10]
        assert np.all(o.eq_residual(sys_, T[sample], xn[sample]) <= 1e-10)


def test_noalloc_rejects_oversize_batch(gpu_lib, pkg, wl):
    lib = _bind(gpu_lib)
    S, logk, cs = wl.tableau(5, 9, seed=4)
    sys_ = pkg.EqSystem()
    pkg.set_eq_system(sys_, S, logk, cs)
    dummy = ctypes.c_void_p(16)                      # never dereferenced: the size check comes first
    st = lib.cl_eq_solve_noalloc(ctypes.byref(sys_), dummy, dummy, dummy, None, None, (1 << 20) + 1,
                                 pkg.EQ_START_COLD, None)
    assert st == pkg.ERR_ARG
    assert b"CL_EQ_NOALLOC_MAX_N" in lib.cl_last_error()
