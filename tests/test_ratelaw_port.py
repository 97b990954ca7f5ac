"""The library's compiled rate laws (include/complab_ratelaw.hpp, built for
the host) against the reference's own rate-law headers compiled from its tree
(oracle/_ref/libzhao.so): the Zhao network's defineRxnKinetics and
defineAbioticRxnKinetics on random voxel states, with the 24-substrate layout
(speciation off) and the 95-substrate one (aqueous complexes summed into the
dissolved totals), every mask class, zero and negative entries, and states
where the per-step stability throttles bind.  Agreement to 1e-13 relative
(absolute 1e-300)."""
import ctypes
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PORT = os.path.join(ROOT, "oracle", "libratelaw_host.so")
REF = os.path.join(ROOT, "oracle", "_ref", "libzhao.so")


def _lib(path, names):
    if not os.path.exists(path):
        pytest.skip("%s not built" % os.path.relpath(path, ROOT))
    lib = ctypes.CDLL(path)
    for n in names:
        getattr(lib, n).restype = None
    return lib


@pytest.fixture(scope="module")
def libs():
    port = _lib(PORT, ["port_zhao_kinetics", "port_zhao_abiotic"])
    ref = _lib(REF, ["ref_zhao_kinetics", "ref_zhao_abiotic"])
    return port, ref


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def _states(n_sub, n, seed):
    rng = np.random.default_rng(seed)
    C = 10.0 ** rng.uniform(-9, -2, (n, n_sub))
    C[rng.random((n, n_sub)) < 0.05] = 0.0
    C[rng.random((n, n_sub)) < 0.02] *= -1e-3          # small negatives, floored by the laws
    B = 10.0 ** rng.uniform(-8, -3.5, (n, 12))        # around the 1e-4 attached carrying capacity
    B[rng.random((n, 12)) < 0.1] = 0.0
    # starve a few voxels so the throttles bind
    C[: n // 8, [0, 1, 4, 5, 6, 7, 8, 9]] *= 1e-6
    mask = rng.integers(0, 4, n)
    return C, B, mask


def _close(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.all(np.abs(a - b) <= 1e-13 * np.maximum(np.abs(b), 1e-300))


@pytest.mark.parametrize("n_sub", [24, 95])
def test_zhao_kinetics_matches_reference_header(libs, n_sub):
    port, ref = libs
    C, B, mask = _states(n_sub, 400, seed=n_sub)
    active = 0
    for v in range(C.shape[0]):
        c, b = np.ascontiguousarray(C[v]), np.ascontiguousarray(B[v])
        sp, bp = np.zeros(n_sub), np.zeros(12)
        sr, br = np.zeros(n_sub), np.zeros(12)
        port.port_zhao_kinetics(_ptr(b), 12, _ptr(c), n_sub, _ptr(sp), _ptr(bp), int(mask[v]))
        ref.ref_zhao_kinetics(_ptr(b), 12, _ptr(c), n_sub, _ptr(sr), _ptr(br), int(mask[v]))
        assert _close(sp, sr), (v, sp, sr)
        assert _close(bp, br), (v, bp, br)
        active += np.count_nonzero(sr) > 0
    # the law acts on the pore and biofilm voxels (mask >= 2), about half of them
    assert active > 150


@pytest.mark.parametrize("n_sub", [24, 95])
def test_zhao_abiotic_matches_reference_header(libs, n_sub):
    port, ref = libs
    C, _, mask = _states(n_sub, 400, seed=100 + n_sub)
    nonzero = 0
    for v in range(C.shape[0]):
        c = np.ascontiguousarray(C[v])
        sp, sr = np.zeros(n_sub), np.zeros(n_sub)
        port.port_zhao_abiotic(_ptr(c), n_sub, _ptr(sp), int(mask[v]))
        ref.ref_zhao_abiotic(_ptr(c), n_sub, _ptr(sr), int(mask[v]))
        assert _close(sp, sr), (v, sp, sr)
        nonzero += np.count_nonzero(sr) > 0
    assert nonzero > 300
