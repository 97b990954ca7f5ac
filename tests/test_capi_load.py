"""The C-ABI library loads without a GPU and exports every entry point the
public header declares, with struct layouts matching the Python binding."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "complab_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cl_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "cl_create" in syms and "cl_step" in syms and "cl_eq_solve_device" in syms
    assert len(syms) >= 30


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg.load_library()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_abi_struct_sizes(pkg):
    pkg.check_abi()


def test_error_paths_without_gpu(pkg):
    """Argument validation runs before any CUDA call: bad configs are refused
    with an error code and a message, never a crash."""
    import ctypes
    lib = pkg.load_library()
    cfg = pkg.make_config(2, 4, 4)          # nx < 3 is invalid
    st = ctypes.c_int(0)
    h = lib.cl_create(ctypes.byref(cfg), None, ctypes.byref(st))
    assert not h and st.value == pkg.ERR_ARG
    assert b"nx" in lib.cl_last_error()
    cfg = pkg.make_config(8, 4, 4, tau_ns=0.5)
    h = lib.cl_create(ctypes.byref(cfg), None, ctypes.byref(st))
    assert not h and st.value == pkg.ERR_ARG


def test_microbe_carrier_validation_without_gpu(pkg):
    """A microbe carried by a solute must name a mobile solute and run the
    rate table: refused otherwise, before any CUDA call."""
    import ctypes
    lib = pkg.load_library()
    st = ctypes.c_int(0)
    sol = [{"c0": 0.1}, {"immobile": True}]
    cfg = pkg.make_config(8, 4, 4, solutes=sol, microbes=1)
    cfg.microbe_carrier[0] = 2                     # solute 1 is immobile
    assert not lib.cl_create(ctypes.byref(cfg), None, ctypes.byref(st)) and st.value == pkg.ERR_ARG
    assert b"microbe_carrier" in lib.cl_last_error()
    cfg.microbe_carrier[0] = 5                     # no such solute
    assert not lib.cl_create(ctypes.byref(cfg), None, ctypes.byref(st)) and st.value == pkg.ERR_ARG
    cfg = pkg.make_config(8, 4, 4, solutes=sol, microbes=1)
    cfg.microbe_carrier[0] = 1
    cfg.rate_law = pkg.RATELAW_ZHAO                # compiled rate laws read sessile biomass
    assert not lib.cl_create(ctypes.byref(cfg), None, ctypes.byref(st)) and st.value == pkg.ERR_ARG
