import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "complb3d-lattice-boltzmann-fba-surrogate-cobrapy-glpk_b200")
sys.path.insert(0, ROOT)


def load_pkg():
    """Import the product package (its directory name is not a Python identifier)."""
    if "complab_b200" in sys.modules:
        return sys.modules["complab_b200"]
    spec = importlib.util.spec_from_file_location("complab_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["complab_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_workloads():
    load_pkg()
    return importlib.import_module("complab_b200.workloads")


def reference_root():
    """The reference source tree, for the CPU tests that read its example
    inputs: $COMPLAB_REFERENCE, else the `reference_path` recorded in
    BASELINE.json at the repository root; None when neither names an existing
    directory (those tests then skip)."""
    cand = os.environ.get("COMPLAB_REFERENCE")
    if not cand:
        try:
            import json
            with open(os.path.join(ROOT, "BASELINE.json")) as f:
                cand = json.load(f).get("reference_path")
        except (OSError, ValueError):
            cand = None
    return cand if cand and os.path.isdir(cand) else None


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libcomplab_gpu.so")


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


@pytest.fixture(scope="session")
def wl():
    return load_workloads()


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as o
    o.lib()
    return o


@pytest.fixture(scope="session")
def gpu_lib(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test without a CUDA device")
    lib = pkg.load_library()
    pkg.check_abi(lib)
    return lib
