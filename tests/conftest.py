import glob
import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "exafmm-beta_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the CUDA path")


def load_package():
    """Import exafmm-beta_b200/ (its directory name is not a Python identifier)."""
    if "exafmm_b200" in sys.modules:
        return sys.modules["exafmm_b200"]
    spec = importlib.util.spec_from_file_location("exafmm_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["exafmm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def ex():
    mod = load_package()
    mod.build()
    return mod


@pytest.fixture(scope="session")
def datasets():
    load_package()
    import exafmm_b200.datasets as d
    return d


@pytest.fixture(scope="session")
def oracle():
    from bindings import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from bindings import Reference, reference_available
    if not reference_available():
        pytest.skip("oracle/_ref was not built here (needs the reference tree)")
    return Reference()


def golden_cases():
    """Free-space solve fixtures (periodic ones, the operator chain, the record formats and
    the MD ABI are separate)."""
    other = ("kernel_kat.npz", "records.npz", "md_gromacs.npz", "md_distributed.npz", "datasets_reference.npz")
    return sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if os.path.basename(p) not in other
                  and not os.path.basename(p).startswith(("periodic_", "inej_", "large_")))


def periodic_golden_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "periodic_*.npz")))


def inej_golden_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "inej_*.npz")))


def load_golden(path):
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def pair_set(p):
    return set(map(tuple, np.asarray(p)[:, :2].tolist()))


def rel_l2(a, b):
    num = float(np.sum((np.asarray(a) - np.asarray(b)) ** 2))
    den = float(np.sum(np.asarray(b) ** 2))
    return float(np.sqrt(num / den)) if den > 0 else float(np.sqrt(num))
