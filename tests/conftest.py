import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100)")


def _has_gpu() -> bool:
    try:
        r = subprocess.run(["nvidia-smi", "-L"], capture_output=True, text=True, timeout=20)
        return r.returncode == 0 and "GPU" in r.stdout
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device on this machine")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build(ref=False)
    return O


@pytest.fixture(scope="session")
def ref(oracle):
    """The reference's own host code (oracle/_ref), when it can be built."""
    if not oracle.ref_available():
        if os.path.isdir(oracle.ref_root()):
            oracle.build(ref=True)
    if not oracle.ref_available():
        pytest.skip("reference sources not present and oracle/_ref not built")
    return oracle


@pytest.fixture(scope="session")
def bvlib():
    import blockvecchia_b200 as bv
    bv.lib()
    return bv


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.fixture(scope="session")
def golden_layout():
    g = golden("layout_2000_150_60.npz")
    return {k: g[k] for k in g.files}
