import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a); run with -m gpu")


def _has_gpu() -> bool:
    try:
        import ctypes
        rt = ctypes.CDLL("libcudart.so.12")
        n = ctypes.c_int(0)
        return rt.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0
    except OSError:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    # GPU tests are selected with -m gpu; they fail (never skip silently) without a GPU.
    pass


@pytest.fixture(scope="session")
def lib():
    import openntc_b200
    return openntc_b200.load()


@pytest.fixture(scope="session")
def oracle():
    from oracle.bindings import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref_rt():
    from oracle.bindings import RefRuntime, REF_RT_SO
    if not REF_RT_SO.exists():
        pytest.skip(f"{REF_RT_SO} not built (make -C oracle ref needs the upstream sources)")
    return RefRuntime()


@pytest.fixture(scope="session")
def materials(tmp_path_factory):
    """Cache of synthetic material sets keyed by (dim, seed, channels)."""
    from openntc_b200.synth import make_material
    base = tmp_path_factory.mktemp("materials")
    cache = {}

    def get(dim, seed, channels=9):
        key = (dim, seed, channels)
        if key not in cache:
            cache[key] = make_material(base / f"m{dim}_{seed}_{channels}", dim, seed, channels)
        return cache[key]

    return get
