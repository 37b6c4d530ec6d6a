import ctypes
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_goldens.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def _cuda_device_count() -> int:
    try:
        cudart = ctypes.CDLL("libcudart.so")
    except OSError:
        try:
            cudart = ctypes.CDLL("/usr/local/cuda/lib64/libcudart.so")
        except OSError:
            return 0
    n = ctypes.c_int(0)
    if cudart.cudaGetDeviceCount(ctypes.byref(n)) != 0:
        return 0
    return n.value


HAVE_GPU = _cuda_device_count() > 0


def pytest_collection_modifyitems(config, items):
    if HAVE_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the native library and the oracle once per session (incremental)."""
    from dpmmsubclusters_gpu_b200 import build as b
    b.build()
    from oracle import oracle as O
    O.build()
    yield


@pytest.fixture(scope="session")
def goldens():
    with open(GOLDEN) as f:
        return json.load(f)["tests"]


def inits(rec):
    """name -> values of the comma initialisers of one golden test (repeated names -> list)."""
    out = {}
    for i in rec["inits"]:
        out.setdefault(i["name"], []).append(np.array(i["values"]))
    return out


def eigen(values, rows, cols):
    """Eigen's comma initialiser fills row by row."""
    return np.asarray(values, dtype=np.float64).reshape(rows, cols)


def uniforms(n, seed):
    """float32 uniforms in (0, 1], the range of curand_uniform."""
    rng = np.random.default_rng(seed)
    return ((rng.integers(0, 1 << 24, size=n) + 1) / float(1 << 24)).astype(np.float32)
