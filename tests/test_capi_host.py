"""CPU-side checks of the C ABI: the library loads and exports every declared entry point,
status handling, and the host-side parsing done before any device work."""
import ctypes
import json
import os
import re

import numpy as np
import pytest

from conftest import HAVE_GPU, ROOT
from dpmmsubclusters_gpu_b200 import capi

HEADER = os.path.join(ROOT, "include", "dpmm_capi.h")


def _declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dpmm_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported():
    names = _declared()
    assert len(names) >= 40
    L = ctypes.CDLL(capi.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_bindings_cover_header():
    assert sorted(capi.SIGNATURES) == _declared()


def test_status_strings_and_version():
    L = capi.lib()
    assert L.dpmm_capi_version() == 1
    for s in range(10):
        assert L.dpmm_status_string(s)
    assert L.dpmm_status_string(0) == b"ok"


def test_create_validates_arguments():
    L = capi.lib()
    d = capi.dpmm_desc()
    h = ctypes.c_void_p()
    d.n_points, d.dim, d.prior_type = 0, 2, 0
    assert L.dpmm_create(ctypes.byref(d), ctypes.byref(h)) == 1      # invalid N
    d.n_points, d.dim = 10, 500
    assert L.dpmm_create(ctypes.byref(d), ctypes.byref(h)) == 1      # Gaussian D > 128
    d.dim, d.prior_type = 2, 7
    assert L.dpmm_create(ctypes.byref(d), ctypes.byref(h)) == 1      # unknown prior
    assert not h.value


def test_matrix_helpers_validate_arguments():
    # checked before any device call: no context, a size outside 1 .. 2048, null arrays
    L = capi.lib()
    a = np.eye(3)
    P = ctypes.POINTER(ctypes.c_double)
    pa = a.ctypes.data_as(P)
    assert L.dpmm_inverse_matrix(None, 3, pa, pa) == 1
    assert L.dpmm_multiply_for_inverse_wishart(None, 3, 3, 3, pa, pa, pa) == 1
    assert L.dpmm_inverse_matrix(None, 0, pa, pa) == 1
    assert L.dpmm_inverse_matrix(None, 4096, None, None) == 1


@pytest.mark.skipif(HAVE_GPU, reason="checks the no-device path")
def test_no_device_status():
    L = capi.lib()
    d = capi.dpmm_desc()
    d.n_points, d.dim = 10, 2
    h = ctypes.c_void_p()
    assert L.dpmm_create(ctypes.byref(d), ctypes.byref(h)) == 9      # DPMM_ERR_NO_DEVICE
    assert b"device" in L.dpmm_last_error()


def test_params_json_errors_reported_before_device(tmp_path):
    npy = tmp_path / "x.npy"
    np.save(npy, np.random.default_rng(0).normal(size=(50, 2)))
    bad = tmp_path / "bad.json"
    bad.write_text('{"alpha": 10.0, "hyper_params": {"k": 1 "v": 5}}')
    L = capi.lib()
    h = ctypes.c_void_p()
    st = L.dpmm_dp_parallel_from_file(str(npy).encode(), str(bad).encode(), 0, None, ctypes.byref(h))
    assert st == 8 and b"JSON" in L.dpmm_last_error()
    st = L.dpmm_dp_parallel_from_file(b"/nonexistent.npy", str(bad).encode(), 0, None, ctypes.byref(h))
    assert st == 8
    # a JSON with // comments (as the reference's fixtures use) parses; without a device the run
    # then stops at device creation
    good = tmp_path / "good.json"
    good.write_text('{\n  // Example for niw\n  "iterations": 3,\n  "hyper_params": {"m": [0.0, 0.0], '
                    '"psi": [[1.0, 0.0], [0.0, 1.0]], "k": 1, "v": 5.0},\n  "outlier_mod": 0\n}\n')
    st = L.dpmm_dp_parallel_from_file(str(npy).encode(), str(good).encode(), 0, None, ctypes.byref(h))
    if HAVE_GPU:
        assert st == 0
        L.dpmm_model_info_free(h)
    else:
        assert st == 9


def test_npy_dtype_rejected_cleanly(tmp_path):
    npy = tmp_path / "c.npy"
    np.save(npy, np.zeros((4, 2), dtype=np.complex64))
    good = tmp_path / "p.json"
    good.write_text("{}")
    L = capi.lib()
    h = ctypes.c_void_p()
    assert L.dpmm_dp_parallel_from_file(str(npy).encode(), str(good).encode(), 0, None, ctypes.byref(h)) == 8


def test_python_api_layout_checks():
    from dpmmsubclusters_gpu_b200 import dp_parallel_sampling_class, niw_hyperparams, prior_type
    with pytest.raises(ValueError):
        dp_parallel_sampling_class(10, np.zeros((2, 9)), 1, prior_type.Gaussian)   # D x N expected
    h = niw_hyperparams(1.0, [0, 0], 5.0, np.eye(2))
    assert h.psi.shape == (2, 2) and h.clone().k == 1.0


def test_golden_fixture_regenerates(tmp_path):
    """The committed golden fixture is what make_golden.py extracts from the reference's tests."""
    from oracle.oracle import reference_dir
    ref = reference_dir()
    if ref is None:
        pytest.skip("reference sources not mounted")
    import subprocess
    import sys
    out = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "golden", "make_golden.py"), ref],
                         capture_output=True, text=True, cwd=tmp_path)
    assert out.returncode == 0, out.stderr
    with open(os.path.join(ROOT, "tests", "golden", "reference_goldens.json")) as f:
        assert json.load(f)["tests"]
