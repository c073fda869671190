"""CPU checks of the C ABI: the library loads, exports every function the
headers declare, and rejects bad arguments before touching a GPU."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import rs_illume_b200 as rb
from rs_illume_b200 import _lib
from tests.conftest import ROOT, has_gpu

DECL = re.compile(r"^\s*(?:const\s+)?(?:int32_t|void|char|const char|float|uint32_t)\s*\*?\s*(ilm_\w+)\s*\(", re.M)


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        names.update(DECL.findall(open(h).read()))
    return sorted(names)


def test_headers_declare_functions():
    names = declared_functions()
    assert "ilm_intersect_closest" in names and "ilm_accel_build" in names and "ilm_wl_ball_rays" in names
    assert len(names) >= 25


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding covers them
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_oracle_library_loads():
    import oracle
    lib = oracle.load()
    assert lib.orc_gamma(3) > 0


def test_null_arguments_rejected_without_gpu():
    lib = _lib.load()
    assert lib.ilm_context_create(None, None) == _lib.ILM_ERR_INVALID_ARGUMENT
    assert lib.ilm_context_destroy(None) == _lib.ILM_ERR_INVALID_ARGUMENT
    assert lib.ilm_intersect_closest(None, 1, None, 10, None, None) == _lib.ILM_ERR_INVALID_ARGUMENT
    assert lib.ilm_intersect_any(None, 1, None, 10, None, None) == _lib.ILM_ERR_INVALID_ARGUMENT
    assert lib.ilm_mesh_upload(None, None, 0, None, 0, None) == _lib.ILM_ERR_INVALID_ARGUMENT
    assert lib.ilm_accel_build(None, None, 0, None, None) == _lib.ILM_ERR_INVALID_ARGUMENT
    assert lib.ilm_device_errors(None, None, 0) == _lib.ILM_ERR_INVALID_ARGUMENT
    assert lib.ilm_synchronize(None, None, 1.0) == _lib.ILM_ERR_INVALID_ARGUMENT
    assert lib.ilm_last_error_string(None) == b"no context"
    assert lib.ilm_host_layout_destroy(None) == _lib.ILM_ERR_INVALID_ARGUMENT


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_context_without_device_fails_loudly():
    h = ctypes.c_void_p()
    assert _lib.load().ilm_context_create(ctypes.byref(h), None) == _lib.ILM_ERR_NO_DEVICE
    with pytest.raises(rb.IllumeError) as e:
        rb.Context(0)
    assert "ILM_ERR_NO_DEVICE" in str(e.value)


def test_record_layouts():
    assert _lib.RAY_DTYPE.itemsize == 32 and _lib.HIT_DTYPE.itemsize == 16
    assert ctypes.sizeof(_lib.ilm_sphere_desc) == 184   # sphere fields + kind, height, inner radius, p1, p2
    assert ctypes.sizeof(_lib.ilm_config) == 20
    r = rb.rays_array([rb.Ray((1, 2, 3), (0, 0, 1), 5.0)])
    assert r["o"][0].tolist() == [1, 2, 3] and r["tmax"][0] == 5.0
    assert np.isinf(rb.rays_array([rb.Ray((0, 0, 0), (1, 0, 0))])["tmax"][0])
