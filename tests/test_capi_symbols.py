"""CPU-only checks of the drop-in boundary: the library loads and exports what the header declares."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER_DIR = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for fn in sorted(os.listdir(HEADER_DIR)):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(HEADER_DIR, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(mhd_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from magnetohydrodynamics_simulator_b200 import capi

    if not os.path.exists(capi.LIB_PATH):
        import __graft_entry__

        __graft_entry__.build()
    return ctypes.CDLL(capi.LIB_PATH)


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ("mhd_create", "mhd_step", "mhd_run", "mhd_cfl_dt", "mhd_divb", "mhd_destroy",
                     "mhd_set_state", "mhd_get_state", "mhd_set_implicit_coefficient"):
        assert required in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings(lib):
    lib.mhd_status_string.restype = ctypes.c_char_p
    for s in range(9):
        assert lib.mhd_status_string(s)


def test_no_device_is_reported_not_faked():
    """Without a GPU the product refuses to run instead of falling back to the CPU."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from magnetohydrodynamics_simulator_b200 import Context, MHDError

    with pytest.raises(MHDError) as e:
        Context(16, 16, 0.1, 0.1, 1e-3)
    assert e.value.status == 6  # MHD_ERR_NO_DEVICE


def test_invalid_parameters_rejected(lib):
    from magnetohydrodynamics_simulator_b200 import capi

    lib = capi.load_library()
    p = capi.Params()
    lib.mhd_default_params(ctypes.byref(p), 1, 16, 0.1, 0.1, 1e-3)
    h = ctypes.c_void_p()
    assert lib.mhd_create(ctypes.byref(p), None, ctypes.byref(h)) == 1  # nx < 2
    lib.mhd_default_params(ctypes.byref(p), 16, 16, -0.1, 0.1, 1e-3)
    assert lib.mhd_create(ctypes.byref(p), None, ctypes.byref(h)) == 1  # dx <= 0
    lib.mhd_default_params(ctypes.byref(p), 16, 16, 0.1, 0.1, -1.0)
    assert lib.mhd_create(ctypes.byref(p), None, ctypes.byref(h)) == 1  # eta < 0


def test_batch_invalid_parameters_rejected(lib):
    from magnetohydrodynamics_simulator_b200 import capi

    lib = capi.load_library()
    arr = (capi.Params * 3)()
    for k in range(3):
        lib.mhd_default_params(ctypes.byref(arr[k]), 16 + k, 16, 0.1, 0.1, 1e-3)
    h = ctypes.c_void_p()
    assert lib.mhd_batch_create(arr, 0, None, ctypes.byref(h)) == 1  # empty batch
    arr[1].nx = 1
    assert lib.mhd_batch_create(arr, 3, None, ctypes.byref(h)) == 1  # one bad instance
    arr[1].nx = 17
    arr[2].ct_mode = 5
    assert lib.mhd_batch_create(arr, 3, None, ctypes.byref(h)) == 1
    assert lib.mhd_batch_step(None, None) == 1
    assert lib.mhd_batch_count(None) == 0


def test_batch_without_device_is_reported_not_faked():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from magnetohydrodynamics_simulator_b200 import Batch, MHDError

    with pytest.raises(MHDError) as e:
        Batch([dict(nx=16, ny=16, dx=0.1, dy=0.1, eta=1e-3)])
    assert e.value.status == 6
