"""The C-ABI library builds, loads and exports every symbol include/okscuda.h
declares (no compute calls: this runs without a GPU)."""
import ctypes
import os

from openkspace_b200 import _lib


def test_header_symbols_all_exported():
    L = _lib.load()
    declared = _lib.header_symbols()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), f"{name} declared in include/okscuda.h but not exported"
    assert set(declared) == set(_lib.SIGNATURES), "ctypes signatures out of sync with the header"


def test_library_is_sm100a_build():
    L = _lib.load()
    assert b"sm_100a" in L.okscuda_version()
    assert os.path.getsize(_lib.LIB_PATH) > 0


def test_create_without_device_fails_cleanly():
    try:
        import torch
        if torch.cuda.is_available():
            return
    except Exception:  # noqa: BLE001
        pass
    L = _lib.load()
    h = ctypes.c_void_p()
    rc = L.okscuda_create(0, ctypes.byref(h))
    assert rc != 0 and not h.value


def test_null_context_is_einval():
    L = _lib.load()
    assert L.okscuda_synchronize(None) == _lib.OKS_EINVAL
    assert L.okscuda_fista_cs(None, None, None, 1, 8, 8, 1, 0.01, None) == _lib.OKS_EINVAL


def test_acquisition_structs_match_the_python_mirror():
    """okscuda_acq_header / okscuda_acq_set as laid out by the compiler equal
    the numpy dtype and ctypes struct the Python host side passes."""
    from openkspace_b200.strategy import HEADER_DTYPE, _AcqSet
    L = _lib.load()
    assert L.okscuda_acq_header_size() == HEADER_DTYPE.itemsize == 40
    assert L.okscuda_acq_set_size() == ctypes.sizeof(_AcqSet)
