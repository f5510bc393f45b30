"""ctypes binding of ``libokscuda.so`` (the C-ABI of ``include/okscuda.h``).

The library is required: importing the compute entry points without it, or
calling them on a machine without a CUDA device, raises -- there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libokscuda.so")
# the bounds-checked build of the same sources (tests select it through
# OKSCUDA_LIB=bounds in a child process)
BOUNDS_LIB_PATH = os.path.join(HERE, "libokscuda_bounds.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "okscuda.h")

OKS_OK = 0
OKS_EINVAL = -1
OKS_ESHAPE = -2
OKS_EODD = -3
OKS_ENOTPD = -4
OKS_ECUDA = -5
OKS_ENOMEM = -6
OKS_EAGAIN = -7
OKS_ETIMEDOUT = -8
OKS_ENOTSUP = -9
OKS_ESKIP = -10

_c = ctypes
_vp = _c.c_void_p
_i = _c.c_int
_f = _c.c_float
_sz = _c.c_size_t

# name -> (restype, argtypes); every symbol include/okscuda.h declares
SIGNATURES = {
    "okscuda_create": (_i, [_i, _c.POINTER(_vp)]),
    "okscuda_destroy": (None, [_vp]),
    "okscuda_last_error": (_i, [_vp, _c.c_char_p, _sz]),
    "okscuda_set_stream": (_i, [_vp, _vp]),
    "okscuda_get_stream": (_vp, [_vp]),
    "okscuda_synchronize": (_i, [_vp]),
    "okscuda_version": (_c.c_char_p, []),
    "okscuda_set_option": (_i, [_vp, _c.c_char_p, _c.c_longlong]),
    "okscuda_autotune": (_i, [_vp, _i, _i, _i, _i, _i, _c.c_char_p, _sz]),
    "okscuda_autotune_table": (_i, [_vp, _c.c_char_p, _sz]),
    "okscuda_autotune_load": (_i, [_vp, _c.c_char_p]),
    "okscuda_malloc": (_i, [_vp, _sz, _c.POINTER(_vp)]),
    "okscuda_free": (_i, [_vp, _vp]),
    "okscuda_upload": (_i, [_vp, _vp, _vp, _sz]),
    "okscuda_download": (_i, [_vp, _vp, _vp, _sz]),
    "okscuda_host_alloc": (_i, [_vp, _sz, _c.POINTER(_vp)]),
    "okscuda_host_free": (_i, [_vp, _vp]),
    "okscuda_centred_fft2": (_i, [_vp, _vp, _i, _i, _i, _i]),
    "okscuda_dft_rows": (_i, [_vp, _vp, _vp, _c.c_longlong, _i, _i, _i, _i]),
    "okscuda_tc_status": (_i, [_vp, _c.POINTER(_i)]),
    "okscuda_debug_bounds": (_i, [_vp, _c.POINTER(_c.c_uint), _i]),
    "okscuda_haar_forward": (_i, [_vp, _vp, _vp, _i, _i, _i]),
    "okscuda_haar_inverse": (_i, [_vp, _vp, _vp, _i, _i, _i]),
    "okscuda_soft_threshold_details": (_i, [_vp, _vp, _i, _i, _i, _f]),
    "okscuda_rss_crop": (_i, [_vp, _vp, _i, _i, _i, _i, _i, _vp]),
    "okscuda_fista_cs": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _f, _vp]),
    "okscuda_cs_slice": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _f, _vp, _vp]),
    "okscuda_cs_volume": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _f, _i, _i, _vp, _vp]),
    "okscuda_cs_slice_noalloc": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _f, _vp]),
    "okscuda_cs_batch": (_i, [_vp, _vp, _i]),
    "okscuda_sense_cs": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _f, _i, _i, _i, _vp, _vp, _vp,
                              _c.POINTER(_c.c_double)]),
    "okscuda_raw_open": (_i, [_c.c_char_p, _c.POINTER(_vp)]),
    "okscuda_raw_acq_set": (_i, [_vp, _vp]),
    "okscuda_raw_info": (_i, [_vp, _c.POINTER(_i), _c.POINTER(_i)]),
    "okscuda_raw_close": (None, [_vp]),
    "okscuda_sense_unfold": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _f, _vp, _vp]),
    "okscuda_percentile": (_i, [_vp, _vp, _c.c_longlong, _f, _c.POINTER(_f)]),
    "okscuda_window_u8": (_i, [_vp, _vp, _c.c_longlong, _f, _f, _i, _vp]),
    "okscuda_write_nifti": (_i, [_vp, _i, _i, _i, _c.c_char_p]),
    "okscuda_write_png": (_i, [_vp, _i, _i, _c.c_char_p]),
    "okscuda_server_create": (_i, [_vp, _vp, _c.POINTER(_vp)]),
    "okscuda_server_destroy": (None, [_vp]),
    "okscuda_server_submit": (_i, [_vp, _vp, _c.POINTER(_c.c_uint64)]),
    "okscuda_server_poll": (_i, [_vp, _c.c_uint64, _c.POINTER(_i)]),
    "okscuda_server_wait": (_i, [_vp, _c.c_uint64, _i]),
    "okscuda_server_stats": (_i, [_vp, _c.POINTER(_c.c_longlong), _c.POINTER(_c.c_longlong),
                                  _c.POINTER(_sz)]),
    "okscuda_prewhiten_fit": (_i, [_vp, _vp, _i, _c.c_longlong, _c.c_longlong, _vp]),
    "okscuda_prewhiten_apply": (_i, [_vp, _vp, _vp, _c.c_longlong, _i, _i]),
    "okscuda_os_remove": (_i, [_vp, _vp, _vp, _c.c_longlong, _i, _i]),
    "okscuda_ifft1_kz": (_i, [_vp, _vp, _i, _i, _i, _i]),
    "okscuda_ifft2": (_i, [_vp, _vp, _c.c_longlong, _i, _i]),
    "okscuda_csrss_default": (None, [_vp]),
    "okscuda_csrss_name": (_c.c_char_p, []),
    "okscuda_acq_header_size": (_c.c_size_t, []),
    "okscuda_acq_set_size": (_c.c_size_t, []),
    "okscuda_csrss_reconstruct": (_i, [_vp, _vp, _vp, _vp, _c.c_longlong, _c.POINTER(_i)]),
    "okscuda_profile_enable": (_i, [_vp, _i]),
    "okscuda_profile_read": (_i, [_vp, _c.c_char_p, _i, _c.POINTER(_c.c_double),
                                  _c.POINTER(_c.c_longlong), _i, _c.POINTER(_i)]),
}

_lib = None


class OksError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def header_symbols() -> list[str]:
    """Function names declared in include/okscuda.h."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(okscuda_[a-z0-9_]+)\s*\(", txt)))


def load(build_if_missing: bool = True):
    """Load the library (building it in-tree when sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    if os.environ.get("OKSCUDA_LIB") == "bounds":
        if not os.path.exists(BOUNDS_LIB_PATH):
            raise OSError(f"{BOUNDS_LIB_PATH} is missing: build it with `python -m openkspace_b200.build`")
        L = ctypes.CDLL(BOUNDS_LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
        return L
    if build_if_missing:
        from . import build as _b
        if _b.needs_build():
            try:
                _b.build()
            except Exception:  # noqa: BLE001 - a prebuilt library may still be loadable
                if not os.path.exists(LIB_PATH):
                    raise
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing: build it with `python -m openkspace_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L
