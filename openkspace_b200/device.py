"""Python host side over the C-ABI: a device context and device arrays.

Mirrors the reference's calling convention (synchronous, one caller per
context) while keeping data on the device between calls.  Every compute call
goes through ``libokscuda.so``; there is no CPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import OksError


class _SliceReq(ctypes.Structure):
    """okscuda_slice_req (include/okscuda.h)."""
    _fields_ = [("d_kspace", ctypes.c_void_p), ("h_mask", ctypes.c_void_p), ("nc", ctypes.c_int),
                ("ny", ctypes.c_int), ("nx", ctypes.c_int), ("iters", ctypes.c_int), ("lambda_", ctypes.c_float),
                ("d_rss", ctypes.c_void_p), ("d_coils", ctypes.c_void_p)]


class DeviceArray:
    """Owned device allocation with a numpy-like shape/dtype."""

    def __init__(self, ctx: "Context", shape, dtype, ptr: int | None = None, owned: bool = True):
        self.ctx = ctx
        self.shape = tuple(int(s) for s in shape)
        self.dtype = np.dtype(dtype)
        self.nbytes = int(np.prod(self.shape, dtype=np.int64)) * self.dtype.itemsize
        if ptr is None:
            p = ctypes.c_void_p()
            ctx.check(ctx.lib.okscuda_malloc(ctx.handle, self.nbytes, ctypes.byref(p)))
            ptr = p.value or 0
            owned = True
        self.ptr = int(ptr)
        self.owned = owned

    def __len__(self):
        return self.shape[0]

    @property
    def size(self):
        return int(np.prod(self.shape, dtype=np.int64))

    def view(self, offset_elems: int, shape) -> "DeviceArray":
        """Non-owning view starting ``offset_elems`` elements in."""
        return DeviceArray(self.ctx, shape, self.dtype, self.ptr + offset_elems * self.dtype.itemsize,
                           owned=False)

    def upload(self, host: np.ndarray) -> "DeviceArray":
        h = np.ascontiguousarray(host, dtype=self.dtype)
        if h.nbytes != self.nbytes:
            raise ValueError(f"upload size {h.nbytes} != {self.nbytes}")
        self.ctx.check(self.ctx.lib.okscuda_upload(self.ctx.handle, self.ptr, h.ctypes.data, h.nbytes))
        self.ctx.synchronize()   # pageable source: keep the host array alive until copied
        return self

    def to_host(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=self.dtype)
        self.ctx.check(self.ctx.lib.okscuda_download(self.ctx.handle, out.ctypes.data, self.ptr, out.nbytes))
        return out

    def free(self):
        if self.owned and self.ptr and self.ctx.handle:
            self.ctx.lib.okscuda_free(self.ctx.handle, self.ptr)
        self.ptr = 0

    def __del__(self):
        try:
            self.free()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


class Context:
    """One ``okscuda_ctx``: a device, a stream, cached FFT plans."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        rc = self.lib.okscuda_create(int(device), ctypes.byref(h))
        if rc != 0:
            raise OksError(rc, f"okscuda_create(device={device}) failed (no CUDA device?)")
        self.handle = h.value
        self.device = device

    def close(self):
        if self.handle:
            self.lib.okscuda_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- plumbing ---------------------------------------------------------
    def last_error(self) -> str:
        buf = ctypes.create_string_buffer(512)
        self.lib.okscuda_last_error(self.handle, buf, 512)
        return buf.value.decode(errors="replace")

    def check(self, rc: int):
        if rc != 0:
            raise OksError(rc, self.last_error())

    def synchronize(self):
        self.check(self.lib.okscuda_synchronize(self.handle))

    def set_stream(self, stream_handle: int | None):
        self.check(self.lib.okscuda_set_stream(self.handle, stream_handle or None))

    def empty(self, shape, dtype=np.complex64) -> DeviceArray:
        return DeviceArray(self, shape, dtype)

    def to_device(self, host: np.ndarray, dtype=None) -> DeviceArray:
        h = np.ascontiguousarray(host, dtype=dtype or host.dtype)
        return DeviceArray(self, h.shape, h.dtype).upload(h)

    def _dev(self, a, dtype=np.complex64) -> tuple[DeviceArray, bool]:
        if isinstance(a, DeviceArray):
            return a, False
        return self.to_device(np.asarray(a), dtype), True

    # -- primitives (reference routines) ----------------------------------
    def centred_fft2(self, x, inverse: bool = False) -> np.ndarray:
        """cs.rs:141-218 on [..., ny, nx] (host in, host out)."""
        h = np.ascontiguousarray(x, dtype=np.complex64)
        ny, nx = h.shape[-2:]
        d = self.to_device(h)
        self.check(self.lib.okscuda_centred_fft2(self.handle, d.ptr, h.size // (ny * nx), ny, nx, int(inverse)))
        return d.to_host()

    def dft_rows(self, x, inverse: bool = False, centred: bool = True, engine: int = 0,
                 in_place: bool = False) -> np.ndarray:
        """Unnormalised (centred) DFT along the last axis: the readout pass of
        cs.rs:141-178.  engine 0 = SIMT FFT, 1 = tcgen05 3xBF16 DFT-as-GEMM."""
        h = np.ascontiguousarray(x, dtype=np.complex64)
        n = h.shape[-1]
        d = self.to_device(h)
        o = d if in_place else self.empty(h.shape)
        self.check(self.lib.okscuda_dft_rows(self.handle, d.ptr, o.ptr, h.size // n, n, int(inverse), int(centred),
                                             int(engine)))
        return o.to_host()

    def tc_status(self) -> int:
        """Reads and clears the tensor-core kernels' bounded-wait error flag."""
        st = ctypes.c_int(0)
        self.check(self.lib.okscuda_tc_status(self.handle, ctypes.byref(st)))
        return st.value

    def haar_forward(self, x) -> np.ndarray:
        h = np.ascontiguousarray(x, dtype=np.complex64)
        ny, nx = h.shape[-2:]
        d = self.to_device(h)
        o = self.empty(h.shape)
        self.check(self.lib.okscuda_haar_forward(self.handle, d.ptr, o.ptr, h.size // (ny * nx), ny, nx))
        return o.to_host()

    def haar_inverse(self, x) -> np.ndarray:
        h = np.ascontiguousarray(x, dtype=np.complex64)
        ny, nx = h.shape[-2:]
        d = self.to_device(h)
        o = self.empty(h.shape)
        self.check(self.lib.okscuda_haar_inverse(self.handle, d.ptr, o.ptr, h.size // (ny * nx), ny, nx))
        return o.to_host()

    def soft_threshold_details(self, x, lam: float) -> np.ndarray:
        h = np.ascontiguousarray(x, dtype=np.complex64)
        ny, nx = h.shape[-2:]
        d = self.to_device(h)
        self.check(self.lib.okscuda_soft_threshold_details(self.handle, d.ptr, h.size // (ny * nx), ny, nx,
                                                           float(lam)))
        return d.to_host()

    def rss_crop(self, coils, crop=None) -> np.ndarray:
        d, _ = self._dev(coils)
        nc, ny, nx = d.shape
        ty, tx = crop if crop is not None else (ny, nx)
        o = self.empty((ty, tx), np.float32)
        self.check(self.lib.okscuda_rss_crop(self.handle, d.ptr, nc, ny, nx, ty, tx, o.ptr))
        return o.to_host()

    # -- FISTA-CS ---------------------------------------------------------
    def fista_cs(self, kspace_zf, mask, iters: int, lam: float, out: DeviceArray | None = None):
        """cs.rs:59-139 batched over leading axes of ``kspace_zf`` [..., ny, nx]
        (host array or DeviceArray).  Returns a host array unless ``out`` is
        given (then ``out`` is filled and returned)."""
        d, _ = self._dev(kspace_zf)
        ny, nx = d.shape[-2:]
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        if m.shape != (ny, nx):
            raise OksError(_lib.OKS_ESHAPE,
                           f"CS: mask shape {m.shape} does not match kspace shape {(ny, nx)}")
        batch = d.size // (ny * nx)
        o = out if out is not None else self.empty(d.shape)
        self.check(self.lib.okscuda_fista_cs(self.handle, d.ptr, m.ctypes.data, batch, ny, nx, int(iters),
                                             float(lam), o.ptr))
        return o if out is not None else o.to_host()

    def fista_cs_single_coil(self, kspace_zf, mask, iters: int, lam: float) -> np.ndarray:
        """Same signature and meaning as the reference (cs.rs:59)."""
        return self.fista_cs(kspace_zf, mask, iters, lam)

    def cs_volume(self, kspace, mask, iters: int, lam: float, crop=None, out: DeviceArray | None = None,
                  coils: DeviceArray | None = None):
        """strategy.rs:849-885 for placed k-space [nc, nz, ny, nx] with masks
        [nz, ny, nx]; one batched launch for every (coil, slice).  Returns the
        RSS volume [nz, ty, tx] (host) unless ``out`` is given."""
        d, _ = self._dev(kspace)
        nc, nz, ny, nx = d.shape
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        if m.shape != (nz, ny, nx):
            raise OksError(_lib.OKS_ESHAPE, f"mask shape {m.shape} != {(nz, ny, nx)}")
        ty, tx = crop if crop is not None else (ny, nx)
        o = out if out is not None else self.empty((nz, ty, tx), np.float32)
        self.check(self.lib.okscuda_cs_volume(self.handle, d.ptr, m.ctypes.data, nc, nz, ny, nx, int(iters),
                                              float(lam), ty, tx, o.ptr, coils.ptr if coils else None))
        return o if out is not None else o.to_host()

    def cs_batch(self, slices, outs=None):
        """okscuda_cs_batch over ``slices`` = [(kspace [nc,ny,nx], mask [ny,nx],
        iters, lambda), ...] (kspace host array or DeviceArray).  Returns the
        RSS images (host) or fills the DeviceArrays in ``outs``."""
        keep = []
        arr = (_SliceReq * max(len(slices), 1))()
        for i, (k, m, iters, lam) in enumerate(slices):
            d, _ = self._dev(k)
            nc, ny, nx = d.shape
            mm = np.ascontiguousarray(m, dtype=np.uint8)
            if mm.shape != (ny, nx):
                raise OksError(_lib.OKS_ESHAPE, f"mask shape {mm.shape} != {(ny, nx)}")
            o = outs[i] if outs is not None else self.empty((ny, nx), np.float32)
            keep += [d, mm, o]
            arr[i] = _SliceReq(d.ptr, mm.ctypes.data, nc, ny, nx, int(iters), float(lam), o.ptr, None)
        self.check(self.lib.okscuda_cs_batch(self.handle, arr, len(slices)))
        if outs is not None:
            return outs
        return [keep[3 * i + 2].to_host() for i in range(len(slices))]

    def sense_cs(self, kspace, mask, iters: int, lam: float, walsh_window: int = 3, walsh_iters: int = 6,
                 power_iters: int = 30):
        """okscuda_sense_cs on one slice: returns (|x|, x, maps, L) on the host."""
        d, _ = self._dev(kspace)
        nc, ny, nx = d.shape
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        if m.shape != (ny, nx):
            raise OksError(_lib.OKS_ESHAPE, f"mask shape {m.shape} != {(ny, nx)}")
        mag = self.empty((ny, nx), np.float32)
        x = self.empty((ny, nx))
        maps = self.empty((nc, ny, nx))
        L = ctypes.c_double()
        self.check(self.lib.okscuda_sense_cs(self.handle, d.ptr, m.ctypes.data, nc, ny, nx, int(iters), float(lam),
                                             int(walsh_window), int(walsh_iters), int(power_iters), mag.ptr, maps.ptr,
                                             x.ptr, ctypes.byref(L)))
        return mag.to_host(), x.to_host(), maps.to_host(), L.value

    def sense_unfold(self, aliased, maps, r: int, ridge: float, gfactor: bool = False):
        """okscuda_sense_unfold (sense.rs:64-252): (unfolded [ny, nx] complex64,
        g-factor [ny, nx] float32 or None) on the host."""
        a, _ = self._dev(aliased)
        m, _ = self._dev(maps)
        nc, ny, nx = a.shape
        out = self.empty((ny, nx))
        g = self.empty((ny, nx), np.float32) if gfactor else None
        self.check(self.lib.okscuda_sense_unfold(self.handle, a.ptr, m.ptr, nc, ny, nx, int(r), float(ridge), out.ptr,
                                                 g.ptr if g is not None else None))
        return out.to_host(), (g.to_host() if g is not None else None)

    def set_option(self, name: str, value: int):
        self.check(self.lib.okscuda_set_option(self.handle, name.encode(), int(value)))

    def autotune(self, kind: int, ny: int, nx: int, nc: int = 8, iters: int = 20) -> dict:
        """Times the engine's plan/launch-shape candidates for one shape and
        keeps the fastest (kind 0: ky-only masks, 1: 2-D masks); returns the
        report (every candidate's time and the choice)."""
        import json
        buf = ctypes.create_string_buffer(1 << 16)
        self.check(self.lib.okscuda_autotune(self.handle, int(kind), int(ny), int(nx), int(nc), int(iters), buf,
                                             len(buf)))
        return json.loads(buf.value.decode())

    def autotune_table(self) -> str:
        buf = ctypes.create_string_buffer(1 << 16)
        self.check(self.lib.okscuda_autotune_table(self.handle, buf, len(buf)))
        return buf.value.decode()

    def autotune_load(self, text: str):
        self.check(self.lib.okscuda_autotune_load(self.handle, text.encode()))

    # -- profiling ----------------------------------------------------------
    def profile(self, on: bool = True):
        self.check(self.lib.okscuda_profile_enable(self.handle, int(on)))

    def profile_read(self) -> dict:
        """{kernel name: (total device ms, launches)} since profile(True)."""
        n = 64
        names = ctypes.create_string_buffer(64 * n)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_longlong * n)()
        found = ctypes.c_int()
        self.check(self.lib.okscuda_profile_read(self.handle, names, 64, ms, cnt, n, ctypes.byref(found)))
        out = {}
        for k in range(min(found.value, n)):
            nm = names.raw[64 * k:64 * (k + 1)].split(b"\0", 1)[0].decode()
            out[nm] = (ms[k], cnt[k])
        return out

    def cs_slice(self, kspace, mask, iters: int, lam: float, return_coils: bool = False):
        """strategy.rs:850-880 for one slice: kspace [nc, ny, nx], mask [ny, nx]."""
        d, _ = self._dev(kspace)
        nc, ny, nx = d.shape
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        if m.shape != (ny, nx):
            raise OksError(_lib.OKS_ESHAPE, f"mask shape {m.shape} != {(ny, nx)}")
        rss = self.empty((ny, nx), np.float32)
        coils = self.empty((nc, ny, nx)) if return_coils else None
        self.check(self.lib.okscuda_cs_slice(self.handle, d.ptr, m.ctypes.data, nc, ny, nx, int(iters),
                                             float(lam), rss.ptr, coils.ptr if coils else None))
        r = rss.to_host()
        return (r, coils.to_host()) if return_coils else r
