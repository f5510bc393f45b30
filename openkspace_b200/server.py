"""Python side of the request server (okscuda_server_*): continuous batching of
per-slice FISTA-CS requests on one device, admission by an HBM budget."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import OksError


class _Cfg(ctypes.Structure):
    """okscuda_server_cfg (include/okscuda.h)."""
    _fields_ = [("max_inflight", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_size_t), ("n_streams", ctypes.c_int),
                ("mode", ctypes.c_int)]


class _Req(ctypes.Structure):
    """okscuda_request (include/okscuda.h)."""
    _fields_ = [("h_kspace", ctypes.c_void_p), ("d_kspace", ctypes.c_void_p), ("h_mask", ctypes.c_void_p),
                ("nc", ctypes.c_int), ("ny", ctypes.c_int), ("nx", ctypes.c_int), ("iters", ctypes.c_int),
                ("lambda_", ctypes.c_float), ("h_rss", ctypes.c_void_p), ("coil_stride", ctypes.c_longlong)]


class Server:
    """okscuda_server_*: ``mode`` 0 (default) one stream per request
    (``n_streams`` streams, 0 = 12); 1 continuous batching (queued requests
    run together as batched passes on ``n_streams`` batch slots, 0 = 6)."""

    def __init__(self, ctx, max_inflight: int = 32, hbm_budget_bytes: int = 0, n_streams: int = 0, mode: int = 0):
        self.ctx = ctx
        self.lib = ctx.lib
        h = ctypes.c_void_p()
        cfg = _Cfg(max_inflight, hbm_budget_bytes, n_streams, mode)
        ctx.check(self.lib.okscuda_server_create(ctx.handle, ctypes.byref(cfg), ctypes.byref(h)))
        self.handle = h.value
        self._live = {}   # id -> buffers kept alive until completion

    def close(self):
        if self.handle:
            self.lib.okscuda_server_destroy(self.handle)
            self.handle = None
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, kspace, mask, iters: int, lam: float, out: np.ndarray | None = None, device=None,
               device_slice=None):
        """Returns (id, out) or raises OksError (code OKS_EAGAIN when refused).
        ``device``: a DeviceArray [nc, ny, nx] in place of host k-space;
        ``device_slice``: (DeviceArray [nc, nz, ny, nx], z) -- slice z of a
        device-resident volume, read in place with the volume's coil stride."""
        stride = 0
        if device_slice is not None:
            vol, z = device_slice
            nc, nz, ny, nx = vol.shape
            hk, dk, keep_k = None, vol.ptr + int(z) * ny * nx * vol.dtype.itemsize, vol
            stride = nz * ny * nx
        elif device is not None:
            nc, ny, nx = device.shape
            hk, dk, keep_k = None, device.ptr, device
        else:
            k = kspace if (isinstance(kspace, np.ndarray) and kspace.dtype == np.complex64
                           and kspace.flags["C_CONTIGUOUS"]) else np.ascontiguousarray(kspace, np.complex64)
            nc, ny, nx = k.shape
            hk, dk, keep_k = k.ctypes.data, None, k
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        o = out if out is not None else np.empty((ny, nx), np.float32)
        req = _Req(hk, dk, m.ctypes.data, nc, ny, nx, int(iters), float(lam), o.ctypes.data, stride)
        rid = ctypes.c_uint64()
        rc = self.lib.okscuda_server_submit(self.handle, ctypes.byref(req), ctypes.byref(rid))
        if rc != 0:
            raise OksError(rc, self.ctx.last_error())
        self._live[rid.value] = (keep_k, m, o)
        return rid.value, o

    def poll(self, rid: int) -> bool:
        done = ctypes.c_int()
        rc = self.lib.okscuda_server_poll(self.handle, rid, ctypes.byref(done))
        if done.value:
            self._live.pop(rid, None)
        if rc != 0:
            raise OksError(rc, self.ctx.last_error())
        return bool(done.value)

    def wait(self, rid: int, timeout_ms: int = 60000):
        rc = self.lib.okscuda_server_wait(self.handle, rid, int(timeout_ms))
        if rc != _lib.OKS_ETIMEDOUT:
            self._live.pop(rid, None)
        if rc != 0:
            raise OksError(rc, self.ctx.last_error())

    def stats(self):
        a, b, c = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_size_t()
        self.ctx.check(self.lib.okscuda_server_stats(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return {"inflight": a.value, "completed": b.value, "reserved_bytes": c.value}
