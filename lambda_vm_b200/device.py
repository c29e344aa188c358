"""Device context and buffers over the C ABI.

Mirrors crypto/math-cuda/src/device.rs: one process-wide backend per GPU
(`backend()`, device.rs:592-619) owning the context, with host<->device copies
and device buffers charged to an HBM budget (device.rs:272-319, VramGate).
"""
import ctypes as C
import threading

import numpy as np

from . import native

_backends = {}
_lock = threading.Lock()


class Backend:
    def __init__(self, device: int = 0, budget_bytes: int = 0):
        L = native.lib()
        h = C.c_void_p()
        native.check(L.sg_ctx_create(device, budget_bytes, C.byref(h)))
        self.h = h
        self.device = device
        self.pass_model = None  # parameters of the installed DFT pass-cost model, if any

    def memory(self):
        a, b = C.c_uint64(), C.c_uint64()
        native.check(native.lib().sg_ctx_memory(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def budget(self) -> int:
        return native.lib().sg_ctx_budget(self.h)

    def launches(self) -> int:
        return native.lib().sg_ctx_launches(self.h)

    def fail_alloc_after(self, n: int):
        native.check(native.lib().sg_ctx_fail_alloc_after(self.h, n))

    def sync(self, stream=None):
        native.check(native.lib().sg_stream_sync(self.h, stream))

    def close(self):
        if self.h:
            native.lib().sg_ctx_destroy(self.h)
            self.h = None


def backend(device: int = 0) -> Backend:
    """Process-wide context for `device` (device::backend()). The committed
    DFT pass-cost model (costmodel.py) chooses its tile widths, unless the
    environment sets SG_PASS_MODEL=0 (the timing probe then decides)."""
    import os
    with _lock:
        b = _backends.get(device)
        if b is None:
            b = Backend(device)
            if os.environ.get("SG_PASS_MODEL", "1") != "0":
                from . import costmodel
                if os.path.exists(costmodel.MODEL):
                    params, _ = costmodel.load_model()
                    costmodel.install(b, params)
                    b.pass_model = params
            _backends[device] = b
        return b


class DeviceBuffer:
    """A device allocation owned by Python; freed on close()/GC."""

    def __init__(self, nbytes: int, be: Backend = None, stream=None):
        self.be = be or backend()
        self.nbytes = int(nbytes)
        self.stream = stream
        p = C.c_void_p()
        native.check(native.lib().sg_dev_alloc(self.be.h, stream, self.nbytes, C.byref(p)))
        self.ptr = p.value or 0

    @classmethod
    def from_host(cls, arr: np.ndarray, be: Backend = None, stream=None):
        a = np.ascontiguousarray(arr)
        b = cls(a.nbytes, be, stream)
        b.upload(a)
        return b

    def upload(self, arr: np.ndarray, offset: int = 0):
        a = np.ascontiguousarray(arr)
        native.check(native.lib().sg_memcpy_h2d(self.be.h, self.stream, self.ptr + offset, a.ctypes.data, a.nbytes))
        native.check(native.lib().sg_stream_sync(self.be.h, self.stream))

    def download(self, dtype=np.uint64, count=None, offset: int = 0):
        dt = np.dtype(dtype)
        n = (self.nbytes - offset) // dt.itemsize if count is None else count
        out = np.empty(n, dt)
        native.check(native.lib().sg_memcpy_d2h(self.be.h, self.stream, out.ctypes.data, self.ptr + offset, out.nbytes))
        native.check(native.lib().sg_stream_sync(self.be.h, self.stream))
        return out

    def close(self):
        if self.ptr:
            native.lib().sg_dev_free(self.be.h, self.stream, self.ptr, self.nbytes)
            self.ptr = 0

    free = close

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PinnedBuffer:
    """Page-locked host memory viewed as a numpy array."""

    def __init__(self, nbytes: int):
        p = C.c_void_p()
        native.check(native.lib().sg_host_alloc(nbytes, C.byref(p)))
        self.ptr = p.value
        self.nbytes = nbytes

    def view(self, dtype=np.uint64, shape=None):
        dt = np.dtype(dtype)
        arr = np.ctypeslib.as_array((C.c_uint8 * self.nbytes).from_address(self.ptr)).view(dt)
        return arr if shape is None else arr.reshape(shape)

    def close(self):
        if self.ptr:
            native.lib().sg_host_free(self.ptr)
            self.ptr = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
