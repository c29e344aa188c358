"""sg_coset_lde_static — the allocation-free coset LDE — against sg_coset_lde.

The allocation-free entry point serves callers that cannot allocate device
memory while they run (for example a serving process that reserved all of its
HBM at start-up and must not grow it mid-request). It keeps its scratch in a
fixed-size static device array instead of allocating, so this test checks that
it returns exactly what the ordinary entry point returns, on two calls in a row
(the second call reuses the scratch the first one left behind), and that a
request larger than the static scratch is rejected with a clear error.
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from lambda_vm_b200 import native
from lambda_vm_b200.device import DeviceBuffer

pytestmark = pytest.mark.gpu
P = 0xFFFFFFFF00000001


def _weights(n, g=3):
    ninv = pow(n, P - 2, P)
    return np.array([ninv * pow(g, i, P) % P for i in range(n)], dtype=np.uint64)


def _both(be, log_n, m, blowup, seed):
    rng = np.random.default_rng(seed)
    n = 1 << log_n
    trace = rng.integers(0, 2**64, size=(n, m), dtype=np.uint64)
    w = _weights(n)
    L = native.lib()
    dt = DeviceBuffer.from_host(trace, be)
    dw = DeviceBuffer.from_host(w, be)
    d_ref = DeviceBuffer(n * blowup * m * 8, be)
    d_static = DeviceBuffer(n * blowup * m * 8, be)
    native.check(L.sg_coset_lde(be.h, None, dt.ptr, n, m, blowup, dw.ptr, d_ref.ptr))
    native.check(L.sg_coset_lde_static(None, dt.ptr, n, m, blowup, dw.ptr, d_static.ptr))
    native.check(L.sg_stream_sync(be.h, None))
    ref = d_ref.download(np.uint64)
    got = d_static.download(np.uint64)
    for b in (dt, dw, d_ref, d_static):
        b.close()
    return ref, got


def test_static_lde_matches_allocating_lde_on_two_calls(be):
    # First call: four-step path (n > 4096); second call: a different shape on
    # the single-pass path, reading scratch the first call left behind.
    ref1, got1 = _both(be, 14, 40, 4, seed=11)
    assert got1.size == ref1.size and (got1 == ref1).all()
    ref2, got2 = _both(be, 10, 7, 8, seed=12)
    assert got2.size == ref2.size and (got2 == ref2).all()


def test_static_lde_rejects_oversized_requests(be):
    L = native.lib()
    n, m, blowup = 1 << 20, 16, 4  # needs (4n + 2nm) * 8 bytes > the static scratch
    assert (blowup * n + 2 * n * m) * 8 > native.SG_STATIC_SCRATCH_BYTES
    rc = L.sg_coset_lde_static(None, C.c_void_p(16), n, m, blowup, C.c_void_p(16), C.c_void_p(16))
    assert rc == native.SG_ERR_INVALID
    assert b"static scratch" in L.sg_last_error()
    # a column count whose scratch size wraps 64 bits is rejected too, before any launch
    for m in (1 << 63, (1 << 64) - 1, (1 << 64) // (2 << 10) + 1):
        rc = L.sg_coset_lde_static(None, C.c_void_p(16), 1 << 10, m, 2, C.c_void_p(16), C.c_void_p(16))
        assert rc == native.SG_ERR_INVALID
        assert b"static scratch" in L.sg_last_error()
