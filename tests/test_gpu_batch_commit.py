"""sg_batch_commit: many tables committed in one call (heaviest first over
internal streams) give, table by table, exactly what sg_lde_commit gives for
that table alone: the same root, LDE and node array. sg_batch_commit_fused
(every table's DFT passes in shared multi-table launches) gives the same."""
import ctypes as C

import numpy as np
import pytest

from lambda_vm_b200 import field as F
from lambda_vm_b200 import native
from lambda_vm_b200.device import DeviceBuffer

pytestmark = pytest.mark.gpu
P = F.P


def _tables(rng, shapes):
    out = []
    for n, m, B, rpl, le in shapes:
        tr = (rng.integers(0, 2**63, size=(n, m), dtype=np.uint64) * np.uint64(2)) % np.uint64(P)
        out.append((tr, n, m, B, rpl, le))
    return out


def _single(be, tr, n, m, B, rpl, le):
    L = native.lib()
    h = C.c_void_p()
    root = (C.c_uint8 * 32)()
    lay = native.LeafLayout(rpl, le, 0, 0)
    w = F.coset_weights(n, 3)
    native.check(L.sg_lde_commit(be.h, None, tr.ctypes.data, 0, n, m, B, w.ctypes.data, C.byref(lay), None,
                                 C.byref(h), root))
    info = native.LdeInfo()
    native.check(L.sg_lde_get_info(h, C.byref(info)))
    lde = np.empty(n * B * m, np.uint64)
    nodes = np.empty((2 * info.leaves_len - 1) * 4, np.uint64)
    native.check(L.sg_memcpy_d2h(be.h, None, lde.ctypes.data, info.d_lde, lde.nbytes))
    native.check(L.sg_memcpy_d2h(be.h, None, nodes.ctypes.data, info.d_nodes, nodes.nbytes))
    L.sg_lde_free(be.h, h)
    return bytes(root), lde, nodes


SHAPES = [(1 << 12, 7, 2, 2, 0), (1 << 6, 33, 4, 1, 1), (1 << 14, 20, 2, 2, 0), (4, 3, 8, 2, 0),
          (1 << 10, 64, 2, 1, 1), (1 << 13, 1, 4, 2, 0), (1 << 9, 300, 2, 2, 0)]
# many tables of shared and distinct pass lengths, widths 1..300, both
# directions' tile widths, single-pass and four-step LDEs, odd and even log n
FUSED_SHAPES = SHAPES + [(1 << 14, 9, 2, 2, 0), (1 << 14, 6, 2, 2, 0), (1 << 16, 40, 2, 2, 0), (1 << 15, 3, 4, 2, 0),
                         (1 << 17, 12, 2, 2, 0), (1 << 20, 16, 2, 2, 0), (1 << 21, 5, 2, 2, 0), (1 << 11, 100, 2, 2, 0),
                         (2, 4, 2, 2, 0), (1 << 18, 33, 4, 2, 0), (1 << 16, 40, 2, 2, 0)]


@pytest.mark.parametrize("on_device,fused", [(False, False), (True, False), (True, True)])
def test_batch_commit_equals_single_commits(be, on_device, fused):
    rng = np.random.default_rng(5)
    shapes = FUSED_SHAPES if fused else SHAPES
    tabs = _tables(rng, shapes)
    L = native.lib()
    keep = []
    descs = (native.TableDesc * len(tabs))()
    for i, (tr, n, m, B, rpl, le) in enumerate(tabs):
        w = F.coset_weights(n, 3)
        if on_device:
            dt, dw = DeviceBuffer.from_host(tr, be), DeviceBuffer.from_host(w, be)
            keep += [dt, dw]
            descs[i] = native.TableDesc(dt.ptr, 1, n, m, B, 1, dw.ptr, native.LeafLayout(rpl, le, 0, 0))
        else:
            keep += [tr, w]
            descs[i] = native.TableDesc(tr.ctypes.data, 0, n, m, B, 0, w.ctypes.data, native.LeafLayout(rpl, le, 0, 0))
    handles = (C.c_void_p * len(tabs))()
    roots = (C.c_uint8 * (32 * len(tabs)))()
    if fused:
        native.check(L.sg_batch_commit_fused(be.h, None, descs, len(tabs), 4, handles, roots))
    else:
        native.check(L.sg_batch_commit(be.h, None, descs, len(tabs), 3, handles, roots))
    for i, t in enumerate(tabs):
        root, lde, nodes = _single(be, *t)
        assert bytes(roots[32 * i:32 * i + 32]) == root
        info = native.LdeInfo()
        native.check(L.sg_lde_get_info(handles[i], C.byref(info)))
        assert bytes(info.root) == root
        got = np.empty_like(lde)
        native.check(L.sg_memcpy_d2h(be.h, None, got.ctypes.data, info.d_lde, got.nbytes))
        assert np.array_equal(got, lde)
        gn = np.empty_like(nodes)
        native.check(L.sg_memcpy_d2h(be.h, None, gn.ctypes.data, info.d_nodes, gn.nbytes))
        assert np.array_equal(gn, nodes)
        L.sg_lde_free_async(be.h, None, handles[i])
    native.check(L.sg_stream_sync(be.h, None))


def test_batch_commit_rejects_bad_table_and_leaks_nothing(be):
    L = native.lib()
    rng = np.random.default_rng(6)
    good = (rng.integers(0, 2**32, size=(256, 5), dtype=np.uint64))
    bad = np.zeros((48, 5), np.uint64)  # 48 rows: not a power of two
    w1, w2 = F.coset_weights(256, 3), np.ones(48, np.uint64)
    descs = (native.TableDesc * 2)()
    descs[0] = native.TableDesc(good.ctypes.data, 0, 256, 5, 2, 0, w1.ctypes.data, native.LeafLayout(0, 0, 0, 0))
    descs[1] = native.TableDesc(bad.ctypes.data, 0, 48, 5, 2, 0, w2.ctypes.data, native.LeafLayout(0, 0, 0, 0))
    # the context keeps one root-of-unity table per LDE size: build it first
    _single(be, good, 256, 5, 2, 2, 0)
    native.check(L.sg_stream_sync(be.h, None))
    before, _ = be.memory()
    handles = (C.c_void_p * 2)()
    rc = L.sg_batch_commit(be.h, None, descs, 2, 2, handles, None)
    assert rc == native.SG_ERR_INVALID
    assert not handles[0] and not handles[1]
    native.check(L.sg_stream_sync(be.h, None))
    after, _ = be.memory()
    assert after == before
    # the fused form rejects host traces and bad shapes before allocating anything
    rc = L.sg_batch_commit_fused(be.h, None, descs, 2, 2, handles, None)
    assert rc == native.SG_ERR_INVALID and not handles[0] and not handles[1]
    native.check(L.sg_stream_sync(be.h, None))
    assert be.memory()[0] == before
