"""Host mirror of the reference's `math-cuda` API (crypto/math-cuda/src/*.rs).

Same function names, argument meaning and results as the Rust seam the stark
crate calls; host arrays are numpy uint64 (field elements) or uint8 (digests),
device-resident results are handles. Errors raise native.SgError (the Rust
side returns Err(DriverError)); nothing falls back to the CPU.
"""
import ctypes as C

import numpy as np

from . import native
from .device import DeviceBuffer, backend

P = 0xFFFFFFFF00000001


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


# ------------------------------------------------------------------ ntt (ntt.rs)
def ntt_forward(coeffs, be=None):
    """ntt::forward (ntt.rs:57): natural-order coefficients -> evaluations.
    1-D input, or a row-major (n, m) batch transformed column by column."""
    return _ntt(coeffs, False, be)


def ntt_inverse(evals, be=None):
    """ntt::inverse (ntt.rs:64): natural-order evaluations -> coefficients (1/n included)."""
    return _ntt(evals, True, be)


def _ntt(x, inverse, be):
    be = be or backend()
    a = _u64(x)
    shape = a.shape
    n = shape[0]
    m = 1 if a.ndim == 1 else int(np.prod(shape[1:]))
    if n <= 1:
        return a.copy()
    d = DeviceBuffer.from_host(a, be)
    f = native.lib().sg_ntt_inverse if inverse else native.lib().sg_ntt_forward
    native.check(f(be.h, None, d.ptr, n, m))
    out = d.download(np.uint64, n * m).reshape(shape)
    d.close()
    return out


# ------------------------------------------------------------------ lde (lde.rs)
def coset_lde_batch_base(row_major, blowup_factor, weights, be=None):
    """Row-major batched coset LDE (lde.rs:1072 batch semantics, row-major like
    Polynomial::coset_lde_full_expand_row_major): (n, m) -> (blowup*n, m)."""
    be = be or backend()
    t = _u64(row_major)
    if t.ndim == 1:
        t = t.reshape(-1, 1)
    n, m = t.shape
    if n == 0 or m == 0:
        return np.zeros((n * blowup_factor, m), np.uint64)
    w = _u64(weights)
    assert w.size == n, "weights length must match n"
    dt = DeviceBuffer.from_host(t, be)
    dw = DeviceBuffer.from_host(w, be)
    do = DeviceBuffer(n * blowup_factor * m * 8, be)
    native.check(native.lib().sg_coset_lde(be.h, None, dt.ptr, n, m, blowup_factor, dw.ptr, do.ptr))
    out = do.download(np.uint64, n * blowup_factor * m).reshape(n * blowup_factor, m)
    for b in (dt, dw, do):
        b.close()
    return out


def coset_lde_base(evals, blowup_factor, weights, be=None):
    """lde::coset_lde_base (lde.rs:990): one column."""
    return coset_lde_batch_base(_u64(evals).reshape(-1, 1), blowup_factor, weights, be).reshape(-1)


class GpuLde:
    """Device-resident LDE + Merkle tree (GpuLdeBase / GpuLdeExt3 + GpuMerkleTree,
    lde.rs:923-988). The LDE stays row-major on the device (the reference
    transposes to column-major; the kernels here read rows directly)."""

    def __init__(self, handle, be):
        self.h = handle
        self.be = be
        info = native.LdeInfo()
        native.check(native.lib().sg_lde_get_info(handle, C.byref(info)))
        self.d_lde = info.d_lde
        self.lde_size = info.lde_rows
        self.row_u64 = info.row_u64
        self.d_nodes = info.d_nodes
        self.leaves_len = info.leaves_len
        self.root = bytes(info.root)

    def lde_host(self):
        out = np.empty(self.lde_size * self.row_u64, np.uint64)
        native.check(native.lib().sg_memcpy_d2h(self.be.h, None, out.ctypes.data, self.d_lde, out.nbytes))
        native.check(native.lib().sg_stream_sync(self.be.h, None))
        return out.reshape(self.lde_size, self.row_u64)

    def nodes_host(self):
        nb = (2 * self.leaves_len - 1) * 32
        out = np.empty(nb, np.uint8)
        native.check(native.lib().sg_memcpy_d2h(self.be.h, None, out.ctypes.data, self.d_nodes, nb))
        native.check(native.lib().sg_stream_sync(self.be.h, None))
        return out.reshape(-1, 32)

    def free(self):
        if self.h:
            native.lib().sg_lde_free(self.be.h, self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _layout(rows_per_leaf=2, little_endian=False, col_range=None):
    c0, c1 = (0, 0) if col_range is None else col_range
    return native.LeafLayout(rows_per_leaf, 1 if little_endian else 0, c0, c1)


def lde_commit(row_major, n, row_u64, blowup_factor, weights, rows_per_leaf=2, little_endian=False,
               col_range=None, retain_host_lde=False, be=None):
    """General LDE + Keccak leaves + Merkle tree on device. Returns (GpuLde, host LDE or empty)."""
    be = be or backend()
    t = _u64(row_major).reshape(-1)
    assert t.size == n * row_u64, "row-major input shape"
    w = _u64(weights)
    assert w.size == n, "weights length must match n"
    lay = _layout(rows_per_leaf, little_endian, col_range)
    host = np.empty((n * blowup_factor, row_u64), np.uint64) if retain_host_lde else None
    h = C.c_void_p()
    root = (C.c_uint8 * 32)()
    native.check(native.lib().sg_lde_commit(be.h, None, t.ctypes.data, 0, n, row_u64, blowup_factor, w.ctypes.data,
                                            C.byref(lay), host.ctypes.data if host is not None else None,
                                            C.byref(h), root))
    return GpuLde(h, be), (host if host is not None else np.empty((0,), np.uint64))


def coset_lde_row_major_with_merkle_tree_keep(row_major, n, m, blowup_factor, weights, retain_host_lde=False,
                                              be=None):
    """lde::coset_lde_row_major_with_merkle_tree_keep (lde.rs:674): base-field
    row-major LDE, row-pair big-endian leaves, resident tree."""
    return lde_commit(row_major, n, m, blowup_factor, weights, 2, False, None, retain_host_lde, be)


def coset_lde_ext3_row_major_with_merkle_tree_keep(row_major, n, m, blowup_factor, weights, retain_host_lde=False,
                                                   be=None):
    """lde::coset_lde_ext3_row_major_with_merkle_tree_keep (lde.rs:855): m ext3
    columns (3m u64 per row, components consecutive)."""
    return lde_commit(row_major, n, 3 * m, blowup_factor, weights, 2, False, None, retain_host_lde, be)


# ------------------------------------------------------------------ merkle (merkle.rs)
def keccak_leaves_row_major(data, rows_per_leaf=2, little_endian=False, col_range=None, be=None):
    """Leaf digests of a row-major (rows, row_u64) matrix, bit-reversed rows
    (commitment.rs:52-107 layout; merkle.rs:33 keccak_leaves_base analog)."""
    be = be or backend()
    d = _u64(data)
    if d.ndim == 1:
        d = d.reshape(-1, 1)
    rows, ru = d.shape
    nl = rows // rows_per_leaf
    dd = DeviceBuffer.from_host(d, be)
    do = DeviceBuffer(nl * 32, be)
    lay = _layout(rows_per_leaf, little_endian, col_range)
    native.check(native.lib().sg_keccak_leaves(be.h, None, dd.ptr, rows, ru, C.byref(lay), do.ptr))
    out = do.download(np.uint8, nl * 32).reshape(nl, 32)
    dd.close()
    do.close()
    return out


def build_merkle_tree_on_device(hashed_leaves, be=None):
    """merkle::build_merkle_tree_on_device (merkle.rs:316): full node array,
    ((2L-1), 32) bytes, root at row 0."""
    be = be or backend()
    lv = np.ascontiguousarray(hashed_leaves, np.uint8).reshape(-1, 32)
    n = lv.shape[0]
    L = native.lib().sg_merkle_leaves_len(n)
    dl = DeviceBuffer.from_host(lv, be)
    dn = DeviceBuffer((2 * L - 1) * 32, be)
    root = (C.c_uint8 * 32)()
    native.check(native.lib().sg_merkle_build(be.h, None, dl.ptr, n, dn.ptr, root))
    out = dn.download(np.uint8).reshape(-1, 32)
    dl.close()
    dn.close()
    return out


def gather_merkle_paths_dev(d_nodes, leaves_len, positions, be=None):
    """merkle::gather_merkle_paths_dev (merkle.rs:358) against a resident tree."""
    be = be or backend()
    pos = np.ascontiguousarray(positions, np.uint32)
    depth = int(leaves_len).bit_length() - 1
    dp = DeviceBuffer.from_host(pos, be)
    do = DeviceBuffer(max(1, pos.size * depth * 32), be)
    native.check(native.lib().sg_merkle_gather_paths(be.h, None, d_nodes, leaves_len, dp.ptr, pos.size, do.ptr))
    out = do.download(np.uint8, pos.size * depth * 32).reshape(pos.size, depth, 32)
    dp.close()
    do.close()
    return out


# ------------------------------------------------------------------ grinding (grinding.rs)
def generate_nonce_gpu(inner_lanes, grinding_factor, be=None):
    """grinding::generate_nonce_gpu (grinding.rs:29): smallest valid nonce."""
    be = be or backend()
    lanes = _u64(inner_lanes)
    out = C.c_uint64()
    native.check(native.lib().sg_grind(be.h, None, lanes.ctypes.data, grinding_factor, C.byref(out)))
    return out.value


def inner_hash_lanes(inner_hash: bytes):
    """stark::grinding::inner_hash_lanes: the 32-byte inner hash as 4 LE u64 lanes."""
    return np.frombuffer(bytes(inner_hash), dtype="<u8").astype(np.uint64)
