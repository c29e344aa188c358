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


# ------------------------------------------------------------------ transcript (host, in the library)
class Transcript:
    """DefaultTranscript (default_transcript.rs:31-146) implemented in libstarkgpu."""

    def __init__(self, data: bytes = b"", _h=None):
        L = native.lib()
        if _h is None:
            buf = (C.c_uint8 * max(1, len(data))).from_buffer_copy(bytes(data) or b"\0")
            _h = L.sg_transcript_new(buf, len(data))
        self.h = _h

    def clone(self):
        return Transcript(_h=native.lib().sg_transcript_clone(self.h))

    def append_bytes(self, data: bytes):
        buf = (C.c_uint8 * max(1, len(data))).from_buffer_copy(bytes(data) or b"\0")
        native.lib().sg_transcript_append(self.h, buf, len(data))

    def append_base(self, v):
        native.lib().sg_transcript_append_base(self.h, int(v))

    def append_ext3(self, v):
        a = _u64(v)
        native.lib().sg_transcript_append_ext3(self.h, a.ctypes.data)

    def append_ext3_many(self, vals):
        """Absorb a sequence of Fp3 elements in order: the same absorption as
        append_ext3 on each (canonical c0 || c1 || c2, big-endian), in one update."""
        a = np.asarray(vals, np.uint64).reshape(-1, 3)
        p = np.uint64(0xFFFFFFFF00000001)
        c = np.where(a >= p, a - p, a)
        self.append_bytes(c.astype(">u8").tobytes())

    def sample(self) -> bytes:
        out = (C.c_uint8 * 32)()
        native.lib().sg_transcript_sample(self.h, out)
        return bytes(out)

    def state(self) -> bytes:
        out = (C.c_uint8 * 32)()
        native.lib().sg_transcript_state(self.h, out)
        return bytes(out)

    def sample_base(self) -> int:
        return native.lib().sg_transcript_sample_base(self.h)

    def sample_ext3(self):
        out = np.zeros(3, np.uint64)
        native.lib().sg_transcript_sample_ext3(self.h, out.ctypes.data)
        return out

    def sample_u64(self, upper: int) -> int:
        return native.lib().sg_transcript_sample_u64(self.h, upper)

    def sample_z_ood(self, trace_len, lde_len, coset_offset):
        out = np.zeros(3, np.uint64)
        native.lib().sg_transcript_sample_z_ood(self.h, trace_len, lde_len, coset_offset, out.ctypes.data)
        return out

    def __del__(self):
        try:
            if self.h:
                native.lib().sg_transcript_free(self.h)
                self.h = None
        except Exception:
            pass


def keccak256(data: bytes) -> bytes:
    buf = (C.c_uint8 * max(1, len(data))).from_buffer_copy(bytes(data) or b"\0")
    out = (C.c_uint8 * 32)()
    native.lib().sg_keccak256(buf, len(data), out)
    return bytes(out)


# ------------------------------------------------------------------ inverse (inverse.rs)
def batch_inverse_ext3(a, be=None):
    """inverse::batch_inverse_ext3 (inverse.rs:53): interleaved ext3 in/out."""
    be = be or backend()
    x = _u64(a).reshape(-1)
    n = x.size // 3
    if n == 0:
        return x.copy()
    d = DeviceBuffer.from_host(x, be)
    z = C.c_int(0)
    native.check(native.lib().sg_batch_inverse_ext3(be.h, None, d.ptr, n, d.ptr, C.byref(z)))
    if z.value:
        raise ZeroDivisionError("batch inverse of a zero element")
    out = d.download(np.uint64, 3 * n)
    d.close()
    return out


def compute_and_invert_denoms_ext3(x, z_scalars, x_minus_z, be=None):
    """inverse::compute_and_invert_denoms_ext3_dev (inverse.rs:241) with host I/O."""
    be = be or backend()
    x = _u64(x)
    z = _u64(z_scalars).reshape(-1)
    n, k = x.size, z.size // 3
    dx = DeviceBuffer.from_host(x, be)
    do = DeviceBuffer(24 * n * k, be)
    zf = C.c_int(0)
    native.check(native.lib().sg_inv_denoms_ext3(be.h, None, dx.ptr, n, z.ctypes.data, k, 1 if x_minus_z else 0,
                                                 do.ptr, C.byref(zf)))
    if zf.value:
        raise ZeroDivisionError("zero denominator")
    out = do.download(np.uint64, 3 * n * k)
    dx.close()
    do.close()
    return out


# ------------------------------------------------------------------ barycentric (barycentric.rs)
def barycentric_multi(data, row_stride, ext3, cols, points, inv_denoms, n, k, be=None):
    """barycentric::barycentric_{base,ext3}_multi_on_device (barycentric.rs:379,449):
    k x cols ext3 sums over a row-major (rows, row_u64) matrix."""
    be = be or backend()
    d = _u64(data)
    ru = d.shape[1]
    dd = DeviceBuffer.from_host(d, be)
    dp = DeviceBuffer.from_host(_u64(points), be)
    di = DeviceBuffer.from_host(_u64(inv_denoms), be)
    do = DeviceBuffer(24 * k * cols, be)
    native.check(native.lib().sg_barycentric_sums(be.h, None, dd.ptr, ru, row_stride, 1 if ext3 else 0, cols, dp.ptr,
                                                  di.ptr, n, k, do.ptr))
    out = do.download(np.uint64, 3 * k * cols)
    for b in (dd, dp, di, do):
        b.close()
    return out


# ------------------------------------------------------------------ DEEP (deep.rs)
def deep_composition_ext3(main, aux, parts, h_ood, trace_ood, gammas_h, gammas_tr, inv_h, inv_t, k,
                           bitrev_out=False, be=None):
    """deep::deep_composition_ext3 (deep.rs:25) over row-major LDEs; returns rows x 3."""
    be = be or backend()
    main, aux, parts = _u64(main), _u64(aux), _u64(parts)
    rows = main.shape[0]
    m = main.shape[1]
    a = aux.shape[1] // 3 if aux.size else 0
    p = parts.shape[1] // 3 if parts.size else 0
    bufs = [DeviceBuffer.from_host(x, be) if x.size else None for x in (main, aux, parts, _u64(inv_h), _u64(inv_t))]
    do = DeviceBuffer(24 * rows, be)
    ptr = [b.ptr if b is not None else None for b in bufs]
    hh, to, gh, gt = _u64(h_ood), _u64(trace_ood), _u64(gammas_h), _u64(gammas_tr)
    native.check(native.lib().sg_deep_composition(be.h, None, ptr[0], m, ptr[1], a, ptr[2], p, rows,
                                                  hh.ctypes.data, to.ctypes.data, gh.ctypes.data, gt.ctypes.data,
                                                  k, ptr[3], ptr[4], 1 if bitrev_out else 0, do.ptr))
    out = do.download(np.uint64, 3 * rows)
    for b in bufs + [do]:
        if b is not None:
            b.close()
    return out


# ------------------------------------------------------------------ FRI (fri.rs)
def fri_fold(evals, inv_tw, zeta, with_leaves=True, be=None):
    """One FRI fold (fri_functions.rs fold_evaluations_in_place) plus, fused, the
    folded layer's leaves and the next twiddles. Returns (folded, tw_next, leaves)."""
    be = be or backend()
    e = _u64(evals).reshape(-1)
    h = e.size // 6
    din = DeviceBuffer.from_host(e, be)
    dtw = DeviceBuffer.from_host(_u64(inv_tw), be)
    dout = DeviceBuffer(24 * h, be)
    dtn = DeviceBuffer(8 * max(1, h // 2), be)
    dl = DeviceBuffer(32 * max(1, h // 2), be) if with_leaves else None
    z = _u64(zeta)
    native.check(native.lib().sg_fri_fold_layer(be.h, None, din.ptr, h, dtw.ptr, z.ctypes.data, dout.ptr, dtn.ptr,
                                                dl.ptr if dl else None))
    out = dout.download(np.uint64, 3 * h)
    tn = dtn.download(np.uint64, h // 2)
    lv = dl.download(np.uint8, 32 * (h // 2)).reshape(-1, 32) if dl else None
    for b in (din, dtw, dout, dtn) + ((dl,) if dl else ()):
        b.close()
    return out, tn, lv


# ------------------------------------------------------------------ LogUp (logup.rs)
def logup_aux_resident(main, desc, alpha_powers, z, be=None):
    """logup::logup_aux_resident (logup.rs:311) over a row-major (n, m) main trace.
    desc: dict with the CSR descriptor fields (LogupDescriptor). Returns
    (aux (n, 3*(num_committed+1)), table_contribution)."""
    be = be or backend()
    main = _u64(main)
    n, m = main.shape
    keep = {}

    def arr(name, dt):
        a = np.ascontiguousarray(desc[name], dt)
        keep[name] = a if a.size else np.zeros(1, dt)
        return keep[name].ctypes.data

    d = native.LogupDesc()
    d.num_interactions = desc["num_interactions"]
    d.bus_ids = arr("bus_ids", np.uint64)
    d.elem_offsets = arr("elem_offsets", np.uint32)
    d.elem_alpha_idx = arr("elem_alpha_idx", np.uint32)
    d.elem_consts = arr("elem_consts", np.uint64)
    d.term_offsets = arr("term_offsets", np.uint32)
    d.term_coefs = arr("term_coefs", np.uint64)
    d.term_cols = arr("term_cols", np.uint32)
    d.num_out_cols = desc["num_out_cols"]
    d.out_col_offsets = arr("out_col_offsets", np.uint32)
    d.out_col_interactions = arr("out_col_interactions", np.uint32)
    d.mult_consts = arr("mult_consts", np.uint64)
    d.mult_term_offsets = arr("mult_term_offsets", np.uint32)
    d.mult_term_coefs = arr("mult_term_coefs", np.uint64)
    d.mult_term_cols = arr("mult_term_cols", np.uint32)
    d.num_committed = desc["num_committed"]
    al = _u64(alpha_powers).reshape(-1)
    W = desc["num_committed"] + 1
    dm = DeviceBuffer.from_host(main, be)
    da = DeviceBuffer(24 * n * W, be)
    L = np.zeros(3, np.uint64)
    zz = _u64(z)
    native.check(native.lib().sg_logup_aux(be.h, None, dm.ptr, n, m, C.byref(d), al.ctypes.data, al.size // 3,
                                           zz.ctypes.data, da.ptr, L.ctypes.data))
    aux = da.download(np.uint64, 3 * n * W).reshape(n, 3 * W)
    dm.close()
    da.close()
    return aux, L


# ------------------------------------------------------------------ constraints (constraint_interp.rs)
def _program_struct(lowered, keep):
    def arr(a, dt):
        a = np.ascontiguousarray(a, dt)
        if a.size == 0:
            a = np.zeros(1, dt)
        keep.append(a)
        return a.ctypes.data

    p = native.DeviceProgram()
    p.nodes = arr(lowered["nodes"], np.uint32)
    p.num_nodes = int(np.asarray(lowered["nodes"]).reshape(-1, 4).shape[0])
    p.base_consts = arr(lowered["base_consts"], np.uint64)
    p.num_base_consts = int(np.asarray(lowered["base_consts"]).size)
    p.ext_consts = arr(lowered["ext_consts"], np.uint64)
    p.num_ext_consts = int(np.asarray(lowered["ext_consts"]).size // 3)
    p.roots = arr(lowered["roots"], np.uint32)
    p.num_roots = int(lowered.get("num_roots", np.asarray(lowered["roots"]).size))
    p.num_base_slots = int(lowered["num_base_slots"])
    p.num_ext_slots = int(lowered["num_ext_slots"])
    p.node_roots = arr(lowered["node_roots"], np.uint32) if lowered.get("node_roots") is not None else None
    p.hand_kernel = int(lowered.get("hand_kernel", 0))
    p.hand_roots = int(lowered.get("hand_roots", 0))
    if lowered.get("logup_desc") is not None:
        d = logup_struct(lowered["logup_desc"], keep)
        keep.append(d)
        p.logup = C.addressof(d)
        p.logup_root = int(lowered["logup_root"])
    return p


def logup_struct(desc, keep):
    """sg_logup_desc of a LogUp descriptor dict (AIR.logup_descriptor()); the
    arrays it points to are appended to keep."""
    def arr(name, dt):
        a = np.ascontiguousarray(desc[name], dt)
        if a.size == 0:
            a = np.zeros(1, dt)
        keep.append(a)
        return a.ctypes.data

    d = native.LogupDesc()
    d.num_interactions = desc["num_interactions"]
    for nm, dt in (("bus_ids", np.uint64), ("elem_offsets", np.uint32), ("elem_alpha_idx", np.uint32),
                   ("elem_consts", np.uint64), ("term_offsets", np.uint32), ("term_coefs", np.uint64),
                   ("term_cols", np.uint32), ("out_col_offsets", np.uint32), ("out_col_interactions", np.uint32),
                   ("mult_consts", np.uint64), ("mult_term_offsets", np.uint32), ("mult_term_coefs", np.uint64),
                   ("mult_term_cols", np.uint32)):
        setattr(d, nm, arr(nm, dt))
    d.num_out_cols = desc["num_out_cols"]
    d.num_committed = desc["num_committed"]
    return d


def eval_constraints_on_device(lowered, main, aux, rap, alpha, table_offset, next_step, composition=None, be=None):
    """constraint_interp::eval_constraints_on_device (constraint_interp.rs:53) when
    composition is None (returns roots x rows x 3), else eval_composition_on_device
    (constraint_interp.rs:353) returning H (rows x 3). composition: dict with beta,
    z_inv, boundary list [(col, is_aux, value3, beta3)], b_z_inv (nb x rows)."""
    be = be or backend()
    keep = []
    prog = _program_struct(lowered, keep)
    main = _u64(main)
    aux = _u64(aux)
    rows, m = main.shape
    a = aux.shape[1] // 3 if aux.size else 0
    dm = DeviceBuffer.from_host(main, be)
    da = DeviceBuffer.from_host(aux, be) if aux.size else None
    rap_a, al_a, off = _u64(rap).reshape(-1), _u64(alpha).reshape(-1), _u64(table_offset)
    bufs = [dm] + ([da] if da else [])
    comp_p = None
    if composition is not None:
        c = native.Composition()
        beta = _u64(composition["beta"]).reshape(-1)
        keep.append(beta)
        c.beta_trans = beta.ctypes.data
        dz = DeviceBuffer.from_host(_u64(composition["z_inv"]), be)
        bufs.append(dz)
        c.d_z_inv = dz.ptr
        c.z_len = int(np.asarray(composition["z_inv"]).size)
        bnd = composition.get("boundary", [])
        c.num_boundary = len(bnd)
        if bnd:
            cols = np.array([b[0] for b in bnd], np.uint64)
            isa = np.array([1 if b[1] else 0 for b in bnd], np.uint64)
            val = _u64([b[2] for b in bnd]).reshape(-1)
            bb = _u64([b[3] for b in bnd]).reshape(-1)
            keep += [cols, isa, val, bb]
            c.b_col, c.b_is_aux, c.b_value, c.b_beta = cols.ctypes.data, isa.ctypes.data, val.ctypes.data, bb.ctypes.data
            dbz = DeviceBuffer.from_host(_u64(composition["b_z_inv"]), be)
            bufs.append(dbz)
            c.d_b_z_inv = dbz.ptr
        comp_p = C.byref(c)
        out_words = 3 * rows
    else:
        out_words = 3 * rows * prog.num_roots
    do = DeviceBuffer(8 * max(1, out_words), be)
    bufs.append(do)
    native.check(native.lib().sg_eval_constraints(be.h, None, C.byref(prog), rap_a.ctypes.data, rap_a.size // 3,
                                                  al_a.ctypes.data, al_a.size // 3, off.ctypes.data, dm.ptr, m,
                                                  da.ptr if da else None, a, rows, next_step, comp_p, do.ptr))
    out = do.download(np.uint64, out_words)
    for b in bufs:
        b.close()
    return out.reshape(rows, 3) if composition is not None else out.reshape(prog.num_roots, rows, 3)


def decompose_d2(h, inv_2x, be=None):
    """decompose_d2_ext3 (constraint_interp.cu:477): returns (H0, H1) each (n, 3)."""
    be = be or backend()
    hh = _u64(h).reshape(-1)
    rows = hh.size // 3
    dh = DeviceBuffer.from_host(hh, be)
    di = DeviceBuffer.from_host(_u64(inv_2x), be)
    do = DeviceBuffer(24 * rows, be)
    native.check(native.lib().sg_decompose_d2(be.h, None, dh.ptr, rows, di.ptr, do.ptr))
    out = do.download(np.uint64, 3 * rows).reshape(rows // 2, 6)
    for b in (dh, di, do):
        b.close()
    return out[:, :3].copy(), out[:, 3:].copy()
