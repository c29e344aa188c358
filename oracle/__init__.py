"""CPU oracle — TEST INFRASTRUCTURE ONLY.

ctypes/numpy wrapper over oracle/liboracle.so, a C restatement of lambda_vm's
CPU proving path (see oracle/oracle.c for the per-function reference
citations). Used by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline legs as the checker; the product (lambda_vm_b200) never imports it.
"""
import ctypes as C
import os

import numpy as np

from . import build as _build

P = 0xFFFFFFFF00000001

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = C.CDLL(path)
        u64, u32, vp, sz = C.c_uint64, C.c_uint32, C.c_void_p, C.c_size_t
        sig = {
            "or_gl_add": (u64, [u64, u64]),
            "or_gl_sub": (u64, [u64, u64]),
            "or_gl_mul": (u64, [u64, u64]),
            "or_gl_neg": (u64, [u64]),
            "or_gl_inv": (u64, [u64]),
            "or_gl_pow": (u64, [u64, u64]),
            "or_gl_canonical": (u64, [u64]),
            "or_gl_root_of_unity": (u64, [u32]),
            "or_fp3_mul": (None, [vp, vp, vp]),
            "or_fp3_inv": (C.c_int, [vp, vp]),
            "or_fft_two_half": (C.c_int, [vp, u64, u64, C.c_int]),
            "or_coset_weights": (None, [u64, u64, vp]),
            "or_coset_lde_row_major": (C.c_int, [vp, u64, u64, u64, vp, vp]),
            "or_keccak_f1600": (None, [vp]),
            "or_keccak256": (None, [vp, sz, vp]),
            "or_leaves_row_major": (C.c_int, [vp, u64, u64, u64, u64, u32, C.c_int, vp]),
            "or_merkle_build": (u64, [vp, u64, vp]),
            "or_merkle_path": (u32, [vp, u64, u64, vp]),
            "or_transcript_size": (sz, []),
            "or_transcript_init": (None, [vp, vp, sz]),
            "or_transcript_append": (None, [vp, vp, sz]),
            "or_transcript_sample": (None, [vp, vp]),
            "or_transcript_state": (None, [vp, vp]),
            "or_transcript_sample_base": (u64, [vp]),
            "or_transcript_sample_ext3": (None, [vp, vp]),
            "or_transcript_sample_u64": (u64, [vp, u64]),
            "or_transcript_append_base": (None, [vp, u64]),
            "or_transcript_append_ext3": (None, [vp, vp]),
            "or_grind_inner_hash": (None, [vp, C.c_uint8, vp]),
            "or_grind_is_valid": (C.c_int, [vp, u64, C.c_uint8]),
            "or_grind": (u64, [vp, C.c_uint8, u64]),
            "or_fp3_batch_inverse": (C.c_int, [vp, u64]),
            "or_fri_fold": (None, [vp, u64, vp, vp, vp]),
            "or_inv_denoms": (C.c_int, [vp, u64, vp, u64, C.c_int, vp]),
            "or_barycentric_sums": (None, [vp, u64, u64, C.c_int, u64, vp, vp, u64, u64, vp]),
            "or_deep": (None, [vp, u64, vp, u64, vp, u64, u64, vp, vp, vp, vp, vp, vp, u64, vp]),
            "or_fri_leaves": (None, [vp, u64, vp]),
            "or_logup_aux": (C.c_int, [vp, u64, u64, u32, vp, vp, vp, vp, vp, vp, vp, u32, vp, vp, vp, vp, vp, vp,
                                       u32, vp, vp, vp, vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


# ---------------- field ----------------
def gl_add(a, b): return lib().or_gl_add(a, b)
def gl_sub(a, b): return lib().or_gl_sub(a, b)
def gl_mul(a, b): return lib().or_gl_mul(a, b)
def gl_neg(a): return lib().or_gl_neg(a)
def gl_inv(a): return lib().or_gl_inv(a)
def gl_pow(a, e): return lib().or_gl_pow(a, e)
def canonical(a): return lib().or_gl_canonical(a)
def root_of_unity(log_n): return lib().or_gl_root_of_unity(log_n)


def canon_array(a):
    a = _u64(a)
    return np.where(a >= np.uint64(P), a - np.uint64(P), a)


def fp3_mul(a, b):
    a, b, out = _u64(a), _u64(b), np.zeros(3, np.uint64)
    lib().or_fp3_mul(_p(a), _p(b), _p(out))
    return out


def fp3_pow(a, e):
    r = np.array([1, 0, 0], np.uint64)
    b = _u64(a).copy()
    while e:
        if e & 1:
            r = fp3_mul(r, b)
        b = fp3_mul(b, b)
        e >>= 1
    return r


def fp3_inv(a):
    a, out = _u64(a), np.zeros(3, np.uint64)
    if lib().or_fp3_inv(_p(a), _p(out)):
        raise ZeroDivisionError("fp3 inverse of zero")
    return out


# ---------------- FFT / LDE ----------------
def fft(buf, inverse=False):
    """Natural-order batched DFT over the rows of a row-major (n, m) array;
    the inverse is unscaled (two_half_fft.rs semantics)."""
    a = _u64(buf).copy()
    n = a.shape[0]
    m = 1 if a.ndim == 1 else a.shape[1]
    rc = lib().or_fft_two_half(_p(a), n, m, 1 if inverse else 0)
    if rc:
        raise ValueError(f"fft rc={rc}")
    return a


def coset_weights(n, offset=3):
    w = np.zeros(n, np.uint64)
    lib().or_coset_weights(n, offset, _p(w))
    return w


def coset_lde_row_major(trace, blowup, weights=None, offset=3):
    """Polynomial::coset_lde_full_expand_row_major on a row-major (n, m) trace."""
    t = _u64(trace)
    if t.ndim == 1:
        t = t.reshape(-1, 1)
    n, m = t.shape
    if weights is None:
        weights = coset_weights(n, offset)
    w = _u64(weights)
    out = np.zeros((n * blowup, m), np.uint64)
    rc = lib().or_coset_lde_row_major(_p(t), n, m, blowup, _p(w), _p(out))
    if rc:
        raise ValueError(f"lde rc={rc}")
    return out


# ---------------- Keccak / Merkle ----------------
def keccak256(data: bytes) -> bytes:
    buf = np.frombuffer(bytes(data) + b"\0", np.uint8)
    out = np.zeros(32, np.uint8)
    lib().or_keccak256(_p(buf), len(data), _p(out))
    return out.tobytes()


def keccak_f1600(state):
    st = _u64(state).copy()
    lib().or_keccak_f1600(_p(st))
    return st


def leaves_row_major(data, rows_per_leaf=2, little_endian=False, col_range=None, row_u64=None):
    """keccak_leaves_bit_reversed_grouped over a row-major (rows, row_u64) array."""
    d = _u64(data)
    if d.ndim == 1:
        d = d.reshape(-1, 1)
    rows = d.shape[0]
    ru = d.shape[1] if row_u64 is None else row_u64
    c0, c1 = (0, ru) if col_range is None else col_range
    out = np.zeros((rows // rows_per_leaf, 32), np.uint8)
    rc = lib().or_leaves_row_major(_p(d), rows, ru, c0, c1, rows_per_leaf, 1 if little_endian else 0, _p(out))
    if rc:
        raise ValueError(f"leaves rc={rc}")
    return out


def merkle_nodes(leaves):
    """Full node array ((2L-1), 32): root at 0, leaves at [L-1, 2L-1)."""
    lv = np.ascontiguousarray(leaves, np.uint8).reshape(-1, 32)
    n = lv.shape[0]
    L = 1
    while L < n:
        L *= 2
    nodes = np.zeros((2 * L - 1, 32), np.uint8)
    lib().or_merkle_build(_p(lv), n, _p(nodes))
    return nodes


def merkle_root(leaves) -> bytes:
    return merkle_nodes(leaves)[0].tobytes()


def merkle_path(nodes, pos):
    nodes = np.ascontiguousarray(nodes, np.uint8)
    L = (nodes.shape[0] + 1) // 2
    out = np.zeros((64, 32), np.uint8)
    d = lib().or_merkle_path(_p(nodes), L, pos, _p(out))
    return out[:d].copy()


# ---------------- transcript ----------------
class Transcript:
    """DefaultTranscript (default_transcript.rs) restated."""

    def __init__(self, data: bytes = b""):
        self._buf = np.zeros(lib().or_transcript_size(), np.uint8)
        d = np.frombuffer(bytes(data) + b"\0", np.uint8)
        lib().or_transcript_init(_p(self._buf), _p(d), len(data))

    def clone(self):
        t = Transcript.__new__(Transcript)
        t._buf = self._buf.copy()
        return t

    def append_bytes(self, data: bytes):
        d = np.frombuffer(bytes(data) + b"\0", np.uint8)
        lib().or_transcript_append(_p(self._buf), _p(d), len(data))

    def append_base(self, v):
        lib().or_transcript_append_base(_p(self._buf), int(v))

    def append_ext3(self, v):
        a = _u64(v)
        lib().or_transcript_append_ext3(_p(self._buf), _p(a))

    def append_ext3_many(self, vals):
        """One append_ext3 per element (default_transcript.rs append semantics)."""
        for v in np.asarray(vals, np.uint64).reshape(-1, 3):
            self.append_ext3(v)

    def sample(self) -> bytes:
        out = np.zeros(32, np.uint8)
        lib().or_transcript_sample(_p(self._buf), _p(out))
        return out.tobytes()

    def state(self) -> bytes:
        out = np.zeros(32, np.uint8)
        lib().or_transcript_state(_p(self._buf), _p(out))
        return out.tobytes()

    def sample_base(self) -> int:
        return lib().or_transcript_sample_base(_p(self._buf))

    def sample_ext3(self):
        out = np.zeros(3, np.uint64)
        lib().or_transcript_sample_ext3(_p(self._buf), _p(out))
        return out

    def sample_u64(self, upper: int) -> int:
        return lib().or_transcript_sample_u64(_p(self._buf), upper)

    def sample_z_ood(self, trace_len, lde_len, offset):
        """IsStarkTranscript::sample_z_ood_with_domain_params (is_transcript.rs:44-75)."""
        off_pow = gl_pow(offset, lde_len)
        blow = lde_len // trace_len
        while True:
            z = self.sample_ext3()
            zt = fp3_pow(z, trace_len)
            in_trace = list(map(int, canon_array(zt))) == [1, 0, 0]
            zl = fp3_pow(zt, blow)
            in_lde = list(map(int, canon_array(zl))) == [canonical(off_pow), 0, 0]
            if not in_trace and not in_lde:
                return z


# ---------------- grinding / FRI / inversion ----------------
def grind_inner_hash(seed: bytes, g: int) -> bytes:
    s = np.frombuffer(bytes(seed), np.uint8).copy()
    out = np.zeros(32, np.uint8)
    lib().or_grind_inner_hash(_p(s), g, _p(out))
    return out.tobytes()


def grind_is_valid(inner: bytes, nonce: int, g: int) -> bool:
    s = np.frombuffer(bytes(inner), np.uint8).copy()
    return bool(lib().or_grind_is_valid(_p(s), nonce, g))


def grind(seed: bytes, g: int, max_nonce: int = 1 << 40) -> int:
    s = np.frombuffer(bytes(seed), np.uint8).copy()
    return lib().or_grind(_p(s), g, max_nonce)


def fp3_batch_inverse(a):
    x = _u64(a).copy()
    if lib().or_fp3_batch_inverse(_p(x), x.size // 3):
        raise ZeroDivisionError("zero in batch inverse")
    return x


def fri_fold(evals, inv_tw, zeta):
    e = _u64(evals).reshape(-1)
    h = e.size // 6
    tw = _u64(inv_tw)
    z = _u64(zeta)
    out = np.zeros(3 * h, np.uint64)
    lib().or_fri_fold(_p(e), h, _p(tw), _p(z), _p(out))
    return out


def fri_number_of_queries(blowup, security_bits=128, grinding=20):
    """GoldilocksCubicProofOptions::with_params (crypto/stark/src/proof/options.rs:106-134):
    Johnson-bound query count."""
    import math
    rate = 1.0 / blowup
    proximity = 1.0 - math.sqrt(rate) - 1.0 / 300.0
    bits_per_query = -math.log2(1.0 - proximity)
    return int(math.ceil((security_bits - grinding) / bits_per_query))


def inv_denoms(x, z, x_minus_z):
    x, z = _u64(x), _u64(z).reshape(-1)
    n, K = x.size, z.size // 3
    out = np.zeros(3 * n * K, np.uint64)
    if lib().or_inv_denoms(_p(x), n, _p(z), K, 1 if x_minus_z else 0, _p(out)):
        raise ZeroDivisionError("zero denominator")
    return out


def barycentric_sums(data, row_stride, ext3, cols, points, invd, n, K):
    d = _u64(data)
    ru = d.shape[1] if d.ndim == 2 else d.size
    out = np.zeros(3 * K * cols, np.uint64)
    lib().or_barycentric_sums(_p(d), ru, row_stride, 1 if ext3 else 0, cols, _p(_u64(points)), _p(_u64(invd)), n, K,
                              _p(out))
    return out


def deep(main, aux, parts, h_ood, trace_ood, gammas_h, gammas_tr, inv_h, inv_t, K):
    main, aux, parts = _u64(main), _u64(aux), _u64(parts)
    rows = main.shape[0]
    m = main.shape[1] if main.ndim == 2 else 0
    A = (aux.shape[1] // 3) if aux.ndim == 2 else 0
    Pp = (parts.shape[1] // 3) if parts.ndim == 2 else 0
    out = np.zeros(3 * rows, np.uint64)
    lib().or_deep(_p(main), m, _p(aux), A, _p(parts), Pp, rows, _p(_u64(h_ood)), _p(_u64(trace_ood)),
                  _p(_u64(gammas_h)), _p(_u64(gammas_tr)), _p(_u64(inv_h)), _p(_u64(inv_t)), K, _p(out))
    return out


def fri_leaves(evals):
    e = _u64(evals).reshape(-1)
    h = e.size // 6
    out = np.zeros((h, 32), np.uint8)
    lib().or_fri_leaves(_p(e), h, _p(out))
    return out


def logup_aux(main, desc, alpha_pows, z):
    """desc: dict of numpy arrays with the CSR descriptor fields."""
    main = _u64(main)
    n, m = main.shape
    u32 = lambda a: np.ascontiguousarray(a, np.uint32)
    d = {k: (u32(v) if v.dtype == np.uint32 else _u64(v)) if isinstance(v, np.ndarray) else v for k, v in desc.items()}
    W = d["num_committed"] + 1
    aux = np.zeros((n, 3 * W), np.uint64)
    L = np.zeros(3, np.uint64)
    keep = [d[k] for k in d if isinstance(d[k], np.ndarray)]
    rc = lib().or_logup_aux(_p(main), n, m, d["num_interactions"], _p(d["bus_ids"]), _p(d["elem_offsets"]),
                            _p(d["elem_alpha_idx"]), _p(d["elem_consts"]), _p(d["term_offsets"]),
                            _p(d["term_coefs"]), _p(d["term_cols"]), d["num_out_cols"], _p(d["out_col_offsets"]),
                            _p(d["out_col_interactions"]), _p(d["mult_consts"]), _p(d["mult_term_offsets"]),
                            _p(d["mult_term_coefs"]), _p(d["mult_term_cols"]), d["num_committed"],
                            _p(_u64(alpha_pows)), _p(_u64(z)), _p(aux), _p(L))
    del keep
    if rc:
        raise ZeroDivisionError("zero fingerprint")
    return aux, L
