"""Multi-table STARK prover over the B200 kernels.

Round structure follows IsStarkProver::multi_prove (crypto/stark/src/prover.rs:3299-4037)
and prove_rounds_2_to_4 (prover.rs:4433-4620):
  R1  per table: coset LDE of the main trace + row-pair Keccak commitment;
      roots absorbed in table order; LogUp challenges [z, alpha] sampled once;
      per-table transcript forks (clone + table index LE bytes when > 1 table).
  aux LogUp aux columns built and committed, root absorbed.
  R2  beta; coefficients beta^i (transition constraints first, then boundary);
      composition H over the LDE; degree-2 split into two parts, each
      extended to the LDE; parts committed, root absorbed.
  R3  z = sample_z_ood; trace columns opened at z and z*w, the parts at z^2, by
      barycentric interpolation over the trace coset; values absorbed.
  R4  gamma; DEEP codeword; FRI commit (fri/mod.rs:27-151) with the terminal
      polynomial; grinding nonce (grinding.rs); query indexes
      sample_u64(lde/2); openings with Merkle paths.
Every heavy step is a C-ABI call into libstarkgpu (the GPU backend below);
the driver only moves challenges and small host values. The same driver runs
over any backend with the same interface.

Differences from the reference protocol, kept deliberately simple: every trace
column is opened at z*w (the reference prunes next-row openings to the columns
constraints read there), and the DEEP coefficients are successive powers of
gamma (parts first, then trace columns column-major over the two points).
"""
import ctypes as C
import math

import numpy as np

from . import field as F
from . import math_cuda as mc
from . import native
from .device import DeviceBuffer, backend as _backend
from .ir import device_program, lowered

P = F.P


class Options:
    def __init__(self, blowup=2, coset_offset=3, grinding=20, final_log_degree=5, queries=None, security=128):
        self.blowup = blowup
        self.coset_offset = coset_offset
        self.grinding = grinding
        self.final_log_degree = final_log_degree
        if queries is None:
            rate = 1.0 / blowup
            prox = 1.0 - math.sqrt(rate) - 1.0 / 300.0
            queries = int(math.ceil((security - grinding) / -math.log2(1.0 - prox)))
        self.queries = queries


def fri_layout(lde_log, blowup_log, k):
    """FriFoldLayout::new (fri/terminal.rs:45-55)."""
    terminal_log = min(blowup_log + k, lde_log)
    total = lde_log - terminal_log
    return {"total_folds": total, "num_committed": max(total - 1, 0), "terminal_len": 1 << terminal_log,
            "effective_k": terminal_log - blowup_log}


def _dft_int(a, w):
    """Radix-2 DFT over Python ints: out[i] = sum_j a[j] w^(ij) mod p."""
    n = len(a)
    if n == 1:
        return list(a)
    w2 = w * w % P
    ev, od = _dft_int(a[0::2], w2), _dft_int(a[1::2], w2)
    out = [0] * n
    t = 1
    h = n // 2
    for k in range(h):
        x = od[k] * t % P
        out[k] = (ev[k] + x) % P
        out[k + h] = (ev[k] - x) % P
        t = t * w % P
    return out


def terminal_coeffs(codeword_br, terminal_offset, eff_k):
    """coeffs_from_terminal_codeword (fri/terminal.rs:72-103): gather the
    size-2^k sub-coset from the bit-reversed codeword and interpolate it on
    the coset terminal_offset * <w^blowup>: c_i = o^-i / keep * sum_j v_j w^-ij."""
    ln = len(codeword_br)
    keep = 1 << eff_k
    blow = ln // keep
    lbits = ln.bit_length() - 1
    cw = np.asarray(codeword_br, np.uint64).reshape(-1, 3)
    sub = [[int(v) % P for v in cw[F.bitrev_int(mm * blow, lbits)]] for mm in range(keep)]
    winv = F.inv_int(F.root_of_unity(eff_k)) if keep > 1 else 1
    oinv = F.inv_int(terminal_offset)
    comps = [_dft_int([sub[j][c] for j in range(keep)], winv) for c in range(3)]
    out = []
    s = F.inv_int(keep)
    for i in range(keep):
        out.append(tuple(comps[c][i] * s % P for c in range(3)))
        s = s * oinv % P
    return out


# ====================================================================== GPU backend
class Mat:
    """A row-major device matrix: rows x cols u64."""

    def __init__(self, buf, rows, cols):
        self.buf, self.rows, self.cols = buf, rows, cols

    @property
    def ptr(self):
        return self.buf.ptr

    def __len__(self):
        return self.rows

    def free(self):
        self.buf.close()


class _Borrowed:
    """Device memory owned by a library handle; closing the view frees nothing."""

    def __init__(self, ptr):
        self.ptr = ptr

    def close(self):
        pass


class _Release:
    """Stream-ordered release of an sg_lde handle (LDE + tree) on a backend's stream."""

    def __init__(self, bk, handle):
        self.bk, self.h = bk, handle

    def __call__(self, bk=None):
        if self.h:
            b = bk or self.bk
            b.L.sg_lde_free_async(b.be.h, b.st, self.h)
            self.h = None


class Tree:
    def __init__(self, buf, leaves_len):
        self.buf, self.leaves_len = buf, leaves_len

    def free(self):
        self.buf.close()


_DOMAINS = {}
_DOMAIN_LOCK = __import__("threading").Lock()


class Domain:
    pass


def _build_domain(bk, log_n, B, g):
    """Set-up vectors of one evaluation domain, as backend matrices."""
    n = 1 << log_n
    N = n * B
    log_N = log_n + (B.bit_length() - 1)
    d = Domain()
    d.log_n, d.log_N, d.n, d.N = log_n, log_N, n, N
    d.weights = bk.upload(F.coset_weights(n, g).reshape(-1, 1))
    d.comp_weights = bk.upload(F.composition_weights(N // 2, g).reshape(-1, 1))
    gn = F.pow_int(g, n)
    wB = F.root_of_unity(B.bit_length() - 1)
    d.z_inv = bk.inv_base(np.array([(gn * pow(wB, k, P) - 1) % P for k in range(B)], np.uint64))
    pts_N = F.coset_points(log_N, g)
    d.z_inv_dev = bk.upload(d.z_inv.reshape(-1, 1))
    d.b_z_inv = bk.upload(bk.inv_base(F.sub(pts_N, np.uint64(1))).reshape(1, -1))  # 1/(x - 1)
    d.inv2x = bk.upload(bk.inv_base(F.add(pts_N[: N // 2], pts_N[: N // 2])).reshape(-1, 1))
    d.pts_N = bk.upload(pts_N.reshape(-1, 1))
    d.pts_n = bk.upload(F.coset_points(log_n, g).reshape(-1, 1))
    tw0 = bk.inv_base(pts_N[: N // 2][F.bitrev_indices(log_N - 1).astype(np.int64)])
    d.tw0 = bk.upload(tw0.reshape(-1, 1))
    return d


class GpuBackend:
    name = "gpu"
    native_rounds = True

    def __init__(self, be=None, stream=None):
        self.be = be or _backend()
        self.L = native.lib()
        self.st = stream

    def _alloc(self, rows, cols):
        return Mat(DeviceBuffer(max(8, 8 * rows * cols), self.be, self.st), rows, cols)

    def transcript(self, label):
        return mc.Transcript(label)

    def upload(self, arr):
        a = np.ascontiguousarray(arr, np.uint64)
        if a.ndim == 1:
            a = a.reshape(-1, 1)
        m = self._alloc(a.shape[0], a.shape[1])
        m.buf.upload(a)
        return m

    def to_host(self, mat):
        return mat.buf.download(np.uint64, mat.rows * mat.cols).reshape(mat.rows, mat.cols)

    def lde(self, mat, blowup, weights):
        """Coset LDE; `weights` is a host array or a device Mat (cached domain weights)."""
        dw = weights if isinstance(weights, Mat) else None
        if dw is None:
            dw = self.upload(np.ascontiguousarray(weights, np.uint64).reshape(-1, 1))
        out = self._alloc(mat.rows * blowup, mat.cols)
        native.check(self.L.sg_coset_lde(self.be.h, self.st, mat.ptr, mat.rows, mat.cols, blowup, dw.ptr, out.ptr))
        if not isinstance(weights, Mat):
            dw.free()
        return out

    def domain(self, log_n, blowup, g):
        """Per-domain set-up vectors, built once per (size, blowup, offset) and
        shared by every table and proof on this context (the reference's
        domain_and_twiddles cache, prover.rs:514-580)."""
        key = (id(self.be), log_n, blowup, g)
        with _DOMAIN_LOCK:
            d = _DOMAINS.get(key)
            if d is None:
                saved, self.st = self.st, None  # build on the legacy stream, visible to all streams after sync
                try:
                    d = _build_domain(self, log_n, blowup, g)
                finally:
                    self.st = saved
                _DOMAINS[key] = d
            return d

    def commit(self, mat, rows_per_leaf=2, little_endian=False):
        nl = mat.rows // rows_per_leaf
        tree = Tree(DeviceBuffer((2 * nl - 1) * 32, self.be, self.st), nl)
        lay = native.LeafLayout(rows_per_leaf, 1 if little_endian else 0, 0, 0)
        leaves = tree.buf.ptr + (nl - 1) * 32
        native.check(self.L.sg_keccak_leaves(self.be.h, self.st, mat.ptr, mat.rows, mat.cols, C.byref(lay), leaves))
        root = (C.c_uint8 * 32)()
        native.check(self.L.sg_merkle_build(self.be.h, self.st, leaves, nl, tree.buf.ptr, root))
        return tree, bytes(root)

    def batch_commit(self, mats, blowup, weights, concurrency=8, fused=False):
        """Commit many main traces in one sg_batch_commit call (row-pair BE
        leaves), or with fused=True in one sg_batch_commit_fused call (every
        table's DFT passes in shared multi-table launches); returns [(lde Mat,
        Tree, root, release)] in table order, where release() returns the LDE
        and tree memory on this backend's stream."""
        n = len(mats)
        descs = (native.TableDesc * n)()
        for i, (m, w) in enumerate(zip(mats, weights)):
            descs[i] = native.TableDesc(m.ptr, 1, m.rows, m.cols, blowup, 1, w.ptr, native.LeafLayout(2, 0, 0, 0))
        handles = (C.c_void_p * n)()
        roots = (C.c_uint8 * (32 * n))()
        if fused:
            native.check(self.L.sg_batch_commit_fused(self.be.h, self.st, descs, n, concurrency, handles, roots))
        else:
            native.check(self.L.sg_batch_commit(self.be.h, self.st, descs, n, concurrency, handles, roots))
        out = []
        for i in range(n):
            info = native.LdeInfo()
            native.check(self.L.sg_lde_get_info(handles[i], C.byref(info)))
            h = handles[i]
            lde = Mat(_Borrowed(info.d_lde), info.lde_rows, info.row_u64)
            tree = Tree(_Borrowed(info.d_nodes), info.leaves_len)
            out.append((lde, tree, bytes(roots[32 * i:32 * i + 32]), _Release(self, h)))
        return out

    def tree_from_leaves(self, leaves_buf, nl):
        tree = Tree(DeviceBuffer((2 * nl - 1) * 32, self.be, self.st), nl)
        root = (C.c_uint8 * 32)()
        native.check(self.L.sg_merkle_build(self.be.h, self.st, leaves_buf.ptr, nl, tree.buf.ptr, root))
        return tree, bytes(root)

    @staticmethod
    def _logup_struct(desc, keep):
        def arr(name, dt):
            a = np.ascontiguousarray(desc[name], dt)
            keep[name] = a if a.size else np.zeros(1, dt)
            return keep[name].ctypes.data

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

    def prove_table_native(self, air, lowered, trace_mat, main_lde, main_tree, t, challenges, alpha_pows, opts):
        """Rounds 2-4 of one table in one library call (sg_prove_table); the
        same proof fields, in the same format, as prove_table's step-by-step path."""
        keep = {}
        B, g = opts.blowup, opts.coset_offset
        dom = self.domain(air.log_n, B, g)
        ld = self._logup_struct(air.logup_descriptor(), keep)
        kp = []
        prog = mc._program_struct(lowered, kp)
        nb = len(air.boundary)
        bcol = np.array([b[0] for b in air.boundary] or [0], np.uint64)
        bis = np.array([1 if b[1] else 0 for b in air.boundary] or [0], np.uint64)
        bval = np.zeros(3 * max(nb, 1), np.uint64)
        ch = np.array([challenges[0], challenges[1]], np.uint64).reshape(-1)
        al = np.ascontiguousarray(alpha_pows, np.uint64).reshape(-1)
        j = native.TableJob(trace_mat.ptr, main_lde.ptr, main_tree.buf.ptr, main_tree.leaves_len, air.n, air.width,
                            B, g, dom.weights.ptr, dom.comp_weights.ptr, dom.z_inv_dev.ptr, dom.b_z_inv.ptr,
                            dom.inv2x.ptr, dom.pts_n.ptr, dom.pts_N.ptr, dom.tw0.ptr, C.addressof(ld),
                            C.addressof(prog), nb, bcol.ctypes.data, bis.ctypes.data, bval.ctypes.data,
                            ch.ctypes.data, al.ctypes.data, len(alpha_pows), opts.queries, opts.grinding,
                            opts.final_log_degree)
        shp = native.ProofShape()
        native.check(self.L.sg_table_proof_shape(C.byref(j), C.byref(shp)))
        A, Q, D, Fl = shp.aux_cols, opts.queries, shp.depth, shp.fri_layers
        W = air.width + A
        u8, u64 = np.uint8, np.uint64
        buf = {"aux_root": np.zeros(32, u8), "comp_root": np.zeros(32, u8), "table_contribution": np.zeros(3, u64),
               "trace_ood": np.zeros((2, W, 3), u64), "parts_ood": np.zeros((2, 3), u64),
               "fri_roots": np.zeros((max(Fl, 1), 32), u8), "fri_final": np.zeros((shp.terminal_coeffs, 3), u64),
               "nonce": np.zeros(1, u64), "iotas": np.zeros(max(Q, 1), u64),
               "open_main": np.zeros((2 * Q, air.width), u64), "open_aux": np.zeros((2 * Q, 3 * A), u64),
               "open_parts": np.zeros((2 * Q, 6), u64), "path_main": np.zeros((Q, D, 32), u8),
               "path_aux": np.zeros((Q, D, 32), u8), "path_parts": np.zeros((Q, D, 32), u8),
               "fri_open": np.zeros((max(Fl, 1), 2 * Q, 3), u64), "fri_paths": np.zeros(max(1, shp.fri_path_bytes), u8)}
        o = native.TableProof(*[buf[k].ctypes.data for k in (
            "aux_root", "comp_root", "table_contribution", "trace_ood", "parts_ood", "fri_roots", "fri_final", "nonce",
            "iotas", "open_main", "open_aux", "open_parts", "path_main", "path_aux", "path_parts", "fri_open",
            "fri_paths")])
        native.check(self.L.sg_prove_table(self.be.h, self.st, t.h, C.byref(j), C.byref(o)))
        fri_paths, off = [], 0
        for li in range(Fl):
            d = D - 1 - li
            fri_paths.append(buf["fri_paths"][off:off + Q * d * 32].reshape(Q, d, 32))
            off += Q * d * 32
        return {"aux_root": buf["aux_root"].tobytes(), "table_contribution": tuple(buf["table_contribution"].tolist()),
                "comp_root": buf["comp_root"].tobytes(),
                "trace_ood": [[tuple(v) for v in row] for row in buf["trace_ood"].tolist()],
                "parts_ood": [tuple(v) for v in buf["parts_ood"].tolist()],
                "fri_roots": [buf["fri_roots"][i].tobytes() for i in range(Fl)],
                "fri_final_coeffs": [tuple(v) for v in buf["fri_final"].tolist()], "nonce": int(buf["nonce"][0]),
                "iotas": buf["iotas"][:Q].tolist(), "open_main": buf["open_main"], "open_aux": buf["open_aux"],
                "open_parts": buf["open_parts"], "path_main": buf["path_main"], "path_aux": buf["path_aux"],
                "path_parts": buf["path_parts"], "fri_open": [buf["fri_open"][i] for i in range(Fl)],
                "fri_paths": fri_paths}

    def logup_aux(self, trace, desc, alpha_pows, z):
        keep = {}

        def arr(name, dt):
            a = np.ascontiguousarray(desc[name], dt)
            keep[name] = a if a.size else np.zeros(1, dt)
            return keep[name].ctypes.data

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
        W = desc["num_committed"] + 1
        al = np.ascontiguousarray(alpha_pows, np.uint64).reshape(-1)
        zz = np.array(z, np.uint64)
        aux = self._alloc(trace.rows, 3 * W)
        L = np.zeros(3, np.uint64)
        native.check(self.L.sg_logup_aux(self.be.h, self.st, trace.ptr, trace.rows, trace.cols, C.byref(d),
                                         al.ctypes.data, al.size // 3, zz.ctypes.data, aux.ptr, L.ctypes.data))
        return aux, F.f3(L)

    def composition(self, program, lowered, main, aux, rap, alpha_pows, offset, next_step, beta, z_inv, boundary,
                    b_z_inv):
        keep = []
        prog = mc._program_struct(lowered, keep)
        c = native.Composition()
        bt = np.ascontiguousarray(beta, np.uint64).reshape(-1)
        dz = DeviceBuffer.from_host(np.ascontiguousarray(z_inv, np.uint64), self.be, self.st)
        c.beta_trans, c.d_z_inv, c.z_len = bt.ctypes.data, dz.ptr, len(z_inv)
        c.num_boundary = len(boundary)
        cols = np.array([b[0] for b in boundary] or [0], np.uint64)
        isa = np.array([1 if b[1] else 0 for b in boundary] or [0], np.uint64)
        val = np.array([b[2] for b in boundary] or [(0, 0, 0)], np.uint64).reshape(-1)
        bb = np.array([b[3] for b in boundary] or [(0, 0, 0)], np.uint64).reshape(-1)
        c.b_col, c.b_is_aux, c.b_value, c.b_beta = cols.ctypes.data, isa.ctypes.data, val.ctypes.data, bb.ctypes.data
        c.d_b_z_inv = b_z_inv.ptr if b_z_inv is not None else None
        rap_a = np.ascontiguousarray(rap, np.uint64).reshape(-1)
        al = np.ascontiguousarray(alpha_pows, np.uint64).reshape(-1)
        off = np.array(offset, np.uint64)
        out = self._alloc(main.rows, 3)
        native.check(self.L.sg_eval_constraints(self.be.h, self.st, C.byref(prog), rap_a.ctypes.data, rap_a.size // 3,
                                                al.ctypes.data, al.size // 3, off.ctypes.data, main.ptr, main.cols,
                                                aux.ptr, aux.cols // 3, main.rows, next_step, C.byref(c), out.ptr))
        dz.close()
        return out

    def decompose(self, h, inv2x):
        out = self._alloc(h.rows // 2, 6)
        native.check(self.L.sg_decompose_d2(self.be.h, self.st, h.ptr, h.rows, inv2x.ptr, out.ptr))
        return out

    def inv_base(self, x):
        """Device vector of base inverses 1/x_i (x host)."""
        x = np.ascontiguousarray(x, np.uint64)
        e = np.zeros((x.size, 3), np.uint64)
        e[:, 0] = x
        m = self.upload(e)
        zf = C.c_int(0)
        native.check(self.L.sg_batch_inverse_ext3(self.be.h, self.st, m.ptr, x.size, m.ptr, C.byref(zf)))
        if zf.value:
            raise ZeroDivisionError("inverse of zero")
        h = self.to_host(m)[:, 0].copy()
        m.free()
        return h

    def inv_denoms(self, pts, zs, x_minus_z):
        z = np.array(zs, np.uint64).reshape(-1)
        k = len(zs)
        out = self._alloc(pts.rows * k, 3)
        zf = C.c_int(0)
        native.check(self.L.sg_inv_denoms_ext3(self.be.h, self.st, pts.ptr, pts.rows, z.ctypes.data, k,
                                               1 if x_minus_z else 0, out.ptr, C.byref(zf)))
        if zf.value:
            raise ZeroDivisionError("zero denominator")
        return out

    def bary(self, mat, stride, ext3, cols, pts, invd, n, k, k0=0):
        """Sums over the k denominator rows k0 .. k0+k-1 of `invd`."""
        out = DeviceBuffer(24 * k * cols, self.be, self.st)
        native.check(self.L.sg_barycentric_sums(self.be.h, self.st, mat.ptr, mat.cols, stride, 1 if ext3 else 0, cols,
                                                pts.ptr, invd.ptr + 24 * k0 * n, n, k, out.ptr))
        r = out.download(np.uint64, 3 * k * cols).reshape(k, cols, 3)
        out.close()
        return r

    def deep(self, main, aux, parts, h_ood, trace_ood, gh, gt, inv_h, inv_t, k):
        out = self._alloc(main.rows, 3)
        arrs = [np.ascontiguousarray(np.array(x, np.uint64).reshape(-1)) for x in (h_ood, trace_ood, gh, gt)]
        native.check(self.L.sg_deep_composition(self.be.h, self.st, main.ptr, main.cols, aux.ptr, aux.cols // 3,
                                                parts.ptr, parts.cols // 3, main.rows, arrs[0].ctypes.data,
                                                arrs[1].ctypes.data, arrs[2].ctypes.data, arrs[3].ctypes.data, k,
                                                inv_h.ptr, inv_t.ptr, 1, out.ptr))
        return out

    def fri_fold(self, ev, tw, zeta, with_leaves):
        h = ev.rows // 2
        out = self._alloc(h, 3)
        twn = self._alloc(max(1, h // 2), 1)
        leaves = DeviceBuffer(32 * max(1, h // 2), self.be, self.st) if with_leaves else None
        z = np.array(zeta, np.uint64)
        native.check(self.L.sg_fri_fold_layer(self.be.h, self.st, ev.ptr, h, tw.ptr, z.ctypes.data, out.ptr, twn.ptr,
                                              leaves.ptr if leaves else None))
        return out, twn, leaves

    def gather(self, mat, rows):
        r = np.ascontiguousarray(rows, np.uint32)
        dr = DeviceBuffer.from_host(r, self.be, self.st)
        out = DeviceBuffer(8 * max(1, r.size * mat.cols), self.be, self.st)
        native.check(self.L.sg_gather_rows(self.be.h, self.st, mat.ptr, mat.cols, mat.rows, 0, mat.cols, dr.ptr,
                                           r.size, out.ptr))
        h = out.download(np.uint64, r.size * mat.cols).reshape(r.size, mat.cols)
        dr.close()
        out.close()
        return h

    def paths(self, tree, positions):
        pos = np.ascontiguousarray(positions, np.uint32)
        depth = tree.leaves_len.bit_length() - 1
        dp = DeviceBuffer.from_host(pos, self.be, self.st)
        out = DeviceBuffer(max(32, pos.size * depth * 32), self.be, self.st)
        native.check(self.L.sg_merkle_gather_paths(self.be.h, self.st, tree.buf.ptr, tree.leaves_len, dp.ptr,
                                                   pos.size, out.ptr))
        h = out.download(np.uint8, pos.size * depth * 32).reshape(pos.size, depth, 32)
        dp.close()
        out.close()
        return h

    def open_many(self, reqs):
        """Query openings in one round trip: reqs is a list of ("rows", Mat,
        rows) and ("paths", Tree, positions); one upload of all indices, one
        kernel per request into one output buffer, one download."""
        idx = [np.ascontiguousarray(r[2], np.uint32) for r in reqs]
        offs, sizes, tot_idx = [], [], 0
        for (kind, obj, _), ix in zip(reqs, idx):
            offs.append(tot_idx)
            tot_idx += ix.size
            sizes.append(ix.size * (obj.cols * 8 if kind == "rows" else (obj.leaves_len.bit_length() - 1) * 32))
        allidx = np.concatenate(idx) if idx else np.zeros(1, np.uint32)
        dix = DeviceBuffer.from_host(allidx if allidx.size else np.zeros(1, np.uint32), self.be, self.st)
        ob = [0]
        for sz in sizes:
            ob.append(ob[-1] + (sz + 7) // 8 * 8)
        out = DeviceBuffer(max(8, ob[-1]), self.be, self.st)
        for (kind, obj, _), ix, off, o in zip(reqs, idx, offs, ob):
            if ix.size == 0:
                continue
            if kind == "rows":
                native.check(self.L.sg_gather_rows(self.be.h, self.st, obj.ptr, obj.cols, obj.rows, 0, obj.cols,
                                                   dix.ptr + 4 * off, ix.size, out.ptr + o))
            else:
                native.check(self.L.sg_merkle_gather_paths(self.be.h, self.st, obj.buf.ptr, obj.leaves_len,
                                                           dix.ptr + 4 * off, ix.size, out.ptr + o))
        host = out.download(np.uint8, ob[-1]) if ob[-1] else np.zeros(0, np.uint8)
        dix.close()
        out.close()
        res = []
        for (kind, obj, _), ix, o, sz in zip(reqs, idx, ob, sizes):
            b = host[o:o + sz]
            if kind == "rows":
                res.append(b.view(np.uint64).reshape(ix.size, obj.cols))
            else:
                res.append(b.reshape(ix.size, obj.leaves_len.bit_length() - 1, 32))
        return res

    def grind(self, state, g):
        inner = mc.keccak256(bytes([0x01, 0x23, 0x45, 0x67, 0x89, 0xAB, 0xCD, 0xED]) + bytes(state) + bytes([g]))
        return mc.generate_nonce_gpu(mc.inner_hash_lanes(inner), g, self.be)

    def free(self, *objs):
        for o in objs:
            if o is not None:
                o.free()


# ====================================================================== the protocol
def _u64le(i):
    return int(i).to_bytes(8, "little")


def _u64be(i):
    return int(i).to_bytes(8, "big")


def _ood_scale(z, n, g):
    """(z^n - g^n) * (1/n) * g^-n  (interpolate_coset_eval_ext_with_g_n_inv, polynomial.rs:207-235)."""
    gn = F.pow_int(g, n)
    s = F.inv_int(n) * F.inv_int(gn) % P
    return F.f3scale(F.f3sub(F.f3pow(z, n), (gn, 0, 0)), s)


def prove_table(bk, air, lowered, trace_mat, main_lde, main_tree, t, challenges, alpha_pows, opts, native_rounds=None):
    """Aux build + rounds 2-4 for one table (prover.rs:3603-3977, 4433-4620).
    On the GPU backend the whole sequence runs as one library call
    (sg_prove_table) unless native_rounds is False, which drives the same steps
    one backend operation at a time from here."""
    if native_rounds is None:
        native_rounds = getattr(bk, "native_rounds", False)
    if native_rounds:
        return bk.prove_table_native(air, lowered, trace_mat, main_lde, main_tree, t, challenges, alpha_pows, opts)
    n, N = air.n, air.n * opts.blowup
    B, g = opts.blowup, opts.coset_offset
    log_n, log_N = air.log_n, air.log_n + (B.bit_length() - 1)
    dom = bk.domain(log_n, B, g)
    proof = {}
    # ---- aux
    aux, Lc = bk.logup_aux(trace_mat, air.logup_descriptor(), alpha_pows, challenges[0])
    aux_lde = bk.lde(aux, B, dom.weights)
    bk.free(aux)
    aux_tree, aux_root = bk.commit(aux_lde)
    t.append_bytes(aux_root)
    proof["aux_root"] = aux_root
    proof["table_contribution"] = Lc
    # ---- R2
    beta = F.f3(t.sample_ext3())
    nroots = lowered.get("num_roots", len(lowered["roots"]))
    ncons = nroots + len(air.boundary)
    coefs = [(1, 0, 0)]
    for _ in range(ncons - 1):
        coefs.append(F.f3mul(coefs[-1], beta))
    beta_t, beta_b = coefs[:nroots], coefs[nroots:]
    offset = F.f3scale(Lc, F.inv_int(n))
    boundary = [(col, is_aux, (0, 0, 0), beta_b[i]) for i, (col, is_aux, _row) in enumerate(air.boundary)]
    H = bk.composition(air.program, lowered, main_lde, aux_lde, [challenges[0], challenges[1]], alpha_pows, offset, B,
                       beta_t, dom.z_inv, boundary, dom.b_z_inv)
    halves = bk.decompose(H, dom.inv2x)
    bk.free(H)
    parts_lde = bk.lde(halves, 2, dom.comp_weights)
    bk.free(halves)
    comp_tree, comp_root = bk.commit(parts_lde)
    t.append_bytes(comp_root)
    proof["comp_root"] = comp_root
    # ---- R3
    z = F.f3(t.sample_z_ood(n, N, g))
    wn = F.root_of_unity(log_n)
    zw = F.f3scale(z, wn)
    z2 = F.f3mul(z, z)
    invd = bk.inv_denoms(dom.pts_n, [z, zw, z2], False)
    # trace columns at z and z*w (denominator rows 0, 1); parts at z^2 (row 2)
    S_main = bk.bary(main_lde, B, False, air.width, dom.pts_n, invd, n, 2)
    S_aux = bk.bary(aux_lde, B, True, air.aux_width, dom.pts_n, invd, n, 2)
    S_parts = bk.bary(parts_lde, B, True, 2, dom.pts_n, invd, n, 1, k0=2)
    bk.free(invd)
    sc = np.array([_ood_scale(p, n, g) for p in (z, zw, z2)], np.uint64)
    tood = np.concatenate([F.f3mul_vec(S_main[:2], sc[:2, None, :]), F.f3mul_vec(S_aux[:2], sc[:2, None, :])],
                          axis=1)  # (2 points, main + aux columns, 3)
    pood = F.f3mul_vec(S_parts[0], sc[2][None, :])  # (2 parts, 3)
    t.append_ext3_many(tood)
    t.append_ext3_many(pood)
    trace_ood = [[tuple(v) for v in row] for row in tood.tolist()]
    parts_ood = [tuple(v) for v in pood.tolist()]
    proof["trace_ood"] = trace_ood
    proof["parts_ood"] = parts_ood
    # ---- R4: DEEP
    gamma = F.f3(t.sample_ext3())
    ncols = air.width + air.aux_width
    gp = [(1, 0, 0)]
    for _ in range(2 + 2 * ncols - 1):
        gp.append(F.f3mul(gp[-1], gamma))
    gh, gt = gp[:2], gp[2:]
    trace_ood_jk = tood.transpose(1, 0, 2).reshape(-1, 3)  # index j*2 + k
    inv_h = bk.inv_denoms(dom.pts_N, [z2], True)
    inv_t = bk.inv_denoms(dom.pts_N, [z, zw], True)
    deep = bk.deep(main_lde, aux_lde, parts_lde, parts_ood, trace_ood_jk, gh, gt, inv_h, inv_t, 2)
    bk.free(inv_h, inv_t)
    # ---- FRI commit (fri/mod.rs:27-151)
    lay = fri_layout(log_N, B.bit_length() - 1, opts.final_log_degree)
    tw, own_tw = dom.tw0, False
    ev = deep
    layers, fri_roots = [], []
    for _ in range(lay["num_committed"]):
        zeta = F.f3(t.sample_ext3())
        ev2, tw2, leaves = bk.fri_fold(ev, tw, zeta, True)
        tree, root = bk.tree_from_leaves(leaves, len(ev2) // 2)
        bk.free(leaves)
        if own_tw:
            bk.free(tw)
        layers.append((ev2, tree))
        fri_roots.append(root)
        t.append_bytes(root)
        ev, tw, own_tw = ev2, tw2, True
    if lay["total_folds"] > 0:
        zeta = F.f3(t.sample_ext3())
        evf, twf, _ = bk.fri_fold(ev, tw, zeta, False)
        bk.free(twf)
        final = bk.to_host(evf)
        bk.free(evf)
    else:
        final = bk.to_host(ev)
    if own_tw:
        bk.free(tw)
    term_off = F.pow_int(g, 1 << lay["total_folds"])
    coeffs = terminal_coeffs(final, term_off, lay["effective_k"])
    t.append_ext3_many(coeffs)
    proof["fri_roots"] = fri_roots
    proof["fri_final_coeffs"] = coeffs
    # ---- grinding + queries
    nonce = bk.grind(t.state(), opts.grinding) if opts.grinding else 0
    if opts.grinding:
        t.append_bytes(_u64be(nonce))
    proof["nonce"] = nonce
    iotas = [t.sample_u64(N // 2) for _ in range(opts.queries)]
    proof["iotas"] = iotas
    # ---- openings: leaf iota of each trace-side tree covers rows br(2i), br(2i+1)
    it = np.asarray(iotas, np.uint64)
    rows = F.bitrev_vec(np.stack([2 * it, 2 * it + 1], axis=1).reshape(-1), log_N).tolist()
    reqs = [("rows", main_lde, rows), ("rows", aux_lde, rows), ("rows", parts_lde, rows),
            ("paths", main_tree, iotas), ("paths", aux_tree, iotas), ("paths", comp_tree, iotas)]
    for li, (lev, ltree) in enumerate(layers):
        leaf = (it >> np.uint64(li + 1)).tolist()
        rr = np.stack([2 * np.asarray(leaf, np.uint64), 2 * np.asarray(leaf, np.uint64) + 1], axis=1).reshape(-1)
        reqs += [("rows", lev, rr.tolist()), ("paths", ltree, leaf)]
    opened = bk.open_many(reqs)
    (proof["open_main"], proof["open_aux"], proof["open_parts"], proof["path_main"], proof["path_aux"],
     proof["path_parts"]) = opened[:6]
    fri_open = opened[6::2]
    fri_paths = opened[7::2]
    proof["fri_open"] = fri_open
    proof["fri_paths"] = fri_paths
    bk.free(deep, aux_lde, parts_lde, aux_tree, comp_tree)
    for lev, ltree in layers:
        bk.free(lev, ltree)
    return proof


def _gen_trace(bk, air, source):
    """`source` is a host array, an int seed for the counter-based synthetic
    trace (generated on the device by the GPU backend, on the host otherwise),
    or a table source with device_trace(bk, air) (the GPU backend writes the
    table on the device) and host_trace(air)."""
    if hasattr(source, "device_trace"):
        return source.device_trace(bk, air) if isinstance(bk, GpuBackend) else bk.upload(source.host_trace(air))
    if isinstance(source, (int, np.integer)):
        if isinstance(bk, GpuBackend):
            m = bk._alloc(air.n, air.width)
            native.check(bk.L.sg_synth_trace(bk.be.h, bk.st, m.ptr, air.n, air.width, int(source), air.k))
            return m
        return bk.upload(air.trace(int(source)))
    return bk.upload(source)


def multi_prove(airs, traces, opts=None, bk=None, label=b"lambda_vm_b200/synthetic-multi-table"):
    """Prove all tables of one multi-table statement, one table after another
    (the plain form); returns the proof dict. `traces` holds host arrays or
    int seeds of counter-based synthetic traces."""
    opts = opts or Options()
    bk = bk or GpuBackend()
    t = bk.transcript(label)
    B, g = opts.blowup, opts.coset_offset
    tabs = []
    for air, tr in zip(airs, traces):
        tm = _gen_trace(bk, air, tr)
        lde = bk.lde(tm, B, bk.domain(air.log_n, B, g).weights)
        tree, root = bk.commit(lde)
        tabs.append((air, tm, lde, tree, root))
    for _, _, _, _, root in tabs:
        t.append_bytes(root)
    challenges = [F.f3(t.sample_ext3()), F.f3(t.sample_ext3())]  # [z, alpha] (lookup.rs:1315-1322)
    alpha = challenges[1]
    max_alpha = max(a.max_alpha for a in airs)
    alpha_pows = [(1, 0, 0)]
    for _ in range(max_alpha - 1):
        alpha_pows.append(F.f3mul(alpha_pows[-1], alpha))
    forks = []
    for i in range(len(tabs)):
        ti = t.clone()
        if len(tabs) > 1:
            ti.append_bytes(_u64le(i))
        forks.append(ti)
    proofs = []
    for i, (air, tm, lde, tree, root) in enumerate(tabs):
        p = prove_table(bk, air, lowered(device_program(air)), tm, lde, tree, forks[i], challenges, alpha_pows, opts)
        p["main_root"] = root
        proofs.append(p)
        bk.free(tm, lde, tree)
    return {"tables": proofs, "challenges": challenges}
