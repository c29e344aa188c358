"""CPU oracle backend for the multi-table prover — TEST INFRASTRUCTURE ONLY.

Implements the same operations as lambda_vm_b200.stark.GpuBackend with the C
oracle (oracle/oracle.c) and plain Python, so a proof produced through the
GPU backend can be compared field for field with one produced entirely on the
CPU. Constraint evaluation walks the UNLOWERED IR program row by row
(constraint_ir/interp.rs semantics), independent of the device lowering.
"""
import numpy as np

import oracle as O

P = O.P


def _c(a):
    return O.canon_array(a)


def _e(x):
    return [int(v) for v in x]


def _f3add(a, b):
    return [O.gl_add(a[i], b[i]) for i in range(3)]


def _f3sub(a, b):
    return [O.gl_sub(a[i], b[i]) for i in range(3)]


def _f3mul(a, b):
    return _e(O.fp3_mul(np.array(a, np.uint64), np.array(b, np.uint64)))


def eval_program_row(prog, row, main, aux, rap, alpha, offset, next_step):
    rows = main.shape[0]
    v = []
    for nd in prog["nodes"]:
        k = nd[0]
        if k == "var":
            _, is_main, off, col = nd
            r = (row + off * next_step) % rows
            v.append([int(main[r, col]), 0, 0] if is_main else _e(aux[r, 3 * col:3 * col + 3]))
        elif k == "cb":
            v.append([prog["base_consts"][nd[1]], 0, 0])
        elif k == "ce":
            v.append(list(prog["ext_consts"][nd[1]]))
        elif k == "rap":
            v.append(_e(rap[nd[1]]))
        elif k == "alpha":
            v.append(_e(alpha[nd[1]]))
        elif k == "off":
            v.append(_e(offset))
        elif k == "add":
            v.append(_f3add(v[nd[1]], v[nd[2]]))
        elif k == "sub":
            v.append(_f3sub(v[nd[1]], v[nd[2]]))
        elif k == "mul":
            v.append(_f3mul(v[nd[1]], v[nd[2]]))
        elif k == "neg":
            v.append([O.gl_neg(x) for x in v[nd[1]]])
        else:
            v.append(list(v[nd[1]]))
    return [v[r] for r in prog["roots"]]


class OracleBackend:
    name = "oracle"

    def transcript(self, label):
        return O.Transcript(label)

    def domain(self, log_n, blowup, g):
        """Domain set-up vectors computed with the oracle (no cache)."""
        class D:
            pass
        n, N = 1 << log_n, (1 << log_n) * blowup
        log_N = N.bit_length() - 1
        d = D()
        d.weights = O.canon_array(O.coset_weights(n, g))
        # composition weights g^-j / (N/2)
        ginv, hinv = O.gl_inv(g), O.gl_inv(N // 2)
        d.comp_weights = np.array([O.canonical(O.gl_mul(hinv, O.gl_pow(ginv, j))) for j in range(N // 2)], np.uint64)
        wN, wn = O.root_of_unity(log_N), O.root_of_unity(log_n)
        pts_N = np.array([O.canonical(O.gl_mul(g, O.gl_pow(wN, i))) for i in range(N)], np.uint64)
        gn, wB = O.gl_pow(g, n), O.root_of_unity(blowup.bit_length() - 1)
        d.z_inv = self.inv_base(np.array([O.gl_sub(O.gl_mul(gn, O.gl_pow(wB, k)), 1) for k in range(blowup)],
                                         np.uint64))
        d.b_z_inv = self.inv_base(np.array([O.gl_sub(int(x), 1) for x in pts_N], np.uint64)).reshape(1, -1)
        d.inv2x = self.inv_base(np.array([O.gl_add(int(x), int(x)) for x in pts_N[: N // 2]], np.uint64)).reshape(-1, 1)
        d.pts_N = pts_N.reshape(-1, 1)
        d.pts_n = np.array([O.canonical(O.gl_mul(g, O.gl_pow(wn, i))) for i in range(n)], np.uint64).reshape(-1, 1)
        br = [int(format(i, f"0{log_N - 1}b")[::-1], 2) if log_N > 1 else 0 for i in range(N // 2)]
        d.tw0 = self.inv_base(pts_N[: N // 2][br]).reshape(-1, 1)
        return d

    def upload(self, arr):
        a = np.ascontiguousarray(arr, np.uint64)
        return a.reshape(-1, 1).copy() if a.ndim == 1 else a.copy()

    def to_host(self, m):
        return m

    def lde(self, mat, blowup, weights):
        return _c(O.coset_lde_row_major(mat, blowup, np.asarray(weights).reshape(-1)))

    def commit(self, mat, rows_per_leaf=2, little_endian=False):
        nodes = O.merkle_nodes(O.leaves_row_major(mat, rows_per_leaf, little_endian))
        return nodes, nodes[0].tobytes()

    def tree_from_leaves(self, leaves, nl):
        nodes = O.merkle_nodes(leaves)
        return nodes, nodes[0].tobytes()

    def logup_aux(self, trace, desc, alpha_pows, z):
        aux, L = O.logup_aux(trace, desc, np.array(alpha_pows, np.uint64), np.array(z, np.uint64))
        return _c(aux), tuple(int(x) for x in _c(L))

    def composition(self, program, lowered, main, aux, rap, alpha_pows, offset, next_step, beta, z_inv, boundary,
                    b_z_inv):
        prog = program
        rows = main.shape[0]
        rap, alpha = np.array(rap, np.uint64), np.array(alpha_pows, np.uint64)
        out = np.zeros((rows, 3), np.uint64)
        for row in range(rows):
            vals = eval_program_row(prog, row, main, aux, rap, alpha, offset, next_step)
            s = [0, 0, 0]
            for c, cv in enumerate(vals):
                s = _f3add(s, _f3mul(list(beta[c]), cv))
            zi = int(z_inv[row % len(z_inv)])
            h = [O.gl_mul(x, zi) for x in s]
            for b, (col, is_aux, value, bb) in enumerate(boundary):
                cell = _e(aux[row, 3 * col:3 * col + 3]) if is_aux else [int(main[row, col]), 0, 0]
                zb = [O.gl_mul(x, int(b_z_inv[b, row])) for x in bb]
                h = _f3add(h, _f3mul(zb, _f3sub(cell, list(value))))
            out[row] = [O.canonical(x) for x in h]
        return out

    def decompose(self, h, inv2x):
        n = h.shape[0] // 2
        two_inv = (P + 1) // 2
        out = np.zeros((n, 6), np.uint64)
        for i in range(n):
            x, y = _e(h[i]), _e(h[i + n])
            w = int(inv2x[i, 0])
            out[i, :3] = [O.canonical(O.gl_mul(O.gl_add(x[k], y[k]), two_inv)) for k in range(3)]
            out[i, 3:] = [O.canonical(O.gl_mul(O.gl_sub(x[k], y[k]), w)) for k in range(3)]
        return out

    def inv_base(self, x):
        x = np.ascontiguousarray(x, np.uint64)
        e = np.zeros((x.size, 3), np.uint64)
        e[:, 0] = x
        return _c(O.fp3_batch_inverse(e.reshape(-1)).reshape(-1, 3)[:, 0])

    def inv_denoms(self, pts, zs, x_minus_z):
        return _c(O.inv_denoms(pts.reshape(-1), np.array(zs, np.uint64), x_minus_z)).reshape(-1, 3)

    def bary(self, mat, stride, ext3, cols, pts, invd, n, k, k0=0):
        sel = np.ascontiguousarray(invd.reshape(-1, 3)[k0 * n:(k0 + k) * n])
        return _c(O.barycentric_sums(mat, stride, ext3, cols, pts.reshape(-1), sel.reshape(-1), n, k)).reshape(k, cols, 3)

    def deep(self, main, aux, parts, h_ood, trace_ood, gh, gt, inv_h, inv_t, k):
        nat = _c(O.deep(main, aux, parts, np.array(h_ood, np.uint64), np.array(trace_ood, np.uint64),
                        np.array(gh, np.uint64), np.array(gt, np.uint64), inv_h.reshape(-1), inv_t.reshape(-1),
                        k)).reshape(-1, 3)
        rows = nat.shape[0]
        lg = rows.bit_length() - 1
        out = np.zeros_like(nat)
        for i in range(rows):
            out[int(format(i, f"0{lg}b")[::-1], 2) if lg else 0] = nat[i]
        return out

    def fri_fold(self, ev, tw, zeta, with_leaves):
        out = _c(O.fri_fold(ev.reshape(-1), tw.reshape(-1), np.array(zeta, np.uint64))).reshape(-1, 3)
        t = tw.reshape(-1)
        twn = np.array([O.canonical(O.gl_mul(int(t[2 * j]), int(t[2 * j]))) for j in range(out.shape[0] // 2)],
                       np.uint64).reshape(-1, 1)
        leaves = O.fri_leaves(out) if with_leaves else None
        return out, twn, leaves

    def gather(self, mat, rows):
        return mat[np.array(rows, np.int64)].copy()

    def paths(self, tree, positions):
        return np.stack([O.merkle_path(tree, int(p)) for p in positions])

    def open_many(self, reqs):
        return [self.gather(obj, ix) if kind == "rows" else self.paths(obj, ix) for kind, obj, ix in reqs]

    def grind(self, state, g):
        return O.grind(bytes(state), g)

    def free(self, *objs):
        pass
