"""GPU parity for the round 2-4 kernels against the CPU oracle (bit-exact on
canonical values): batch inversion and denominators (inverse.rs tests
batch_inverse.rs, compute_and_invert_denoms.rs), barycentric sums
(barycentric_multi.rs), DEEP (deep.rs), FRI fold + layer leaves
(fri_layer_tree.rs), LogUp aux (lookup.rs term / accumulated columns)."""
import numpy as np
import pytest

import oracle as O
from lambda_vm_b200 import math_cuda as mc

pytestmark = pytest.mark.gpu
P = O.P


def rf(rng, shape):
    x = rng.integers(0, 2**64, size=shape, dtype=np.uint64)
    return np.where(x >= np.uint64(P), x - np.uint64(P), x)


@pytest.mark.parametrize("n", [1, 3, 4, 31, 32, 127, 128, 129, 1000, 4096, 100003])
def test_batch_inverse_matches_oracle(be, n):
    rng = np.random.default_rng(n)
    a = rf(rng, (n, 3)).reshape(-1)
    got = mc.batch_inverse_ext3(a, be)
    assert (got == O.canon_array(O.fp3_batch_inverse(a))).all()


def test_batch_inverse_reports_zero(be):
    a = np.ones(3 * 40, np.uint64)
    a[3 * 17:3 * 18] = 0
    with pytest.raises(ZeroDivisionError):
        mc.batch_inverse_ext3(a, be)


@pytest.mark.parametrize("n,k,sign", [(1, 1, 0), (64, 2, 0), (1000, 3, 1), (4096, 8, 1), (50000, 2, 0),
                                      # a thread's chunk of 12 denominators wraps across several points
                                      (1, 8, 1), (5, 7, 0), (11, 3, 1)])
def test_inv_denoms_match_oracle(be, n, k, sign):
    rng = np.random.default_rng(n + k)
    x = rf(rng, (n,))
    z = rf(rng, (k, 3))
    got = mc.compute_and_invert_denoms_ext3(x, z, sign, be)
    assert (got == O.canon_array(O.inv_denoms(x, z, sign))).all()


@pytest.mark.parametrize("rows,ru,cols,ext3,stride,k", [
    (64, 5, 5, False, 1, 1), (256, 7, 7, False, 2, 3), (1024, 12, 4, True, 4, 2), (4096, 300, 300, False, 2, 8),
    (2048, 30, 10, True, 2, 5), (16384, 16, 16, False, 4, 2),
    # point counts that end inside a weight batch and inside a prefetch group
    (3000, 9, 9, False, 3, 2), (96, 9, 3, True, 1, 8), (1000, 600, 600, False, 1, 1)])
def test_barycentric_sums_match_oracle(be, rows, ru, cols, ext3, stride, k):
    rng = np.random.default_rng(rows + cols)
    data = rf(rng, (rows, ru))
    n = rows // stride
    pts = rf(rng, (n,))
    invd = rf(rng, (k * n * 3,))
    got = mc.barycentric_multi(data, stride, ext3, cols, pts, invd, n, k, be)
    want = O.canon_array(O.barycentric_sums(data, stride, ext3, cols, pts, invd, n, k))
    assert (got == want).all()


@pytest.mark.parametrize("rows,m,a,p,k", [(32, 3, 1, 1, 1), (256, 17, 2, 2, 2), (1024, 64, 5, 2, 3),
                                          (4096, 300, 0, 2, 2), (2048, 8, 40, 1, 8), (64, 1, 1, 1, 2),
                                          (128, 2, 1, 2, 2)])
def test_deep_matches_oracle(be, rows, m, a, p, k):
    rng = np.random.default_rng(rows + m + a)
    main = rf(rng, (rows, m))
    aux = rf(rng, (rows, 3 * a))
    parts = rf(rng, (rows, 3 * p))
    h_ood, gh = rf(rng, (3 * p,)), rf(rng, (3 * p,))
    t_ood, gt = rf(rng, (3 * (m + a) * k,)), rf(rng, (3 * (m + a) * k,))
    inv_h, inv_t = rf(rng, (3 * rows,)), rf(rng, (3 * k * rows,))
    want = O.canon_array(O.deep(main, aux if a else np.zeros((rows, 0), np.uint64),
                                parts, h_ood, t_ood, gh, gt, inv_h, inv_t, k)).reshape(rows, 3)
    got = mc.deep_composition_ext3(main, aux, parts, h_ood, t_ood, gh, gt, inv_h, inv_t, k, False, be).reshape(rows, 3)
    assert (got == want).all()
    gotb = mc.deep_composition_ext3(main, aux, parts, h_ood, t_ood, gh, gt, inv_h, inv_t, k, True, be).reshape(rows, 3)
    lg = rows.bit_length() - 1
    br = [int(format(i, f"0{lg}b")[::-1], 2) for i in range(rows)]
    assert (gotb[br] == want).all()


@pytest.mark.parametrize("rows,m,a,k", [(256, 17, 2, 2), (1024, 64, 5, 3), (128, 1, 0, 2)])
def test_deep_with_power_coefficients_matches_oracle(be, rows, m, a, k):
    """Trace coefficients that are successive powers of one gamma (the
    prover's): the kernel then accumulates one column sum a row and scales
    it by gamma^k; against the oracle's full sums. A single broken power
    falls back to the general kernel, also against the oracle."""
    rng = np.random.default_rng(7 * rows + m)
    main, aux, parts = rf(rng, (rows, m)), rf(rng, (rows, 3 * a)), rf(rng, (rows, 3 * 2))
    h_ood, gh = rf(rng, (3 * 2,)), rf(rng, (3 * 2,))
    t_ood = rf(rng, (3 * (m + a) * k,))
    gamma = np.array([int(v) for v in rf(rng, (3,))], np.uint64)
    gt = np.zeros(3 * (m + a) * k, np.uint64)
    pw = np.array([1, 0, 0], np.uint64)
    for q in range(2 + (m + a) * k):
        if q >= 2:
            gt[3 * (q - 2):3 * (q - 1)] = pw
        pw = O.fp3_mul(pw, gamma)
    inv_h, inv_t = rf(rng, (3 * rows,)), rf(rng, (3 * k * rows,))
    for broken in (False, True):
        g = gt.copy()
        if broken:
            g[3 * ((m + a) * k - 1)] ^= np.uint64(1)
        want = O.canon_array(O.deep(main, aux if a else np.zeros((rows, 0), np.uint64),
                                    parts, h_ood, t_ood, gh, g, inv_h, inv_t, k)).reshape(rows, 3)
        got = mc.deep_composition_ext3(main, aux, parts, h_ood, t_ood, gh, g, inv_h, inv_t, k, False,
                                       be).reshape(rows, 3)
        assert (got == want).all(), broken


@pytest.mark.parametrize("h", [1, 2, 4, 64, 1024, 1 << 15])
def test_fri_fold_layer_matches_oracle(be, h):
    rng = np.random.default_rng(h)
    ev = rf(rng, (2 * h, 3)).reshape(-1)
    tw = rf(rng, (h,))
    zeta = rf(rng, (3,))
    out, tn, lv = mc.fri_fold(ev, tw, zeta, with_leaves=h >= 2, be=be)
    want = O.canon_array(O.fri_fold(ev, tw, zeta))
    assert (out == want).all()
    if h >= 2:
        assert all(int(tn[j]) == O.canonical(O.gl_mul(int(tw[2 * j]), int(tw[2 * j]))) for j in range(h // 2))
        assert (lv == O.fri_leaves(want)).all()


def random_logup_desc(rng, m, K, n_out, n_committed):
    def rp():
        return int(rng.integers(0, 2**64, dtype=np.uint64)) % P

    eo, ea, ec, to, tc, tl = [0], [], [], [0], [], []
    for k in range(K):
        for e in range(int(rng.integers(1, 4))):
            ea.append(int(rng.integers(0, 5)))
            ec.append(rp())
            for t in range(int(rng.integers(0, 4))):
                tc.append(rp())
                tl.append(int(rng.integers(0, m)))
            to.append(len(tc))
        eo.append(len(ea))
    ints = list(range(K))
    rng.shuffle(ints)
    oo, oi = [0], []
    per = [[] for _ in range(n_out)]
    for i, k in enumerate(ints):
        per[i % n_out].append(k)
    for c in range(n_out):
        oi += per[c]
        oo.append(len(oi))
    mo, mk, ml = [0], [], []
    for k in range(K):
        for t in range(int(rng.integers(0, 3))):
            mk.append(rp())
            ml.append(int(rng.integers(0, m)))
        mo.append(len(mk))
    u32 = lambda x: np.array(x, np.uint32)
    u64 = lambda x: np.array(x, np.uint64)
    return {"num_interactions": K, "bus_ids": u64(rng.integers(0, 1 << 20, size=K)), "elem_offsets": u32(eo),
            "elem_alpha_idx": u32(ea), "elem_consts": u64(ec), "term_offsets": u32(to), "term_coefs": u64(tc),
            "term_cols": u32(tl), "num_out_cols": n_out, "out_col_offsets": u32(oo), "out_col_interactions": u32(oi),
            "mult_consts": u64(rng.integers(0, 1 << 16, size=K)), "mult_term_offsets": u32(mo),
            "mult_term_coefs": u64(mk), "mult_term_cols": u32(ml), "num_committed": n_committed}


@pytest.mark.parametrize("n,m,K,n_out,n_comm", [(1, 4, 1, 1, 0), (8, 5, 3, 2, 1), (1024, 12, 7, 4, 3),
                                                (4096, 40, 12, 6, 5), (3000, 9, 2, 1, 0), (65536, 20, 5, 3, 2)])
def test_logup_aux_matches_oracle(be, n, m, K, n_out, n_comm):
    rng = np.random.default_rng(n + K)
    main = rng.integers(0, 1 << 16, size=(n, m)).astype(np.uint64)
    desc = random_logup_desc(rng, m, K, n_out, n_comm)
    alpha = rf(rng, (5, 3))
    z = rf(rng, (3,))
    aux, L = mc.logup_aux_resident(main, desc, alpha, z, be)
    want_aux, want_L = O.logup_aux(main, desc, alpha, z)
    assert (aux == O.canon_array(want_aux)).all()
    assert (L == O.canon_array(want_L)).all()


@pytest.mark.parametrize("n0,layers", [(64, 3), (1024, 7), (1 << 14, 5)])
def test_fri_commit_state_matches_oracle_chain(be, n0, layers):
    """sg_fri (FriCommitState): each committed layer's evaluations, leaves and
    root follow the oracle's fold chain, the twiddles square from layer to
    layer, and the final fold matches."""
    import ctypes as C
    from lambda_vm_b200 import native
    L = native.lib()
    rng = np.random.default_rng(n0)
    ev = rf(rng, (n0, 3)).reshape(-1)
    tw = rf(rng, (n0 // 2,))
    f = C.c_void_p()
    native.check(L.sg_fri_begin(be.h, None, ev.ctypes.data, 0, tw.ctypes.data, 0, n0, C.byref(f)))
    try:
        cur, ctw = O.canon_array(ev), tw.copy()
        for li in range(layers):
            zeta = rf(rng, (3,))
            root = (C.c_uint8 * 32)()
            host = np.zeros(3 * (len(cur) // 6), np.uint64)
            native.check(L.sg_fri_fold_commit_layer(f, zeta.ctypes.data, root, host.ctypes.data))
            want = O.canon_array(O.fri_fold(cur, ctw, zeta))
            assert (host == want.reshape(-1)).all()
            nodes = O.merkle_nodes(O.fri_leaves(want))
            assert bytes(root) == nodes[0].tobytes()
            d_ev, n, d_nodes, nl = C.c_void_p(), C.c_uint64(), C.c_void_p(), C.c_uint64()
            native.check(L.sg_fri_layer(f, li, C.byref(d_ev), C.byref(n), C.byref(d_nodes), C.byref(nl)))
            assert n.value == len(want.reshape(-1)) // 3 and nl.value == n.value // 2
            cur = want.reshape(-1)
            ctw = np.array([O.canonical(O.gl_mul(int(ctw[2 * j]), int(ctw[2 * j]))) for j in range(len(ctw) // 2)],
                           np.uint64)
        assert L.sg_fri_num_layers(f) == layers
        zeta = rf(rng, (3,))
        fin = np.zeros(3 * (len(cur) // 6), np.uint64)
        native.check(L.sg_fri_fold_final(f, zeta.ctypes.data, fin.ctypes.data))
        assert (fin == O.canon_array(O.fri_fold(cur, ctw, zeta)).reshape(-1)).all()
        assert L.sg_fri_fold_final(f, zeta.ctypes.data, None) == native.SG_ERR_INVALID
    finally:
        L.sg_fri_free(f)


def test_split_commit_matches_two_column_range_trees(be):
    """sg_lde_commit_split (coset_lde_row_major_split_trees): one LDE, a main
    tree over columns [split, m) and a precomputed tree over [0, split)."""
    import ctypes as C
    from lambda_vm_b200 import native
    L = native.lib()
    rng = np.random.default_rng(77)
    n, m, B, split = 1 << 9, 11, 4, 4
    t = rf(rng, (n, m))
    w = O.coset_weights(n, 3)
    Lv = n * B // 2
    pre = C.c_void_p()
    native.check(L.sg_dev_alloc(be.h, None, (2 * Lv - 1) * 32, C.byref(pre)))
    h = C.c_void_p()
    root, root_pre = (C.c_uint8 * 32)(), (C.c_uint8 * 32)()
    host = np.zeros((n * B, m), np.uint64)
    native.check(L.sg_lde_commit_split(be.h, None, t.ctypes.data, 0, n, m, B, w.ctypes.data, split, 1,
                                       host.ctypes.data, C.byref(h), root, pre, root_pre))
    lde = O.canon_array(O.coset_lde_row_major(t, B, w))
    assert (host == lde).all()
    assert bytes(root) == O.merkle_nodes(O.leaves_row_major(lde, 2, False, col_range=(split, m)))[0].tobytes()
    assert bytes(root_pre) == O.merkle_nodes(O.leaves_row_major(lde, 2, False, col_range=(0, split)))[0].tobytes()
    L.sg_lde_free(be.h, h)
    L.sg_dev_free(be.h, None, pre, (2 * Lv - 1) * 32)
