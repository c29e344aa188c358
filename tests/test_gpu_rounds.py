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


@pytest.mark.parametrize("n,k,sign", [(1, 1, 0), (64, 2, 0), (1000, 3, 1), (4096, 8, 1), (50000, 2, 0)])
def test_inv_denoms_match_oracle(be, n, k, sign):
    rng = np.random.default_rng(n + k)
    x = rf(rng, (n,))
    z = rf(rng, (k, 3))
    got = mc.compute_and_invert_denoms_ext3(x, z, sign, be)
    assert (got == O.canon_array(O.inv_denoms(x, z, sign))).all()


@pytest.mark.parametrize("rows,ru,cols,ext3,stride,k", [
    (64, 5, 5, False, 1, 1), (256, 7, 7, False, 2, 3), (1024, 12, 4, True, 4, 2), (4096, 300, 300, False, 2, 8),
    (2048, 30, 10, True, 2, 5), (16384, 16, 16, False, 4, 2)])
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
                                          (4096, 300, 0, 2, 2), (2048, 8, 40, 1, 8)])
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
