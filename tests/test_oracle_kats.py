"""Pins the CPU oracle to the reference's own known-answer vectors and to
independent mathematical cross-checks (no GPU). The vectors are text-extracted
from lambda_vm's test sources by tests/golden/extract_kats.py."""
import json
import os

import numpy as np
import pytest

import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
KATS = json.load(open(os.path.join(GOLDEN, "reference_kats.json")))
P = O.P


def rand_field(rng, shape):
    x = rng.integers(0, 2**64, size=shape, dtype=np.uint64)
    return np.where(x >= np.uint64(P), x - np.uint64(P), x)


# ---- crypto/ethrex-crypto/src/tests/keccak_tests.rs:57-79
@pytest.mark.parametrize("kat", KATS["keccak256"], ids=lambda k: repr(k["msg"][:12]))
def test_keccak256_kat(kat):
    assert O.keccak256(kat["msg"].encode()).hex() == kat["digest"]


def test_keccak_sponge_block_boundaries():
    # Rate-boundary lengths (keccak_tests.rs:40-52) must agree between the
    # one-shot and the streamed transcript absorber.
    for n in (0, 1, 135, 136, 137, 271, 272, 273):
        data = bytes((i * 7 + 3) & 0xFF for i in range(n))
        t = O.Transcript(b"")
        t.append_bytes(data)
        assert t.state() == O.keccak256(data)


# ---- crypto/crypto/src/tests/default_transcript_tests.rs:253-281
def test_transcript_duplex_kat():
    k = KATS["transcript"]
    t = O.Transcript(k["label"].encode())
    assert [t.sample_base() for _ in range(5)] == k["base"]
    assert t.sample_u64(1 << k["u64_bound_log2"]) == k["u64"]
    te = O.Transcript(k["label"].encode())
    te.append_bytes(k["ext3_phase"].encode())
    assert [int(x) for x in te.sample_ext3()] == k["ext3"]


def test_transcript_clone_replays():
    t = O.Transcript(b"snapshot")
    t.sample_base()
    s = t.clone()
    assert [t.sample_base() for _ in range(6)] == [s.sample_base() for _ in range(6)]


# ---- crypto/stark/src/tests/proof_options_tests.rs:4-40
@pytest.mark.parametrize("q", KATS["fri_queries"], ids=lambda q: f"b{q['blowup']}g{q['grinding']}")
def test_fri_query_count(q):
    assert O.fri_number_of_queries(q["blowup"], q["security_bits"], q["grinding"]) == q["queries"]


# ---- crypto/math-cuda/tests/ntt_known.rs:22-125 (closed-form NTT vectors)
@pytest.mark.parametrize("log_n", [4, 8])
def test_ntt_one_plus_x(log_n):
    n = 1 << log_n
    x = np.zeros(n, np.uint64)
    x[0] = x[1] = 1
    y = O.canon_array(O.fft(x))
    w = O.root_of_unity(log_n)
    c = 1
    for i in range(n):
        assert int(y[i]) == O.canonical(O.gl_add(1, c))
        c = O.gl_mul(c, w)


def test_ntt_x_half_alternates():
    n = 256
    x = np.zeros(n, np.uint64)
    x[n // 2] = 1
    y = O.canon_array(O.fft(x))
    assert all(int(y[i]) == (1 if i % 2 == 0 else P - 1) for i in range(n))


def test_root_of_unity_orders():
    for k in range(1, 33):
        w = O.root_of_unity(k)
        assert O.canonical(O.gl_pow(w, 1 << k)) == 1
        assert O.canonical(O.gl_pow(w, 1 << (k - 1))) == P - 1


def naive_dft(x, omega):
    n = len(x)
    out = []
    for k in range(n):
        acc, wk, p = 0, O.gl_pow(omega, k), 1
        for i in range(n):
            acc = O.gl_add(acc, O.gl_mul(int(x[i]), p))
            p = O.gl_mul(p, wk)
        out.append(O.canonical(acc))
    return np.array(out, np.uint64)


@pytest.mark.parametrize("log_n", [0, 1, 2, 3, 5, 6])
def test_two_half_fft_matches_naive_dft(log_n):
    rng = np.random.default_rng(log_n)
    n = 1 << log_n
    x = rand_field(rng, (n, 3))
    fw = O.canon_array(O.fft(x))
    iv = O.canon_array(O.fft(x, inverse=True))
    w = O.root_of_unity(log_n)
    winv = O.gl_inv(w) if log_n else 1
    for c in range(3):
        assert (fw[:, c] == naive_dft(x[:, c], w)).all()
        assert (iv[:, c] == naive_dft(x[:, c], winv)).all()


@pytest.mark.parametrize("log_n,blowup", [(0, 2), (2, 2), (3, 4), (4, 8), (5, 2)])
def test_coset_lde_is_interpolant_on_coset(log_n, blowup):
    """LDE[k] = P(g * w_{Bn}^k) where P interpolates the column on <w_n>."""
    rng = np.random.default_rng(100 + log_n)
    n = 1 << log_n
    m = 2
    t = rand_field(rng, (n, m))
    lde = O.canon_array(O.coset_lde_row_major(t, blowup))
    wn = O.root_of_unity(log_n)
    coeffs = [naive_dft(t[:, c], O.gl_inv(wn) if log_n else 1) for c in range(m)]
    ninv = O.gl_inv(n)
    wbn = O.root_of_unity(log_n + (blowup.bit_length() - 1))
    for k in range(n * blowup):
        x = O.gl_mul(3, O.gl_pow(wbn, k))
        for c in range(m):
            acc = 0
            for i in reversed(range(n)):
                acc = O.gl_add(O.gl_mul(acc, x), O.gl_mul(int(coeffs[c][i]), ninv))
            assert int(lde[k, c]) == O.canonical(acc)


def test_leaves_layout_matches_manual_bytes():
    rng = np.random.default_rng(7)
    rows, m = 8, 5
    d = rand_field(rng, (rows, m))
    for R in (1, 2):
        for le in (False, True):
            got = O.leaves_row_major(d, R, le)
            for li in range(rows // R):
                buf = b""
                for k in range(R):
                    r = int("{:03b}".format(li * R + k)[::-1], 2)
                    for c in range(m):
                        buf += int(d[r, c]).to_bytes(8, "little" if le else "big")
                assert got[li].tobytes() == O.keccak256(buf)


def test_merkle_tree_matches_manual():
    rng = np.random.default_rng(8)
    for n in (1, 2, 3, 4, 5, 8):
        lv = rng.integers(0, 256, size=(n, 32), dtype=np.uint8)
        nodes = O.merkle_nodes(lv)
        L = 1
        while L < n:
            L *= 2
        level = [lv[min(i, n - 1)].tobytes() for i in range(L)]
        while len(level) > 1:
            level = [O.keccak256(level[2 * i] + level[2 * i + 1]) for i in range(len(level) // 2)]
        assert nodes[0].tobytes() == level[0]
        for pos in range(n):
            path = O.merkle_path(nodes, pos)
            h = nodes[L - 1 + pos].tobytes()
            idx = pos
            for sib in path:
                h = O.keccak256(h + sib.tobytes()) if idx % 2 == 0 else O.keccak256(sib.tobytes() + h)
                idx //= 2
            assert h == nodes[0].tobytes()


def test_fp3_inverse_and_batch_inverse():
    rng = np.random.default_rng(9)
    a = rand_field(rng, (17, 3))
    binv = O.fp3_batch_inverse(a.reshape(-1)).reshape(-1, 3)
    for i in range(17):
        one = O.canon_array(O.fp3_mul(a[i], binv[i]))
        assert list(map(int, one)) == [1, 0, 0]
        assert (O.canon_array(O.fp3_inv(a[i])) == O.canon_array(binv[i])).all()


def test_fri_fold_is_even_plus_zeta_odd():
    """fold(p)(x^2) = 2 (p_even(x^2) + zeta p_odd(x^2)) (fri_functions.rs:8-29)."""
    rng = np.random.default_rng(10)
    deg = 8
    coeffs = rand_field(rng, (deg, 3))
    zeta = rand_field(rng, (3,))
    xs = [O.gl_mul(5, O.gl_pow(O.root_of_unity(4), i)) for i in range(4)]

    def ev(cs, x):
        acc = np.zeros(3, np.uint64)
        for c in reversed(cs):
            acc = np.array([O.gl_add(O.gl_mul(int(acc[k]), x), int(c[k])) for k in range(3)], np.uint64)
        return acc

    evals = []
    for x in xs:
        evals.append(ev(coeffs, x))
        evals.append(ev(coeffs, O.gl_neg(x)))
    inv_tw = np.array([O.gl_inv(x) for x in xs], np.uint64)
    out = O.fri_fold(np.array(evals).reshape(-1), inv_tw, zeta).reshape(-1, 3)
    for j, x in enumerate(xs):
        x2 = O.gl_mul(x, x)
        e = ev(coeffs[0::2], x2)
        o = ev(coeffs[1::2], x2)
        zo = O.fp3_mul(zeta, o)
        want = [O.canonical(O.gl_mul(2, O.gl_add(int(e[k]), int(zo[k])))) for k in range(3)]
        assert list(map(int, O.canon_array(out[j]))) == want


def test_grinding_smallest_nonce():
    seed = bytes(range(32))
    g = 8
    inner = O.grind_inner_hash(seed, g)
    nonce = O.grind(seed, g)
    assert O.grind_is_valid(inner, nonce, g)
    assert not any(O.grind_is_valid(inner, k, g) for k in range(nonce))


@pytest.mark.parametrize("kat", KATS["grinding"], ids=lambda k: f"g{k['grinding_factor']}-{k['nonce']}")
def test_grinding_kat(kat):
    """grinding_tests.rs: Hash(Hash(prefix || seed || g) || nonce_be) validity."""
    inner = O.grind_inner_hash(bytes(kat["seed"]), kat["grinding_factor"])
    assert O.grind_is_valid(inner, kat["nonce"], kat["grinding_factor"]) == kat["valid"]


def test_grinding_search_returns_smallest_nonce_below_the_kat():
    # the g = 10 vector's nonce is valid, so the smallest valid nonce is <= it
    kat = next(k for k in KATS["grinding"] if k["grinding_factor"] == 10 and k["valid"])
    seed, g = bytes(kat["seed"]), kat["grinding_factor"]
    nonce = O.grind(seed, g)
    inner = O.grind_inner_hash(seed, g)
    assert nonce <= kat["nonce"] and O.grind_is_valid(inner, nonce, g)
    assert not any(O.grind_is_valid(inner, k, g) for k in range(nonce))


def test_terminal_roundtrip():
    """terminal_tests.rs test_terminal_roundtrip: coefficients 1..8 evaluated on
    the offset-3 coset of 16 points (FRI bit-reversed order) come back from
    coeffs_from_terminal_codeword with k = 3."""
    from lambda_vm_b200 import field as F
    from lambda_vm_b200.stark import terminal_coeffs
    P = F.P
    w16 = F.root_of_unity(4)
    evals = []
    for i in range(16):
        x = 3 * pow(w16, i, P) % P
        evals.append(sum(c * pow(x, j, P) for j, c in enumerate(range(1, 9))) % P)
    br = [evals[int(format(i, "04b")[::-1], 2)] for i in range(16)]
    cw = np.zeros((16, 3), np.uint64)
    cw[:, 0] = br
    assert terminal_coeffs(cw, 3, 3) == [(c, 0, 0) for c in range(1, 9)]
