"""GPU parity: NTT, coset LDE, Keccak leaves, Merkle tree/paths, LDE+commit and
grinding through the C ABI, bit-exact against the CPU oracle (canonical
values; digests byte for byte). Modelled on crypto/math-cuda/tests/{ntt.rs,
ntt_known.rs, lde.rs, lde_batch.rs, keccak_leaves.rs, merkle_tree.rs,
merkle_root_parity.rs, merkle_gather.rs, grinding.rs}."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from lambda_vm_b200 import math_cuda as mc
from lambda_vm_b200 import native

pytestmark = pytest.mark.gpu
P = O.P


def rand_field(rng, shape):
    x = rng.integers(0, 2**64, size=shape, dtype=np.uint64)
    return np.where(x >= np.uint64(P), x - np.uint64(P), x)


def rand_raw(rng, shape):
    """Non-canonical inputs too: the reference accepts any u64 representative."""
    return rng.integers(0, 2**64, size=shape, dtype=np.uint64)


# ---------------------------------------------------------------- NTT
@pytest.mark.parametrize("log_n", [1, 2, 4, 5, 8, 10, 11, 12, 13, 16])
@pytest.mark.parametrize("m", [1, 3, 16])
def test_ntt_forward_inverse_match_oracle(be, log_n, m):
    rng = np.random.default_rng(log_n * 31 + m)
    n = 1 << log_n
    x = rand_raw(rng, (n, m))
    fw = mc.ntt_forward(x, be)
    assert (fw == O.canon_array(O.fft(x))).all()
    iv = mc.ntt_inverse(x, be)
    ninv = O.gl_inv(n)
    want = O.canon_array(O.fft(x, inverse=True))
    want = np.array([[O.canonical(O.gl_mul(int(v), ninv)) for v in row] for row in want], np.uint64)
    assert (iv == want).all()
    assert (mc.ntt_inverse(fw, be) == O.canon_array(x)).all()


def test_ntt_known_polynomials(be):
    # ntt_known.rs:22-125
    for log_n in (4, 8):
        n = 1 << log_n
        x = np.zeros(n, np.uint64)
        x[0] = x[1] = 1
        y = mc.ntt_forward(x, be)
        w = O.root_of_unity(log_n)
        c = 1
        for i in range(n):
            assert int(y[i]) == O.canonical(O.gl_add(1, c))
            c = O.gl_mul(c, w)
    n = 256
    x = np.zeros(n, np.uint64)
    x[n // 2] = 1
    y = mc.ntt_forward(x, be)
    assert all(int(y[i]) == (1 if i % 2 == 0 else P - 1) for i in range(n))


# ---------------------------------------------------------------- coset LDE
LDE_CASES = [(0, 1, 2), (1, 1, 2), (1, 5, 4), (3, 8, 2), (5, 3, 8), (7, 17, 4), (10, 8, 2), (12, 4, 4),
             (13, 9, 2), (14, 16, 4), (15, 3, 2), (16, 33, 2), (17, 8, 4), (13, 256, 4), (12, 1, 16)]


@pytest.mark.parametrize("log_n,m,blowup", LDE_CASES)
def test_coset_lde_matches_oracle(be, log_n, m, blowup):
    rng = np.random.default_rng(1000 + log_n * 7 + m)
    n = 1 << log_n
    t = rand_raw(rng, (n, m))
    w = O.coset_weights(n, 3)
    got = mc.coset_lde_batch_base(t, blowup, w, be)
    want = O.canon_array(O.coset_lde_row_major(t, blowup, w))
    assert got.shape == want.shape
    assert (got == want).all()


def test_coset_lde_arbitrary_weights(be):
    """The weights are an input (lde.rs takes them from the caller)."""
    rng = np.random.default_rng(5)
    n, m = 1 << 14, 5
    t = rand_field(rng, (n, m))
    w = rand_field(rng, (n,))
    assert (mc.coset_lde_batch_base(t, 2, w, be) == O.canon_array(O.coset_lde_row_major(t, 2, w))).all()


def test_coset_lde_single_column(be):
    rng = np.random.default_rng(6)
    n = 1 << 9
    t = rand_field(rng, (n,))
    w = O.coset_weights(n, 7)
    got = mc.coset_lde_base(t, 4, w, be)
    assert (got == O.canon_array(O.coset_lde_row_major(t, 4, w)).reshape(-1)).all()


# ---------------------------------------------------------------- leaves / tree
@pytest.mark.parametrize("rows,ru,R,le,cr", [
    (2, 1, 1, False, None), (2, 1, 2, False, None), (8, 5, 2, False, None), (8, 5, 1, True, None),
    (64, 17, 2, False, None), (64, 16, 1, False, None), (256, 256, 1, True, None), (256, 256, 2, False, None),
    (128, 24, 2, False, None), (1024, 300, 2, False, None), (512, 40, 2, False, (0, 13)),
    (512, 40, 2, False, (13, 40)), (4096, 3, 2, True, None)])
def test_keccak_leaves_match_oracle(be, rows, ru, R, le, cr):
    rng = np.random.default_rng(rows + ru)
    d = rand_raw(rng, (rows, ru))
    got = mc.keccak_leaves_row_major(d, R, le, cr, be)
    want = O.leaves_row_major(d, R, le, cr)
    assert (got == want).all()


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 8, 128, 255, 256, 257, 1000, 1 << 12, (1 << 16) + 3])
def test_merkle_tree_matches_oracle(be, n):
    rng = np.random.default_rng(n)
    lv = rng.integers(0, 256, size=(n, 32), dtype=np.uint8)
    got = mc.build_merkle_tree_on_device(lv, be)
    want = O.merkle_nodes(lv)
    assert got.shape == want.shape
    assert (got == want).all()


# ---------------------------------------------------------------- LDE + commit
@pytest.mark.parametrize("log_n,m,blowup,R,le", [
    (3, 4, 2, 2, False), (8, 7, 4, 2, False), (10, 64, 2, 2, False), (13, 32, 4, 1, True),
    (14, 12, 2, 2, False), (12, 256, 4, 1, True), (11, 3 * 5, 2, 2, False),
    # host traces of >= 64 columns are uploaded in 32-column chunks; one-row
    # leaves are then absorbed in 17-lane windows as the chunks complete
    (10, 300, 2, 1, False), (9, 130, 4, 1, True), (11, 200, 2, 2, False), (8, 128, 8, 1, False),
    (10, 64, 2, 1, False), (9, 63, 2, 1, True), (10, 97, 2, 1, True), (9, 65, 4, 2, False)])
def test_lde_commit_root_matches_oracle(be, log_n, m, blowup, R, le):
    """merkle_root_parity.rs: GPU LDE + leaves + tree root == CPU row-major
    LDE + commit_rows_bit_reversed."""
    rng = np.random.default_rng(2000 + log_n)
    n = 1 << log_n
    t = rand_raw(rng, (n, m))
    w = O.coset_weights(n, 3)
    h, host = mc.lde_commit(t, n, m, blowup, w, R, le, None, True, be)
    lde = O.canon_array(O.coset_lde_row_major(t, blowup, w))
    assert (host == lde).all()
    nodes = O.merkle_nodes(O.leaves_row_major(lde, R, le))
    assert h.root == nodes[0].tobytes()
    assert (h.nodes_host() == nodes).all()
    # authentication paths from the resident tree (merkle_gather.rs)
    pos = rng.integers(0, h.leaves_len, size=37).astype(np.uint32)
    paths = mc.gather_merkle_paths_dev(h.d_nodes, h.leaves_len, pos, be)
    for q, p in enumerate(pos):
        assert (paths[q] == O.merkle_path(nodes, int(p))).all()
    h.free()


def test_reference_entry_point_row_pair_big_endian(be):
    rng = np.random.default_rng(77)
    n, m = 1 << 9, 11
    t = rand_field(rng, (n, m))
    w = O.coset_weights(n, 3)
    h, host = mc.coset_lde_row_major_with_merkle_tree_keep(t, n, m, 2, w, retain_host_lde=False, be=be)
    assert host.size == 0
    lde = O.canon_array(O.coset_lde_row_major(t, 2, w))
    assert h.root == O.merkle_root(O.leaves_row_major(lde, 2, False))
    assert (h.lde_host() == lde).all()
    h.free()


def test_ext3_commit_is_interleaved_columns(be):
    rng = np.random.default_rng(78)
    n, m = 1 << 8, 4
    t = rand_field(rng, (n, 3 * m))
    w = O.coset_weights(n, 3)
    h, host = mc.coset_lde_ext3_row_major_with_merkle_tree_keep(t, n, m, 4, w, retain_host_lde=True, be=be)
    lde = O.canon_array(O.coset_lde_row_major(t, 4, w))
    assert (host == lde).all()
    assert h.root == O.merkle_root(O.leaves_row_major(lde, 2, False))
    h.free()


# ---------------------------------------------------------------- grinding
@pytest.mark.parametrize("g", [1, 4, 10, 16])
def test_grinding_smallest_nonce(be, g):
    seed = bytes((i * 13 + g) & 0xFF for i in range(32))
    inner = O.grind_inner_hash(seed, g)
    nonce = mc.generate_nonce_gpu(mc.inner_hash_lanes(inner), g, be)
    assert O.grind_is_valid(inner, nonce, g)
    assert nonce == O.grind(seed, g)


def _grinding_kats():
    import json
    import os
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))
    return [k for k in d["grinding"] if k["valid"] and k["grinding_factor"] <= 20]


@pytest.mark.parametrize("kat", _grinding_kats(), ids=lambda k: f"g{k['grinding_factor']}")
def test_grinding_reference_vectors(be, kat):
    """grinding_tests.rs vectors: the device search returns the smallest valid
    nonce, which is at most the reference test's valid nonce."""
    seed, g = bytes(kat["seed"]), kat["grinding_factor"]
    inner = O.grind_inner_hash(seed, g)
    nonce = mc.generate_nonce_gpu(mc.inner_hash_lanes(inner), g, be)
    assert nonce <= kat["nonce"] and O.grind_is_valid(inner, nonce, g)
    assert nonce == O.grind(seed, g)


# ---------------------------------------------------------------- errors
def test_invalid_shapes_raise_status(be):
    from lambda_vm_b200.native import SgError
    with pytest.raises(SgError):
        mc.coset_lde_batch_base(np.zeros((3, 2), np.uint64), 2, np.zeros(3, np.uint64), be)
    with pytest.raises(SgError):
        mc.coset_lde_batch_base(np.zeros((4, 2), np.uint64), 3, np.zeros(4, np.uint64), be)


def test_injected_allocation_failure_is_reported(be):
    from lambda_vm_b200.native import SgError, SG_ERR_OOM
    rng = np.random.default_rng(3)
    t = rand_field(rng, (64, 4))
    w = O.coset_weights(64, 3)
    be.fail_alloc_after(2)
    with pytest.raises(SgError) as e:
        mc.lde_commit(t, 64, 4, 2, w, be=be)
    be.fail_alloc_after(0)
    assert e.value.code == SG_ERR_OOM
    h, _ = mc.lde_commit(t, 64, 4, 2, w, be=be)  # context still usable
    assert h.root == O.merkle_root(O.leaves_row_major(O.coset_lde_row_major(t, 2, w), 2, False))
    h.free()


@pytest.mark.parametrize("log_n", [16, 18, 20, 22])
def test_every_dft_tile_width_gives_the_same_lde(be, log_n):
    """The tile autotuner only regroups columns into tiles: every compiled
    width of the pass length (2^(log_n/2) points) yields the identical LDE."""
    import ctypes as C
    from lambda_vm_b200 import native
    L = native.lib()
    log_len = log_n // 2
    cols = (C.c_uint32 * 4)()
    cost = (C.c_float * 4)()
    cnt = C.c_uint32()
    native.check(L.sg_ctx_dft_tuning(be.h, None, log_len, cols, cost, C.byref(cnt)))
    widths = [cols[i] for i in range(cnt.value)]
    assert cnt.value >= 2 and all(cost[i] > 0 for i in range(cnt.value))
    rng = np.random.default_rng(log_n)
    n, m = 1 << log_n, 7
    t = rand_raw(rng, (n, m))
    w = O.coset_weights(n, 3)
    outs = []
    try:
        for c in widths + [0]:
            native.check(L.sg_ctx_dft_tiles(be.h, log_len, c))
            outs.append(mc.coset_lde_batch_base(t, 2, w, be=be))
    finally:
        native.check(L.sg_ctx_dft_tiles(be.h, log_len, 0))
    for o in outs[1:]:
        assert (o == outs[0]).all()
    # and the oracle at every length, 2^11-point passes (log_n 22) included
    assert (outs[0] == O.canon_array(O.coset_lde_row_major(t, 2, w))).all()
    with pytest.raises(native.SgError):
        native.check(L.sg_ctx_dft_tiles(be.h, log_len, 5))


def test_lde_rejects_sizes_that_overflow(be):
    """A column count whose matrix size wraps 64 bits is an argument error,
    raised before any allocation or launch."""
    L = native.lib()
    for m in (1 << 61, (1 << 64) - 1):
        rc = L.sg_coset_lde(be.h, None, C.c_void_p(16), 1 << 10, m, 4, C.c_void_p(16), C.c_void_p(16))
        assert rc == native.SG_ERR_INVALID
        assert b"overflows" in L.sg_last_error()
