"""Device Goldilocks / Fp3 arithmetic against exact Python integers, on edge
values (0, 1, p - 1, p, p + 1, 2^32 - 1, 2^63, 2^64 - 1, ...) crossed with each
other and on seeded random words, including non-canonical inputs."""
import itertools

import numpy as np
import pytest

from lambda_vm_b200 import native
from lambda_vm_b200.device import DeviceBuffer

pytestmark = pytest.mark.gpu
P = (1 << 64) - (1 << 32) + 1
M64 = (1 << 64) - 1
EDGE = [0, 1, 2, 3, P - 2, P - 1, P, P + 1, (1 << 32) - 1, 1 << 32, (1 << 32) + 1, 1 << 63, (1 << 63) + 1,
        M64 - 1, M64, (M64 - (1 << 32)) + 2, 0xFFFFFFFE00000001, 0xFFFFFFFF00000000]


def _pairs(rng, extra=4000):
    e = list(itertools.product(EDGE, EDGE))
    r = [(int(x), int(y)) for x, y in zip(rng.integers(0, 2**64, size=extra, dtype=np.uint64),
                                          rng.integers(0, 2**64, size=extra, dtype=np.uint64))]
    top = [(int(x), int(y)) for x, y in zip(rng.integers(2**64 - 2**34, 2**64, size=extra, dtype=np.uint64),
                                            rng.integers(2**64 - 2**34, 2**64, size=extra, dtype=np.uint64))]
    return e + r + top


def _run(be, op, a, b, width=1):
    L = native.lib()
    da = DeviceBuffer.from_host(np.array(a, np.uint64), be)
    db = DeviceBuffer.from_host(np.array(b, np.uint64), be)
    n = len(a) // width
    do = DeviceBuffer(8 * len(a), be)
    native.check(L.sg_field_ops(be.h, None, op, da.ptr, db.ptr, do.ptr, n))
    out = do.download(np.uint64, len(a))
    for x in (da, db, do):
        x.close()
    return [int(v) for v in out]


@pytest.mark.parametrize("op,fn", [(0, lambda x, y: x + y), (1, lambda x, y: x - y), (2, lambda x, y: x * y),
                                   (6, lambda x, y: x * x)])
def test_base_ops(be, op, fn):
    pairs = _pairs(np.random.default_rng(op))
    a, b = [x for x, _ in pairs], [y for _, y in pairs]
    got = _run(be, op, a, b)
    for x, y, g in zip(a, b, got):
        assert g <= M64 and g % P == fn(x, y) % P, (op, hex(x), hex(y), hex(g))


def test_canon_neg_inv(be):
    rng = np.random.default_rng(9)
    a = EDGE + [int(v) for v in rng.integers(0, 2**64, size=2000, dtype=np.uint64)]
    for g, x in zip(_run(be, 3, a, a), a):
        assert g == x % P
    for g, x in zip(_run(be, 4, a, a), a):
        assert g % P == (-x) % P
    for g, x in zip(_run(be, 5, a, a), a):
        assert (x % P == 0 and g % P == 0) or (g * x) % P == 1


def test_reduce128(be):
    pairs = _pairs(np.random.default_rng(5))
    lo, hi = [x for x, _ in pairs], [y for _, y in pairs]
    for g, x, y in zip(_run(be, 9, lo, hi), lo, hi):
        assert g <= M64 and g % P == (x + (y << 64)) % P


def test_mul_by_power_of_two(be):
    # every exponent 0..95 (2^96 = -1 covers the rest), each on the edge values
    # and on random words; the DFT butterflies multiply by these constants
    rng = np.random.default_rng(8)
    xs = EDGE + [int(v) for v in rng.integers(0, 2**64, size=40, dtype=np.uint64)]
    a = [x for x in xs for _ in range(96)]
    b = [s for _ in xs for s in range(96)]
    for g, x, s in zip(_run(be, 11, a, b), a, b):
        assert g <= M64 and g % P == (x << s) % P, (hex(x), s, hex(g))


def test_unreduced_sums(be):
    rng = np.random.default_rng(6)
    a = [int(v) for v in rng.integers(2**63, 2**64, size=512, dtype=np.uint64)] + EDGE
    b = [int(v) for v in rng.integers(2**63, 2**64, size=512, dtype=np.uint64)] + EDGE[::-1]
    n = len(a)
    got = _run(be, 10, a, b)
    for i in range(n):
        assert got[i] % P == sum(a[i] * b[(i + j) % n] for j in range(16)) % P


def _f3mul(x, y):
    a0, a1, a2 = x
    b0, b1, b2 = y
    return ((a0 * b0 + 2 * (a1 * b2 + a2 * b1)) % P, (a0 * b1 + a1 * b0 + 2 * a2 * b2) % P,
            (a0 * b2 + a1 * b1 + a2 * b0) % P)


def test_fp3_mul_and_inverse(be):
    rng = np.random.default_rng(7)
    vals = [tuple(int(v) for v in rng.integers(0, 2**64, size=3, dtype=np.uint64)) for _ in range(1500)]
    vals += [(e, f, g) for e, f, g in itertools.product([0, 1, P - 1, P, M64], repeat=3)]
    other = vals[1:] + vals[:1]
    flat = lambda vs: [c for v in vs for c in v]
    got = _run(be, 7, flat(vals), flat(other), width=3)
    for i, (x, y) in enumerate(zip(vals, other)):
        assert tuple(g % P for g in got[3 * i:3 * i + 3]) == _f3mul(x, y)
    inv = _run(be, 8, flat(vals), flat(vals), width=3)
    for i, x in enumerate(vals):
        r = tuple(g % P for g in inv[3 * i:3 * i + 3])
        if all(c % P == 0 for c in x):
            assert r == (0, 0, 0)
        else:
            assert _f3mul(tuple(c % P for c in x), r) == (1, 0, 0)
