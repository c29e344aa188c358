"""Vectorised host-side Goldilocks helpers (numpy) for prover set-up data:
coset points, LDE weights, zerofier inputs, synthetic traces. The proving
arithmetic itself runs on the GPU; these only build inputs of size O(N)."""
import numpy as np

P = 0xFFFFFFFF00000001
_P = np.uint64(P)
_EPS = np.uint64(0xFFFFFFFF)
_M32 = np.uint64(0xFFFFFFFF)
GENERATOR_2ADIC = 1753635133440165772


def canon(a):
    a = np.asarray(a, dtype=np.uint64)
    return np.where(a >= _P, a - _P, a)


def add(a, b):
    a, b = canon(a), canon(b)
    s = a + b
    over = s < a
    s = np.where(over, s + _EPS, s)
    return canon(s)


def sub(a, b):
    a, b = canon(a), canon(b)
    return np.where(a >= b, a - b, a + (_P - b))


def mul(a, b):
    """a*b mod p, elementwise, via the 64x64->128 product in 32-bit limbs."""
    a = np.asarray(a, dtype=np.uint64)
    b = np.asarray(b, dtype=np.uint64)
    with np.errstate(over="ignore"):
        a0, a1 = a & _M32, a >> np.uint64(32)
        b0, b1 = b & _M32, b >> np.uint64(32)
        p00, p01, p10, p11 = a0 * b0, a0 * b1, a1 * b0, a1 * b1
        mid = p01 + p10
        mid_carry = (mid < p01).astype(np.uint64)
        lo = p00 + (mid << np.uint64(32))
        lo_carry = (lo < p00).astype(np.uint64)
        hi = p11 + (mid >> np.uint64(32)) + (mid_carry << np.uint64(32)) + lo_carry
        # reduce128: lo - hi_hi, + hi_lo * EPS
        hh, hl = hi >> np.uint64(32), hi & _M32
        t0 = lo - hh
        t0 = np.where(lo < hh, t0 - _EPS, t0)
        t1 = (hl << np.uint64(32)) - hl
        r = t0 + t1
        r = np.where(r < t0, r + _EPS, r)
    return canon(r)


def pow_int(a, e):
    return pow(int(a) % P, int(e), P)


def inv_int(a):
    return pow(int(a) % P, P - 2, P)


def root_of_unity(log_n):
    r = GENERATOR_2ADIC
    for _ in range(32 - log_n):
        r = r * r % P
    return r if log_n else 1


def powers(base, count, start=1):
    """[start * base^i for i < count] without a sequential loop over count."""
    base = int(base) % P
    if count == 0:
        return np.zeros(0, np.uint64)
    blk = 1 << 10
    lo = np.empty(min(blk, count), np.uint64)
    c = 1
    for i in range(lo.size):
        lo[i] = c
        c = c * base % P
    nhi = (count + blk - 1) // blk
    hi = np.empty(nhi, np.uint64)
    step = pow(base, blk, P)
    c = int(start) % P
    for i in range(nhi):
        hi[i] = c
        c = c * step % P
    out = mul(np.repeat(hi, blk)[:count], np.tile(lo, nhi)[:count])
    return out


def coset_points(log_n, offset):
    """offset * w_n^i for i < n."""
    return powers(root_of_unity(log_n), 1 << log_n, offset)


def coset_weights(n, offset):
    """g^i / n (crypto/stark/src/prover.rs:458-467)."""
    return powers(offset, n, inv_int(n))


def composition_weights(half, offset):
    """g^-j / half (prover.rs:419-437 CompositionLdeTwiddles)."""
    return powers(inv_int(offset), half, inv_int(half))


def bitrev_indices(log_n):
    n = 1 << log_n
    i = np.arange(n, dtype=np.uint64)
    r = np.zeros(n, dtype=np.uint64)
    for b in range(log_n):
        r |= ((i >> np.uint64(b)) & np.uint64(1)) << np.uint64(log_n - 1 - b)
    return r


def bitrev_vec(idx, bits):
    """Bit-reversal of each index of `idx` (array-like) over `bits` bits."""
    i = np.asarray(idx, dtype=np.uint64)
    r = np.zeros_like(i)
    for b in range(bits):
        r |= ((i >> np.uint64(b)) & np.uint64(1)) << np.uint64(bits - 1 - b)
    return r


def f3mul_vec(a, b):
    """Fp3 products of (..., 3) uint64 arrays, with broadcasting; canonical output."""
    a = np.asarray(a, np.uint64)
    b = np.asarray(b, np.uint64)
    a0, a1, a2 = a[..., 0], a[..., 1], a[..., 2]
    b0, b1, b2 = b[..., 0], b[..., 1], b[..., 2]
    t = add(mul(a1, b2), mul(a2, b1))
    c0 = add(mul(a0, b0), add(t, t))
    u = mul(a2, b2)
    c1 = add(add(mul(a0, b1), mul(a1, b0)), add(u, u))
    c2 = add(add(mul(a0, b2), mul(a1, b1)), mul(a2, b0))
    return canon(np.stack(np.broadcast_arrays(c0, c1, c2), axis=-1))


# ---------------- scalar Fp3 helpers (Python ints) for the few host-side
# extension-field values (challenges, OOD scalars, terminal polynomial).
def f3(x):
    return tuple(int(v) % P for v in x)


def f3add(a, b):
    return tuple((a[i] + b[i]) % P for i in range(3))


def f3sub(a, b):
    return tuple((a[i] - b[i]) % P for i in range(3))


def f3mul(a, b):
    a0, a1, a2 = a
    b0, b1, b2 = b
    return ((a0 * b0 + 2 * (a1 * b2 + a2 * b1)) % P, (a0 * b1 + a1 * b0 + 2 * a2 * b2) % P,
            (a0 * b2 + a1 * b1 + a2 * b0) % P)


def f3scale(a, s):
    return tuple(v * (int(s) % P) % P for v in a)


def f3pow(a, e):
    r, b = (1, 0, 0), f3(a)
    while e:
        if e & 1:
            r = f3mul(r, b)
        b = f3mul(b, b)
        e >>= 1
    return r


def f3inv(a):
    a0, a1, a2 = f3(a)
    nrm = (a0 ** 3 + 2 * a1 ** 3 + 4 * a2 ** 3 - 6 * a0 * a1 * a2) % P
    ni = pow(nrm, P - 2, P)
    return ((a0 * a0 - 2 * a1 * a2) * ni % P, (2 * a2 * a2 - a0 * a1) * ni % P, (a1 * a1 - a0 * a2) * ni % P)


def bitrev_int(i, bits):
    return int(format(i, f"0{bits}b")[::-1], 2) if bits else 0
