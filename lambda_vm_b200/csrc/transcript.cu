// Host-side pieces of the prover runtime: Goldilocks / Fp3 arithmetic on the
// CPU (for the few scalars the host folds: OOD constants, terminal FRI
// polynomial) and the Fiat-Shamir transcript.
//
// The transcript restates crypto/crypto/src/fiat_shamir/default_transcript.rs:31-146:
// a Keccak-256 hash chain; sample() = finalize, byte-reverse, absorb the
// reversed digest; field and index sampling read big-endian u64 candidates
// from a 32-byte duplex buffer (4 per squeeze), invalidated by every absorb;
// rejection sampling below p; sample_u64 uses the modulo threshold. The
// out-of-domain sampler follows is_transcript.rs:44-75.
#include <stdint.h>
#include <string.h>

#include <new>

#include "../../include/starkgpu.h"
#include "fs.cuh"

typedef unsigned __int128 u128;
static const uint64_t P = 0xFFFFFFFF00000001ULL;

extern "C" {

uint64_t sg_host_gl_canon(uint64_t a) { return a >= P ? a - P : a; }
uint64_t sg_host_gl_add(uint64_t a, uint64_t b) {
    const uint64_t x = sg_host_gl_canon(a), y = sg_host_gl_canon(b);
    uint64_t s = x + y;
    if (s < x) s += 0xFFFFFFFFull;  // the carry 2^64 = 2^32 - 1 (mod p); no second carry (x + y < 2p)
    return sg_host_gl_canon(s);
}
uint64_t sg_host_gl_sub(uint64_t a, uint64_t b) {
    uint64_t x = sg_host_gl_canon(a), y = sg_host_gl_canon(b);
    return x >= y ? x - y : x + (P - y);
}
// A 128-bit product reduced with 2^64 = 2^32 - 1 and 2^96 = -1 (mod p):
// lo + hl 2^64 + hh 2^96 = lo - hh + hl (2^32 - 1), each step folding its
// borrow or carry back in once (the sums leave no second one).
uint64_t sg_host_gl_mul(uint64_t a, uint64_t b) {
    const u128 x = (u128)a * b;
    const uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64), hh = hi >> 32, hl = hi & 0xFFFFFFFFull;
    uint64_t t = lo - hh;
    if (lo < hh) t -= 0xFFFFFFFFull;
    const uint64_t u = hl * 0xFFFFFFFFull;
    uint64_t r = t + u;
    if (r < u) r += 0xFFFFFFFFull;
    return sg_host_gl_canon(r);
}
uint64_t sg_host_gl_pow(uint64_t a, uint64_t e) {
    uint64_t r = 1, b = sg_host_gl_canon(a);
    while (e) {
        if (e & 1) r = sg_host_gl_mul(r, b);
        b = sg_host_gl_mul(b, b);
        e >>= 1;
    }
    return r;
}
uint64_t sg_host_gl_inv(uint64_t a) { return sg_host_gl_pow(a, P - 2); }

void sg_host_fp3_add(const uint64_t* a, const uint64_t* b, uint64_t* c) {
    for (int i = 0; i < 3; ++i) c[i] = sg_host_gl_add(a[i], b[i]);
}
void sg_host_fp3_sub(const uint64_t* a, const uint64_t* b, uint64_t* c) {
    for (int i = 0; i < 3; ++i) c[i] = sg_host_gl_sub(a[i], b[i]);
}
void sg_host_fp3_mul(const uint64_t* a, const uint64_t* b, uint64_t* c) {
    // (a0 + a1 w + a2 w^2)(b0 + b1 w + b2 w^2), w^3 = 2
    u128 t0 = (u128)a[0] * b[0] % P, t1, t2;
    uint64_t r0 = sg_host_gl_add((uint64_t)t0, sg_host_gl_mul(2, sg_host_gl_add(sg_host_gl_mul(a[1], b[2]),
                                                                                     sg_host_gl_mul(a[2], b[1]))));
    t1 = sg_host_gl_add(sg_host_gl_add(sg_host_gl_mul(a[0], b[1]), sg_host_gl_mul(a[1], b[0])),
                        sg_host_gl_mul(2, sg_host_gl_mul(a[2], b[2])));
    t2 = sg_host_gl_add(sg_host_gl_add(sg_host_gl_mul(a[0], b[2]), sg_host_gl_mul(a[1], b[1])),
                        sg_host_gl_mul(a[2], b[0]));
    c[0] = r0;
    c[1] = (uint64_t)t1;
    c[2] = (uint64_t)t2;
}
void sg_host_fp3_pow(const uint64_t* a, uint64_t e, uint64_t* out) {
    uint64_t r[3] = {1, 0, 0}, b[3] = {a[0], a[1], a[2]};
    while (e) {
        if (e & 1) sg_host_fp3_mul(r, b, r);
        sg_host_fp3_mul(b, b, b);
        e >>= 1;
    }
    memcpy(out, r, 24);
}
int sg_host_fp3_inv(const uint64_t* a, uint64_t* out) {
    // norm N = a0^3 + 2 a1^3 + 4 a2^3 - 6 a0 a1 a2; inverse = adj / N
    uint64_t a0 = a[0], a1 = a[1], a2 = a[2];
    uint64_t a0s = sg_host_gl_mul(a0, a0), a1s = sg_host_gl_mul(a1, a1), a2s = sg_host_gl_mul(a2, a2);
    uint64_t nrm = sg_host_gl_mul(a0s, a0);
    nrm = sg_host_gl_add(nrm, sg_host_gl_mul(2, sg_host_gl_mul(a1s, a1)));
    nrm = sg_host_gl_add(nrm, sg_host_gl_mul(4, sg_host_gl_mul(a2s, a2)));
    nrm = sg_host_gl_sub(nrm, sg_host_gl_mul(6, sg_host_gl_mul(sg_host_gl_mul(a0, a1), a2)));
    if (nrm == 0) return -1;
    uint64_t ni = sg_host_gl_inv(nrm);
    out[0] = sg_host_gl_mul(sg_host_gl_sub(a0s, sg_host_gl_mul(2, sg_host_gl_mul(a1, a2))), ni);
    out[1] = sg_host_gl_mul(sg_host_gl_sub(sg_host_gl_mul(2, a2s), sg_host_gl_mul(a0, a1)), ni);
    out[2] = sg_host_gl_mul(sg_host_gl_sub(a1s, sg_host_gl_mul(a0, a2)), ni);
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------- Keccak-256 (host)
namespace {

const uint64_t RC[24] = {
    0x0000000000000001ULL, 0x0000000000008082ULL, 0x800000000000808aULL, 0x8000000080008000ULL,
    0x000000000000808bULL, 0x0000000080000001ULL, 0x8000000080008081ULL, 0x8000000000008009ULL,
    0x000000000000008aULL, 0x0000000000000088ULL, 0x0000000080008009ULL, 0x000000008000000aULL,
    0x000000008000808bULL, 0x800000000000008bULL, 0x8000000000008089ULL, 0x8000000000008003ULL,
    0x8000000000008002ULL, 0x8000000000000080ULL, 0x000000000000800aULL, 0x800000008000000aULL,
    0x8000000080008081ULL, 0x8000000000008080ULL, 0x0000000080000001ULL, 0x8000000080008008ULL};
// rho offsets, lane x + 5y
const unsigned RHO[25] = {0, 1, 62, 28, 27, 36, 44, 6, 55, 20, 3, 10, 43, 25, 39, 41, 45, 15, 21, 8, 18, 2, 61, 56, 14};

inline uint64_t rol(uint64_t x, unsigned r) { return r ? (x << r) | (x >> (64 - r)) : x; }

void keccak_f(uint64_t* A) {
    for (int round = 0; round < 24; ++round) {
        uint64_t C[5], D[5], B[25];
        for (int x = 0; x < 5; ++x) C[x] = A[x] ^ A[x + 5] ^ A[x + 10] ^ A[x + 15] ^ A[x + 20];
        for (int x = 0; x < 5; ++x) D[x] = C[(x + 4) % 5] ^ rol(C[(x + 1) % 5], 1);
        for (int y = 0; y < 5; ++y)
            for (int x = 0; x < 5; ++x) B[y + 5 * ((2 * x + 3 * y) % 5)] = rol(A[x + 5 * y] ^ D[x], RHO[x + 5 * y]);
        for (int y = 0; y < 5; ++y)
            for (int x = 0; x < 5; ++x)
                A[x + 5 * y] = B[x + 5 * y] ^ (~B[(x + 1) % 5 + 5 * y] & B[(x + 2) % 5 + 5 * y]);
        A[0] ^= RC[round];
    }
}

}  // namespace

void fs::host_permute(uint64_t st[25]) { keccak_f(st); }

extern "C" {

void sg_keccak256(const uint8_t* data, uint64_t len, uint8_t out[32]) {
    fs::State k;
    fs::init(k, data, len);
    fs::final_digest(k, out);
}

sg_transcript* sg_transcript_new(const uint8_t* data, uint64_t len) {
    sg_transcript* t = new (std::nothrow) sg_transcript;
    if (!t) return nullptr;
    fs::init(t->s, data, len);
    return t;
}

sg_transcript* sg_transcript_clone(const sg_transcript* t) {
    sg_transcript* c = new (std::nothrow) sg_transcript;
    if (c) *c = *t;
    return c;
}

void sg_transcript_free(sg_transcript* t) { delete t; }

void sg_transcript_append(sg_transcript* t, const uint8_t* data, uint64_t len) { fs::append(t->s, data, len); }

void sg_transcript_append_base(sg_transcript* t, uint64_t v) { fs::append_u64_be(t->s, fs::canon(v)); }

void sg_transcript_append_ext3(sg_transcript* t, const uint64_t v[3]) { fs::append_ext3(t->s, v); }

void sg_transcript_sample(sg_transcript* t, uint8_t out[32]) { fs::sample(t->s, out); }

void sg_transcript_state(const sg_transcript* t, uint8_t out[32]) { fs::final_digest(t->s, out); }

uint64_t sg_transcript_sample_base(sg_transcript* t) { return fs::sample_base(t->s); }

void sg_transcript_sample_ext3(sg_transcript* t, uint64_t out[3]) { fs::sample_ext3(t->s, out); }

uint64_t sg_transcript_sample_u64(sg_transcript* t, uint64_t upper) { return fs::sample_u64(t->s, upper); }

void sg_transcript_sample_z_ood(sg_transcript* t, uint64_t trace_len, uint64_t lde_len, uint64_t coset_offset,
                                uint64_t out[3]) {
    const uint64_t off_pow = sg_host_gl_pow(coset_offset, lde_len);
    const uint64_t blowup = lde_len / trace_len;
    for (;;) {
        uint64_t z[3];
        sg_transcript_sample_ext3(t, z);
        uint64_t zt[3], zl[3];
        sg_host_fp3_pow(z, trace_len, zt);
        const bool in_trace = zt[0] == 1 && zt[1] == 0 && zt[2] == 0;
        sg_host_fp3_pow(zt, blowup, zl);
        const bool in_lde = zl[0] == off_pow && zl[1] == 0 && zl[2] == 0;
        if (!in_trace && !in_lde) {
            memcpy(out, z, 24);
            return;
        }
    }
}

}  // extern "C"
