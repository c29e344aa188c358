// Goldilocks (p = 2^64 - 2^32 + 1) and its cubic extension Fp3 = Fp[w]/(w^3 - 2)
// for sm_100a. Same field semantics as crypto/math/src/field/goldilocks.rs:72-216
// and extensions_goldilocks.rs:280-420: values live in [0, 2^64), reduced mod p
// but not necessarily canonical; gl_canon() maps to [0, p) at the boundaries
// (hashing, host output). All arithmetic is exact 64-bit modular integer math
// written as explicit 32-bit carry chains so the INT pipes see the minimum.
#pragma once
#include <stdint.h>

#define GL_P 0xFFFFFFFF00000001ULL
#define GL_EPS 0xFFFFFFFFULL

namespace gl {

__device__ __forceinline__ uint32_t lo32(uint64_t x) { return (uint32_t)x; }
__device__ __forceinline__ uint32_t hi32(uint64_t x) { return (uint32_t)(x >> 32); }
__device__ __forceinline__ uint64_t pack(uint32_t lo, uint32_t hi) {
    return ((uint64_t)hi << 32) | lo;
}

__device__ __forceinline__ uint64_t canon(uint64_t a) { return a >= GL_P ? a - GL_P : a; }

// a + b mod p. The carry c of the 64-bit sum is folded as c * EPS with a
// 32-bit multiply-add (FMA pipe), whose own carry w is folded the same way;
// that second fold cannot carry (after a wrap the sum is < EPS - 1). The
// additions and the two carry reads stay on the ALU pipe, which the
// butterflies saturate, while the FMA pipe has room.
__device__ __forceinline__ uint64_t add(uint64_t a, uint64_t b) {
    uint32_t r0, r1, c, w;
    asm("add.cc.u32 %0, %3, %5;\n\t"
        "addc.cc.u32 %1, %4, %6;\n\t"
        "addc.u32 %2, 0, 0;"
        : "=r"(r0), "=r"(r1), "=r"(c)
        : "r"(lo32(a)), "r"(hi32(a)), "r"(lo32(b)), "r"(hi32(b)));
    asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
        "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
        "addc.u32 %2, 0, 0;"
        : "+r"(r0), "+r"(r1), "=r"(w)
        : "r"(c), "r"(0xFFFFFFFFu));
    asm("mad.lo.cc.u32 %0, %2, %3, %0;\n\t"
        "madc.hi.u32 %1, %2, %3, %1;"
        : "+r"(r0), "+r"(r1)
        : "r"(w), "r"(0xFFFFFFFFu));
    return pack(r0, r1);
}

// a - b mod p.
__device__ __forceinline__ uint64_t sub(uint64_t a, uint64_t b) {
    uint32_t r0, r1, br;
    asm("sub.cc.u32 %0, %3, %5;\n\t"
        "subc.cc.u32 %1, %4, %6;\n\t"
        "subc.u32 %2, 0, 0;"
        : "=r"(r0), "=r"(r1), "=r"(br)
        : "r"(lo32(a)), "r"(hi32(a)), "r"(lo32(b)), "r"(hi32(b)));
    uint32_t br2;
    asm("sub.cc.u32 %0, %0, %3;\n\t"
        "subc.cc.u32 %1, %1, 0;\n\t"
        "subc.u32 %2, 0, 0;"
        : "+r"(r0), "+r"(r1), "=r"(br2)
        : "r"(br));  // br is 0 or 0xFFFFFFFF == EPS
    uint64_t r = pack(r0, r1);
    if (br2) r -= GL_EPS;  // r >= 2^64 - EPS after a second wrap, so this cannot borrow
    return r;
}

// Reduce the 128-bit value (x3:x2:x1:x0) mod p using 2^64 = EPS, 2^96 = -1:
// V = (x1:x0) + x2 * EPS - x3. The x2 * EPS term is a 32x32 multiply-add on
// the FMA pipe into the low word pair (S < 2^65, carry c); subtracting x3
// leaves c' = c - borrow in {-1, 0, 1}, and V = s + c' * 2^64 = s + c' * EPS
// with no further wrap (S <= 2^65 - 2^33, so s + EPS < 2^64 when c' = 1; and
// c' = -1 only when s >= 2^64 - x3 > EPS). c' * EPS mod 2^64 has low word -c'
// and high word sign(c').
__device__ __forceinline__ uint64_t reduce128(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3) {
    uint32_t s0, s1, c;
    asm("mad.lo.cc.u32 %0, %3, %5, %4;\n\t"
        "madc.hi.cc.u32 %1, %3, %5, %6;\n\t"
        "addc.u32 %2, 0, 0;"
        : "=r"(s0), "=r"(s1), "=r"(c)
        : "r"(x2), "r"(x0), "r"(0xFFFFFFFFu), "r"(x1));
    asm("sub.cc.u32 %0, %0, %3;\n\t"
        "subc.cc.u32 %1, %1, 0;\n\t"
        "subc.u32 %2, %2, 0;"
        : "+r"(s0), "+r"(s1), "+r"(c)
        : "r"(x3));
    const uint32_t lo = 0u - c, hi = (uint32_t)((int32_t)c >> 31);
    asm("add.cc.u32 %0, %0, %2;\n\t"
        "addc.u32 %1, %1, %3;"
        : "+r"(s0), "+r"(s1)
        : "r"(lo), "r"(hi));
    return pack(s0, s1);
}

// Full 64x64 -> 128 product as four 32-bit limbs.
__device__ __forceinline__ void mul128(uint64_t a, uint64_t b, uint32_t& r0, uint32_t& r1, uint32_t& r2,
                                       uint32_t& r3) {
    uint32_t a0 = lo32(a), a1 = hi32(a), b0 = lo32(b), b1 = hi32(b);
    asm("mul.lo.u32 %0, %4, %6;\n\t"
        "mul.hi.u32 %1, %4, %6;\n\t"
        "mad.lo.cc.u32 %1, %4, %7, %1;\n\t"
        "madc.hi.u32 %2, %4, %7, 0;\n\t"
        "mad.lo.cc.u32 %1, %5, %6, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
        "madc.hi.u32 %3, %5, %7, 0;\n\t"
        "mad.lo.cc.u32 %2, %5, %7, %2;\n\t"
        "addc.u32 %3, %3, 0;"
        : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
        : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint64_t mul(uint64_t a, uint64_t b) {
    uint32_t r0, r1, r2, r3;
    mul128(a, b, r0, r1, r2, r3);
    return reduce128(r0, r1, r2, r3);
}

// Reduce the 96-bit value (w2:w1:w0) mod p: S = (w1:w0) + w2 * EPS < 2^65
// (2^64 = EPS) as multiply-adds, then its carry c folded as c * EPS, which
// cannot wrap again (S - 2^64 <= 2^64 - 2^33 when c = 1). Every step but the
// carry read is a 32-bit multiply-add (FMA pipe).
__device__ __forceinline__ uint64_t reduce96(uint32_t w0, uint32_t w1, uint32_t w2) {
    uint32_t s0, s1, c;
    asm("mad.lo.cc.u32 %0, %3, %5, %4;\n\t"
        "madc.hi.cc.u32 %1, %3, %5, %6;\n\t"
        "addc.u32 %2, 0, 0;"
        : "=r"(s0), "=r"(s1), "=r"(c)
        : "r"(w2), "r"(w0), "r"(0xFFFFFFFFu), "r"(w1));
    asm("mad.lo.cc.u32 %0, %2, %3, %0;\n\t"
        "madc.hi.u32 %1, %2, %3, %1;"
        : "+r"(s0), "+r"(s1)
        : "r"(c), "r"(0xFFFFFFFFu));
    return pack(s0, s1);
}

// (w2:w1:w0) = x * k exactly, for a 32-bit k (four multiply-adds).
__device__ __forceinline__ void mul_wide_k32(uint64_t x, uint32_t k, uint32_t& w0, uint32_t& w1, uint32_t& w2) {
    asm("mul.lo.u32 %0, %3, %5;\n\t"
        "mul.hi.u32 %1, %3, %5;\n\t"
        "mad.lo.cc.u32 %1, %4, %5, %1;\n\t"
        "madc.hi.u32 %2, %4, %5, 0;"
        : "=r"(w0), "=r"(w1), "=r"(w2)
        : "r"(lo32(x)), "r"(hi32(x)), "r"(k));
}

// x * k mod p for a 32-bit k: the 96-bit product, reduced.
__device__ __forceinline__ uint64_t mul_k32(uint64_t x, uint32_t k) {
    uint32_t w0, w1, w2;
    mul_wide_k32(x, k, w0, w1, w2);
    return reduce96(w0, w1, w2);
}

// x * 2^S mod p for a compile-time 0 <= S < 96 (2^96 = -1, so every power of
// two is +-2^S with S in this range), from y = x * 2^(S mod 32) as three
// exact words (w2:w1:w0) placed S div 32 words up:
//   S < 32:  reduce96(w0, w1, w2)
//   S < 64:  words (w2:w1:w0:0): reduce128
//   S >= 64: w0 2^64 + w1 2^96 + w2 2^128 = w0 EPS - (w2:w1)
// (2^64 = EPS, 2^96 = -1, 2^128 = -2^32). Of the forms measured in the DFT's
// register butterflies, this mix of FMA-pipe and ALU-pipe work was fastest.
template <int S>
__device__ __forceinline__ uint64_t mul_2exp(uint64_t x) {
    static_assert(S >= 0 && S < 96, "exponent out of range");
    if constexpr (S == 0) {
        return x;
    } else if constexpr (S == 32) {
        return reduce96(0, lo32(x), hi32(x));
    } else if constexpr (S == 64) {
        return mul_k32(x, 0xFFFFFFFFu);
    } else {
        // y = x * 2^r as three words by funnel shifts (ALU pipe: this form
        // measured 1 % faster in the DFT than four multiply-adds)
        constexpr int r = S % 32;
        const uint32_t w0 = lo32(x) << r, w1 = __funnelshift_l(lo32(x), hi32(x), r), w2 = hi32(x) >> (32 - r);
        if constexpr (S < 32) {
            return reduce96(w0, w1, w2);
        } else if constexpr (S < 64) {
            return reduce128(0, w0, w1, w2);
        } else {
            uint32_t t0, t1;
            asm("mul.lo.u32 %0, %2, %3;\n\t"
                "mul.hi.u32 %1, %2, %3;"
                : "=r"(t0), "=r"(t1)
                : "r"(w0), "r"(0xFFFFFFFFu));
            return sub(pack(t0, t1), pack(w1, w2));
        }
    }
}

__device__ __forceinline__ uint64_t sqr(uint64_t a) { return mul(a, a); }

__device__ __forceinline__ uint64_t neg(uint64_t a) {
    uint64_t c = canon(a);
    return c == 0 ? 0 : GL_P - c;
}

__device__ __forceinline__ uint64_t pow(uint64_t a, uint64_t e) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = mul(r, a);
        a = mul(a, a);
        e >>= 1;
    }
    return r;
}

// x^(2^n) by n squarings.
__device__ __forceinline__ uint64_t sqn(uint64_t x, int n) {
    for (int i = 0; i < n; ++i) x = mul(x, x);
    return x;
}

// a^(p-2) = a^-1 (0 -> 0) by an addition chain: p - 2 = (2^31 - 1) 2^33 +
// (2^32 - 1), and t_k = a^(2^k - 1) doubles as t_{j+k} = t_j^(2^k) t_k. 64
// squarings and 9 products against 127 for square-and-multiply: the inverse
// is a single dependent chain, so its length is its latency.
__device__ __forceinline__ uint64_t inv(uint64_t a) {
    const uint64_t t2 = mul(sqr(a), a);           // 2^2 - 1
    const uint64_t t3 = mul(sqr(t2), a);          // 2^3 - 1
    const uint64_t t6 = mul(sqn(t3, 3), t3);      // 2^6 - 1
    const uint64_t t12 = mul(sqn(t6, 6), t6);     // 2^12 - 1
    const uint64_t t24 = mul(sqn(t12, 12), t12);  // 2^24 - 1
    const uint64_t t30 = mul(sqn(t24, 6), t6);    // 2^30 - 1
    const uint64_t t31 = mul(sqr(t30), a);        // 2^31 - 1
    const uint64_t t32 = mul(sqr(t31), a);        // 2^32 - 1
    return mul(sqn(t31, 33), t32);                // (2^31 - 1) 2^33 + 2^32 - 1
}

// ---------------------------------------------------------------- Fp3
struct fe3 {
    uint64_t c0, c1, c2;
};

__device__ __forceinline__ fe3 f3(uint64_t a, uint64_t b, uint64_t c) { return fe3{a, b, c}; }
__device__ __forceinline__ fe3 add3(fe3 a, fe3 b) { return fe3{add(a.c0, b.c0), add(a.c1, b.c1), add(a.c2, b.c2)}; }
__device__ __forceinline__ fe3 sub3(fe3 a, fe3 b) { return fe3{sub(a.c0, b.c0), sub(a.c1, b.c1), sub(a.c2, b.c2)}; }
__device__ __forceinline__ fe3 mulb3(fe3 a, uint64_t s) { return fe3{mul(a.c0, s), mul(a.c1, s), mul(a.c2, s)}; }

// Accumulate three 128-bit products and reduce once: sum overflow past 2^128
// folds 2^128 = EPS^2 mod p (same identity as goldilocks.rs dot_product_3).
__device__ __forceinline__ uint64_t dot3(uint64_t a0, uint64_t b0, uint64_t a1, uint64_t b1, uint64_t a2,
                                         uint64_t b2) {
    uint32_t s0, s1, s2, s3, t0, t1, t2, t3, ov;
    mul128(a0, b0, s0, s1, s2, s3);
    mul128(a1, b1, t0, t1, t2, t3);
    asm("add.cc.u32 %0, %0, %5;\n\t"
        "addc.cc.u32 %1, %1, %6;\n\t"
        "addc.cc.u32 %2, %2, %7;\n\t"
        "addc.cc.u32 %3, %3, %8;\n\t"
        "addc.u32 %4, 0, 0;"
        : "+r"(s0), "+r"(s1), "+r"(s2), "+r"(s3), "=r"(ov)
        : "r"(t0), "r"(t1), "r"(t2), "r"(t3));
    mul128(a2, b2, t0, t1, t2, t3);
    asm("add.cc.u32 %0, %0, %5;\n\t"
        "addc.cc.u32 %1, %1, %6;\n\t"
        "addc.cc.u32 %2, %2, %7;\n\t"
        "addc.cc.u32 %3, %3, %8;\n\t"
        "addc.u32 %4, %4, 0;"
        : "+r"(s0), "+r"(s1), "+r"(s2), "+r"(s3), "+r"(ov)
        : "r"(t0), "r"(t1), "r"(t2), "r"(t3));
    uint64_t r = reduce128(s0, s1, s2, s3);
    // EPS^2 = 2^64 - 2^33 + 1 < p; add it `ov` (0..2) times.
    const uint64_t EPS2 = 0xFFFFFFFE00000001ULL;
    if (ov) {
        r = add(r, EPS2);
        if (ov > 1) r = add(r, EPS2);
    }
    return r;
}

__device__ __forceinline__ fe3 mul3(fe3 a, fe3 b) {
    uint64_t b1_2 = add(b.c1, b.c1), b2_2 = add(b.c2, b.c2);
    return fe3{dot3(a.c0, b.c0, a.c1, b2_2, a.c2, b1_2), dot3(a.c0, b.c1, a.c1, b.c0, a.c2, b2_2),
               dot3(a.c0, b.c2, a.c1, b.c1, a.c2, b.c0)};
}

// ---------------------------------------------------------------- lazily reduced sums of products
// A sum of up to 2^32 products of two u64 is exact in 160 bits; it is reduced
// once at the end with 2^128 = -2^32 (mod p). One product then costs the
// 32-bit partial products plus a 5-limb carry chain, instead of a full
// reduction and a modular add.
struct wacc {
    uint32_t w0, w1, w2, w3, w4;
};

__device__ __forceinline__ wacc wzero() { return wacc{0, 0, 0, 0, 0}; }

__device__ __forceinline__ void wmac(wacc& a, uint64_t x, uint64_t y) {
    uint32_t t0, t1, t2, t3;
    mul128(x, y, t0, t1, t2, t3);
    asm("add.cc.u32 %0, %0, %5;\n\t"
        "addc.cc.u32 %1, %1, %6;\n\t"
        "addc.cc.u32 %2, %2, %7;\n\t"
        "addc.cc.u32 %3, %3, %8;\n\t"
        "addc.u32 %4, %4, 0;"
        : "+r"(a.w0), "+r"(a.w1), "+r"(a.w2), "+r"(a.w3), "+r"(a.w4)
        : "r"(t0), "r"(t1), "r"(t2), "r"(t3));
}

__device__ __forceinline__ uint64_t wreduce(const wacc& a) {
    return sub(reduce128(a.w0, a.w1, a.w2, a.w3), pack(0u, a.w4));
}

struct wacc3 {
    wacc c0, c1, c2;
};

__device__ __forceinline__ wacc3 wzero3() { return wacc3{wzero(), wzero(), wzero()}; }

// acc += g * t (ext3 times base)
__device__ __forceinline__ void wmacb3(wacc3& a, const fe3& g, uint64_t t) {
    wmac(a.c0, g.c0, t);
    wmac(a.c1, g.c1, t);
    wmac(a.c2, g.c2, t);
}

// acc += x * y (ext3 times ext3, w^3 = 2); y2 = (2 y1, 2 y2) precomputed by the caller.
__device__ __forceinline__ void wmac3(wacc3& a, const fe3& x, const fe3& y, uint64_t y1_2, uint64_t y2_2) {
    wmac(a.c0, x.c0, y.c0);
    wmac(a.c0, x.c1, y2_2);
    wmac(a.c0, x.c2, y1_2);
    wmac(a.c1, x.c0, y.c1);
    wmac(a.c1, x.c1, y.c0);
    wmac(a.c1, x.c2, y2_2);
    wmac(a.c2, x.c0, y.c2);
    wmac(a.c2, x.c1, y.c1);
    wmac(a.c2, x.c2, y.c0);
}

__device__ __forceinline__ fe3 wreduce3(const wacc3& a) { return fe3{wreduce(a.c0), wreduce(a.c1), wreduce(a.c2)}; }

// Norm-based inverse (extensions_goldilocks.rs:359-390). Returns 0 for 0.
__device__ __forceinline__ fe3 inv3(fe3 a) {
    uint64_t a0s = sqr(a.c0), a1s = sqr(a.c1), a2s = sqr(a.c2);
    uint64_t a0c = mul(a0s, a.c0), a1c = mul(a1s, a.c1), a2c = mul(a2s, a.c2);
    uint64_t a012 = mul(mul(a.c0, a.c1), a.c2);
    uint64_t a1c2 = add(a1c, a1c);
    uint64_t a2c4 = add(a2c, a2c);
    a2c4 = add(a2c4, a2c4);
    uint64_t six = add(add(a012, a012), a012);
    six = add(six, six);
    uint64_t norm = sub(add(add(a0c, a1c2), a2c4), six);
    uint64_t ni = inv(canon(norm));
    uint64_t a1a2 = mul(a.c1, a.c2), a0a1 = mul(a.c0, a.c1), a0a2 = mul(a.c0, a.c2);
    return fe3{mul(sub(a0s, add(a1a2, a1a2)), ni), mul(sub(add(a2s, a2s), a0a1), ni), mul(sub(a1s, a0a2), ni)};
}

__device__ __forceinline__ fe3 canon3(fe3 a) { return fe3{canon(a.c0), canon(a.c1), canon(a.c2)}; }

}  // namespace gl

// ---------------------------------------------------------------- host-side constexpr field math
// Used to bake roots of unity into kernels as compile-time constants.
namespace glc {
constexpr uint64_t P = GL_P;
constexpr uint64_t mul(uint64_t a, uint64_t b) {
    return (uint64_t)(((unsigned __int128)a * b) % P);
}
constexpr uint64_t pow(uint64_t a, uint64_t e) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = mul(r, a);
        a = mul(a, a);
        e >>= 1;
    }
    return r;
}
// Primitive 2^k-th root of unity, derived from the two-adic generator
// 1753635133440165772 exactly as traits.rs:83-95 does (repeated squaring).
constexpr uint64_t root(uint32_t log_n) {
    uint64_t r = 1753635133440165772ULL;
    for (uint32_t i = 0; i < 32 - log_n; i++) r = mul(r, r);
    return log_n == 0 ? 1 : r;
}
// The S in [0, 192) with 2^S = v (2 has order 192), or -1 when v is not a
// power of two. Every 64th root of unity is one: omega_64 is 2^39 here.
constexpr int log2_of(uint64_t v) {
    uint64_t c = 1;
    for (int s = 0; s < 192; ++s) {
        if (c == v) return s;
        c = mul(c, 2);
    }
    return -1;
}
constexpr uint64_t inv(uint64_t a) { return pow(a, P - 2); }
}  // namespace glc
