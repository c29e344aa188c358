// keccak-f[1600] constants, and the KECCAK chip table's constraints as a
// hand-written kernel.
//
// The KECCAK table (lambda_vm_b200/rv64_air.py KeccakAir) has 2605 columns and
// 3383 base-field constraints of a few regular shapes (bit checks, XORs of
// three bits, the parity of five, 16-bit limbs of XORed or chi-ed bits). The
// generic constraint walk spends ~120 instructions a program node on them;
// this kernel evaluates the same polynomials directly, one thread per LDE
// row, and folds them into the composition under the same constraint indices
// (the KeccakAir emission order; the kernel's own order keeps column reads
// few), so its sum equals the walk's exactly
// (field arithmetic is exact: any evaluation of a polynomial gives the same
// value). The table's LogUp constraints come from its descriptor
// (k_logup_constraints).
#pragma once

#include <stdint.h>

#include "gl.cuh"

namespace sg {

// keccak-f[1600]'s round constants and rotation offsets, derived from their
// definitions in FIPS 202 (the rc(t) LFSR over x^8 + x^6 + x^5 + x^4 + 1, the
// (x, y) -> (y, 2x + 3y) walk), for the host executor and the kernels.
struct KeccakTables {
    uint64_t rc[24];
    int rot[25];  // by lane x + 5y
    KeccakTables() {
        auto rc_bit = [](int t) {
            if (t % 255 == 0) return 1u;
            unsigned r = 1;
            for (int i = 0; i < t % 255; ++i) {
                r <<= 1;
                if (r & 0x100) r ^= 0x171;
            }
            return r & 1u;
        };
        for (int ir = 0; ir < 24; ++ir) {
            uint64_t c = 0;
            for (int j = 0; j < 7; ++j) c |= (uint64_t)rc_bit(j + 7 * ir) << ((1 << j) - 1);
            rc[ir] = c;
        }
        rot[0] = 0;
        int x = 1, y = 0;
        for (int t = 0; t < 24; ++t) {
            rot[x + 5 * y] = ((t + 1) * (t + 2) / 2) % 64;
            const int nx = y, ny = (2 * x + 3 * y) % 5;
            x = nx, y = ny;
        }
    }
};
inline const KeccakTables& keccak_tables() {
    static const KeccakTables t;
    return t;
}
struct KeccakConsts {
    uint64_t rc[24];
    int rot[25];
};
inline KeccakConsts keccak_consts() {
    KeccakConsts k;
    for (int i = 0; i < 24; ++i) k.rc[i] = keccak_tables().rc[i];
    for (int i = 0; i < 25; ++i) k.rot[i] = keccak_tables().rot[i];
    return k;
}

// Column layout of the KECCAK table (rv64_air.py).
constexpr uint32_t KAIR_R = 0, KAIR_A = 24, KAIR_C = 124, KAIR_CP = 444, KAIR_AP = 764, KAIR_OUT = 2364,
                   KAIR_B00 = 2464, KAIR_BASE = 2528, KAIR_CLK = 2529, KAIR_TOLD = 2530, KAIR_TD = 2555,
                   KAIR_WIDTH = 2605, KAIR_CONSTRAINTS = 3383;

// The cells a KECCAK-table row reads: the main LDE column-major (cm, m x rows)
// or row-major (rm, rows x m).
struct KRow {
    const uint64_t* cm;
    const uint64_t* rm;
    uint64_t rows, row, rn;  // this row and its frame successor
    __device__ __forceinline__ uint64_t at(uint64_t r, uint32_t col) const {
        return cm ? cm[(uint64_t)col * rows + r] : rm[r * KAIR_WIDTH + col];
    }
    __device__ __forceinline__ uint64_t M(uint32_t col) const { return at(row, col); }
    __device__ __forceinline__ uint64_t N(uint32_t col) const { return at(rn, col); }
};

__device__ __forceinline__ uint64_t kbool(uint64_t v) { return gl::mul(v, gl::sub(v, 1)); }
__device__ __forceinline__ uint64_t kxor2(uint64_t x, uint64_t y) {
    const uint64_t p = gl::mul(x, y);
    return gl::sub(gl::add(x, y), gl::add(p, p));
}
// x ^ y ^ z of bits, as x' + w - 2 x' w with w = y ^ z
__device__ __forceinline__ uint64_t kxor3(uint64_t x, uint64_t y, uint64_t z) { return kxor2(x, kxor2(y, z)); }
__device__ __forceinline__ uint64_t kdbl(uint64_t v) { return gl::add(v, v); }

// Where a kernel puts each constraint: mode 0 folds beta_c C_c into the
// row's sum (kept unreduced, reduced once per row by total()); mode 1 writes
// C_c to out[c * rows + row]. c is the constraint's index in the table's
// program: given, or the next one after the previous put.
struct KSink {
    const uint64_t* beta;
    int mode;
    uint64_t* out;
    uint64_t rows, row;
    gl::wacc3 sum;
    uint32_t next;
    __device__ __forceinline__ void put(uint64_t v) { put(next, v); }
    __device__ __forceinline__ gl::fe3 total() const { return gl::wreduce3(sum); }
    __device__ __forceinline__ void put(uint32_t c, uint64_t v) {
        next = c + 1;
        if (mode == 1) {
            uint64_t* o = out + 3 * ((uint64_t)c * rows + row);
            o[0] = gl::canon(v), o[1] = 0, o[2] = 0;
        } else {
            const gl::fe3 b{__ldg(beta + 3 * c), __ldg(beta + 3 * c + 1), __ldg(beta + 3 * c + 2)};
            gl::wmacb3(sum, b, v);
        }
    }
};

// chi's output bit z of lane (X, Y): B[X][Y] ^ (~B[X+1][Y] & B[X+2][Y]), where
// B[X][Y] = rot(A'[x][y], r[x][y]) with (X, Y) = (y, 2x + 3y): y = X, x = 3 (Y - 3X) mod 5.
__device__ __forceinline__ uint64_t kB(const KRow& w, const KeccakConsts& kc, int X, int Y, int z) {
    const int y = X, x = (3 * ((Y - 3 * X) % 5 + 5)) % 5;
    const int rr = kc.rot[x + 5 * y];
    return w.M(KAIR_AP + 64 * (x + 5 * y) + ((z - rr) & 63));
}
__device__ __forceinline__ uint64_t kchi(const KRow& w, const KeccakConsts& kc, int X, int Y, int z) {
    const uint64_t b0 = kB(w, kc, X, Y, z), b1 = kB(w, kc, (X + 1) % 5, Y, z), b2 = kB(w, kc, (X + 2) % 5, Y, z);
    return kxor2(b0, gl::mul(gl::sub(1, b1), b2));
}

// One thread per LDE row; mode 0 writes the row's sum over the 3383
// constraints to out (rows ext3), mode 1 every constraint's value. The
// constraints are evaluated in an order that reads each column few times
// (the A' bits twice: once per (x, z) with C, C' and the A limbs, once per
// (Y, z) for chi's five lanes) and folded under their indices in the table's
// program:
//   0..23 round flags boolean, 24 their sum boolean;
//   25 + 7 (64 x + z) + {0: C, 1: C', 2 + y: A'[x + 5y]} booleans;
//   2265 + z lane-0-before-iota bits boolean;
//   2329 + 2 (64 x + z) + {0: C' = C ^ C[x-1] ^ C[x+1] rotated, 1: parity};
//   2969 + 5 (4 x + l) + y: A[x + 5y] limb l from A' ^ C ^ C';
//   3069 + 4 (5 X + Y - 1) + l: OUT limb l of lane (X, Y) != (0, 0) from chi;
//   3165 + z: lane 0's chi bit; 3229 + l: lane 0's OUT limb after iota;
//   3233.. the transitions and the timestamp gaps, in program order.
static __global__ void k_keccak_constraints(const uint64_t* __restrict__ cm, const uint64_t* __restrict__ rm, uint64_t rows,
                                     uint64_t next_step, KeccakConsts kc, const uint64_t* __restrict__ beta, int mode,
                                     uint64_t* __restrict__ out) {
    for (uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; row < rows;
         row += (uint64_t)gridDim.x * blockDim.x) {
        KRow w{cm, rm, rows, row, row + next_step >= rows ? row + next_step - rows : row + next_step};
        KSink s{beta, mode, out, rows, row, gl::wzero3(), 0};
        uint64_t act = 0;
        for (int i = 0; i < 24; ++i) {
            const uint64_t r = w.M(KAIR_R + i);
            s.put(i, kbool(r));
            act = gl::add(act, r);
        }
        s.put(24, kbool(act));
        // per (x, z): the C, C' and A' bits, theta, and the A limbs (z descending inside a limb)
        for (int x = 0; x < 5; ++x)
            for (int l = 0; l < 4; ++l) {
                uint64_t acc[5] = {0, 0, 0, 0, 0};
                for (int i = 15; i >= 0; --i) {
                    const int z = 16 * l + i;
                    const uint32_t b = 25 + 7 * (64 * x + z), t = 2329 + 2 * (64 * x + z);
                    const uint64_t c = w.M(KAIR_C + 64 * x + z), cp = w.M(KAIR_CP + 64 * x + z);
                    uint64_t ap[5];
#pragma unroll
                    for (int y = 0; y < 5; ++y) ap[y] = w.M(KAIR_AP + 64 * (x + 5 * y) + z);
                    s.put(b, kbool(c));
                    s.put(b + 1, kbool(cp));
#pragma unroll
                    for (int y = 0; y < 5; ++y) s.put(b + 2 + y, kbool(ap[y]));
                    s.put(t, gl::sub(cp, kxor3(c, w.M(KAIR_C + 64 * ((x + 4) % 5) + z),
                                               w.M(KAIR_C + 64 * ((x + 1) % 5) + ((z + 63) & 63)))));
                    uint64_t par = 0;
#pragma unroll
                    for (int y = 0; y < 5; ++y) par = gl::add(par, ap[y]);
                    par = gl::sub(par, cp);
                    s.put(t + 1, gl::mul(gl::mul(par, gl::sub(par, 2)), gl::sub(par, 4)));
#pragma unroll
                    for (int y = 0; y < 5; ++y) acc[y] = gl::add(kdbl(acc[y]), kxor3(ap[y], c, cp));
                }
#pragma unroll
                for (int y = 0; y < 5; ++y) s.put(2969 + 5 * (4 * x + l) + y, gl::sub(w.M(KAIR_A + 4 * (x + 5 * y) + l), acc[y]));
            }
        for (int z = 0; z < 64; ++z) s.put(2265 + z, kbool(w.M(KAIR_B00 + z)));
        // chi per output row Y: the five lanes' rho-pi bits at z, each read once
        for (int Y = 0; Y < 5; ++Y)
            for (int l = 0; l < 4; ++l) {
                uint64_t acc[5] = {0, 0, 0, 0, 0};
                for (int i = 15; i >= 0; --i) {
                    const int z = 16 * l + i;
                    uint64_t bb[5], ch[5];
#pragma unroll
                    for (int X = 0; X < 5; ++X) bb[X] = kB(w, kc, X, Y, z);
#pragma unroll
                    for (int X = 0; X < 5; ++X) ch[X] = kxor2(bb[X], gl::mul(gl::sub(1, bb[(X + 1) % 5]), bb[(X + 2) % 5]));
#pragma unroll
                    for (int X = 0; X < 5; ++X) acc[X] = gl::add(kdbl(acc[X]), ch[X]);
                    if (Y == 0) s.put(3165 + z, gl::sub(w.M(KAIR_B00 + z), ch[0]));
                }
#pragma unroll
                for (int X = 0; X < 5; ++X)
                    if (X || Y)
                        s.put(3069 + 4 * (5 * X + Y - 1) + l, gl::sub(w.M(KAIR_OUT + 4 * (X + 5 * Y) + l), acc[X]));
            }
        // lane 0 after iota with the flags' round constant
        for (int l = 0; l < 4; ++l) {
            uint64_t acc = 0;
            for (int i = 15; i >= 0; --i) {
                const int z = 16 * l + i;
                uint64_t rcz = 0;
                bool any = false;
                for (int ir = 0; ir < 24; ++ir)
                    if ((kc.rc[ir] >> z) & 1) rcz = gl::add(rcz, w.M(KAIR_R + ir)), any = true;
                const uint64_t b = w.M(KAIR_B00 + z);
                acc = gl::add(kdbl(acc), any ? kxor2(b, rcz) : b);
            }
            s.put(3229 + l, gl::sub(w.M(KAIR_OUT + l), acc));
        }
        // transitions inside a permutation
        uint32_t c = 3233;
        uint64_t g = 0;
        for (int i = 0; i < 23; ++i) {
            const uint64_t r = w.M(KAIR_R + i);
            s.put(c++, gl::sub(w.N(KAIR_R + i + 1), r));
            g = gl::add(g, r);
        }
        for (int k = 0; k < 100; ++k) s.put(c++, gl::mul(g, gl::sub(w.N(KAIR_A + k), w.M(KAIR_OUT + k))));
        s.put(c++, gl::mul(g, gl::sub(w.N(KAIR_BASE), w.M(KAIR_BASE))));
        s.put(c++, gl::mul(g, gl::sub(w.N(KAIR_CLK), w.M(KAIR_CLK))));
        // reads of earlier timestamps
        const uint64_t r0 = w.M(KAIR_R), clk = w.M(KAIR_CLK);
        for (int i = 0; i < 25; ++i) {
            const uint64_t gap = gl::sub(gl::sub(clk, w.M(KAIR_TOLD + i)), 1);
            const uint64_t v = gl::add(w.M(KAIR_TD + 2 * i), gl::mul(1ull << 16, w.M(KAIR_TD + 2 * i + 1)));
            s.put(c++, gl::mul(r0, gl::sub(gap, v)));
        }
        if (mode == 0) {
            const gl::fe3 sum = s.total();
            uint64_t* o = out + 3 * row;
            o[0] = sum.c0, o[1] = sum.c1, o[2] = sum.c2;
        }
    }
}

}  // namespace sg
