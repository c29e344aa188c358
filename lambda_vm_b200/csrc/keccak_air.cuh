// keccak-f[1600] constants, and the KECCAK chip table's constraints as a
// hand-written kernel.
//
// The KECCAK table (lambda_vm_b200/rv64_air.py KeccakAir) has 2605 columns and
// 3383 base-field constraints of a few regular shapes (bit checks, XORs of
// three bits, the parity of five, 16-bit limbs of XORed or chi-ed bits). The
// generic constraint walk spends ~120 instructions a program node on them;
// this kernel evaluates the same polynomials directly, one thread per LDE
// row, and folds them into the composition with the same constraint indices
// (the KeccakAir emission order), so its sum equals the walk's exactly
// (field arithmetic is exact: any evaluation of a polynomial gives the same
// value). The LogUp constraints of the table stay with the walk.
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

// Where the kernel puts each constraint: mode 0 folds beta_c C_c into the
// row's sum; mode 1 writes C_c to out[c * rows + row].
struct KSink {
    const uint64_t* beta;
    int mode;
    uint64_t* out;
    uint64_t rows, row;
    uint32_t c;
    gl::fe3 sum;
    __device__ __forceinline__ void put(uint64_t v) {
        if (mode == 1) {
            uint64_t* o = out + 3 * ((uint64_t)c * rows + row);
            o[0] = gl::canon(v), o[1] = 0, o[2] = 0;
        } else {
            const gl::fe3 b{__ldg(beta + 3 * c), __ldg(beta + 3 * c + 1), __ldg(beta + 3 * c + 2)};
            sum = gl::add3(sum, gl::mulb3(b, v));
        }
        ++c;
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
// constraints to out (rows ext3), mode 1 every constraint's value.
static __global__ void k_keccak_constraints(const uint64_t* __restrict__ cm, const uint64_t* __restrict__ rm, uint64_t rows,
                                     uint64_t next_step, KeccakConsts kc, const uint64_t* __restrict__ beta, int mode,
                                     uint64_t* __restrict__ out) {
    for (uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; row < rows;
         row += (uint64_t)gridDim.x * blockDim.x) {
        KRow w{cm, rm, rows, row, row + next_step >= rows ? row + next_step - rows : row + next_step};
        KSink s{beta, mode, out, rows, row, 0, gl::fe3{0, 0, 0}};
        // bit checks: the round flags and their sum, C, C', A' per (x, z), lane 0 before iota
        uint64_t act = 0;
        for (int i = 0; i < 24; ++i) {
            const uint64_t r = w.M(KAIR_R + i);
            s.put(kbool(r));
            act = gl::add(act, r);
        }
        s.put(kbool(act));
        for (int x = 0; x < 5; ++x)
            for (int z = 0; z < 64; ++z) {
                s.put(kbool(w.M(KAIR_C + 64 * x + z)));
                s.put(kbool(w.M(KAIR_CP + 64 * x + z)));
                for (int y = 0; y < 5; ++y) s.put(kbool(w.M(KAIR_AP + 64 * (x + 5 * y) + z)));
            }
        for (int z = 0; z < 64; ++z) s.put(kbool(w.M(KAIR_B00 + z)));
        // theta: C' = C ^ C[x-1] ^ rot(C[x+1], 1); the five A' bits and C' have even parity
        for (int x = 0; x < 5; ++x)
            for (int z = 0; z < 64; ++z) {
                const uint64_t cp = w.M(KAIR_CP + 64 * x + z);
                s.put(gl::sub(cp, kxor3(w.M(KAIR_C + 64 * x + z), w.M(KAIR_C + 64 * ((x + 4) % 5) + z),
                                        w.M(KAIR_C + 64 * ((x + 1) % 5) + ((z + 63) & 63)))));
                uint64_t t = 0;
                for (int y = 0; y < 5; ++y) t = gl::add(t, w.M(KAIR_AP + 64 * (x + 5 * y) + z));
                t = gl::sub(t, cp);
                s.put(gl::mul(gl::mul(t, gl::sub(t, 2)), gl::sub(t, 4)));
            }
        // A's limbs are the bits A' ^ C ^ C' (lanes of a column innermost)
        for (int x = 0; x < 5; ++x)
            for (int l = 0; l < 4; ++l)
                for (int y = 0; y < 5; ++y) {
                    uint64_t acc = 0;
                    for (int i = 15; i >= 0; --i) {
                        const int z = 16 * l + i;
                        acc = gl::add(kdbl(acc), kxor3(w.M(KAIR_AP + 64 * (x + 5 * y) + z), w.M(KAIR_C + 64 * x + z),
                                                       w.M(KAIR_CP + 64 * x + z)));
                    }
                    s.put(gl::sub(w.M(KAIR_A + 4 * (x + 5 * y) + l), acc));
                }
        // OUT's limbs (lanes other than 0) are chi of rho-pi of A'
        for (int x = 0; x < 5; ++x)
            for (int y = 0; y < 5; ++y) {
                if (x == 0 && y == 0) continue;
                for (int l = 0; l < 4; ++l) {
                    uint64_t acc = 0;
                    for (int i = 15; i >= 0; --i) acc = gl::add(kdbl(acc), kchi(w, kc, x, y, 16 * l + i));
                    s.put(gl::sub(w.M(KAIR_OUT + 4 * (x + 5 * y) + l), acc));
                }
            }
        // lane 0 before iota, bit by bit; then iota with the flags' round constant
        for (int z = 0; z < 64; ++z) s.put(gl::sub(w.M(KAIR_B00 + z), kchi(w, kc, 0, 0, z)));
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
            s.put(gl::sub(w.M(KAIR_OUT + l), acc));
        }
        // transitions inside a permutation
        uint64_t g = 0;
        for (int i = 0; i < 23; ++i) {
            const uint64_t r = w.M(KAIR_R + i);
            s.put(gl::sub(w.N(KAIR_R + i + 1), r));
            g = gl::add(g, r);
        }
        for (int c = 0; c < 100; ++c) s.put(gl::mul(g, gl::sub(w.N(KAIR_A + c), w.M(KAIR_OUT + c))));
        s.put(gl::mul(g, gl::sub(w.N(KAIR_BASE), w.M(KAIR_BASE))));
        s.put(gl::mul(g, gl::sub(w.N(KAIR_CLK), w.M(KAIR_CLK))));
        // reads of earlier timestamps
        const uint64_t r0 = w.M(KAIR_R), clk = w.M(KAIR_CLK);
        for (int i = 0; i < 25; ++i) {
            const uint64_t gap = gl::sub(gl::sub(clk, w.M(KAIR_TOLD + i)), 1);
            const uint64_t v = gl::add(w.M(KAIR_TD + 2 * i), gl::mul(1ull << 16, w.M(KAIR_TD + 2 * i + 1)));
            s.put(gl::mul(r0, gl::sub(gap, v)));
        }
        if (mode == 0) {
            uint64_t* o = out + 3 * row;
            o[0] = s.sum.c0, o[1] = s.sum.c1, o[2] = s.sum.c2;
        }
    }
}

}  // namespace sg
