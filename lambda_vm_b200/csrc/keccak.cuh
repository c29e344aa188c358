// Keccak-f[1600] for sm_100a with the whole 25-lane state in registers.
// Rounds are fully unrolled with compile-time lane indices, so theta/rho/pi/chi
// become straight-line LOP3 (3-input XOR / ANDNOT-XOR) and funnel-shift
// rotations on the INT pipes; pi is pure register renaming.
// Sponge framing is original Keccak-256 (pad 0x01 ... 0x80, rate 136 bytes),
// the variant the reference's sha3::Keccak256 computes.
#pragma once
#include <stdint.h>

namespace kc {

__device__ __constant__ static const uint64_t RC[24] = {
    0x0000000000000001ULL, 0x0000000000008082ULL, 0x800000000000808aULL, 0x8000000080008000ULL,
    0x000000000000808bULL, 0x0000000080000001ULL, 0x8000000080008081ULL, 0x8000000000008009ULL,
    0x000000000000008aULL, 0x0000000000000088ULL, 0x0000000080008009ULL, 0x000000008000000aULL,
    0x000000008000808bULL, 0x800000000000008bULL, 0x8000000000008089ULL, 0x8000000000008003ULL,
    0x8000000000008002ULL, 0x8000000000000080ULL, 0x000000000000800aULL, 0x800000008000000aULL,
    0x8000000080008081ULL, 0x8000000000008080ULL, 0x0000000080000001ULL, 0x8000000080008008ULL};

template <int R>
__device__ __forceinline__ uint64_t rotl(uint64_t x) {
    if constexpr (R == 0) {
        return x;
    } else if constexpr (R == 32) {
        return (x << 32) | (x >> 32);
    } else {
        uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32), rl, rh;
        if constexpr (R < 32) {
            rh = __funnelshift_l(lo, hi, R);
            rl = __funnelshift_l(hi, lo, R);
        } else {
            rh = __funnelshift_l(hi, lo, R - 32);
            rl = __funnelshift_l(lo, hi, R - 32);
        }
        return ((uint64_t)rh << 32) | rl;
    }
}

__device__ __forceinline__ uint64_t xor5(uint64_t a, uint64_t b, uint64_t c, uint64_t d, uint64_t e) {
    return a ^ b ^ c ^ d ^ e;
}

// chi: a ^ (~b & c)
__device__ __forceinline__ uint64_t chi(uint64_t a, uint64_t b, uint64_t c) { return a ^ ((~b) & c); }

// One Keccak-f[1600] permutation. Lane (x, y) lives at s[x + 5y]; rho/pi
// destinations B[y + 5((2x+3y) mod 5)] and rotation offsets are the Keccak
// specification's, written out so every index is a compile-time constant.
__device__ __forceinline__ void permute(uint64_t s[25]) {
    // The round loop stays rolled: a fully unrolled permutation is ~5k
    // instructions and thrashes the instruction cache once inlined at several
    // call sites; within a round every lane index is still a constant.
#pragma unroll 1
    for (int round = 0; round < 24; ++round) {
        // theta: A[x,y] ^= C[x-1] ^ rotl1(C[x+1]), written as one 3-input XOR
        // per lane half (a single LOP3) instead of materialising D first.
        uint64_t C[5], R[5];
#pragma unroll
        for (int x = 0; x < 5; ++x) C[x] = xor5(s[x], s[x + 5], s[x + 10], s[x + 15], s[x + 20]);
#pragma unroll
        for (int x = 0; x < 5; ++x) R[x] = rotl<1>(C[x]);
#define D(x) C[((x) + 4) % 5] ^ R[((x) + 1) % 5]
        uint64_t B[25];
        // B[y + 5*((2x+3y)%5)] = rot(A[x+5y] ^ D[x], r[x][y])
        B[0] = s[0] ^ D(0);
        B[10] = rotl<1>(s[1] ^ D(1));
        B[20] = rotl<62>(s[2] ^ D(2));
        B[5] = rotl<28>(s[3] ^ D(3));
        B[15] = rotl<27>(s[4] ^ D(4));
        B[16] = rotl<36>(s[5] ^ D(0));
        B[1] = rotl<44>(s[6] ^ D(1));
        B[11] = rotl<6>(s[7] ^ D(2));
        B[21] = rotl<55>(s[8] ^ D(3));
        B[6] = rotl<20>(s[9] ^ D(4));
        B[7] = rotl<3>(s[10] ^ D(0));
        B[17] = rotl<10>(s[11] ^ D(1));
        B[2] = rotl<43>(s[12] ^ D(2));
        B[12] = rotl<25>(s[13] ^ D(3));
        B[22] = rotl<39>(s[14] ^ D(4));
        B[23] = rotl<41>(s[15] ^ D(0));
        B[8] = rotl<45>(s[16] ^ D(1));
        B[18] = rotl<15>(s[17] ^ D(2));
        B[3] = rotl<21>(s[18] ^ D(3));
        B[13] = rotl<8>(s[19] ^ D(4));
        B[14] = rotl<18>(s[20] ^ D(0));
        B[24] = rotl<2>(s[21] ^ D(1));
        B[9] = rotl<61>(s[22] ^ D(2));
        B[19] = rotl<56>(s[23] ^ D(3));
        B[4] = rotl<14>(s[24] ^ D(4));
#pragma unroll
        for (int y = 0; y < 5; ++y) {
#pragma unroll
            for (int x = 0; x < 5; ++x) s[x + 5 * y] = chi(B[x + 5 * y], B[(x + 1) % 5 + 5 * y], B[(x + 2) % 5 + 5 * y]);
        }
#undef D
        s[0] ^= RC[round];
    }
}

__device__ __forceinline__ uint64_t bswap64(uint64_t x) {
    uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
    return ((uint64_t)__byte_perm(lo, 0, 0x0123) << 32) | __byte_perm(hi, 0, 0x0123);
}

// Lane-granular Keccak-256 absorber: every input here is a whole number of
// 8-byte lanes (field elements, 32-byte digests), so absorption XORs lanes
// directly and permutes every 17 lanes.
struct Sponge {
    uint64_t s[25];
    uint32_t pos;
    __device__ __forceinline__ void init() {
#pragma unroll
        for (int i = 0; i < 25; ++i) s[i] = 0;
        pos = 0;
    }
    __device__ __forceinline__ void lane(uint64_t v) {
        // Runtime index into a register array would spill; dispatch via unrolled compare.
#pragma unroll
        for (int i = 0; i < 17; ++i)
            if (pos == (uint32_t)i) s[i] ^= v;
        if (++pos == 17) {
            permute(s);
            pos = 0;
        }
    }
    __device__ __forceinline__ void finish() {
#pragma unroll
        for (int i = 0; i < 17; ++i)
            if (pos == (uint32_t)i) s[i] ^= 0x01ULL;
        s[16] ^= 0x8000000000000000ULL;
        permute(s);
    }
};

}  // namespace kc
