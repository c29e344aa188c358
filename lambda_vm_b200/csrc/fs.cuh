// The Fiat-Shamir transcript state and its operations, compiled for both the
// host and the device from one definition, so a transcript can be advanced by
// device threads (the FRI commit phase, grinding and query sampling of a table
// run without host round trips) and handed back to the host bit for bit.
//
// Semantics restate crypto/crypto/src/fiat_shamir/default_transcript.rs:31-146:
// a Keccak-256 hash chain; sample() = finalize, byte-reverse, restart the
// hasher on the reversed digest; field and index sampling read big-endian u64
// candidates from a 32-byte buffer (4 per squeeze), invalidated by every
// absorb; rejection sampling below p; sample_u64 uses the modulo threshold.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#include "keccak.cuh"
#define FS_HD __host__ __device__
#else
#define FS_HD
#endif

namespace fs {

constexpr uint64_t P = 0xFFFFFFFF00000001ULL;

struct State {
    uint64_t st[25];     // Keccak-256 sponge lanes
    uint8_t buf[136];    // pending rate bytes
    uint32_t pos;        // bytes pending in buf
    uint8_t out_buf[32]; // duplex sample buffer
    uint32_t out_pos;    // next unread byte of out_buf (32 = empty)
};

// Keccak-f[1600] on the host (transcript.cu); the device uses the register
// implementation of keccak.cuh.
void host_permute(uint64_t st[25]);

FS_HD inline void permute(uint64_t st[25]) {
#ifdef __CUDA_ARCH__
    uint64_t s[25];
    for (int i = 0; i < 25; ++i) s[i] = st[i];
    kc::permute(s);
    for (int i = 0; i < 25; ++i) st[i] = s[i];
#else
    host_permute(st);
#endif
}

FS_HD inline void copy_bytes(uint8_t* d, const uint8_t* s, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i) d[i] = s[i];
}

FS_HD inline void reset_hasher(State& t) {
    for (int i = 0; i < 25; ++i) t.st[i] = 0;
    t.pos = 0;
}

FS_HD inline void absorb_block(uint64_t st[25], const uint8_t* b) {
    for (int i = 0; i < 17; ++i) {
        uint64_t v = 0;
        for (int k = 7; k >= 0; --k) v = (v << 8) | b[8 * i + k];  // little-endian lanes
        st[i] ^= v;
    }
    permute(st);
}

FS_HD inline void update(State& t, const uint8_t* d, uint64_t n) {
    while (n) {
        uint64_t c = 136 - t.pos;
        if (c > n) c = n;
        copy_bytes(t.buf + t.pos, d, (uint32_t)c);
        t.pos += (uint32_t)c;
        d += c;
        n -= c;
        if (t.pos == 136) {
            absorb_block(t.st, t.buf);
            t.pos = 0;
        }
    }
}

// Digest of everything absorbed so far (the hasher itself is not advanced).
FS_HD inline void final_digest(const State& t, uint8_t out[32]) {
    uint64_t st[25];
    uint8_t b[136];
    for (int i = 0; i < 25; ++i) st[i] = t.st[i];
    for (uint32_t i = 0; i < 136; ++i) b[i] = i < t.pos ? t.buf[i] : 0;
    b[t.pos] ^= 0x01;
    b[135] ^= 0x80;
    absorb_block(st, b);
    for (int i = 0; i < 4; ++i)
        for (int k = 0; k < 8; ++k) out[8 * i + k] = (uint8_t)(st[i] >> (8 * k));
}

FS_HD inline void init(State& t, const uint8_t* d, uint64_t n) {
    reset_hasher(t);
    for (int i = 0; i < 32; ++i) t.out_buf[i] = 0;
    t.out_pos = 32;
    update(t, d, n);
}

FS_HD inline void append(State& t, const uint8_t* d, uint64_t n) {
    t.out_pos = 32;
    update(t, d, n);
}

FS_HD inline uint64_t canon(uint64_t a) { return a >= P ? a - P : a; }

FS_HD inline void append_u64_be(State& t, uint64_t v) {
    uint8_t b[8];
    for (int i = 0; i < 8; ++i) b[i] = (uint8_t)(v >> (56 - 8 * i));
    append(t, b, 8);
}

FS_HD inline void append_ext3(State& t, const uint64_t v[3]) {
    uint8_t b[24];
    for (int k = 0; k < 3; ++k) {
        const uint64_t c = canon(v[k]);
        for (int i = 0; i < 8; ++i) b[8 * k + i] = (uint8_t)(c >> (56 - 8 * i));
    }
    append(t, b, 24);
}

FS_HD inline void sample(State& t, uint8_t out[32]) {
    uint8_t d[32];
    final_digest(t, d);
    for (int i = 0; i < 32; ++i) out[i] = d[31 - i];
    reset_hasher(t);
    update(t, out, 32);
    t.out_pos = 32;
}

FS_HD inline uint64_t next_u64(State& t) {
    if (t.out_pos + 8 > 32) {
        uint8_t s[32];
        sample(t, s);
        copy_bytes(t.out_buf, s, 32);
        t.out_pos = 0;
    }
    uint64_t v = 0;
    for (int i = 0; i < 8; ++i) v = (v << 8) | t.out_buf[t.out_pos + i];
    t.out_pos += 8;
    return v;
}

FS_HD inline uint64_t sample_base(State& t) {
    for (;;) {
        const uint64_t c = next_u64(t);
        if (c < P) return c;
    }
}

FS_HD inline void sample_ext3(State& t, uint64_t out[3]) {
    for (int i = 0; i < 3; ++i) out[i] = sample_base(t);
}

FS_HD inline uint64_t sample_u64(State& t, uint64_t upper) {
    if (upper == 0) return 0;
    const uint64_t thr = (0 - upper) % upper;
    for (;;) {
        const uint64_t c = next_u64(t);
        if (c >= thr) return c % upper;
    }
}

}  // namespace fs

// The library's transcript handle: exactly the shared state.
struct sg_transcript {
    fs::State s;
};
