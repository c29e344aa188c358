/* A foreign (non-Python) host of the C ABI: commits a seeded trace through
 * sg_lde_commit from host memory, gathers two authentication paths, runs a
 * grinding search and prints the root, the paths' first siblings and the
 * nonce as hex, one per line. Built by the tests with plain gcc against
 * include/starkgpu.h and libstarkgpu.so. Exit status 0 on success, 1 on any
 * library error (printed from sg_last_error). */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "starkgpu.h"

static const uint64_t P = 0xFFFFFFFF00000001ULL;

static uint64_t mulmod(uint64_t a, uint64_t b) { return (uint64_t)(((unsigned __int128)a * b) % P); }
static uint64_t powmod(uint64_t a, uint64_t e) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = mulmod(r, a);
        a = mulmod(a, a);
        e >>= 1;
    }
    return r;
}

static int fail(const char* what) {
    fprintf(stderr, "%s: %s\n", what, sg_last_error());
    return 1;
}

int main(int argc, char** argv) {
    const uint64_t n = argc > 1 ? strtoull(argv[1], 0, 10) : 1024, m = argc > 2 ? strtoull(argv[2], 0, 10) : 20;
    const uint32_t blowup = 4;
    uint64_t* trace = malloc(n * m * 8);
    uint64_t* weights = malloc(n * 8);
    uint64_t x = 0x9E3779B97F4A7C15ULL;
    for (uint64_t i = 0; i < n * m; ++i) {  /* xorshift64 */
        x ^= x << 13;
        x ^= x >> 7;
        x ^= x << 17;
        trace[i] = x % P;
    }
    /* coset weights g^i / n, g = 3 */
    const uint64_t ninv = powmod(n % P, P - 2);
    uint64_t w = ninv;
    for (uint64_t i = 0; i < n; ++i) {
        weights[i] = w;
        w = mulmod(w, 3);
    }
    sg_ctx* ctx = 0;
    if (sg_ctx_create(0, 0, &ctx)) return fail("sg_ctx_create");
    sg_lde* lde = 0;
    uint8_t root[32];
    if (sg_lde_commit(ctx, 0, trace, 0, n, m, blowup, weights, 0, 0, &lde, root)) return fail("sg_lde_commit");
    sg_lde_info info;
    if (sg_lde_get_info(lde, &info)) return fail("sg_lde_get_info");
    for (int i = 0; i < 32; ++i) printf("%02x", root[i]);
    printf("\n");
    uint32_t pos[2] = {0, (uint32_t)(info.leaves_len - 1)};
    uint32_t* d_pos = 0;
    uint8_t* d_paths = 0;
    uint32_t depth = 0;
    while ((1ULL << depth) < info.leaves_len) ++depth;
    if (sg_dev_alloc(ctx, 0, sizeof(pos), (void**)&d_pos)) return fail("sg_dev_alloc");
    if (sg_dev_alloc(ctx, 0, 2ull * depth * 32, (void**)&d_paths)) return fail("sg_dev_alloc");
    if (sg_memcpy_h2d(ctx, 0, d_pos, pos, sizeof(pos))) return fail("sg_memcpy_h2d");
    if (sg_merkle_gather_paths(ctx, 0, info.d_nodes, info.leaves_len, d_pos, 2, d_paths)) return fail("paths");
    uint8_t* paths = malloc(2ull * depth * 32);
    if (sg_memcpy_d2h(ctx, 0, paths, d_paths, 2ull * depth * 32)) return fail("sg_memcpy_d2h");
    if (sg_stream_sync(ctx, 0)) return fail("sg_stream_sync");
    for (int q = 0; q < 2; ++q) {
        for (int i = 0; i < 32; ++i) printf("%02x", paths[(uint64_t)q * depth * 32 + i]);
        printf("\n");
    }
    uint64_t lanes[4];
    for (int i = 0; i < 4; ++i) {
        lanes[i] = 0;
        for (int b = 0; b < 8; ++b) lanes[i] |= (uint64_t)root[8 * i + b] << (8 * b);
    }
    uint64_t nonce = 0;
    if (sg_grind(ctx, 0, lanes, 12, &nonce)) return fail("sg_grind");
    printf("%llu\n", (unsigned long long)nonce);
    sg_dev_free(ctx, 0, d_pos, sizeof(pos));
    sg_dev_free(ctx, 0, d_paths, 2ull * depth * 32);
    sg_lde_free(ctx, lde);
    sg_ctx_destroy(ctx);
    free(trace);
    free(weights);
    free(paths);
    return 0;
}
