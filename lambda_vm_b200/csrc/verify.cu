// Batched proof verification: the query phase of the STARK verifier for many
// tables of many proofs in one launch (crypto/stark/src/verifier.rs
// multi_verify :1178-1430, step 3 of verify: the openings' Merkle paths, the
// DEEP composition values at the opened rows, the FRI fold chain and the
// terminal polynomial).
//
// The transcript is a serial hash chain, so the host replays it per table
// (lambda_vm_b200/verifier.py) and hands the derived values in; what remains
// is independent per (table, query) and is one thread each here. A thread
// hashes its three row-pair leaves (every element canonical and big-endian,
// crypto/stark/src/commitment.rs:52-107), walks their authentication paths
// (merkle_tree/utils.rs:68-96 node rule), forms the DEEP values at both
// opened rows, then folds through every FRI layer checking the opened pair
// and its path (fri/mod.rs:153-205), and evaluates the terminal polynomial
// (fri/terminal.rs:72-103). Field equality is tested on canonical values.
#include <string.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "gl.cuh"
#include "keccak.cuh"

namespace sg {
namespace {

using gl::fe3;

struct VerifyDesc {
    sg_verify_table t;
    uint64_t first;  // index of this table's first query in the launch
};

__device__ __forceinline__ fe3 c3(const uint64_t* p, uint64_t i) { return fe3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ fe3 base3(uint64_t x) { return fe3{x, 0, 0}; }
__device__ __forceinline__ bool eq3(fe3 a, fe3 b) {
    a = gl::canon3(a), b = gl::canon3(b);
    return a.c0 == b.c0 && a.c1 == b.c1 && a.c2 == b.c2;
}

__device__ __forceinline__ uint64_t brev(uint64_t x, uint32_t bits) { return bits ? __brevll(x) >> (64 - bits) : 0; }

// Keccak-256 sponge fed one 8-byte lane at a time (rate 17 lanes).
struct Sponge {
    uint64_t s[25];
    uint32_t pos;
    __device__ void init() {
        for (int i = 0; i < 25; ++i) s[i] = 0;
        pos = 0;
    }
    __device__ void lane(uint64_t v) {
        s[pos] ^= v;
        if (++pos == 17) {
            kc::permute(s);
            pos = 0;
        }
    }
    __device__ void finish(uint64_t d[4]) {
        s[pos] ^= 0x01ULL;
        s[16] ^= 0x8000000000000000ULL;
        kc::permute(s);
        for (int i = 0; i < 4; ++i) d[i] = s[i];
    }
};

// Leaf of two rows of `w` field elements, canonical big-endian.
__device__ void row_pair_leaf(const uint64_t* r0, const uint64_t* r1, uint32_t w, uint64_t d[4]) {
    Sponge sp;
    sp.init();
    for (uint32_t i = 0; i < w; ++i) sp.lane(kc::bswap64(gl::canon(r0[i])));
    for (uint32_t i = 0; i < w; ++i) sp.lane(kc::bswap64(gl::canon(r1[i])));
    sp.finish(d);
}

// Walk an authentication path (siblings leaf first) and compare with the root.
__device__ bool path_ok(uint64_t h[4], uint64_t idx, const uint8_t* path, uint32_t depth, const uint8_t* root) {
    for (uint32_t d = 0; d < depth; ++d) {
        const uint64_t* sib = reinterpret_cast<const uint64_t*>(path + 32ull * d);
        uint64_t s[25];
        for (int i = 0; i < 25; ++i) s[i] = 0;
        const uint64_t* l = (idx & 1) ? sib : h;
        const uint64_t* r = (idx & 1) ? h : sib;
        for (int i = 0; i < 4; ++i) {
            s[i] = l[i];
            s[4 + i] = r[i];
        }
        s[8] = 0x01ULL;
        s[16] = 0x8000000000000000ULL;
        kc::permute(s);
        for (int i = 0; i < 4; ++i) h[i] = s[i];
        idx >>= 1;
    }
    const uint64_t* rt = reinterpret_cast<const uint64_t*>(root);
    return h[0] == rt[0] && h[1] == rt[1] && h[2] == rt[2] && h[3] == rt[3];
}

// DEEP composition value at the LDE point x from one opened row of each
// commitment: sum_j gh_j (H_j(x) - H_j(z^2)) / (x - z^2)
//            + sum_j [gt_2j (t_j(x) - t_j(z)) / (x - z) + gt_2j+1 (t_j(x) - t_j(zw)) / (x - zw)]
// (crypto/stark/src/prover.rs:2400-2608).
__device__ fe3 deep_at(const sg_verify_table& T, uint64_t x, const uint64_t* rm, const uint64_t* ra,
                       const uint64_t* rp) {
    const uint64_t* C = T.consts;
    const uint32_t m = T.m, W = T.m + T.aux_cols;
    const fe3 z = c3(C, 0), zw = c3(C, 1), z2 = c3(C, 2);
    fe3 ah{0, 0, 0}, a0{0, 0, 0}, a1{0, 0, 0};
    for (int j = 0; j < 2; ++j)
        ah = gl::add3(ah, gl::mul3(c3(C, 3 + j), gl::sub3(c3(rp, j), c3(C, 5 + j))));
    const uint64_t gt0 = 7, td0 = 7 + 2ull * W;
    for (uint32_t j = 0; j < W; ++j) {
        const fe3 tv = j < m ? base3(rm[j]) : c3(ra, j - m);
        a0 = gl::add3(a0, gl::mul3(c3(C, gt0 + 2ull * j), gl::sub3(tv, c3(C, td0 + j))));
        a1 = gl::add3(a1, gl::mul3(c3(C, gt0 + 2ull * j + 1), gl::sub3(tv, c3(C, td0 + W + j))));
    }
    const fe3 ih = gl::inv3(gl::sub3(base3(x), z2));
    const fe3 i0 = gl::inv3(gl::sub3(base3(x), z));
    const fe3 i1 = gl::inv3(gl::sub3(base3(x), zw));
    return gl::add3(gl::add3(gl::mul3(ah, ih), gl::mul3(a0, i0)), gl::mul3(a1, i1));
}

__device__ uint32_t check_query(const sg_verify_table& T, uint32_t q) {
    const uint32_t logN = T.log_N, Q = T.queries, D = logN - 1;
    const uint64_t iota = T.iotas[q];
    const uint32_t W = T.m + T.aux_cols;
    const uint8_t* roots = T.roots;
    uint64_t h[4];
    // openings of the three trace commitments
    const uint64_t* om = T.open_main + 2ull * q * T.m;
    row_pair_leaf(om, om + T.m, T.m, h);
    if (!path_ok(h, iota, T.path_main + (uint64_t)q * D * 32, D, roots)) return 1;
    const uint64_t* oa = T.open_aux + 2ull * q * 3 * T.aux_cols;
    row_pair_leaf(oa, oa + 3 * T.aux_cols, 3 * T.aux_cols, h);
    if (!path_ok(h, iota, T.path_aux + (uint64_t)q * D * 32, D, roots + 32)) return 2;
    const uint64_t* op = T.open_parts + 2ull * q * 6;
    row_pair_leaf(op, op + 6, 6, h);
    if (!path_ok(h, iota, T.path_parts + (uint64_t)q * D * 32, D, roots + 64)) return 3;
    if (T.total_folds == 0) return 0;
    // DEEP values at rows br(2 iota), br(2 iota + 1): x = g w^r
    const uint64_t* C = T.consts;
    const uint64_t zeta_at = 7 + 4ull * W, coef_at = zeta_at + T.total_folds;
    const uint64_t r0 = brev(2 * iota, logN), r1 = brev(2 * iota + 1, logN);
    const fe3 d0 = deep_at(T, gl::mul(T.coset_offset, gl::pow(T.omega_N, r0)), om, oa, op);
    const fe3 d1 = deep_at(T, gl::mul(T.coset_offset, gl::pow(T.omega_N, r1)), om + T.m, oa + 3 * T.aux_cols, op + 6);
    // first fold at x0 = g w^br(iota, logN - 1)
    const uint64_t x0 = gl::mul(T.coset_offset, gl::pow(T.omega_N, brev(iota, logN - 1)));
    fe3 v = gl::add3(gl::add3(d0, d1), gl::mulb3(gl::mul3(c3(C, zeta_at), gl::sub3(d0, d1)), gl::inv(gl::canon(x0))));
    const uint8_t* fpath = T.fri_paths;
    for (uint32_t li = 0; li < T.fri_layers; ++li) {
        const uint32_t f = li + 1;
        const uint64_t pos = iota >> li, leaf = pos >> 1;
        const uint64_t* pr = T.fri_open + (uint64_t)li * 2 * Q * 3 + 6ull * q;
        const fe3 a = c3(pr, 0), b = c3(pr, 1);
        if (!eq3((pos & 1) ? b : a, v)) return 4 | (f << 8);
        Sponge sp;
        sp.init();
        const uint64_t lanes[6] = {a.c0, a.c1, a.c2, b.c0, b.c1, b.c2};
        for (int i = 0; i < 6; ++i) sp.lane(kc::bswap64(gl::canon(lanes[i])));
        sp.finish(h);
        const uint32_t depth = logN - 2 - li;
        if (!path_ok(h, leaf, fpath + (uint64_t)q * depth * 32, depth, roots + 96 + 32ull * li)) return 5 | (f << 8);
        fpath += (uint64_t)Q * depth * 32;
        uint64_t xj = gl::mul(T.coset_offset, gl::pow(T.omega_N, brev(leaf << f, logN - 1)));
        for (uint32_t s = 0; s < f; ++s) xj = gl::sqr(xj);
        v = gl::add3(gl::add3(a, b), gl::mulb3(gl::mul3(c3(C, zeta_at + f), gl::sub3(a, b)), gl::inv(gl::canon(xj))));
    }
    // terminal polynomial at x_t = offset * wT^br(p, terminal_log)
    const uint64_t pt = iota >> (T.total_folds - 1);
    const uint64_t xt = gl::mul(T.terminal_offset, gl::pow(T.omega_T, brev(pt, T.terminal_log)));
    fe3 ev{0, 0, 0};
    for (uint32_t i = T.num_coeffs; i-- > 0;) ev = gl::add3(gl::mulb3(ev, xt), c3(C, coef_at + i));
    if (!eq3(ev, v)) return 6;
    return 0;
}

__global__ void __launch_bounds__(128) k_verify_queries(const VerifyDesc* __restrict__ d, uint32_t count,
                                                        uint64_t total, uint32_t* __restrict__ status) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    uint32_t lo = 0, hi = count;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (d[mid].first <= g)
            lo = mid;
        else
            hi = mid;
    }
    status[g] = check_query(d[lo].t, (uint32_t)(g - d[lo].first));
}

}  // namespace
}  // namespace sg

using namespace sg;

extern "C" int sg_verify_queries(sg_ctx* c, void* stream, const sg_verify_table* tables, uint32_t count,
                                 uint32_t* status_out) {
    SG_CHECK_ARG(c && (count == 0 || (tables && status_out)), "null argument");
    SG_ENTER(ctx_of(c));
    Ctx* ctx = ctx_of(c);
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<VerifyDesc> d(count);
    uint64_t total = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const sg_verify_table& t = tables[i];
        SG_CHECK_ARG(t.log_N >= 2 && t.log_N <= 32 && t.log_N > t.log_n, "LDE size out of range");
        SG_CHECK_ARG(t.total_folds < t.log_N && t.fri_layers == (t.total_folds ? t.total_folds - 1 : 0),
                     "FRI layer count");
        SG_CHECK_ARG(t.terminal_log <= t.log_N && t.terminal_log + t.total_folds == t.log_N, "terminal size");
        SG_CHECK_ARG(t.consts && t.roots && t.iotas && t.open_main && t.open_parts && t.path_main && t.path_aux &&
                         t.path_parts && (t.aux_cols == 0 || t.open_aux) && (t.fri_layers == 0 || (t.fri_open && t.fri_paths)),
                     "null table array");
        d[i].t = t;
        d[i].first = total;
        total += t.queries;
    }
    if (total == 0) return SG_OK;
    VerifyDesc* dd = nullptr;
    uint32_t* ds = nullptr;
    SG_TRY(dev_alloc(ctx, st, count * sizeof(VerifyDesc), (void**)&dd));
    int rc = dev_alloc(ctx, st, total * 4, (void**)&ds);
    cudaError_t e = cudaSuccess;
    if (rc == SG_OK) e = cudaMemcpyAsync(dd, d.data(), count * sizeof(VerifyDesc), cudaMemcpyHostToDevice, st);
    if (rc == SG_OK && e == cudaSuccess) {
        k_verify_queries<<<(unsigned)((total + 127) / 128), 128, 0, st>>>(dd, count, total, ds);
        rc = check_launch(ctx, "k_verify_queries");
    }
    if (rc == SG_OK && e == cudaSuccess) e = cudaMemcpyAsync(status_out, ds, total * 4, cudaMemcpyDeviceToHost, st);
    if (rc == SG_OK && e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (rc == SG_OK && e != cudaSuccess) {
        set_error(std::string("verify queries: ") + cudaGetErrorString(e));
        rc = SG_ERR_CUDA;
    }
    dev_free(ctx, st, ds, total * 4);
    dev_free(ctx, st, dd, count * sizeof(VerifyDesc));
    return rc;
}
