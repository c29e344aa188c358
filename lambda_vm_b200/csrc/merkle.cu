// Keccak-256 Merkle commitment kernels for sm_100a.
//
// Reference behaviour:
//  * leaves: crypto/stark/src/commitment.rs:52-107 (keccak_leaves_bit_reversed_grouped)
//    — leaf i hashes rows br(R*i) .. br(R*i + R - 1) of the natural-order LDE,
//    each row's columns in order, every element canonical and big-endian
//    (goldilocks.rs:440-444). A little-endian variant serves the per-row LE
//    commitment layout.
//  * inner tree: crypto/crypto/src/merkle_tree/utils.rs:68-96 — node array of
//    2L-1 digests, root at 0, leaves at [L-1, 2L-1), parent = Keccak(left || right).
//  * paths: merkle.rs build_merkle_path — sibling per level, leaf first.
//  * grinding: crypto/stark/src/grinding.rs:45-104 — smallest nonce whose
//    Keccak(inner || nonce_be) head (BE u64) is below 2^(64-g).
//
// One thread owns one sponge: Keccak is a serial chain of permutations, and
// with the state in registers the kernels are bound by INT issue, not HBM.
// The tree kernel reduces 8 levels per launch inside shared memory.
#include "common.cuh"
#include "gl.cuh"
#include "keccak.cuh"

namespace sg {

template <bool LE>
__global__ void __launch_bounds__(128) k_leaves(const uint64_t* __restrict__ data, uint64_t row_u64, uint64_t c0,
                                                uint64_t w, uint32_t R, uint32_t log_rows, uint64_t num_leaves,
                                                uint64_t* __restrict__ out) {
    const uint64_t leaf = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (leaf >= num_leaves) return;
    auto row_of = [&](uint64_t r) -> const uint64_t* {
        const uint64_t br = log_rows ? (__brevll(r) >> (64 - log_rows)) : 0;
        return data + br * row_u64 + c0;
    };
    uint64_t s[25];
#pragma unroll
    for (int i = 0; i < 25; ++i) s[i] = 0;
    const uint64_t total = (uint64_t)R * w;
    const uint64_t* row = row_of(leaf * R);
    uint32_t k = 0;
    uint64_t c = 0;
    auto next = [&]() -> uint64_t {
        uint64_t v = gl::canon(__ldg(row + c));
        if (++c == w) {
            c = 0;
            ++k;
            if (k < R) row = row_of(leaf * R + k);
        }
        return LE ? v : kc::bswap64(v);
    };
    const uint64_t full = total / 17;
    const uint32_t rem = (uint32_t)(total % 17);
    for (uint64_t b = 0; b < full; ++b) {
#pragma unroll
        for (int i = 0; i < 17; ++i) s[i] ^= next();
        kc::permute(s);
    }
#pragma unroll
    for (int i = 0; i < 17; ++i) {
        if ((uint32_t)i < rem) s[i] ^= next();
        if ((uint32_t)i == rem) s[i] ^= 0x01ULL;
    }
    s[16] ^= 0x8000000000000000ULL;
    kc::permute(s);
    uint64_t* o = out + leaf * 4;
    o[0] = s[0];
    o[1] = s[1];
    o[2] = s[2];
    o[3] = s[3];
}

// Per-row leaves absorbed one column window at a time, for commits whose
// columns arrive in chunks: window [c0, c0 + w) of every leaf's row is
// absorbed into that leaf's sponge, which lives in HBM between windows
// (structure of arrays: lane j of leaf i at state[j * L + i], so every load
// and store is coalesced). Windows start on sponge-block boundaries (c0 a
// multiple of 17 lanes); the last one absorbs the remainder, pads, permutes
// and writes the digest. The absorbed byte stream, and so the digest, is the
// one k_leaves produces for rows_per_leaf = 1.
template <bool LE>
__global__ void __launch_bounds__(128) k_leaves_window(const uint64_t* __restrict__ data, uint64_t row_u64,
                                                       uint64_t c0, uint64_t w, uint32_t log_rows, uint64_t L,
                                                       uint64_t* __restrict__ state, int first, int last,
                                                       uint64_t* __restrict__ out) {
    const uint64_t leaf = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (leaf >= L) return;
    const uint64_t br = log_rows ? (__brevll(leaf) >> (64 - log_rows)) : 0;
    const uint64_t* row = data + br * row_u64 + c0;
    uint64_t s[25];
#pragma unroll
    for (int i = 0; i < 25; ++i) s[i] = first ? 0 : state[(uint64_t)i * L + leaf];
    auto lane = [&](uint64_t c) {
        const uint64_t v = gl::canon(__ldg(row + c));
        return LE ? v : kc::bswap64(v);
    };
    const uint64_t full = w / 17;
    for (uint64_t b = 0; b < full; ++b) {
#pragma unroll
        for (int i = 0; i < 17; ++i) s[i] ^= lane(b * 17 + i);
        kc::permute(s);
    }
    if (last) {
        const uint32_t rem = (uint32_t)(w % 17);
#pragma unroll
        for (int i = 0; i < 17; ++i) {
            if ((uint32_t)i < rem) s[i] ^= lane(full * 17 + i);
            if ((uint32_t)i == rem) s[i] ^= 0x01ULL;
        }
        s[16] ^= 0x8000000000000000ULL;
        kc::permute(s);
        uint64_t* o = out + leaf * 4;
#pragma unroll
        for (int i = 0; i < 4; ++i) o[i] = s[i];
    } else {
#pragma unroll
        for (int i = 0; i < 25; ++i) state[(uint64_t)i * L + leaf] = s[i];
    }
}

int leaves_window(Ctx* ctx, cudaStream_t st, const uint64_t* data, uint64_t num_rows, uint64_t row_u64, uint64_t c0,
                  uint64_t w, int little_endian, uint64_t* state, int first, int last, uint8_t* out) {
    SG_CHECK_ARG(c0 % 17 == 0 && (last || w % 17 == 0), "leaf windows must cover whole sponge blocks");
    const int lr = log2_exact(num_rows);
    SG_CHECK_ARG(lr >= 0, "num_rows must be a power of two");
    const unsigned grid = (unsigned)((num_rows + 127) / 128);
    if (little_endian)
        k_leaves_window<true><<<grid, 128, 0, st>>>(data, row_u64, c0, w, lr, num_rows, state, first, last,
                                                   (uint64_t*)out);
    else
        k_leaves_window<false><<<grid, 128, 0, st>>>(data, row_u64, c0, w, lr, num_rows, state, first, last,
                                                    (uint64_t*)out);
    return check_launch(ctx, "k_leaves_window");
}

__device__ __forceinline__ void hash_pair(const uint64_t* l, const uint64_t* r, uint64_t* d) {
    uint64_t s[25];
#pragma unroll
    for (int i = 0; i < 25; ++i) s[i] = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        s[i] = l[i];
        s[4 + i] = r[i];
    }
    s[8] = 0x01ULL;
    s[16] = 0x8000000000000000ULL;
    kc::permute(s);
#pragma unroll
    for (int i = 0; i < 4; ++i) d[i] = s[i];
}

// Reduce `levels` tree levels above child level jc (2^jc nodes, starting at
// node index 2^jc - 1). CTA b owns children [b*2^levels, (b+1)*2^levels).
__global__ void __launch_bounds__(128) k_merkle_levels(uint64_t* nodes, uint32_t jc, uint32_t levels) {
    __shared__ uint64_t sh[128 * 4];
    const uint32_t t = threadIdx.x;
    const uint64_t b = blockIdx.x;
    uint32_t active = 1u << (levels - 1);
    uint64_t d[4];
    if (t < active) {
        const uint64_t child = ((1ULL << jc) - 1) + (b << levels) + 2 * t;
        hash_pair(nodes + child * 4, nodes + (child + 1) * 4, d);
        const uint64_t parent = ((1ULL << (jc - 1)) - 1) + (b << (levels - 1)) + t;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            nodes[parent * 4 + i] = d[i];
            sh[t * 4 + i] = d[i];
        }
    }
    __syncthreads();
    for (uint32_t lvl = 1; lvl < levels; ++lvl) {
        active >>= 1;
        if (t < active) hash_pair(sh + 8 * t, sh + 8 * t + 4, d);
        __syncthreads();
        if (t < active) {
            const uint32_t j = jc - 1 - lvl;
            const uint64_t parent = ((1ULL << j) - 1) + (b << (levels - 1 - lvl)) + t;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                nodes[parent * 4 + i] = d[i];
                sh[t * 4 + i] = d[i];
            }
        }
        __syncthreads();
    }
}

// One tree level with one thread per parent: level jc (2^jc nodes) -> jc - 1.
// Used for the wide bottom levels, where every thread of every warp has a
// pair to hash; the fused kernel above takes over once a level is narrow.
__global__ void __launch_bounds__(128) k_merkle_level(uint64_t* nodes, uint32_t jc) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t parents = 1ULL << (jc - 1);
    if (t >= parents) return;
    const uint64_t child = ((1ULL << jc) - 1) + 2 * t;
    uint64_t d[4];
    hash_pair(nodes + child * 4, nodes + (child + 1) * 4, d);
    const uint64_t parent = (parents - 1) + t;
#pragma unroll
    for (int i = 0; i < 4; ++i) nodes[parent * 4 + i] = d[i];
}

int leaves_row_major(Ctx* ctx, cudaStream_t st, const uint64_t* data, uint64_t num_rows, uint64_t row_u64,
                     uint64_t col_start, uint64_t col_end, uint32_t rows_per_leaf, int little_endian,
                     uint8_t* out) {
    if (num_rows == 0) return SG_OK;
    const int lr = log2_exact(num_rows);
    SG_CHECK_ARG(lr >= 0, "num_rows must be a power of two");
    SG_CHECK_ARG(rows_per_leaf >= 1 && num_rows % rows_per_leaf == 0, "rows_per_leaf must divide num_rows");
    SG_CHECK_ARG(col_start < col_end && col_end <= row_u64, "column range");
    SG_CHECK_ARG(((uintptr_t)out & 7) == 0, "leaf output must be 8-byte aligned");
    const uint64_t nl = num_rows / rows_per_leaf;
    const unsigned grid = (unsigned)((nl + 127) / 128);
    if (little_endian)
        k_leaves<true><<<grid, 128, 0, st>>>(data, row_u64, col_start, col_end - col_start, rows_per_leaf, lr, nl,
                                             (uint64_t*)out);
    else
        k_leaves<false><<<grid, 128, 0, st>>>(data, row_u64, col_start, col_end - col_start, rows_per_leaf, lr, nl,
                                              (uint64_t*)out);
    return check_launch(ctx, "k_leaves");
}

int merkle_inner(Ctx* ctx, cudaStream_t st, uint8_t* nodes, uint64_t L) {
    const int lg = log2_exact(L);
    SG_CHECK_ARG(lg >= 0, "leaf count must be a power of two");
    SG_CHECK_ARG(((uintptr_t)nodes & 7) == 0, "node buffer must be 8-byte aligned");
    uint32_t jc = (uint32_t)lg;
    // Levels with at least 2^14 parents: one full-width launch per level.
    while (jc > 14) {
        const uint64_t parents = 1ULL << (jc - 1);
        k_merkle_level<<<(unsigned)((parents + 127) / 128), 128, 0, st>>>((uint64_t*)nodes, jc);
        SG_TRY(check_launch(ctx, "k_merkle_level"));
        --jc;
    }
    while (jc > 0) {
        const uint32_t levels = jc < 8 ? jc : 8;
        const uint64_t ctas = 1ULL << (jc - levels);
        k_merkle_levels<<<(unsigned)ctas, 1u << (levels - 1), 0, st>>>((uint64_t*)nodes, jc, levels);
        SG_TRY(check_launch(ctx, "k_merkle_levels"));
        jc -= levels;
    }
    return SG_OK;
}

// Leaf padding to a power of two: copies of the last leaf (merkle_tree/utils.rs:46-52).
__global__ void k_pad_leaves(uint64_t* leaves, uint64_t n, uint64_t L) {
    const uint64_t i = n + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L) return;
#pragma unroll
    for (int k = 0; k < 4; ++k) leaves[i * 4 + k] = leaves[(n - 1) * 4 + k];
}

int pad_leaves(Ctx* ctx, cudaStream_t st, uint8_t* leaves, uint64_t n, uint64_t L) {
    if (L <= n) return SG_OK;
    k_pad_leaves<<<(unsigned)((L - n + 255) / 256), 256, 0, st>>>((uint64_t*)leaves, n, L);
    return check_launch(ctx, "k_pad_leaves");
}

// ---------------------------------------------------------------- paths
__global__ void k_gather_paths(const uint64_t* nodes, uint64_t L, uint32_t depth, const uint32_t* pos, uint32_t nq,
                               uint64_t* out) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (uint64_t)nq * depth) return;
    const uint32_t q = (uint32_t)(g / depth), lvl = (uint32_t)(g % depth);
    if ((uint64_t)pos[q] >= L) {  // out-of-range query: emit a zero node, touch nothing else
#pragma unroll
        for (int i = 0; i < 4; ++i) out[g * 4 + i] = 0;
        return;
    }
    uint64_t node = (uint64_t)pos[q] + L - 1;
    for (uint32_t i = 0; i < lvl; ++i) node = (node & 1) ? (node >> 1) : ((node - 1) >> 1);
    const uint64_t sib = (node & 1) ? node + 1 : node - 1;
#pragma unroll
    for (int i = 0; i < 4; ++i) out[g * 4 + i] = nodes[sib * 4 + i];
}

// ---------------------------------------------------------------- grinding
__global__ void __launch_bounds__(256) k_grind(uint64_t h0, uint64_t h1, uint64_t h2, uint64_t h3, uint64_t limit,
                                               uint64_t base, uint64_t count, unsigned long long* best) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        const uint64_t nonce = base + i;
        if (nonce < base) break;  // u64 wrap
        if (nonce >= *(volatile unsigned long long*)best) break;
        uint64_t s[25];
#pragma unroll
        for (int k = 0; k < 25; ++k) s[k] = 0;
        s[0] = h0;
        s[1] = h1;
        s[2] = h2;
        s[3] = h3;
        s[4] = kc::bswap64(nonce);
        s[5] = 0x01ULL;
        s[16] = 0x8000000000000000ULL;
        kc::permute(s);
        if (kc::bswap64(s[0]) < limit) atomicMin(best, (unsigned long long)nonce);
    }
}

}  // namespace sg

using namespace sg;

extern "C" int sg_merkle_gather_paths(sg_ctx* c, void* stream, const uint8_t* d_nodes, uint64_t leaves_len,
                                      const uint32_t* d_positions, uint32_t num_queries, uint8_t* d_out) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    SG_CHECK_ARG(ctx, "null context");
    SG_ENTER(ctx);
    const int lg = log2_exact(leaves_len);
    SG_CHECK_ARG(lg >= 0, "leaves_len must be a power of two");
    if (num_queries == 0 || lg == 0) return SG_OK;
    const uint64_t tot = (uint64_t)num_queries * lg;
    k_gather_paths<<<(unsigned)((tot + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        (const uint64_t*)d_nodes, leaves_len, (uint32_t)lg, d_positions, num_queries, (uint64_t*)d_out);
    return check_launch(ctx, "k_gather_paths");
}

// Grid of the grinding search: exactly the CTAs that are resident at once.
// The search must return the smallest valid nonce, so it can only stop once
// every smaller nonce is checked; CTAs beyond the resident ones would start
// late on the low nonces of each sweep and hold the whole search open.
static int grind_grid(unsigned* grid) {
    KernelInfo ki;
    SG_TRY(kernel_info((const void*)k_grind, 0, 256, &ki));
    *grid = (unsigned)ki.sms * (unsigned)ki.blocks_per_sm;
    return SG_OK;
}

extern "C" int sg_grind(sg_ctx* c, void* stream, const uint64_t inner_lanes[4], uint8_t grinding_factor,
                        uint64_t* nonce_out) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    SG_CHECK_ARG(ctx && inner_lanes && nonce_out, "null argument");
    SG_ENTER(ctx);
    SG_CHECK_ARG(grinding_factor >= 1 && grinding_factor <= 64, "grinding factor must be in 1..=64");
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t limit = grinding_factor == 64 ? 1ULL : (1ULL << (64 - grinding_factor));
    const uint64_t expected = grinding_factor >= 63 ? ~0ULL : (1ULL << grinding_factor);
    uint64_t count = expected > (1ULL << 25) ? (1ULL << 28) : (expected * 8 < (1ULL << 20) ? (1ULL << 20) : expected * 8);
    unsigned grid = 0;
    SG_TRY(grind_grid(&grid));
    unsigned long long* d_best = nullptr;
    SG_TRY(dev_alloc(ctx, st, 8, (void**)&d_best));
    int rc = SG_OK;
    uint64_t base = 0;
    *nonce_out = ~0ULL;
    for (;;) {
        const unsigned long long init = ~0ULL;
        unsigned long long host = 0;
        cudaError_t e = cudaMemcpyAsync(d_best, &init, 8, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            k_grind<<<grid, 256, 0, st>>>(inner_lanes[0], inner_lanes[1], inner_lanes[2], inner_lanes[3], limit,
                                               base, count, d_best);
            rc = check_launch(ctx, "k_grind");
            if (rc != SG_OK) break;
            e = cudaMemcpyAsync(&host, d_best, 8, cudaMemcpyDeviceToHost, st);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            set_error(std::string("grind: ") + cudaGetErrorString(e));
            rc = SG_ERR_CUDA;
            break;
        }
        if (host != ~0ULL) {
            *nonce_out = host;
            break;
        }
        if (base + count < base) {
            set_error("grind: nonce space exhausted");
            rc = SG_ERR_INVALID;
            break;
        }
        base += count;
    }
    int rf = dev_free(ctx, st, d_best, 8);
    return rc != SG_OK ? rc : rf;
}
