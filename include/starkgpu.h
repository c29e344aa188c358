/*
 * starkgpu — B200 (sm_100a) proving backend for lambda_vm's Goldilocks STARK.
 *
 * C ABI that replaces the `math-cuda` crate's public surface
 * (crypto/math-cuda/src/lib.rs:8-31), the seam through which the stark crate
 * (crypto/stark/src/gpu_lde.rs, logup_gpu.rs, grinding.rs, fri/mod.rs) reaches
 * the GPU. Each entry below names the reference function it stands in for.
 *
 * Conventions
 *  - Every function returns an int status (SG_OK or an SG_ERR_* code); it never
 *    aborts and never falls back to the CPU. sg_last_error() gives the message
 *    of the last failure on the calling thread.
 *  - `stream` is a cudaStream_t (NULL = legacy default stream). Work is
 *    enqueued on it; functions that return host data synchronize it.
 *  - Field elements cross as u64 in [0, 2^64) (reduced mod p, any
 *    representative); every output this library writes is canonical (< p).
 *    Ext3 elements are 3 consecutive u64 (c0, c1, c2) with w^3 = 2.
 *  - Matrices are row-major: element (row r, column c) at [r * row_stride + c].
 *  - Device pointers are named d_*; host pointers have no prefix.
 *  - One context per GPU; a context is safe to use from several threads.
 */
#ifndef STARKGPU_H
#define STARKGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define SG_API __attribute__((visibility("default")))
#else
#define SG_API
#endif

#define SG_OK 0
#define SG_ERR_INVALID 1     /* bad argument (shape, size, alignment, null) */
#define SG_ERR_CUDA 2        /* a CUDA runtime call failed */
#define SG_ERR_OOM 3         /* device allocation failed */
#define SG_ERR_BUDGET 4      /* request exceeds the context's HBM budget */
#define SG_ERR_UNSUPPORTED 5 /* valid request outside what the kernels cover */

typedef struct sg_ctx sg_ctx;
/* Device-resident LDE of one table plus its Merkle tree (GpuLdeBase /
 * GpuLdeExt3 + GpuMerkleTree, crypto/math-cuda/src/lde.rs:923-988). */
typedef struct sg_lde sg_lde;

typedef struct {
    uint64_t* d_lde;       /* (lde_rows x row_u64) row-major, natural order, canonical */
    uint64_t lde_rows;     /* n * blowup */
    uint64_t row_u64;      /* u64 per LDE row (m for base tables, 3m for ext3) */
    uint8_t* d_nodes;      /* (2L-1) x 32 bytes, root at 0, leaves at [L-1, 2L-1); NULL if no tree */
    uint64_t leaves_len;   /* L */
    uint8_t root[32];      /* Merkle root (node 0) */
} sg_lde_info;

/* Leaf layout of a commitment (crypto/stark/src/commitment.rs:52-107). */
typedef struct {
    uint32_t rows_per_leaf; /* 2 = the prover's row-pair leaf (ROWS_PER_LEAF); 1 = per-row */
    uint32_t little_endian; /* 0 = canonical big-endian bytes (reference); 1 = little-endian */
    uint64_t col_start;     /* hashed column range [col_start, col_end) in u64 lanes; */
    uint64_t col_end;       /* col_end = 0 means the whole row */
} sg_leaf_layout;

/* ---- context / runtime: replaces device::backend() (crypto/math-cuda/src/device.rs:592) ---- */
SG_API int sg_ctx_create(int device, uint64_t hbm_budget_bytes, sg_ctx** out);
SG_API void sg_ctx_destroy(sg_ctx* ctx);
SG_API const char* sg_last_error(void);
/* Bytes currently held by the context and the high-water mark. */
SG_API int sg_ctx_memory(sg_ctx* ctx, uint64_t* in_use, uint64_t* peak);
/* Kernels launched through this context so far (for launch accounting). */
SG_API uint64_t sg_ctx_launches(sg_ctx* ctx);
/* Test hook for host-side failure handling: the n-th device allocation from
 * now (n >= 1) fails with SG_ERR_OOM; n = 0 disarms. */
SG_API int sg_ctx_fail_alloc_after(sg_ctx* ctx, int64_t n);

/* Stream-ordered device memory charged to the context budget. */
SG_API int sg_dev_alloc(sg_ctx* ctx, void* stream, uint64_t bytes, void** d_out);
SG_API int sg_dev_free(sg_ctx* ctx, void* stream, void* d_ptr, uint64_t bytes);
SG_API int sg_memcpy_h2d(sg_ctx* ctx, void* stream, void* d_dst, const void* src, uint64_t bytes);
SG_API int sg_memcpy_d2h(sg_ctx* ctx, void* stream, void* dst, const void* d_src, uint64_t bytes);
SG_API int sg_stream_sync(sg_ctx* ctx, void* stream);
/* Page-locked host memory for fast transfers. */
SG_API int sg_host_alloc(uint64_t bytes, void** out);
SG_API int sg_host_free(void* p);

/* ---- NTT: replaces ntt::forward / ntt::inverse (crypto/math-cuda/src/ntt.rs:57-66),
 *      batched over the m columns of a row-major n x m matrix, in place,
 *      natural order in and out; the inverse includes the 1/n scaling. ---- */
SG_API int sg_ntt_forward(sg_ctx* ctx, void* stream, uint64_t* d_data, uint64_t n, uint64_t m);
SG_API int sg_ntt_inverse(sg_ctx* ctx, void* stream, uint64_t* d_data, uint64_t n, uint64_t m);

/* ---- coset LDE: replaces lde::coset_lde_base / coset_lde_batch_base
 *      (crypto/math-cuda/src/lde.rs:990,1072) and the CPU
 *      Polynomial::coset_lde_full_expand_row_major (crypto/math/src/polynomial.rs:527).
 *      d_trace: n x m row-major; d_weights: n coset weights (g^i / n, prover.rs:458-467);
 *      d_out: (blowup*n) x m row-major, natural order, canonical. ---- */
SG_API int sg_coset_lde(sg_ctx* ctx, void* stream, const uint64_t* d_trace, uint64_t n, uint64_t m, uint32_t blowup,
                 const uint64_t* d_weights, uint64_t* d_out);

/* ---- allocation-free coset LDE. No counterpart in the reference: an extra
 *      entry point for callers that cannot allocate device memory at call time
 *      (a serving process that reserves all of its HBM at start-up and must not
 *      grow it mid-request, or an FFI host that wants no hidden allocation and
 *      no context object). Same arguments and result as sg_coset_lde, but no
 *      context and no allocation: its scratch is a static device array of
 *      SG_STATIC_SCRATCH_BYTES per GPU, held until the process exits. Requires
 *      (blowup*n + 2*n*m) * 8 <= SG_STATIC_SCRATCH_BYTES, else SG_ERR_INVALID.
 *      The first call on a device (with that device current) looks up the
 *      array's device address; make it before any stream capture. Calls share
 *      the array, so calls that overlap on the GPU race and must be serialized
 *      by the caller. ---- */
#define SG_STATIC_SCRATCH_BYTES (32ull << 20)
SG_API int sg_coset_lde_static(void* stream, const uint64_t* d_trace, uint64_t n, uint64_t m, uint32_t blowup,
                               const uint64_t* d_weights, uint64_t* d_out);

/* ---- leaves: replaces merkle::keccak_leaves_base / keccak_leaves_ext3
 *      (crypto/math-cuda/src/merkle.rs:33,83) over a row-major matrix
 *      (num_rows x row_u64). d_leaves_out: num_rows/rows_per_leaf x 32 bytes,
 *      8-byte aligned. ---- */
SG_API int sg_keccak_leaves(sg_ctx* ctx, void* stream, const uint64_t* d_data, uint64_t num_rows, uint64_t row_u64,
                     const sg_leaf_layout* layout, uint8_t* d_leaves_out);

/* ---- tree: replaces merkle::build_merkle_tree_on_device (crypto/math-cuda/src/merkle.rs:316).
 *      Leaves are padded to a power of two by repeating the last one
 *      (merkle_tree/utils.rs:46-52). d_nodes receives (2L-1) x 32 bytes; the root
 *      is copied to root_out (host, may be NULL). ---- */
SG_API int sg_merkle_build(sg_ctx* ctx, void* stream, const uint8_t* d_leaves, uint64_t num_leaves, uint8_t* d_nodes,
                    uint8_t root_out[32]);
/* Number of leaves L the tree over num_leaves leaves has (next power of two). */
SG_API uint64_t sg_merkle_leaves_len(uint64_t num_leaves);

/* ---- paths: replaces merkle::gather_merkle_paths_dev (crypto/math-cuda/src/merkle.rs:358).
 *      d_out: num_queries x log2(leaves_len) x 32 bytes, sibling per level, leaf first. ---- */
SG_API int sg_merkle_gather_paths(sg_ctx* ctx, void* stream, const uint8_t* d_nodes, uint64_t leaves_len,
                           const uint32_t* d_positions, uint32_t num_queries, uint8_t* d_out);

/* ---- LDE + commit: replaces lde::coset_lde_row_major_with_merkle_tree_keep
 *      (crypto/math-cuda/src/lde.rs:674; base field, row-pair big-endian leaves)
 *      and lde::coset_lde_ext3_row_major_with_merkle_tree_keep (lde.rs:855;
 *      pass row_u64 = 3m). `trace` is n x row_u64 row-major, on the host when
 *      trace_on_device == 0 (the reference's `row_major` slice) or on the device
 *      otherwise (`predev`). `weights` (n entries) is a host array.
 *      layout == NULL selects the reference layout {2, BE, all columns}.
 *      When host_lde_out != NULL the LDE is also copied back (retain_host_lde).
 *      The returned handle keeps the LDE and tree resident; root_out gets the root. ---- */
SG_API int sg_lde_commit(sg_ctx* ctx, void* stream, const uint64_t* trace, int trace_on_device, uint64_t n,
                  uint64_t row_u64, uint32_t blowup, const uint64_t* weights, const sg_leaf_layout* layout,
                  uint64_t* host_lde_out, sg_lde** out, uint8_t root_out[32]);
SG_API int sg_lde_get_info(const sg_lde* lde, sg_lde_info* info);
SG_API void sg_lde_free(sg_ctx* ctx, sg_lde* lde);

/* ---- grinding: replaces grinding::generate_nonce_gpu (crypto/math-cuda/src/grinding.rs:29).
 *      inner_lanes: the 32-byte inner hash as four little-endian u64 lanes
 *      (stark::grinding::inner_hash_lanes). Returns the smallest valid nonce. ---- */
SG_API int sg_grind(sg_ctx* ctx, void* stream, const uint64_t inner_lanes[4], uint8_t grinding_factor, uint64_t* nonce_out);

#ifdef __cplusplus
}
#endif
#endif /* STARKGPU_H */
