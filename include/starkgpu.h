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
/* The context's HBM budget in bytes. */
SG_API uint64_t sg_ctx_budget(sg_ctx* ctx);
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
/* Non-blocking CUDA streams owned by the caller (one per concurrent table driver,
 * the reference's 32-stream pool, device.rs:139-143,500-503). */
SG_API int sg_stream_create(sg_ctx* ctx, void** stream_out);
SG_API int sg_stream_destroy(sg_ctx* ctx, void* stream);
/* The same with a scheduling priority (lower numbers run first; the device's
 * range comes from sg_stream_priority_range, greatest = the most urgent). The
 * proof server gives its large jobs the urgent end so that small jobs running
 * beside them fill gaps instead of stretching them. Streams a call creates
 * internally (batched commits, host-trace uploads) take the caller stream's
 * priority. No counterpart in the reference (its stream pool has one level). */
SG_API int sg_stream_create_priority(sg_ctx* ctx, int priority, void** stream_out);
SG_API int sg_stream_priority_range(sg_ctx* ctx, int* least, int* greatest);
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
/* ---- DFT tile autotuning (no reference counterpart: the reference fixes its
 *      kernels' launch shapes). Each pass of 2^log_len points can run with
 *      several compiled tile widths (columns per tile; 4/8/16 for lengths
 *      2^8..2^10, 4/8 for 2^11). On a context's first pass of a length, every
 *      width is timed on the same work and its time per column kept; a pass
 *      over m columns then uses the width minimising ceil(m/C)*C*cost(C),
 *      keeping the default width (16 up to 2^10, 8 at 2^11) unless another is
 *      at least 3 % cheaper; a context with a learned pass-cost model
 *      (sg_ctx_set_pass_model, below) predicts each width's pass time instead
 *      and never times. Results never depend on the width. sg_ctx_dft_tiles pins a width for a
 *      length (cols = 0: automatic); sg_ctx_dft_tuning reports the widths and
 *      their time per column (ms), timing them on `stream` first if needed. ---- */
SG_API int sg_ctx_dft_tiles(sg_ctx* ctx, uint32_t log_len, uint32_t cols);
SG_API int sg_ctx_dft_tuning(sg_ctx* ctx, void* stream, uint32_t log_len, uint32_t* cols, float* cost_per_col,
                             uint32_t* count);

/* ---- allocation-free coset LDE. No counterpart in the reference: an extra
 *      entry point for callers that cannot allocate device memory at call time
 *      (a serving process that reserves all of its HBM at start-up and must not
 *      grow it mid-request, or an FFI host that wants no hidden allocation and
 *      no context object). Same arguments and result as sg_coset_lde, but no
 *      context and no allocation: its scratch is a static device array of
 *      SG_STATIC_SCRATCH_BYTES per GPU, held until the process exits. Requires
 *      (max(blowup*n, 3) + 2*n*m) * 8 <= SG_STATIC_SCRATCH_BYTES, else
 *      SG_ERR_INVALID. It runs on the calling thread's current device; each
 *      GPU has its own array, and the first call on a device (with that device
 *      current) looks up that array's device address and sets the DFT kernels'
 *      shared-memory limit there, so make it before any stream capture. Calls
 *      share the array, so calls that overlap on the GPU race and must be
 *      serialized by the caller. ---- */
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
/* ---- split commitment: replaces coset_lde_row_major_split_trees
 *      (crypto/math-cuda/src/lde.rs:726): one LDE, two row-pair big-endian trees,
 *      columns [split_col, row_u64) in the returned handle (root_out) and, when
 *      build_pre != 0, the precomputed columns [0, split_col) into the caller's
 *      device node buffer d_pre_nodes ((blowup*n - 1) * 32 bytes; root_pre_out). ---- */
SG_API int sg_lde_commit_split(sg_ctx* ctx, void* stream, const uint64_t* trace, int trace_on_device, uint64_t n,
                               uint64_t row_u64, uint32_t blowup, const uint64_t* weights, uint64_t split_col,
                               int build_pre, uint64_t* host_lde_out, sg_lde** out, uint8_t root_out[32],
                               uint8_t* d_pre_nodes, uint8_t root_pre_out[32]);
/* Stream-ordered release of a handle: its memory returns to the pool after
 * the work already queued on `stream`; no device-wide wait. */
SG_API void sg_lde_free_async(sg_ctx* ctx, void* stream, sg_lde* lde);

/* ---- batched commit: the batched form of the per-table commits that
 *      crypto/stark/src/prover.rs:1132-1398 (commit_main_trace) runs through
 *      coset_lde_row_major_with_merkle_tree_keep (crypto/math-cuda/src/lde.rs:674)
 *      once per table, under the table scheduler (prover.rs:749-790).
 *      Commits `count` tables in one call: heaviest first, spread over
 *      `concurrency` internal streams that start after the work already on
 *      `stream` and that `stream` waits for; returns when every root is on the
 *      host. out_ldes[i] / roots_out[32*i] belong to tables[i], each identical
 *      to what sg_lde_commit returns for that table alone. On failure no handle
 *      is returned. ---- */
typedef struct sg_table_desc {
    const uint64_t* trace;   /* n x row_u64 row-major */
    int trace_on_device;     /* nonzero: device pointer, else host */
    uint64_t n;              /* power of two >= 2 */
    uint64_t row_u64;
    uint32_t blowup;         /* power of two */
    int weights_on_device;   /* nonzero: device pointer, else host */
    const uint64_t* weights; /* n coset weights g^i / n */
    sg_leaf_layout layout;   /* rows_per_leaf == 0 selects {2, BE, all columns} */
} sg_table_desc;
SG_API int sg_batch_commit(sg_ctx* ctx, void* stream, const sg_table_desc* tables, uint32_t count,
                           uint32_t concurrency, sg_lde** out_ldes, uint8_t* roots_out);
/* The same commitments with the tables' LDEs fused: every pass of every table
 * goes into one persistent multi-table DFT launch per (step, pass length,
 * tile width, direction), so small tables share the grid with large ones
 * instead of running as launches of a few CTAs (4 steps x a few launches in
 * all, against 4 per table). Each table's leaves and tree follow, heaviest
 * first over `concurrency` streams that start when the LDEs are done.
 * Traces must be device-resident. Same handles and roots as sg_batch_commit. */
SG_API int sg_batch_commit_fused(sg_ctx* ctx, void* stream, const sg_table_desc* tables, uint32_t count,
                                 uint32_t concurrency, sg_lde** out_ldes, uint8_t* roots_out);

/* ---- grinding: replaces grinding::generate_nonce_gpu (crypto/math-cuda/src/grinding.rs:29).
 *      inner_lanes: the 32-byte inner hash as four little-endian u64 lanes
 *      (stark::grinding::inner_hash_lanes). Returns the smallest valid nonce. ---- */
SG_API int sg_grind(sg_ctx* ctx, void* stream, const uint64_t inner_lanes[4], uint8_t grinding_factor, uint64_t* nonce_out);


/* ---- Fiat-Shamir transcript: replaces DefaultTranscript
 *      (crypto/crypto/src/fiat_shamir/default_transcript.rs:31-146) and
 *      IsStarkTranscript::sample_z_ood_with_domain_params (is_transcript.rs:44-75).
 *      Host-side; field elements are absorbed as canonical big-endian bytes. ---- */
typedef struct sg_transcript sg_transcript;
SG_API sg_transcript* sg_transcript_new(const uint8_t* data, uint64_t len);
SG_API sg_transcript* sg_transcript_clone(const sg_transcript* t);
SG_API void sg_transcript_free(sg_transcript* t);
SG_API void sg_transcript_append(sg_transcript* t, const uint8_t* data, uint64_t len);
SG_API void sg_transcript_append_base(sg_transcript* t, uint64_t v);
SG_API void sg_transcript_append_ext3(sg_transcript* t, const uint64_t v[3]);
SG_API void sg_transcript_sample(sg_transcript* t, uint8_t out[32]);
SG_API void sg_transcript_state(const sg_transcript* t, uint8_t out[32]);
SG_API uint64_t sg_transcript_sample_base(sg_transcript* t);
SG_API void sg_transcript_sample_ext3(sg_transcript* t, uint64_t out[3]);
SG_API uint64_t sg_transcript_sample_u64(sg_transcript* t, uint64_t upper_bound);
SG_API void sg_transcript_sample_z_ood(sg_transcript* t, uint64_t trace_len, uint64_t lde_len, uint64_t coset_offset,
                                       uint64_t out[3]);
/* Keccak-256 (original padding) of a host buffer. */
SG_API void sg_keccak256(const uint8_t* data, uint64_t len, uint8_t out[32]);

/* ---- batch inversion: replaces inverse::batch_inverse_ext3 / _dev
 *      (crypto/math-cuda/src/inverse.rs:53,157). n ext3 elements in, their
 *      inverses out (may alias). zero_found (host, may be NULL) reports a zero
 *      input, for which the outputs are undefined (the reference errors). ---- */
SG_API int sg_batch_inverse_ext3(sg_ctx* ctx, void* stream, const uint64_t* d_in, uint64_t n, uint64_t* d_out,
                                 int* zero_found);
/* ---- inverse denominators: replaces inverse::compute_and_invert_denoms_ext3_dev
 *      (inverse.rs:241). d_out[k*n + i] = 1/(z_k - x_i) (x_minus_z = 0, R3 OOD)
 *      or 1/(x_i - z_k) (x_minus_z = 1, R4 DEEP); z_host: k ext3 scalars. ---- */
SG_API int sg_inv_denoms_ext3(sg_ctx* ctx, void* stream, const uint64_t* d_x, uint64_t n, const uint64_t* z_host,
                              uint32_t k, int x_minus_z, uint64_t* d_out, int* zero_found);
/* ---- barycentric OOD sums: replaces barycentric::barycentric_{base,ext3}_multi_on_device
 *      (crypto/math-cuda/src/barycentric.rs:379,449). For each of k <= 8 points
 *      and each column c < cols: d_out[k*cols + c] (ext3) =
 *      sum_{i<n} points[i] * col_c(row i*row_stride) * inv_denoms[k*n + i].
 *      d_data is row-major (row_u64 u64 per row); ext3 != 0 reads 3-u64 elements. ---- */
SG_API int sg_barycentric_sums(sg_ctx* ctx, void* stream, const uint64_t* d_data, uint64_t row_u64,
                               uint64_t row_stride, int ext3, uint64_t cols, const uint64_t* d_points,
                               const uint64_t* d_inv_denoms, uint64_t n, uint32_t k, uint64_t* d_out);
/* ---- DEEP composition: replaces deep::deep_composition_ext3_fully_resident_keep
 *      (crypto/math-cuda/src/deep.rs:316). Per LDE row i:
 *        sum_j gh_j (H_j(x_i) - h_ood_j) inv_h[i] + sum_{j,k} gt_{jk} (t_j(x_i) - t_ood_{jk}) inv_t[k*rows+i]
 *      main rows x m (base), aux rows x a (ext3), parts rows x p (ext3), all row-major;
 *      h_ood/gammas_h: p ext3 (host); trace_ood/gammas_tr: (m+a)*k ext3 (host, index j*k+kk).
 *      bitrev_out != 0 writes row i at bit-reversed position (FRI order). ---- */
SG_API int sg_deep_composition(sg_ctx* ctx, void* stream, const uint64_t* d_main, uint64_t m, const uint64_t* d_aux,
                               uint64_t a, const uint64_t* d_parts, uint64_t p, uint64_t rows, const uint64_t* h_ood,
                               const uint64_t* trace_ood, const uint64_t* gammas_h, const uint64_t* gammas_tr,
                               uint32_t k, const uint64_t* d_inv_h, const uint64_t* d_inv_t, int bitrev_out,
                               uint64_t* d_out);
/* ---- FRI fold: replaces the fold of FriCommitState::fold_and_commit_layer
 *      (crypto/math-cuda/src/fri.rs:110; fri_functions.rs:15-61). d_in: 2h ext3 in
 *      bit-reversed order; d_out[j] = (lo+hi) + inv_tw[j]*zeta*(lo-hi). Optionally
 *      writes the next layer's twiddles tw[2j]^2 (h/2) and the folded layer's
 *      Merkle leaves Keccak(out[2j] || out[2j+1]) (h/2 x 32 bytes). ---- */
SG_API int sg_fri_fold_layer(sg_ctx* ctx, void* stream, const uint64_t* d_in, uint64_t h, const uint64_t* d_inv_tw,
                             const uint64_t zeta[3], uint64_t* d_out, uint64_t* d_inv_tw_next, uint8_t* d_leaves);
/* ---- stateful FRI commit phase: replaces FriCommitState (crypto/math-cuda/src/fri.rs:48-255).
 *      sg_fri_begin (FriCommitState::new / new_dev): the bit-reversed layer-0 ext3
 *      evaluations (3*n0 u64; a device buffer is borrowed, a host one copied) and
 *      their inverse twiddles (n0/2 u64).
 *      sg_fri_fold_commit_layer (fold_and_commit_layer): fold with zeta, commit the
 *      ext3 pair leaves, root to root_out, optionally the folded evaluations to
 *      host_evals_out (want_host). sg_fri_fold_final: the last fold, uncommitted.
 *      Every committed layer stays resident (sg_fri_layer) until sg_fri_free. ---- */
typedef struct sg_fri sg_fri;
SG_API int sg_fri_begin(sg_ctx* ctx, void* stream, const uint64_t* evals, int evals_on_device, const uint64_t* inv_tw,
                        int tw_on_device, uint64_t n0, sg_fri** out);
SG_API int sg_fri_fold_commit_layer(sg_fri* fri, const uint64_t zeta[3], uint8_t root_out[32],
                                    uint64_t* host_evals_out);
SG_API int sg_fri_fold_final(sg_fri* fri, const uint64_t zeta[3], uint64_t* host_evals_out);
SG_API uint32_t sg_fri_num_layers(const sg_fri* fri);
SG_API int sg_fri_layer(const sg_fri* fri, uint32_t layer, const uint64_t** d_evals, uint64_t* n,
                        const uint8_t** d_nodes, uint64_t* leaves_len);
SG_API void sg_fri_free(sg_fri* fri);
/* FRI layer leaves over n ext3 evaluations (keccak_fri_leaves_ext3, keccak.cu:384). */
SG_API int sg_fri_leaves(sg_ctx* ctx, void* stream, const uint64_t* d_evals, uint64_t n, uint8_t* d_leaves);
/* ---- row gathers for query openings: replaces barycentric::gather_rows_{base,ext3}_on_device
 *      (barycentric.rs:522,561) and fri::gather_ext3_at (fri.rs:260): d_out[q*width + c] =
 *      d_data[rows[q]*row_u64 + col0 + c]. ---- */
SG_API int sg_gather_rows(sg_ctx* ctx, void* stream, const uint64_t* d_data, uint64_t row_u64, uint64_t nrows,
                          uint64_t col0, uint64_t width, const uint32_t* d_rows, uint32_t nq, uint64_t* d_out);

/* LogUp CSR descriptor (crypto/math-cuda/src/logup.rs:26-44), host arrays. */
typedef struct {
    uint32_t num_interactions;
    const uint64_t* bus_ids;              /* [K] */
    const uint32_t* elem_offsets;         /* [K+1] */
    const uint32_t* elem_alpha_idx;       /* [elems] */
    const uint64_t* elem_consts;          /* [elems] */
    const uint32_t* term_offsets;         /* [elems+1] */
    const uint64_t* term_coefs;           /* [terms] */
    const uint32_t* term_cols;            /* [terms] */
    uint32_t num_out_cols;                /* committed + virtual term columns */
    const uint32_t* out_col_offsets;      /* [num_out_cols+1] */
    const uint32_t* out_col_interactions; /* [...] */
    const uint64_t* mult_consts;          /* [K] */
    const uint32_t* mult_term_offsets;    /* [K+1] */
    const uint64_t* mult_term_coefs;      /* [...] */
    const uint32_t* mult_term_cols;       /* [...] */
    uint32_t num_committed;               /* the first num_committed out columns are committed */
} sg_logup_desc;
/* ---- LogUp aux build: replaces logup::logup_aux_resident (crypto/math-cuda/src/logup.rs:311;
 *      CPU lookup.rs:1660-1842). d_main: n x m row-major. d_aux: n x (num_committed+1)
 *      ext3 row-major: committed term columns then the accumulated column.
 *      alpha_powers: num_alpha ext3 (host). Writes the table contribution L. ---- */
SG_API int sg_logup_aux(sg_ctx* ctx, void* stream, const uint64_t* d_main, uint64_t n, uint64_t m,
                        const sg_logup_desc* desc, const uint64_t* alpha_powers, uint32_t num_alpha,
                        const uint64_t z[3], uint64_t* d_aux, uint64_t table_contribution[3]);


/* Lowered constraint program (DeviceProgram, crypto/stark/src/constraint_ir/device.rs):
 * nodes are {op, a, b, res} u32 quadruples with the reference's OP_* tags,
 * operand encoding (kind << 29 | payload) and RES_EXT_BIT slot packing.
 * node_roots NULL: the reference's shape (each constraint's value pinned in
 * the slot `roots` names until the walk ends). node_roots set (num_nodes
 * entries): a streaming program, as lambda_vm_b200/ir.py lowers by default —
 * node_roots[i] is the constraint instruction i completes (0xFFFFFFFF: none;
 * each constraint exactly once; `roots` unused), and operands may also be
 * trace reads, kind 7 with payload aux << 28 | frame offset << 20 | column. */
typedef struct {
    const uint32_t* nodes;
    uint32_t num_nodes;
    const uint64_t* base_consts;
    uint32_t num_base_consts;
    const uint64_t* ext_consts; /* 3 u64 per constant */
    uint32_t num_ext_consts;
    const uint32_t* roots;      /* slot | RES_EXT_BIT, one per constraint */
    uint32_t num_roots;
    uint32_t num_base_slots;
    uint32_t num_ext_slots;
    const uint32_t* node_roots; /* NULL, or num_nodes entries (streaming program) */
    uint32_t hand_kernel;       /* 0; SG_AIR_KECCAK: constraints [0, hand_roots) are the KECCAK chip
                                   table's (main width 2605); SG_AIR_CPU | chips << 8: the RV64 CPU table's
                                   with that chip set (width 200 without chips, else 234; chips as
                                   SG_RV64_CHIP_*); SG_AIR_SHIFT: the SHIFT chip table's (width 148). The
                                   library's own kernel evaluates those; the nodes complete the rest */
    uint32_t hand_roots;
    const sg_logup_desc* logup; /* NULL, or the table's LogUp descriptor in its standard layout (committed
                                   columns = interaction pairs (2p, 2p+1), then one accumulated column over
                                   the one or two interactions left): the library evaluates the table's
                                   LogUp constraints (lookup.rs:2185-2290: aux_p fa fb - ma fb - mb fa per
                                   pair, then delta f - m or delta f1 f2 - m1 f2 - m2 f1 with delta =
                                   aux'_acc - aux_acc - sum_p aux_p + table_offset; fingerprints from
                                   z = rap[0] and the alpha table) as constraints [logup_root,
                                   logup_root + num_committed + 1), which no node completes (streaming
                                   programs only) */
    uint32_t logup_root;
} sg_device_program;
#define SG_AIR_KECCAK 1u
#define SG_AIR_CPU 2u
#define SG_AIR_SHIFT 3u

/* Composition accumulation (CompositionAccum, crypto/math-cuda/src/constraint_interp.rs:157). */
typedef struct {
    const uint64_t* beta_trans; /* host: num_roots ext3 */
    const uint64_t* d_z_inv;    /* device: z_len base values, used cyclically (row % z_len) */
    uint64_t z_len;
    uint32_t num_boundary;
    const uint64_t* b_col;      /* host: num_boundary */
    const uint64_t* b_is_aux;   /* host: num_boundary (0 = main, 1 = aux) */
    const uint64_t* b_value;    /* host: num_boundary ext3 */
    const uint64_t* b_beta;     /* host: num_boundary ext3 */
    const uint64_t* d_b_z_inv;  /* device: num_boundary x rows base values */
} sg_composition;

/* ---- constraint evaluation: replaces constraint_interp::eval_composition_on_device
 *      (crypto/math-cuda/src/constraint_interp.rs:353; kernel semantics of
 *      constraint_interp.cu:379-468) when comp != NULL: d_out = H, rows ext3;
 *      and constraint_interp::eval_constraints_on_device (constraint_interp.rs:53)
 *      when comp == NULL: d_out = per-constraint evals [c*rows + row] ext3.
 *      Trace frames read row (row + offset*next_step) mod rows of the row-major
 *      main (rows x m) and aux (rows x a ext3) LDEs. rap/alpha: host ext3 tables. ---- */
SG_API int sg_eval_constraints(sg_ctx* ctx, void* stream, const sg_device_program* prog, const uint64_t* rap,
                               uint32_t n_rap, const uint64_t* alpha, uint32_t n_alpha,
                               const uint64_t table_offset[3], const uint64_t* d_main, uint64_t m,
                               const uint64_t* d_aux, uint64_t a, uint64_t rows, uint64_t next_step,
                               const sg_composition* comp, uint64_t* d_out);
/* ---- degree-2 composition split: replaces decompose_d2_ext3 (constraint_interp.cu:477;
 *      prover.rs:1557-1662). d_h: lde_rows ext3; d_inv_2x: lde_rows/2 values 1/(2x_i);
 *      d_out: lde_rows/2 rows of [H0, H1] (6 u64 per row). ---- */
SG_API int sg_decompose_d2(sg_ctx* ctx, void* stream, const uint64_t* d_h, uint64_t lde_rows, const uint64_t* d_inv_2x,
                           uint64_t* d_out);

/* ---- one table's rounds 2-4 in one call: the per-table body of the prover
 *      (crypto/stark/src/prover.rs:3603-3977 rounds 2-3, 4433-4620 round 4,
 *      fri/mod.rs:27-205 FRI commit and queries) over the kernels above:
 *      LogUp aux + commit, beta, composition + decomposition + parts commit,
 *      z_ood, OOD values (main and aux at z and z*w, parts at z^2), gamma,
 *      DEEP, FRI layers, terminal coefficients, grinding, query indexes and
 *      openings. `t` is the table's transcript fork (advanced in place).
 *      Row-pair big-endian leaves throughout; the table's boundary
 *      constraints are described by (b_col, b_is_aux, b_value) with their
 *      zerofier inverses in d_b_z_inv. ---- */
typedef struct sg_table_job {
    /* main trace and its R1 commitment (device) */
    const uint64_t* d_trace;      /* n x m */
    const uint64_t* d_main_lde;   /* N x m, N = n * blowup */
    const uint8_t* d_main_nodes;  /* node array of the main tree */
    uint64_t main_leaves_len;     /* N / 2 */
    uint64_t n, m;
    uint32_t blowup;
    uint64_t coset_offset;
    /* domain vectors (device) */
    const uint64_t* d_weights;      /* n: g^i / n */
    const uint64_t* d_comp_weights; /* N/2: g^-j / (N/2) */
    const uint64_t* d_z_inv;        /* blowup: 1 / (x^n - 1), cyclic over rows */
    const uint64_t* d_b_z_inv;      /* num_boundary x N: boundary zerofier inverses */
    const uint64_t* d_inv2x;        /* N/2: 1 / (2 x_i) */
    const uint64_t* d_pts_n;        /* n: g * w_n^i */
    const uint64_t* d_pts_N;        /* N: g * w_N^i */
    const uint64_t* d_tw0;          /* N/2: 1 / x over the bit-reversed first FRI layer */
    /* AIR */
    const sg_logup_desc* logup;
    const sg_device_program* program;
    uint32_t num_boundary;
    const uint64_t* b_col;    /* host: num_boundary */
    const uint64_t* b_is_aux; /* host: num_boundary */
    const uint64_t* b_value;  /* host: num_boundary ext3 */
    /* challenges shared by the tables of the proof (host) */
    const uint64_t* lookup_challenges; /* 2 ext3: LogUp z, alpha */
    const uint64_t* alpha_pows;
    uint32_t n_alpha;
    /* options */
    uint32_t queries;
    uint32_t grinding;
    uint32_t final_log_degree;
} sg_table_job;

/* Sizes of a table proof: A = aux_cols ext3 columns, W = m + A, Q = queries,
 * D = depth (log2 N - 1), F = fri_layers committed FRI layers. */
typedef struct sg_proof_shape {
    uint64_t aux_cols;
    uint32_t total_folds;
    uint32_t fri_layers;
    uint32_t terminal_coeffs;
    uint32_t depth;
    uint64_t fri_path_bytes; /* sum over layers l < F of Q * (D - 1 - l) * 32 */
} sg_proof_shape;
SG_API int sg_table_proof_shape(const sg_table_job* job, sg_proof_shape* shape);

/* Caller-allocated host outputs of sg_prove_table. */
typedef struct sg_table_proof {
    uint8_t* aux_root;            /* 32 */
    uint8_t* comp_root;           /* 32 */
    uint64_t* table_contribution; /* ext3 */
    uint64_t* trace_ood;          /* 2 x W ext3: [point][column], main then aux */
    uint64_t* parts_ood;          /* 2 ext3 */
    uint8_t* fri_roots;           /* F x 32 */
    uint64_t* fri_final;          /* terminal_coeffs ext3 */
    uint64_t* nonce;              /* 1 */
    uint64_t* iotas;              /* Q */
    uint64_t* open_main;          /* 2Q x m */
    uint64_t* open_aux;           /* 2Q x 3A */
    uint64_t* open_parts;         /* 2Q x 6 */
    uint8_t* path_main;           /* Q x D x 32 */
    uint8_t* path_aux;            /* Q x D x 32 */
    uint8_t* path_parts;          /* Q x D x 32 */
    uint64_t* fri_open;           /* F x 2Q ext3 */
    uint8_t* fri_paths;           /* layer after layer: Q x (D - 1 - l) x 32 */
} sg_table_proof;
SG_API int sg_prove_table(sg_ctx* ctx, void* stream, sg_transcript* t, const sg_table_job* job,
                          sg_table_proof* out);

/* ---- device field arithmetic self-test (no reference counterpart; the reference
 *      fuzzes its host field code): d_out[i] = op(d_a[i], d_b[i]) for op
 *      0 add, 1 sub, 2 mul, 3 canon, 4 neg, 5 inv, 6 sqr, 7 Fp3 mul, 8 Fp3 inverse
 *      (3 u64 per element for 7 and 8), 9 reduce of the 128-bit (d_b[i]:d_a[i]),
 *      10 sum_{j<16} d_a[i] * d_b[(i+j) mod n] accumulated unreduced, 11 d_a[i] *
 *      2^(d_b[i] mod 96) by the shift-and-reduce product the DFT butterflies use.
 *      Outputs are reduced mod p but not necessarily canonical (except 3). ---- */
SG_API int sg_field_ops(sg_ctx* ctx, void* stream, uint32_t op, const uint64_t* d_a, const uint64_t* d_b,
                        uint64_t* d_out, uint64_t n);

/* ---- synthetic chip-table trace (benchmark input generator; no counterpart in the
 *      reference, whose traces come from the VM executor): n x w row-major,
 *      element (r, c) = splitmix64(splitmix64(seed) + r*w + c) mod p, column w-2 a
 *      16-bit multiplicity, column w-1 = sum_{j<k} c_j(r) c_j(r+1 mod n). ---- */
SG_API int sg_synth_trace(sg_ctx* ctx, void* stream, uint64_t* d_out, uint64_t n, uint64_t w, uint64_t seed,
                          uint32_t k_checksum);

/* ---- batched proof verification on the GPU: the query phase of
 *      crypto/stark/src/verifier.rs (multi_verify, :1178-1430) for many tables
 *      of many proofs in one launch, one thread per (table, query). The host
 *      replays each table's transcript first (challenges, the composition
 *      identity at z, grinding, the query indexes) and passes the values below;
 *      the kernel checks, per query: the main, aux and composition openings'
 *      Merkle paths (row-pair big-endian leaves), the DEEP values at both
 *      opened rows, every FRI layer's opened value and path, and the terminal
 *      polynomial. Ext3 constants are 3 u64 each; every pointer inside the
 *      descriptor is a device pointer. status_out (host) gets one word per
 *      (table, query) in order: 0 = accepted, else code | layer << 8 with code
 *      1 main path, 2 aux path, 3 composition path, 4 FRI value, 5 FRI path,
 *      6 terminal polynomial. ---- */
typedef struct {
    uint32_t log_n, log_N;         /* trace and LDE sizes, log2 */
    uint32_t m, aux_cols;          /* main columns (base), aux columns (ext3) */
    uint32_t queries, fri_layers;  /* committed FRI layers */
    uint32_t total_folds, terminal_log, num_coeffs, pad_;
    uint64_t coset_offset, omega_N, terminal_offset, omega_T;
    /* ext3 constants, packed: z, z*w, z^2, gh[2], pood[2], gt[2*(m+A)] (column
     * major: gt[2j+k]), tood[2][m+A] (point major), zetas[total_folds], coeffs */
    const uint64_t* consts;
    const uint8_t* roots;          /* main, aux, composition, then fri_layers roots, 32 bytes each */
    const uint64_t* iotas;         /* queries */
    const uint64_t* open_main;     /* 2Q x m */
    const uint64_t* open_aux;      /* 2Q x 3A */
    const uint64_t* open_parts;    /* 2Q x 6 */
    const uint8_t* path_main;      /* Q x (log_N - 1) x 32, leaf first */
    const uint8_t* path_aux;
    const uint8_t* path_parts;
    const uint64_t* fri_open;      /* fri_layers x 2Q x 3 */
    const uint8_t* fri_paths;      /* layer after layer: Q x (log_N - 2 - l) x 32 */
} sg_verify_table;
SG_API int sg_verify_queries(sg_ctx* ctx, void* stream, const sg_verify_table* tables, uint32_t count,
                             uint32_t* status_out);

/* ---- RV64 front-end: execute a guest of RV64I-subset words (ADD, SUB, XOR,
 *      OR, AND, ADDI, XORI, ORI, ANDI, SLLI, SRLI, LUI, LD, SD, BEQ, BNE, ECALL:
 *      a7 = 93 exits, a7 = 2^64 - 2 applies keccak-f[1600] to the 25 lanes at
 *      a0; executor/src/vm semantics, the keccak ecall as
 *      executor/src/vm/instruction/execution.rs:649-670) from pc 0 with zeroed
 *      data memory, at most max_steps instructions, on the host. Fills *info
 *      (executed instructions, final a0, shifts executed, memory cells
 *      touched, keccak ecalls, SG_RV64_CHIP_* bits of the chips the run
 *      needs). Each optional output gets one record per event (size them from
 *      a first call without outputs): rows_out (8 words per executed
 *      instruction: pc | op << 32 | rd << 40 | rs1 << 48 | rs2 << 56, imm, a,
 *      b, r, memory address, the cell's previous value and timestamp; op is
 *      the ROM opcode id, 18 for a keccak ecall), regs_out (the 32 registers
 *      before every SG_RV64_REG_CHUNK-th row of an n_rows table, the final
 *      registers past the halt), counts_out (nwords: how many rows of an
 *      n_rows table execute instruction i, the halting ECALL repeated to the
 *      end), shifts_out (dir, a, amount), cells_out (address, final value,
 *      final timestamp; ascending addresses), keccak_out (timestamp, state
 *      address, 25 input lanes, the 25 cells' previous timestamps). No
 *      counterpart in the reference's math-cuda (it is the executor and trace
 *      builder of the VM crates, restricted to this subset). ---- */
#define SG_RV64_CPU_CORE_WIDTH 200
#define SG_RV64_CPU_WIDTH 234
#define SG_RV64_REG_CHUNK 64
#define SG_RV64_MEMORY_WIDTH 8
#define SG_RV64_CHIP_BITWISE 1u
#define SG_RV64_CHIP_SHIFT 2u
#define SG_RV64_CHIP_MEMORY 4u
#define SG_RV64_CHIP_KECCAK 8u
typedef struct {
    uint64_t cycles, a0, shifts, cells, keccak_calls;
    uint32_t chips, reserved;
} sg_rv64_info;
SG_API int sg_rv64_run(const uint32_t* words, uint32_t nwords, uint64_t max_steps, uint64_t n_rows,
                       uint64_t* rows_out, uint64_t* regs_out, uint64_t* counts_out, uint64_t* shifts_out,
                       uint64_t* cells_out, uint64_t* keccak_out, sg_rv64_info* info);
/* sg_rv64_run, also counting the lookups as the machine runs (both need
 * rows_out): range_counts (65536) gets how many times the CPU table (every
 * one of its n_rows rows) and the KECCAK table look each 16-bit value up in
 * RANGE; bitwise_counts (3 x 65536: XOR, OR, AND) how many times the CPU
 * table looks each byte pair x << 8 | y up in BITWISE. */
SG_API int sg_rv64_run_counted(const uint32_t* words, uint32_t nwords, uint64_t max_steps, uint64_t n_rows,
                               uint64_t* rows_out, uint64_t* regs_out, uint64_t* counts_out, uint64_t* shifts_out,
                               uint64_t* cells_out, uint64_t* keccak_out, uint64_t* range_counts,
                               uint64_t* bitwise_counts, sg_rv64_info* info);
/* sg_rv64_run_counted in one run: the library keeps the outputs, in buffers
 * that grow as the machine runs (the row records in one anonymous mapping
 * grown with mremap, so nothing is copied), for an n_rows table of the power
 * of two >= max(2, cycles) rows. sg_rv64_trace_part gives a part's words in
 * place (SG_RV64_PART_*: rows 8 per instruction, regs 32 per 64-row chunk,
 * counts nwords, shifts 3 per shift, cells 3 per touched cell, keccak 52 per
 * ecall, range_counts 65536, bitwise_counts 3 x 65536), valid until
 * sg_rv64_trace_free. */
typedef struct sg_rv64_trace sg_rv64_trace;
#define SG_RV64_PART_ROWS 0u
#define SG_RV64_PART_REGS 1u
#define SG_RV64_PART_COUNTS 2u
#define SG_RV64_PART_SHIFTS 3u
#define SG_RV64_PART_CELLS 4u
#define SG_RV64_PART_KECCAK 5u
#define SG_RV64_PART_RANGE_COUNTS 6u
#define SG_RV64_PART_BITWISE_COUNTS 7u
SG_API int sg_rv64_exec(const uint32_t* words, uint32_t nwords, uint64_t max_steps, sg_rv64_trace** out,
                        sg_rv64_info* info);
SG_API int sg_rv64_trace_part(const sg_rv64_trace* trace, uint32_t part, const uint64_t** data, uint64_t* words);
SG_API void sg_rv64_trace_free(sg_rv64_trace* trace);
/* The CPU table (n_rows x width u64, row-major, into device memory) written on
 * the device from sg_rv64_run's `count` row records and register snapshots
 * (host arrays): width SG_RV64_CPU_CORE_WIDTH (no chip instruction executed)
 * or SG_RV64_CPU_WIDTH; rows past the execution repeat the halting row, the
 * last row ends the cycle. Layout: lambda_vm_b200/rv64_air.py's CpuAir. */
SG_API int sg_rv64_cpu_table(sg_ctx* ctx, void* stream, const uint64_t* rows, uint64_t count, const uint64_t* regs,
                             uint64_t n_rows, uint32_t width, uint64_t* d_out);
/* The chip tables written on the device from sg_rv64_run's events (host
 * arrays), so the host neither builds nor uploads them: d_out gets the KECCAK table
 * (n_rows x 2605: 24 rows per ecall, the rest zero) from `count` 52-word ecall
 * records, or the SHIFT table (n_rows x 148, padding rows shift 0 by 0) from
 * `count` 3-word shift records. Layouts: lambda_vm_b200/rv64_air.py's
 * KeccakAir and ShiftAir. Asynchronous on `stream`. */
SG_API int sg_rv64_keccak_table(sg_ctx* ctx, void* stream, const uint64_t* calls, uint64_t count, uint64_t n_rows,
                                uint64_t* d_out);
SG_API int sg_rv64_shift_table(sg_ctx* ctx, void* stream, const uint64_t* shifts, uint64_t count, uint64_t n_rows,
                               uint64_t* d_out);
/* The MEMORY table (n_rows x SG_RV64_MEMORY_WIDTH: address, final value's low
 * and high 32 bits, final timestamp, active, not-the-wrap-row, the gap to the
 * next address in two 16-bit pieces) written on the device from sg_rv64_run's
 * `count` >= 1 cells (address, final value, final timestamp; addresses
 * ascending multiples of 8 below 2^32, else SG_ERR_INVALID); rows past the
 * cells continue the addresses in steps of 8. Layout:
 * lambda_vm_b200/rv64_air.py's MemoryAir. Asynchronous on `stream`. */
SG_API int sg_rv64_memory_table(sg_ctx* ctx, void* stream, const uint64_t* cells, uint64_t count, uint64_t n_rows,
                                uint64_t* d_out);

/* ---- DFT pass log: the autotuner's measurements. No counterpart in the
 *      reference (its NTT has one fixed plan). While enabled, every DFT pass
 *      launched through the context is bracketed by CUDA events; _read waits for
 *      them and returns one record per pass (its shape, the tile width used and
 *      its device time), oldest first, then clears the log. ---- */
typedef struct {
    uint32_t log_len;  /* points per tile, log2 */
    uint32_t cols;     /* tile width (columns per tile) */
    uint32_t inverse;  /* 1: inverse transform */
    uint32_t reps;     /* coset repetitions per tile (blowup for the LDE's first forward pass) */
    uint32_t pre;      /* 1: per-point coset-shift factors before the transform */
    uint32_t post;     /* 0 none, 1 four-step twiddles, 2 coset weights, 3 scalar */
    uint32_t canon;    /* 1: canonical output */
    uint32_t pad_;
    uint64_t tiles;    /* point tiles (each is log_len points x all columns) */
    uint64_t m;        /* columns */
    float ms;          /* device time of the launch */
    float pad2_;
} sg_pass_record;
SG_API int sg_ctx_pass_log(sg_ctx* ctx, int enable);
SG_API int sg_ctx_pass_log_read(sg_ctx* ctx, sg_pass_record* out, uint32_t capacity, uint32_t* count);

/* ---- learned pass-cost model. No counterpart in the reference. A small MLP
 *      (SG_MLP_IN inputs, two hidden layers of SG_MLP_HIDDEN ReLU units, one
 *      output) predicts log(ms) of a DFT pass from its shape and tile width;
 *      trained on the GPU by these kernels from pass-log measurements, it then
 *      chooses each pass's tile width in place of the timing probe.
 *      Parameters are fp32, laid out W1[H][IN], b1[H], W2[H][H], b2[H], w3[H], b3.
 *      _loss_grad: mean squared error over n samples (x: n x SG_MLP_IN row-major,
 *      y: n targets) and its gradient, one forward and backward pass, reduced in a
 *      fixed order (deterministic). _train: `steps` Adam steps on the full batch
 *      (lr, beta1 0.9, beta2 0.999, eps 1e-8), params updated in place; the final
 *      loss is written to loss_out. _predict: y = model(x). All device pointers.
 *      sg_ctx_set_pass_model installs host-side parameters in the context (count
 *      = SG_MLP_PARAMS; count 0 removes them): pass tile widths are then the
 *      model's choice, and the timing probe never runs. ---- */
#define SG_MLP_IN 16
#define SG_MLP_HIDDEN 32
#define SG_MLP_PARAMS (SG_MLP_HIDDEN * SG_MLP_IN + SG_MLP_HIDDEN + SG_MLP_HIDDEN * SG_MLP_HIDDEN + SG_MLP_HIDDEN + \
                       SG_MLP_HIDDEN + 1)
SG_API int sg_mlp_loss_grad(sg_ctx* ctx, void* stream, const float* d_x, const float* d_y, uint32_t n,
                            const float* d_params, float* d_grad, float* d_loss);
SG_API int sg_mlp_train(sg_ctx* ctx, void* stream, const float* d_x, const float* d_y, uint32_t n, float* d_params,
                        uint32_t steps, float lr, float* loss_out);
SG_API int sg_mlp_predict(sg_ctx* ctx, void* stream, const float* d_x, uint32_t n, const float* d_params,
                          float* d_out);
/* Feature vector of one DFT pass with tile width `cols` (host function; the
 * same features the model is trained on). */
SG_API void sg_pass_features(uint32_t log_len, uint64_t tiles, uint64_t m, uint32_t cols, uint32_t reps,
                             uint32_t inverse, uint32_t pre, uint32_t post, uint32_t canon, float out[SG_MLP_IN]);
SG_API int sg_ctx_set_pass_model(sg_ctx* ctx, const float* params, uint32_t count);

#ifdef __cplusplus
}
#endif
#endif /* STARKGPU_H */
