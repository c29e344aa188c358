// Internal runtime shared by the C-ABI entry points: error reporting, the
// per-GPU context (stream-ordered allocator under an HBM budget, cached
// twiddle tables) and launch helpers. Nothing here is exported.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/starkgpu.h"

// Host-side field helpers (transcript.cu); internal to the library.
extern "C" {
uint64_t sg_host_gl_canon(uint64_t a);
uint64_t sg_host_gl_add(uint64_t a, uint64_t b);
uint64_t sg_host_gl_sub(uint64_t a, uint64_t b);
uint64_t sg_host_gl_mul(uint64_t a, uint64_t b);
uint64_t sg_host_gl_pow(uint64_t a, uint64_t e);
uint64_t sg_host_gl_inv(uint64_t a);
void sg_host_fp3_add(const uint64_t* a, const uint64_t* b, uint64_t* c);
void sg_host_fp3_sub(const uint64_t* a, const uint64_t* b, uint64_t* c);
void sg_host_fp3_mul(const uint64_t* a, const uint64_t* b, uint64_t* c);
void sg_host_fp3_pow(const uint64_t* a, uint64_t e, uint64_t* out);
int sg_host_fp3_inv(const uint64_t* a, uint64_t* out);
}

namespace sg {

void set_error(const std::string& msg);
const char* last_error();

#define SG_CHECK_ARG(cond, msg)                               \
    do {                                                      \
        if (!(cond)) {                                        \
            ::sg::set_error(std::string("invalid argument: ") + (msg)); \
            return SG_ERR_INVALID;                            \
        }                                                     \
    } while (0)

#define SG_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t _e = (call);                                                        \
        if (_e != cudaSuccess) {                                                        \
            ::sg::set_error(std::string(#call) + ": " + cudaGetErrorString(_e));         \
            return _e == cudaErrorMemoryAllocation ? SG_ERR_OOM : SG_ERR_CUDA;          \
        }                                                                               \
    } while (0)

#define SG_TRY(call)               \
    do {                           \
        int _rc = (call);          \
        if (_rc != SG_OK) return _rc; \
    } while (0)

struct Ctx {
    int device = 0;
    uint64_t budget = 0;              // bytes this context may hold on the device
    std::atomic<uint64_t> in_use{0};  // bytes currently allocated through this context
    std::atomic<uint64_t> peak{0};
    std::atomic<uint64_t> launches{0};  // kernels launched through this context
    std::mutex mu;
    // W_N[e] = omega_N^e for N = 2^log, keyed by log. Device-resident, built once.
    std::map<uint32_t, uint64_t*> roots;
    // Fault injection for host-side failure tests: when > 0, the next
    // allocation that would bring the count to zero fails with SG_ERR_OOM.
    std::atomic<int64_t> fail_alloc_after{-1};
    // Stream-ordered block cache: freed blocks stay with the context, keyed by
    // capacity, each with the event recorded on the freeing stream; a later
    // allocation on any stream waits on that event before reusing the block.
    // Steady-state proofs then allocate without driver calls (growing the
    // driver pool maps physical memory and can stall for hundreds of ms).
    struct Cached {
        void* p;
        uint64_t cap;
        cudaEvent_t ev;
    };
    std::mutex cache_mu;
    std::multimap<uint64_t, Cached> free_blocks;
    std::map<void*, uint64_t> live_cap;
    std::vector<cudaEvent_t> spare_events;
    uint64_t cached_bytes = 0;
    // DFT tile widths per tile length 2^logL (ntt.cu): the compiled widths and
    // their measured time per column, filled on first use; `forced` pins a
    // width (0 = automatic). Contexts that must not allocate never tune.
    struct TileTune {
        int n = 0;
        int cols[4] = {0, 0, 0, 0};
        float cost[4] = {0, 0, 0, 0};
        int forced = 0;
    };
    TileTune tiles[13];
    std::mutex tune_mu;
    bool autotune = true;
    // Page-locked staging for uploads from pageable host memory (api.cu): two
    // halves of stage_bytes, each with the event of the copy that last read it.
    std::mutex stage_mu;
    void* stage = nullptr;
    uint64_t stage_bytes = 0;
    cudaEvent_t stage_free[2] = {nullptr, nullptr};
    // DFT pass log (ntt.cu, sg_ctx_pass_log): each pass with its events while on.
    struct PassLog {
        sg_pass_record rec;
        cudaEvent_t e0, e1;
    };
    std::atomic<bool> passlog_on{false};
    std::mutex passlog_mu;
    std::vector<PassLog> passlog;
    // Learned pass-cost model (mlp.cu): when set, DFT tile widths are its choice.
    std::vector<float> pass_model;
};

// Host-side prediction of the pass-cost model (mlp.cu): log(ms) for features x.
float mlp_predict_host(const float* params, const float* x);

// Return every cached block to the driver pool (on OOM, and at teardown).
void trim_cache(Ctx* ctx);

// Stream-ordered allocation charged against the context budget.
int dev_alloc(Ctx* ctx, cudaStream_t st, uint64_t bytes, void** out);
int dev_free(Ctx* ctx, cudaStream_t st, void* p, uint64_t bytes);

// Copy `bytes` of host memory to device memory `dst` in `st`'s order (api.cu).
// Page-locked memory goes up directly; pageable memory goes through the
// context's page-locked staging, host threads copying one chunk into a
// staging half while the previous chunk's DMA is in flight (the driver's own
// staging of a pageable copy runs at a few GB/s).
// `check`, when given, is called on every byte range [lo, hi) of the upload
// by the host thread that copies it (while the bytes are in its cache); a
// false return makes the call fail with SG_ERR_INVALID once the copies are
// enqueued (the caller frees `dst` in stream order).
int upload_host(Ctx* ctx, cudaStream_t st, const void* host, uint64_t bytes, void* dst,
                const std::function<bool(uint64_t lo, uint64_t hi)>& check = nullptr);

// f(lo, hi) over contiguous slices of [0, n), at least `grain` items a slice,
// on up to 16 host threads; the calling thread takes the first slice.
template <class F>
void host_parallel(uint64_t n, uint64_t grain, F f) {
    const unsigned hw = std::thread::hardware_concurrency();
    const uint64_t T = std::max<uint64_t>(1, std::min<uint64_t>({hw ? hw : 1u, 16u, n / (grain ? grain : 1)}));
    std::vector<std::thread> th;
    for (uint64_t t = 1; t < T; ++t) th.emplace_back([&f, n, T, t] { f(n * t / T, n * (t + 1) / T); });
    f(0, n / T);
    for (auto& x : th) x.join();
}

// Table of omega_{2^log}^e, e in [0, 2^log), cached per context.
int roots_table(Ctx* ctx, cudaStream_t st, uint32_t log, const uint64_t** out);

inline int log2_exact(uint64_t n) {
    if (n == 0 || (n & (n - 1))) return -1;
    int l = 0;
    while ((1ULL << l) < n) ++l;
    return l;
}

// Make the context's GPU current on the calling thread. CUDA's current device
// is per host thread and a thread that never chose one runs on device 0, so
// every entry point that takes a context calls this before any CUDA call:
// worker threads of a table scheduler or a proof server then launch on the
// context's GPU whichever thread they are. Cheap when it is already current.
inline Ctx* ctx_of(sg_ctx* c) { return reinterpret_cast<Ctx*>(c); }
inline int enter(Ctx* ctx) {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur == ctx->device) return SG_OK;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) {
        set_error(std::string("cudaSetDevice(") + std::to_string(ctx->device) + "): " + cudaGetErrorString(e));
        return SG_ERR_CUDA;
    }
    return SG_OK;
}
#define SG_ENTER(ctx) SG_TRY(::sg::enter(ctx))

// Launch facts of one kernel on the current device: its SM count and how many
// CTAs of `threads` threads and `smem` dynamic shared memory bytes fit on one
// SM. The first query per (kernel, device) also raises the kernel's dynamic
// shared-memory limit when smem exceeds 48 KB; that attribute is per device,
// so each GPU of a process gets it on its first launch there.
struct KernelInfo {
    int sms = 0;
    int blocks_per_sm = 0;
};
int kernel_info(const void* fn, size_t smem, int threads, KernelInfo* out);

inline int check_launch(Ctx* ctx, const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string(what) + ": " + cudaGetErrorString(e));
        return SG_ERR_CUDA;
    }
    ctx->launches.fetch_add(1, std::memory_order_relaxed);
    return SG_OK;
}

// ---- internal kernel drivers (ntt.cu, merkle.cu) ----
enum Dir { FWD = 0, INV = 1 };
// Batched natural-order DFT over the rows of a row-major n x m matrix.
int ntt_rows(Ctx* ctx, cudaStream_t st, uint64_t* d, uint64_t n, uint64_t m, int inverse, int scale_inverse);
// Coset LDE: out ((B*n) x m, row-major, canonical) from trace (n x m) and coset weights.
int coset_lde(Ctx* ctx, cudaStream_t st, const uint64_t* trace, uint64_t n, uint64_t m, uint64_t blowup,
              const uint64_t* weights, uint64_t* out);
// The same over m columns of wider row-major matrices: trace rows of trace_ld
// u64, output rows of out_ld u64 (a column range of each, by pointer offset).
int coset_lde_ld(Ctx* ctx, cudaStream_t st, const uint64_t* trace, uint64_t trace_ld, uint64_t n, uint64_t m,
                 uint64_t blowup, const uint64_t* weights, uint64_t* out, uint64_t out_ld);
// One table's LDE for lde_multi: its input, output and scratch (coef n x m,
// tmp n x m when n > 4096).
struct LdeJob {
    const uint64_t* trace;
    uint64_t trace_ld, n, m, blowup;
    const uint64_t* weights;
    uint64_t* out;
    uint64_t out_ld;
    uint64_t* coef;
    uint64_t* tmp;
};
// The LDEs of many tables with one multi-table launch per pass group.
int lde_multi(Ctx* ctx, cudaStream_t st, const LdeJob* jobs, uint32_t count);
int leaves_row_major(Ctx* ctx, cudaStream_t st, const uint64_t* data, uint64_t num_rows, uint64_t row_u64,
                     uint64_t col_start, uint64_t col_end, uint32_t rows_per_leaf, int little_endian,
                     uint8_t* out);
int merkle_inner(Ctx* ctx, cudaStream_t st, uint8_t* nodes, uint64_t num_leaves_pow2);

// FRI commit steps on the device (rounds.cu). fri_state_load_dev puts a host
// transcript state (an fs::State) into device memory; fri_challenge_dev
// absorbs d_root (32 bytes, or nothing when null; copied to d_root_out) into
// the state at d_state and samples the next challenge into d_zeta (3 u64),
// which fri_fold_dev's fold reads.
int fri_state_load_dev(Ctx* ctx, cudaStream_t st, const void* host_state, void* d_state);
int fri_challenge_dev(Ctx* ctx, cudaStream_t st, void* d_state, const uint8_t* d_root, uint8_t* d_root_out,
                      uint64_t* d_zeta);
int fri_fold_dev(Ctx* ctx, cudaStream_t st, const uint64_t* d_in, uint64_t h, const uint64_t* d_inv_tw,
                 const uint64_t* d_zeta, uint64_t* d_out, uint64_t* d_inv_tw_next, uint8_t* d_leaves);
// One-row leaves absorbed in column windows [c0, c0 + w) with the sponge
// state (25 x num_rows u64) kept in HBM between windows; see merkle.cu.
int leaves_window(Ctx* ctx, cudaStream_t st, const uint64_t* data, uint64_t num_rows, uint64_t row_u64, uint64_t c0,
                  uint64_t w, int little_endian, uint64_t* state, int first, int last, uint8_t* out);
int pad_leaves(Ctx* ctx, cudaStream_t st, uint8_t* leaves, uint64_t n, uint64_t L);

}  // namespace sg
