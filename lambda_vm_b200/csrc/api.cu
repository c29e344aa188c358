// C-ABI entry points: context, memory, NTT/LDE, leaves, tree, LDE + commit.
// The per-function reference correspondences are listed in include/starkgpu.h.
#include <string.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

namespace sg {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
const char* last_error() { return g_err.c_str(); }

// Capacity classes: 512-byte granularity up to 2 MiB, then eight classes per
// power of two (at most 12.5 % slack), so freed blocks fit later requests of
// nearby sizes.
static uint64_t cap_of(uint64_t b) {
    if (b <= (2ull << 20)) return (b + 511) & ~511ull;
    const int lg = 63 - __builtin_clzll(b);
    const uint64_t step = 1ull << (lg - 3);
    return (b + step - 1) & ~(step - 1);
}

void trim_cache(Ctx* ctx) {
    std::vector<Ctx::Cached> blocks;
    {
        std::lock_guard<std::mutex> g(ctx->cache_mu);
        for (auto& kv : ctx->free_blocks) blocks.push_back(kv.second);
        ctx->free_blocks.clear();
        ctx->cached_bytes = 0;
    }
    for (auto& b : blocks) {
        cudaEventSynchronize(b.ev);
        cudaFree(b.p);
        cudaEventDestroy(b.ev);
    }
}

int dev_alloc(Ctx* ctx, cudaStream_t st, uint64_t bytes, void** out) {
    *out = nullptr;
    if (bytes == 0) return SG_OK;
    int64_t f = ctx->fail_alloc_after.load();
    if (f > 0) {
        if (ctx->fail_alloc_after.fetch_sub(1) == 1) {
            set_error("injected allocation failure");
            return SG_ERR_OOM;
        }
    }
    uint64_t cur = ctx->in_use.fetch_add(bytes) + bytes;
    if (cur > ctx->budget) {
        ctx->in_use.fetch_sub(bytes);
        set_error("HBM budget exceeded: need " + std::to_string(bytes) + " bytes, budget " +
                  std::to_string(ctx->budget) + ", in use " + std::to_string(cur - bytes));
        return SG_ERR_BUDGET;
    }
    uint64_t pk = ctx->peak.load();
    while (cur > pk && !ctx->peak.compare_exchange_weak(pk, cur)) {
    }
    const uint64_t cap = cap_of(bytes);
    {
        std::lock_guard<std::mutex> g(ctx->cache_mu);
        auto it = ctx->free_blocks.lower_bound(cap);
        if (it != ctx->free_blocks.end() && it->first <= cap + cap / 4) {
            Ctx::Cached b = it->second;
            ctx->free_blocks.erase(it);
            ctx->cached_bytes -= b.cap;
            ctx->live_cap[b.p] = b.cap;
            // The block's last use was on the freeing stream: order this stream after it.
            cudaError_t e = cudaStreamWaitEvent(st, b.ev, 0);
            ctx->spare_events.push_back(b.ev);
            if (e != cudaSuccess) {
                ctx->live_cap.erase(b.p);
                ctx->in_use.fetch_sub(bytes);
                set_error(std::string("cudaStreamWaitEvent: ") + cudaGetErrorString(e));
                return SG_ERR_CUDA;
            }
            *out = b.p;
            return SG_OK;
        }
    }
    cudaError_t e = cudaMallocAsync(out, cap, st);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        trim_cache(ctx);
        e = cudaMallocAsync(out, cap, st);
    }
    if (e != cudaSuccess) {
        ctx->in_use.fetch_sub(bytes);
        *out = nullptr;
        set_error(std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? SG_ERR_OOM : SG_ERR_CUDA;
    }
    std::lock_guard<std::mutex> g(ctx->cache_mu);
    ctx->live_cap[*out] = cap;
    return SG_OK;
}

int dev_free(Ctx* ctx, cudaStream_t st, void* p, uint64_t bytes) {
    if (!p) return SG_OK;
    ctx->in_use.fetch_sub(bytes);
    cudaEvent_t ev = nullptr;
    uint64_t cap = 0;
    {
        std::lock_guard<std::mutex> g(ctx->cache_mu);
        auto it = ctx->live_cap.find(p);
        if (it == ctx->live_cap.end()) {
            set_error("dev_free: pointer not allocated by this context");
            return SG_ERR_INVALID;
        }
        cap = it->second;
        ctx->live_cap.erase(it);
        if (!ctx->spare_events.empty()) {
            ev = ctx->spare_events.back();
            ctx->spare_events.pop_back();
        }
    }
    cudaError_t e = ev ? cudaSuccess : cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ev, st);
    if (e != cudaSuccess) {
        // Without an event the block cannot be reused safely: hand it back to the pool.
        if (ev) cudaEventDestroy(ev);
        cudaError_t e2 = cudaFreeAsync(p, st);
        set_error(std::string("dev_free: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
        return SG_ERR_CUDA;
    }
    std::lock_guard<std::mutex> g(ctx->cache_mu);
    ctx->free_blocks.insert({cap, Ctx::Cached{p, cap, ev}});
    ctx->cached_bytes += cap;
    return SG_OK;
}

int kernel_info(const void* fn, size_t smem, int threads, KernelInfo* out) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, KernelInfo> cache;
    int dev = 0;
    SG_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find({fn, dev});
    if (it != cache.end()) {
        *out = it->second;
        return SG_OK;
    }
    KernelInfo k;
    if (smem > 48 * 1024) SG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    SG_CUDA(cudaDeviceGetAttribute(&k.sms, cudaDevAttrMultiProcessorCount, dev));
    SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k.blocks_per_sm, fn, threads, smem));
    if (k.sms < 1) k.sms = 1;
    if (k.blocks_per_sm < 1) k.blocks_per_sm = 1;
    cache[{fn, dev}] = k;
    *out = k;
    return SG_OK;
}

}  // namespace sg

using namespace sg;

struct sg_lde {
    uint64_t* d_lde = nullptr;
    uint64_t lde_rows = 0, row_u64 = 0;
    uint8_t* d_nodes = nullptr;
    uint64_t leaves_len = 0;
    uint8_t root[32] = {0};
};

static Ctx* C(sg_ctx* c) { return reinterpret_cast<Ctx*>(c); }

extern "C" {

const char* sg_last_error(void) { return last_error(); }

int sg_ctx_create(int device, uint64_t budget, sg_ctx** out) {
    SG_CHECK_ARG(out, "null output");
    *out = nullptr;
    int count = 0;
    SG_CUDA(cudaGetDeviceCount(&count));
    SG_CHECK_ARG(device >= 0 && device < count, "device index out of range");
    SG_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    SG_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) {
        set_error("this library is built for sm_100a (B200); found sm_" + std::to_string(prop.major) +
                  std::to_string(prop.minor));
        return SG_ERR_UNSUPPORTED;
    }
    Ctx* ctx = new Ctx();
    ctx->device = device;
    size_t free_b = 0, total_b = 0;
    SG_CUDA(cudaMemGetInfo(&free_b, &total_b));
    ctx->budget = budget ? budget : (uint64_t)(0.9 * (double)free_b);
    // Keep freed blocks in the stream-ordered pool instead of returning them to
    // the driver each time: repeated commits then allocate without syscalls.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = ctx->budget;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    *out = reinterpret_cast<sg_ctx*>(ctx);
    return SG_OK;
}

void sg_ctx_destroy(sg_ctx* c) {
    Ctx* ctx = C(c);
    if (!ctx) return;
    enter(ctx);  // best effort: teardown continues either way
    cudaDeviceSynchronize();
    trim_cache(ctx);
    for (auto& kv : ctx->live_cap) cudaFree(kv.first);
    for (auto ev : ctx->spare_events) cudaEventDestroy(ev);
    for (auto& kv : ctx->roots) cudaFree(kv.second);
    for (auto e : ctx->stage_free)
        if (e) cudaEventDestroy(e);
    if (ctx->stage) cudaFreeHost(ctx->stage);
    delete ctx;
}

int sg_ctx_memory(sg_ctx* c, uint64_t* in_use, uint64_t* peak) {
    SG_CHECK_ARG(c, "null context");
    SG_ENTER(ctx_of(c));
    if (in_use) *in_use = C(c)->in_use.load();
    if (peak) *peak = C(c)->peak.load();
    return SG_OK;
}

uint64_t sg_ctx_launches(sg_ctx* c) { return c ? C(c)->launches.load() : 0; }

uint64_t sg_ctx_budget(sg_ctx* c) { return c ? C(c)->budget : 0; }

int sg_ctx_fail_alloc_after(sg_ctx* c, int64_t n) {
    SG_CHECK_ARG(c && n >= 0, "bad argument");
    SG_ENTER(ctx_of(c));
    C(c)->fail_alloc_after.store(n == 0 ? -1 : n);
    return SG_OK;
}

int sg_dev_alloc(sg_ctx* c, void* stream, uint64_t bytes, void** d_out) {
    SG_CHECK_ARG(c && d_out, "null argument");
    SG_ENTER(ctx_of(c));
    return dev_alloc(C(c), (cudaStream_t)stream, bytes, d_out);
}

int sg_dev_free(sg_ctx* c, void* stream, void* p, uint64_t bytes) {
    SG_CHECK_ARG(c, "null context");
    SG_ENTER(ctx_of(c));
    return dev_free(C(c), (cudaStream_t)stream, p, bytes);
}

int sg_memcpy_h2d(sg_ctx* c, void* stream, void* dst, const void* src, uint64_t bytes) {
    SG_CHECK_ARG(c, "null context");
    SG_ENTER(ctx_of(c));
    if (!bytes) return SG_OK;
    SG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream));
    return SG_OK;
}

int sg_memcpy_d2h(sg_ctx* c, void* stream, void* dst, const void* src, uint64_t bytes) {
    SG_CHECK_ARG(c, "null context");
    SG_ENTER(ctx_of(c));
    if (!bytes) return SG_OK;
    SG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    return SG_OK;
}

int sg_stream_sync(sg_ctx* c, void* stream) {
    SG_CHECK_ARG(c, "null context");
    SG_ENTER(ctx_of(c));
    SG_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return SG_OK;
}

int sg_stream_create(sg_ctx* c, void** out) {
    SG_CHECK_ARG(c && out, "null argument");
    SG_ENTER(ctx_of(c));
    cudaStream_t st;
    SG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    *out = (void*)st;
    return SG_OK;
}

int sg_stream_create_priority(sg_ctx* c, int priority, void** out) {
    SG_CHECK_ARG(c && out, "null argument");
    SG_ENTER(ctx_of(c));
    cudaStream_t st;
    SG_CUDA(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, priority));
    *out = (void*)st;
    return SG_OK;
}

int sg_stream_priority_range(sg_ctx* c, int* least, int* greatest) {
    SG_CHECK_ARG(c && least && greatest, "null argument");
    SG_ENTER(ctx_of(c));
    SG_CUDA(cudaDeviceGetStreamPriorityRange(least, greatest));
    return SG_OK;
}

int sg_stream_destroy(sg_ctx* c, void* stream) {
    SG_CHECK_ARG(c, "null context");
    SG_ENTER(ctx_of(c));
    if (stream) SG_CUDA(cudaStreamDestroy((cudaStream_t)stream));
    return SG_OK;
}

int sg_host_alloc(uint64_t bytes, void** out) {
    SG_CHECK_ARG(out, "null output");
    SG_CUDA(cudaMallocHost(out, bytes ? bytes : 1));
    return SG_OK;
}

int sg_host_free(void* p) {
    if (p) SG_CUDA(cudaFreeHost(p));
    return SG_OK;
}

int sg_ntt_forward(sg_ctx* c, void* stream, uint64_t* d, uint64_t n, uint64_t m) {
    SG_CHECK_ARG(c, "null context");
    SG_ENTER(ctx_of(c));
    return ntt_rows(C(c), (cudaStream_t)stream, d, n, m, 0, 0);
}

int sg_ntt_inverse(sg_ctx* c, void* stream, uint64_t* d, uint64_t n, uint64_t m) {
    SG_CHECK_ARG(c, "null context");
    SG_ENTER(ctx_of(c));
    return ntt_rows(C(c), (cudaStream_t)stream, d, n, m, 1, 1);
}

int sg_coset_lde(sg_ctx* c, void* stream, const uint64_t* d_trace, uint64_t n, uint64_t m, uint32_t blowup,
                 const uint64_t* d_weights, uint64_t* d_out) {
    SG_CHECK_ARG(c, "null context");
    SG_ENTER(ctx_of(c));
    SG_CHECK_ARG(blowup >= 1, "blowup must be >= 1");
    if (n == 0 || m == 0) return SG_OK;
    SG_CHECK_ARG(d_trace && d_weights && d_out, "null buffer");
    return coset_lde(C(c), (cudaStream_t)stream, d_trace, n, m, blowup, d_weights, d_out);
}

static int resolve_layout(const sg_leaf_layout* lay, uint64_t row_u64, uint32_t* R, int* le, uint64_t* c0,
                          uint64_t* c1) {
    sg_leaf_layout d = {2, 0, 0, 0};
    if (!lay) lay = &d;
    *R = lay->rows_per_leaf;
    *le = lay->little_endian ? 1 : 0;
    *c0 = lay->col_start;
    *c1 = lay->col_end ? lay->col_end : row_u64;
    SG_CHECK_ARG(*R >= 1, "rows_per_leaf must be >= 1");
    SG_CHECK_ARG(*c0 < *c1 && *c1 <= row_u64, "leaf column range");
    return SG_OK;
}

int sg_keccak_leaves(sg_ctx* c, void* stream, const uint64_t* d_data, uint64_t num_rows, uint64_t row_u64,
                     const sg_leaf_layout* layout, uint8_t* d_out) {
    SG_CHECK_ARG(c, "null context");
    SG_ENTER(ctx_of(c));
    if (num_rows == 0) return SG_OK;
    uint32_t R;
    int le;
    uint64_t c0, c1;
    SG_TRY(resolve_layout(layout, row_u64, &R, &le, &c0, &c1));
    return leaves_row_major(C(c), (cudaStream_t)stream, d_data, num_rows, row_u64, c0, c1, R, le, d_out);
}

uint64_t sg_merkle_leaves_len(uint64_t num_leaves) {
    uint64_t L = 1;
    while (L < num_leaves) L <<= 1;
    return num_leaves ? L : 0;
}

int sg_merkle_build(sg_ctx* c, void* stream, const uint8_t* d_leaves, uint64_t num_leaves, uint8_t* d_nodes,
                    uint8_t root_out[32]) {
    SG_CHECK_ARG(c, "null context");
    SG_ENTER(ctx_of(c));
    SG_CHECK_ARG(num_leaves > 0, "empty leaf set");
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t L = sg_merkle_leaves_len(num_leaves);
    uint8_t* leaf_dst = d_nodes + (L - 1) * 32;
    if (leaf_dst != d_leaves) SG_CUDA(cudaMemcpyAsync(leaf_dst, d_leaves, num_leaves * 32, cudaMemcpyDeviceToDevice, st));
    SG_TRY(pad_leaves(C(c), st, leaf_dst, num_leaves, L));
    SG_TRY(merkle_inner(C(c), st, d_nodes, L));
    if (root_out) {
        SG_CUDA(cudaMemcpyAsync(root_out, d_nodes, 32, cudaMemcpyDeviceToHost, st));
        SG_CUDA(cudaStreamSynchronize(st));
    }
    return SG_OK;
}

}  // extern "C"

// Host trace -> LDE with the upload overlapped: the columns go up in chunks
// of kChunkCols on a copy stream (one strided copy each), and each chunk's
// LDE starts on `st` as soon as its copy lands, so the PCIe transfer of the
// later chunks runs under the DFT passes of the earlier ones. With a
// page-locked host trace the copies are asynchronous; with pageable memory
// they are staged by the driver and the overlap is lost, not the result.
static constexpr uint64_t kChunkCols = 32;  // fastest of 16/24/32/48/64 at 2^20 x 256

// A non-blocking stream with the scheduling priority of `like` (the legacy
// default stream counts as the default priority).
static cudaError_t new_stream_like(cudaStream_t like, cudaStream_t* out) {
    int prio = 0;
    if (like && cudaStreamGetPriority(like, &prio) != cudaSuccess) prio = 0;
    return cudaStreamCreateWithPriority(out, cudaStreamNonBlocking, prio);
}

// Copy columns [c0, c0 + w) of an n x m row-major host matrix into a dense
// n x w buffer, rows split across host threads (each row is one w*8-byte copy).
static void gather_columns(uint64_t* dst, const uint64_t* src, uint64_t n, uint64_t m, uint64_t c0, uint64_t w) {
    const unsigned hw = std::thread::hardware_concurrency();
    const uint64_t T = std::max<uint64_t>(1, std::min<uint64_t>({hw ? hw : 1u, 16u, (n + 4095) / 4096}));
    auto part = [&](uint64_t t) {
        const uint64_t r0 = n * t / T, r1 = n * (t + 1) / T;
        for (uint64_t r = r0; r < r1; ++r) memcpy(dst + r * w, src + r * m + c0, w * 8);
    };
    std::vector<std::thread> th;
    for (uint64_t t = 1; t < T; ++t) th.emplace_back(part, t);
    part(0);
    for (auto& x : th) x.join();
}

// Page-locked staging for host traces in pageable memory: two halves of at
// least `half_bytes`, kept by the context and reused by later calls. The
// DMA engine can read only page-locked memory, so a pageable copy is staged
// by the driver one small bounce buffer at a time (2 GiB took 350 ms); here
// host threads gather a column chunk into one half while the previous chunk
// goes up from the other. Called with ctx->stage_mu held.
static int stage_reserve(Ctx* ctx, uint64_t half_bytes) {
    if (ctx->stage && ctx->stage_bytes >= half_bytes) return SG_OK;
    for (auto& e : ctx->stage_free)
        if (e) SG_CUDA(cudaEventSynchronize(e));
    if (ctx->stage) {
        cudaFreeHost(ctx->stage);
        ctx->stage = nullptr;
        ctx->stage_bytes = 0;
    }
    SG_CUDA(cudaMallocHost(&ctx->stage, 2 * half_bytes));
    ctx->stage_bytes = half_bytes;
    for (auto& e : ctx->stage_free)
        if (!e) SG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return SG_OK;
}

int sg::upload_host(Ctx* ctx, cudaStream_t st, const void* host, uint64_t bytes, void* dst,
                    const std::function<bool(uint64_t lo, uint64_t hi)>& check) {
    if (!bytes) return SG_OK;
    std::atomic<bool> bad{false};
    cudaPointerAttributes pa;
    const bool pageable = cudaPointerGetAttributes(&pa, host) != cudaSuccess || pa.type == cudaMemoryTypeUnregistered;
    cudaGetLastError();
    constexpr uint64_t kDirect = 4ull << 20, kPiece = 32ull << 20;
    if (!pageable || bytes <= kDirect) {
        if (check) host_parallel(bytes, 1ull << 20, [&](uint64_t lo, uint64_t hi) {
            if (!check(lo, hi)) bad = true;
        });
        SG_CHECK_ARG(!bad.load(), "bad input records");
        SG_CUDA(cudaMemcpyAsync(dst, host, bytes, cudaMemcpyHostToDevice, st));
        return SG_OK;
    }
    std::lock_guard<std::mutex> lock(ctx->stage_mu);
    SG_TRY(stage_reserve(ctx, std::min(bytes, kPiece)));
    const uint64_t piece = std::min(ctx->stage_bytes, kPiece);
    // the first pieces are small, so the device starts copying soon (the
    // host fills a piece before its copy can start); then they double
    uint64_t len = std::min<uint64_t>(piece, kDirect);
    for (uint64_t off = 0, k = 0; off < bytes; off += len, len = std::min(2 * len, piece), ++k) {
        len = std::min(len, bytes - off);
        uint8_t* half = (uint8_t*)ctx->stage + (k & 1) * ctx->stage_bytes;
        const uint8_t* src = (const uint8_t*)host + off;
        // the half is free once its previous copy (this call's or an earlier one's) has left it
        SG_CUDA(cudaEventSynchronize(ctx->stage_free[k & 1]));
        host_parallel(len, 1ull << 20, [&](uint64_t lo, uint64_t hi) {
            memcpy(half + lo, src + lo, hi - lo);
            if (check && !check(off + lo, off + hi)) bad = true;
        });
        SG_CUDA(cudaMemcpyAsync((uint8_t*)dst + off, half, len, cudaMemcpyHostToDevice, st));
        SG_CUDA(cudaEventRecord(ctx->stage_free[k & 1], st));
    }
    SG_CHECK_ARG(!bad.load(), "bad input records");
    return SG_OK;
}

// When `leaves` is non-null the commit's leaves are one LDE row each over the
// whole row: they are then absorbed window by window as the LDE columns
// complete (whole 17-lane sponge blocks), so hashing also runs under the
// upload, and the digests land in `leaves` when the last window is done.
struct LeafSink {
    uint8_t* leaves;
    int little_endian;
    uint64_t* state;  // 25 x lde_rows u64
};

static int upload_and_lde(Ctx* ctx, cudaStream_t st, const uint64_t* h_trace, uint64_t* d_trace, uint64_t n,
                          uint64_t m, uint64_t blowup, const uint64_t* d_w, uint64_t* d_lde,
                          const LeafSink* sink = nullptr) {
    const uint64_t chunk = m >= 2 * kChunkCols ? kChunkCols : m;
    const uint64_t nchunks = (m + chunk - 1) / chunk;
    cudaStream_t cs = nullptr;
    uint64_t absorbed = 0;  // leaf columns absorbed so far (a multiple of 17)
    std::vector<cudaEvent_t> ev(nchunks + 1, nullptr);
    int rc = SG_OK;
    auto ok = [&](cudaError_t e, const char* what) {
        if (e != cudaSuccess && rc == SG_OK) {
            set_error(std::string("trace upload: ") + what + ": " + cudaGetErrorString(e));
            rc = SG_ERR_CUDA;
        }
        return rc == SG_OK;
    };
    if (ok(new_stream_like(st, &cs), "stream")) {
        for (auto& e : ev)
            if (!ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event")) break;
    }
    // the copy stream starts after d_trace is valid in `st`'s order
    if (rc == SG_OK && ok(cudaEventRecord(ev[nchunks], st), "record")) ok(cudaStreamWaitEvent(cs, ev[nchunks], 0), "wait");
    // pageable host memory goes through the context's page-locked staging
    cudaPointerAttributes pa;
    const bool pageable = cudaPointerGetAttributes(&pa, h_trace) != cudaSuccess || pa.type == cudaMemoryTypeUnregistered;
    cudaGetLastError();
    std::unique_lock<std::mutex> stage_lock(ctx->stage_mu, std::defer_lock);
    if (pageable && rc == SG_OK) {
        stage_lock.lock();
        rc = stage_reserve(ctx, n * chunk * 8);
    }
    for (uint64_t k = 0; k < nchunks && rc == SG_OK; ++k) {
        const uint64_t c0 = k * chunk, w = m - c0 < chunk ? m - c0 : chunk;
        if (pageable) {
            // wait until the half's previous copy (this call's or an earlier one's) has left it
            uint64_t* half = (uint64_t*)ctx->stage + (k & 1) * (ctx->stage_bytes / 8);
            if (!ok(cudaEventSynchronize(ctx->stage_free[k & 1]), "staging wait")) break;
            gather_columns(half, h_trace, n, m, c0, w);
            if (!ok(cudaMemcpy2DAsync(d_trace + c0, m * 8, half, w * 8, w * 8, n, cudaMemcpyHostToDevice, cs),
                    "copy") ||
                !ok(cudaEventRecord(ctx->stage_free[k & 1], cs), "record"))
                break;
        } else if (!ok(cudaMemcpy2DAsync(d_trace + c0, m * 8, h_trace + c0, m * 8, w * 8, n, cudaMemcpyHostToDevice,
                                         cs),
                       "copy")) {
            break;
        }
        if (!ok(cudaEventRecord(ev[k], cs), "record") || !ok(cudaStreamWaitEvent(st, ev[k], 0), "wait")) break;
        rc = coset_lde_ld(ctx, st, d_trace + c0, m, n, w, blowup, d_w, d_lde + c0, m);
        if (rc == SG_OK && sink) {
            // absorb every whole sponge block now complete; the tail with the last chunk
            const uint64_t done = (c0 + w == m) ? m : (c0 + w) / 17 * 17;
            const uint64_t from = absorbed;
            if (done > from || c0 + w == m) {
                rc = leaves_window(ctx, st, d_lde, n * blowup, m, from, done - from, sink->little_endian,
                                   sink->state, from == 0, c0 + w == m, sink->leaves);
                absorbed = done;
            }
        }
    }
    // On success the copy stream's work is ordered before `st` through the
    // events; after a failure part of it may not be, so drain it before the
    // caller frees the buffers. Its resources are released once it completes.
    if (cs && rc != SG_OK) cudaStreamSynchronize(cs);
    if (cs) cudaStreamDestroy(cs);
    for (auto e : ev)
        if (e) cudaEventDestroy(e);
    return rc;
}

// Enqueue one table's commit on `st` without waiting on the host: weights and
// trace upload (when given on the host), coset LDE, leaves and tree; the root
// is node 0 of the handle's node array. On failure nothing stays allocated and
// *out is null.
static int commit_enqueue(Ctx* ctx, cudaStream_t st, const uint64_t* trace, int trace_on_device, uint64_t n,
                          uint64_t row_u64, uint32_t blowup, const uint64_t* weights, int weights_on_device,
                          const sg_leaf_layout* layout, uint64_t* host_lde_out, sg_lde** out) {
    SG_CHECK_ARG(out && trace && weights, "null argument");
    *out = nullptr;
    SG_CHECK_ARG(n >= 2 && log2_exact(n) >= 0, "n must be a power of two >= 2");
    SG_CHECK_ARG(blowup >= 1 && log2_exact(blowup) >= 0, "blowup must be a power of two");
    SG_CHECK_ARG(row_u64 >= 1, "row width must be >= 1");
    uint32_t R;
    int le;
    uint64_t c0, c1;
    SG_TRY(resolve_layout(layout, row_u64, &R, &le, &c0, &c1));
    const uint64_t lde_rows = n * blowup;
    SG_CHECK_ARG(lde_rows % R == 0, "rows_per_leaf must divide the LDE size");
    const uint64_t L = lde_rows / R;  // power of two
    sg_lde* h = new sg_lde();
    h->lde_rows = lde_rows;
    h->row_u64 = row_u64;
    h->leaves_len = L;
    uint64_t* d_trace = nullptr;
    uint64_t* d_w = nullptr;
    uint64_t* d_state = nullptr;
    const uint64_t trace_bytes = n * row_u64 * 8;
    int rc = SG_OK;
    do {
        rc = dev_alloc(ctx, st, lde_rows * row_u64 * 8, (void**)&h->d_lde);
        if (rc) break;
        rc = dev_alloc(ctx, st, (2 * L - 1) * 32, (void**)&h->d_nodes);
        if (rc) break;
        const uint64_t* w = weights;
        if (!weights_on_device) {
            rc = dev_alloc(ctx, st, n * 8, (void**)&d_w);
            if (rc) break;
            if (cudaMemcpyAsync(d_w, weights, n * 8, cudaMemcpyHostToDevice, st) != cudaSuccess) {
                set_error("weights upload failed");
                rc = SG_ERR_CUDA;
                break;
            }
            w = d_w;
        }
        uint8_t* leaf_out = h->d_nodes + (L - 1) * 32;
        bool leaves_done = false;
        if (trace_on_device) {
            rc = coset_lde(ctx, st, trace, n, row_u64, blowup, w, h->d_lde);
        } else {
            rc = dev_alloc(ctx, st, trace_bytes, (void**)&d_trace);
            if (rc) break;
            // one-row leaves over whole rows are hashed as the columns arrive
            if (R == 1 && c0 == 0 && c1 == row_u64 && row_u64 >= 2 * kChunkCols) {
                rc = dev_alloc(ctx, st, 25 * lde_rows * 8, (void**)&d_state);
                if (rc) break;
                LeafSink sink{leaf_out, le, d_state};
                rc = upload_and_lde(ctx, st, trace, d_trace, n, row_u64, blowup, w, h->d_lde, &sink);
                leaves_done = true;
            } else {
                rc = upload_and_lde(ctx, st, trace, d_trace, n, row_u64, blowup, w, h->d_lde);
            }
        }
        if (rc) break;
        if (!leaves_done) rc = leaves_row_major(ctx, st, h->d_lde, lde_rows, row_u64, c0, c1, R, le, leaf_out);
        if (rc) break;
        rc = merkle_inner(ctx, st, h->d_nodes, L);
        if (rc) break;
        if (host_lde_out &&
            cudaMemcpyAsync(host_lde_out, h->d_lde, lde_rows * row_u64 * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess) {
            set_error("LDE download failed");
            rc = SG_ERR_CUDA;
            break;
        }
    } while (0);
    // Stream-ordered frees: the memory returns to the pool after the kernels that read it.
    if (d_trace) dev_free(ctx, st, d_trace, trace_bytes);
    if (d_w) dev_free(ctx, st, d_w, n * 8);
    if (d_state) dev_free(ctx, st, d_state, 25 * lde_rows * 8);
    if (rc != SG_OK) {
        if (h->d_lde) dev_free(ctx, st, h->d_lde, lde_rows * row_u64 * 8);
        if (h->d_nodes) dev_free(ctx, st, h->d_nodes, (2 * L - 1) * 32);
        delete h;
        return rc;
    }
    *out = h;
    return SG_OK;
}


extern "C" {

int sg_lde_commit(sg_ctx* c, void* stream, const uint64_t* trace, int trace_on_device, uint64_t n, uint64_t row_u64,
                  uint32_t blowup, const uint64_t* weights, const sg_leaf_layout* layout, uint64_t* host_lde_out,
                  sg_lde** out, uint8_t root_out[32]) {
    SG_CHECK_ARG(c && out, "null argument");
    SG_ENTER(ctx_of(c));
    *out = nullptr;
    Ctx* ctx = C(c);
    cudaStream_t st = (cudaStream_t)stream;
    sg_lde* h = nullptr;
    SG_TRY(commit_enqueue(ctx, st, trace, trace_on_device, n, row_u64, blowup, weights, 0, layout, host_lde_out, &h));
    cudaError_t e = cudaMemcpyAsync(h->root, h->d_nodes, 32, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_error(std::string("lde commit: ") + cudaGetErrorString(e));
        sg_lde_free(c, h);
        return SG_ERR_CUDA;
    }
    if (root_out) memcpy(root_out, h->root, 32);
    *out = h;
    return SG_OK;
}

int sg_lde_commit_split(sg_ctx* c, void* stream, const uint64_t* trace, int trace_on_device, uint64_t n,
                        uint64_t row_u64, uint32_t blowup, const uint64_t* weights, uint64_t split_col, int build_pre,
                        uint64_t* host_lde_out, sg_lde** out, uint8_t root_out[32], uint8_t* d_pre_nodes,
                        uint8_t root_pre_out[32]) {
    SG_CHECK_ARG(c && out, "null argument");
    SG_ENTER(ctx_of(c));
    *out = nullptr;
    SG_CHECK_ARG(split_col > 0 && split_col < row_u64, "split inside the row");
    SG_CHECK_ARG(!build_pre || d_pre_nodes, "the precomputed tree needs a node buffer");
    Ctx* ctx = C(c);
    cudaStream_t st = (cudaStream_t)stream;
    const sg_leaf_layout main_cols{2, 0, split_col, row_u64};
    sg_lde* h = nullptr;
    SG_TRY(commit_enqueue(ctx, st, trace, trace_on_device, n, row_u64, blowup, weights, 0, &main_cols, host_lde_out,
                          &h));
    int rc = SG_OK;
    const uint64_t L = h->leaves_len;
    if (build_pre) {
        rc = leaves_row_major(ctx, st, h->d_lde, h->lde_rows, row_u64, 0, split_col, 2, 0, d_pre_nodes + (L - 1) * 32);
        if (rc == SG_OK) rc = merkle_inner(ctx, st, d_pre_nodes, L);
    }
    uint8_t pre[32];
    cudaError_t e = rc == SG_OK ? cudaMemcpyAsync(h->root, h->d_nodes, 32, cudaMemcpyDeviceToHost, st) : cudaSuccess;
    if (rc == SG_OK && e == cudaSuccess && build_pre) e = cudaMemcpyAsync(pre, d_pre_nodes, 32, cudaMemcpyDeviceToHost, st);
    if (rc == SG_OK && e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (rc == SG_OK && e != cudaSuccess) {
        set_error(std::string("lde commit split: ") + cudaGetErrorString(e));
        rc = SG_ERR_CUDA;
    }
    if (rc != SG_OK) {
        sg_lde_free(c, h);
        return rc;
    }
    if (root_out) memcpy(root_out, h->root, 32);
    if (build_pre && root_pre_out) memcpy(root_pre_out, pre, 32);
    *out = h;
    return SG_OK;
}

int sg_batch_commit(sg_ctx* c, void* stream, const sg_table_desc* tables, uint32_t count, uint32_t concurrency,
                    sg_lde** out_ldes, uint8_t* roots_out) {
    SG_CHECK_ARG(c && (count == 0 || (tables && out_ldes)), "null argument");
    SG_ENTER(ctx_of(c));
    for (uint32_t i = 0; i < count; ++i) out_ldes[i] = nullptr;
    if (count == 0) return SG_OK;
    Ctx* ctx = C(c);
    cudaStream_t caller = (cudaStream_t)stream;
    // Heaviest first (crypto/stark/src/prover.rs:785): the long tables start
    // at once and the short ones fill the gaps behind them.
    std::vector<uint32_t> order(count);
    for (uint32_t i = 0; i < count; ++i) order[i] = i;
    auto weight = [&](uint32_t i) { return (double)tables[i].n * tables[i].blowup * tables[i].row_u64; };
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return weight(x) > weight(y); });
    uint32_t k = concurrency == 0 ? 1 : concurrency;
    if (k > count) k = count;
    if (k > 32) k = 32;
    // Roots are gathered on the device and read back with one copy after the join.
    uint8_t* d_roots = nullptr;
    SG_TRY(dev_alloc(ctx, caller, 32ull * count, (void**)&d_roots));
    std::vector<uint8_t> roots(32ull * count);
    std::vector<cudaStream_t> streams(k, nullptr);
    std::vector<cudaEvent_t> done(k, nullptr);
    cudaEvent_t start = nullptr;
    int rc = SG_OK;
    auto cuda_ok = [&](cudaError_t e, const char* what) {
        if (e != cudaSuccess && rc == SG_OK) {
            set_error(std::string("batch commit: ") + what + ": " + cudaGetErrorString(e));
            rc = SG_ERR_CUDA;
        }
        return e == cudaSuccess;
    };
    if (cuda_ok(cudaEventCreateWithFlags(&start, cudaEventDisableTiming), "event") &&
        cuda_ok(cudaEventRecord(start, caller), "event record")) {
        for (uint32_t s = 0; s < k && rc == SG_OK; ++s) {
            if (!cuda_ok(new_stream_like(caller, &streams[s]), "stream")) break;
            if (!cuda_ok(cudaEventCreateWithFlags(&done[s], cudaEventDisableTiming), "event")) break;
            cuda_ok(cudaStreamWaitEvent(streams[s], start, 0), "stream wait");
        }
    }
    for (uint32_t j = 0; j < count && rc == SG_OK; ++j) {
        const uint32_t i = order[j];
        const sg_table_desc& d = tables[i];
        const sg_leaf_layout* lay = d.layout.rows_per_leaf ? &d.layout : nullptr;
        rc = commit_enqueue(ctx, streams[j % k], d.trace, d.trace_on_device, d.n, d.row_u64, d.blowup, d.weights,
                            d.weights_on_device, lay, nullptr, &out_ldes[i]);
        if (rc == SG_OK)
            cuda_ok(cudaMemcpyAsync(d_roots + 32ull * i, out_ldes[i]->d_nodes, 32, cudaMemcpyDeviceToDevice,
                                    streams[j % k]),
                    "root copy");
    }
    // Join: the caller's stream waits for every driver stream; the roots are
    // host-visible once it drains.
    for (uint32_t s = 0; s < k; ++s) {
        if (streams[s] && done[s]) {
            cuda_ok(cudaEventRecord(done[s], streams[s]), "event record");
            cuda_ok(cudaStreamWaitEvent(caller, done[s], 0), "stream wait");
        }
    }
    if (rc == SG_OK) cuda_ok(cudaMemcpyAsync(roots.data(), d_roots, 32ull * count, cudaMemcpyDeviceToHost, caller),
                             "roots download");
    for (uint32_t s = 0; s < k; ++s)
        if (streams[s]) cuda_ok(cudaStreamSynchronize(streams[s]), "sync");
    cuda_ok(cudaStreamSynchronize(caller), "sync");
    dev_free(ctx, caller, d_roots, 32ull * count);
    for (uint32_t s = 0; s < k; ++s) {
        if (done[s]) cudaEventDestroy(done[s]);
        if (streams[s]) cudaStreamDestroy(streams[s]);
    }
    if (start) cudaEventDestroy(start);
    if (rc != SG_OK) {
        for (uint32_t i = 0; i < count; ++i) {
            if (out_ldes[i]) {
                dev_free(ctx, caller, out_ldes[i]->d_lde, out_ldes[i]->lde_rows * out_ldes[i]->row_u64 * 8);
                dev_free(ctx, caller, out_ldes[i]->d_nodes, (2 * out_ldes[i]->leaves_len - 1) * 32);
                delete out_ldes[i];
                out_ldes[i] = nullptr;
            }
        }
        return rc;
    }
    for (uint32_t i = 0; i < count; ++i) {
        memcpy(out_ldes[i]->root, roots.data() + 32ull * i, 32);
        if (roots_out) memcpy(roots_out + 32ull * i, out_ldes[i]->root, 32);
    }
    return SG_OK;
}

int sg_batch_commit_fused(sg_ctx* c, void* stream, const sg_table_desc* tables, uint32_t count, uint32_t concurrency,
                          sg_lde** out_ldes, uint8_t* roots_out) {
    SG_CHECK_ARG(c && (count == 0 || (tables && out_ldes)), "null argument");
    SG_ENTER(ctx_of(c));
    for (uint32_t i = 0; i < count; ++i) out_ldes[i] = nullptr;
    if (count == 0) return SG_OK;
    Ctx* ctx = C(c);
    cudaStream_t st = (cudaStream_t)stream;
    struct Held {
        uint64_t* coef = nullptr;
        uint64_t* tmp = nullptr;
        uint64_t* w = nullptr;
        uint64_t coef_b = 0, w_b = 0;
    };
    std::vector<Held> held(count);
    std::vector<LdeJob> jobs(count);
    uint8_t* d_roots = nullptr;
    int rc = SG_OK;
    for (uint32_t i = 0; i < count && rc == SG_OK; ++i) {
        const sg_table_desc& d = tables[i];
        SG_CHECK_ARG(d.trace && d.weights, "null trace or weights");
        SG_CHECK_ARG(d.trace_on_device, "the fused batch commit takes device-resident traces");
        SG_CHECK_ARG(d.n >= 2 && log2_exact(d.n) >= 0, "n must be a power of two >= 2");
        SG_CHECK_ARG(d.blowup >= 1 && log2_exact(d.blowup) >= 0, "blowup must be a power of two");
        SG_CHECK_ARG(d.row_u64 >= 1, "row width must be >= 1");
        uint32_t R;
        int le;
        uint64_t c0, c1;
        const sg_leaf_layout* lay = d.layout.rows_per_leaf ? &d.layout : nullptr;
        SG_TRY(resolve_layout(lay, d.row_u64, &R, &le, &c0, &c1));
        const uint64_t lde_rows = d.n * d.blowup;
        SG_CHECK_ARG(lde_rows % R == 0, "rows_per_leaf must divide the LDE size");
        SG_CHECK_ARG(d.row_u64 <= (~0ULL / 8) / lde_rows, "matrix size overflows 64 bits");
    }
    for (uint32_t i = 0; i < count && rc == SG_OK; ++i) {
        const sg_table_desc& d = tables[i];
        const uint64_t lde_rows = d.n * d.blowup;
        const uint32_t R = d.layout.rows_per_leaf ? d.layout.rows_per_leaf : 2;
        const uint64_t L = lde_rows / R;
        sg_lde* h = new sg_lde();
        h->lde_rows = lde_rows;
        h->row_u64 = d.row_u64;
        h->leaves_len = L;
        out_ldes[i] = h;
        rc = dev_alloc(ctx, st, lde_rows * d.row_u64 * 8, (void**)&h->d_lde);
        if (rc == SG_OK) rc = dev_alloc(ctx, st, (2 * L - 1) * 32, (void**)&h->d_nodes);
        Held& hd = held[i];
        hd.coef_b = d.n * d.row_u64 * 8;
        if (rc == SG_OK) rc = dev_alloc(ctx, st, hd.coef_b, (void**)&hd.coef);
        if (rc == SG_OK && d.n > 4096) rc = dev_alloc(ctx, st, hd.coef_b, (void**)&hd.tmp);
        const uint64_t* w = d.weights;
        if (rc == SG_OK && !d.weights_on_device) {
            hd.w_b = d.n * 8;
            rc = dev_alloc(ctx, st, hd.w_b, (void**)&hd.w);
            if (rc == SG_OK && cudaMemcpyAsync(hd.w, d.weights, hd.w_b, cudaMemcpyHostToDevice, st) != cudaSuccess) {
                set_error("fused batch commit: weights upload failed");
                rc = SG_ERR_CUDA;
            }
            w = hd.w;
        }
        jobs[i] = LdeJob{d.trace, d.row_u64, d.n, d.row_u64, d.blowup, w, h->d_lde, d.row_u64, hd.coef, hd.tmp};
    }
    if (rc == SG_OK) rc = dev_alloc(ctx, st, 32ull * count, (void**)&d_roots);
    // every table's LDE: one multi-table launch per pass group
    if (rc == SG_OK) rc = lde_multi(ctx, st, jobs.data(), count);
    // then each table's leaves and tree, heaviest first over k streams that
    // start after the LDEs (the hashing of small tables overlaps the large ones)
    uint32_t k = concurrency == 0 ? 1 : (concurrency > 32 ? 32 : concurrency);
    if (k > count) k = count;
    std::vector<cudaStream_t> streams(k, nullptr);
    std::vector<cudaEvent_t> done(k, nullptr);
    cudaEvent_t lde_done = nullptr;
    auto cuda_ok = [&](cudaError_t e, const char* what) {
        if (e != cudaSuccess && rc == SG_OK) {
            set_error(std::string("fused batch commit: ") + what + ": " + cudaGetErrorString(e));
            rc = SG_ERR_CUDA;
        }
        return rc == SG_OK;
    };
    if (rc == SG_OK && cuda_ok(cudaEventCreateWithFlags(&lde_done, cudaEventDisableTiming), "event") &&
        cuda_ok(cudaEventRecord(lde_done, st), "event record")) {
        for (uint32_t s = 0; s < k && rc == SG_OK; ++s) {
            if (!cuda_ok(new_stream_like(st, &streams[s]), "stream")) break;
            if (!cuda_ok(cudaEventCreateWithFlags(&done[s], cudaEventDisableTiming), "event")) break;
            cuda_ok(cudaStreamWaitEvent(streams[s], lde_done, 0), "stream wait");
        }
    }
    std::vector<uint32_t> order(count);
    for (uint32_t i = 0; i < count; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
        return (double)tables[x].n * tables[x].blowup * tables[x].row_u64 >
               (double)tables[y].n * tables[y].blowup * tables[y].row_u64;
    });
    for (uint32_t j = 0; j < count && rc == SG_OK; ++j) {
        const uint32_t i = order[j];
        cudaStream_t ss = streams[j % k];
        const sg_table_desc& d = tables[i];
        sg_lde* h = out_ldes[i];
        uint32_t R;
        int le;
        uint64_t c0, c1;
        const sg_leaf_layout* lay = d.layout.rows_per_leaf ? &d.layout : nullptr;
        rc = resolve_layout(lay, d.row_u64, &R, &le, &c0, &c1);
        if (rc == SG_OK)
            rc = leaves_row_major(ctx, ss, h->d_lde, h->lde_rows, d.row_u64, c0, c1, R, le,
                                  h->d_nodes + (h->leaves_len - 1) * 32);
        if (rc == SG_OK) rc = merkle_inner(ctx, ss, h->d_nodes, h->leaves_len);
        if (rc == SG_OK)
            cuda_ok(cudaMemcpyAsync(d_roots + 32ull * i, h->d_nodes, 32, cudaMemcpyDeviceToDevice, ss), "root copy");
    }
    // join: `st` waits for every hashing stream
    for (uint32_t s = 0; s < k; ++s) {
        if (streams[s] && done[s]) {
            cudaError_t e = cudaEventRecord(done[s], streams[s]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(st, done[s], 0);
            if (e != cudaSuccess) {
                cudaStreamSynchronize(streams[s]);
                cuda_ok(e, "join");
            }
        }
    }
    std::vector<uint8_t> roots(32ull * count);
    if (rc == SG_OK) {
        cudaError_t e = cudaMemcpyAsync(roots.data(), d_roots, 32ull * count, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            set_error(std::string("fused batch commit: ") + cudaGetErrorString(e));
            rc = SG_ERR_CUDA;
        }
    }
    for (uint32_t s = 0; s < k; ++s) {
        if (streams[s]) {
            if (rc != SG_OK) cudaStreamSynchronize(streams[s]);
            cudaStreamDestroy(streams[s]);
        }
        if (done[s]) cudaEventDestroy(done[s]);
    }
    if (lde_done) cudaEventDestroy(lde_done);
    for (uint32_t i = 0; i < count; ++i) {
        dev_free(ctx, st, held[i].coef, held[i].coef_b);
        dev_free(ctx, st, held[i].tmp, held[i].coef_b);
        dev_free(ctx, st, held[i].w, held[i].w_b);
    }
    dev_free(ctx, st, d_roots, 32ull * count);
    if (rc != SG_OK) {
        cudaStreamSynchronize(st);
        for (uint32_t i = 0; i < count; ++i) {
            sg_lde* h = out_ldes[i];
            if (!h) continue;
            dev_free(ctx, st, h->d_lde, h->lde_rows * h->row_u64 * 8);
            dev_free(ctx, st, h->d_nodes, (2 * h->leaves_len - 1) * 32);
            delete h;
            out_ldes[i] = nullptr;
        }
        return rc;
    }
    for (uint32_t i = 0; i < count; ++i) {
        memcpy(out_ldes[i]->root, roots.data() + 32ull * i, 32);
        if (roots_out) memcpy(roots_out + 32ull * i, out_ldes[i]->root, 32);
    }
    return SG_OK;
}

void sg_lde_free_async(sg_ctx* c, void* stream, sg_lde* h) {
    if (!c || !h) return;
    Ctx* ctx = C(c);
    enter(ctx);  // best effort: the handle is released either way
    cudaStream_t st = (cudaStream_t)stream;
    dev_free(ctx, st, h->d_lde, h->lde_rows * h->row_u64 * 8);
    dev_free(ctx, st, h->d_nodes, (2 * h->leaves_len - 1) * 32);
    delete h;
}

int sg_lde_get_info(const sg_lde* h, sg_lde_info* info) {
    SG_CHECK_ARG(h && info, "null argument");
    info->d_lde = h->d_lde;
    info->lde_rows = h->lde_rows;
    info->row_u64 = h->row_u64;
    info->d_nodes = h->d_nodes;
    info->leaves_len = h->leaves_len;
    memcpy(info->root, h->root, 32);
    return SG_OK;
}

void sg_lde_free(sg_ctx* c, sg_lde* h) {
    if (!c || !h) return;
    Ctx* ctx = C(c);
    enter(ctx);  // best effort: the handle is released either way
    // Freed on the legacy stream: ordered after all prior work that used the handle.
    cudaDeviceSynchronize();
    dev_free(ctx, nullptr, h->d_lde, h->lde_rows * h->row_u64 * 8);
    dev_free(ctx, nullptr, h->d_nodes, (2 * h->leaves_len - 1) * 32);
    delete h;
}

}  // extern "C"
