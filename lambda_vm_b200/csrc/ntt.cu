// Batched Goldilocks DFT / coset LDE over row-major matrices for sm_100a.
//
// Reference behaviour: crypto/math/src/polynomial.rs:527-608
// (coset_lde_full_expand_row_major: iDFT(n) -> x g^i/n -> zero-pad -> DFT(B n),
// natural-order output) and crypto/math-cuda/src/ntt.rs:57-66 (natural-order
// forward / inverse NTT, the inverse scaled by 1/n).
//
// Design. Every pass is one kernel, `k_dft_pass`: a CTA owns a tile of L points
// (rows) x C columns, stages it in shared memory in bit-reversed point order
// (coalesced C*8-byte row segments from HBM), runs an in-place radix-2^q DIT
// whose 2^q-point butterfly networks live in registers (q <= 5, so at most
// two shared-memory round trips for L = 1024), and writes the tile back.
// Per-point factors (coset weights, four-step twiddles, coset shifts) depend
// only on the row, so each is fetched once per tile into shared memory and
// reused by all C columns.
//
// Sizes above 4096 use the four-step split n = N1 * N2:
//   step 1: for each j2, DFT_N1 over rows i*N2 + j2, times w_n^{j2 k1}, written in place;
//   step 2: for each k1, DFT_N2 over the contiguous rows k1*N2 + j, written to rows k1 + N1*k2.
// The LDE runs iDFT (steps I1, I2; the coset weights are folded into I2's
// store), then for each coset shift j in [0, B) the forward DFT of
// c_i * w_{Bn}^{ij} (steps F1, F2). F1 writes its B outputs straight into the
// LDE buffer at the rows F2 later reads and overwrites, so F2 runs in place and
// the LDE needs no scratch beyond two n x m buffers.
#include "common.cuh"
#include "gl.cuh"

namespace sg {

struct W64 {
    uint64_t v[64];
    constexpr W64() : v() {
        uint64_t w = glc::root(6), c = 1;
        for (int i = 0; i < 64; ++i) {
            v[i] = c;
            c = glc::mul(c, w);
        }
    }
};
// omega_64^e with omega_64 derived from the reference's two-adic generator.
__constant__ W64 c_w64 = W64();

// 2^Q-point DFT on registers: bit-reversed input order, natural output order.
template <int Q, bool INVD>
__device__ __forceinline__ void dit_reg(uint64_t* v) {
    constexpr int R = 1 << Q;
#pragma unroll
    for (int h = 1; h < R; h <<= 1) {
#pragma unroll
        for (int b = 0; b < R; b += 2 * h) {
#pragma unroll
            for (int j = 0; j < h; ++j) {
                uint64_t a = v[b + j], t = v[b + j + h];
                if (j != 0) {
                    const int e = j * (64 / (2 * h));
                    t = gl::mul(t, INVD ? c_w64.v[(64 - e) & 63] : c_w64.v[e]);
                }
                v[b + j] = gl::add(a, t);
                v[b + j + h] = gl::sub(a, t);
            }
        }
    }
}

template <int Q>
__device__ __forceinline__ uint32_t brev_q(uint32_t r) {
    return __brev(r) >> (32 - Q);
}

__device__ __forceinline__ uint32_t spad(uint32_t i) { return i + (i >> 5); }

struct PassArgs {
    const uint64_t* in;
    uint64_t* out;
    uint64_t m;  // columns == row stride in u64
    uint32_t logL;
    uint32_t inverse;
    // row(tile, point, rep) = tile*ts + point*ps + rep*rs
    uint64_t in_ts, in_ps;
    uint64_t out_ts, out_ps, out_rs;
    uint32_t reps;
    const uint64_t* W;  // W[e] = omega_{2^logW}^e
    uint32_t logW;
    uint32_t pre_kind;   // 0: none, 1: omega_{2^pre_log}^{in_row * rep}
    uint32_t pre_log;
    uint32_t post_kind;  // 0: none, 1: omega_{2^post_log}^{+-(tile*k)}, 2: weights[out_row], 3: scalar
    uint32_t post_log;
    const uint64_t* weights;
    uint64_t scalar;
    uint32_t canon_out;
};

// One in-place radix-2^Q DIT stage over all C columns of the tile.
template <int Q>
__device__ __forceinline__ void dit_stage(uint64_t* S, const uint64_t* WL, uint32_t logL, int C, uint32_t cs,
                                          uint32_t logNs, bool inv) {
    constexpr uint32_t R = 1u << Q;
    const uint32_t L = 1u << logL;
    const uint32_t per_col = L >> Q;
    const uint32_t items = (uint32_t)C * per_col;
    const uint32_t Ns = 1u << logNs;
    for (uint32_t w = threadIdx.x; w < items; w += blockDim.x) {
        const uint32_t c = w >> (logL - Q);
        const uint32_t j = w & (per_col - 1);
        const uint32_t k = j & (Ns - 1);
        const uint32_t base = ((j >> logNs) << (logNs + Q)) + k;
        uint64_t* col = S + (size_t)c * cs;
        uint64_t v[R];
#pragma unroll
        for (uint32_t r = 0; r < R; ++r) v[r] = col[spad(base + r * Ns)];
        if (logNs > 0) {
            // twiddle omega_{Ns R}^{k * brev(r)} = omega_L^{k * brev(r) * L / (Ns R)}
            const uint32_t sh = logL - logNs - Q;
#pragma unroll
            for (uint32_t r = 1; r < R; ++r) v[r] = gl::mul(v[r], WL[(k * brev_q<Q>(r)) << sh]);
        }
        if (inv)
            dit_reg<Q, true>(v);
        else
            dit_reg<Q, false>(v);
#pragma unroll
        for (uint32_t r = 0; r < R; ++r) col[spad(base + r * Ns)] = v[r];
    }
}

__device__ void tile_dft(uint64_t* S, const uint64_t* WL, uint32_t logL, int C, uint32_t cs, bool inv) {
    const int nst = (int)(logL + 4) / 5;
    uint32_t rem = logL, logNs = 0;
    for (int s = 0; s < nst; ++s) {
        const uint32_t q = (rem + (nst - s) - 1) / (nst - s);
        switch (q) {
            case 1: dit_stage<1>(S, WL, logL, C, cs, logNs, inv); break;
            case 2: dit_stage<2>(S, WL, logL, C, cs, logNs, inv); break;
            case 3: dit_stage<3>(S, WL, logL, C, cs, logNs, inv); break;
            case 4: dit_stage<4>(S, WL, logL, C, cs, logNs, inv); break;
            default: dit_stage<5>(S, WL, logL, C, cs, logNs, inv); break;
        }
        rem -= q;
        logNs += q;
        __syncthreads();
    }
}

__device__ __forceinline__ uint64_t wlookup(const uint64_t* W, uint32_t logW, uint32_t logM, uint64_t e, bool inv) {
    // omega_{2^logM}^{+-e}
    const uint64_t mask = (1ULL << logW) - 1;
    uint64_t idx = (e << (logW - logM)) & mask;
    if (inv) idx = (mask + 1 - idx) & mask;
    return W[idx];
}

template <int C>
__global__ void __launch_bounds__(256) k_dft_pass(PassArgs a) {
    extern __shared__ uint64_t sm[];
    const uint32_t L = 1u << a.logL;
    const uint32_t cs = L + (L >> 5) + 1;  // padded smem column stride (u64)
    uint64_t* S = sm;
    uint64_t* WL = S + (size_t)C * cs;
    uint64_t* F = WL + L;
    const uint64_t tile = blockIdx.x;
    const uint64_t col0 = (uint64_t)blockIdx.y * C;
    const uint32_t ncols = (uint32_t)min((uint64_t)C, a.m - col0);
    const bool inv = a.inverse != 0;
    const uint32_t T = blockDim.x;

    for (uint32_t e = threadIdx.x; e < L; e += T) WL[e] = wlookup(a.W, a.logW, a.logL, e, inv);

    for (uint32_t rep = 0; rep < a.reps; ++rep) {
        if (a.pre_kind == 1) {
            const uint64_t pmask = (1ULL << a.pre_log) - 1;
            for (uint32_t i = threadIdx.x; i < L; i += T) {
                const uint64_t row = tile * a.in_ts + (uint64_t)i * a.in_ps;
                F[i] = wlookup(a.W, a.logW, a.pre_log, (row * rep) & pmask, false);
            }
        }
        __syncthreads();
        // load (coalesced along columns), bit-reverse the point index into smem
        const uint32_t tot = L * C;
        for (uint32_t e = threadIdx.x; e < tot; e += T) {
            const uint32_t i = e / C, c = e % C;
            uint64_t v = 0;
            if (c < ncols) {
                const uint64_t row = tile * a.in_ts + (uint64_t)i * a.in_ps;
                v = a.in[row * a.m + col0 + c];
                if (a.pre_kind == 1) v = gl::mul(v, F[i]);
            }
            const uint32_t p = a.logL ? (__brev(i) >> (32 - a.logL)) : 0;
            S[(size_t)c * cs + spad(p)] = v;
        }
        __syncthreads();
        tile_dft(S, WL, a.logL, C, cs, inv);
        if (a.post_kind == 1) {
            const uint64_t pmask = (1ULL << a.post_log) - 1;
            for (uint32_t k = threadIdx.x; k < L; k += T)
                F[k] = wlookup(a.W, a.logW, a.post_log, (tile * k) & pmask, inv);
        } else if (a.post_kind == 2) {
            for (uint32_t k = threadIdx.x; k < L; k += T)
                F[k] = a.weights[tile * a.out_ts + (uint64_t)k * a.out_ps + (uint64_t)rep * a.out_rs];
        }
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < tot; e += T) {
            const uint32_t k = e / C, c = e % C;
            if (c < ncols) {
                uint64_t v = S[(size_t)c * cs + spad(k)];
                if (a.post_kind == 1 || a.post_kind == 2)
                    v = gl::mul(v, F[k]);
                else if (a.post_kind == 3)
                    v = gl::mul(v, a.scalar);
                if (a.canon_out) v = gl::canon(v);
                const uint64_t row = tile * a.out_ts + (uint64_t)k * a.out_ps + (uint64_t)rep * a.out_rs;
                a.out[row * a.m + col0 + c] = v;
            }
        }
        __syncthreads();
    }
}

static int cols_for(uint32_t logL) { return logL <= 9 ? 16 : (logL <= 11 ? 8 : 4); }

template <int C>
static int launch_pass(Ctx* ctx, cudaStream_t st, const PassArgs& a, uint64_t ntiles) {
    const uint32_t L = 1u << a.logL;
    const size_t smem = ((size_t)C * (L + (L >> 5) + 1) + 2 * (size_t)L) * sizeof(uint64_t);
    static bool configured = false;
    if (!configured) {
        SG_CUDA(cudaFuncSetAttribute(k_dft_pass<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
        configured = true;
    }
    const uint64_t ctiles = (a.m + C - 1) / C;
    if (ntiles > 0x7fffffffULL || ctiles > 65535) {
        set_error("dft pass grid too large");
        return SG_ERR_UNSUPPORTED;
    }
    dim3 grid((unsigned)ntiles, (unsigned)ctiles);
    k_dft_pass<C><<<grid, 256, smem, st>>>(a);
    return check_launch(ctx, "k_dft_pass");
}

static int run_pass(Ctx* ctx, cudaStream_t st, const PassArgs& a, uint64_t ntiles) {
    if (a.logL > 12) {
        set_error("dft pass longer than 4096 points");
        return SG_ERR_UNSUPPORTED;
    }
    switch (cols_for(a.logL)) {
        case 16: return launch_pass<16>(ctx, st, a, ntiles);
        case 8: return launch_pass<8>(ctx, st, a, ntiles);
        default: return launch_pass<4>(ctx, st, a, ntiles);
    }
}

static PassArgs base_args(const uint64_t* in, uint64_t* out, uint64_t m, uint32_t logL, bool inv, const uint64_t* W,
                          uint32_t logW) {
    PassArgs a{};
    a.in = in;
    a.out = out;
    a.m = m;
    a.logL = logL;
    a.inverse = inv ? 1 : 0;
    a.reps = 1;
    a.W = W;
    a.logW = logW;
    return a;
}

int ntt_rows(Ctx* ctx, cudaStream_t st, uint64_t* d, uint64_t n, uint64_t m, int inverse, int scale_inverse) {
    if (n <= 1 || m == 0) return SG_OK;
    const int logn = log2_exact(n);
    SG_CHECK_ARG(logn > 0 && logn <= 32, "n must be a power of two <= 2^32");
    if (logn > 24) {
        set_error("NTT longer than 2^24 rows is not supported by the two-pass kernel");
        return SG_ERR_UNSUPPORTED;
    }
    const uint64_t* W = nullptr;
    SG_TRY(roots_table(ctx, st, (uint32_t)logn, &W));
    uint64_t ninv = 0;
    if (inverse && scale_inverse) {
        // 1/n = p - (p-1)/n for n | p-1
        ninv = GL_P - (GL_P - 1) / n;
    }
    if (logn <= 12) {
        PassArgs a = base_args(d, d, m, logn, inverse, W, logn);
        a.in_ps = 1;
        a.out_ps = 1;
        if (ninv) {
            a.post_kind = 3;
            a.scalar = ninv;
        }
        a.canon_out = 1;
        return run_pass(ctx, st, a, 1);
    }
    const uint32_t l1 = logn / 2, l2 = logn - l1;
    const uint64_t N1 = 1ULL << l1, N2 = 1ULL << l2;
    // step 1 in place
    PassArgs s1 = base_args(d, d, m, l1, inverse, W, logn);
    s1.in_ts = 1;
    s1.in_ps = N2;
    s1.out_ts = 1;
    s1.out_ps = N2;
    s1.post_kind = 1;
    s1.post_log = logn;
    SG_TRY(run_pass(ctx, st, s1, N2));
    uint64_t* tmp = nullptr;
    SG_TRY(dev_alloc(ctx, st, n * m * 8, (void**)&tmp));
    PassArgs s2 = base_args(d, tmp, m, l2, inverse, W, logn);
    s2.in_ts = N2;
    s2.in_ps = 1;
    s2.out_ts = 1;
    s2.out_ps = N1;
    if (ninv) {
        s2.post_kind = 3;
        s2.scalar = ninv;
    }
    s2.canon_out = 1;
    int rc = run_pass(ctx, st, s2, N1);
    if (rc == SG_OK) {
        cudaError_t e = cudaMemcpyAsync(d, tmp, n * m * 8, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) {
            set_error(std::string("ntt copy-back: ") + cudaGetErrorString(e));
            rc = SG_ERR_CUDA;
        }
    }
    int rc2 = dev_free(ctx, st, tmp, n * m * 8);
    return rc != SG_OK ? rc : rc2;
}

int coset_lde(Ctx* ctx, cudaStream_t st, const uint64_t* trace, uint64_t n, uint64_t m, uint64_t blowup,
              const uint64_t* weights, uint64_t* out) {
    if (n == 0 || m == 0) return SG_OK;
    const int logn = log2_exact(n), logB = log2_exact(blowup);
    SG_CHECK_ARG(logn >= 0, "n must be a power of two");
    SG_CHECK_ARG(logB >= 0, "blowup must be a power of two");
    const int logN = logn + logB;
    SG_CHECK_ARG(logN <= 32, "LDE size must be <= 2^32 (TWO_ADICITY)");
    if (logn > 24) {
        set_error("traces longer than 2^24 rows are not supported by the two-pass kernel");
        return SG_ERR_UNSUPPORTED;
    }
    const uint64_t* W = nullptr;
    SG_TRY(roots_table(ctx, st, (uint32_t)logN, &W));
    uint64_t* coef = nullptr;
    SG_TRY(dev_alloc(ctx, st, n * m * 8, (void**)&coef));
    int rc = SG_OK;
    if (logn <= 12) {
        PassArgs I = base_args(trace, coef, m, logn, true, W, logN);
        I.in_ps = 1;
        I.out_ps = 1;
        I.post_kind = 2;
        I.weights = weights;
        rc = run_pass(ctx, st, I, 1);
        if (rc == SG_OK) {
            PassArgs F = base_args(coef, out, m, logn, false, W, logN);
            F.in_ps = 1;
            F.reps = (uint32_t)blowup;
            F.pre_kind = 1;
            F.pre_log = logN;
            F.out_ps = blowup;
            F.out_rs = 1;
            F.canon_out = 1;
            rc = run_pass(ctx, st, F, 1);
        }
    } else {
        const uint32_t l1 = logn / 2, l2 = logn - l1;
        const uint64_t N1 = 1ULL << l1, N2 = 1ULL << l2;
        uint64_t* tmp = nullptr;
        rc = dev_alloc(ctx, st, n * m * 8, (void**)&tmp);
        if (rc == SG_OK) {
            PassArgs I1 = base_args(trace, tmp, m, l1, true, W, logN);
            I1.in_ts = 1;
            I1.in_ps = N2;
            I1.out_ts = 1;
            I1.out_ps = N2;
            I1.post_kind = 1;
            I1.post_log = logn;
            rc = run_pass(ctx, st, I1, N2);
            if (rc == SG_OK) {
                PassArgs I2 = base_args(tmp, coef, m, l2, true, W, logN);
                I2.in_ts = N2;
                I2.in_ps = 1;
                I2.out_ts = 1;
                I2.out_ps = N1;
                I2.post_kind = 2;
                I2.weights = weights;
                rc = run_pass(ctx, st, I2, N1);
            }
            int rf = dev_free(ctx, st, tmp, n * m * 8);
            if (rc == SG_OK) rc = rf;
        }
        if (rc == SG_OK) {
            PassArgs F1 = base_args(coef, out, m, l1, false, W, logN);
            F1.in_ts = 1;
            F1.in_ps = N2;
            F1.reps = (uint32_t)blowup;
            F1.pre_kind = 1;
            F1.pre_log = logN;
            F1.post_kind = 1;
            F1.post_log = logn;
            F1.out_ts = blowup * N1;
            F1.out_ps = blowup;
            F1.out_rs = 1;
            rc = run_pass(ctx, st, F1, N2);
        }
        if (rc == SG_OK) {
            PassArgs F2 = base_args(out, out, m, l2, false, W, logN);
            F2.in_ts = 1;
            F2.in_ps = blowup * N1;
            F2.out_ts = 1;
            F2.out_ps = blowup * N1;
            F2.canon_out = 1;
            rc = run_pass(ctx, st, F2, N1 * blowup);
        }
    }
    int rf = dev_free(ctx, st, coef, n * m * 8);
    return rc != SG_OK ? rc : rf;
}

// W[e] = omega^e for e in [0, N): each thread raises omega to its own exponent.
__global__ void k_roots(uint64_t* W, uint64_t N, uint64_t omega) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < N) W[e] = gl::canon(gl::pow(omega, e));
}

int roots_table(Ctx* ctx, cudaStream_t st, uint32_t log, const uint64_t** out) {
    std::lock_guard<std::mutex> g(ctx->mu);
    auto it = ctx->roots.find(log);
    if (it != ctx->roots.end()) {
        *out = it->second;
        return SG_OK;
    }
    const uint64_t N = 1ULL << log;
    uint64_t* W = nullptr;
    // Tables persist for the context lifetime: plain cudaMalloc, charged to the budget.
    if (ctx->in_use.load() + N * 8 > ctx->budget) {
        set_error("HBM budget exceeded by twiddle table");
        return SG_ERR_BUDGET;
    }
    SG_CUDA(cudaMalloc((void**)&W, N * 8));
    ctx->in_use.fetch_add(N * 8);
    const uint64_t omega = glc::root(log);
    k_roots<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(W, N, omega);
    int rc = check_launch(ctx, "k_roots");
    if (rc != SG_OK) return rc;
    // Other streams may read the table next: finish building it before publishing.
    SG_CUDA(cudaStreamSynchronize(st));
    ctx->roots[log] = W;
    *out = W;
    return SG_OK;
}

}  // namespace sg

// ---------------------------------------------------------------- allocation-free coset LDE
//
// sg_coset_lde_static computes exactly what sg_coset_lde computes, for callers
// that cannot allocate device memory at call time: a serving process that
// reserves its whole HBM allowance when it starts and treats any later
// cudaMalloc as a failure (under co-tenant memory pressure such a call can
// fail, and cudaMalloc/cudaFree can synchronize the device and stall the other
// proofs in flight), or a foreign-language host that wants one call with no
// hidden allocation and no context object to manage.
//
// Its scratch (the omega table, the coefficient matrix and the four-step
// intermediate) lives in one file-scope device array of SG_STATIC_SCRATCH_BYTES
// that every GPU which loads this library holds until the process exits. The
// array's host-side name is only a stand-in for the symbol, so the first call
// on each device, with that device current, looks up its device address with
// cudaGetSymbolAddress and caches it; make that first call before any stream
// capture. All calls share the array: two calls that overlap on the GPU (on
// different streams, or from different threads) race on it and must be
// serialized by the caller. Nothing needs clearing between calls, because each
// call writes every scratch word before it reads it.
namespace sg {

static __device__ __align__(256) uint64_t g_lde_scratch[SG_STATIC_SCRATCH_BYTES / sizeof(uint64_t)];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
uint64_t* g_static_scratch[kMaxDevices] = {};
Ctx g_static_ctx;  // launch accounting only; it never allocates

int static_scratch(uint64_t** out) {
    int dev = 0;
    SG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device index out of range for the static scratch table");
        return SG_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> g(g_static_mu);
    if (!g_static_scratch[dev]) {
        void* p = nullptr;
        SG_CUDA(cudaGetSymbolAddress(&p, g_lde_scratch));
        g_static_scratch[dev] = (uint64_t*)p;
    }
    *out = g_static_scratch[dev];
    return SG_OK;
}
}  // namespace

}  // namespace sg

extern "C" int sg_coset_lde_static(void* stream, const uint64_t* d_trace, uint64_t n, uint64_t m, uint32_t blowup,
                                   const uint64_t* d_weights, uint64_t* d_out) {
    using namespace sg;
    if (n == 0 || m == 0) return SG_OK;
    SG_CHECK_ARG(d_trace && d_weights && d_out, "null buffer");
    const int logn = log2_exact(n), logB = log2_exact(blowup);
    SG_CHECK_ARG(logn >= 0, "n must be a power of two");
    SG_CHECK_ARG(logB >= 0, "blowup must be a power of two");
    const int logN = logn + logB;
    SG_CHECK_ARG(logN <= 32 && logn <= 24, "LDE size out of range");
    const uint64_t N = 1ULL << logN;
    const uint64_t need = N + 2 * n * m;  // u64 words: omega table + coefficients + four-step intermediate
    if (need > SG_STATIC_SCRATCH_BYTES / sizeof(uint64_t)) {
        set_error("sg_coset_lde_static: needs " + std::to_string(need * 8) +
                  " bytes of scratch ((blowup*n + 2*n*m) * 8) but the static scratch holds " +
                  std::to_string((unsigned long long)SG_STATIC_SCRATCH_BYTES) + "; use sg_coset_lde");
        return SG_ERR_INVALID;
    }
    uint64_t* scratch = nullptr;
    SG_TRY(static_scratch(&scratch));
    cudaStream_t st = (cudaStream_t)stream;
    Ctx* ctx = &g_static_ctx;
    uint64_t* W = scratch;
    uint64_t* coef = scratch + N;
    uint64_t* tmp = coef + n * m;
    k_roots<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(W, N, glc::root((uint32_t)logN));
    SG_TRY(check_launch(ctx, "k_roots"));
    if (logn <= 12) {
        PassArgs I = base_args(d_trace, coef, m, logn, true, W, logN);
        I.in_ps = 1;
        I.out_ps = 1;
        I.post_kind = 2;
        I.weights = d_weights;
        SG_TRY(run_pass(ctx, st, I, 1));
        PassArgs F = base_args(coef, d_out, m, logn, false, W, logN);
        F.in_ps = 1;
        F.reps = blowup;
        F.pre_kind = 1;
        F.pre_log = logN;
        F.out_ps = blowup;
        F.out_rs = 1;
        F.canon_out = 1;
        return run_pass(ctx, st, F, 1);
    }
    const uint32_t l1 = logn / 2, l2 = logn - l1;
    const uint64_t N1 = 1ULL << l1, N2 = 1ULL << l2;
    PassArgs I1 = base_args(d_trace, tmp, m, l1, true, W, logN);
    I1.in_ts = 1;
    I1.in_ps = N2;
    I1.out_ts = 1;
    I1.out_ps = N2;
    I1.post_kind = 1;
    I1.post_log = logn;
    SG_TRY(run_pass(ctx, st, I1, N2));
    PassArgs I2 = base_args(tmp, coef, m, l2, true, W, logN);
    I2.in_ts = N2;
    I2.in_ps = 1;
    I2.out_ts = 1;
    I2.out_ps = N1;
    I2.post_kind = 2;
    I2.weights = d_weights;
    SG_TRY(run_pass(ctx, st, I2, N1));
    PassArgs F1 = base_args(coef, d_out, m, l1, false, W, logN);
    F1.in_ts = 1;
    F1.in_ps = N2;
    F1.reps = blowup;
    F1.pre_kind = 1;
    F1.pre_log = logN;
    F1.post_kind = 1;
    F1.post_log = logn;
    F1.out_ts = (uint64_t)blowup * N1;
    F1.out_ps = blowup;
    F1.out_rs = 1;
    SG_TRY(run_pass(ctx, st, F1, N2));
    PassArgs F2 = base_args(d_out, d_out, m, l2, false, W, logN);
    F2.in_ts = 1;
    F2.in_ps = (uint64_t)blowup * N1;
    F2.out_ts = 1;
    F2.out_ps = (uint64_t)blowup * N1;
    F2.canon_out = 1;
    return run_pass(ctx, st, F2, N1 * blowup);
}
