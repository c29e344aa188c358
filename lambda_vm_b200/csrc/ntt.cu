// Batched Goldilocks DFT / coset LDE over row-major matrices for sm_100a.
//
// Reference behaviour: crypto/math/src/polynomial.rs:527-608
// (coset_lde_full_expand_row_major: iDFT(n) -> x g^i/n -> zero-pad -> DFT(B n),
// natural-order output) and crypto/math-cuda/src/ntt.rs:57-66 (natural-order
// forward / inverse NTT, the inverse scaled by 1/n).
//
// Design. Every pass is one launch of `k_dft<LOGL>`, a persistent kernel whose
// CTAs walk tiles of L = 2^LOGL points (rows) x C columns. The DFT of a tile is
// an in-place radix-2^q decimation-in-time whose 2^q-point butterfly networks
// live in registers (q <= 5); the stage plan is fixed at compile time per L:
//   stage 1 gathers its 2^q1 inputs straight from HBM (bit-reversed point
//           order is just an address permutation), with coalesced C*8-byte
//           row segments, and leaves its outputs in shared memory;
//   middle stages (L > 1024 only) run in place in shared memory;
//   the last stage reads shared memory and writes its outputs straight to HBM.
// So an L = 1024 tile costs one shared-memory round trip. Per-point factors
// (coset weights, four-step twiddles, coset shifts) depend only on the row, so
// each is computed once per tile and shared by its C columns; all roots of
// unity come from two small tables (omega_N^e = lo[e mod 2^h] * hi[e >> h])
// that stay in L1, instead of an N-entry table read with a large stride.
//
// Sizes above 4096 use the four-step split n = N1 * N2:
//   step 1: for each j2, DFT_N1 over rows i*N2 + j2, times w_n^{j2 k1}, written in place;
//   step 2: for each k1, DFT_N2 over the contiguous rows k1*N2 + j, written to rows k1 + N1*k2.
// The LDE runs iDFT (steps I1, I2; the coset weights are folded into I2's
// store), then for each coset shift j in [0, B) the forward DFT of
// c_i * w_{Bn}^{ij} (steps F1, F2). F1 writes its B outputs straight into the
// LDE buffer at the rows F2 later reads and overwrites, so F2 runs in place and
// the LDE needs no scratch beyond two n x m buffers.
#include <algorithm>
#include <utility>

#include "common.cuh"
#include "gl.cuh"

namespace sg {

// f(integral_constant<int, 0>) ... f(integral_constant<int, N-1>), so loop
// indices are compile-time constants inside f.
template <typename F, int... I>
__device__ __forceinline__ void static_for_(F&& f, std::integer_sequence<int, I...>) {
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f) {
    static_for_(f, std::make_integer_sequence<int, N>{});
}

// One radix-2 butterfly (a, t) -> (a + w t, a - w t) with w = omega_64^E.
// Every 64th root of unity is +-2^S (S < 96), so w t is a shift-and-reduce
// product of 32-bit constants (gl::mul_2exp) instead of a full 64x64
// multiply, and a negative w swaps the two outputs instead of negating.
template <int E>
__device__ __forceinline__ void bfly_w64(uint64_t& x, uint64_t& y) {
    constexpr int S = glc::log2_of(glc::pow(glc::root(6), (uint64_t)E));
    static_assert(S >= 0, "64th roots of unity are powers of two");
    const uint64_t a = x, t = gl::mul_2exp<S % 96>(y);
    if constexpr (S >= 96) {
        x = gl::sub(a, t);
        y = gl::add(a, t);
    } else {
        x = gl::add(a, t);
        y = gl::sub(a, t);
    }
}

// 2^Q-point DFT on registers: bit-reversed input order, natural output order.
template <int Q, bool INVD>
__device__ __forceinline__ void dit_reg(uint64_t* v) {
    constexpr int R = 1 << Q;
    static_for<Q>([&](auto lh) {
        constexpr int h = 1 << decltype(lh)::value;
        static_for<R / (2 * h)>([&](auto bi) {
            constexpr int b = decltype(bi)::value * 2 * h;
            static_for<h>([&](auto ji) {
                constexpr int j = decltype(ji)::value;
                constexpr int e = j * (64 / (2 * h));
                bfly_w64<INVD ? (64 - e) & 63 : e>(v[b + j], v[b + j + h]);
            });
        });
    });
}

template <int Q>
__device__ __forceinline__ uint32_t brev_q(uint32_t r) {
    if constexpr (Q == 0)
        return 0;
    else
        return __brev(r) >> (32 - Q);
}

// omega_N^e = lo[e & (2^h - 1)] * hi[e >> h], N = 2^logN.
struct Tw {
    const uint64_t* lo;
    const uint64_t* hi;
    uint32_t h;
    uint32_t logN;
};

__device__ __forceinline__ uint64_t tw_pow(const Tw& t, uint64_t e) {
    return gl::mul(__ldg(t.lo + (e & ((1ULL << t.h) - 1))), __ldg(t.hi + (e >> t.h)));
}

// omega_{2^logM}^{+-x}
__device__ __forceinline__ uint64_t tw_root(const Tw& t, uint32_t logM, uint64_t x, bool inv) {
    const uint64_t mask = (1ULL << t.logN) - 1;
    uint64_t e = (x << (t.logN - logM)) & mask;
    if (inv) e = (mask + 1 - e) & mask;
    return tw_pow(t, e);
}

struct PassArgs {
    const uint64_t* in;
    uint64_t* out;
    uint64_t m;               // columns transformed
    uint64_t in_ld, out_ld;   // row strides of in / out in u64 (>= m)
    uint32_t logL;
    uint32_t inverse;
    // row(tile, point, rep) = tile*ts + point*ps + rep*rs
    uint64_t in_ts, in_ps;
    uint64_t out_ts, out_ps, out_rs;
    uint32_t reps;
    Tw tw;
    uint32_t pre_kind;   // 0: none, 1: omega_{2^pre_log}^{in_row * rep}
    uint32_t pre_log;
    uint32_t post_kind;  // 0: none, 1: omega_{2^post_log}^{+-(tile*k)}, 2: weights[out_row], 3: scalar
    uint32_t post_log;
    const uint64_t* weights;
    uint64_t scalar;
    uint32_t canon_out;
};

// Compile-time stage plan per tile: 2^LOGL points x CC columns. A tile runs
// NST register stages of at most 2^QM points each (larger radices first):
// 2^5 where a thread may hold 128 registers (tiles of 8+ columns; a 2^10
// pass is then 2^5 x 2^5, one shared-memory round trip and 31/32 general
// twiddle products a point instead of 2^4 x 2^3 x 2^3 with 7/4), 2^4 for
// the 4-column tiles, planned at four 256-thread CTAs per SM (64 registers):
// 2^5 stages at two CTAs per SM measured slower on the narrow LDEs those
// tiles serve (2^20 x 3 columns, blowup 2: 0.42 against 0.35 ms).
// The column count is a tuning choice: several are compiled per tile length
// and the context picks one per call (see pick_cols).
// Default (and untuned) columns per tile for 2^logL-point passes.
__host__ __device__ constexpr int default_cols(int logL) {
    return logL <= 7 ? 32 : (logL <= 10 ? 16 : (logL == 11 ? 8 : 4));
}
template <int LOGL, int CC>
struct Plan {
    static constexpr int QM = CC <= 4 ? 4 : 5;
    static constexpr int NST = LOGL == 0 ? 0 : (LOGL <= 5 ? 1 : ((LOGL + QM - 1) / QM < 2 ? 2 : (LOGL + QM - 1) / QM));
    static constexpr int q(int s) { return NST == 0 ? 0 : LOGL / NST + (s < LOGL % NST ? 1 : 0); }
    static constexpr int lgns(int s) { return s == 0 ? 0 : lgns(s - 1) + q(s - 1); }
    static constexpr int Q1 = q(0);
    static constexpr int C = CC;
    static constexpr int T = LOGL >= 11 ? 512 : (LOGL == 10 && C >= 16 ? 512 : 256);
    // CTAs per SM the register allocation must allow (64K registers per SM).
    // 512-thread tiles are planned at one CTA per SM (up to 128 registers a
    // thread); the 2^10-point ones hold 155 KB of shared memory, so a second
    // CTA would not fit beside them in any case.
    static constexpr int MINB = T <= 256 ? (C <= 4 && LOGL >= 10 ? 4 : 2) : 1;
    static constexpr uint32_t L = 1u << LOGL;
    static constexpr uint32_t CS0 = L + (NST > 1 ? (L >> Q1) : 0);
    static constexpr uint32_t CP = C < 16 ? C : 16;
    static constexpr uint32_t CSMOD = 16 / CP;  // column stride = CSMOD (mod 16): no bank conflicts
    static constexpr uint32_t CS = CS0 + ((CSMOD + 16 - CS0 % 16) % 16);
    static constexpr uint32_t S_WORDS = NST > 1 ? C * CS : 0;
    static constexpr uint32_t WL_WORDS = NST > 1 ? L : 0;
    static constexpr uint32_t F_WORDS = NST > 1 ? L : 2 * L;  // one buffer reused for pre and post
    static constexpr size_t SMEM = (size_t)(S_WORDS + WL_WORDS + F_WORDS) * 8;
    static_assert(NST < 2 || q(0) <= 5, "register stage wider than 32 points");
};

template <int LOGL, int C>
__device__ __forceinline__ uint32_t tpad(uint32_t p) {
    using PL = Plan<LOGL, C>;
    if constexpr (PL::NST > 1)
        return p + (p >> PL::Q1);
    else
        return p;
}

__device__ __forceinline__ uint64_t finish(const PassArgs& a, uint64_t v, uint64_t f) {
    if (a.post_kind == 1 || a.post_kind == 2)
        v = gl::mul(v, f);
    else if (a.post_kind == 3)
        v = gl::mul(v, a.scalar);
    return a.canon_out ? gl::canon(v) : v;
}

// Middle stage: in place in shared memory.
template <int LOGL, int C_, int Q, int LOGNS, bool INV>
__device__ __forceinline__ void mid_stage(uint64_t* S, const uint64_t* WL) {
    using PL = Plan<LOGL, C_>;
    constexpr uint32_t R = 1u << Q, Ns = 1u << LOGNS, per_col = PL::L >> Q;
    constexpr uint32_t items = PL::C * per_col;
    for (uint32_t w = threadIdx.x; w < items; w += PL::T) {
        const uint32_t c = w % PL::C, j = w / PL::C;
        const uint32_t k = j & (Ns - 1);
        const uint32_t base = ((j >> LOGNS) << (LOGNS + Q)) + k;
        uint64_t* col = S + c * PL::CS;
        uint64_t v[R];
#pragma unroll
        for (uint32_t r = 0; r < R; ++r) v[r] = col[tpad<LOGL, C_>(base + r * Ns)];
        constexpr uint32_t sh = LOGL - LOGNS - Q;
#pragma unroll
        for (uint32_t r = 1; r < R; ++r) v[r] = gl::mul(v[r], WL[(k * brev_q<Q>(r)) << sh]);
        dit_reg<Q, INV>(v);
#pragma unroll
        for (uint32_t r = 0; r < R; ++r) col[tpad<LOGL, C_>(base + r * Ns)] = v[r];
    }
}

// Stages 1 .. NST-2, each separated from the next by a barrier.
template <int LOGL, int C_, int STG, bool INV>
__device__ __forceinline__ void mid_stages(uint64_t* S, const uint64_t* WL) {
    using PL = Plan<LOGL, C_>;
    if constexpr (STG < PL::NST - 1) {
        if constexpr (STG > 1) __syncthreads();
        mid_stage<LOGL, C_, PL::q(STG), PL::lgns(STG), INV>(S, WL);
        mid_stages<LOGL, C_, STG + 1, INV>(S, WL);
    }
}

template <int LOGL, int C_, bool INV>
__device__ __forceinline__ void tile_body(const PassArgs& a, uint64_t* S, const uint64_t* WL, uint64_t* F,
                                          uint64_t pt, uint64_t col0, uint32_t ncols, uint32_t rep) {
    using PL = Plan<LOGL, C_>;
    constexpr uint32_t L = PL::L, C = PL::C, T = PL::T;
    uint64_t* Fpre = F;
    uint64_t* Fpost = PL::NST > 1 ? F : F + L;
    // coset-shift pre factors omega^(row * rep): rep 0 scales by omega^0 = 1
    const bool pre = a.pre_kind == 1 && rep != 0;
    // ---- pre factors
    if (pre) {
        const uint64_t pmask = (1ULL << a.pre_log) - 1;
        for (uint32_t i = threadIdx.x; i < L; i += T) {
            const uint64_t row = pt * a.in_ts + (uint64_t)i * a.in_ps;
            Fpre[i] = tw_root(a.tw, a.pre_log, (row * rep) & pmask, false);
        }
    }
    if constexpr (PL::NST <= 1) {
        if (a.post_kind == 1) {
            const uint64_t pmask = (1ULL << a.post_log) - 1;
            for (uint32_t k = threadIdx.x; k < L; k += T)
                Fpost[k] = tw_root(a.tw, a.post_log, (pt * k) & pmask, INV);
        } else if (a.post_kind == 2) {
            for (uint32_t k = threadIdx.x; k < L; k += T)
                Fpost[k] = a.weights[pt * a.out_ts + (uint64_t)k * a.out_ps + (uint64_t)rep * a.out_rs];
        }
    }
    __syncthreads();
    const uint64_t* in = a.in + (pt * a.in_ts) * a.in_ld + col0;
    uint64_t* out = a.out + (pt * a.out_ts + (uint64_t)rep * a.out_rs) * a.out_ld + col0;
    const uint64_t ip = a.in_ps * a.in_ld, op = a.out_ps * a.out_ld;
    if constexpr (PL::NST == 0) {
        for (uint32_t c = threadIdx.x; c < C; c += T) {
            if (c < ncols) {
                uint64_t v = in[c];
                if (pre) v = gl::mul(v, Fpre[0]);
                out[c] = finish(a, v, Fpost[0]);
            }
        }
        return;
    } else {
        // ---- stage 1: HBM -> registers -> (smem | HBM)
        constexpr int Q = PL::Q1;
        constexpr uint32_t R = 1u << Q, per_col = L >> Q, items = C * per_col;
        for (uint32_t w = threadIdx.x; w < items; w += T) {
            const uint32_t c = w % C, j = w / C;
            const uint32_t jb = brev_q<LOGL - Q>(j);
            uint64_t v[R];
            if (c < ncols) {
                const uint64_t* src = in + (uint64_t)jb * ip + c;
#pragma unroll
                for (uint32_t r = 0; r < R; ++r) v[r] = __ldg(src + (uint64_t)(brev_q<Q>(r) * per_col) * ip);
                if (pre) {
#pragma unroll
                    for (uint32_t r = 0; r < R; ++r) v[r] = gl::mul(v[r], Fpre[jb + brev_q<Q>(r) * per_col]);
                }
            } else {
#pragma unroll
                for (uint32_t r = 0; r < R; ++r) v[r] = 0;
            }
            dit_reg<Q, INV>(v);
            if constexpr (PL::NST == 1) {
                if (c < ncols) {
#pragma unroll
                    for (uint32_t q = 0; q < R; ++q) out[(uint64_t)q * op + c] = finish(a, v[q], Fpost[q]);
                }
            } else {
                uint64_t* col = S + c * PL::CS;
#pragma unroll
                for (uint32_t q = 0; q < R; ++q) col[tpad<LOGL, C_>(j * R + q)] = v[q];
            }
        }
    }
    if constexpr (PL::NST > 1) {
        __syncthreads();
        // post factors reuse the pre-factor buffer (stage 1 has finished reading it)
        if (a.post_kind == 1) {
            const uint64_t pmask = (1ULL << a.post_log) - 1;
            for (uint32_t k = threadIdx.x; k < L; k += T)
                Fpost[k] = tw_root(a.tw, a.post_log, (pt * k) & pmask, INV);
        } else if (a.post_kind == 2) {
            for (uint32_t k = threadIdx.x; k < L; k += T)
                Fpost[k] = a.weights[pt * a.out_ts + (uint64_t)k * a.out_ps + (uint64_t)rep * a.out_rs];
        }
        mid_stages<LOGL, C_, 1, INV>(S, WL);
        __syncthreads();
        // ---- last stage: smem -> registers -> HBM
        constexpr int Q = PL::q(PL::NST - 1);
        constexpr int LOGNS = LOGL - Q;
        constexpr uint32_t R = 1u << Q, Ns = 1u << LOGNS, items = C * Ns;
        for (uint32_t w = threadIdx.x; w < items; w += T) {
            const uint32_t c = w % C, k = w / C;
            const uint64_t* col = S + c * PL::CS;
            uint64_t v[R];
#pragma unroll
            for (uint32_t r = 0; r < R; ++r) v[r] = col[tpad<LOGL, C_>(k + r * Ns)];
#pragma unroll
            for (uint32_t r = 1; r < R; ++r) v[r] = gl::mul(v[r], WL[k * brev_q<Q>(r)]);
            dit_reg<Q, INV>(v);
            if (c < ncols) {
#pragma unroll
                for (uint32_t q = 0; q < R; ++q)
                    out[(uint64_t)(k + q * Ns) * op + c] = finish(a, v[q], Fpost[k + q * Ns]);
            }
        }
    }
}

// One instantiation per (tile length, columns, direction): each launch carries
// only the butterfly code it runs, which keeps the unrolled networks in the
// I-cache.
template <int LOGL, int C_, bool INV>
__global__ void __launch_bounds__(Plan<LOGL, C_>::T, Plan<LOGL, C_>::MINB)
    k_dft(PassArgs a, uint64_t ntiles, uint32_t ctiles) {
    using PL = Plan<LOGL, C_>;
    extern __shared__ uint64_t sm[];
    uint64_t* S = sm;
    uint64_t* WL = S + PL::S_WORDS;
    uint64_t* F = WL + PL::WL_WORDS;
    if constexpr (PL::NST > 1) {
        for (uint32_t e = threadIdx.x; e < PL::L; e += PL::T) WL[e] = tw_root(a.tw, LOGL, e, INV);
    }
    const uint64_t total = ntiles * ctiles;
    for (uint64_t t = blockIdx.x; t < total; t += gridDim.x) {
        const uint64_t pt = t / ctiles;
        const uint64_t col0 = (t % ctiles) * PL::C;
        const uint32_t ncols = (uint32_t)min((uint64_t)PL::C, a.m - col0);
        for (uint32_t rep = 0; rep < a.reps; ++rep) {
            __syncthreads();  // the previous tile is done with S and F
            tile_body<LOGL, C_, INV>(a, S, WL, F, pt, col0, ncols, rep);
        }
    }
}

// Passes of many tables that share a tile length, width and direction, in one
// persistent launch. Descriptor d owns the global tiles [first, first +
// ntiles * ctiles); a CTA finds the descriptor of each tile it takes by binary
// search and keeps its arguments in shared memory while it works on tiles of
// the same descriptor (the grid walks descriptors in order, so a CTA switches
// rarely). Small tables then share the persistent grid with large ones
// instead of running as launches of a few CTAs each.
struct PassDesc {
    PassArgs a;
    uint64_t ntiles;
    uint64_t first;
    uint32_t ctiles;
};

template <int LOGL, int C_, bool INV>
__global__ void __launch_bounds__(Plan<LOGL, C_>::T, Plan<LOGL, C_>::MINB)
    k_dft_multi(const PassDesc* __restrict__ descs, uint32_t count, uint64_t total) {
    using PL = Plan<LOGL, C_>;
    extern __shared__ uint64_t sm[];
    __shared__ PassArgs sa;
    uint64_t* S = sm;
    uint64_t* WL = S + PL::S_WORDS;
    uint64_t* F = WL + PL::WL_WORDS;
    if constexpr (PL::NST > 1) {
        // omega_{2^LOGL} is the same from every table's root table
        const Tw tw = descs[0].a.tw;
        for (uint32_t e = threadIdx.x; e < PL::L; e += PL::T) WL[e] = tw_root(tw, LOGL, e, INV);
    }
    uint32_t cur = count;  // the descriptor whose arguments are in `sa`
    for (uint64_t t = blockIdx.x; t < total; t += gridDim.x) {
        uint32_t lo = 0, hi = count;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (descs[mid].first <= t)
                lo = mid;
            else
                hi = mid;
        }
        if (lo != cur) {
            __syncthreads();  // every thread is done with the previous descriptor's arguments
            if (threadIdx.x == 0) sa = descs[lo].a;
            cur = lo;
            __syncthreads();
        }
        const uint64_t lt = t - descs[lo].first;
        const uint32_t ctiles = descs[lo].ctiles;
        const uint64_t pt = lt / ctiles;
        const uint64_t col0 = (lt % ctiles) * PL::C;
        const uint32_t ncols = (uint32_t)min((uint64_t)PL::C, sa.m - col0);
        for (uint32_t rep = 0; rep < sa.reps; ++rep) {
            __syncthreads();  // the previous tile is done with S and F
            tile_body<LOGL, C_, INV>(sa, S, WL, F, pt, col0, ncols, rep);
        }
    }
}

template <int LOGL, int C_, bool INV>
static int launch_multi_dir(Ctx* ctx, cudaStream_t st, const PassDesc* d, uint32_t count, uint64_t total) {
    using PL = Plan<LOGL, C_>;
    KernelInfo ki;
    SG_TRY(kernel_info((const void*)k_dft_multi<LOGL, C_, INV>, PL::SMEM, PL::T, &ki));
    const uint64_t cap = (uint64_t)ki.sms * ki.blocks_per_sm;
    k_dft_multi<LOGL, C_, INV><<<(unsigned)(total < cap ? total : cap), PL::T, PL::SMEM, st>>>(d, count, total);
    return check_launch(ctx, "k_dft_multi");
}

template <int LOGL, int C_>
static int launch_multi(Ctx* ctx, cudaStream_t st, bool inv, const PassDesc* d, uint32_t count, uint64_t total) {
    return inv ? launch_multi_dir<LOGL, C_, true>(ctx, st, d, count, total)
               : launch_multi_dir<LOGL, C_, false>(ctx, st, d, count, total);
}

template <int LOGL, int C_, bool INV>
static int launch_dft_dir(Ctx* ctx, cudaStream_t st, const PassArgs& a, uint64_t ntiles) {
    using PL = Plan<LOGL, C_>;
    KernelInfo ki;
    SG_TRY(kernel_info((const void*)k_dft<LOGL, C_, INV>, PL::SMEM, PL::T, &ki));
    const int blocks_per_sm = ki.blocks_per_sm, num_sms = ki.sms;
    const uint64_t ctiles = (a.m + PL::C - 1) / PL::C;
    if (ctiles > 0xffffffffULL) {
        set_error("too many columns");
        return SG_ERR_UNSUPPORTED;
    }
    const uint64_t total = ntiles * ctiles;
    const uint64_t grid = total < (uint64_t)num_sms * blocks_per_sm ? total : (uint64_t)num_sms * blocks_per_sm;
    k_dft<LOGL, C_, INV><<<(unsigned)grid, PL::T, PL::SMEM, st>>>(a, ntiles, (uint32_t)ctiles);
    return check_launch(ctx, "k_dft");
}

template <int LOGL, int C_>
static int launch_dft(Ctx* ctx, cudaStream_t st, const PassArgs& a, uint64_t ntiles) {
    return a.inverse ? launch_dft_dir<LOGL, C_, true>(ctx, st, a, ntiles)
                     : launch_dft_dir<LOGL, C_, false>(ctx, st, a, ntiles);
}

// Tile-width variants compiled per tile length (columns per tile).
static int tile_variants(uint32_t logL, int* out) {
    if (logL >= 8 && logL <= 10) {
        out[0] = 4, out[1] = 8, out[2] = 16;
        return 3;
    }
    if (logL == 11) {
        out[0] = 4, out[1] = 8;
        return 2;
    }
    out[0] = default_cols((int)logL);
    return 1;
}

static int launch_cols(Ctx* ctx, cudaStream_t st, const PassArgs& a, uint64_t ntiles, int cols) {
    switch (a.logL) {
        case 0: return launch_dft<0, default_cols(0)>(ctx, st, a, ntiles);
        case 1: return launch_dft<1, default_cols(1)>(ctx, st, a, ntiles);
        case 2: return launch_dft<2, default_cols(2)>(ctx, st, a, ntiles);
        case 3: return launch_dft<3, default_cols(3)>(ctx, st, a, ntiles);
        case 4: return launch_dft<4, default_cols(4)>(ctx, st, a, ntiles);
        case 5: return launch_dft<5, default_cols(5)>(ctx, st, a, ntiles);
        case 6: return launch_dft<6, default_cols(6)>(ctx, st, a, ntiles);
        case 7: return launch_dft<7, default_cols(7)>(ctx, st, a, ntiles);
        case 8:
            return cols == 4 ? launch_dft<8, 4>(ctx, st, a, ntiles)
                             : (cols == 8 ? launch_dft<8, 8>(ctx, st, a, ntiles) : launch_dft<8, 16>(ctx, st, a, ntiles));
        case 9:
            return cols == 4 ? launch_dft<9, 4>(ctx, st, a, ntiles)
                             : (cols == 8 ? launch_dft<9, 8>(ctx, st, a, ntiles) : launch_dft<9, 16>(ctx, st, a, ntiles));
        case 10:
            return cols == 4 ? launch_dft<10, 4>(ctx, st, a, ntiles)
                             : (cols == 8 ? launch_dft<10, 8>(ctx, st, a, ntiles)
                                          : launch_dft<10, 16>(ctx, st, a, ntiles));
        case 11: return cols == 4 ? launch_dft<11, 4>(ctx, st, a, ntiles) : launch_dft<11, 8>(ctx, st, a, ntiles);
        case 12: return launch_dft<12, default_cols(12)>(ctx, st, a, ntiles);
        default: set_error("dft pass longer than 4096 points"); return SG_ERR_UNSUPPORTED;
    }
}

static int launch_multi_cols(Ctx* ctx, cudaStream_t st, uint32_t logL, int cols, bool inv, const PassDesc* d,
                             uint32_t count, uint64_t total) {
    switch (logL) {
        case 0: return launch_multi<0, default_cols(0)>(ctx, st, inv, d, count, total);
        case 1: return launch_multi<1, default_cols(1)>(ctx, st, inv, d, count, total);
        case 2: return launch_multi<2, default_cols(2)>(ctx, st, inv, d, count, total);
        case 3: return launch_multi<3, default_cols(3)>(ctx, st, inv, d, count, total);
        case 4: return launch_multi<4, default_cols(4)>(ctx, st, inv, d, count, total);
        case 5: return launch_multi<5, default_cols(5)>(ctx, st, inv, d, count, total);
        case 6: return launch_multi<6, default_cols(6)>(ctx, st, inv, d, count, total);
        case 7: return launch_multi<7, default_cols(7)>(ctx, st, inv, d, count, total);
        case 8:
            return cols == 4 ? launch_multi<8, 4>(ctx, st, inv, d, count, total)
                             : (cols == 8 ? launch_multi<8, 8>(ctx, st, inv, d, count, total)
                                          : launch_multi<8, 16>(ctx, st, inv, d, count, total));
        case 9:
            return cols == 4 ? launch_multi<9, 4>(ctx, st, inv, d, count, total)
                             : (cols == 8 ? launch_multi<9, 8>(ctx, st, inv, d, count, total)
                                          : launch_multi<9, 16>(ctx, st, inv, d, count, total));
        case 10:
            return cols == 4 ? launch_multi<10, 4>(ctx, st, inv, d, count, total)
                             : (cols == 8 ? launch_multi<10, 8>(ctx, st, inv, d, count, total)
                                          : launch_multi<10, 16>(ctx, st, inv, d, count, total));
        case 11:
            return cols == 4 ? launch_multi<11, 4>(ctx, st, inv, d, count, total)
                             : launch_multi<11, 8>(ctx, st, inv, d, count, total);
        case 12: return launch_multi<12, default_cols(12)>(ctx, st, inv, d, count, total);
        default: set_error("dft pass longer than 4096 points"); return SG_ERR_UNSUPPORTED;
    }
}

static int ctx_tw(Ctx* ctx, cudaStream_t st, uint32_t logN, Tw* tw);
static PassArgs base_args(const uint64_t* in, uint64_t* out, uint64_t m, uint32_t logL, bool inv, const Tw& tw);

// Tile-width autotuner. The first pass of each tile length on a context times
// every compiled width on the same work (2^logL points x 16 columns x 296
// tiles, one forward pass, in place on a scratch buffer) and keeps each
// width's time per column; a pass over m columns then uses the width that
// minimises ceil(m / C) * C * cost(C), so narrow matrices (LogUp aux, the
// composition parts) get narrow tiles and wide ones keep the 128-byte rows.
// Widths only change how columns are grouped into tiles, never a value.
static int tune_tiles(Ctx* ctx, cudaStream_t st, uint32_t logL) {
    int vs[4];
    const int nv = tile_variants(logL, vs);
    Ctx::TileTune& tt = ctx->tiles[logL];
    if (nv == 1) {
        tt.n = 1, tt.cols[0] = vs[0], tt.cost[0] = 1.0f;
        return SG_OK;
    }
    // Two 16-column tiles per SM. These stay in L2; a larger, HBM-resident
    // buffer of contiguous tiles was measured to rank the widths unlike the
    // strided four-step passes do (8 and 16 columns tied at 2^10, where real
    // 2^20-row passes run 7 % faster at 16).
    const uint64_t L = 1ULL << logL, m = 16, tiles = 296;
    uint64_t* scratch = nullptr;
    SG_TRY(dev_alloc(ctx, st, L * m * tiles * 8, (void**)&scratch));
    int rc = SG_OK;
    Tw tw;
    rc = ctx_tw(ctx, st, logL, &tw);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (rc == SG_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) {
        set_error("tile tuning: event creation failed");
        rc = SG_ERR_CUDA;
    }
    if (rc == SG_OK && cudaMemsetAsync(scratch, 0, L * m * tiles * 8, st) != cudaSuccess) {
        set_error("tile tuning: memset failed");
        rc = SG_ERR_CUDA;
    }
    // Three rounds over the widths in turn, each width's cost the fastest of
    // its rounds: a clock ramp or a noisy neighbour then cannot pick a width.
    PassArgs a = base_args(scratch, scratch, m, logL, false, tw);
    a.in_ts = L, a.in_ps = 1, a.out_ts = L, a.out_ps = 1;
    for (int v = 0; v < nv && rc == SG_OK; ++v) {
        tt.cols[v] = vs[v];
        tt.cost[v] = 1e30f;
        rc = launch_cols(ctx, st, a, tiles, vs[v]);  // warm-up (first launch sets up the kernel)
    }
    for (int round = 0; round < 3 && rc == SG_OK; ++round) {
        for (int v = 0; v < nv && rc == SG_OK; ++v) {
            cudaEventRecord(e0, st);
            for (int r = 0; r < 8 && rc == SG_OK; ++r) rc = launch_cols(ctx, st, a, tiles, vs[v]);
            if (rc != SG_OK) break;
            cudaEventRecord(e1, st);
            float ms = 0;
            if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                set_error("tile tuning: timing failed");
                rc = SG_ERR_CUDA;
                break;
            }
            const float c = ms / (8.0f * (float)m);
            if (c < tt.cost[v]) tt.cost[v] = c;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    int rf = dev_free(ctx, st, scratch, L * m * tiles * 8);
    if (rc == SG_OK) tt.n = nv;
    return rc != SG_OK ? rc : rf;
}

static int pick_cols(Ctx* ctx, cudaStream_t st, const PassArgs& a, uint64_t ntiles, int* cols) {
    const uint32_t logL = a.logL;
    const uint64_t m = a.m;
    int vs[4];
    const int nv = tile_variants(logL, vs);
    *cols = default_cols((int)logL);
    if (nv == 1 || !ctx->autotune) return SG_OK;
    {
        std::lock_guard<std::mutex> g(ctx->tune_mu);
        const int forced = ctx->tiles[logL].forced;
        if (forced) {
            *cols = forced;
            return SG_OK;
        }
        // With a learned pass-cost model installed, each compiled width's pass
        // time is predicted from the pass's shape and the fastest is taken; no
        // timing probe runs.
        if (!ctx->pass_model.empty()) {
            float best = 0;
            for (int v = 0; v < nv; ++v) {
                float x[SG_MLP_IN];
                sg_pass_features(logL, ntiles, m, (uint32_t)vs[v], a.reps, a.inverse, a.pre_kind ? 1 : 0,
                                 a.post_kind, a.canon_out, x);
                const float t = mlp_predict_host(ctx->pass_model.data(), x);
                if (v == 0 || t < best) best = t, *cols = vs[v];
            }
            return SG_OK;
        }
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return SG_OK;
    std::lock_guard<std::mutex> g(ctx->tune_mu);
    Ctx::TileTune& tt = ctx->tiles[logL];
    if (tt.n == 0) SG_TRY(tune_tiles(ctx, st, logL));
    // Padded work times cost per column; the default width keeps the pass
    // unless another is at least 3 % cheaper (the timing pass is a proxy:
    // closer calls than that follow the measured default).
    const int def = *cols;
    double best = 0, at_def = -1;
    for (int v = 0; v < tt.n; ++v) {
        const double c = (double)((m + tt.cols[v] - 1) / tt.cols[v] * tt.cols[v]) * tt.cost[v];
        if (tt.cols[v] == def) at_def = c;
        if (v == 0 || c < best) best = c, *cols = tt.cols[v];
    }
    if (at_def >= 0 && best > 0.97 * at_def) *cols = def;
    return SG_OK;
}

static int run_pass(Ctx* ctx, cudaStream_t st, const PassArgs& a, uint64_t ntiles) {
    int cols = 0;
    SG_TRY(pick_cols(ctx, st, a, ntiles, &cols));
    if (!ctx->passlog_on.load(std::memory_order_relaxed)) return launch_cols(ctx, st, a, ntiles, cols);
    // pass log: the launch between two events, read back by sg_ctx_pass_log_read
    Ctx::PassLog r{};
    r.rec.log_len = a.logL, r.rec.cols = (uint32_t)cols, r.rec.inverse = a.inverse, r.rec.reps = a.reps;
    r.rec.pre = a.pre_kind ? 1 : 0, r.rec.post = a.post_kind, r.rec.canon = a.canon_out;
    r.rec.tiles = ntiles, r.rec.m = a.m;
    SG_CUDA(cudaEventCreate(&r.e0));
    cudaError_t e = cudaEventCreate(&r.e1);
    if (e == cudaSuccess) e = cudaEventRecord(r.e0, st);
    int rc = e == cudaSuccess ? launch_cols(ctx, st, a, ntiles, cols) : SG_ERR_CUDA;
    if (rc == SG_OK) e = cudaEventRecord(r.e1, st);
    if (e != cudaSuccess || rc != SG_OK) {
        if (e != cudaSuccess) set_error(std::string("pass log: ") + cudaGetErrorString(e));
        cudaEventDestroy(r.e0);
        if (r.e1) cudaEventDestroy(r.e1);
        return rc != SG_OK ? rc : SG_ERR_CUDA;
    }
    std::lock_guard<std::mutex> g(ctx->passlog_mu);
    ctx->passlog.push_back(r);
    return SG_OK;
}

static PassArgs base_args(const uint64_t* in, uint64_t* out, uint64_t m, uint32_t logL, bool inv, const Tw& tw) {
    PassArgs a{};
    a.in = in;
    a.out = out;
    a.m = m;
    a.in_ld = m;
    a.out_ld = m;
    a.logL = logL;
    a.inverse = inv ? 1 : 0;
    a.reps = 1;
    a.tw = tw;
    return a;
}

// Two-level root tables for N = 2^logN: lo = omega^[0, 2^h), hi = omega^(2^h * [0, 2^(logN-h))).
static inline uint32_t tw_h(uint32_t logN) { return (logN + 1) / 2; }
static inline uint64_t tw_words(uint32_t logN) { return (1ULL << tw_h(logN)) + (1ULL << (logN - tw_h(logN))); }

__global__ void k_tw_tables(uint64_t* lo, uint64_t nlo, uint64_t* hi, uint64_t nhi, uint64_t omega, uint32_t h) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nlo) lo[e] = gl::canon(gl::pow(omega, e));
    if (e < nhi) hi[e] = gl::canon(gl::pow(omega, e << h));
}

static int build_tw(Ctx* ctx, cudaStream_t st, uint32_t logN, uint64_t* mem, Tw* out) {
    const uint32_t h = tw_h(logN);
    const uint64_t nlo = 1ULL << h, nhi = 1ULL << (logN - h);
    const uint64_t mx = nlo > nhi ? nlo : nhi;
    k_tw_tables<<<(unsigned)((mx + 255) / 256), 256, 0, st>>>(mem, nlo, mem + nlo, nhi, glc::root(logN), h);
    SG_TRY(check_launch(ctx, "k_tw_tables"));
    out->lo = mem;
    out->hi = mem + nlo;
    out->h = h;
    out->logN = logN;
    return SG_OK;
}

int roots_table(Ctx* ctx, cudaStream_t st, uint32_t log, const uint64_t** out) {
    std::lock_guard<std::mutex> g(ctx->mu);
    auto it = ctx->roots.find(log);
    if (it != ctx->roots.end()) {
        *out = it->second;
        return SG_OK;
    }
    const uint64_t words = tw_words(log);
    uint64_t* mem = nullptr;
    // Tables persist for the context lifetime: plain cudaMalloc, charged to the budget.
    if (ctx->in_use.load() + words * 8 > ctx->budget) {
        set_error("HBM budget exceeded by twiddle table");
        return SG_ERR_BUDGET;
    }
    SG_CUDA(cudaMalloc((void**)&mem, words * 8));
    ctx->in_use.fetch_add(words * 8);
    Tw tw;
    int rc = build_tw(ctx, st, log, mem, &tw);
    if (rc != SG_OK) return rc;
    // Other streams may read the table next: finish building it before publishing.
    SG_CUDA(cudaStreamSynchronize(st));
    ctx->roots[log] = mem;
    *out = mem;
    return SG_OK;
}

static int ctx_tw(Ctx* ctx, cudaStream_t st, uint32_t logN, Tw* tw) {
    const uint64_t* mem = nullptr;
    SG_TRY(roots_table(ctx, st, logN, &mem));
    tw->h = tw_h(logN);
    tw->logN = logN;
    tw->lo = mem;
    tw->hi = mem + (1ULL << tw->h);
    return SG_OK;
}

int ntt_rows(Ctx* ctx, cudaStream_t st, uint64_t* d, uint64_t n, uint64_t m, int inverse, int scale_inverse) {
    if (n <= 1 || m == 0) return SG_OK;
    const int logn = log2_exact(n);
    SG_CHECK_ARG(logn > 0 && logn <= 32, "n must be a power of two <= 2^32");
    if (logn > 24) {
        set_error("NTT longer than 2^24 rows is not supported by the two-pass kernel");
        return SG_ERR_UNSUPPORTED;
    }
    Tw tw;
    SG_TRY(ctx_tw(ctx, st, (uint32_t)logn, &tw));
    uint64_t ninv = 0;
    if (inverse && scale_inverse) {
        // 1/n = p - (p-1)/n for n | p-1
        ninv = GL_P - (GL_P - 1) / n;
    }
    if (logn <= 12) {
        PassArgs a = base_args(d, d, m, logn, inverse, tw);
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
    PassArgs s1 = base_args(d, d, m, l1, inverse, tw);
    s1.in_ts = 1;
    s1.in_ps = N2;
    s1.out_ts = 1;
    s1.out_ps = N2;
    s1.post_kind = 1;
    s1.post_log = logn;
    SG_TRY(run_pass(ctx, st, s1, N2));
    uint64_t* tmp = nullptr;
    SG_TRY(dev_alloc(ctx, st, n * m * 8, (void**)&tmp));
    PassArgs s2 = base_args(d, tmp, m, l2, inverse, tw);
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

// The LDE pass sequence over caller-provided scratch: coef (n x m) always,
// tmp (n x m) when n > 4096. Each pass goes to `emit(step, args, ntiles)`,
// which runs it now (one table) or plans it for the multi-table launcher.
// Steps 0..3 are I1, I2, F1, F2 (a single-pass LDE uses steps 1 and 3);
// passes of one step of different tables never depend on each other.
template <typename Emit>
static int lde_passes_to(Emit&& emit, const uint64_t* trace, uint64_t trace_ld, uint64_t n, uint64_t m,
                         uint64_t blowup, const uint64_t* weights, uint64_t* out, uint64_t out_ld, const Tw& tw,
                         uint64_t* coef, uint64_t* tmp) {
    const int logn = log2_exact(n), logN = (int)tw.logN;
    if (logn <= 12) {
        PassArgs I = base_args(trace, coef, m, logn, true, tw);
        I.in_ld = trace_ld;
        I.in_ps = 1;
        I.out_ps = 1;
        I.post_kind = 2;
        I.weights = weights;
        SG_TRY(emit(1, I, 1));
        PassArgs F = base_args(coef, out, m, logn, false, tw);
        F.out_ld = out_ld;
        F.in_ps = 1;
        F.reps = (uint32_t)blowup;
        F.pre_kind = 1;
        F.pre_log = logN;
        F.out_ps = blowup;
        F.out_rs = 1;
        F.canon_out = 1;
        return emit(3, F, 1);
    }
    const uint32_t l1 = logn / 2, l2 = logn - l1;
    const uint64_t N1 = 1ULL << l1, N2 = 1ULL << l2;
    PassArgs I1 = base_args(trace, tmp, m, l1, true, tw);
    I1.in_ld = trace_ld;
    I1.in_ts = 1;
    I1.in_ps = N2;
    I1.out_ts = 1;
    I1.out_ps = N2;
    I1.post_kind = 1;
    I1.post_log = logn;
    SG_TRY(emit(0, I1, N2));
    PassArgs I2 = base_args(tmp, coef, m, l2, true, tw);
    I2.in_ts = N2;
    I2.in_ps = 1;
    I2.out_ts = 1;
    I2.out_ps = N1;
    I2.post_kind = 2;
    I2.weights = weights;
    SG_TRY(emit(1, I2, N1));
    PassArgs F1 = base_args(coef, out, m, l1, false, tw);
    F1.out_ld = out_ld;
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
    SG_TRY(emit(2, F1, N2));
    PassArgs F2 = base_args(out, out, m, l2, false, tw);
    F2.in_ld = out_ld;
    F2.out_ld = out_ld;
    F2.in_ts = 1;
    F2.in_ps = blowup * N1;
    F2.out_ts = 1;
    F2.out_ps = blowup * N1;
    F2.canon_out = 1;
    return emit(3, F2, N1 * blowup);
}

static int lde_passes(Ctx* ctx, cudaStream_t st, const uint64_t* trace, uint64_t trace_ld, uint64_t n, uint64_t m,
                      uint64_t blowup, const uint64_t* weights, uint64_t* out, uint64_t out_ld, const Tw& tw,
                      uint64_t* coef, uint64_t* tmp) {
    auto now = [&](int, const PassArgs& a, uint64_t ntiles) { return run_pass(ctx, st, a, ntiles); };
    return lde_passes_to(now, trace, trace_ld, n, m, blowup, weights, out, out_ld, tw, coef, tmp);
}

int coset_lde(Ctx* ctx, cudaStream_t st, const uint64_t* trace, uint64_t n, uint64_t m, uint64_t blowup,
              const uint64_t* weights, uint64_t* out) {
    return coset_lde_ld(ctx, st, trace, m, n, m, blowup, weights, out, m);
}

int coset_lde_ld(Ctx* ctx, cudaStream_t st, const uint64_t* trace, uint64_t trace_ld, uint64_t n, uint64_t m,
                 uint64_t blowup, const uint64_t* weights, uint64_t* out, uint64_t out_ld) {
    if (n == 0 || m == 0) return SG_OK;
    SG_CHECK_ARG(trace_ld >= m && out_ld >= m, "row stride smaller than the column count");
    const int logn = log2_exact(n), logB = log2_exact(blowup);
    SG_CHECK_ARG(logn >= 0, "n must be a power of two");
    SG_CHECK_ARG(logB >= 0, "blowup must be a power of two");
    const int logN = logn + logB;
    SG_CHECK_ARG(logN <= 32, "LDE size must be <= 2^32 (TWO_ADICITY)");
    SG_CHECK_ARG(trace_ld <= (~0ULL / 8) >> logn && out_ld <= (~0ULL / 8) >> logN, "matrix size overflows 64 bits");
    if (logn > 24) {
        set_error("traces longer than 2^24 rows are not supported by the two-pass kernel");
        return SG_ERR_UNSUPPORTED;
    }
    Tw tw;
    SG_TRY(ctx_tw(ctx, st, (uint32_t)logN, &tw));
    uint64_t* coef = nullptr;
    uint64_t* tmp = nullptr;
    SG_TRY(dev_alloc(ctx, st, n * m * 8, (void**)&coef));
    int rc = SG_OK;
    if (logn > 12) rc = dev_alloc(ctx, st, n * m * 8, (void**)&tmp);
    if (rc == SG_OK) rc = lde_passes(ctx, st, trace, trace_ld, n, m, blowup, weights, out, out_ld, tw, coef, tmp);
    int rf = dev_free(ctx, st, tmp, n * m * 8);
    int rf2 = dev_free(ctx, st, coef, n * m * 8);
    if (rc != SG_OK) return rc;
    return rf != SG_OK ? rf : rf2;
}

// The LDEs of many tables, the passes of each step grouped by (tile length,
// width, direction) into one multi-table launch each: 4 steps x a few
// groups of launches for any number of tables. Every job brings its own
// scratch (coef always, tmp when n > 4096) and its output buffer.
int lde_multi(Ctx* ctx, cudaStream_t st, const LdeJob* jobs, uint32_t count) {
    struct Planned {
        int step, cols;
        PassArgs a;
        uint64_t ntiles;
    };
    std::vector<Planned> plan;
    for (uint32_t i = 0; i < count; ++i) {
        const LdeJob& j = jobs[i];
        if (j.n == 0 || j.m == 0) continue;
        const int logn = log2_exact(j.n), logB = log2_exact(j.blowup);
        SG_CHECK_ARG(logn >= 0 && logB >= 0 && logn <= 24 && logn + logB <= 32, "LDE size out of range");
        SG_CHECK_ARG(j.n <= 4096 || j.tmp, "a four-step LDE needs its tmp scratch");
        Tw tw;
        SG_TRY(ctx_tw(ctx, st, (uint32_t)(logn + logB), &tw));
        auto record = [&](int step, const PassArgs& a, uint64_t ntiles) {
            int cols = 0;
            SG_TRY(pick_cols(ctx, st, a, ntiles, &cols));
            plan.push_back({step, cols, a, ntiles});
            return SG_OK;
        };
        SG_TRY(lde_passes_to(record, j.trace, j.trace_ld, j.n, j.m, j.blowup, j.weights, j.out, j.out_ld, tw, j.coef,
                             j.tmp));
    }
    if (plan.empty()) return SG_OK;
    std::stable_sort(plan.begin(), plan.end(), [](const Planned& x, const Planned& y) {
        if (x.step != y.step) return x.step < y.step;
        if (x.a.logL != y.a.logL) return x.a.logL < y.a.logL;
        if (x.cols != y.cols) return x.cols < y.cols;
        return x.a.inverse < y.a.inverse;
    });
    // one descriptor array for every group, uploaded once before any launch
    std::vector<PassDesc> descs(plan.size());
    struct Group {
        size_t begin, end;
        uint64_t total;
    };
    std::vector<Group> groups;
    for (size_t i = 0; i < plan.size(); ++i) {
        const Planned& p = plan[i];
        if (groups.empty() || p.step != plan[groups.back().begin].step || p.a.logL != plan[groups.back().begin].a.logL ||
            p.cols != plan[groups.back().begin].cols || p.a.inverse != plan[groups.back().begin].a.inverse)
            groups.push_back({i, i, 0});
        Group& g = groups.back();
        const uint64_t ctiles = (p.a.m + (uint64_t)p.cols - 1) / (uint64_t)p.cols;
        SG_CHECK_ARG(ctiles <= 0xffffffffULL, "too many columns");
        descs[i] = PassDesc{p.a, p.ntiles, g.total, (uint32_t)ctiles};
        g.total += p.ntiles * ctiles;
        g.end = i + 1;
    }
    PassDesc* d_descs = nullptr;
    const uint64_t bytes = descs.size() * sizeof(PassDesc);
    SG_TRY(dev_alloc(ctx, st, bytes, (void**)&d_descs));
    int rc = SG_OK;
    if (cudaMemcpyAsync(d_descs, descs.data(), bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        set_error("multi-table DFT: descriptor upload failed");
        rc = SG_ERR_CUDA;
    }
    for (const Group& g : groups) {
        if (rc != SG_OK) break;
        const Planned& p = plan[g.begin];
        rc = launch_multi_cols(ctx, st, p.a.logL, p.cols, p.a.inverse != 0, d_descs + g.begin,
                               (uint32_t)(g.end - g.begin), g.total);
    }
    const int rf = dev_free(ctx, st, d_descs, bytes);
    return rc != SG_OK ? rc : rf;
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
Ctx g_static_ctx;  // launch accounting only; it never allocates (so it never tunes tiles)
const bool g_static_ctx_fixed = (g_static_ctx.autotune = false, true);

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
    // u64 words needed: the two-level root tables (tw_words(logN) <= max(N, 3))
    // + coefficients + four-step intermediate (n x m each). Bounded by
    // division, so no m wraps tw_region + 2*n*m into range.
    const uint64_t tw_region = N > 3 ? N : 3;
    const uint64_t cap = SG_STATIC_SCRATCH_BYTES / sizeof(uint64_t);
    if (tw_region > cap || m > (cap - tw_region) / (2 * n)) {
        set_error("sg_coset_lde_static: n=" + std::to_string(n) + " m=" + std::to_string(m) +
                  " blowup=" + std::to_string(blowup) +
                  " needs (max(blowup*n, 3) + 2*n*m) * 8 bytes of scratch, more than the static scratch holds (" +
                  std::to_string((unsigned long long)SG_STATIC_SCRATCH_BYTES) + " bytes); use sg_coset_lde");
        return SG_ERR_INVALID;
    }
    uint64_t* scratch = nullptr;
    SG_TRY(static_scratch(&scratch));
    cudaStream_t st = (cudaStream_t)stream;
    Ctx* ctx = &g_static_ctx;
    // Scratch layout: [root tables | coefficients (n x m) | four-step intermediate (n x m)].
    Tw tw;
    SG_TRY(build_tw(ctx, st, (uint32_t)logN, scratch, &tw));
    uint64_t* coef = scratch + tw_region;
    uint64_t* tmp = coef + n * m;
    return lde_passes(ctx, st, d_trace, m, n, m, blowup, d_weights, d_out, m, tw, coef, tmp);
}

extern "C" int sg_ctx_pass_log(sg_ctx* c, int enable) {
    using namespace sg;
    SG_CHECK_ARG(c, "null context");
    reinterpret_cast<Ctx*>(c)->passlog_on.store(enable != 0);
    return SG_OK;
}

extern "C" int sg_ctx_pass_log_read(sg_ctx* c, sg_pass_record* out, uint32_t capacity, uint32_t* count) {
    using namespace sg;
    SG_CHECK_ARG(c && count && (out || capacity == 0), "null argument");
    SG_ENTER(ctx_of(c));
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    std::vector<Ctx::PassLog> log;
    {
        std::lock_guard<std::mutex> g(ctx->passlog_mu);
        log.swap(ctx->passlog);
    }
    int rc = SG_OK;
    uint32_t k = 0;
    for (auto& r : log) {
        float ms = 0;
        if (rc == SG_OK) {
            cudaError_t e = cudaEventSynchronize(r.e1);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, r.e0, r.e1);
            if (e != cudaSuccess) {
                set_error(std::string("pass log: ") + cudaGetErrorString(e));
                rc = SG_ERR_CUDA;
            }
        }
        if (rc == SG_OK && k < capacity) {
            out[k] = r.rec;
            out[k].ms = ms;
            ++k;
        }
        cudaEventDestroy(r.e0);
        cudaEventDestroy(r.e1);
    }
    *count = k;
    return rc;
}

extern "C" int sg_ctx_dft_tiles(sg_ctx* c, uint32_t log_len, uint32_t cols) {
    using namespace sg;
    SG_CHECK_ARG(c && log_len <= 12, "null context or tile length above 2^12");
    SG_ENTER(ctx_of(c));
    int vs[4];
    const int nv = tile_variants(log_len, vs);
    bool ok = cols == 0;
    for (int v = 0; v < nv; ++v) ok = ok || (int)cols == vs[v];
    SG_CHECK_ARG(ok, "no compiled tile of that width for this length");
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    std::lock_guard<std::mutex> g(ctx->tune_mu);
    ctx->tiles[log_len].forced = (int)cols;
    return SG_OK;
}

extern "C" int sg_ctx_dft_tuning(sg_ctx* c, void* stream, uint32_t log_len, uint32_t* cols, float* cost_per_col,
                                 uint32_t* count) {
    using namespace sg;
    SG_CHECK_ARG(c && cols && cost_per_col && count && log_len <= 12, "null argument or tile length above 2^12");
    SG_ENTER(ctx_of(c));
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    std::lock_guard<std::mutex> g(ctx->tune_mu);
    Ctx::TileTune& tt = ctx->tiles[log_len];
    if (tt.n == 0) SG_TRY(tune_tiles(ctx, (cudaStream_t)stream, log_len));
    for (int v = 0; v < tt.n; ++v) {
        cols[v] = (uint32_t)tt.cols[v];
        cost_per_col[v] = tt.cost[v];
    }
    *count = (uint32_t)tt.n;
    return SG_OK;
}
