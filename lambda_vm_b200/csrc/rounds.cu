// Round 2-4 kernels of the STARK prover for sm_100a: batch inversion and
// inverse denominators, barycentric OOD sums, DEEP composition, FRI folding
// with the next layer's leaves fused in, LogUp auxiliary columns, row gathers.
//
// Reference behaviour (CPU semantics the kernels reproduce):
//  * inversion:   FieldElement::inplace_batch_inverse; denominators per
//                 crypto/math-cuda/src/inverse.rs:226-300 (DenomSign).
//  * barycentric: polynomial.rs:207-235 inner sum; barycentric.cu:210-323.
//  * DEEP:        prover.rs:2400-2608 / deep.cu:30-115.
//  * FRI:         fri/fri_functions.rs:15-61, FRI leaves keccak.cu:384.
//  * LogUp:       lookup.rs:1660-1842 with the CSR descriptor of
//                 crypto/math-cuda/src/logup.rs:26-44.
// All layouts are row-major; ext3 values are 3 consecutive u64.
#include <vector>

#include "common.cuh"
#include "gl.cuh"
#include "keccak.cuh"
#include "fs.cuh"

namespace sg {

using gl::fe3;

__device__ __forceinline__ fe3 ld3(const uint64_t* p) { return fe3{p[0], p[1], p[2]}; }
__device__ __forceinline__ void st3(uint64_t* p, fe3 v) {
    p[0] = v.c0;
    p[1] = v.c1;
    p[2] = v.c2;
}
__device__ __forceinline__ fe3 one3() { return fe3{1, 0, 0}; }
__device__ __forceinline__ fe3 zero3() { return fe3{0, 0, 0}; }
__device__ __forceinline__ fe3 shfl_up3(fe3 v, int d) {
    return fe3{__shfl_up_sync(0xffffffffu, v.c0, d), __shfl_up_sync(0xffffffffu, v.c1, d),
               __shfl_up_sync(0xffffffffu, v.c2, d)};
}
__device__ __forceinline__ fe3 shfl_down3(fe3 v, int d) {
    return fe3{__shfl_down_sync(0xffffffffu, v.c0, d), __shfl_down_sync(0xffffffffu, v.c1, d),
               __shfl_down_sync(0xffffffffu, v.c2, d)};
}
__device__ __forceinline__ fe3 shfl3(fe3 v, int src) {
    return fe3{__shfl_sync(0xffffffffu, v.c0, src), __shfl_sync(0xffffffffu, v.c1, src),
               __shfl_sync(0xffffffffu, v.c2, src)};
}
__device__ __forceinline__ bool is_zero3(fe3 v) {
    return gl::canon(v.c0) == 0 && gl::canon(v.c1) == 0 && gl::canon(v.c2) == 0;
}

// ---------------------------------------------------------------- batch inversion
// Montgomery's trick in one pass: each thread owns BI_CH consecutive elements,
// a warp prefix/suffix scan of the thread products gives every thread the
// inverse of its own product from ONE Fp3 inversion per warp (lane 0), and the
// thread then unwinds its chunk. No global scan, no second pass. Lane 0's
// inversion is a serial chain the other lanes wait on, so a warp covers
// 32 * BI_CH elements to spread it (and the scans) thin; the unwind reloads
// the inputs instead of holding them in registers, each before its own
// output is stored (the inversion may run in place). 2^22 x 3 DEEP
// denominators: 4 elements a thread 1.24 ms, 8: 0.82, 12: 0.72, 16: 1.24
// (153 registers, one block per SM); one inversion per block instead of per
// warp: 0.79 (the block waits on one thread's chain).
#define BI_CH 12

struct LoadPlain {
    const uint64_t* in;
    struct Cur {
        uint64_t base;
    };
    __device__ __forceinline__ Cur start(uint64_t base) const { return Cur{base}; }
    __device__ __forceinline__ fe3 at(const Cur& c, int j) const { return ld3(in + 3 * (c.base + j)); }
};
// Denominators z_k - x_i (sign 0) or x_i - z_k (sign 1), element idx = k*n + i.
// A thread's cursor divides once; its later elements step (k, i) forward.
struct LoadDenom {
    const uint64_t* x;
    const uint64_t* z;
    uint64_t n;
    int x_minus_z;
    struct Cur {
        uint64_t k, i;
    };
    __device__ __forceinline__ Cur start(uint64_t base) const {
        const uint64_t k = base / n;
        return Cur{k, base - k * n};
    }
    __device__ __forceinline__ fe3 at(const Cur& c, int j) const {
        uint64_t k = c.k, i = c.i + (uint64_t)j;
        while (i >= n) i -= n, ++k;
        const fe3 zk = ld3(z + 3 * k);
        const uint64_t xi = x[i];
        return x_minus_z ? fe3{gl::sub(xi, zk.c0), gl::neg(zk.c1), gl::neg(zk.c2)}
                         : fe3{gl::sub(zk.c0, xi), zk.c1, zk.c2};
    }
};

template <class Load>
__global__ void __launch_bounds__(256) k_batch_inv(Load load, uint64_t total, uint64_t* out, unsigned* zero_flag) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t base = tid * BI_CH;
    const int lane = threadIdx.x & 31;
    const typename Load::Cur cur = load.start(base < total ? base : 0);
    // prefix products of the chunk; elements past the end count as 1
    fe3 p[BI_CH];
    p[0] = base < total ? load.at(cur, 0) : one3();
#pragma unroll
    for (int i = 1; i < BI_CH; ++i) p[i] = base + i < total ? gl::mul3(p[i - 1], load.at(cur, i)) : p[i - 1];
    const fe3 tot = p[BI_CH - 1];
    fe3 incl = tot, sinc = tot;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const fe3 v = shfl_up3(incl, off);
        if (lane >= off) incl = gl::mul3(v, incl);
        const fe3 w = shfl_down3(sinc, off);
        if (lane + off < 32) sinc = gl::mul3(sinc, w);
    }
    fe3 excl = shfl_up3(incl, 1);
    if (lane == 0) excl = one3();
    fe3 sexcl = shfl_down3(sinc, 1);
    if (lane == 31) sexcl = one3();
    const fe3 T = shfl3(incl, 31);
    fe3 Tinv = zero3();
    if (lane == 0) {
        if (is_zero3(T)) atomicOr(zero_flag, 1u);
        Tinv = gl::inv3(T);
    }
    Tinv = shfl3(Tinv, 0);
    // (excl * tot)^-1 = T^-1 * sexcl ; tot^-1 = that * excl
    fe3 inv = gl::mul3(gl::mul3(Tinv, sexcl), excl);
#pragma unroll
    for (int i = BI_CH - 1; i >= 1; --i) {
        if (base + i < total) {
            const fe3 a = load.at(cur, i);  // before the store: out may alias the input
            st3(out + 3 * (base + i), gl::canon3(gl::mul3(inv, p[i - 1])));
            inv = gl::mul3(inv, a);
        }
    }
    if (base < total) st3(out + 3 * base, gl::canon3(inv));
}

template <class Load>
static int batch_inv_launch(Ctx* ctx, cudaStream_t st, Load load, uint64_t total, uint64_t* out, int* zero_out) {
    if (total == 0) return SG_OK;
    unsigned* d_flag = nullptr;
    SG_TRY(dev_alloc(ctx, st, sizeof(unsigned), (void**)&d_flag));
    int rc = SG_OK;
    if (cudaMemsetAsync(d_flag, 0, sizeof(unsigned), st) != cudaSuccess) {
        set_error("batch inverse: flag reset failed");
        rc = SG_ERR_CUDA;
    }
    if (rc == SG_OK) {
        const uint64_t threads = (total + BI_CH - 1) / BI_CH;
        k_batch_inv<Load><<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(load, total, out, d_flag);
        rc = check_launch(ctx, "k_batch_inv");
    }
    if (rc == SG_OK && zero_out) {
        unsigned h = 0;
        if (cudaMemcpyAsync(&h, d_flag, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            set_error("batch inverse: flag readback failed");
            rc = SG_ERR_CUDA;
        }
        *zero_out = h ? 1 : 0;
    }
    int rf = dev_free(ctx, st, d_flag, sizeof(unsigned));
    return rc != SG_OK ? rc : rf;
}

// ---------------------------------------------------------------- barycentric sums
// out_partial[(chunk * K + k) * cols + c] = sum over the chunk's rows i of
//   points[i] * col_c(row i*stride) * inv_denoms[k][i]
#define BARY_MAX_K 8
#define BARY_PF 4  // rows in flight per thread: 4, 8, 16 measured 1.60, 1.79, 1.78 ms (2^20 x 256, K = 2)
// Block = RL row lanes x CT columns (thread t: lane t / CT, column t % CT of
// the block's column tile). The chunk's rows go in batches of RB: the block
// first forms the row weights W[r][k] = points[i] * inv_denoms[k][i] of the
// batch in shared memory (coalesced loads, one product per row instead of one
// per cell), then lane r walks rows r, r+RL, ... of the batch, so narrow tables
// still fill the block and each warp reads whole row segments. The lanes'
// sums meet in the same shared memory; one partial per (chunk, k, column)
// goes to k_bary_combine.
template <bool EXT3, int K>
__global__ void __launch_bounds__(512) k_bary(const uint64_t* __restrict__ data, uint64_t row_u64, uint64_t stride,
                                              uint64_t cols, uint32_t CT, uint32_t RL, uint32_t RB,
                                              const uint64_t* __restrict__ points,
                                              const uint64_t* __restrict__ invd, uint64_t n, uint64_t chunk_len,
                                              uint64_t* __restrict__ partial) {
    extern __shared__ uint64_t bary_sm[];  // batch weights [RB][K] ext3, then lane sums [RL][CT][K] ext3
    const uint32_t lane = threadIdx.x / CT, cl = threadIdx.x % CT;
    const uint64_t c = (uint64_t)blockIdx.x * CT + cl;
    const bool active = lane < RL && c < cols;
    // Row sums are accumulated unreduced (160-bit, at most 3n products each)
    // and reduced once per thread.
    gl::wacc3 wa[K];
#pragma unroll
    for (int k = 0; k < K; ++k) wa[k] = gl::wzero3();
    const uint64_t i0 = blockIdx.y * chunk_len, i1 = min(n, i0 + chunk_len);
    for (uint64_t b0 = i0; b0 < i1; b0 += RB) {
        const uint32_t nb = (uint32_t)min((uint64_t)RB, i1 - b0);
        __syncthreads();  // the previous batch's weights are consumed
        for (uint32_t e = threadIdx.x; e < nb * K; e += blockDim.x) {
            const uint32_t r = e / K, k = e % K;
            const uint64_t i = b0 + r;
            const uint64_t* dp = invd + 3 * (k * n + i);
            st3(bary_sm + 3 * e, gl::mulb3(fe3{__ldg(dp), __ldg(dp + 1), __ldg(dp + 2)}, __ldg(points + i)));
        }
        __syncthreads();
        if (active) {
            if (EXT3) {
#pragma unroll 4
                for (uint32_t r = lane; r < nb; r += RL) {
                    const uint64_t* row = data + (b0 + r) * stride * row_u64;
                    const uint64_t* wr = bary_sm + 3 * ((uint64_t)r * K);
                    const fe3 t{__ldg(row + 3 * c), __ldg(row + 3 * c + 1), __ldg(row + 3 * c + 2)};
                    const uint64_t t1_2 = gl::add(t.c1, t.c1), t2_2 = gl::add(t.c2, t.c2);
#pragma unroll
                    for (int k = 0; k < K; ++k) gl::wmac3(wa[k], ld3(wr + 3 * k), t, t1_2, t2_2);
                }
            } else {
                // BARY_PF rows' loads issued together, then their products:
                // the loop is bound by load latency, not arithmetic
                for (uint32_t r = lane; r < nb; r += BARY_PF * RL) {
                    uint64_t t[BARY_PF];
#pragma unroll
                    for (int u = 0; u < BARY_PF; ++u) {
                        const uint32_t ru = r + u * RL;
                        t[u] = ru < nb ? __ldg(data + (b0 + ru) * stride * row_u64 + c) : 0;
                    }
#pragma unroll
                    for (int u = 0; u < BARY_PF; ++u) {
                        const uint32_t ru = r + u * RL;
                        if (ru < nb) {
                            const uint64_t* wr = bary_sm + 3 * ((uint64_t)ru * K);
#pragma unroll
                            for (int k = 0; k < K; ++k) gl::wmacb3(wa[k], ld3(wr + 3 * k), t[u]);
                        }
                    }
                }
            }
        }
    }
    fe3 acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = gl::wreduce3(wa[k]);
    __syncthreads();  // the weights are consumed; the buffer takes the lane sums
    if (lane < RL) {
#pragma unroll
        for (int k = 0; k < K; ++k) st3(bary_sm + 3 * (((uint64_t)lane * CT + cl) * K + k), acc[k]);
    }
    __syncthreads();
    if (lane == 0 && c < cols) {
        for (uint32_t r = 1; r < RL; ++r) {
#pragma unroll
            for (int k = 0; k < K; ++k) acc[k] = gl::add3(acc[k], ld3(bary_sm + 3 * (((uint64_t)r * CT + cl) * K + k)));
        }
#pragma unroll
        for (int k = 0; k < K; ++k) st3(partial + 3 * ((blockIdx.y * (uint64_t)K + k) * cols + c), acc[k]);
    }
}

typedef void (*bary_fn)(const uint64_t*, uint64_t, uint64_t, uint64_t, uint32_t, uint32_t, uint32_t,
                        const uint64_t*, const uint64_t*, uint64_t, uint64_t, uint64_t*);
template <bool EXT3>
static bary_fn bary_kernel(uint32_t K) {
    switch (K) {
        case 1: return k_bary<EXT3, 1>;
        case 2: return k_bary<EXT3, 2>;
        case 3: return k_bary<EXT3, 3>;
        case 4: return k_bary<EXT3, 4>;
        case 5: return k_bary<EXT3, 5>;
        case 6: return k_bary<EXT3, 6>;
        case 7: return k_bary<EXT3, 7>;
        default: return k_bary<EXT3, 8>;
    }
}

// One warp per output: lanes sum strided chunk partials, then a shuffle tree.
__global__ void k_bary_combine(const uint64_t* partial, uint64_t chunks, uint64_t per_chunk, uint64_t* out) {
    const uint64_t t = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const uint32_t lane = threadIdx.x % 32;
    if (t >= per_chunk) return;  // whole warp leaves together
    fe3 s = zero3();
    for (uint64_t ch = lane; ch < chunks; ch += 32) s = gl::add3(s, ld3(partial + 3 * (ch * per_chunk + t)));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const fe3 o{__shfl_down_sync(0xffffffffu, s.c0, off), __shfl_down_sync(0xffffffffu, s.c1, off),
                    __shfl_down_sync(0xffffffffu, s.c2, off)};
        s = gl::add3(s, o);
    }
    if (lane == 0) st3(out + 3 * t, gl::canon3(s));
}

// ---------------------------------------------------------------- DEEP
// One thread per LDE row, templated on the number K of trace opening points:
//   result = inv_h * (sum_j g_j H_j(x) - c_h)
//          + sum_k inv_t[k] * (sum_j g'_{jk} t_j(x) - c_k)
// with c_h = sum_j g_j H_j(z^P) and c_k = sum_j g'_{jk} t_j(z w^k) folded on
// the host: the same field value as summing g (t - t_ood) term by term.
// The coefficient loads are uniform across the warp (broadcast); each
// thread streams its own row, whose 32-byte sectors stay in L1 across the
// consecutive column reads that share them. The row is read two columns per
// 16-byte load where it is 16-byte aligned: a warp's load touches 32 rows'
// sectors either way, so pairs halve the L1 lookups, which bound this kernel.
#define DEEP_MAX_K 8
// POW: the trace coefficients are gam_tr[j K + k] = rho_k gam_tr[j K] (the
// prover's successive powers of one gamma give rho_k = gamma^k), so each
// row's K column sums are rho_k times the first: one sum is accumulated
// (half the products at K = 2) and the others are one product each. rho
// (K ext3, rho_0 = 1) follows the constants in `consts`.
template <int K, bool POW>
__global__ void __launch_bounds__(128) k_deep(const uint64_t* __restrict__ main, uint64_t m,
                                              const uint64_t* __restrict__ aux, uint64_t A,
                                              const uint64_t* __restrict__ parts, uint64_t P, uint64_t rows,
                                              uint32_t log_rows, const uint64_t* __restrict__ gam_h,
                                              const uint64_t* __restrict__ gam_tr, const uint64_t* __restrict__ consts,
                                              const uint64_t* __restrict__ inv_h, const uint64_t* __restrict__ inv_t,
                                              int bitrev_out, uint64_t* __restrict__ out) {
    constexpr int KS = POW ? 1 : K;  // column sums accumulated
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    // Column sums are accumulated unreduced (160-bit) and reduced once per row.
    gl::wacc3 acc[K > 0 ? K : 1];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = gl::wzero3();
    const uint64_t* mrow = main + i * m;
    auto col = [&](uint64_t j, uint64_t t) {
        const uint64_t* g = gam_tr + 3 * j * K;
#pragma unroll
        for (int k = 0; k < (K < KS ? K : KS); ++k)
            gl::wmacb3(acc[k], fe3{__ldg(g + 3 * k), __ldg(g + 3 * k + 1), __ldg(g + 3 * k + 2)}, t);
    };
    uint64_t j = 0;
    if (m > 0 && ((uintptr_t)mrow & 15)) col(j++, __ldg(mrow));
    for (; j + 1 < m; j += 2) {
        const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(mrow + j));
        col(j, v.x);
        col(j + 1, v.y);
    }
    if (j < m) col(j, __ldg(mrow + j));
    const uint64_t* arow = aux + i * A * 3;
    for (uint64_t j = 0; j < A; ++j) {
        const fe3 t{__ldg(arow + 3 * j), __ldg(arow + 3 * j + 1), __ldg(arow + 3 * j + 2)};
        const uint64_t t1_2 = gl::add(t.c1, t.c1), t2_2 = gl::add(t.c2, t.c2);
        const uint64_t* g = gam_tr + 3 * (m + j) * K;
#pragma unroll
        for (int k = 0; k < (K < KS ? K : KS); ++k)
            gl::wmac3(acc[k], fe3{__ldg(g + 3 * k), __ldg(g + 3 * k + 1), __ldg(g + 3 * k + 2)}, t, t1_2, t2_2);
    }
    gl::wacc3 acch = gl::wzero3();
    const uint64_t* prow = parts + i * P * 3;
    for (uint64_t j = 0; j < P; ++j) {
        const fe3 h{__ldg(prow + 3 * j), __ldg(prow + 3 * j + 1), __ldg(prow + 3 * j + 2)};
        gl::wmac3(acch, fe3{__ldg(gam_h + 3 * j), __ldg(gam_h + 3 * j + 1), __ldg(gam_h + 3 * j + 2)}, h,
                  gl::add(h.c1, h.c1), gl::add(h.c2, h.c2));
    }
    fe3 sk[K > 0 ? K : 1];
#pragma unroll
    for (int k = 0; k < K; ++k)
        sk[k] = !POW ? gl::wreduce3(acc[k])
              : k == 0 ? gl::wreduce3(acc[0])
                       : gl::mul3(ld3(consts + 3 * (1 + K + k)), sk[0]);
    const fe3 sh = gl::wreduce3(acch);
    fe3 r = gl::mul3(ld3(inv_h + 3 * i), gl::sub3(sh, ld3(consts)));
#pragma unroll
    for (int k = 0; k < K; ++k)
        r = gl::add3(r, gl::mul3(ld3(inv_t + 3 * (k * rows + i)), gl::sub3(sk[k], ld3(consts + 3 * (1 + k)))));
    const uint64_t o = bitrev_out ? (log_rows ? (__brevll(i) >> (64 - log_rows)) : 0) : i;
    st3(out + 3 * o, gl::canon3(r));
}

typedef void (*deep_fn)(const uint64_t*, uint64_t, const uint64_t*, uint64_t, const uint64_t*, uint64_t, uint64_t,
                        uint32_t, const uint64_t*, const uint64_t*, const uint64_t*, const uint64_t*, const uint64_t*,
                        int, uint64_t*);
template <bool POW>
static deep_fn deep_kernel_t(uint32_t K) {
    switch (K) {
        case 0: return k_deep<0, POW>;
        case 1: return k_deep<1, POW>;
        case 2: return k_deep<2, POW>;
        case 3: return k_deep<3, POW>;
        case 4: return k_deep<4, POW>;
        case 5: return k_deep<5, POW>;
        case 6: return k_deep<6, POW>;
        case 7: return k_deep<7, POW>;
        default: return k_deep<8, POW>;
    }
}
static deep_fn deep_kernel(uint32_t K, bool pow) { return pow ? deep_kernel_t<true>(K) : deep_kernel_t<false>(K); }

// ---------------------------------------------------------------- FRI
// Fold one layer (evaluations in bit-reversed order, pairs (2j, 2j+1) are
// x_j and -x_j) and, fused in the same pass, hash the folded layer's leaf
// pairs and derive the next layer's inverse twiddles tw'[j] = tw[2j]^2.
// Each thread produces folded outputs 2t and 2t+1, i.e. exactly leaf t.
__device__ __forceinline__ fe3 fold_one(const uint64_t* in, uint64_t j, uint64_t tw, fe3 zeta) {
    const fe3 lo = ld3(in + 6 * j), hi = ld3(in + 6 * j + 3);
    return gl::add3(gl::add3(lo, hi), gl::mulb3(gl::mul3(zeta, gl::sub3(lo, hi)), tw));
}

// zeta is (z0, z1, z2), or read from device memory when dz is non-null.
__global__ void __launch_bounds__(128) k_fri_fold(const uint64_t* in, uint64_t h, const uint64_t* tw, uint64_t z0,
                                                  uint64_t z1, uint64_t z2, const uint64_t* dz, uint64_t* out,
                                                  uint64_t* tw_next, uint64_t* leaves) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const fe3 zeta = dz ? fe3{dz[0], dz[1], dz[2]} : fe3{z0, z1, z2};
    if (2 * t >= h) return;
    const uint64_t tw0 = tw[2 * t];
    const fe3 a = gl::canon3(fold_one(in, 2 * t, tw0, zeta));
    st3(out + 6 * t, a);
    if (2 * t + 1 < h) {
        const fe3 b = gl::canon3(fold_one(in, 2 * t + 1, tw[2 * t + 1], zeta));
        st3(out + 6 * t + 3, b);
        if (tw_next) tw_next[t] = gl::canon(gl::sqr(tw0));
        if (leaves) {
            // Keccak-256 of 48 bytes: 6 big-endian lanes, pad at lane 6.
            uint64_t s[25];
#pragma unroll
            for (int q = 0; q < 25; ++q) s[q] = 0;
            s[0] = kc::bswap64(a.c0);
            s[1] = kc::bswap64(a.c1);
            s[2] = kc::bswap64(a.c2);
            s[3] = kc::bswap64(b.c0);
            s[4] = kc::bswap64(b.c1);
            s[5] = kc::bswap64(b.c2);
            s[6] = 0x01ULL;
            s[16] = 0x8000000000000000ULL;
            kc::permute(s);
#pragma unroll
            for (int q = 0; q < 4; ++q) leaves[4 * t + q] = s[q];
        }
    }
}

// Leaves of an already-folded layer (pairs of consecutive ext3 values).
__global__ void __launch_bounds__(128) k_fri_leaves(const uint64_t* ev, uint64_t nleaves, uint64_t* leaves) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nleaves) return;
    uint64_t s[25];
#pragma unroll
    for (int q = 0; q < 25; ++q) s[q] = 0;
#pragma unroll
    for (int q = 0; q < 6; ++q) s[q] = kc::bswap64(gl::canon(ev[6 * t + q]));
    s[6] = 0x01ULL;
    s[16] = 0x8000000000000000ULL;
    kc::permute(s);
#pragma unroll
    for (int q = 0; q < 4; ++q) leaves[4 * t + q] = s[q];
}

// ---------------------------------------------------------------- gathers
// out[q * width + c] = data[rows[q] * row_u64 + col0 + c] for c < width.
__global__ void k_gather_rows(const uint64_t* data, uint64_t row_u64, uint64_t nrows, uint64_t col0, uint64_t width,
                              const uint32_t* rows, uint32_t nq, uint64_t* out) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (uint64_t)nq * width) return;
    const uint64_t q = g / width, c = g - q * width;
    const uint64_t r = rows[q];
    out[g] = r < nrows ? data[r * row_u64 + col0 + c] : 0;
}

// ---------------------------------------------------------------- LogUp
// fingerprints fp[k*n + r] = z - (bus_id_k + sum_e alpha^{ai_e} (c_e + sum_t coef_t main[r][col_t]))
struct LogupDesc {
    uint32_t K;
    const uint64_t* bus_ids;
    const uint32_t* elem_off;
    const uint32_t* elem_alpha;
    const uint64_t* elem_const;
    const uint32_t* term_off;
    const uint64_t* term_coef;
    const uint32_t* term_col;
    uint32_t n_out;
    const uint32_t* out_off;
    const uint32_t* out_int;
    const uint64_t* mult_const;
    const uint32_t* mterm_off;
    const uint64_t* mterm_coef;
    const uint32_t* mterm_col;
    uint32_t n_committed;
    const uint64_t* alpha_pows;
};

__global__ void k_logup_fp(const uint64_t* main, uint64_t n, uint64_t m, LogupDesc d, uint64_t z0, uint64_t z1,
                           uint64_t z2, uint64_t* fp) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (uint64_t)d.K * n) return;
    const uint32_t k = (uint32_t)(g / n);
    const uint64_t r = g - (uint64_t)k * n;
    const uint64_t* row = main + r * m;
    fe3 lc{d.bus_ids[k], 0, 0};
    for (uint32_t e = d.elem_off[k]; e < d.elem_off[k + 1]; ++e) {
        uint64_t base = d.elem_const[e];
        for (uint32_t t = d.term_off[e]; t < d.term_off[e + 1]; ++t)
            base = gl::add(base, gl::mul(d.term_coef[t], row[d.term_col[t]]));
        lc = gl::add3(lc, gl::mulb3(ld3(d.alpha_pows + 3 * d.elem_alpha[e]), base));
    }
    st3(fp + 3 * g, gl::sub3(fe3{z0, z1, z2}, lc));
}

// Terms per row: committed columns go to aux[r][c]; row sums to rsum[r].
__global__ void k_logup_terms(const uint64_t* main, uint64_t n, uint64_t m, LogupDesc d, const uint64_t* recip,
                              uint64_t* aux, uint64_t* rsum) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint64_t* row = main + r * m;
    const uint64_t W = (uint64_t)d.n_committed + 1;
    fe3 s = zero3();
    for (uint32_t c = 0; c < d.n_out; ++c) {
        fe3 term = zero3();
        for (uint32_t ki = d.out_off[c]; ki < d.out_off[c + 1]; ++ki) {
            const uint32_t k = d.out_int[ki];
            uint64_t mu = d.mult_const[k];
            for (uint32_t t = d.mterm_off[k]; t < d.mterm_off[k + 1]; ++t)
                mu = gl::add(mu, gl::mul(d.mterm_coef[t], row[d.mterm_col[t]]));
            term = gl::add3(term, gl::mulb3(ld3(recip + 3 * ((uint64_t)k * n + r)), mu));
        }
        if (c < d.n_committed) st3(aux + 3 * (r * W + c), gl::canon3(term));
        s = gl::add3(s, term);
    }
    st3(rsum + 3 * r, s);
}

// Segment sums of rsum over SEG rows.
#define LG_SEG 1024
__global__ void __launch_bounds__(256) k_seg_sum(const uint64_t* rsum, uint64_t n, uint64_t* seg) {
    __shared__ uint64_t sh[3 * 8];
    const uint64_t s0 = (uint64_t)blockIdx.x * LG_SEG;
    fe3 acc = zero3();
    for (uint64_t r = s0 + threadIdx.x; r < min(n, s0 + LG_SEG); r += blockDim.x) acc = gl::add3(acc, ld3(rsum + 3 * r));
    for (int off = 16; off >= 1; off >>= 1) acc = gl::add3(acc, shfl_down3(acc, off));
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) st3(sh + 3 * w, acc);
    __syncthreads();
    if (threadIdx.x == 0) {
        fe3 t = zero3();
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t = gl::add3(t, ld3(sh + 3 * q));
        st3(seg + 3 * blockIdx.x, t);
    }
}

// Exclusive prefix of the segment sums, total L and offset L/n (one thread:
// at most n/1024 segments).
__global__ void k_seg_scan(uint64_t* seg, uint64_t nseg, uint64_t ninv, uint64_t* L_off) {
    if (threadIdx.x || blockIdx.x) return;
    fe3 run = zero3();
    for (uint64_t s = 0; s < nseg; ++s) {
        const fe3 v = ld3(seg + 3 * s);
        st3(seg + 3 * s, run);
        run = gl::add3(run, v);
    }
    st3(L_off, gl::canon3(run));
    st3(L_off + 3, gl::mulb3(run, ninv));
}

// acc[r] = (sum_{r' < r} rsum[r']) - r * (L / n), written to aux column W-1.
__global__ void __launch_bounds__(1024) k_logup_acc(const uint64_t* rsum, uint64_t n, const uint64_t* seg,
                                                    const uint64_t* L_off, uint64_t W, uint64_t* aux) {
    __shared__ uint64_t wsum[3 * 32];
    const uint64_t r = (uint64_t)blockIdx.x * LG_SEG + threadIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    fe3 v = r < n ? ld3(rsum + 3 * r) : zero3();
    fe3 incl = v;
    for (int off = 1; off < 32; off <<= 1) {
        const fe3 u = shfl_up3(incl, off);
        if (lane >= off) incl = gl::add3(incl, u);
    }
    if (lane == 31) st3(wsum + 3 * w, incl);
    __syncthreads();
    if (w == 0) {
        fe3 x = ld3(wsum + 3 * lane);
        fe3 xi = x;
        for (int off = 1; off < 32; off <<= 1) {
            const fe3 u = shfl_up3(xi, off);
            if (lane >= off) xi = gl::add3(xi, u);
        }
        st3(wsum + 3 * lane, gl::sub3(xi, x));  // exclusive warp prefix
    }
    __syncthreads();
    if (r >= n) return;
    const fe3 excl = gl::add3(gl::add3(ld3(seg + 3 * blockIdx.x), ld3(wsum + 3 * w)), gl::sub3(incl, v));
    const fe3 off = ld3(L_off + 3);
    st3(aux + 3 * (r * W + (W - 1)), gl::canon3(gl::sub3(excl, gl::mulb3(off, r % GL_P))));
}

}  // namespace sg

using namespace sg;

static Ctx* CX(sg_ctx* c) { return reinterpret_cast<Ctx*>(c); }

extern "C" {

int sg_batch_inverse_ext3(sg_ctx* c, void* stream, const uint64_t* d_in, uint64_t n, uint64_t* d_out,
                          int* zero_found) {
    SG_CHECK_ARG(c && (n == 0 || (d_in && d_out)), "null argument");
    SG_ENTER(ctx_of(c));
    return batch_inv_launch(CX(c), (cudaStream_t)stream, LoadPlain{d_in}, n, d_out, zero_found);
}

int sg_inv_denoms_ext3(sg_ctx* c, void* stream, const uint64_t* d_x, uint64_t n, const uint64_t* z_host, uint32_t k,
                       int x_minus_z, uint64_t* d_out, int* zero_found) {
    SG_CHECK_ARG(c && z_host && (n == 0 || (d_x && d_out)), "null argument");
    SG_ENTER(ctx_of(c));
    Ctx* ctx = CX(c);
    cudaStream_t st = (cudaStream_t)stream;
    if (n == 0 || k == 0) return SG_OK;
    uint64_t* d_z = nullptr;
    SG_TRY(dev_alloc(ctx, st, 24ull * k, (void**)&d_z));
    int rc = SG_OK;
    if (cudaMemcpyAsync(d_z, z_host, 24ull * k, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        set_error("inv_denoms: z upload failed");
        rc = SG_ERR_CUDA;
    }
    if (rc == SG_OK) rc = batch_inv_launch(ctx, st, LoadDenom{d_x, d_z, n, x_minus_z}, n * k, d_out, zero_found);
    int rf = dev_free(ctx, st, d_z, 24ull * k);
    return rc != SG_OK ? rc : rf;
}

int sg_barycentric_sums(sg_ctx* c, void* stream, const uint64_t* d_data, uint64_t row_u64, uint64_t row_stride,
                        int ext3, uint64_t cols, const uint64_t* d_points, const uint64_t* d_inv_denoms, uint64_t n,
                        uint32_t k, uint64_t* d_out) {
    SG_CHECK_ARG(c, "null context");
    SG_ENTER(ctx_of(c));
    SG_CHECK_ARG(k >= 1 && k <= BARY_MAX_K, "1 <= k <= 8 evaluation points");
    SG_CHECK_ARG(cols * (ext3 ? 3 : 1) <= row_u64, "columns exceed the row width");
    Ctx* ctx = CX(c);
    cudaStream_t st = (cudaStream_t)stream;
    if (cols == 0) return SG_OK;
    if (n == 0) {
        SG_CUDA(cudaMemsetAsync(d_out, 0, 24ull * k * cols, st));
        return SG_OK;
    }
    // Column tile of at most 512 threads; row lanes fill the block to >= 256 threads.
    const uint64_t ctiles = (cols + 511) / 512;
    const uint32_t CT = (uint32_t)((cols + ctiles - 1) / ctiles);
    const uint32_t RL = CT >= 256 ? 1u : 256u / CT;
    const uint32_t threads = (RL * CT + 31) / 32 * 32;
    // weight batches of at least 64 rows, a whole number of row lanes
    const uint32_t RB = RL >= 64 ? RL : (64 + RL - 1) / RL * RL;
    const size_t smem = 24ull * k * (RB > RL * CT ? RB : RL * CT);
    // About four blocks of work per SM in total, each chunk at least RL rows.
    uint64_t chunks = (148 * 4 + ctiles - 1) / ctiles;
    const uint64_t max_chunks = (n + RL - 1) / RL;
    if (chunks > max_chunks) chunks = max_chunks;
    if (chunks > 65535) chunks = 65535;
    const uint64_t chunk_len = (n + chunks - 1) / chunks;
    chunks = (n + chunk_len - 1) / chunk_len;
    uint64_t* part = nullptr;
    SG_TRY(dev_alloc(ctx, st, 24ull * chunks * k * cols, (void**)&part));
    dim3 grid((unsigned)ctiles, (unsigned)chunks);
    bary_fn fn = ext3 ? bary_kernel<true>(k) : bary_kernel<false>(k);
    if (smem > 48 * 1024) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    fn<<<grid, threads, smem, st>>>(d_data, row_u64, row_stride, cols, CT, RL, RB, d_points, d_inv_denoms, n, chunk_len,
                                    part);
    int rc = check_launch(ctx, "k_bary");
    if (rc == SG_OK) {
        const uint64_t per = (uint64_t)k * cols;
        k_bary_combine<<<(unsigned)((per * 32 + 255) / 256), 256, 0, st>>>(part, chunks, per, d_out);
        rc = check_launch(ctx, "k_bary_combine");
    }
    int rf = dev_free(ctx, st, part, 24ull * chunks * k * cols);
    return rc != SG_OK ? rc : rf;
}

int sg_deep_composition(sg_ctx* c, void* stream, const uint64_t* d_main, uint64_t m, const uint64_t* d_aux,
                        uint64_t a, const uint64_t* d_parts, uint64_t p, uint64_t rows, const uint64_t* h_ood,
                        const uint64_t* trace_ood, const uint64_t* gammas_h, const uint64_t* gammas_tr, uint32_t k,
                        const uint64_t* d_inv_h, const uint64_t* d_inv_t, int bitrev_out, uint64_t* d_out) {
    SG_CHECK_ARG(c && h_ood && trace_ood && gammas_h && gammas_tr, "null argument");
    SG_ENTER(ctx_of(c));
    SG_CHECK_ARG(k <= DEEP_MAX_K, "at most 8 evaluation points");
    const int lr = log2_exact(rows);
    SG_CHECK_ARG(!bitrev_out || lr >= 0, "bit-reversed output needs a power-of-two row count");
    Ctx* ctx = CX(c);
    cudaStream_t st = (cudaStream_t)stream;
    if (rows == 0) return SG_OK;
    // Host side: fold the OOD terms into constants c_h, c_k (field identities).
    const uint64_t ng_h = 3 * p, ng_t = 3 * (m + a) * k;
    auto mulc = [](const uint64_t* x, const uint64_t* y, uint64_t* o) { sg_host_fp3_mul(x, y, o); };
    uint64_t ch[3] = {0, 0, 0};
    for (uint64_t j = 0; j < p; ++j) {
        uint64_t t[3];
        mulc(gammas_h + 3 * j, h_ood + 3 * j, t);
        sg_host_fp3_add(ch, t, ch);
    }
    std::vector<uint64_t> consts(3 * (1 + k), 0);
    consts[0] = ch[0];
    consts[1] = ch[1];
    consts[2] = ch[2];
    for (uint32_t kk = 0; kk < k; ++kk) {
        uint64_t acc[3] = {0, 0, 0};
        for (uint64_t j = 0; j < m + a; ++j) {
            uint64_t t[3];
            mulc(gammas_tr + 3 * (j * k + kk), trace_ood + 3 * (j * k + kk), t);
            sg_host_fp3_add(acc, t, acc);
        }
        consts[3 * (1 + kk)] = acc[0];
        consts[3 * (1 + kk) + 1] = acc[1];
        consts[3 * (1 + kk) + 2] = acc[2];
    }
    // When every column's coefficients are rho_kk times its first (the
    // prover's powers of one gamma), the kernel accumulates one sum a row:
    // rho_kk = g[kk] / g[0] from column 0, checked on every column.
    bool pow = k > 1;
    std::vector<uint64_t> rho(3 * k, 0);
    if (pow) {
        uint64_t g0i[3];
        pow = sg_host_fp3_inv(gammas_tr, g0i) == 0;
        for (uint32_t kk = 0; pow && kk < k; ++kk) mulc(gammas_tr + 3 * kk, g0i, rho.data() + 3 * kk);
        for (uint64_t j = 1; pow && j < m + a; ++j)
            for (uint32_t kk = 1; pow && kk < k; ++kk) {
                uint64_t t[3];
                mulc(rho.data() + 3 * kk, gammas_tr + 3 * (j * k), t);
                const uint64_t* g = gammas_tr + 3 * (j * k + kk);
                pow = t[0] == sg_host_gl_canon(g[0]) && t[1] == sg_host_gl_canon(g[1]) && t[2] == sg_host_gl_canon(g[2]);
            }
    }
    if (pow) consts.insert(consts.end(), rho.begin(), rho.end());
    uint64_t* d_g = nullptr;
    const uint64_t gbytes = 8 * (ng_h + ng_t + consts.size());
    SG_TRY(dev_alloc(ctx, st, gbytes, (void**)&d_g));
    int rc = SG_OK;
    if (cudaMemcpyAsync(d_g, gammas_h, 8 * ng_h, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(d_g + ng_h, gammas_tr, 8 * ng_t, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(d_g + ng_h + ng_t, consts.data(), 8 * consts.size(), cudaMemcpyHostToDevice, st) != cudaSuccess) {
        set_error("deep: coefficient upload failed");
        rc = SG_ERR_CUDA;
    }
    if (rc == SG_OK) {
        deep_kernel(k, pow)<<<(unsigned)((rows + 127) / 128), 128, 0, st>>>(d_main, m, d_aux, a, d_parts, p, rows,
                                                                        lr < 0 ? 0 : (uint32_t)lr, d_g, d_g + ng_h,
                                                                        d_g + ng_h + ng_t, d_inv_h, d_inv_t,
                                                                        bitrev_out, d_out);
        rc = check_launch(ctx, "k_deep");
        // keep host vectors alive until the copies have been consumed
        if (rc == SG_OK && cudaStreamSynchronize(st) != cudaSuccess) {
            set_error("deep: sync failed");
            rc = SG_ERR_CUDA;
        }
    }
    int rf = dev_free(ctx, st, d_g, gbytes);
    return rc != SG_OK ? rc : rf;
}

int sg_fri_fold_layer(sg_ctx* c, void* stream, const uint64_t* d_in, uint64_t h, const uint64_t* d_inv_tw,
                      const uint64_t zeta[3], uint64_t* d_out, uint64_t* d_inv_tw_next, uint8_t* d_leaves) {
    SG_CHECK_ARG(c && zeta, "null argument");
    SG_ENTER(ctx_of(c));
    SG_CHECK_ARG(!d_leaves || (h % 2 == 0), "leaves need an even folded length");
    if (h == 0) return SG_OK;
    const uint64_t threads = (h + 1) / 2;
    k_fri_fold<<<(unsigned)((threads + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        d_in, h, d_inv_tw, zeta[0], zeta[1], zeta[2], nullptr, d_out, d_inv_tw_next, (uint64_t*)d_leaves);
    return check_launch(CX(c), "k_fri_fold");
}

int sg_fri_leaves(sg_ctx* c, void* stream, const uint64_t* d_evals, uint64_t n, uint8_t* d_leaves) {
    SG_CHECK_ARG(c, "null context");
    SG_ENTER(ctx_of(c));
    SG_CHECK_ARG(n % 2 == 0, "FRI leaves hash pairs: even length required");
    if (n == 0) return SG_OK;
    k_fri_leaves<<<(unsigned)((n / 2 + 127) / 128), 128, 0, (cudaStream_t)stream>>>(d_evals, n / 2,
                                                                                     (uint64_t*)d_leaves);
    return check_launch(CX(c), "k_fri_leaves");
}

int sg_gather_rows(sg_ctx* c, void* stream, const uint64_t* d_data, uint64_t row_u64, uint64_t nrows, uint64_t col0,
                   uint64_t width, const uint32_t* d_rows, uint32_t nq, uint64_t* d_out) {
    SG_CHECK_ARG(c, "null context");
    SG_ENTER(ctx_of(c));
    SG_CHECK_ARG(col0 + width <= row_u64, "column range exceeds the row");
    const uint64_t tot = (uint64_t)nq * width;
    if (tot == 0) return SG_OK;
    k_gather_rows<<<(unsigned)((tot + 255) / 256), 256, 0, (cudaStream_t)stream>>>(d_data, row_u64, nrows, col0,
                                                                                  width, d_rows, nq, d_out);
    return check_launch(CX(c), "k_gather_rows");
}

int sg_logup_aux(sg_ctx* c, void* stream, const uint64_t* d_main, uint64_t n, uint64_t m, const sg_logup_desc* hd,
                 const uint64_t* alpha_powers, uint32_t num_alpha, const uint64_t z[3], uint64_t* d_aux,
                 uint64_t table_contribution[3]) {
    SG_CHECK_ARG(c && hd && z && table_contribution, "null argument");
    SG_ENTER(ctx_of(c));
    SG_CHECK_ARG(n >= 1, "n must be >= 1");
    SG_CHECK_ARG(hd->num_committed <= hd->num_out_cols, "committed columns exceed output columns");
    Ctx* ctx = CX(c);
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t K = hd->num_interactions, NO = hd->num_out_cols;
    const uint32_t ne = K ? hd->elem_offsets[K] : 0, nt = ne ? hd->term_offsets[ne] : 0;
    const uint32_t noi = NO ? hd->out_col_offsets[NO] : 0, nmt = K ? hd->mult_term_offsets[K] : 0;
    // Validate CSR indices on the host: every column index must be < m and
    // every interaction index < K, so the kernels never read out of bounds.
    for (uint32_t t = 0; t < nt; ++t) SG_CHECK_ARG(hd->term_cols[t] < m, "fingerprint term column out of range");
    for (uint32_t t = 0; t < nmt; ++t) SG_CHECK_ARG(hd->mult_term_cols[t] < m, "multiplicity column out of range");
    for (uint32_t t = 0; t < noi; ++t) SG_CHECK_ARG(hd->out_col_interactions[t] < K, "interaction index out of range");
    for (uint32_t e = 0; e < ne; ++e) SG_CHECK_ARG(hd->elem_alpha_idx[e] < num_alpha, "alpha power index out of range");
    for (uint32_t k = 0; k < K; ++k) SG_CHECK_ARG(hd->elem_offsets[k] <= hd->elem_offsets[k + 1], "elem offsets");
    for (uint32_t e = 0; e < ne; ++e) SG_CHECK_ARG(hd->term_offsets[e] <= hd->term_offsets[e + 1], "term offsets");
    for (uint32_t o = 0; o < NO; ++o) SG_CHECK_ARG(hd->out_col_offsets[o] <= hd->out_col_offsets[o + 1], "out offsets");
    for (uint32_t k = 0; k < K; ++k)
        SG_CHECK_ARG(hd->mult_term_offsets[k] <= hd->mult_term_offsets[k + 1], "mult offsets");
    // One device blob for the descriptor.
    std::vector<uint64_t> blob;
    auto put64 = [&](const uint64_t* p, size_t cnt) {
        size_t o = blob.size();
        blob.insert(blob.end(), p, p + cnt);
        return o;
    };
    auto put32 = [&](const uint32_t* p, size_t cnt) {
        size_t o = blob.size();
        for (size_t i = 0; i < cnt; i += 2) {
            uint64_t lo = p[i], hi = i + 1 < cnt ? p[i + 1] : 0;
            blob.push_back(lo | (hi << 32));
        }
        if (cnt == 0) blob.push_back(0);
        return o;
    };
    const uint32_t zero32[2] = {0, 0};
    const size_t o_bus = put64(hd->bus_ids, K), o_eo = put32(K ? hd->elem_offsets : zero32, K + 1),
                 o_ea = put32(hd->elem_alpha_idx, ne), o_ec = put64(hd->elem_consts, ne),
                 o_to = put32(ne ? hd->term_offsets : zero32, ne + 1), o_tc = put64(hd->term_coefs, nt),
                 o_tl = put32(hd->term_cols, nt), o_oo = put32(NO ? hd->out_col_offsets : zero32, NO + 1),
                 o_oi = put32(hd->out_col_interactions, noi), o_mc = put64(hd->mult_consts, K),
                 o_mo = put32(K ? hd->mult_term_offsets : zero32, K + 1), o_mk = put64(hd->mult_term_coefs, nmt),
                 o_ml = put32(hd->mult_term_cols, nmt), o_al = put64(alpha_powers, 3ull * num_alpha);
    blob.push_back(0);
    const uint64_t W = (uint64_t)hd->num_committed + 1;
    const uint64_t nseg = (n + LG_SEG - 1) / LG_SEG;
    uint64_t *d_blob = nullptr, *d_fp = nullptr, *d_rs = nullptr, *d_seg = nullptr;
    const uint64_t bb = 8 * blob.size(), fb = 24ull * (uint64_t)K * n + 24, rb = 24ull * n, sb = 24ull * (nseg + 2);
    int rc = dev_alloc(ctx, st, bb, (void**)&d_blob);
    if (rc == SG_OK) rc = dev_alloc(ctx, st, fb, (void**)&d_fp);
    if (rc == SG_OK) rc = dev_alloc(ctx, st, rb, (void**)&d_rs);
    if (rc == SG_OK) rc = dev_alloc(ctx, st, sb, (void**)&d_seg);
    if (rc == SG_OK && cudaMemcpyAsync(d_blob, blob.data(), bb, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        set_error("logup: descriptor upload failed");
        rc = SG_ERR_CUDA;
    }
    if (rc == SG_OK) {
        auto u32p = [&](size_t o) { return (const uint32_t*)(d_blob + o); };
        LogupDesc d{K,          d_blob + o_bus, u32p(o_eo),     u32p(o_ea),     d_blob + o_ec,
                    u32p(o_to), d_blob + o_tc,  u32p(o_tl),     NO,             u32p(o_oo),
                    u32p(o_oi), d_blob + o_mc,  u32p(o_mo),     d_blob + o_mk,  u32p(o_ml),
                    hd->num_committed, d_blob + o_al};
        if (K) {
            const uint64_t tot = (uint64_t)K * n;
            k_logup_fp<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(d_main, n, m, d, z[0], z[1], z[2], d_fp);
            rc = check_launch(ctx, "k_logup_fp");
            int zf = 0;
            if (rc == SG_OK) rc = batch_inv_launch(ctx, st, LoadPlain{d_fp}, tot, d_fp, &zf);
            if (rc == SG_OK && zf) {
                set_error("logup: a fingerprint is zero (challenge collides with a row value)");
                rc = SG_ERR_INVALID;
            }
        }
        if (rc == SG_OK) {
            k_logup_terms<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(d_main, n, m, d, d_fp, d_aux, d_rs);
            rc = check_launch(ctx, "k_logup_terms");
        }
        if (rc == SG_OK) {
            k_seg_sum<<<(unsigned)nseg, 256, 0, st>>>(d_rs, n, d_seg + 6);
            rc = check_launch(ctx, "k_seg_sum");
        }
        if (rc == SG_OK) {
            const uint64_t ninv = sg_host_gl_inv(n % GL_P);
            k_seg_scan<<<1, 32, 0, st>>>(d_seg + 6, nseg, ninv, d_seg);
            rc = check_launch(ctx, "k_seg_scan");
        }
        if (rc == SG_OK) {
            k_logup_acc<<<(unsigned)nseg, LG_SEG, 0, st>>>(d_rs, n, d_seg + 6, d_seg, W, d_aux);
            rc = check_launch(ctx, "k_logup_acc");
        }
        if (rc == SG_OK && (cudaMemcpyAsync(table_contribution, d_seg, 24, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                            cudaStreamSynchronize(st) != cudaSuccess)) {
            set_error("logup: contribution readback failed");
            rc = SG_ERR_CUDA;
        }
    }
    dev_free(ctx, st, d_seg, sb);
    dev_free(ctx, st, d_rs, rb);
    dev_free(ctx, st, d_fp, fb);
    dev_free(ctx, st, d_blob, bb);
    return rc;
}

}  // extern "C"

// ---------------------------------------------------------------- FRI commit state
// The stateful form of the FRI commit phase (FriCommitState, crypto/math-cuda/src/fri.rs:48-255):
// it owns the current codeword and twiddles, and every committed layer's
// evaluations and Merkle tree stay resident for the query phase.
struct sg_fri {
    sg::Ctx* ctx;
    cudaStream_t st;
    uint64_t* cur;      // current evaluations (3 * n u64)
    uint64_t n;
    bool own_cur;       // false while cur is the caller's layer-0 buffer
    uint64_t* tw;       // inverse twiddles of the current layer (n / 2 u64)
    struct Layer {
        uint64_t* evals;
        uint64_t n;
        uint8_t* nodes;
        uint64_t leaves;
    };
    std::vector<Layer> layers;
    uint64_t* final_evals = nullptr;
    uint64_t final_n = 0;
};

extern "C" {

int sg_fri_begin(sg_ctx* c, void* stream, const uint64_t* evals, int evals_on_device, const uint64_t* inv_tw,
                 int tw_on_device, uint64_t n0, sg_fri** out) {
    using namespace sg;
    SG_CHECK_ARG(c && evals && inv_tw && out, "null argument");
    SG_ENTER(ctx_of(c));
    SG_CHECK_ARG(n0 >= 2 && log2_exact(n0) >= 0, "n0 must be a power of two >= 2");
    *out = nullptr;
    Ctx* ctx = CX(c);
    cudaStream_t st = (cudaStream_t)stream;
    sg_fri* f = new sg_fri{ctx, st, nullptr, n0, false, nullptr, {}};
    int rc = SG_OK;
    if (evals_on_device) {
        f->cur = const_cast<uint64_t*>(evals);
    } else {
        rc = dev_alloc(ctx, st, 24 * n0, (void**)&f->cur);
        f->own_cur = rc == SG_OK;
        if (rc == SG_OK && cudaMemcpyAsync(f->cur, evals, 24 * n0, cudaMemcpyHostToDevice, st) != cudaSuccess) {
            set_error("fri: evaluations upload failed");
            rc = SG_ERR_CUDA;
        }
    }
    if (rc == SG_OK) rc = dev_alloc(ctx, st, 8 * (n0 / 2), (void**)&f->tw);
    if (rc == SG_OK && cudaMemcpyAsync(f->tw, inv_tw, 8 * (n0 / 2),
                                       tw_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                       st) != cudaSuccess) {
        set_error("fri: twiddles upload failed");
        rc = SG_ERR_CUDA;
    }
    if (rc != SG_OK) {
        sg_fri_free(f);
        return rc;
    }
    *out = f;
    return SG_OK;
}

static int fri_fold_step(sg_fri* f, const uint64_t zeta[3], bool commit, uint8_t root_out[32],
                         uint64_t* host_evals_out) {
    using namespace sg;
    SG_CHECK_ARG(f && zeta, "null argument");
    SG_CHECK_ARG(!f->final_evals, "the final fold has been taken");
    const uint64_t h = f->n / 2;
    SG_CHECK_ARG(h >= (commit ? 2u : 1u), "codeword too short for another fold");
    Ctx* ctx = f->ctx;
    SG_ENTER(ctx);
    uint64_t *out = nullptr, *twn = nullptr;
    uint8_t* nodes = nullptr;
    const uint64_t nl = h / 2;
    int rc = dev_alloc(ctx, f->st, 24 * h, (void**)&out);
    if (rc == SG_OK) rc = dev_alloc(ctx, f->st, 8 * (nl ? nl : 1), (void**)&twn);
    if (rc == SG_OK && commit) rc = dev_alloc(ctx, f->st, (2 * nl - 1) * 32, (void**)&nodes);
    if (rc == SG_OK)
        rc = sg_fri_fold_layer(reinterpret_cast<sg_ctx*>(ctx), f->st, f->cur, h, f->tw, zeta, out, twn,
                               commit ? nodes + (nl - 1) * 32 : nullptr);
    if (rc == SG_OK && commit) rc = merkle_inner(ctx, f->st, nodes, nl);
    cudaError_t e = cudaSuccess;
    if (rc == SG_OK && commit && root_out) e = cudaMemcpyAsync(root_out, nodes, 32, cudaMemcpyDeviceToHost, f->st);
    if (rc == SG_OK && e == cudaSuccess && host_evals_out)
        e = cudaMemcpyAsync(host_evals_out, out, 24 * h, cudaMemcpyDeviceToHost, f->st);
    if (rc == SG_OK && e == cudaSuccess) e = cudaStreamSynchronize(f->st);
    if (rc == SG_OK && e != cudaSuccess) {
        set_error(std::string("fri fold: ") + cudaGetErrorString(e));
        rc = SG_ERR_CUDA;
    }
    if (rc != SG_OK) {
        dev_free(ctx, f->st, out, 24 * h);
        dev_free(ctx, f->st, twn, 8 * (nl ? nl : 1));
        dev_free(ctx, f->st, nodes, (2 * nl - 1) * 32);
        return rc;
    }
    if (f->own_cur && f->layers.empty()) dev_free(ctx, f->st, f->cur, 24 * f->n);  // the uploaded layer 0
    dev_free(ctx, f->st, f->tw, 8 * (f->n / 2 ? f->n / 2 : 1));
    f->tw = twn;
    if (commit) {
        f->layers.push_back({out, h, nodes, nl});
    } else {
        f->final_evals = out;
        f->final_n = h;
    }
    f->cur = out;
    f->n = h;
    return SG_OK;
}

int sg_fri_fold_commit_layer(sg_fri* f, const uint64_t zeta[3], uint8_t root_out[32], uint64_t* host_evals_out) {
    return fri_fold_step(f, zeta, true, root_out, host_evals_out);
}

int sg_fri_fold_final(sg_fri* f, const uint64_t zeta[3], uint64_t* host_evals_out) {
    return fri_fold_step(f, zeta, false, nullptr, host_evals_out);
}

uint32_t sg_fri_num_layers(const sg_fri* f) { return f ? (uint32_t)f->layers.size() : 0; }

int sg_fri_layer(const sg_fri* f, uint32_t layer, const uint64_t** d_evals, uint64_t* n, const uint8_t** d_nodes,
                 uint64_t* leaves_len) {
    SG_CHECK_ARG(f && layer < f->layers.size(), "no such FRI layer");
    const auto& L = f->layers[layer];
    if (d_evals) *d_evals = L.evals;
    if (n) *n = L.n;
    if (d_nodes) *d_nodes = L.nodes;
    if (leaves_len) *leaves_len = L.leaves;
    return SG_OK;
}

void sg_fri_free(sg_fri* f) {
    using namespace sg;
    if (!f) return;
    Ctx* ctx = f->ctx;
    enter(ctx);  // best effort: the layers are released either way
    for (auto& L : f->layers) {
        dev_free(ctx, f->st, L.evals, 24 * L.n);
        dev_free(ctx, f->st, L.nodes, (2 * L.leaves - 1) * 32);
    }
    if (f->final_evals) dev_free(ctx, f->st, f->final_evals, 24 * f->final_n);
    if (f->own_cur && f->layers.empty() && !f->final_evals) dev_free(ctx, f->st, f->cur, 24 * f->n);
    if (f->tw) dev_free(ctx, f->st, f->tw, 8 * (f->n / 2 ? f->n / 2 : 1));
    delete f;
}

}  // extern "C"

// ---------------------------------------------------------------- field self-test
// Element-wise Goldilocks / Fp3 operations on device vectors, for checking the
// device arithmetic (add, sub, mul, reduce, Fp3 mul / inverse, the lazily
// reduced sums) against exact integer arithmetic on the host. Ops:
//   0 add, 1 sub, 2 mul, 3 canon(a), 4 neg(a), 5 inv(a), 6 sqr(a),
//   7 Fp3 mul (a, b, out: 3 u64 per element), 8 Fp3 inverse (a),
//   9 reduce128 of (a = low 64 bits, b = high 64 bits),
//   10 sum of a[i] * b[j] for j < 16 accumulated unreduced (wacc) then reduced.
namespace sg {
// gl::mul_2exp<S> for a runtime S < 96 (a chain of compile-time cases).
template <int S>
__device__ __forceinline__ uint64_t mul_2exp_rt(uint64_t x, uint32_t s) {
    if constexpr (S == 96)
        return 0;
    else
        return s == S ? gl::mul_2exp<S>(x) : mul_2exp_rt<S + 1>(x, s);
}

__global__ void k_field_ops(uint32_t op, const uint64_t* a, const uint64_t* b, uint64_t* out, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    switch (op) {
        case 0: out[i] = gl::add(a[i], b[i]); break;
        case 1: out[i] = gl::sub(a[i], b[i]); break;
        case 2: out[i] = gl::mul(a[i], b[i]); break;
        case 3: out[i] = gl::canon(a[i]); break;
        case 4: out[i] = gl::neg(a[i]); break;
        case 5: out[i] = gl::inv(gl::canon(a[i])); break;
        case 6: out[i] = gl::sqr(a[i]); break;
        case 7: st3(out + 3 * i, gl::mul3(ld3(a + 3 * i), ld3(b + 3 * i))); break;
        case 8: st3(out + 3 * i, gl::inv3(ld3(a + 3 * i))); break;
        case 9:
            out[i] = gl::reduce128((uint32_t)a[i], (uint32_t)(a[i] >> 32), (uint32_t)b[i], (uint32_t)(b[i] >> 32));
            break;
        case 10: {
            gl::wacc w = gl::wzero();
            for (uint64_t j = 0; j < 16; ++j) gl::wmac(w, a[i], b[(i + j) % n]);
            out[i] = gl::wreduce(w);
            break;
        }
        case 11: out[i] = mul_2exp_rt<0>(a[i], (uint32_t)(b[i] % 96)); break;
        default: break;
    }
}
}  // namespace sg

extern "C" int sg_field_ops(sg_ctx* c, void* stream, uint32_t op, const uint64_t* d_a, const uint64_t* d_b,
                            uint64_t* d_out, uint64_t n) {
    using namespace sg;
    SG_CHECK_ARG(c && op <= 11, "null context or unknown op");
    SG_ENTER(ctx_of(c));
    if (n == 0) return SG_OK;
    k_field_ops<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(op, d_a, d_b, d_out, n);
    return check_launch(CX(c), "k_field_ops");
}

// ---- FRI commit phase without host round trips (fri/mod.rs:27-151): the
// transcript steps between layers run on the device on a copy of the
// transcript, so a table's layers are all enqueued before anything is read
// back.
namespace sg {

// Absorb the previous layer's root when there is one (and keep a copy of it
// at root_out), then sample the next folding challenge into zeta. One thread:
// a step is one or two permutations.
__global__ void k_fri_challenge(fs::State* ts, const uint8_t* root, uint8_t* root_out, uint64_t* zeta) {
    if (threadIdx.x || blockIdx.x) return;
    fs::State s = *ts;
    if (root) {
        fs::append(s, root, 32);
        for (int i = 0; i < 32; ++i) root_out[i] = root[i];
    }
    uint64_t z[3];
    fs::sample_ext3(s, z);
    zeta[0] = z[0], zeta[1] = z[1], zeta[2] = z[2];
    *ts = s;
}

// The host transcript's state into device memory, as a kernel argument (no
// copy from pageable memory, which would wait for the stream).
__global__ void k_fs_load(fs::State s, fs::State* ts) {
    if (threadIdx.x || blockIdx.x) return;
    *ts = s;
}

int fri_state_load_dev(Ctx* ctx, cudaStream_t st, const void* host_state, void* d_state) {
    k_fs_load<<<1, 32, 0, st>>>(*(const fs::State*)host_state, (fs::State*)d_state);
    return check_launch(ctx, "k_fs_load");
}

int fri_challenge_dev(Ctx* ctx, cudaStream_t st, void* d_state, const uint8_t* d_root, uint8_t* d_root_out,
                      uint64_t* d_zeta) {
    k_fri_challenge<<<1, 32, 0, st>>>((fs::State*)d_state, d_root, d_root_out, d_zeta);
    return check_launch(ctx, "k_fri_challenge");
}

int fri_fold_dev(Ctx* ctx, cudaStream_t st, const uint64_t* d_in, uint64_t h, const uint64_t* d_inv_tw,
                 const uint64_t* d_zeta, uint64_t* d_out, uint64_t* d_inv_tw_next, uint8_t* d_leaves) {
    if (h == 0) return SG_OK;
    const uint64_t threads = (h + 1) / 2;
    k_fri_fold<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(d_in, h, d_inv_tw, 0, 0, 0, d_zeta, d_out,
                                                                  d_inv_tw_next, (uint64_t*)d_leaves);
    return check_launch(ctx, "k_fri_fold");
}

}  // namespace sg
