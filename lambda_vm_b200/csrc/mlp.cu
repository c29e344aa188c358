// Learned cost model of the DFT passes: a small MLP trained on the GPU.
//
// The tile width of each DFT pass (columns per tile) is a runtime choice
// (ntt.cu). The timing probe that picks it measures every width on one proxy
// shape per pass length, which ranks widths unlike the real passes do for
// some shapes (narrow matrices, few tiles, the four-step passes). This file
// holds a model that predicts log(ms) of a pass from its shape and width,
// trained from the pass log (sg_ctx_pass_log) by the kernels below, and the
// host-side prediction the tile chooser uses once a model is installed.
//
// Network: SG_MLP_IN inputs -> H ReLU -> H ReLU -> 1 (H = SG_MLP_HIDDEN),
// fp32, parameters laid out W1[H][IN], b1[H], W2[H][H], b2[H], w3[H], b3.
// Loss: mean squared error over the batch. Gradients are formed per block of
// kSamplesPerBlock samples (per-sample activations staged in shared memory,
// each parameter's sum over the block's samples by one thread) and the block
// partials reduced in a fixed order, so a gradient is reproducible bit for
// bit. Adam (beta1 0.9, beta2 0.999, eps 1e-8) updates the parameters in place.
#include <math.h>

#include "common.cuh"

namespace sg {

constexpr int IN = SG_MLP_IN, H = SG_MLP_HIDDEN, NP = SG_MLP_PARAMS;
constexpr int OW1 = 0, OB1 = OW1 + H * IN, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H, OB3 = OW3 + H;
static_assert(OB3 + 1 == NP, "parameter layout");
constexpr int kSamplesPerBlock = 128;

// Per-sample forward pass: h1, h2 (post-ReLU) and the output.
template <typename P>
__host__ __device__ inline float mlp_forward(const P& p, const float* x, float* h1, float* h2) {
    for (int j = 0; j < H; ++j) {
        float s = p(OB1 + j);
        for (int i = 0; i < IN; ++i) s += p(OW1 + j * IN + i) * x[i];
        h1[j] = s > 0.f ? s : 0.f;
    }
    for (int k = 0; k < H; ++k) {
        float s = p(OB2 + k);
        for (int j = 0; j < H; ++j) s += p(OW2 + k * H + j) * h1[j];
        h2[k] = s > 0.f ? s : 0.f;
    }
    float y = p(OB3);
    for (int k = 0; k < H; ++k) y += p(OW3 + k) * h2[k];
    return y;
}

// Staged per sample in shared memory: x, h1, h2, e1 (dL/d pre-activation of
// layer 1), e2 (of layer 2), d (dL/dy).
constexpr int kRow = IN + 4 * H + 1;

__global__ void __launch_bounds__(kSamplesPerBlock) k_mlp_block_grad(const float* __restrict__ X,
                                                                     const float* __restrict__ Y, uint32_t n,
                                                                     const float* __restrict__ params,
                                                                     float* __restrict__ partial,
                                                                     float* __restrict__ loss_partial) {
    extern __shared__ float sm[];
    float* w = sm;                           // NP parameters
    float* rows = sm + NP;                   // kSamplesPerBlock x kRow
    for (int i = threadIdx.x; i < NP; i += blockDim.x) w[i] = params[i];
    __syncthreads();
    const uint32_t s = blockIdx.x * kSamplesPerBlock + threadIdx.x;
    float* r = rows + threadIdx.x * kRow;
    float* x = r;
    float* h1 = x + IN;
    float* h2 = h1 + H;
    float* e1 = h2 + H;
    float* e2 = e1 + H;
    float* d = e2 + H;
    float sq = 0.f;
    if (s < n) {
        for (int i = 0; i < IN; ++i) x[i] = X[(uint64_t)s * IN + i];
        auto P = [&](int i) { return w[i]; };
        const float y = mlp_forward(P, x, h1, h2);
        const float diff = y - Y[s];
        sq = diff * diff;
        const float g = 2.f * diff / (float)n;
        *d = g;
        for (int k = 0; k < H; ++k) e2[k] = h2[k] > 0.f ? g * w[OW3 + k] : 0.f;
        for (int j = 0; j < H; ++j) {
            float t = 0.f;
            for (int k = 0; k < H; ++k) t += w[OW2 + k * H + j] * e2[k];
            e1[j] = h1[j] > 0.f ? t : 0.f;
        }
    } else {
        for (int i = 0; i < kRow; ++i) r[i] = 0.f;
    }
    __syncthreads();
    // Each thread sums some parameters' gradients over the block's samples, in sample order.
    for (int p = threadIdx.x; p < NP; p += blockDim.x) {
        float acc = 0.f;
        for (int t = 0; t < kSamplesPerBlock; ++t) {
            const float* q = rows + t * kRow;
            const float *qx = q, *qh1 = q + IN, *qh2 = qh1 + H, *qe1 = qh2 + H, *qe2 = qe1 + H, qd = q[kRow - 1];
            float v;
            if (p < OB1) v = qe1[(p - OW1) / IN] * qx[(p - OW1) % IN];
            else if (p < OW2) v = qe1[p - OB1];
            else if (p < OB2) v = qe2[(p - OW2) / H] * qh1[(p - OW2) % H];
            else if (p < OW3) v = qe2[p - OB2];
            else if (p < OB3) v = qd * qh2[p - OW3];
            else v = qd;
            acc += v;
        }
        partial[(uint64_t)blockIdx.x * NP + p] = acc;
    }
    // block loss partial: a fixed-order tree over the threads' squared errors
    __shared__ float red[kSamplesPerBlock];
    red[threadIdx.x] = sq;
    __syncthreads();
    for (int off = kSamplesPerBlock / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss_partial[blockIdx.x] = red[0];
}

// grad[p] = sum over blocks of partial[b][p], blocks in order; loss likewise / n.
__global__ void k_mlp_reduce(const float* __restrict__ partial, const float* __restrict__ loss_partial,
                             uint32_t blocks, uint32_t n, float* __restrict__ grad, float* __restrict__ loss) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < NP) {
        float acc = 0.f;
        for (uint32_t b = 0; b < blocks; ++b) acc += partial[(uint64_t)b * NP + p];
        grad[p] = acc;
    }
    if (p == 0 && loss) {
        float acc = 0.f;
        for (uint32_t b = 0; b < blocks; ++b) acc += loss_partial[b];
        *loss = acc / (float)n;
    }
}

__global__ void k_mlp_adam(float* __restrict__ params, const float* __restrict__ grad, float* __restrict__ m1,
                           float* __restrict__ m2, float lr, float c1, float c2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NP) return;
    const float g = grad[p];
    const float a = 0.9f * m1[p] + 0.1f * g;
    const float b = 0.999f * m2[p] + 0.001f * g * g;
    m1[p] = a;
    m2[p] = b;
    params[p] -= lr * (a / c1) / (sqrtf(b / c2) + 1e-8f);
}

__global__ void k_mlp_predict(const float* __restrict__ X, uint32_t n, const float* __restrict__ params,
                              float* __restrict__ out) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float x[IN], h1[H], h2[H];
    for (int i = 0; i < IN; ++i) x[i] = X[(uint64_t)s * IN + i];
    auto P = [&](int i) { return __ldg(params + i); };
    out[s] = mlp_forward(P, x, h1, h2);
}

static int loss_grad(Ctx* ctx, cudaStream_t st, const float* X, const float* Y, uint32_t n, const float* params,
                     float* grad, float* loss, float* partial, float* loss_partial) {
    const uint32_t blocks = (n + kSamplesPerBlock - 1) / kSamplesPerBlock;
    const size_t smem = (size_t)(NP + kSamplesPerBlock * kRow) * sizeof(float);
    KernelInfo ki;
    SG_TRY(kernel_info((const void*)k_mlp_block_grad, smem, kSamplesPerBlock, &ki));
    k_mlp_block_grad<<<blocks, kSamplesPerBlock, smem, st>>>(X, Y, n, params, partial, loss_partial);
    SG_TRY(check_launch(ctx, "k_mlp_block_grad"));
    k_mlp_reduce<<<(NP + 255) / 256, 256, 0, st>>>(partial, loss_partial, blocks, n, grad, loss);
    return check_launch(ctx, "k_mlp_reduce");
}

float mlp_predict_host(const float* params, const float* x) {
    float h1[H], h2[H];
    auto P = [&](int i) { return params[i]; };
    return mlp_forward(P, x, h1, h2);
}

}  // namespace sg

using namespace sg;

extern "C" {

void sg_pass_features(uint32_t log_len, uint64_t tiles, uint64_t m, uint32_t cols, uint32_t reps, uint32_t inverse,
                      uint32_t pre, uint32_t post, uint32_t canon, float out[SG_MLP_IN]) {
    const double ct = cols ? (double)((m + cols - 1) / cols) : 1.0;
    const double padded = ct * (double)cols;
    const double mm = m ? (double)m : 1.0;
    const double work = (double)tiles * (double)(1ull << log_len) * padded * (double)(reps ? reps : 1);
    out[0] = (float)(((double)log_len - 8.0) / 3.0);
    out[1] = (float)(log2((double)(tiles ? tiles : 1)) / 14.0);
    out[2] = (float)(log2(mm) / 9.0);
    out[3] = cols == 4 ? 1.f : 0.f;
    out[4] = cols == 8 ? 1.f : 0.f;
    out[5] = cols == 16 ? 1.f : 0.f;
    out[6] = (float)(log2(ct) / 7.0);
    out[7] = (float)(padded / mm - 1.0);
    out[8] = (float)(log2((double)(reps ? reps : 1)) / 3.0);
    out[9] = inverse ? 1.f : 0.f;
    out[10] = pre ? 1.f : 0.f;
    out[11] = post == 1 ? 1.f : 0.f;
    out[12] = post == 2 ? 1.f : 0.f;
    out[13] = post == 3 ? 1.f : 0.f;
    out[14] = canon ? 1.f : 0.f;
    out[15] = (float)(log2(work > 1.0 ? work : 1.0) / 32.0);
}

int sg_mlp_loss_grad(sg_ctx* c, void* stream, const float* d_x, const float* d_y, uint32_t n, const float* d_params,
                     float* d_grad, float* d_loss) {
    SG_CHECK_ARG(c && d_x && d_y && d_params && d_grad && n > 0, "null argument or empty batch");
    SG_ENTER(ctx_of(c));
    Ctx* ctx = ctx_of(c);
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t blocks = (n + kSamplesPerBlock - 1) / kSamplesPerBlock;
    float *partial = nullptr, *lp = nullptr;
    SG_TRY(dev_alloc(ctx, st, (uint64_t)blocks * NP * 4, (void**)&partial));
    int rc = dev_alloc(ctx, st, (uint64_t)blocks * 4, (void**)&lp);
    if (rc == SG_OK) rc = loss_grad(ctx, st, d_x, d_y, n, d_params, d_grad, d_loss, partial, lp);
    dev_free(ctx, st, partial, (uint64_t)blocks * NP * 4);
    dev_free(ctx, st, lp, (uint64_t)blocks * 4);
    return rc;
}

int sg_mlp_train(sg_ctx* c, void* stream, const float* d_x, const float* d_y, uint32_t n, float* d_params,
                 uint32_t steps, float lr, float* loss_out) {
    SG_CHECK_ARG(c && d_x && d_y && d_params && n > 0, "null argument or empty batch");
    SG_ENTER(ctx_of(c));
    Ctx* ctx = ctx_of(c);
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t blocks = (n + kSamplesPerBlock - 1) / kSamplesPerBlock;
    // scratch: block partials, loss partials, gradient, Adam moments, loss
    const uint64_t words = (uint64_t)blocks * NP + blocks + 3ull * NP + 1;
    float* mem = nullptr;
    SG_TRY(dev_alloc(ctx, st, words * 4, (void**)&mem));
    float* partial = mem;
    float* lp = partial + (uint64_t)blocks * NP;
    float* grad = lp + blocks;
    float* m1 = grad + NP;
    float* m2 = m1 + NP;
    float* loss = m2 + NP;
    int rc = SG_OK;
    if (cudaMemsetAsync(m1, 0, 2ull * NP * 4, st) != cudaSuccess) {
        set_error("mlp train: memset failed");
        rc = SG_ERR_CUDA;
    }
    double b1t = 1.0, b2t = 1.0;
    for (uint32_t t = 0; t < steps && rc == SG_OK; ++t) {
        rc = loss_grad(ctx, st, d_x, d_y, n, d_params, grad, nullptr, partial, lp);
        if (rc != SG_OK) break;
        b1t *= 0.9, b2t *= 0.999;
        k_mlp_adam<<<(NP + 255) / 256, 256, 0, st>>>(d_params, grad, m1, m2, lr, (float)(1.0 - b1t),
                                                      (float)(1.0 - b2t));
        rc = check_launch(ctx, "k_mlp_adam");
    }
    if (rc == SG_OK) rc = loss_grad(ctx, st, d_x, d_y, n, d_params, grad, loss, partial, lp);
    if (rc == SG_OK && loss_out) {
        cudaError_t e = cudaMemcpyAsync(loss_out, loss, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            set_error(std::string("mlp train: ") + cudaGetErrorString(e));
            rc = SG_ERR_CUDA;
        }
    }
    dev_free(ctx, st, mem, words * 4);
    return rc;
}

int sg_mlp_predict(sg_ctx* c, void* stream, const float* d_x, uint32_t n, const float* d_params, float* d_out) {
    SG_CHECK_ARG(c && d_x && d_params && d_out, "null argument");
    SG_ENTER(ctx_of(c));
    if (n == 0) return SG_OK;
    k_mlp_predict<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(d_x, n, d_params, d_out);
    return check_launch(ctx_of(c), "k_mlp_predict");
}

int sg_ctx_set_pass_model(sg_ctx* c, const float* params, uint32_t count) {
    SG_CHECK_ARG(c, "null context");
    SG_CHECK_ARG(count == 0 || (params && count == (uint32_t)NP), "a pass model has SG_MLP_PARAMS parameters");
    Ctx* ctx = ctx_of(c);
    std::lock_guard<std::mutex> g(ctx->tune_mu);
    if (count == 0)
        ctx->pass_model.clear();
    else
        ctx->pass_model.assign(params, params + count);
    return SG_OK;
}

}  // extern "C"
