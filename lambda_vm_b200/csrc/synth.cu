// Deterministic synthetic chip-table traces generated on the device, for the
// multi-table proving benchmarks (seeded synthetic inputs stand in for VM
// traces). Element (r, c) of a table with seed s is a splitmix64 draw on the
// counter r*w + c, reduced to [0, p); the multiplicity column keeps 16 bits;
// the checksum column is sum_{j<k} c_j(r) c_j(r+1 mod n). The host generator
// in lambda_vm_b200/air.py computes the identical values.
#include "common.cuh"
#include "gl.cuh"

namespace sg {

__device__ __host__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__global__ void k_synth_values(uint64_t* out, uint64_t n, uint64_t w, uint64_t key, uint64_t mult_col) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n * w) return;
    const uint64_t c = g % w;
    uint64_t v = splitmix64(key + g);
    if (c == mult_col)
        v &= 0xFFFFULL;
    else
        v = v >= GL_P ? v - GL_P : v;
    out[g] = v;
}

__global__ void k_synth_checksum(uint64_t* t, uint64_t n, uint64_t w, uint32_t k, uint64_t sum_col) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint64_t rn = r + 1 == n ? 0 : r + 1;
    uint64_t s = 0;
    for (uint32_t j = 0; j < k; ++j) s = gl::add(s, gl::mul(t[r * w + j], t[rn * w + j]));
    t[r * w + sum_col] = gl::canon(s);
}

}  // namespace sg

using namespace sg;

extern "C" int sg_synth_trace(sg_ctx* c, void* stream, uint64_t* d_out, uint64_t n, uint64_t w, uint64_t seed,
                              uint32_t k_checksum) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    SG_CHECK_ARG(ctx && d_out, "null argument");
    SG_ENTER(ctx);
    SG_CHECK_ARG(w >= 3 && k_checksum <= w - 2, "width must be >= 3 and k <= width - 2");
    if (n == 0) return SG_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t key = splitmix64(seed);
    const uint64_t tot = n * w;
    k_synth_values<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(d_out, n, w, key, w - 2);
    SG_TRY(check_launch(ctx, "k_synth_values"));
    k_synth_checksum<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_out, n, w, k_checksum, w - 1);
    return check_launch(ctx, "k_synth_checksum");
}
