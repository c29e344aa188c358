// Host-side check of the library's device guard (sg::enter in
// lambda_vm_b200/csrc/common.cuh) without a GPU: compiled with g++ against a
// fake CUDA runtime (fake_cuda/cuda_runtime.h) whose current device is
// per-thread, like the real one. A context made for device 3 is entered from
// fresh worker threads, which start on device 0 as CUDA threads do; each must
// end on device 3, and a thread already there must not switch again.
#include <stdio.h>

#include <atomic>
#include <thread>
#include <vector>

#include "../../lambda_vm_b200/csrc/common.cuh"

static thread_local int g_current = 0;  // a new CUDA host thread starts on device 0
static std::atomic<int> g_switches{0};
static const int kDevices = 4;

cudaError_t cudaGetDevice(int* device) {
    *device = g_current;
    return cudaSuccess;
}
cudaError_t cudaSetDevice(int device) {
    if (device < 0 || device >= kDevices) return cudaErrorInvalidDevice;
    g_current = device;
    g_switches.fetch_add(1);
    return cudaSuccess;
}
cudaError_t cudaGetLastError(void) { return cudaSuccess; }
const char* cudaGetErrorString(cudaError_t e) { return e == cudaSuccess ? "no error" : "invalid device ordinal"; }

namespace sg {
static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
const char* last_error() { return g_err.c_str(); }
}  // namespace sg

int main() {
    sg::Ctx ctx;
    ctx.device = 3;
    const int workers = 8;
    std::atomic<int> bad{0};
    std::vector<std::thread> ts;
    for (int w = 0; w < workers; ++w) {
        ts.emplace_back([&] {
            if (g_current != 0) bad.fetch_add(1);
            for (int call = 0; call < 5; ++call) {  // several entry points in a row
                if (sg::enter(&ctx) != SG_OK || g_current != 3) bad.fetch_add(1);
            }
        });
    }
    for (auto& t : ts) t.join();
    if (bad.load()) {
        printf("FAIL: %d worker calls did not run on the context's device\n", bad.load());
        return 1;
    }
    if (g_switches.load() != workers) {
        printf("FAIL: %d device switches for %d threads (one per thread expected)\n", g_switches.load(), workers);
        return 1;
    }
    sg::Ctx bad_ctx;
    bad_ctx.device = 9;  // no such device: the entry point reports it
    if (sg::enter(&bad_ctx) != SG_ERR_CUDA || std::string(sg::last_error()).find("cudaSetDevice(9)") == std::string::npos) {
        printf("FAIL: a missing device was not reported\n");
        return 1;
    }
    printf("ok\n");
    return 0;
}
