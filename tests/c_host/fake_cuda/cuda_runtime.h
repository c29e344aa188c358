/* A stand-in for cuda_runtime.h with just the declarations the library's
 * internal runtime header (lambda_vm_b200/csrc/common.cuh) uses, so its host
 * logic compiles with plain g++ and runs on a machine without a GPU. The test
 * that includes it defines these functions over a fake per-thread device. */
#pragma once
#include <stddef.h>

typedef enum {
    cudaSuccess = 0,
    cudaErrorMemoryAllocation = 2,
    cudaErrorInvalidDevice = 101,
} cudaError_t;
typedef void* cudaStream_t;
typedef void* cudaEvent_t;

cudaError_t cudaGetDevice(int* device);
cudaError_t cudaSetDevice(int device);
cudaError_t cudaGetLastError(void);
const char* cudaGetErrorString(cudaError_t e);
