/*
 * fake_cuda.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Host stand-ins for the CUDA runtime calls that the model upload
 * (fn_upload, fibrenet_b200/csrc/fn_engine.cu) and context set-up make, so
 * the upload's host logic -- argument checks, bead ordering, conversions,
 * chain-form detection, the helper threads -- runs in the CPU test suite.
 * Force-included before fn_engine.cu in the test harness only: "device"
 * buffers become host memory, copies become memcpy, and no kernel runs (the
 * launchers are stubs in harness.cu).  The library itself never sees it.
 */
#pragma once
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>

static inline cudaError_t hu_ok() { return cudaSuccess; }
static inline cudaError_t hu_malloc(void** p, size_t n) {
    *p = std::malloc(n);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
static inline cudaError_t hu_free(void* p) {
    std::free(p);
    return cudaSuccess;
}
static inline cudaError_t hu_copy(void* d, const void* s, size_t n) {
    std::memcpy(d, s, n);
    return cudaSuccess;
}
static inline cudaError_t hu_set(void* d, int v, size_t n) {
    std::memset(d, v, n);
    return cudaSuccess;
}
static inline cudaError_t hu_count(int* n) {
    *n = 1;
    return cudaSuccess;
}
static inline cudaError_t hu_device(int* d) {
    *d = 0;
    return cudaSuccess;
}
static inline cudaError_t hu_attr(int* v) {
    *v = 227 * 1024; /* a B200's opt-in shared memory per block */
    return cudaSuccess;
}
static inline cudaError_t hu_pool(cudaMemPool_t* p) {
    static int token;
    *p = reinterpret_cast<cudaMemPool_t>(&token);
    return cudaSuccess;
}
static inline cudaError_t hu_stream(cudaStream_t* s) {
    *s = nullptr;
    return cudaSuccess;
}

#define cudaSetDevice(d) hu_ok()
#define cudaGetDeviceCount(n) hu_count(n)
#define cudaGetDevice(d) hu_device(d)
#define cudaDeviceGetAttribute(v, a, d) hu_attr(v)
#define cudaStreamCreateWithFlags(s, f) hu_stream(s)
#define cudaStreamSynchronize(s) hu_ok()
#define cudaStreamDestroy(s) hu_ok()
#define cudaEventDestroy(e) hu_ok()
#define cudaMalloc(p, n) hu_malloc((void**)(p), n)
#define cudaFree(p) hu_free((void*)(p))
#define cudaMallocAsync(p, n, st) hu_malloc((void**)(p), n)
#define cudaMallocFromPoolAsync(p, n, pl, st) hu_malloc((void**)(p), n)
#define cudaMemPoolCreate(pl, props) hu_pool(pl)
#define cudaMemPoolSetAttribute(pl, a, v) hu_ok()
#define cudaFreeAsync(p, st) hu_free((void*)(p))
#define cudaMemcpyAsync(d, s, n, k, st) hu_copy(d, s, n)
#define cudaMemcpy(d, s, n, k) hu_copy(d, s, n)
#define cudaMemsetAsync(d, v, n, st) hu_set(d, v, n)
