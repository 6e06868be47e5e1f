// Small CUDA helpers shared by the build and count translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <vector>

#include "kd_internal.h"

namespace kd {

struct Error {
    int code;
    char msg[200];
};

[[noreturn]] inline void raise(int code, const char *what, cudaError_t e = cudaSuccess)
{
    Error err;
    err.code = code;
    if (e != cudaSuccess)
        snprintf(err.msg, sizeof err.msg, "%s: %s", what, cudaGetErrorString(e));
    else
        snprintf(err.msg, sizeof err.msg, "%s", what);
    throw err;
}

inline void check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) raise(e == cudaErrorMemoryAllocation ? KD_ENOMEM : KD_ECUDA, what, e);
}

// Stream-ordered allocations owned by one call; anything not released to a
// longer-lived owner is freed when the call ends.
struct Pool {
    cudaStream_t s;
    std::vector<void *> ptrs;
    size_t bytes = 0;
    explicit Pool(cudaStream_t st) : s(st) {}
    template <class T> T *alloc(size_t n)
    {
        void *p = nullptr;
        size_t b = (n ? n : 1) * sizeof(T);
        cudaError_t e = cudaMallocAsync(&p, b, s);
        if (e != cudaSuccess) {
            cudaGetLastError();
            raise(KD_ENOMEM, "device allocation failed", e);
        }
        ptrs.push_back(p);
        bytes += b;
        return (T *)p;
    }
    // n elements from a given memory pool (stream-ordered like alloc)
    template <class T> T *alloc_from(cudaMemPool_t mp, size_t n)
    {
        void *p = nullptr;
        size_t b = (n ? n : 1) * sizeof(T);
        cudaError_t e = cudaMallocFromPoolAsync(&p, b, mp, s);
        if (e != cudaSuccess) {
            cudaGetLastError();
            raise(KD_ENOMEM, "device allocation failed", e);
        }
        ptrs.push_back(p);
        bytes += b;
        return (T *)p;
    }
    // hand ownership of p to the caller (it will not be freed by ~Pool)
    template <class T> T *keep(T *p)
    {
        for (auto &q : ptrs)
            if (q == (void *)p) q = nullptr;
        return p;
    }
    ~Pool()
    {
        for (void *p : ptrs)
            if (p) cudaFreeAsync(p, s);
    }
};

// One non-blocking stream per API call: calls on different threads do not
// serialise on each other's work.
struct Stream {
    cudaStream_t s = nullptr;
    Stream() { check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate"); }
    ~Stream()
    {
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    }
    void sync() { check(cudaStreamSynchronize(s), "kernel execution"); }
};

// Keep freed device memory cached in the stream-ordered pool so repeated
// builds and counts do not pay for fresh allocations.
void init_device();

inline unsigned blocks_for(long long n, int threads)
{
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 0x7fffffff) b = 0x7fffffff;
    return (unsigned)b;
}

#define KD_LAUNCH_CHECK(what) ::kd::check(cudaGetLastError(), what)

}  // namespace kd
