// Small CUDA helpers shared by the build and count translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <cstring>
#include <mutex>
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

// Stream-ordered memory pools of their own, per device, beside the default
// pool that every other build and count array comes from (its release
// threshold raised, like the default pool's):
//   kPoolNodes   the node arrays that builds copy to the host.  A node array
//                still being copied while a count runs (deferred builds)
//                would otherwise sit inside a cached block of the default
//                pool that the count's tile-record buffer could have reused.
//   kPoolRecords the counts' tile-record buffers (gigabytes, one per count
//                in flight).  In the default pool, the catalogs and build
//                temporaries of many trees fragment the cached memory, and a
//                count whose record buffer finds no cached block large enough
//                makes the pool map new memory (hundreds of ms for 10 GB).
// Either falls back to the default pool where a pool cannot be made.
enum { kPoolNodes = 0, kPoolRecords = 1 };
inline cudaMemPool_t side_pool(int which)
{
    static std::mutex mu;
    static cudaMemPool_t pools[2][64] = {};
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    cudaMemPool_t def = nullptr;
    if (dev < 0 || dev >= 64 || which < 0 || which > 1) {
        check(cudaDeviceGetDefaultMemPool(&def, dev), "cudaDeviceGetDefaultMemPool");
        return def;
    }
    std::lock_guard<std::mutex> g(mu);
    if (!pools[which][dev]) {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof props);
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
            cudaGetLastError();
            check(cudaDeviceGetDefaultMemPool(&def, dev), "cudaDeviceGetDefaultMemPool");
            return def;
        }
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &thr);
        pools[which][dev] = p;
    }
    return pools[which][dev];
}

// Device memory a pool holds but has not handed out (reusable at once).
inline size_t pool_idle_bytes(cudaMemPool_t p)
{
    uint64_t reserved = 0, used = 0;
    if (cudaMemPoolGetAttribute(p, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess ||
        cudaMemPoolGetAttribute(p, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return reserved > used ? (size_t)(reserved - used) : 0;
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
