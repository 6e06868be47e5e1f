// Device-wide scans and a stable LSD radix sort of (key, value) pairs, the
// sorting primitives of the tree build (the stable dedup and superkey sorts
// of kdbuild.c:98-243 become radix sorts over the keys' varying bits) and of
// the counting layout.
//
// Scan: reduce-then-scan over tiles of kScanTile elements (tile totals, one
// block scans the totals, every tile scans itself from its offset).
// Sort: one pass per digit of up to 8 bits; per pass each tile counts its
// digits, a scan of the digit-major count table (digit 0 of every tile, then
// digit 1, ...) gives every (digit, tile) its output offset, and each tile
// scatters its keys in order: each warp owns a contiguous run of the tile's
// keys, the warps' digit counts are scanned in warp order, and within a
// round of 32 keys equal digits are ranked by lane, so equal keys keep their
// input order (stable).
//
// Temporary storage is the caller's (a Pool or a carved scratch array): the
// *_temp_bytes functions give its size.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace kd {
namespace sort {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

struct SumOp {
    template <class T> __device__ __forceinline__ T operator()(T a, T b) const { return a + b; }
    template <class T> __host__ __device__ static T identity() { return T(0); }
};
struct MaxOp {
    template <class T> __device__ __forceinline__ T operator()(T a, T b) const { return a > b ? a : b; }
    template <class T> __host__ __device__ static T identity()
    {
        return std::is_signed<T>::value ? (T)((unsigned long long)1 << (8 * sizeof(T) - 1)) : T(0);
    }
};

// Inclusive scan of one value per thread over the block (warp shuffles,
// then the scanned warp totals in sw); *total = the block's total.  sw stays
// valid until the next call.
template <class T, class Op>
__device__ __forceinline__ T block_incl_scan(T v, Op op, T *sw, T *total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const T u = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) v = op(u, v);
    }
    if (lane == 31) sw[w] = v;
    __syncthreads();
    if (w == 0) {
        T x = lane < nw ? sw[lane] : Op::template identity<T>();
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const T u = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x = op(u, x);
        }
        if (lane < nw) sw[lane] = x;
    }
    __syncthreads();
    if (w > 0) v = op(sw[w - 1], v);
    *total = sw[nw - 1];
    return v;
}

// Exclusive scan of one value per thread over the block.
template <class T, class Op>
__device__ __forceinline__ T block_excl_scan(T v, Op op, T *sw, T *total)
{
    const T inc = block_incl_scan<T>(v, op, sw, total);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T prev = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0) prev = w ? sw[w - 1] : Op::template identity<T>();
    __syncthreads();  // sw is rewritten by the next call
    return prev;
}

template <class T, class Op>
__global__ void __launch_bounds__(kScanThreads) k_tile_reduce(const T *in, long long n, T *tot, Op op)
{
    __shared__ T sw[kScanThreads / 32];
    const long long base = (long long)blockIdx.x * kScanTile;
    T acc = Op::template identity<T>();
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        const long long j = base + (long long)i * kScanThreads + threadIdx.x;
        if (j < n) acc = op(acc, in[j]);
    }
    T total;
    block_incl_scan<T>(acc, op, sw, &total);
    if (threadIdx.x == 0) tot[blockIdx.x] = total;
}

// exclusive scan of the tile totals, in place, by one block of 1024 threads
template <class T, class Op>
__global__ void __launch_bounds__(1024) k_scan_totals(T *tot, long long ntiles, Op op)
{
    __shared__ T sw[32];
    T carry = Op::template identity<T>();
    for (long long b = 0; b < ntiles; b += blockDim.x) {
        const long long j = b + threadIdx.x;
        const T v = j < ntiles ? tot[j] : Op::template identity<T>();
        T total;
        const T ex = block_excl_scan<T>(v, op, sw, &total);
        if (j < ntiles) tot[j] = op(carry, ex);
        carry = op(carry, total);
    }
}

// each tile scans itself from its offset; a thread owns kScanItems
// consecutive elements
template <class T, class Op, bool INCLUSIVE>
__global__ void __launch_bounds__(kScanThreads) k_tile_scan(const T *in, T *out, long long n,
                                                            const T *off, Op op)
{
    __shared__ T sw[kScanThreads / 32];
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    T v[kScanItems];
    T acc = Op::template identity<T>();
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        v[i] = base + i < n ? in[base + i] : Op::template identity<T>();
        acc = op(acc, v[i]);
    }
    T total;
    T run = op(off[blockIdx.x], block_excl_scan<T>(acc, op, sw, &total));
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        if (INCLUSIVE) {
            run = op(run, v[i]);
            if (base + i < n) out[base + i] = run;
        } else {
            if (base + i < n) out[base + i] = run;
            run = op(run, v[i]);
        }
    }
}

inline long long scan_tiles(long long n) { return n > 0 ? (n + kScanTile - 1) / kScanTile : 1; }

template <class T> inline size_t scan_temp_bytes(long long n)
{
    return sizeof(T) * (size_t)scan_tiles(n);
}

// out = scan of in (n elements; in and out may alias), temp of
// scan_temp_bytes<T>(n) bytes
template <class T, class Op, bool INCLUSIVE>
inline cudaError_t scan(void *temp, const T *in, T *out, long long n, Op op, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    const long long nt = scan_tiles(n);
    T *tot = (T *)temp;
    k_tile_reduce<T, Op><<<(unsigned)nt, kScanThreads, 0, s>>>(in, n, tot, op);
    k_scan_totals<T, Op><<<1, 1024, 0, s>>>(tot, nt, op);
    k_tile_scan<T, Op, INCLUSIVE><<<(unsigned)nt, kScanThreads, 0, s>>>(in, out, n, tot, op);
    return cudaGetLastError();
}

// ------------------------------------------------------------------- sort

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortRounds = 8;                       // rounds of 32 keys per warp
constexpr int kSortTile = kSortThreads * kSortRounds;  // keys per tile
constexpr int kRadixBits = 8;
constexpr int kBins = 1 << kRadixBits;

inline long long sort_tiles(long long n) { return n > 0 ? (n + kSortTile - 1) / kSortTile : 1; }

template <class K> __device__ __forceinline__ int digit_of(K k, int shift, int mask)
{
    return (int)((k >> shift) & (K)mask);
}

// counts[d * ntiles + tile]: keys of the tile with digit d
template <class K>
__global__ void __launch_bounds__(kSortThreads) k_digit_count(const K *keys, long long n, int shift,
                                                              int mask, unsigned *counts,
                                                              long long ntiles)
{
    __shared__ unsigned h[kBins];
    for (int d = threadIdx.x; d < kBins; d += blockDim.x) h[d] = 0;
    __syncthreads();
    const long long base = (long long)blockIdx.x * kSortTile;
    for (int i = threadIdx.x; i < kSortTile; i += blockDim.x) {
        const long long j = base + i;
        if (j < n) atomicAdd(&h[digit_of(keys[j], shift, mask)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d <= mask; d += blockDim.x)
        counts[(long long)d * ntiles + blockIdx.x] = h[d];
}

// Stable scatter of one tile to offsets[d * ntiles + tile] + rank.  The
// tile is first ordered by digit in shared memory (ranks from per-warp digit
// counts and warp matching of equal digits, as the tile's keys come: warp,
// then round, then lane), then written out in that order, so that each
// thread's consecutive stores of one digit land on consecutive addresses
// (runs of ~8 keys per digit per tile at 256 digits) instead of 32 scattered
// addresses per store instruction.
template <class K, class V>
__global__ void __launch_bounds__(kSortThreads) k_digit_scatter(const K *kin, K *kout, const V *vin,
                                                                V *vout, long long n, int shift,
                                                                int mask, const unsigned *offsets,
                                                                long long ntiles)
{
    __shared__ unsigned wc[kSortWarps][kBins];  // per-warp counts, then tile-local positions
    __shared__ unsigned tstart[kBins];          // first tile-local position of each digit
    __shared__ unsigned gofs[kBins];            // first output position of each digit
    __shared__ unsigned wsum[kSortWarps];
    __shared__ K skey[kSortTile];
    __shared__ V sval[kSortTile];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kSortWarps * kBins; i += blockDim.x) (&wc[0][0])[i] = 0;
    __syncthreads();
    // warp w owns keys [w * 32 * kSortRounds, (w + 1) * 32 * kSortRounds) of the tile
    const long long tbase = (long long)blockIdx.x * kSortTile;
    const long long base = tbase + (long long)w * 32 * kSortRounds;
    int dg[kSortRounds];
#pragma unroll
    for (int r = 0; r < kSortRounds; r++) {
        const long long j = base + r * 32 + lane;
        const bool v = j < n;
        dg[r] = v ? digit_of(kin[j], shift, mask) : -1;
        const unsigned act = __ballot_sync(0xffffffffu, v);
        if (v) {
            const unsigned peers = __match_any_sync(act, dg[r]);
            if (lane == __ffs(peers) - 1) wc[w][dg[r]] += __popc(peers);
        }
        __syncwarp();
    }
    __syncthreads();
    // digit totals of the tile, their exclusive scan (one digit per thread),
    // and each warp's first position within its digit
    static_assert(kBins == kSortThreads, "one digit per thread");
    {
        const int d = threadIdx.x;
        unsigned tot = 0;
#pragma unroll
        for (int k = 0; k < kSortWarps; k++) tot += wc[k][d];
        unsigned inc = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) wsum[w] = inc;
        __syncthreads();
        unsigned before = 0;
        for (int k = 0; k < w; k++) before += wsum[k];
        unsigned run = before + inc - tot;
        tstart[d] = run;
        gofs[d] = d <= mask ? offsets[(long long)d * ntiles + blockIdx.x] : 0u;
#pragma unroll
        for (int k = 0; k < kSortWarps; k++) {
            const unsigned c = wc[k][d];
            wc[k][d] = run;
            run += c;
        }
    }
    __syncthreads();
    // the tile in digit order, in shared memory
#pragma unroll
    for (int r = 0; r < kSortRounds; r++) {
        const long long j = base + r * 32 + lane;
        const bool v = dg[r] >= 0;
        const unsigned act = __ballot_sync(0xffffffffu, v);
        if (v) {
            const unsigned peers = __match_any_sync(act, dg[r]);
            const unsigned pos = wc[w][dg[r]] + __popc(peers & ((1u << lane) - 1u));
            skey[pos] = kin[j];
            sval[pos] = vin[j];
            __syncwarp(act);
            if (lane == __ffs(peers) - 1) wc[w][dg[r]] += __popc(peers);
        }
        __syncwarp();
    }
    __syncthreads();
    // written out in that order: consecutive positions of a digit go to
    // consecutive output addresses
    const long long left = n - tbase;
    const int cnt = left < kSortTile ? (int)left : kSortTile;
    for (int i = threadIdx.x; i < cnt; i += kSortThreads) {
        const K k = skey[i];
        const int d = digit_of(k, shift, mask);
        const unsigned dst = gofs[d] + ((unsigned)i - tstart[d]);
        kout[dst] = k;
        vout[dst] = sval[i];
    }
}

// temp bytes of sort_pairs for n keys: the digit count table, its scan's
// tile totals and one spare key/value buffer pair
template <class K, class V> inline size_t sort_temp_bytes(long long n)
{
    const long long ntiles = sort_tiles(n), nc = ntiles * kBins;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    return al(sizeof(unsigned) * (size_t)nc) + al(scan_temp_bytes<unsigned>(nc)) +
           al(sizeof(K) * (size_t)(n > 0 ? n : 1)) + al(sizeof(V) * (size_t)(n > 0 ? n : 1));
}

// Stable sort of n (key, value) pairs by key bits [b0, b1): kin/vin are
// read, kout/vout receive the result; temp of sort_temp_bytes<K, V>(n).
template <class K, class V>
inline cudaError_t sort_pairs(void *temp, const K *kin, K *kout, const V *vin, V *vout, long long n,
                              int b0, int b1, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    const long long ntiles = sort_tiles(n), nc = ntiles * kBins;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    char *t = (char *)temp;
    unsigned *counts = (unsigned *)t;
    t += al(sizeof(unsigned) * (size_t)nc);
    void *scan_tmp = t;
    t += al(scan_temp_bytes<unsigned>(nc));
    K *k2 = (K *)t;
    t += al(sizeof(K) * (size_t)n);
    V *v2 = (V *)t;
    const int npass = b1 > b0 ? (b1 - b0 + kRadixBits - 1) / kRadixBits : 0;
    if (npass == 0) {
        cudaError_t e = cudaMemcpyAsync(kout, kin, sizeof(K) * (size_t)n, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(vout, vin, sizeof(V) * (size_t)n, cudaMemcpyDeviceToDevice, s);
        return e;
    }
    // ping-pong so that the last pass writes kout/vout
    const K *ks = kin;
    const V *vs = vin;
    for (int p = 0; p < npass; p++) {
        const int shift = b0 + p * kRadixBits;
        const int bits = (b1 - shift) < kRadixBits ? (b1 - shift) : kRadixBits;
        const int mask = (1 << bits) - 1;
        const bool last = p == npass - 1;
        K *kd = ((npass - 1 - p) & 1) ? k2 : kout;
        V *vd = ((npass - 1 - p) & 1) ? v2 : vout;
        if (last) {
            kd = kout;
            vd = vout;
        }
        k_digit_count<K><<<(unsigned)ntiles, kSortThreads, 0, s>>>(ks, n, shift, mask, counts, ntiles);
        cudaError_t e = scan<unsigned, SumOp, false>(scan_tmp, counts, counts, (long long)(mask + 1) * ntiles,
                                                     SumOp(), s);
        if (e != cudaSuccess) return e;
        k_digit_scatter<K, V><<<(unsigned)ntiles, kSortThreads, 0, s>>>(ks, kd, vs, vd, n, shift, mask,
                                                                        counts, ntiles);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        ks = kd;
        vs = vd;
    }
    return cudaSuccess;
}

}  // namespace sort
}  // namespace kd
