// GPU tree build for corruscant's tree_construct (kdbuild.c:451-537).
//
// Produces, on the device, the same node array and in-order permutation the
// reference's recursive presort-median build produces (semantic fields:
// coordinates, field, weight, has_lchild, has_rchild, dim), and from that tree
// the counting layout used by kd_count.cu (see kd_internal.h).
//
// Reference semantics reproduced (kdbuild.c line numbers):
//   dedup            : stable lexicographic (x,y,z) sort with '==' compares
//                      (so -0.0 == +0.0), first occurrence keeps its field,
//                      weight = run length, >= 256 copies is an error
//                      (:82-96, :98-152, :479-511)
//   argsorts         : the three cyclic superkey orders of the unique points
//                      (:59-80, :158-243)
//   median           : (l+r+1)/2, rounding right (:52-55)
//   split dimension  : max_variance_dim over subtrees of 4+ points: per
//                      dimension a sequential sum in that dimension's superkey
//                      order, mean by division, sequential fused
//                      multiply-add sum of squared deviations, first strict
//                      maximum wins (:308-351, :383-386)
//   partition        : stable split of the other orders around the median
//                      (:251-291)
//   base cases       : sizes 1, 2, 3 taken from the superkey-0 order (:402-418)
//   heap layout      : root 1, children 2p and 2p+1, memsize = pow2ceil (:435-449)
//
// GPU formulation (not the reference's recursion): all subtrees of one depth
// are processed together.  Positions of the three superkey-ordered index arrays
// are grouped in contiguous segments, one per subtree.  A level computes every
// segment's split dimension, writes the level's nodes, then moves every
// position to its child segment with a stable segmented partition (two global
// prefix sums packed into one 64-bit scan).  Split dimensions of large
// segments come from a parallel variance with a rigorous error interval around
// the value the reference's sequential sums produce; only when the intervals of
// the best and another dimension overlap is the sequential computation run.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <exception>
#include <memory>
#include <new>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "kd_cuda_util.cuh"
#include "kd_sort.cuh"

namespace kd {

struct alignas(8) NodeRec {
    double v[3];
    uint32_t fw;    // field:8 | weight:8 << 8  (kdtree.h:15-16)
    uint32_t pad0;
    uint32_t flags; // has_lchild:1 | has_rchild:1 << 1 | dim:8 << 2 (kdtree.h:21-24)
    uint32_t pad1;
};
static_assert(sizeof(NodeRec) == 40, "node_t is 40 bytes");

// Segments up to this size get the exact sequential variance directly;
// larger ones first try the parallel sums with a rigorous interval (one
// thread walking thousands of gathered points is slow: ~1 us per point).
constexpr int kSmallSeg = 256;
// Positions per block in the parallel variance kernels (<= kSmallSeg + 1 so a
// block touches at most two segments).
constexpr int kVarChunk = 256;   // positions per k_var_par block
constexpr int kVarThreads = 64;  // threads per k_var_par block (4 positions each)

// Once per device (any thread may get here first; doing it twice is harmless):
// keep freed stream-ordered allocations in the device's pool instead of
// returning them to the driver at every synchronisation.
void init_device()
{
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0;
    if (bit && (done.load() & bit)) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    cudaGetLastError();
    done.fetch_or(bit);
}

// Order-preserving 64-bit key of a double; -0.0 maps to +0.0's key so that
// key equality is C '==' equality for non-NaN values.
__device__ __forceinline__ uint64_t okey(double v)
{
    if (v == 0.0) v = 0.0;
    uint64_t b = (uint64_t)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__device__ __forceinline__ void set_err(int *err, int code) { atomicCAS(err, 0, code); }

// ------------------------------------------------------------ dedup stage

__global__ void k_prep(const double *__restrict__ xyz, int n, uint64_t *kx, uint64_t *ky,
                       uint64_t *kz, int *iota, int *err, unsigned long long *maxabs)
{
    unsigned long long m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double x = xyz[3 * (size_t)i], y = xyz[3 * (size_t)i + 1], z = xyz[3 * (size_t)i + 2];
        if (isnan(x) || isnan(y) || isnan(z)) set_err(err, KD_ENAN);
        kx[i] = okey(x);
        ky[i] = okey(y);
        kz[i] = okey(z);
        iota[i] = i;
        unsigned long long a = (unsigned long long)__double_as_longlong(fabs(x));
        unsigned long long b = (unsigned long long)__double_as_longlong(fabs(y));
        unsigned long long c = (unsigned long long)__double_as_longlong(fabs(z));
        m = max(m, max(a, max(b, c)));
    }
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxabs, m);
}

// OR of (k_i xor k_0) for each key array: the bits that actually vary.
__global__ void k_keyvary(const uint64_t *kx, const uint64_t *ky, const uint64_t *kz, int n,
                          unsigned long long *vary)
{
    uint64_t ax = 0, ay = 0, az = 0;
    uint64_t x0 = kx[0], y0 = ky[0], z0 = kz[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        ax |= kx[i] ^ x0;
        ay |= ky[i] ^ y0;
        az |= kz[i] ^ z0;
    }
    for (int o = 16; o; o >>= 1) {
        ax |= __shfl_xor_sync(0xffffffffu, ax, o);
        ay |= __shfl_xor_sync(0xffffffffu, ay, o);
        az |= __shfl_xor_sync(0xffffffffu, az, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicOr(vary + 0, (unsigned long long)ax);
        atomicOr(vary + 1, (unsigned long long)ay);
        atomicOr(vary + 2, (unsigned long long)az);
    }
}

__global__ void k_gather_u64(const uint64_t *__restrict__ src, const int *__restrict__ idx, int n,
                             uint64_t *dst)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = src[idx[i]];
}

__global__ void k_heads(const int *__restrict__ p, const uint64_t *kx, const uint64_t *ky,
                        const uint64_t *kz, int n, int *head)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int h = 1;
        if (i > 0) {
            int a = p[i], b = p[i - 1];
            h = (kx[a] != kx[b]) | (ky[a] != ky[b]) | (kz[a] != kz[b]);
        }
        head[i] = h;
    }
}

struct UniqueArrays {
    double *ux, *uy, *uz;
    int *ufield, *uw, *urep, *uhead;
    uint64_t *ukx, *uky, *ukz;
};

// cls[i] = 1-based class number of dedup-sorted position i
__global__ void k_unique(const int *__restrict__ p, const int *__restrict__ head,
                         const int *__restrict__ cls, int n, const double *__restrict__ xyz,
                         const int *__restrict__ fin, const uint64_t *kx, const uint64_t *ky,
                         const uint64_t *kz, UniqueArrays u, int n_u)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!head[i]) continue;
        int c = cls[i] - 1, r = p[i];
        u.ux[c] = xyz[3 * (size_t)r];
        u.uy[c] = xyz[3 * (size_t)r + 1];
        u.uz[c] = xyz[3 * (size_t)r + 2];
        u.ufield[c] = fin ? (fin[r] & 0xFF) : 0;
        u.urep[c] = r;
        u.uhead[c] = i;
        u.ukx[c] = kx[r];
        u.uky[c] = ky[r];
        u.ukz[c] = kz[r];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) u.uhead[n_u] = n;
}

struct FieldInfo {
    int min_qf, max_qf, max_tf, split;
};

__global__ void k_weights(UniqueArrays u, int n_u, const int *__restrict__ p,
                          const int *__restrict__ cls, const int *__restrict__ fin, int n,
                          int heavy_ok, int *err, FieldInfo *fi)
{
    int maxtf = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n_u; c += gridDim.x * blockDim.x) {
        int w = u.uhead[c + 1] - u.uhead[c];
        u.uw[c] = w;
        if (w > 255 && !heavy_ok) set_err(err, KD_EDUP);
        maxtf = max(maxtf, u.ufield[c]);
    }
    int minq = 0x7fffffff, maxq = -0x7fffffff, split = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int qf = fin ? fin[p[i]] : 0;
        int tf = u.ufield[cls[i] - 1];
        minq = min(minq, qf);
        maxq = max(maxq, qf);
        split |= (qf != tf);
    }
    for (int o = 16; o; o >>= 1) {
        maxtf = max(maxtf, __shfl_xor_sync(0xffffffffu, maxtf, o));
        minq = min(minq, __shfl_xor_sync(0xffffffffu, minq, o));
        maxq = max(maxq, __shfl_xor_sync(0xffffffffu, maxq, o));
        split |= __shfl_xor_sync(0xffffffffu, split, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&fi->max_tf, maxtf);
        atomicMin(&fi->min_qf, minq);
        atomicMax(&fi->max_qf, maxq);
        atomicOr(&fi->split, split);
    }
}

// ------------------------------------------------------------ level loop

struct Segs {
    int *p, *l, *r;   // heap id and in-order range of each segment
    int *count;       // device count
};

struct LevelBufs {
    int *tdim;
    unsigned char *big, *fallback;
    double *acc;      // per big segment: S0 S1 S2 A0 A1 A2 V0 V1 V2
    int cap_big;
    int *rank;        // exclusive scan of "has children"
    int *haskids;
};

__global__ void k_seg_setup(Segs sg, int ub, LevelBufs lb)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ub) return;
    int ns = *sg.count;
    if (s >= ns) {
        lb.haskids[s] = 0;
        return;
    }
    int size = sg.r[s] - sg.l[s] + 1;
    int big = size > kSmallSeg && s < lb.cap_big;
    lb.big[s] = (unsigned char)big;
    lb.fallback[s] = 0;
    lb.tdim[s] = 0;
    lb.haskids[s] = size >= 4;
    if (big)
        for (int k = 0; k < 9; k++) lb.acc[9 * (size_t)s + k] = 0.0;
}

// Parallel sums for big segments: pass 0 accumulates S_j = sum v_j and
// A_j = sum |v_j|; pass 1 accumulates V_j = sum (v_j - S_j/n)^2.
// c0, c1, c2: the x of the point at each position of superkey order 0, the
// y along order 1, the z along order 2 (carried through the partitions), so
// a segment's coordinates are read contiguously; the parallel sums do not
// depend on the order within a segment
template <int PASS>
__global__ void __launch_bounds__(kVarThreads) k_var_par(int n_u, const int *__restrict__ pos_seg,
                                                         Segs sg, LevelBufs lb,
                                                         const double *__restrict__ c0,
                                                         const double *__restrict__ c1,
                                                         const double *__restrict__ c2)
{
    // pass 0: S0 S1 S2 A0 A1 A2; pass 1: V0 V1 V2
    constexpr int NV = PASS == 0 ? 6 : 3;
    constexpr int PER = kVarChunk / kVarThreads;
    constexpr int NW = kVarThreads / 32;
    __shared__ double wsum[NW][2][NV];
    __shared__ double mu_sh[2][3];
    __shared__ int wmin[NW];
    const int base = blockIdx.x * kVarChunk;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int seg[PER];
    int smin = 0x7fffffff;
#pragma unroll
    for (int k = 0; k < PER; k++) {
        const int i = base + threadIdx.x + kVarThreads * k;
        seg[k] = -1;
        if (i < n_u) {
            const int s = pos_seg[i];
            if (s >= 0 && lb.big[s]) {
                seg[k] = s;
                smin = min(smin, s);
            }
        }
    }
    smin = __reduce_min_sync(0xffffffffu, smin);
    if (lane == 0) wmin[w] = smin;
    __syncthreads();
    int s0 = wmin[0];
#pragma unroll
    for (int q = 1; q < NW; q++) s0 = min(s0, wmin[q]);
    if (s0 == 0x7fffffff) return;
    if (PASS == 1) {  // the means of the chunk's first two segments, once
        if (threadIdx.x < 6) {
            const int q = threadIdx.x / 3, j = threadIdx.x % 3, sq = s0 + q;
            mu_sh[q][j] = sq < *sg.count
                              ? lb.acc[9 * (size_t)sq + j] / (double)(sg.r[sq] - sg.l[sq] + 1)
                              : 0.0;
        }
        __syncthreads();
    }
    double a[2][NV];
#pragma unroll
    for (int q = 0; q < 2; q++)
#pragma unroll
        for (int j = 0; j < NV; j++) a[q][j] = 0.0;
    bool second = false;
#pragma unroll
    for (int k = 0; k < PER; k++) {
        const int s = seg[k];
        if (s < 0) continue;
        const int i = base + threadIdx.x + kVarThreads * k;
        const double v[3] = {c0[i], c1[i], c2[i]};
        double c[NV];
        const int slot = s - s0;
        if (PASS == 0) {
#pragma unroll
            for (int j = 0; j < 3; j++) {
                c[j] = v[j];
                c[3 + j] = fabs(v[j]);
            }
        } else {
            const double n = (double)(sg.r[s] - sg.l[s] + 1);
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const double mu = slot < 2 ? mu_sh[slot][j] : lb.acc[9 * (size_t)s + j] / n;
                const double d = v[j] - mu;
                c[j] = d * d;
            }
        }
        if (slot == 0) {
#pragma unroll
            for (int j = 0; j < NV; j++) a[0][j] += c[j];
        } else if (slot == 1) {
            second = true;
#pragma unroll
            for (int j = 0; j < NV; j++) a[1][j] += c[j];
        } else {  // a third segment in one chunk: segments this small are rare
#pragma unroll
            for (int j = 0; j < NV; j++)
                atomicAdd(&lb.acc[9 * (size_t)s + (PASS == 0 ? 0 : 6) + j], c[j]);
        }
    }
    // warp sums; the second segment's only where a lane of the warp holds one
    const bool two = __any_sync(0xffffffffu, second);
#pragma unroll
    for (int q = 0; q < 2; q++) {
        if (q == 1 && !two) {
            if (lane < NV) wsum[w][1][lane] = 0.0;
            break;
        }
#pragma unroll
        for (int j = 0; j < NV; j++) {
            double v = a[q][j];
#pragma unroll
            for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) wsum[w][q][j] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x < 2 * NV) {
        const int q = threadIdx.x / NV, j = threadIdx.x % NV, s = s0 + q;
        double v = wsum[0][q][j];
#pragma unroll
        for (int x = 1; x < NW; x++) v += wsum[x][q][j];
        if (v != 0.0 && s < *sg.count && lb.big[s])
            atomicAdd(&lb.acc[9 * (size_t)s + (PASS == 0 ? 0 : 6) + j], v);
    }
}

__device__ __forceinline__ double gam(double m)
{
    const double u = 1.1102230246251565e-16;  // 2^-53
    return m * u / (1.0 - m * u);
}

// Decide the split dimension of a big segment from rigorous intervals around
// the reference's rounded variances, or mark it for the sequential fallback.
__global__ void k_var_decide(Segs sg, int ub, LevelBufs lb)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ub || s >= *sg.count || !lb.big[s]) return;
    const double u = 1.1102230246251565e-16;
    double n = (double)(sg.r[s] - sg.l[s] + 1);
    const double *a = lb.acc + 9 * (size_t)s;
    double lo[3], hi[3];
    for (int j = 0; j < 3; j++) {
        double A = a[3 + j] * (1.0 + gam(n));
        double dmu = (gam(n - 1) * (1.0 + u) + u) * A / n * (1.0 + 4 * u);
        double V = a[6 + j];
        double nd2 = n * dmu * dmu * (1.0 + 4 * u);
        double l = V / (1.0 + gam(n + 2)) - nd2;
        if (l < 0) l = 0;
        lo[j] = (1.0 - gam(n + 1)) * (1.0 - u) * (1.0 - u) * l * (1.0 - 1e-14);
        hi[j] = (1.0 + gam(n + 1)) * (1.0 + u) * (1.0 + u) * (V / (1.0 - gam(n + 2)) + nd2) *
                (1.0 + 1e-14);
    }
    int c = 0;
    if (a[7] > a[6 + c]) c = 1;
    if (a[8] > a[6 + c]) c = 2;
    bool ok = true;
    for (int j = 0; j < 3; j++)
        if (j != c && !(lo[c] > hi[j])) ok = false;
    if (ok) lb.tdim[s] = c;
    else lb.fallback[s] = 1;
}

// max_variance_dim exactly as the reference evaluates it (kdbuild.c:308-351),
// one thread per segment; the three dimensions' chains are independent and
// are interleaved for latency hiding without changing any chain's order.
// c0, c1, c2 as for k_var_par: c_j[i] is coordinate j of the point at
// position i of superkey order j, so the sums below run over exactly the
// values, in exactly the order, of the reference's loops over args[j]
__global__ void k_var_seq(Segs sg, int ub, LevelBufs lb, const double *__restrict__ c0,
                          const double *__restrict__ c1, const double *__restrict__ c2)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ub || s >= *sg.count) return;
    int l = sg.l[s], r = sg.r[s];
    int size = r - l + 1;
    if (size < 4) return;
    if (lb.big[s] && !lb.fallback[s]) return;
    double m0 = 0.0, m1 = 0.0, m2 = 0.0;
    int i = l;
    for (; i + 4 <= r + 1; i += 4) {
        double v0[4], v1[4], v2[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            v0[k] = c0[i + k];
            v1[k] = c1[i + k];
            v2[k] = c2[i + k];
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            m0 = __dadd_rn(m0, v0[k]);
            m1 = __dadd_rn(m1, v1[k]);
            m2 = __dadd_rn(m2, v2[k]);
        }
    }
    for (; i <= r; i++) {
        m0 = __dadd_rn(m0, c0[i]);
        m1 = __dadd_rn(m1, c1[i]);
        m2 = __dadd_rn(m2, c2[i]);
    }
    double nn = (double)size;
    m0 = __ddiv_rn(m0, nn);
    m1 = __ddiv_rn(m1, nn);
    m2 = __ddiv_rn(m2, nn);
    double q0 = 0.0, q1 = 0.0, q2 = 0.0;
    i = l;
    for (; i + 4 <= r + 1; i += 4) {
        double v0[4], v1[4], v2[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            v0[k] = c0[i + k];
            v1[k] = c1[i + k];
            v2[k] = c2[i + k];
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            double d0 = __dsub_rn(v0[k], m0), d1 = __dsub_rn(v1[k], m1), d2 = __dsub_rn(v2[k], m2);
            q0 = __fma_rn(d0, d0, q0);
            q1 = __fma_rn(d1, d1, q1);
            q2 = __fma_rn(d2, d2, q2);
        }
    }
    for (; i <= r; i++) {
        double d0 = __dsub_rn(c0[i], m0), d1 = __dsub_rn(c1[i], m1), d2 = __dsub_rn(c2[i], m2);
        q0 = __fma_rn(d0, d0, q0);
        q1 = __fma_rn(d1, d1, q1);
        q2 = __fma_rn(d2, d2, q2);
    }
    int dim = 0;
    double mx = q0;
    if (q1 > mx) {
        mx = q1;
        dim = 1;
    }
    if (q2 > mx) dim = 2;
    lb.tdim[s] = dim;
}

struct TreeOut {
    NodeRec *nodes;
    int *npoint;
    unsigned char *ndim;
    int *inorder_u;
    int memsize;
};

__device__ __forceinline__ void put_node(TreeOut t, const UniqueArrays &u, int hp, int pt, int dim,
                                         int hl, int hr, int pos, int *err)
{
    if (hp >= t.memsize) {
        set_err(err, KD_EINTERNAL);
        return;
    }
    NodeRec rec;
    rec.v[0] = u.ux[pt];
    rec.v[1] = u.uy[pt];
    rec.v[2] = u.uz[pt];
    rec.fw = (uint32_t)u.ufield[pt] | ((uint32_t)u.uw[pt] << 8);
    rec.pad0 = 0;
    rec.flags = (uint32_t)hl | ((uint32_t)hr << 1) | ((uint32_t)dim << 2);
    rec.pad1 = 0;
    t.nodes[hp] = rec;
    t.npoint[hp] = pt;
    t.ndim[hp] = (unsigned char)dim;
    t.inorder_u[pos] = pt;
}

__global__ void k_level_nodes(Segs sg, int ub, LevelBufs lb, const int *__restrict__ a0,
                              const int *__restrict__ a1, const int *__restrict__ a2,
                              UniqueArrays u, TreeOut t, int *err)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ub || s >= *sg.count) return;
    int p = sg.p[s], l = sg.l[s], r = sg.r[s];
    int size = r - l + 1;
    if (size >= 4) {
        int med = (l + r + 1) / 2;
        int d = lb.tdim[s];
        const int *ad = d == 0 ? a0 : (d == 1 ? a1 : a2);
        put_node(t, u, p, ad[med], d, 1, 1, med, err);
    } else if (size == 3) {
        put_node(t, u, p, a0[l + 1], 0, 1, 1, l + 1, err);
        put_node(t, u, 2 * p, a0[l], 0, 0, 0, l, err);
        put_node(t, u, 2 * p + 1, a0[r], 0, 0, 0, r, err);
    } else if (size == 2) {
        put_node(t, u, p, a0[r], 0, 1, 0, r, err);
        put_node(t, u, 2 * p, a0[l], 0, 0, 0, l, err);
    } else if (size == 1) {
        put_node(t, u, p, a0[l], 0, 0, 0, l, err);
    }
}

// side of every point of a splitting segment: 0 left, 1 right, 2 median
__global__ void k_mark(int n_u, const int *__restrict__ pos_seg, Segs sg, LevelBufs lb,
                       const int *__restrict__ a0, const int *__restrict__ a1,
                       const int *__restrict__ a2, unsigned char *side)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_u; i += gridDim.x * blockDim.x) {
        int s = pos_seg[i];
        if (s < 0) continue;
        int l = sg.l[s], r = sg.r[s];
        if (r - l + 1 < 4) continue;
        int med = (l + r + 1) / 2;
        int d = lb.tdim[s];
        const int *ad = d == 0 ? a0 : (d == 1 ? a1 : a2);
        side[ad[i]] = i < med ? 0 : (i == med ? 2 : 1);
    }
}

// ---- Stable three-way partition of the three superkey orders, one level.
// Within every splitting segment [l, r] (at least four points, median
// position med = (l + r + 1) / 2), the points of each order d go, in their
// order, to [l, med) when k_mark put them left of the median (side 0), to
// (med, r] when right (side 1), the median point itself to med; positions
// outside splitting segments stay.  The destination of a point is its
// segment's start plus the number of same-side points before it in the
// segment: a segmented prefix count, computed in three launches over tiles of
// kPtTile positions that handle all three orders at once (per-tile counts, one
// block scanning the tile counts, then the move), with no waiting between
// blocks.  Counts inside a tile fit 16 bits: left | right << 16 in a word.
constexpr int kPtThreads = 256;
constexpr int kPtItems = 8;  // consecutive positions per thread
constexpr int kPtTile = kPtThreads * kPtItems;

struct PartIO {
    const int *a[3];     // superkey orders (point ids by position)
    int *ao[3];          // partitioned orders
    const double *c[3];  // coordinate d of the point at each position of order d
    double *co[3];       // the same, partitioned
};

// kPtItems consecutive ints from p + base (vector loads when all are in range)
__device__ __forceinline__ void load8(const int *__restrict__ p, int base, int n, int (&x)[kPtItems])
{
    static_assert(kPtItems == 8, "two int4 loads per thread");
    if (base + kPtItems <= n) {
        const int4 u = __ldg(reinterpret_cast<const int4 *>(p + base));
        const int4 w = __ldg(reinterpret_cast<const int4 *>(p + base) + 1);
        x[0] = u.x, x[1] = u.y, x[2] = u.z, x[3] = u.w;
        x[4] = w.x, x[5] = w.y, x[6] = w.z, x[7] = w.w;
    } else {
#pragma unroll
        for (int k = 0; k < kPtItems; k++) x[k] = base + k < n ? p[base + k] : -1;
    }
}

// the splitting segment of each of a thread's positions (-1: none) and the
// positions that start one
__device__ __forceinline__ unsigned split_segs(int base, int n_u, const int *__restrict__ pos_seg,
                                               Segs sg, int (&sgi)[kPtItems])
{
    load8(pos_seg, base, n_u, sgi);
    unsigned headmask = 0;
#pragma unroll
    for (int k = 0; k < kPtItems; k++) {
        const int s = sgi[k];
        if (s < 0) continue;
        const int l = sg.l[s], r = sg.r[s];
        if (r - l + 1 < 4) sgi[k] = -1;
        else if (base + k == l) headmask |= 1u << k;
    }
    return headmask;
}

__device__ __forceinline__ unsigned side_count(int sd)
{
    return sd == 0 ? 1u : (sd == 1 ? 0x10000u : 0u);
}

// inclusive segmented scan over the lanes of a warp: a lane's value restarts
// at a lane holding a head (f = 1)
template <int NV>
__device__ __forceinline__ void warp_seg_scan(unsigned &f, unsigned (&v)[NV], int lane)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned pf = __shfl_up_sync(0xffffffffu, f, o);
        unsigned pv[NV];
#pragma unroll
        for (int k = 0; k < NV; k++) pv[k] = __shfl_up_sync(0xffffffffu, v[k], o);
        if (lane >= o) {
            if (!f)
#pragma unroll
                for (int k = 0; k < NV; k++) v[k] += pv[k];
            f |= pf;
        }
    }
}

// Per tile: (a head in the tile?, the three orders' packed side counts from
// the tile's last head, or from its start when it has none).  Also stores
// the three sides of every position, sd_pos[i] = side0 | side1 << 8 |
// side2 << 16 (3: not in a splitting segment), so that the move reads them
// in order instead of gathering side[] by point again.
__global__ void __launch_bounds__(kPtThreads) k_part_count(int n_u, const int *__restrict__ pos_seg,
                                                           Segs sg, const int *__restrict__ a0,
                                                           const int *__restrict__ a1,
                                                           const int *__restrict__ a2,
                                                           const unsigned char *__restrict__ side,
                                                           unsigned *sd_pos, uint4 *tagg)
{
    constexpr int NW = kPtThreads / 32;
    __shared__ unsigned wf[NW], wv[NW][3];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int base = blockIdx.x * kPtTile + threadIdx.x * kPtItems;
    int sgi[kPtItems];
    const unsigned headmask = split_segs(base, n_u, pos_seg, sg, sgi);
    unsigned sdw[kPtItems];
#pragma unroll
    for (int k = 0; k < kPtItems; k++) sdw[k] = 0x030303u;
    {
        const int *ad[3] = {a0, a1, a2};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            int pt[kPtItems];
            load8(ad[d], base, n_u, pt);
#pragma unroll
            for (int k = 0; k < kPtItems; k++)
                if (sgi[k] >= 0)
                    sdw[k] = (sdw[k] & ~(0xffu << (8 * d))) | ((unsigned)side[pt[k]] << (8 * d));
        }
    }
    unsigned f = 0, v[3] = {0u, 0u, 0u};
#pragma unroll
    for (int k = 0; k < kPtItems; k++) {
        if (headmask >> k & 1) {
            f = 1;
            v[0] = v[1] = v[2] = 0;
        }
#pragma unroll
        for (int d = 0; d < 3; d++) v[d] += side_count((sdw[k] >> (8 * d)) & 0xff);
    }
    if (base + kPtItems <= n_u) {
        reinterpret_cast<uint4 *>(sd_pos + base)[0] = make_uint4(sdw[0], sdw[1], sdw[2], sdw[3]);
        reinterpret_cast<uint4 *>(sd_pos + base)[1] = make_uint4(sdw[4], sdw[5], sdw[6], sdw[7]);
    } else {
#pragma unroll
        for (int k = 0; k < kPtItems; k++)
            if (base + k < n_u) sd_pos[base + k] = sdw[k];
    }
    warp_seg_scan<3>(f, v, lane);
    if (lane == 31) {
        wf[w] = f;
        wv[w][0] = v[0];
        wv[w][1] = v[1];
        wv[w][2] = v[2];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned F = 0, V[3] = {0u, 0u, 0u};
        for (int q = 0; q < NW; q++) {
            for (int k = 0; k < 3; k++) V[k] = wf[q] ? wv[q][k] : V[k] + wv[q][k];
            F |= wf[q];
        }
        tagg[blockIdx.x] = make_uint4(F, V[0], V[1], V[2]);
    }
}


__device__ __forceinline__ void unpack_counts(const uint4 &g, unsigned (&x)[6])
{
    x[0] = g.y & 0xffffu;
    x[1] = g.y >> 16;
    x[2] = g.z & 0xffffu;
    x[3] = g.z >> 16;
    x[4] = g.w & 0xffffu;
    x[5] = g.w >> 16;
}

// One block: for every tile, the side counts (left, right for each order, 32
// bits each) from the last head before the tile: carry[2t], carry[2t+1].
__global__ void __launch_bounds__(1024) k_part_carry(int ntiles, const uint4 *__restrict__ tagg,
                                                     uint4 *carry)
{
    __shared__ unsigned sf[32], sv[32][6];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int per = (ntiles + 1023) / 1024;
    const int j0 = min(ntiles, t * per), j1 = min(ntiles, j0 + per);
    unsigned f = 0, v[6] = {0u, 0u, 0u, 0u, 0u, 0u};
    for (int j = j0; j < j1; j++) {
        const uint4 g = tagg[j];
        unsigned x[6];
        unpack_counts(g, x);
        for (int k = 0; k < 6; k++) v[k] = g.x ? x[k] : v[k] + x[k];
        f |= g.x;
    }
    unsigned fi = f, vi[6];
    for (int k = 0; k < 6; k++) vi[k] = v[k];
    warp_seg_scan<6>(fi, vi, lane);
    if (lane == 31) {
        sf[w] = fi;
        for (int k = 0; k < 6; k++) sv[w][k] = vi[k];
    }
    __syncthreads();
    // everything before this thread's tiles: the earlier warps, then the
    // earlier lanes of this warp
    unsigned pv[6] = {0u, 0u, 0u, 0u, 0u, 0u};
    for (int q = 0; q < w; q++)
        for (int k = 0; k < 6; k++) pv[k] = sf[q] ? sv[q][k] : pv[k] + sv[q][k];
    unsigned ef = __shfl_up_sync(0xffffffffu, fi, 1), ev[6];
    for (int k = 0; k < 6; k++) ev[k] = __shfl_up_sync(0xffffffffu, vi[k], 1);
    if (lane == 0) {
        ef = 0;
        for (int k = 0; k < 6; k++) ev[k] = 0;
    }
    unsigned cv[6];
    for (int k = 0; k < 6; k++) cv[k] = ef ? ev[k] : pv[k] + ev[k];
    for (int j = j0; j < j1; j++) {
        carry[2 * (size_t)j] = make_uint4(cv[0], cv[1], cv[2], cv[3]);
        carry[2 * (size_t)j + 1] = make_uint4(cv[4], cv[5], 0u, 0u);
        const uint4 g = tagg[j];
        unsigned x[6];
        unpack_counts(g, x);
        for (int k = 0; k < 6; k++) cv[k] = g.x ? x[k] : cv[k] + x[k];
    }
}

// The move: every position's point id and carried coordinate, in each of the
// three orders, to its place (see above).
__global__ void __launch_bounds__(kPtThreads, 3) k_part_move(int n_u, const int *__restrict__ pos_seg,
                                                             Segs sg, PartIO io,
                                                             const unsigned *__restrict__ sd_pos,
                                                             const uint4 *__restrict__ carry,
                                                             int *err)
{
    constexpr int NW = kPtThreads / 32;
    __shared__ unsigned wf[NW], wv[NW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int base = blockIdx.x * kPtTile + threadIdx.x * kPtItems;
    const bool full = base + kPtItems <= n_u;
    int sgi[kPtItems], sdp[kPtItems];
    const unsigned headmask = split_segs(base, n_u, pos_seg, sg, sgi);
    load8(reinterpret_cast<const int *>(sd_pos), base, n_u, sdp);
    const uint4 c0 = carry[2 * (size_t)blockIdx.x], c1 = carry[2 * (size_t)blockIdx.x + 1];
#pragma unroll 1
    for (int d = 0; d < 3; d++) {
        // (selects rather than indexing io and the carry by d, which would
        // put them in local memory)
        const int *__restrict__ ain = d == 0 ? io.a[0] : (d == 1 ? io.a[1] : io.a[2]);
        int *__restrict__ aout = d == 0 ? io.ao[0] : (d == 1 ? io.ao[1] : io.ao[2]);
        const double *__restrict__ cin = d == 0 ? io.c[0] : (d == 1 ? io.c[1] : io.c[2]);
        double *__restrict__ cout = d == 0 ? io.co[0] : (d == 1 ? io.co[1] : io.co[2]);
        const unsigned crl = d == 0 ? c0.x : (d == 1 ? c0.z : c1.x);
        const unsigned crr = d == 0 ? c0.y : (d == 1 ? c0.w : c1.y);
        int sd[kPtItems];
        unsigned f = 0, v = 0;
#pragma unroll
        for (int k = 0; k < kPtItems; k++) {
            sd[k] = ((unsigned)sdp[k] >> (8 * d)) & 0xffu;
            if (headmask >> k & 1) {
                f = 1;
                v = 0;
            }
            v += side_count(sd[k]);
        }
        unsigned vi[1] = {v};
        unsigned fi = f;
        warp_seg_scan<1>(fi, vi, lane);
        if (lane == 31) {
            wf[w] = fi;
            wv[w] = vi[0];
        }
        __syncthreads();
        unsigned pf = 0, pv = 0;
        for (int q = 0; q < w; q++) {
            pv = wf[q] ? wv[q] : pv + wv[q];
            pf |= wf[q];
        }
        unsigned ef = __shfl_up_sync(0xffffffffu, fi, 1);
        unsigned ev = __shfl_up_sync(0xffffffffu, vi[0], 1);
        if (lane == 0) ef = ev = 0;
        // the tile's counts before this thread's first position
        unsigned runf = pf | ef, runv = ef ? ev : pv + ev;
        __syncthreads();  // wf / wv are written again for the next order
        int pt[kPtItems];
        double cv[kPtItems];
        load8(ain, base, n_u, pt);
        if (full) {
            const double2 *cp = reinterpret_cast<const double2 *>(cin + base);
#pragma unroll
            for (int k = 0; k < kPtItems / 2; k++) {
                const double2 t = __ldg(cp + k);
                cv[2 * k] = t.x;
                cv[2 * k + 1] = t.y;
            }
        } else {
#pragma unroll
            for (int k = 0; k < kPtItems; k++) cv[k] = base + k < n_u ? cin[base + k] : 0.0;
        }
#pragma unroll
        for (int k = 0; k < kPtItems; k++) {
            const int i = base + k;
            if (i >= n_u) break;
            int dst = i;
            if (sgi[k] >= 0) {
                if (headmask >> k & 1) {
                    runf = 1;
                    runv = 0;
                }
                unsigned L = runv & 0xffffu, R = runv >> 16;
                if (!runf) {  // the segment began in an earlier tile
                    L += crl;
                    R += crr;
                }
                const int s = sgi[k], l = sg.l[s], r = sg.r[s], med = (l + r + 1) / 2;
                dst = sd[k] == 0 ? l + (int)L : (sd[k] == 1 ? med + 1 + (int)R : med);
                if (dst < l || dst > r) {
                    set_err(err, KD_EINTERNAL);
                    dst = -1;
                }
                runv += side_count(sd[k]);
            }
            if (dst >= 0) {
                aout[dst] = pt[k];
                cout[dst] = cv[k];
            }
        }
    }
}

__global__ void k_children(Segs cur, int ub, LevelBufs lb, Segs nxt, int cap, int *err)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ub) return;
    int ns = *cur.count;
    if (s == 0) *nxt.count = ns > 0 ? 2 * (lb.rank[ns - 1] + lb.haskids[ns - 1]) : 0;
    if (s >= ns || !lb.haskids[s]) return;
    int p = cur.p[s], l = cur.l[s], r = cur.r[s];
    int med = (l + r + 1) / 2;
    int c = 2 * lb.rank[s];
    if (c + 1 >= cap) {
        set_err(err, KD_EINTERNAL);
        return;
    }
    nxt.p[c] = 2 * p;
    nxt.l[c] = l;
    nxt.r[c] = med - 1;
    nxt.p[c + 1] = 2 * p + 1;
    nxt.l[c + 1] = med + 1;
    nxt.r[c + 1] = r;
}

__global__ void k_next_pos(int n_u, const int *__restrict__ pos_seg, Segs sg, LevelBufs lb,
                           int *pos_next)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_u; i += gridDim.x * blockDim.x) {
        int s = pos_seg[i];
        int v = -1;
        if (s >= 0 && lb.haskids[s]) {
            int med = (sg.l[s] + sg.r[s] + 1) / 2;
            if (i != med) v = 2 * lb.rank[s] + (i > med);
        }
        pos_next[i] = v;
    }
}

__global__ void k_inorder_rep(int n_u, const int *__restrict__ inorder_u,
                              const int *__restrict__ urep, int *out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_u; i += gridDim.x * blockDim.x)
        out[i] = urep[inorder_u[i]];
}

// ------------------------------------------------------------ counting layout

// in-order range of heap id h at depth D (the range recursion is data
// independent: med = (l+r+1)/2, children (l, med-1) and (med+1, r))
__device__ __forceinline__ void heap_range(int n_u, int h, int D, int &l, int &r)
{
    l = 0;
    r = n_u - 1;
    for (int b = D - 1; b >= 0; b--) {
        int med = (l + r + 1) / 2;
        if ((h >> b) & 1) l = med + 1;
        else r = med - 1;
    }
}

__device__ __forceinline__ int superkey_cmp(const UniqueArrays &u, int a, int b, int msd)
{
    for (int k = 0; k < 3; k++) {
        int d = (msd + k) % 3;
        uint64_t ka = d == 0 ? u.ukx[a] : (d == 1 ? u.uky[a] : u.ukz[a]);
        uint64_t kb = d == 0 ? u.ukx[b] : (d == 1 ? u.uky[b] : u.ukz[b]);
        if (ka != kb) return ka < kb ? -1 : 1;
    }
    return 0;
}

// Each node above the counting leaves holds one point; it is placed in the
// leaf (below its left child, on whose side of the split plane it lies) whose
// cell contains it, following the splits of the nodes below.
__global__ void k_anc_leaf(int nleaves, const int *__restrict__ npoint,
                           const unsigned char *__restrict__ ndim, UniqueArrays u, int *anc_leaf,
                           int *extra_cnt)
{
    int h = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (h >= nleaves) return;
    int pt = npoint[h];
    int c = 2 * h;
    while (c < nleaves) c = 2 * c + (superkey_cmp(u, pt, npoint[c], ndim[c]) > 0);
    int leaf = c - nleaves;
    anc_leaf[h - 1] = leaf;
    atomicAdd(&extra_cnt[leaf], 1);
}

__global__ void k_leaf_ucount(int n_u, int D, int nleaves, const int *__restrict__ extra_cnt,
                              int *ucount)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nleaves) return;
    int l, r;
    heap_range(n_u, nleaves + j, D, l, r);
    ucount[j] = (r - l + 1) + (extra_cnt ? extra_cnt[j] : 0);
}

__global__ void k_cpos_sub(int n_u, int D, int nleaves, const int *__restrict__ ustart,
                           const int *__restrict__ inorder_u, int *cpos)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nleaves) return;
    int l, r;
    heap_range(n_u, nleaves + j, D, l, r);
    int base = ustart[j];
    for (int i = l; i <= r; i++) cpos[inorder_u[i]] = base + (i - l);
}

// sorted (leaf, ancestor) pairs -> counting positions of ancestor points
__global__ void k_cpos_extra(int nanc, int n_u, int D, int nleaves,
                             const int *__restrict__ sleaf, const int *__restrict__ sanc,
                             const int *__restrict__ extra_start, const int *__restrict__ ustart,
                             const int *__restrict__ npoint, int *cpos)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nanc) return;
    int j = sleaf[k];
    int l, r;
    heap_range(n_u, nleaves + j, D, l, r);
    cpos[npoint[sanc[k]]] = ustart[j] + (r - l + 1) + (k - extra_start[j]);
}

__global__ void k_scatter_w(int n_u, const int *__restrict__ cpos, const int *__restrict__ uw,
                            int *wc)
{
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < n_u; u += gridDim.x * blockDim.x)
        wc[cpos[u]] = uw[u];
}

struct RawOut {
    double *x, *y, *z;
    int *qf, *tf;
};

__global__ void k_raw_scatter(int n, const int *__restrict__ p, const int *__restrict__ cls,
                              const int *__restrict__ uhead, const int *__restrict__ cpos,
                              const int *__restrict__ rstart, const double *__restrict__ xyz,
                              const int *__restrict__ fin, const int *__restrict__ ufield,
                              RawOut o, int split)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int r = p[i], c = cls[i] - 1;
        int pos = rstart[cpos[c]] + (i - uhead[c]);
        o.x[pos] = xyz[3 * (size_t)r];
        o.y[pos] = xyz[3 * (size_t)r + 1];
        o.z[pos] = xyz[3 * (size_t)r + 2];
        o.qf[pos] = fin ? fin[r] : 0;
        if (split) o.tf[pos] = ufield[c];
    }
}

__global__ void k_leaf_rstart(int nleaves, const int *__restrict__ ustart,
                              const int *__restrict__ rstart, int *leaf_r)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j > nleaves) return;
    leaf_r[j] = rstart[ustart[j]];
}

// key (leaf, tree field) per raw position; flag when a leaf is out of order
__global__ void k_leaf_keys(int nleaves, const int *__restrict__ leaf_r,
                            const int *__restrict__ tf, unsigned *key, int *unsorted)
{
    int j = blockIdx.x;
    if (j >= nleaves) return;
    int a = leaf_r[j], b = leaf_r[j + 1];
    int bad = 0;
    for (int i = a + threadIdx.x; i < b; i += blockDim.x) {
        key[i] = ((unsigned)j << 8) | (unsigned)tf[i];
        if (i > a && tf[i] < tf[i - 1]) bad = 1;
    }
    if (bad) atomicOr(unsorted, 1);
}

template <class T>
__global__ void k_gather(const T *__restrict__ src, const int *__restrict__ idx, int n, T *dst)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = src[idx[i]];
}

// group heads (leaf or tree-field change) carry their own index, others 0;
// an inclusive max-scan then gives every position its group start
__global__ void k_group_heads(int n, const unsigned *__restrict__ key, int *gh)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        gh[i] = (i == 0 || key[i] != key[i - 1]) ? i : 0;
}

// a run starts at every KD_RUN_MAX-th point of a group
__global__ void k_run_heads(int n, const int *__restrict__ gs, int *head)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        head[i] = ((i - gs[i]) % KD_RUN_MAX) == 0;
}

__global__ void k_runs(int n, const unsigned *__restrict__ key, const int *__restrict__ head,
                       const int *__restrict__ rid, int nleaves, int *run_start, int *run_tf,
                       int *run_leaf, int *leaf_run)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!head[i]) continue;
        int r = rid[i] - 1;
        run_start[r] = i;
        run_tf[r] = (int)(key[i] & 0xFF);
        unsigned leaf = key[i] >> 8;
        run_leaf[r] = (int)leaf;
        if (i == 0 || (key[i - 1] >> 8) != leaf) leaf_run[leaf] = r;
    }
}

__global__ void k_run_len(int nruns, int n, int nleaves, const int *__restrict__ run_start,
                          int *run_len, int *leaf_run)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r == 0) leaf_run[nleaves] = nruns;
    if (r >= nruns) return;
    int e = r + 1 < nruns ? run_start[r + 1] : n;
    run_len[r] = e - run_start[r];
}

struct Summ {
    double *box;
    int *count, *tf, *qf;
};

// one warp per leaf
__global__ void k_leaf_summary(int nleaves, const int *__restrict__ leaf_r, RawOut o, Summ sm)
{
    int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= nleaves) return;
    int a = leaf_r[w], b = leaf_r[w + 1];
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    int tf0 = o.tf[a], qf0 = o.qf[a];
    int tfm = 0, qfm = 0;
    for (int i = a + lane; i < b; i += 32) {
        double v[3] = {o.x[i], o.y[i], o.z[i]};
        for (int d = 0; d < 3; d++) {
            lo[d] = fmin(lo[d], v[d]);
            hi[d] = fmax(hi[d], v[d]);
        }
        tfm |= o.tf[i] != tf0;
        qfm |= o.qf[i] != qf0;
    }
    for (int off = 16; off; off >>= 1)
        for (int d = 0; d < 3; d++) {
            lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], off));
            hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], off));
        }
    tfm = __any_sync(0xffffffffu, tfm);
    qfm = __any_sync(0xffffffffu, qfm);
    if (lane == 0) {
        int h = nleaves + w;
        for (int d = 0; d < 3; d++) {
            sm.box[6 * (size_t)h + d] = lo[d];
            sm.box[6 * (size_t)h + 3 + d] = hi[d];
        }
        sm.count[h] = b - a;
        sm.tf[h] = tfm ? -1 : tf0;
        sm.qf[h] = qfm ? -1 : qf0;
    }
}

// leaf centres and each raw point in FP32 relative to its leaf's centre,
// stored ready for the tile kernel's distance expansion
__global__ void k_leaf_rel(int nleaves, const int *__restrict__ leaf_r, RawOut o,
                           const double *__restrict__ box, double *leaf_c, float4 *t4,
                           unsigned long long *hdiag)
{
    int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= nleaves) return;
    const double *b = box + 6 * (size_t)(nleaves + w);
    double cx = 0.5 * (b[0] + b[3]), cy = 0.5 * (b[1] + b[4]), cz = 0.5 * (b[2] + b[5]);
    if (lane == 0) {
        leaf_c[3 * (size_t)w] = cx;
        leaf_c[3 * (size_t)w + 1] = cy;
        leaf_c[3 * (size_t)w + 2] = cz;
        double hx = 0.5 * (b[3] - b[0]), hy = 0.5 * (b[4] - b[1]), hz = 0.5 * (b[5] - b[2]);
        double h = sqrt(hx * hx + hy * hy + hz * hz);
        atomicMax(hdiag, (unsigned long long)__double_as_longlong(h));
    }
    // (-2 t, |t|^2) of t = fl32(p - centre); |t|^2 is exact in FP64 from the
    // FP32 components and rounded once
    for (int i = leaf_r[w] + lane; i < leaf_r[w + 1]; i += 32) {
        float tx = (float)(o.x[i] - cx), ty = (float)(o.y[i] - cy), tz = (float)(o.z[i] - cz);
        double tn = (double)tx * tx + (double)ty * ty + (double)tz * tz;
        t4[i] = make_float4(-2.0f * tx, -2.0f * ty, -2.0f * tz, (float)tn);
    }
}

__global__ void k_internal_summary(int lo_h, int hi_h, Summ sm)
{
    int h = lo_h + blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= hi_h) return;
    int a = 2 * h, b = 2 * h + 1;
    for (int d = 0; d < 3; d++) {
        sm.box[6 * (size_t)h + d] = fmin(sm.box[6 * (size_t)a + d], sm.box[6 * (size_t)b + d]);
        sm.box[6 * (size_t)h + 3 + d] =
            fmax(sm.box[6 * (size_t)a + 3 + d], sm.box[6 * (size_t)b + 3 + d]);
    }
    sm.count[h] = sm.count[a] + sm.count[b];
    sm.tf[h] = (sm.tf[a] >= 0 && sm.tf[a] == sm.tf[b]) ? sm.tf[a] : -1;
    sm.qf[h] = (sm.qf[a] >= 0 && sm.qf[a] == sm.qf[b]) ? sm.qf[a] : -1;
}

// query blocks: each depth-DB subtree's raw range split into equal parts of
// at most KD_BLOCK_MAX points
__global__ void k_block_count(int nb_nodes, int span, const int *__restrict__ leaf_r, int *nblk)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nb_nodes) return;
    int len = leaf_r[(k + 1) * span] - leaf_r[k * span];
    nblk[k] = (len + KD_BLOCK_MAX - 1) / KD_BLOCK_MAX;
}

__global__ void k_block_fill(int nb_nodes, int span, const int *__restrict__ leaf_r,
                             const int *__restrict__ nblk, const int *__restrict__ boff,
                             int *bstart, int *blen)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nb_nodes) return;
    int a = leaf_r[k * span], len = leaf_r[(k + 1) * span] - a;
    int nb = nblk[k];
    for (int j = 0; j < nb; j++) {
        int s = a + (int)((long long)len * j / nb), e = a + (int)((long long)len * (j + 1) / nb);
        bstart[boff[k] + j] = s;
        blen[boff[k] + j] = e - s;
    }
}

// one CTA of KD_BLOCK_MAX threads per query block: box and single own field
__global__ void __launch_bounds__(KD_BLOCK_MAX) k_block_boxes(int nblocks, const int *bstart,
                                                             const int *blen, RawOut o,
                                                             double *bbox, int *bqf)
{
    constexpr int W = KD_BLOCK_MAX / 32;
    __shared__ double sw[W][6];
    __shared__ int sq[W];
    int b = blockIdx.x;
    if (b >= nblocks) return;
    int t = threadIdx.x, w = t >> 5, lane = t & 31;
    int len = blen[b], s = bstart[b];
    bool valid = t < len;
    double lo[3], hi[3];
    int qf = valid ? o.qf[s + t] : 0x7fffffff;
    for (int d = 0; d < 3; d++) {
        double v = valid ? (d == 0 ? o.x[s + t] : (d == 1 ? o.y[s + t] : o.z[s + t])) : 0.0;
        lo[d] = valid ? v : INFINITY;
        hi[d] = valid ? v : -INFINITY;
    }
    int q0 = __shfl_sync(0xffffffffu, qf, 0);
    int mixed = valid && qf != q0;
    for (int off = 16; off; off >>= 1)
        for (int d = 0; d < 3; d++) {
            lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], off));
            hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], off));
        }
    mixed = __any_sync(0xffffffffu, mixed);
    if (lane == 0) {
        for (int d = 0; d < 3; d++) {
            sw[w][d] = lo[d];
            sw[w][3 + d] = hi[d];
        }
        sq[w] = (32 * w >= len) ? -2 : (mixed ? -1 : q0);
    }
    __syncthreads();
    if (t == 0) {
        double L[3] = {INFINITY, INFINITY, INFINITY}, H[3] = {-INFINITY, -INFINITY, -INFINITY};
        int q = -2;
        for (int k = 0; k < W; k++) {
            for (int d = 0; d < 3; d++) {
                L[d] = fmin(L[d], sw[k][d]);
                H[d] = fmax(H[d], sw[k][3 + d]);
            }
            if (sq[k] == -2) continue;
            if (sq[k] == -1 || (q != -2 && q != sq[k])) q = -1;
            else if (q == -2) q = sq[k];
        }
        for (int d = 0; d < 3; d++) {
            bbox[6 * (size_t)b + d] = L[d];
            bbox[6 * (size_t)b + 3 + d] = H[d];
        }
        bqf[b] = q < 0 ? -1 : q;
    }
}

// ------------------------------------------------------------ helpers

// Stable radix sort of (key, value) pairs by key bits [b0, b1) and device
// scans: the project's own (kd_sort.cuh), temporaries from the call's pool.
// Keys are unsigned or non-negative.
template <class K, class V>
static void sort_pairs(Pool &pool, cudaStream_t s, const K *kin, K *kout, const V *vin, V *vout,
                       int n, int b0, int b1)
{
    char *tmp = pool.alloc<char>(sort::sort_temp_bytes<K, V>(n));
    check(sort::sort_pairs<K, V>(tmp, kin, kout, vin, vout, n, b0, b1, s), "radix sort");
}

template <class T>
static void excl_sum(Pool &pool, cudaStream_t s, const T *in, T *out, int n)
{
    char *tmp = pool.alloc<char>(sort::scan_temp_bytes<T>(n));
    check(sort::scan<T, sort::SumOp, false>(tmp, in, out, n, sort::SumOp(), s), "scan");
}

template <class T>
static void incl_sum(Pool &pool, cudaStream_t s, const T *in, T *out, int n)
{
    char *tmp = pool.alloc<char>(sort::scan_temp_bytes<T>(n));
    check(sort::scan<T, sort::SumOp, true>(tmp, in, out, n, sort::SumOp(), s), "scan");
}

template <class T>
static void incl_max(Pool &pool, cudaStream_t s, const T *in, T *out, int n)
{
    char *tmp = pool.alloc<char>(sort::scan_temp_bytes<T>(n));
    check(sort::scan<T, sort::MaxOp, true>(tmp, in, out, n, sort::MaxOp(), s), "max scan");
}

static int bit_hi(unsigned long long v) { return v ? 64 - __builtin_clzll(v) : 0; }
static int bit_lo(unsigned long long v) { return v ? __builtin_ctzll(v) : 0; }

static const int TPB = 256;

static unsigned grid_for(long long n)
{
    long long b = (n + TPB - 1) / TPB;
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (unsigned)b;
}

template <class T> static T read1(const T *d, cudaStream_t s)
{
    T v;
    check(cudaMemcpyAsync(&v, d, sizeof(T), cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaStreamSynchronize(s), "sync");
    return v;
}

static void copy_to_pageable(void *dst, const void *src, size_t bytes);
static void copy_from_host(void *dst, const void *src, size_t bytes, cudaStream_t s);

// Touch one byte of every 4 KiB page of [p, p + bytes), split over up to 16
// threads, so that the pages are resident before they are copied into.
static void prefault(void *p, size_t bytes)
{
    if (bytes < ((size_t)64 << 20)) return;
    const unsigned hw = std::thread::hardware_concurrency();
    const int nthr = (int)std::max(1u, std::min(16u, hw ? hw : 1u));
    auto touch = [p, bytes, nthr](int t) {
        volatile char *c = (volatile char *)p;
        const size_t a = bytes * t / nthr, b = bytes * (t + 1) / nthr;
        for (size_t i = a & ~(size_t)4095; i < b; i += 4096)
            if (i >= a) c[i] = 0;
    };
    std::vector<std::thread> th;
    try {
        for (int t = 1; t < nthr; t++) th.emplace_back(touch, t);
    } catch (const std::exception &) {
    }
    touch(0);
    for (int t = (int)th.size() + 1; t < nthr; t++) touch(t);  // threads not started
    for (auto &x : th) x.join();
}

static double wall_ms()
{
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
}

// The node array's way to the caller's host array (see build_impl): the
// per-level items the build queues, the copier thread that drains them, and,
// for a deferred build, the device node array it reads until it is done.
struct NodeCopy {
    kd_node_sink *sink = nullptr;
    void *host = nullptr;
    bool handed = false;
    std::thread th;
    std::mutex mu;
    std::condition_variable cv;
    struct Item {
        cudaEvent_t ev;
        size_t off, len;
    };
    std::vector<Item> items;
    size_t next = 0;     // first item the copier has not taken
    bool closed = false; // no more items
    std::vector<cudaEvent_t> events;
    int code = 0;
    char msg[160] = "";
    double ms = 0;
    // deferred builds: the device node array (freed once the copy is done)
    // and the one-time join
    void *dnodes = nullptr;
    std::once_flag joined;
    void push(cudaEvent_t ev, size_t off, size_t len)
    {
        std::lock_guard<std::mutex> g(mu);
        items.push_back({ev, off, len});
        cv.notify_one();
    }
    void close()
    {
        std::lock_guard<std::mutex> g(mu);
        closed = true;
        cv.notify_one();
    }
    ~NodeCopy()
    {
        close();
        if (th.joinable()) th.join();
        for (auto e : events) cudaEventDestroy(e);
        if (dnodes) cudaFree(dnodes);
        if (host && !handed) sink->release(host);
    }
};

static void build_impl(const double *h_xyz, const int *h_fields, int n, int num_fields,
                       int query_only, kd_node_sink *sink, int deferred, kd_catalog *cat)
{
    init_device();
    Stream st;
    cudaStream_t s = st.s;
    Pool pool(s);     // temporaries
    Pool keep(s);     // catalog arrays (released to the catalog on success)
    // phase boundaries: start, dedup, argsorts, levels, layout, end
    cudaEvent_t ph[6] = {};
    struct EvRelease {
        cudaEvent_t *e;
        ~EvRelease()
        {
            for (int i = 0; i < 6; i++)
                if (e[i]) cudaEventDestroy(e[i]);
        }
    } ev_release{ph};
    for (auto &e : ph) check(cudaEventCreate(&e), "cudaEventCreate");
    check(cudaEventRecord(ph[0], s), "event");

    // ---- inputs
    double *xyz = pool.alloc<double>(3 * (size_t)n);
    copy_from_host(xyz, h_xyz, sizeof(double) * 3 * (size_t)n, s);
    int *fin = nullptr;
    if (h_fields) {
        fin = pool.alloc<int>(n);
        copy_from_host(fin, h_fields, sizeof(int) * (size_t)n, s);
    }
    int *err = pool.alloc<int>(1);
    unsigned long long *misc = pool.alloc<unsigned long long>(4);
    check(cudaMemsetAsync(err, 0, sizeof(int), s), "memset");
    check(cudaMemsetAsync(misc, 0, 4 * sizeof(unsigned long long), s), "memset");

    uint64_t *kx = pool.alloc<uint64_t>(n), *ky = pool.alloc<uint64_t>(n),
             *kz = pool.alloc<uint64_t>(n);
    int *iota = pool.alloc<int>(n);
    k_prep<<<grid_for(n), TPB, 0, s>>>(xyz, n, kx, ky, kz, iota, err, misc + 3);
    k_keyvary<<<grid_for(n), TPB, 0, s>>>(kx, ky, kz, n, misc);
    KD_LAUNCH_CHECK("k_prep");
    unsigned long long hv[4];
    check(cudaMemcpyAsync(hv, misc, sizeof hv, cudaMemcpyDeviceToHost, s), "D2H");
    int herr = 0;
    check(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    st.sync();
    if (herr) raise(herr, "NaN coordinate in tree points");
    double maxabs;
    memcpy(&maxabs, &hv[3], sizeof maxabs);

    check(cudaEventRecord(ph[1], s), "event");
    // ---- stable lexicographic sort (LSD: z, then y, then x)
    uint64_t *ktmp = pool.alloc<uint64_t>(n), *ksrt = pool.alloc<uint64_t>(n);
    int *pa = pool.alloc<int>(n), *pb = pool.alloc<int>(n);
    check(cudaMemcpyAsync(pa, iota, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, s), "copy");
    const uint64_t *keys[3] = {kz, ky, kx};
    unsigned long long vary[3] = {hv[2], hv[1], hv[0]};
    for (int k = 0; k < 3; k++) {
        if (!vary[k]) continue;  // constant key: a stable sort is the identity
        k_gather_u64<<<grid_for(n), TPB, 0, s>>>(keys[k], pa, n, ktmp);
        sort_pairs(pool, s, ktmp, ksrt, pa, pb, n, bit_lo(vary[k]), bit_hi(vary[k]));
        std::swap(pa, pb);
    }
    int *p3 = pa;

    // ---- runs of equal points
    int *head = pool.alloc<int>(n), *cls = pool.alloc<int>(n);
    k_heads<<<grid_for(n), TPB, 0, s>>>(p3, kx, ky, kz, n, head);
    incl_sum(pool, s, head, cls, n);
    int n_u = read1(cls + (n - 1), s);

    UniqueArrays u;
    u.ux = pool.alloc<double>(n_u);
    u.uy = pool.alloc<double>(n_u);
    u.uz = pool.alloc<double>(n_u);
    u.ufield = pool.alloc<int>(n_u);
    u.uw = pool.alloc<int>(n_u);
    u.urep = pool.alloc<int>(n_u);
    u.uhead = pool.alloc<int>(n_u + 1);
    u.ukx = pool.alloc<uint64_t>(n_u);
    u.uky = pool.alloc<uint64_t>(n_u);
    u.ukz = pool.alloc<uint64_t>(n_u);
    k_unique<<<grid_for(n), TPB, 0, s>>>(p3, head, cls, n, xyz, fin, kx, ky, kz, u, n_u);
    FieldInfo *fi = pool.alloc<FieldInfo>(1);
    FieldInfo fi0 = {0x7fffffff, -0x7fffffff, 0, 0};
    check(cudaMemcpyAsync(fi, &fi0, sizeof fi0, cudaMemcpyHostToDevice, s), "H2D");
    k_weights<<<grid_for(std::max(n, n_u)), TPB, 0, s>>>(u, n_u, p3, cls, fin, n, query_only, err, fi);
    KD_LAUNCH_CHECK("k_weights");
    FieldInfo hfi;
    check(cudaMemcpyAsync(&hfi, fi, sizeof hfi, cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    st.sync();
    if (herr) raise(herr, "a point is repeated 256 or more times (the node weight is 8 bits)");

    check(cudaEventRecord(ph[2], s), "event");
    // ---- superkey argsorts of the unique points (dedup order = superkey 0)
    int *A[3], *B[3];
    for (int d = 0; d < 3; d++) {
        A[d] = pool.alloc<int>(n_u);
        B[d] = pool.alloc<int>(n_u);
    }
    check(cudaMemcpyAsync(A[0], iota, sizeof(int) * (size_t)n_u, cudaMemcpyDeviceToDevice, s),
          "copy");
    // superkey 2 = (z, x, y): stable sort of the (x, y, z) order by z
    // (only the bits that vary among the points: the same order)
    sort_pairs(pool, s, u.ukz, ksrt, (const int *)iota, A[2], n_u, bit_lo(hv[2]), bit_hi(hv[2]));
    // superkey 1 = (y, z, x): stable sort of the (z, x, y) order by y
    k_gather_u64<<<grid_for(n_u), TPB, 0, s>>>(u.uky, A[2], n_u, ktmp);
    sort_pairs(pool, s, ktmp, ksrt, (const int *)A[2], A[1], n_u, bit_lo(hv[1]), bit_hi(hv[1]));
    // coordinate d of the point at every position of order d, partitioned
    // along with the order (the variance passes then read contiguously)
    double *C[3], *CB[3];
    {
        const double *uc[3] = {u.ux, u.uy, u.uz};
        for (int d = 0; d < 3; d++) {
            C[d] = pool.alloc<double>(n_u);
            CB[d] = pool.alloc<double>(n_u);
            k_gather<double><<<grid_for(n_u), TPB, 0, s>>>(uc[d], A[d], n_u, C[d]);
        }
    }

    check(cudaEventRecord(ph[3], s), "event");
    // ---- tree
    int memsize = 2;
    {
        int x = n_u, e = 1;
        while (x > 1) {
            x /= 2;
            e++;
        }
        memsize = 1 << e;
    }
    TreeOut to;
    to.memsize = memsize;
    to.nodes = sink ? keep.alloc_from<NodeRec>(side_pool(kPoolNodes), memsize) : keep.alloc<NodeRec>(memsize);
    to.npoint = pool.alloc<int>(memsize);
    to.ndim = pool.alloc<unsigned char>(memsize);
    to.inorder_u = pool.alloc<int>(n_u);
    check(cudaMemsetAsync(to.nodes, 0, sizeof(NodeRec) * (size_t)memsize, s), "memset");
    check(cudaMemsetAsync(to.npoint, 0xff, sizeof(int) * (size_t)memsize, s), "memset");
    check(cudaMemsetAsync(to.ndim, 0, (size_t)memsize, s), "memset");

    int cap = n_u / 2 + 16;
    Segs sg[2];
    for (int k = 0; k < 2; k++) {
        sg[k].p = pool.alloc<int>(cap);
        sg[k].l = pool.alloc<int>(cap);
        sg[k].r = pool.alloc<int>(cap);
        sg[k].count = pool.alloc<int>(1);
    }
    LevelBufs lb;
    lb.cap_big = n_u / kSmallSeg + 16;
    lb.tdim = pool.alloc<int>(cap);
    lb.big = pool.alloc<unsigned char>(cap);
    lb.fallback = pool.alloc<unsigned char>(cap);
    lb.acc = pool.alloc<double>(9 * (size_t)lb.cap_big);
    lb.rank = pool.alloc<int>(cap);
    lb.haskids = pool.alloc<int>(cap);
    int *pos[2] = {pool.alloc<int>(n_u), pool.alloc<int>(n_u)};
    unsigned char *side = pool.alloc<unsigned char>(n_u);
    const int ntiles = (int)((n_u + (long long)kPtTile - 1) / kPtTile);
    uint4 *tagg = pool.alloc<uint4>(ntiles), *tcarry = pool.alloc<uint4>(2 * (size_t)ntiles);
    unsigned *sd_pos = pool.alloc<unsigned>(n_u);
    {
        int one = 1, zero = 0, last = n_u - 1;
        check(cudaMemcpyAsync(sg[0].count, &one, sizeof(int), cudaMemcpyHostToDevice, s), "H2D");
        check(cudaMemcpyAsync(sg[0].p, &one, sizeof(int), cudaMemcpyHostToDevice, s), "H2D");
        check(cudaMemcpyAsync(sg[0].l, &zero, sizeof(int), cudaMemcpyHostToDevice, s), "H2D");
        check(cudaMemcpyAsync(sg[0].r, &last, sizeof(int), cudaMemcpyHostToDevice, s), "H2D");
        check(cudaMemsetAsync(pos[0], 0, sizeof(int) * (size_t)n_u, s), "memset");
        st.sync();  // the host scalars above go out of scope
    }
    // The node array goes to the caller's host array level by level while
    // the tree is built: iteration lev of the loop below writes the heap
    // slots of level lev (and, for segments of at most three points, their
    // children), so once it has run, every slot below 2^(lev+1) is final.
    // The build records an event after each iteration and queues that
    // level's slots; a second host thread waits for each event and copies
    // the slots (pinned staging, DMA on its own stream) while the build
    // goes on, then the rest once the loop ends, during the counting layout.
    std::unique_ptr<NodeCopy> ncu(new NodeCopy);
    NodeCopy &nc = *ncu;
    const size_t node_bytes = sizeof(NodeRec) * (size_t)memsize;
    size_t node_queued = sizeof(NodeRec);  // slot 0 is never written: it stays zero
    // queue the node slots [node_queued, upto) once the stream reaches here
    auto queue_nodes = [&](size_t upto) {
        if (!sink || upto <= node_queued) return;
        cudaEvent_t ev = nullptr;
        check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
        nc.events.push_back(ev);
        check(cudaEventRecord(ev, s), "event");
        nc.push(ev, node_queued, upto - node_queued);
        node_queued = upto;
    };
    if (sink) {
        nc.sink = sink;
        nc.host = sink->alloc(node_bytes);
        if (!nc.host) raise(KD_ENOMEM, "out of host memory for the node array");
        memset(nc.host, 0, sizeof(NodeRec));
        int dev = 0;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        const char *src = (const char *)to.nodes;
        NodeCopy *ncp = &nc;
        auto job = [ncp, dev, src, node_bytes] {
            const double t0 = wall_ms();
            try {
                check(cudaSetDevice(dev), "cudaSetDevice");
                // fault the whole host array in first, on parallel threads,
                // while the first levels are built: the copies then write
                // resident pages instead of taking a page fault (and the
                // kernel's zeroing of a fresh page) at every page
                prefault(ncp->host, node_bytes);
                for (;;) {
                    NodeCopy::Item it;
                    {
                        std::unique_lock<std::mutex> g(ncp->mu);
                        ncp->cv.wait(g, [ncp] { return ncp->next < ncp->items.size() || ncp->closed; });
                        if (ncp->next == ncp->items.size()) break;
                        it = ncp->items[ncp->next++];
                    }
                    check(cudaEventSynchronize(it.ev), "node copy wait");
                    copy_to_pageable((char *)ncp->host + it.off, src + it.off, it.len);
                }
            } catch (const Error &e) {
                ncp->code = e.code;
                snprintf(ncp->msg, sizeof ncp->msg, "node copy: %.140s", e.msg);
            } catch (const std::exception &e) {
                ncp->code = KD_EINTERNAL;
                snprintf(ncp->msg, sizeof ncp->msg, "node copy: %s", e.what());
            }
            ncp->ms = wall_ms() - t0;
        };
        try {
            nc.th = std::thread(job);
        } catch (const std::exception &) {
            // no thread to spare: the copy runs on this thread at the end
        }
    }

    // the partition kernels read and write these with 16-byte vector
    // accesses at multiples of 8 elements: stream-ordered allocations are
    // aligned far beyond that, which is checked here rather than assumed
    {
        const void *vec[] = {pos[0], pos[1], A[0], A[1], A[2], B[0], B[1], B[2],
                             C[0],   C[1],   C[2], CB[0], CB[1], CB[2], sd_pos};
        for (const void *p : vec)
            if ((reinterpret_cast<uintptr_t>(p) & 15) != 0)
                raise(KD_EINTERNAL, "build array not 16-byte aligned");
    }
    int cur = 0, nlevels = 0;
    for (int lev = 0; (1LL << lev) <= (long long)n_u; lev++) {
        nlevels = lev + 1;
        long long ub64 = std::min<long long>(1LL << lev, cap);
        int ub = (int)ub64;
        unsigned gs = blocks_for(ub, TPB);
        Segs S = sg[cur], N = sg[cur ^ 1];
        k_seg_setup<<<gs, TPB, 0, s>>>(S, ub, lb);
        long long maxsize = (long long)n_u >> lev;
        if (maxsize > kSmallSeg) {
            unsigned gv = blocks_for(n_u, kVarChunk);
            k_var_par<0><<<gv, kVarThreads, 0, s>>>(n_u, pos[cur], S, lb, C[0], C[1], C[2]);
            k_var_par<1><<<gv, kVarThreads, 0, s>>>(n_u, pos[cur], S, lb, C[0], C[1], C[2]);
            k_var_decide<<<gs, TPB, 0, s>>>(S, ub, lb);
        }
        k_var_seq<<<blocks_for(ub, 64), 64, 0, s>>>(S, ub, lb, C[0], C[1], C[2]);
        k_level_nodes<<<gs, TPB, 0, s>>>(S, ub, lb, A[0], A[1], A[2], u, to, err);
        KD_LAUNCH_CHECK("level kernels");
        if (maxsize < 4) break;  // every segment of this level was a base case
        // levels 0 .. lev are final: copy their slots once they are large
        // enough to be worth a copy of their own
        {
            const size_t upto = sizeof(NodeRec) * std::min<size_t>((size_t)2 << lev, memsize);
            if (upto - node_queued >= ((size_t)4 << 20)) queue_nodes(upto);
        }
        k_mark<<<grid_for(n_u), TPB, 0, s>>>(n_u, pos[cur], S, lb, A[0], A[1], A[2], side);
        {
            k_part_count<<<ntiles, kPtThreads, 0, s>>>(n_u, pos[cur], S, A[0], A[1], A[2], side,
                                                       sd_pos, tagg);
            k_part_carry<<<1, 1024, 0, s>>>(ntiles, tagg, tcarry);
            PartIO io;
            for (int d = 0; d < 3; d++) {
                io.a[d] = A[d];
                io.ao[d] = B[d];
                io.c[d] = C[d];
                io.co[d] = CB[d];
            }
            k_part_move<<<ntiles, kPtThreads, 0, s>>>(n_u, pos[cur], S, io, sd_pos, tcarry, err);
            for (int d = 0; d < 3; d++) {
                std::swap(A[d], B[d]);
                std::swap(C[d], CB[d]);
            }
        }
        excl_sum(pool, s, lb.haskids, lb.rank, ub);
        k_children<<<gs, TPB, 0, s>>>(S, ub, lb, N, cap, err);
        k_next_pos<<<grid_for(n_u), TPB, 0, s>>>(n_u, pos[cur], S, lb, pos[cur ^ 1]);
        KD_LAUNCH_CHECK("partition kernels");
        cur ^= 1;
    }
    // every slot is final: queue the rest and let the copier finish it while
    // the counting layout is built
    queue_nodes(node_bytes);
    nc.close();
    if (sink && !nc.th.joinable()) {  // no copier thread: copy here
        for (auto &it : nc.items) {
            check(cudaEventSynchronize(it.ev), "node copy wait");
            copy_to_pageable((char *)nc.host + it.off, (const char *)to.nodes + it.off, it.len);
        }
    }
    int *inorder_rep = keep.alloc<int>(n_u);
    k_inorder_rep<<<grid_for(n_u), TPB, 0, s>>>(n_u, to.inorder_u, u.urep, inorder_rep);
    check(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    st.sync();
    if (herr) raise(herr, "tree build exceeded an internal bound");

    check(cudaEventRecord(ph[4], s), "event");
    // ---- counting layout
    int D = 0;
    while ((long long)KD_LEAF_TARGET << D < (long long)n_u) D++;
    if (D > 24) raise(KD_EINVAL, "tree too large for the counting layout (more than 2^29 points)");
    int nleaves = 1 << D;
    int *extra_cnt = pool.alloc<int>(nleaves);
    check(cudaMemsetAsync(extra_cnt, 0, sizeof(int) * (size_t)nleaves, s), "memset");
    int nanc = nleaves - 1;
    int *anc_leaf = pool.alloc<int>(std::max(nanc, 1)), *anc_id = pool.alloc<int>(std::max(nanc, 1));
    int *sleaf = pool.alloc<int>(std::max(nanc, 1)), *sanc = pool.alloc<int>(std::max(nanc, 1));
    int *extra_start = pool.alloc<int>(nleaves);
    if (nanc > 0) {
        k_anc_leaf<<<blocks_for(nanc, TPB), TPB, 0, s>>>(nleaves, to.npoint, to.ndim, u, anc_leaf,
                                                          extra_cnt);
        // ancestor ids 1..nanc in order; a stable sort by leaf keeps that order
        k_gather<int><<<grid_for(nanc), TPB, 0, s>>>(iota + 1, iota, nanc, anc_id);
        sort_pairs(pool, s, (const int *)anc_leaf, sleaf, (const int *)anc_id, sanc, nanc, 0,
                   std::max(1, D));
        excl_sum(pool, s, extra_cnt, extra_start, nleaves);
    }
    int *ucount = pool.alloc<int>(nleaves + 1), *ustart = pool.alloc<int>(nleaves + 1);
    k_leaf_ucount<<<blocks_for(nleaves, TPB), TPB, 0, s>>>(n_u, D, nleaves,
                                                           nanc > 0 ? extra_cnt : nullptr, ucount);
    check(cudaMemsetAsync(ucount + nleaves, 0, sizeof(int), s), "memset");
    excl_sum(pool, s, ucount, ustart, nleaves + 1);
    int *cpos = pool.alloc<int>(n_u);
    k_cpos_sub<<<blocks_for(nleaves, TPB), TPB, 0, s>>>(n_u, D, nleaves, ustart, to.inorder_u,
                                                        cpos);
    if (nanc > 0)
        k_cpos_extra<<<blocks_for(nanc, TPB), TPB, 0, s>>>(nanc, n_u, D, nleaves, sleaf, sanc,
                                                           extra_start, ustart, to.npoint, cpos);
    int *wc = pool.alloc<int>(n_u + 1), *rstart = pool.alloc<int>(n_u + 1);
    k_scatter_w<<<grid_for(n_u), TPB, 0, s>>>(n_u, cpos, u.uw, wc);
    check(cudaMemsetAsync(wc + n_u, 0, sizeof(int), s), "memset");
    excl_sum(pool, s, wc, rstart, n_u + 1);

    int split = hfi.split ? 1 : 0;
    RawOut ro;
    ro.x = keep.alloc<double>(n);
    ro.y = keep.alloc<double>(n);
    ro.z = keep.alloc<double>(n);
    ro.qf = keep.alloc<int>(n);
    ro.tf = split ? keep.alloc<int>(n) : ro.qf;
    k_raw_scatter<<<grid_for(n), TPB, 0, s>>>(n, p3, cls, u.uhead, cpos, rstart, xyz, fin,
                                              u.ufield, ro, split);
    int *leaf_r = keep.alloc<int>(nleaves + 1);
    k_leaf_rstart<<<blocks_for(nleaves + 1, TPB), TPB, 0, s>>>(nleaves, ustart, rstart, leaf_r);
    KD_LAUNCH_CHECK("layout kernels");

    // group each leaf's points by tree field (stable), then cut runs
    unsigned *key = pool.alloc<unsigned>(n), *key2 = pool.alloc<unsigned>(n);
    int *unsorted = pool.alloc<int>(1);
    check(cudaMemsetAsync(unsorted, 0, sizeof(int), s), "memset");
    k_leaf_keys<<<nleaves, 64, 0, s>>>(nleaves, leaf_r, ro.tf, key, unsorted);
    if (read1(unsorted, s)) {
        int *perm = pool.alloc<int>(n);
        sort_pairs(pool, s, (const unsigned *)key, key2, (const int *)iota, perm, n, 0, D + 8);
        std::swap(key, key2);
        double *tmpd = pool.alloc<double>(n);
        int *tmpi = pool.alloc<int>(n);
        double *dd[3] = {ro.x, ro.y, ro.z};
        for (int d = 0; d < 3; d++) {
            k_gather<double><<<grid_for(n), TPB, 0, s>>>(dd[d], perm, n, tmpd);
            check(cudaMemcpyAsync(dd[d], tmpd, sizeof(double) * (size_t)n,
                                  cudaMemcpyDeviceToDevice, s), "copy");
        }
        int *ii[2] = {ro.qf, ro.tf};
        for (int k = 0; k < (split ? 2 : 1); k++) {
            k_gather<int><<<grid_for(n), TPB, 0, s>>>(ii[k], perm, n, tmpi);
            check(cudaMemcpyAsync(ii[k], tmpi, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice,
                                  s), "copy");
        }
    }
    int *rhead = pool.alloc<int>(n), *rid = pool.alloc<int>(n);
    {
        int *gh = pool.alloc<int>(n), *gs = pool.alloc<int>(n);
        k_group_heads<<<grid_for(n), TPB, 0, s>>>(n, key, gh);
        incl_max(pool, s, (const int *)gh, gs, n);
        k_run_heads<<<grid_for(n), TPB, 0, s>>>(n, gs, rhead);
    }
    incl_sum(pool, s, rhead, rid, n);
    int nruns = read1(rid + (n - 1), s);
    int *run_start = keep.alloc<int>(nruns), *run_len = keep.alloc<int>(nruns),
        *run_tf = keep.alloc<int>(nruns), *run_leaf = keep.alloc<int>(nruns),
        *leaf_run = keep.alloc<int>(nleaves + 1);
    k_runs<<<grid_for(n), TPB, 0, s>>>(n, key, rhead, rid, nleaves, run_start, run_tf, run_leaf,
                                       leaf_run);
    k_run_len<<<blocks_for(nruns + 1, TPB), TPB, 0, s>>>(nruns, n, nleaves, run_start, run_len,
                                                          leaf_run);

    // counting-tree summaries
    int nnodes = 2 * nleaves;
    Summ sm;
    sm.box = keep.alloc<double>(6 * (size_t)nnodes);
    sm.count = keep.alloc<int>(nnodes);
    sm.tf = keep.alloc<int>(nnodes);
    sm.qf = keep.alloc<int>(nnodes);
    k_leaf_summary<<<blocks_for((long long)nleaves * 32, TPB), TPB, 0, s>>>(nleaves, leaf_r, ro,
                                                                             sm);
    for (int d = D - 1; d >= 0; d--)
        k_internal_summary<<<blocks_for(1 << d, TPB), TPB, 0, s>>>(1 << d, 2 << d, sm);
    double *leaf_c = keep.alloc<double>(3 * (size_t)nleaves);
    float4 *t4 = keep.alloc<float4>(n);
    unsigned long long *hdiag = pool.alloc<unsigned long long>(1);
    check(cudaMemsetAsync(hdiag, 0, sizeof(unsigned long long), s), "memset");
    k_leaf_rel<<<blocks_for((long long)nleaves * 32, TPB), TPB, 0, s>>>(nleaves, leaf_r, ro, sm.box,
                                                                         leaf_c, t4, hdiag);
    double leaf_hdiag = 0;
    {
        unsigned long long hb = read1(hdiag, s);
        memcpy(&leaf_hdiag, &hb, sizeof leaf_hdiag);
    }

    // query blocks: each 16-leaf subtree cut into equal chunks of <= 128
    int DB = std::max(0, D - 4);
    int nbn = 1 << DB, span = nleaves / nbn;
    int *nblk = pool.alloc<int>(nbn + 1), *boff = pool.alloc<int>(nbn + 1);
    k_block_count<<<blocks_for(nbn, TPB), TPB, 0, s>>>(nbn, span, leaf_r, nblk);
    check(cudaMemsetAsync(nblk + nbn, 0, sizeof(int), s), "memset");
    excl_sum(pool, s, nblk, boff, nbn + 1);
    int nblocks = read1(boff + nbn, s);
    int *bstart = keep.alloc<int>(nblocks), *blen = keep.alloc<int>(nblocks),
        *bqf = keep.alloc<int>(nblocks);
    double *bbox = keep.alloc<double>(6 * (size_t)nblocks);
    k_block_fill<<<blocks_for(nbn, TPB), TPB, 0, s>>>(nbn, span, leaf_r, nblk, boff, bstart, blen);
    k_block_boxes<<<nblocks, KD_BLOCK_MAX, 0, s>>>(nblocks, bstart, blen, ro, bbox, bqf);
    KD_LAUNCH_CHECK("summary kernels");
    check(cudaEventRecord(ph[5], s), "event");
    st.sync();
    kd_build_stats bs;
    memset(&bs, 0, sizeof bs);
    if (!deferred || !sink) {
        const double wait0 = wall_ms();
        if (nc.th.joinable()) nc.th.join();
        const double waited = wall_ms() - wait0;
        if (nc.code) raise(nc.code, nc.msg);
        bs.ms_node_copy = nc.ms;
        bs.ms_node_wait = waited;
    }
    {
        float ms[5] = {0, 0, 0, 0, 0}, tot = 0;
        for (int i = 0; i < 5; i++) cudaEventElapsedTime(&ms[i], ph[i], ph[i + 1]);
        cudaEventElapsedTime(&tot, ph[0], ph[5]);
        bs.ms_prep = ms[0];
        bs.ms_dedup = ms[1];
        bs.ms_argsort = ms[2];
        bs.ms_levels = ms[3];
        bs.ms_layout = ms[4];
        bs.ms_device = tot;
        bs.levels = nlevels;
        bs.n_unique = n_u;
    }

    // ---- hand the kept arrays to the catalog
    memset(cat, 0, sizeof *cat);
    check(cudaGetDevice(&cat->device), "cudaGetDevice");
    cat->n_raw = n;
    cat->n_u = n_u;
    cat->memsize = memsize;
    cat->num_fields = num_fields;
    cat->min_qf = h_fields ? hfi.min_qf : 0;
    cat->max_qf = h_fields ? hfi.max_qf : 0;
    cat->max_tf = hfi.max_tf;
    cat->fields_split = split;
    cat->max_abs = maxabs;
    if (sink) {
        // the host holds the node array; the device copy is freed with the
        // pool, or, while a deferred copy still reads it, once that is done
        sink->nodes = nc.host;
        nc.handed = true;
        nc.sink = nullptr;
        cat->d_nodes = nullptr;
    } else {
        cat->d_nodes = keep.keep(to.nodes);
    }
    cat->d_inorder_rep = keep.keep(inorder_rep);
    cat->d_x = keep.keep(ro.x);
    cat->d_y = keep.keep(ro.y);
    cat->d_z = keep.keep(ro.z);
    cat->d_qf = keep.keep(ro.qf);
    cat->d_tf = split ? keep.keep(ro.tf) : ro.qf;
    cat->depth = D;
    cat->nleaves = nleaves;
    cat->d_box = keep.keep(sm.box);
    cat->d_ncount = keep.keep(sm.count);
    cat->d_ntf = keep.keep(sm.tf);
    cat->d_nqf = keep.keep(sm.qf);
    cat->d_leaf_run = keep.keep(leaf_run);
    cat->d_leaf_pos = keep.keep(leaf_r);
    cat->nruns = nruns;
    cat->d_run_start = keep.keep(run_start);
    cat->d_run_len = keep.keep(run_len);
    cat->d_run_tf = keep.keep(run_tf);
    cat->d_run_leaf = keep.keep(run_leaf);
    cat->d_t4 = keep.keep(t4);
    cat->d_leaf_c = keep.keep(leaf_c);
    cat->leaf_hdiag = leaf_hdiag;
    cat->nblocks = nblocks;
    cat->d_blk_start = keep.keep(bstart);
    cat->d_blk_len = keep.keep(blen);
    cat->d_blk_qf = keep.keep(bqf);
    cat->d_blk_box = keep.keep(bbox);
    cat->device_bytes = keep.bytes;
    cat->bstats = bs;
    if (sink && deferred) {
        nc.dnodes = keep.keep(to.nodes);
        cat->pending = ncu.release();
    }
}

}  // namespace kd

static int build_entry(const double *h_xyz, const int *h_fields, int n, int num_fields,
                       int query_only, kd_node_sink *sink, int deferred, kd_catalog *cat)
{
    if (n < 1) {
        kd_set_error(KD_EINVAL, "a tree needs at least one point");
        return KD_EINVAL;
    }
    try {
        kd::build_impl(h_xyz, h_fields, n, num_fields, query_only, sink, deferred, cat);
        return KD_OK;
    } catch (const kd::Error &e) {
        kd_set_error(e.code, "%s", e.msg);
        return e.code;
    } catch (const std::bad_alloc &) {
        kd_set_error(KD_ENOMEM, "out of host memory");
        return KD_ENOMEM;
    } catch (const std::exception &e) {
        kd_set_error(KD_EINTERNAL, "host error: %s", e.what());
        return KD_EINTERNAL;
    }
}

extern "C" int kdg_build(const double *h_xyz, const int *h_fields, int n, int num_fields,
                         int query_only, kd_catalog *cat)
{
    return build_entry(h_xyz, h_fields, n, num_fields, query_only, nullptr, 0, cat);
}

extern "C" int kdg_build_tree(const double *h_xyz, const int *h_fields, int n, int num_fields,
                              kd_node_sink *sink, int deferred, kd_catalog *cat)
{
    if (!sink || !sink->alloc || !sink->release) {
        kd_set_error(KD_EINVAL, "kdg_build_tree: no node array sink");
        return KD_EINVAL;
    }
    sink->nodes = nullptr;
    return build_entry(h_xyz, h_fields, n, num_fields, 0, sink, deferred, cat);
}

// Runs a catalog operation on the catalog's device, then restores the
// calling thread's device.
struct OnDevice {
    int prev = 0;
    explicit OnDevice(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~OnDevice() { cudaSetDevice(prev); }
};

namespace kd {

// Device -> pageable host copy of the node array returned by tree_construct
// (1.3 GB at 20M points), one queued item at a time.  A plain cudaMemcpy into
// pageable memory goes through the driver's own staging, one copy at a time
// for the whole process, and at the speed of the page faults of its one
// copying thread; it also makes every other pageable transfer of the process
// (the build's own small reads of device scalars) queue behind it.  Here the
// data goes through two pinned staging chunks (the next chunk's DMA overlaps
// the current one's host copy) and each chunk is copied into the destination
// by several threads, which take the destination's first-touch page faults in
// parallel.
namespace {
struct Staging {
    static constexpr size_t kChunk = size_t(32) << 20;
    void *pin[2] = {nullptr, nullptr};
};
// pinned staging pairs kept for the life of the process (allocating pinned
// memory per copy costs more than the copy): one per copy running at once,
// at most kMaxStaging (a batch of many small deferred builds would otherwise
// pin 64 MB per build); a copy that finds them all in use waits for one
constexpr int kMaxStaging = 4;
std::mutex g_stage_mu;
std::condition_variable g_stage_cv;
std::vector<Staging *> g_stage_free;
int g_stage_made = 0;
struct StagingLease {
    Staging *st = nullptr;
    StagingLease()
    {
        {
            std::unique_lock<std::mutex> g(g_stage_mu);
            g_stage_cv.wait(g, [] { return !g_stage_free.empty() || g_stage_made < kMaxStaging; });
            if (!g_stage_free.empty()) {
                st = g_stage_free.back();
                g_stage_free.pop_back();
                return;
            }
            g_stage_made++;  // this thread makes the next pair
        }
        std::unique_ptr<Staging> n(new Staging);
        for (int i = 0; i < 2; i++)
            if (cudaHostAlloc(&n->pin[i], Staging::kChunk, cudaHostAllocPortable) != cudaSuccess) {
                cudaGetLastError();
                for (int j = 0; j < i; j++) cudaFreeHost(n->pin[j]);
                {
                    std::lock_guard<std::mutex> g(g_stage_mu);
                    g_stage_made--;
                }
                g_stage_cv.notify_one();
                raise(KD_ENOMEM, "out of pinned host memory for the node array copy");
            }
        st = n.release();
    }
    ~StagingLease()
    {
        {
            std::lock_guard<std::mutex> g(g_stage_mu);
            g_stage_free.push_back(st);
        }
        g_stage_cv.notify_one();
    }
};
// Host copies of a transfer's chunks fanned out over a pool of threads made
// once for the whole transfer (a 32 MB chunk takes ~1 ms; creating threads
// per chunk would cost a good part of that).  Transfers under 4 MB are
// copied by the calling thread alone.
struct FanOut {
    int nthr = 1;
    std::vector<std::thread> th;
    std::mutex mu;
    std::condition_variable go, done;
    size_t gen = 0;
    int pending = 0;
    bool stop = false;
    char *to = nullptr;
    const char *from = nullptr;
    size_t len = 0;
    explicit FanOut(size_t bytes)
    {
        const unsigned hw = std::thread::hardware_concurrency();
        nthr = bytes < (size_t(4) << 20) ? 1 : (int)std::max(1u, std::min(16u, hw ? hw : 1u));
        try {
            for (int t = 1; t < nthr; t++) th.emplace_back(&FanOut::worker, this, t);
        } catch (const std::exception &) {  // fewer threads: the rest is copied by this one
        }
    }
    void slice(int t, char *d, const char *f, size_t n)
    {
        const size_t a = n * t / nthr, b = n * (t + 1) / nthr;
        std::memcpy(d + a, f + a, b - a);
    }
    void worker(int t)
    {
        size_t seen = 0;
        std::unique_lock<std::mutex> g(mu);
        for (;;) {
            go.wait(g, [&] { return stop || gen != seen; });
            if (stop) return;
            seen = gen;
            char *d = to;
            const char *f = from;
            const size_t n = len;
            g.unlock();
            slice(t, d, f, n);
            g.lock();
            if (--pending == 0) done.notify_one();
        }
    }
    void copy(char *d, const char *f, size_t n)
    {
        {
            std::lock_guard<std::mutex> g(mu);
            to = d;
            from = f;
            len = n;
            pending = (int)th.size();
            gen++;
        }
        go.notify_all();
        // slices of the threads that could not be started are done here
        for (int t = (int)th.size() + 1; t < nthr; t++) slice(t, d, f, n);
        slice(0, d, f, n);
        std::unique_lock<std::mutex> g(mu);
        done.wait(g, [&] { return pending == 0; });
    }
    ~FanOut()
    {
        {
            std::lock_guard<std::mutex> g(mu);
            stop = true;
        }
        go.notify_all();
        for (auto &x : th) x.join();
    }
};
}  // namespace

// Host -> device copy of a build's input on stream s.  Pinned (or managed)
// memory, and anything under 32 MB (where starting the copying threads
// costs more than it saves), is one cudaMemcpyAsync.  Pageable memory
// otherwise takes the driver's own staging path at about 10 GB/s (50 ms for
// the 560 MB of a 20M-point catalog); here several threads copy each 32 MB
// chunk into a pinned staging buffer while the previous chunk's DMA runs.
// Returns once the last DMA has finished (the staging pair is then free).
static void copy_from_host(void *dst, const void *src, size_t bytes, cudaStream_t s)
{
    if (bytes == 0) return;
    bool plain = bytes < (size_t(32) << 20);
    if (!plain) {
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, src) == cudaSuccess)
            plain = at.type != cudaMemoryTypeUnregistered;
        else
            cudaGetLastError();  // not known to the runtime: pageable
    }
    if (plain) {
        check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "H2D");
        return;
    }
    const size_t chunk = Staging::kChunk;
    StagingLease lease;
    void *const *pin = lease.st->pin;
    cudaEvent_t done[2] = {nullptr, nullptr};
    struct Release {
        cudaEvent_t *ev;
        ~Release()
        {
            for (int i = 0; i < 2; i++)
                if (ev[i]) {
                    cudaEventSynchronize(ev[i]);  // no DMA may still read the staging
                    cudaEventDestroy(ev[i]);
                }
        }
    } rel{done};
    for (int i = 0; i < 2; i++)
        check(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming), "cudaEventCreate");
    FanOut fan(bytes);
    const size_t nch = (bytes + chunk - 1) / chunk;
    for (size_t c = 0; c < nch; c++) {
        const int b = (int)(c & 1);
        if (c >= 2) check(cudaEventSynchronize(done[b]), "H2D wait");  // its last DMA is done
        const size_t off = c * chunk, len = std::min(chunk, bytes - off);
        fan.copy((char *)pin[b], (const char *)src + off, len);
        check(cudaMemcpyAsync((char *)dst + off, pin[b], len, cudaMemcpyHostToDevice, s), "H2D");
        check(cudaEventRecord(done[b], s), "event");
    }
    for (int b = 0; b < 2; b++) check(cudaEventSynchronize(done[b]), "H2D wait");
}

static void copy_to_pageable(void *dst, const void *src, size_t bytes)
{
    const size_t chunk = Staging::kChunk;
    if (bytes == 0) return;
    StagingLease lease;
    void *const *pin = lease.st->pin;
    Stream st;
    cudaEvent_t done[2] = {nullptr, nullptr};
    struct Release {
        cudaEvent_t *ev;
        ~Release()
        {
            for (int i = 0; i < 2; i++)
                if (ev[i]) cudaEventDestroy(ev[i]);
        }
    } rel{done};
    for (int i = 0; i < 2; i++)
        check(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming), "cudaEventCreate");
    const size_t nch = (bytes + chunk - 1) / chunk;
    auto issue = [&](size_t c) {
        const size_t off = c * chunk, len = std::min(chunk, bytes - off);
        check(cudaMemcpyAsync(pin[c & 1], (const char *)src + off, len, cudaMemcpyDeviceToHost, st.s),
              "D2H");
        check(cudaEventRecord(done[c & 1], st.s), "event");
    };
    FanOut fan(bytes);

    issue(0);
    for (size_t c = 0; c < nch; c++) {
        check(cudaEventSynchronize(done[c & 1]), "D2H wait");
        if (c + 1 < nch) issue(c + 1);  // into the other buffer, already drained
        const size_t off = c * chunk, len = std::min(chunk, bytes - off);
        fan.copy((char *)dst + off, (const char *)pin[c & 1], len);
    }
}

}  // namespace kd

extern "C" int kdg_copy_inorder(const kd_catalog *cat, int *h_perm)
{
    OnDevice on(cat->device);
    cudaError_t e = cudaMemcpy(h_perm, cat->d_inorder_rep, sizeof(int) * (size_t)cat->n_u,
                               cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        kd_set_error(KD_ECUDA, "permutation copy: %s", cudaGetErrorString(e));
        return KD_ECUDA;
    }
    return KD_OK;
}

extern "C" int kdg_wait_nodes(kd_catalog *cat)
{
    kd::NodeCopy *nc = (kd::NodeCopy *)cat->pending;
    if (!nc) return KD_OK;
    std::call_once(nc->joined, [nc, cat] {
        const double w0 = kd::wall_ms();
        if (nc->th.joinable()) nc->th.join();
        cat->bstats.ms_node_wait = kd::wall_ms() - w0;
        cat->bstats.ms_node_copy = nc->ms;
        OnDevice on(cat->device);
        // the copier has finished reading it: a stream-ordered free, so that
        // a count still running on the device is not waited for
        if (nc->dnodes) cudaFreeAsync(nc->dnodes, cudaStreamPerThread);
        nc->dnodes = nullptr;
    });
    if (nc->code) {
        kd_set_error(nc->code, "%s", nc->msg);
        return nc->code;
    }
    return KD_OK;
}

extern "C" void kdg_free(kd_catalog *cat)
{
    if (cat->pending) {
        kdg_wait_nodes(cat);
        OnDevice on(cat->device);
        delete (kd::NodeCopy *)cat->pending;
        cat->pending = nullptr;
    }
    OnDevice on(cat->device);
    void *ptrs[] = {cat->d_nodes,    cat->d_inorder_rep, cat->d_x,       cat->d_y,
                    cat->d_z,        cat->d_qf,          cat->fields_split ? cat->d_tf : nullptr,
                    cat->d_box,      cat->d_ncount,      cat->d_ntf,     cat->d_nqf,
                    cat->d_leaf_run, cat->d_leaf_pos,    cat->d_run_start, cat->d_run_len,
                    cat->d_run_tf,
                    cat->d_run_leaf, cat->d_t4,          cat->d_leaf_c,
                    cat->d_blk_start, cat->d_blk_len,    cat->d_blk_qf,  cat->d_blk_box};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    memset(cat, 0, sizeof *cat);
}
