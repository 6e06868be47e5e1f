// Pair counting for corruscant's pair_count (kdquery.c:62-113, :165-249),
// batched over all bin edges at once.
//
// Semantics kept from the reference (proved equivalent in DESIGN.md): the
// reference traversal counts, for every query point q and every tree node t,
// weight(t) if fl(d2) < fl(r*r), where d2 is evaluated as
//     dx = t.x - q.x, ...;  d2 = dx*dx;  d2 = fma(dy,dy,d2);  d2 = fma(dz,dz,d2)
// (kdquery.c:39-47 as the reference build compiles it) and its pruning
// (kdquery.c:96-104) never drops such a pair.  Here a pair lands in bin e, the
// first sorted squared edge with d2 < rsq[e]; cumulative sums over e give the
// reference's per-radius counts.
//
// Work decomposition (B200-first, not the reference's per-query recursion):
//   k_traverse : one warp per query block walks the tree-side counting tree
//                with box-box distance bounds.  Node pairs beyond the last
//                edge are pruned, node pairs entirely inside one bin are
//                accepted as count(block) x count(node), and leaf pairs are
//                emitted as tiles (block, run) with a per-warp active edge
//                range.  Run twice: once to count tiles, once to write them.
//   k_tiles    : one CTA (8 warps, one query point per thread) per query
//                block streams its tree runs through shared memory (double
//                buffered, one barrier per run).  Mixed mode: FP32 distances
//                relative to the block centre, binned against the active edges
//                with a saturating ramp that is exactly 0 or 1 outside a
//                rigorous error band; a tile with any pair inside the band is
//                recomputed for that thread in FP64 with the reference's
//                operation order.  FP64 mode: every distance in FP64.
//                Per-thread bin counters live in shared memory and are
//                reduced per warp into the global (bin, qfield, tfield)
//                histogram when the tree field changes.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "kd_cuda_util.cuh"

namespace kd {

constexpr int kTravWarps = 4;
constexpr int kStack = 2048;
constexpr int kTileThreads = KD_BLOCK_MAX;

struct TreeSide {
    const double *x, *y, *z;
    const double *box;
    const int *count, *tf, *leaf_run;
    const int *run_start, *run_len, *run_tf;
    int D, nleaves;
};

struct QuerySide {
    const double *x, *y, *z;
    const int *qf;
    const int *blk_start, *blk_len, *blk_qf;
    const double *blk_box, *blk_wbox;
};

// Bins a pair of boxes can reach: pairs land in bins elo..ehi (ne = beyond
// every edge).  The box bounds are exact for the points' true distances; the
// relative margin covers the FP64 rounding of the reference's d2 and of this
// bound computation.
__device__ __forceinline__ void bin_range(const double *a, const double *b,
                                          const double *__restrict__ rsq, int ne, int &elo,
                                          int &ehi)
{
    double dmin2 = 0.0, dmax2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        double g = fmax(0.0, fmax(b[d] - a[3 + d], a[d] - b[3 + d]));
        double sp = fmax(b[3 + d] - a[d], a[3 + d] - b[d]);
        dmin2 += g * g;
        dmax2 += sp * sp;
    }
    double lo = dmin2 * (1.0 - 1e-12), hi = dmax2 * (1.0 + 1e-12);
    int l = 0, h = ne;  // first e with rsq[e] > lo
    while (l < h) {
        int m = (l + h) >> 1;
        if (rsq[m] > lo) h = m;
        else l = m + 1;
    }
    elo = l;
    h = ne;  // first e with rsq[e] > hi
    while (l < h) {
        int m = (l + h) >> 1;
        if (rsq[m] > hi) h = m;
        else l = m + 1;
    }
    ehi = l;
}

struct TravOut {
    int *count;                 // COUNT pass: tiles per block
    const long long *off;       // FILL pass: batch-relative tile offsets
    unsigned *run;              // FILL: tree run of each tile
    unsigned short *code;       // FILL: KD_WARPS codes per tile (k0 | K << 8)
    unsigned long long *H;
    int Fqe, Fte;
    unsigned long long *accepted;
    int *err;
};

template <bool FILL>
__global__ void __launch_bounds__(32 * kTravWarps) k_traverse(TreeSide T, QuerySide Q,
                                                             const double *__restrict__ g_rsq,
                                                             int ne, int b0, int b1, TravOut o)
{
    __shared__ int stack[kTravWarps][kStack];
    __shared__ double rsq[KD_MAX_EDGES];
    __shared__ double wb[kTravWarps][KD_WARPS * 6 + 6];
    for (int k = threadIdx.x; k < ne; k += blockDim.x) rsq[k] = g_rsq[k];
    __syncthreads();
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int b = b0 + blockIdx.x * kTravWarps + w;
    if (b >= b1) return;
    int alen = Q.blk_len[b], aqf = Q.blk_qf[b];
    int nw = (alen + 31) >> 5;
    double *bb = wb[w];
    for (int k = lane; k < 6; k += 32) bb[k] = Q.blk_box[6 * (size_t)b + k];
    for (int k = lane; k < KD_WARPS * 6; k += 32) bb[6 + k] = Q.blk_wbox[(size_t)b * KD_WARPS * 6 + k];
    int *st = stack[w];
    if (lane == 0) st[0] = 1;
    __syncwarp();
    int sp = 1;
    long long emitted = 0;
    long long base = FILL ? o.off[b - b0] : 0;
    unsigned long long acc_pairs = 0;
    long long guard = 8LL * 2 * T.nleaves + 64;
    while (sp > 0) {
        if (--guard < 0) {
            if (lane == 0) atomicCAS(o.err, 0, KD_EINTERNAL);
            break;
        }
        int nb = min(sp, 32);
        int h = lane < nb ? st[sp - nb + lane] : 0;
        __syncwarp();
        sp -= nb;
        int act = 0, nr = 0, leaf = 0;
        if (h) {
            int elo, ehi;
            bin_range(bb, T.box + 6 * (size_t)h, rsq, ne, elo, ehi);
            if (elo >= ne) {
                act = 0;
            } else if (elo == ehi && aqf >= 0 && T.tf[h] >= 0) {
                if (FILL) {
                    unsigned long long c = (unsigned long long)alen * (unsigned long long)T.count[h];
                    atomicAdd(&o.H[((size_t)elo * o.Fqe + aqf) * o.Fte + T.tf[h]], c);
                    acc_pairs += c;
                }
            } else if (h >= T.nleaves) {
                act = 2;
                leaf = h - T.nleaves;
                nr = T.leaf_run[leaf + 1] - T.leaf_run[leaf];
            } else {
                act = 1;
            }
        }
        int push = act == 1 ? 2 : 0;
        int ps = push;
        for (int off = 1; off < 32; off <<= 1) {
            int v = __shfl_up_sync(0xffffffffu, ps, off);
            if (lane >= off) ps += v;
        }
        int ptot = __shfl_sync(0xffffffffu, ps, 31);
        if (sp + ptot > kStack) {
            if (lane == 0) atomicCAS(o.err, 0, KD_EINTERNAL);
            break;
        }
        if (act == 1) {
            st[sp + ps - 2] = 2 * h + 1;
            st[sp + ps - 1] = 2 * h;
        }
        sp += ptot;
        int es = act == 2 ? nr : 0;
        for (int off = 1; off < 32; off <<= 1) {
            int v = __shfl_up_sync(0xffffffffu, es, off);
            if (lane >= off) es += v;
        }
        int etot = __shfl_sync(0xffffffffu, es, 31);
        if (FILL && act == 2) {
            unsigned short codes[KD_WARPS];
            const double *tb = T.box + 6 * (size_t)h;
            for (int ww = 0; ww < KD_WARPS; ww++) {
                if (ww < nw) {
                    int elo, ehi;
                    bin_range(bb + 6 + 6 * ww, tb, rsq, ne, elo, ehi);
                    codes[ww] = (unsigned short)(elo | ((ehi - elo) << 8));
                } else {
                    codes[ww] = (unsigned short)ne;
                }
            }
            int r0 = T.leaf_run[leaf];
            for (int k = 0; k < nr; k++) {
                long long idx = base + emitted + es - nr + k;
                o.run[idx] = (unsigned)(r0 + k);
                uint4 *cp = (uint4 *)(o.code + idx * KD_WARPS);
                uint4 v;
                v.x = codes[0] | ((unsigned)codes[1] << 16);
                v.y = codes[2] | ((unsigned)codes[3] << 16);
                v.z = codes[4] | ((unsigned)codes[5] << 16);
                v.w = codes[6] | ((unsigned)codes[7] << 16);
                *cp = v;
            }
        }
        emitted += etot;
        __syncwarp();
    }
    if (!FILL && lane == 0) o.count[b - b0] = (int)emitted;
    if (FILL) {
        for (int off = 16; off; off >>= 1) acc_pairs += __shfl_xor_sync(0xffffffffu, acc_pairs, off);
        if (lane == 0 && acc_pairs) atomicAdd(o.accepted, acc_pairs);
    }
}

// Rigorous half-width E of the uncertain band around edge R.
// Geometry of a tile: query points within Rq of the warp centre o, tree points
// within hT of their leaf centre c; both sides are re-centred on c in FP32:
//   q' = fl(fl(q - o) - fl(c - o)),   t' = fl(t - c),   T = fl(|t'|^2),
//   s  = fma(q'z, -2t'z, fma(q'y, -2t'y, fma(q'x, -2t'x, T)))   (= |t'-q'|^2 - |q'|^2)
//   a  = fl(A - |q'|^2 / 4E),  A = fl(1/2 + R / 4E),   c = sat(a - s / 4E)
// c is exactly 1 when s is more than 2E below R - |q'|^2, 0 when more than 2E
// above.  Every pair that is counted or lies within E of the edge has
// d2 <= 2R, so |q - c| <= P = sqrt(2R) + hT, and for such pairs the FP32
// quantity s - (R - |q'|^2) differs from d2 - R by at most
//   u32 [ 2 sqrt(2R)(2P + 2Rq + hT) + 4 hT^2 + 6 P hT + 5 P^2 + 3 R ]
// (coordinate rounding 2 sqrt(d2) eta with eta <= u32 (2P + 2Rq + hT), the
// roundings of T, of the FMA chain for s and for |q'|^2, and of the threshold
// a).  E adds 25%, a term for the FP64 reference's own rounding, and is rounded
// up to a power of two so that 1/(4E) is exact in FP32.  Pairs with d2 > 2R
// have an FP32 value far above the band (its error grows like u32 d2).
__device__ __forceinline__ double band_halfwidth(double R, double Rq, double hT)
{
    const double u32 = 5.9604644775390625e-08;  // 2^-24
    const double sr = sqrt(2.0 * R);
    const double P = sr + hT;
    double e = 2.0 * sr * (2.0 * P + 2.0 * Rq + hT) + 4.0 * hT * hT + 6.0 * P * hT +
               5.0 * P * P + 3.0 * R;
    double E = 1.25 * u32 * e + 1e-15 * R + 1e-30;
    int ex;
    frexp(E, &ex);
    return ldexp(1.0, ex);
}

// saturating FMA: clamp(a*b + c, 0, 1) in one instruction (NaN -> 0)
__device__ __forceinline__ float fma_sat(float a, float b, float c)
{
    float d;
    asm("fma.rn.sat.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// FP32 pass of one lane's query over a run and K (<= 4) edges.  Each pair
// gives c_k = sat(a_k + s * nsl_k), exactly 0 or 1 outside the band and in
// [1/4, 3/4] inside it.  sum_k acc_k equals acc2 = sum c^2 bit for bit when
// every c is 0 or 1; a band pair makes them differ by at least 3/16, far
// above the FP32 rounding of these short sums (<= 256 terms of at most 1).
template <int K>
__device__ __forceinline__ bool fp32_run(const float4 *__restrict__ t, int rl, float qx, float qy,
                                         float qz, const float *a, const float *nsl, int *cnt)
{
    float acc[K], acc2 = 0.0f;
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = 0.0f;
    int j = 0;
    for (; j + 2 <= rl; j += 2) {
        const float4 t0 = __ldg(t + j), t1 = __ldg(t + j + 1);
        const float s0 = fmaf(qz, t0.z, fmaf(qy, t0.y, fmaf(qx, t0.x, t0.w)));
        const float s1 = fmaf(qz, t1.z, fmaf(qy, t1.y, fmaf(qx, t1.x, t1.w)));
#pragma unroll
        for (int k = 0; k < K; k++) {
            const float c0 = fma_sat(s0, nsl[k], a[k]);
            const float c1 = fma_sat(s1, nsl[k], a[k]);
            acc[k] += c0;
            acc2 = fmaf(c0, c0, acc2);
            acc[k] += c1;
            acc2 = fmaf(c1, c1, acc2);
        }
    }
    if (j < rl) {
        const float4 t0 = __ldg(t + j);
        const float s0 = fmaf(qz, t0.z, fmaf(qy, t0.y, fmaf(qx, t0.x, t0.w)));
#pragma unroll
        for (int k = 0; k < K; k++) {
            const float c0 = fma_sat(s0, nsl[k], a[k]);
            acc[k] += c0;
            acc2 = fmaf(c0, c0, acc2);
        }
    }
    float tot = 0.0f;
#pragma unroll
    for (int k = 0; k < K; k++) {
        tot += acc[k];
        cnt[k] = __float2int_rn(acc[k]);
    }
    return tot == acc2;
}

// reference-order FP64 distance (kdquery.c:39-47 as compiled)
__device__ __forceinline__ double d2_ref(double tx, double ty, double tz, double qx, double qy,
                                         double qz)
{
    double dx = __dsub_rn(tx, qx), dy = __dsub_rn(ty, qy), dz = __dsub_rn(tz, qz);
    double s = __dmul_rn(dx, dx);
    s = __fma_rn(dy, dy, s);
    return __fma_rn(dz, dz, s);
}

// Exact pass in FP64 with the reference's operation order: cumulative counts
// of pairs with d2 < R[k] for the kn (<= 4) edges, packed one per byte (a run
// has at most KD_RUN_MAX = 64 points).  Used for FP64 mode, band rechecks and
// infinite radii; kept out of line so the FP32 loop stays small.
__device__ __noinline__ unsigned exact_pass(const double *__restrict__ tx,
                                            const double *__restrict__ ty,
                                            const double *__restrict__ tz, int rl, double qx,
                                            double qy, double qz, const double *R, int kn)
{
    int c4[4] = {0, 0, 0, 0};
    for (int j = 0; j < rl; j++) {
        const double d2 = d2_ref(__ldg(tx + j), __ldg(ty + j), __ldg(tz + j), qx, qy, qz);
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (k < kn) c4[k] += d2 < R[k];
    }
    return (unsigned)c4[0] | ((unsigned)c4[1] << 8) | ((unsigned)c4[2] << 16) |
           ((unsigned)c4[3] << 24);
}

struct TileArgs {
    TreeSide T;
    const float4 *t4;     // tree points: (-2t, |t|^2), t relative to the leaf centre
    const int *run_leaf;
    const double *leaf_c; // 3 per leaf
    double hT;            // largest leaf half-diagonal
    QuerySide Q;
    const double *rsq;
    int ne;
    int b0, b1;
    const long long *off;
    const unsigned *run;
    const unsigned short *code;
    unsigned long long *H;
    int Fqe, Fte;
    int *work;
    unsigned long long *stats;  // tested, rechecked, accepted, wide, edge-pairs, warp tiles
};

constexpr int kTileWarps = KD_BLOCK_MAX / 32;

// One warp = one work item: 32 query points (a warp's slice of a query block)
// against that block's list of tree runs.  Warps never wait for each other;
// tree points are read with broadcast loads (the block's 8 warps walk the
// same runs, so they hit in L1).
template <int MODE>
__global__ void __launch_bounds__(32 * kTileWarps, 3) k_tiles(TileArgs A)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int ne = A.ne;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    int *P = (int *)smem;                                           // (ne+1) x 256
    double *R = (double *)(P + (size_t)(ne + 1) * kTileThreads);    // ne
    float *Aw = (float *)(R + KD_MAX_EDGES) + w * 2 * KD_MAX_EDGES; // per warp: A_k
    float *nsl = Aw + KD_MAX_EDGES;                                 //           -1/(4E_k)

    for (int k = tid; k < ne; k += blockDim.x) R[k] = A.rsq[k];
    __syncthreads();
    unsigned long long pairs = 0, rechecked = 0, wide = 0, kpairs = 0, wtiles = 0;
    int *Pt = P + tid;

    while (true) {
        int item = 0;
        if (lane == 0) item = atomicAdd(A.work, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        const int b = A.b0 + item / kTileWarps, wi = item % kTileWarps;
        if (b >= A.b1) break;
        const int qlen = A.Q.blk_len[b] - 32 * wi;
        if (qlen <= 0) continue;
        const int qs = A.Q.blk_start[b] + 32 * wi;
        const long long eoff = A.off[b - A.b0];
        const int ecnt = (int)(A.off[b - A.b0 + 1] - eoff);
        const double *bx = A.Q.blk_wbox + ((size_t)b * KD_WARPS + wi) * 6;
        const double ox = 0.5 * (bx[0] + bx[3]), oy = 0.5 * (bx[1] + bx[4]),
                     oz = 0.5 * (bx[2] + bx[5]);
        const bool valid = lane < qlen;
        double qxd = ox, qyd = oy, qzd = oz;
        int qf = 0;
        if (valid) {
            qxd = A.Q.x[qs + lane];
            qyd = A.Q.y[qs + lane];
            qzd = A.Q.z[qs + lane];
            qf = A.Q.qf[qs + lane];
        }
        const int q0 = __shfl_sync(0xffffffffu, qf, 0);
        const int wq = __all_sync(0xffffffffu, !valid || qf == q0) ? q0 : -1;
        const float qwx = (float)(qxd - ox), qwy = (float)(qyd - oy), qwz = (float)(qzd - oz);
        if (MODE == KD_MODE_MIXED) {
            const double hx = 0.5 * (bx[3] - bx[0]), hy = 0.5 * (bx[4] - bx[1]),
                         hz = 0.5 * (bx[5] - bx[2]);
            const double Rq = sqrt(hx * hx + hy * hy + hz * hz) * (1.0 + 1e-12);
            for (int k = lane; k < ne; k += 32) {
                if (isfinite(R[k])) {
                    const double inv4e = 0.25 / band_halfwidth(R[k], Rq, A.hT);
                    nsl[k] = (float)(-inv4e);
                    Aw[k] = (float)(0.5 + R[k] * inv4e);
                } else {
                    nsl[k] = 0.0f;
                    Aw[k] = 0.0f;
                }
            }
        }
        for (int e = 0; e <= ne; e++) Pt[(size_t)e * kTileThreads] = 0;
        __syncwarp();
        int cur_tf = -1;
        long long since = 0;

        auto flush = [&](int tf) {
            for (int e = 0; e < ne; e++) {
                int v = Pt[(size_t)e * kTileThreads];
                Pt[(size_t)e * kTileThreads] = 0;
                if (wq >= 0) {
                    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                    if (lane == 0 && v)
                        atomicAdd(&A.H[((size_t)e * A.Fqe + wq) * A.Fte + tf], (unsigned long long)v);
                } else if (valid && v) {
                    atomicAdd(&A.H[((size_t)e * A.Fqe + qf) * A.Fte + tf], (unsigned long long)v);
                }
            }
            Pt[(size_t)ne * kTileThreads] = 0;
        };

        for (int i = 0; i < ecnt; i++) {
            const unsigned code = A.code[(eoff + i) * KD_WARPS + wi];
            const int k0 = code & 0xFF, K = code >> 8;
            if (k0 >= ne) continue;  // beyond every edge for this warp
            const unsigned run = A.run[eoff + i];
            const int rs = A.T.run_start[run], rl = A.T.run_len[run], tf = A.T.run_tf[run];
            if (tf != cur_tf || since > (1LL << 30)) {
                if (cur_tf >= 0) flush(cur_tf);
                cur_tf = tf;
                since = 0;
            }
            since += rl;
            if (K == 0) {
                if (valid) Pt[(size_t)k0 * kTileThreads] += rl;
                continue;
            }
            wtiles++;
            // edges k0 .. k0+K-1 in passes of at most four; pairs land in
            // bins k0 .. k0+K (the last: beyond the active edges)
            const bool fp32 = MODE == KD_MODE_MIXED && isfinite(R[k0 + K - 1]);
            float qx = 0.0f, qy = 0.0f, qz = 0.0f, qn = 0.0f;
            if (fp32) {
                const int leaf = A.run_leaf[run];
                const float dx = (float)(A.leaf_c[3 * (size_t)leaf] - ox);
                const float dy = (float)(A.leaf_c[3 * (size_t)leaf + 1] - oy);
                const float dz = (float)(A.leaf_c[3 * (size_t)leaf + 2] - oz);
                qx = qwx - dx;
                qy = qwy - dy;
                qz = qwz - dz;
                qn = fmaf(qz, qz, fmaf(qy, qy, qx * qx));
            }
            if (!valid) continue;
            int prev = 0;
            for (int kb = 0; kb < K; kb += 4) {
                const int kn = min(4, K - kb);
                int cnt[4] = {0, 0, 0, 0};
                bool ok = false;
                if (fp32) {
                    float a[4], sl[4];
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        sl[k] = k < kn ? nsl[k0 + kb + k] : 0.0f;
                        a[k] = k < kn ? fmaf(qn, sl[k], Aw[k0 + kb + k]) : 0.0f;
                    }
                    const float4 *t = A.t4 + rs;
                    switch (kn) {
                    case 1: ok = fp32_run<1>(t, rl, qx, qy, qz, a, sl, cnt); break;
                    case 2: ok = fp32_run<2>(t, rl, qx, qy, qz, a, sl, cnt); break;
                    case 3: ok = fp32_run<3>(t, rl, qx, qy, qz, a, sl, cnt); break;
                    default: ok = fp32_run<4>(t, rl, qx, qy, qz, a, sl, cnt); break;
                    }
                    if (!ok) rechecked += rl;
                }
                if (!ok) {
                    const unsigned pk = exact_pass(A.T.x + rs, A.T.y + rs, A.T.z + rs, rl, qxd, qyd,
                                                   qzd, R + k0 + kb, kn);
#pragma unroll
                    for (int k = 0; k < 4; k++) cnt[k] = (pk >> (8 * k)) & 0xFF;
                }
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (k < kn) {
                        Pt[(size_t)(k0 + kb + k) * kTileThreads] += cnt[k] - prev;
                        prev = cnt[k];
                    }
            }
            Pt[(size_t)(k0 + K) * kTileThreads] += rl - prev;
            if (K > 4) wide += rl;
            kpairs += (unsigned long long)rl * K;
            pairs += rl;
        }
        if (cur_tf >= 0) flush(cur_tf);
        __syncwarp();
    }
    for (int o = 16; o; o >>= 1) {
        pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
        rechecked += __shfl_xor_sync(0xffffffffu, rechecked, o);
        wide += __shfl_xor_sync(0xffffffffu, wide, o);
        kpairs += __shfl_xor_sync(0xffffffffu, kpairs, o);
    }
    if (lane == 0) {
        if (pairs) atomicAdd(&A.stats[0], pairs);
        if (rechecked) atomicAdd(&A.stats[1], rechecked);
        if (wide) atomicAdd(&A.stats[3], wide);
        if (kpairs) atomicAdd(&A.stats[4], kpairs);
        if (wtiles) atomicAdd(&A.stats[5], wtiles);
    }
}

static size_t tile_smem(int ne, int mode)
{
    (void)mode;
    return sizeof(int) * (size_t)(ne + 1) * kTileThreads + sizeof(double) * KD_MAX_EDGES +
           sizeof(float) * 2 * KD_MAX_EDGES * kTileWarps;
}

struct Events {
    cudaEvent_t e[8];
    Events()
    {
        for (auto &x : e) check(cudaEventCreate(&x), "cudaEventCreate");
    }
    ~Events()
    {
        for (auto &x : e) cudaEventDestroy(x);
    }
};

static float elapsed(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

static void count_impl(const kd_catalog *tc, const kd_catalog *qc, const double *h_rsq, int ne,
                       int mode, long long *hist, kd_count_stats *stats)
{
    init_device();
    Stream st;
    cudaStream_t s = st.s;
    Pool pool(s);
    Events ev;
    int launches = 0, tile_launches = 0;

    TreeSide T;
    T.x = tc->d_x;
    T.y = tc->d_y;
    T.z = tc->d_z;
    T.box = tc->d_box;
    T.count = tc->d_ncount;
    T.tf = tc->d_ntf;
    T.leaf_run = tc->d_leaf_run;
    T.run_start = tc->d_run_start;
    T.run_len = tc->d_run_len;
    T.run_tf = tc->d_run_tf;
    T.D = tc->depth;
    T.nleaves = tc->nleaves;
    QuerySide Q;
    Q.x = qc->d_x;
    Q.y = qc->d_y;
    Q.z = qc->d_z;
    Q.qf = qc->d_qf;
    Q.blk_start = qc->d_blk_start;
    Q.blk_len = qc->d_blk_len;
    Q.blk_qf = qc->d_blk_qf;
    Q.blk_box = qc->d_blk_box;
    Q.blk_wbox = qc->d_blk_wbox;

    const int Fqe = qc->max_qf + 1, Fte = tc->max_tf + 1;
    const size_t hsz = (size_t)(ne + 1) * Fqe * Fte;
    unsigned long long *H = pool.alloc<unsigned long long>(hsz);
    unsigned long long *dstats = pool.alloc<unsigned long long>(8);
    int *err = pool.alloc<int>(1);
    int *work = pool.alloc<int>(1);
    double *rsq = pool.alloc<double>(std::max(ne, 1));
    check(cudaEventRecord(ev.e[0], s), "event");
    check(cudaMemsetAsync(H, 0, sizeof(unsigned long long) * hsz, s), "memset");
    check(cudaMemsetAsync(dstats, 0, sizeof(unsigned long long) * 8, s), "memset");
    check(cudaMemsetAsync(err, 0, sizeof(int), s), "memset");
    check(cudaMemcpyAsync(rsq, h_rsq, sizeof(double) * ne, cudaMemcpyHostToDevice, s), "H2D");

    const int nb = qc->nblocks;
    int *cnt = pool.alloc<int>(nb);
    TravOut to;
    memset(&to, 0, sizeof to);
    to.count = cnt;
    to.H = H;
    to.Fqe = Fqe;
    to.Fte = Fte;
    to.accepted = dstats + 2;
    to.err = err;
    unsigned tgrid = blocks_for(nb, kTravWarps);
    k_traverse<false><<<tgrid, 32 * kTravWarps, 0, s>>>(T, Q, rsq, ne, 0, nb, to);
    launches++;
    KD_LAUNCH_CHECK("k_traverse(count)");
    std::vector<int> hcnt(nb);
    check(cudaMemcpyAsync(hcnt.data(), cnt, sizeof(int) * (size_t)nb, cudaMemcpyDeviceToHost, s),
          "D2H");
    st.sync();
    int herr = 0;
    check(cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost), "D2H");
    if (herr) raise(herr, "node-pair traversal exceeded its stack");

    // batches of query blocks whose tiles fit the tile buffer
    long long total = 0;
    for (int v : hcnt) total += v;
    size_t freeb = 0, totb = 0;
    cudaMemGetInfo(&freeb, &totb);
    long long cap = std::max<long long>(1 << 20, std::min<long long>(256LL << 20, (long long)(freeb / 4 / 20)));
    cap = std::min<long long>(cap, std::max<long long>(total, 1));
    unsigned *run = pool.alloc<unsigned>(cap);
    unsigned short *code = pool.alloc<unsigned short>(cap * KD_WARPS);
    long long *off = pool.alloc<long long>(nb + 1);
    std::vector<long long> hoff(nb + 1);

    size_t smem = tile_smem(ne, mode);
    auto kern = mode == KD_MODE_MIXED ? k_tiles<KD_MODE_MIXED> : k_tiles<KD_MODE_FP64>;
    check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
          "smem attribute");
    int dev = 0, nsm = 148, occ = 1;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kTileThreads, smem), "occupancy");
    occ = std::max(occ, 1);

    float ms_trav = 0, ms_tiles = 0;
    int b0 = 0;
    while (b0 < nb) {
        long long acc = 0;
        int b1 = b0;
        hoff[0] = 0;
        while (b1 < nb && (b1 == b0 || acc + hcnt[b1] <= cap)) {
            acc += hcnt[b1];
            b1++;
            hoff[b1 - b0] = acc;
        }
        check(cudaMemcpyAsync(off, hoff.data(), sizeof(long long) * (size_t)(b1 - b0 + 1),
                              cudaMemcpyHostToDevice, s), "H2D");
        TravOut tf = to;
        tf.off = off;
        tf.run = run;
        tf.code = code;
        check(cudaEventRecord(ev.e[1], s), "event");
        k_traverse<true><<<blocks_for(b1 - b0, kTravWarps), 32 * kTravWarps, 0, s>>>(T, Q, rsq, ne,
                                                                                      b0, b1, tf);
        launches++;
        KD_LAUNCH_CHECK("k_traverse(fill)");
        check(cudaEventRecord(ev.e[2], s), "event");
        TileArgs ta;
        ta.T = T;
        ta.t4 = (const float4 *)tc->d_t4;
        ta.run_leaf = tc->d_run_leaf;
        ta.leaf_c = tc->d_leaf_c;
        ta.hT = tc->leaf_hdiag * (1.0 + 1e-12);
        ta.Q = Q;
        ta.rsq = rsq;
        ta.ne = ne;
        ta.b0 = b0;
        ta.b1 = b1;
        ta.off = off;
        ta.run = run;
        ta.code = code;
        ta.H = H;
        ta.Fqe = Fqe;
        ta.Fte = Fte;
        ta.work = work;
        ta.stats = dstats;
        check(cudaMemsetAsync(work, 0, sizeof(int), s), "memset");
        int grid = (int)std::min<long long>((long long)(b1 - b0), (long long)nsm * occ);
        kern<<<grid, kTileThreads, smem, s>>>(ta);
        launches++;
        tile_launches++;
        KD_LAUNCH_CHECK("k_tiles");
        check(cudaEventRecord(ev.e[3], s), "event");
        st.sync();
        ms_trav += elapsed(ev.e[1], ev.e[2]);
        ms_tiles += elapsed(ev.e[2], ev.e[3]);
        b0 = b1;
    }
    check(cudaEventRecord(ev.e[4], s), "event");
    std::vector<unsigned long long> hh(hsz);
    unsigned long long hs[8];
    check(cudaMemcpyAsync(hh.data(), H, sizeof(unsigned long long) * hsz, cudaMemcpyDeviceToHost, s),
          "D2H");
    check(cudaMemcpyAsync(hs, dstats, sizeof hs, cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    st.sync();
    if (herr) raise(herr, "node-pair traversal exceeded its stack");
    for (size_t i = 0; i < hsz; i++) hist[i] = (long long)hh[i];
    if (stats) {
        stats->pairs_tested = (long long)hs[0];
        stats->pairs_rechecked = (long long)hs[1];
        stats->pairs_accepted = (long long)hs[2];
        stats->pairs_wide = (long long)hs[3];
        stats->edge_pairs = (long long)hs[4];
        stats->warp_tiles = (long long)hs[5];
        stats->entries = total;
        stats->ms_traverse = ms_trav + 0.0;
        stats->ms_tiles = ms_tiles;
        stats->ms_total = elapsed(ev.e[0], ev.e[4]);
        stats->tile_launches = tile_launches;
        stats->launches = launches;
    }
}

}  // namespace kd

extern "C" int kdg_count(const kd_catalog *tree, const kd_catalog *query, const double *rsq,
                         int ne, int mode, long long *hist, kd_count_stats *stats)
{
    if (ne < 1 || ne > KD_MAX_EDGES) {
        kd_set_error(KD_EINVAL, "between 1 and %d distinct radii per count", KD_MAX_EDGES);
        return KD_EINVAL;
    }
    try {
        kd::count_impl(tree, query, rsq, ne, mode, hist, stats);
        return KD_OK;
    } catch (const kd::Error &e) {
        kd_set_error(e.code, "%s", e.msg);
        return e.code;
    }
}
