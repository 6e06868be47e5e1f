// Pair counting for corruscant's pair_count (kdquery.c:62-113, :165-249),
// batched over all bin edges at once.
//
// Semantics kept from the reference: the reference traversal counts, for
// every query point q and every tree node t, weight(t) if fl(d2) < fl(r*r),
// where d2 is evaluated as
//     dx = t.x - q.x, ...;  d2 = dx*dx;  d2 = fma(dy,dy,d2);  d2 = fma(dz,dz,d2)
// (kdquery.c:39-47 as the reference build compiles it), and its pruning
// (kdquery.c:96-104) never drops such a pair.  Here a pair lands in bin e, the
// first sorted squared edge with d2 < rsq[e]; cumulative sums over e give the
// reference's per-radius counts.
//
// Work decomposition (B200-first, not the reference's per-query recursion):
//   k_traverse : one warp per query block (<= 128 points) walks the tree-side
//                counting tree with box-box distance bounds.  Node pairs
//                beyond the last edge are pruned, node pairs inside one bin
//                are accepted as count(block) x count(node), and leaf pairs
//                become tile records (tree run, active edge range).  Run twice:
//                once to count the tiles, once to write them.
//   k_tiles    : one warp per query block, four query points per lane, walks
//                its tile records.  Each tree run is staged into the warp's
//                shared memory (the next run's loads already in flight) and
//                every staged point is compared with the lane's four queries.
//                Mixed mode: FP32 distances relative to the block centre,
//                binned against the active edges with a saturating ramp that
//                is exactly 0 or 1 outside a rigorous error band; a query
//                with any pair of the run inside the band is recounted in
//                FP64 with the reference's operation order.  FP64 mode: every
//                distance in FP64.  Per-query bin counters live in shared
//                memory and are reduced per (own field) into the global
//                (bin, qfield, tfield) histogram when the tree field changes.

#include <algorithm>
#include <exception>
#include <new>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <mutex>
#include <vector>

#include "kd_cuda_util.cuh"
#include "kd_sort.cuh"

namespace kd {

constexpr int kTravWarps = 4;
// Node-pair stack per traversal warp.  A round pops the top min(sp, 32)
// entries and pushes at most two children for each, so the stack grows by at
// most 32 entries per tree level: at most 32 * D + 64 entries for a counting
// tree of depth D <= 24 (832).  A push past the end stops the count with
// KD_EINTERNAL instead of writing out of bounds.  4 KB per warp (rather
// than 8) lets the count pass run more warps per SM: the traversal of the
// clustered 1M / 20M batch takes 16.3 ms instead of 19.5.
constexpr int kStack = 1024;
static_assert(kStack >= 32 * 24 + 64, "stack bound of a depth-24 counting tree");
constexpr int kQ = KD_QPL;              // query points per lane
constexpr int kTileWarpsPerCta = 4;
constexpr int kMaxDistinctQf = 8;       // own fields reduced per warp at a flush
constexpr int kPass32 = 4;              // edges per FP32 pass (register budget)
constexpr int kStageMax = KD_RUN_MAX;  // points staged per pass

constexpr int kCoopMax = 32;            // rechecks of a run done by the whole warp
constexpr int kShardChunk = 32;         // blocks per interleaved shard chunk
constexpr int kRunPerLane = KD_RUN_MAX / 32;  // staged run points per lane
// FP32 tiles only where every staged value and square stays far inside FP32
// range: tree and query points within kFp32Span of the block centre (their
// squares and products below 1e30 < FLT_MAX) and squared edges below 1e30.
// Records beyond that (coordinates or radii of 1e15 and more) are counted
// by the exact FP64 path, as infinite radii are.
constexpr double kFp32Span = 1e15;
constexpr double kFp32MaxR = 1e30;
// A run's exact counts travel one per byte (recounts) and its FP32 band sums
// stay small (at most 4 * KD_RUN_MAX terms in [0, 1]): both need short runs.
static_assert(KD_RUN_MAX % 32 == 0 && KD_RUN_MAX <= 128, "runs of 32..128 points");

struct TreeSide {
    const double *box;
    const int *count, *tf, *leaf_run, *leaf_pos;
    const int *run_start, *run_len, *run_tf;
    int D, nleaves;
};

struct QuerySide {
    const double *x, *y, *z;
    const int *qf;
    const int *blk_start, *blk_len, *blk_qf;
    const double *blk_box;
};

// One (tree, query tree) count of a batch.  A batch numbers the query blocks
// of all its jobs consecutively: job j owns global blocks [jblk[j], jblk[j+1]).
struct JobDesc {
    TreeSide T;
    QuerySide Q;
    const double *tx, *ty, *tz;  // tree points, FP64, counting order
    const float4 *t4;            // tree points: (-2 t_r, |t_r|^2), t_r relative to leaf centre
    const double *leaf_c;        // 3 per leaf
    double hT;                   // largest leaf half-diagonal, with margin
    unsigned long long *H;       // (ne + 1) x Fqe x Fte bin histogram
    // Symmetric job (tree and query are one catalog whose points all have own
    // field == tree field): a block counts only tree points at or after its
    // own first point; points inside the block as ordered pairs into H, points
    // after it once into H2, and the host adds H2 and its field transpose.
    unsigned long long *H2;
    int Fqe, Fte;
    int sym, pad_;
};
static_assert(sizeof(JobDesc) % 8 == 0, "JobDesc is copied in 8-byte words");

// the job owning global block g: the last j with jblk[j] <= g (an empty job
// shares its start with the next one, which is then the one found)
__device__ __forceinline__ int job_of(const int *__restrict__ jblk, int njobs, int g)
{
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jblk[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

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

// A tile record: x = run start, y = leaf, z = run length | tree field << 8 |
// first active edge << 16 | active edge count << 24.
struct TravOut {
    const int *gmap;         // shard-local block index -> global block (NULL: identity)
    int *count;              // COUNT pass: tiles per block
    const long long *off;    // FILL pass: launch-relative tile offsets
    uint4 *rec;              // FILL: tile records
    unsigned long long *accepted;
    int *err;
};

// one warp per shard-local block index i in [g0, g1) (global block o.gmap[i])
template <bool FILL>
__global__ void __launch_bounds__(32 * kTravWarps) k_traverse(const JobDesc *__restrict__ jobs,
                                                             const int *__restrict__ jblk,
                                                             int njobs,
                                                             const double *__restrict__ g_rsq,
                                                             int ne, int g0, int g1, TravOut o)
{
    __shared__ int stack[kTravWarps][kStack];
    __shared__ double rsq[KD_MAX_EDGES];
    __shared__ double wb[kTravWarps][6];
    for (int k = threadIdx.x; k < ne; k += blockDim.x) rsq[k] = g_rsq[k];
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int li = g0 + blockIdx.x * kTravWarps + w;
    if (li >= g1) return;
    const int g = o.gmap ? o.gmap[li] : li;
    const int j = job_of(jblk, njobs, g);
    const int b = g - jblk[j];
    const TreeSide T = jobs[j].T;
    const QuerySide Q = jobs[j].Q;
    unsigned long long *const H = jobs[j].H, *const H2 = jobs[j].H2;
    const int Fqe = jobs[j].Fqe, Fte = jobs[j].Fte;
    const bool sym = jobs[j].sym != 0;
    const int alen = Q.blk_len[b], aqf = Q.blk_qf[b];
    const int qb0 = Q.blk_start[b], qb1 = qb0 + alen;  // the block's raw positions
    double *bb = wb[w];
    if (lane < 6) bb[lane] = Q.blk_box[6 * (size_t)b + lane];
    int *st = stack[w];
    if (lane == 0) st[0] = 1;
    __syncwarp();
    int sp = 1;
    long long emitted = 0;
    const long long base = FILL ? o.off[li - g0] : 0;
    unsigned long long acc_pairs = 0, blocked_pairs = 0;
    long long guard = 4LL * T.nleaves + 64;
    while (sp > 0) {
        if (--guard < 0) {
            if (lane == 0) atomicCAS(o.err, 0, KD_EINTERNAL);
            break;
        }
        const int nb = min(sp, 32);
        const int h = lane < nb ? st[sp - nb + lane] : 0;
        __syncwarp();
        sp -= nb;
        int act = 0, nr = 0, leaf = 0, elo = 0, ehi = 0;
        if (h) {
            // symmetric jobs: the node's raw positions [nlo, nhi) against the
            // block's [qb0, qb1): before it -> nothing (the other side's block
            // counts these pairs), after it -> once into H2, overlapping ->
            // descend, runs cut at the block's ends
            int nlo = 0, nhi = 0;
            if (sym) {
                const int sh = T.D - (31 - __clz(h));
                nlo = T.leaf_pos[(h << sh) - T.nleaves];
                nhi = T.leaf_pos[((h + 1) << sh) - T.nleaves];
            }
            const bool after = sym && nlo >= qb1;
            if (sym && nhi <= qb0) {
                act = 0;
            } else {
                bin_range(bb, T.box + 6 * (size_t)h, rsq, ne, elo, ehi);
                const bool whole = !sym || after || (nlo >= qb0 && nhi <= qb1);
                if (elo >= ne) {
                    act = 0;
                } else if (whole && elo == ehi && aqf >= 0 && T.tf[h] >= 0) {
                    if (FILL) {
                        const unsigned long long c =
                            (unsigned long long)alen * (unsigned long long)T.count[h];
                        atomicAdd(&(after ? H2 : H)[((size_t)elo * Fqe + aqf) * Fte + T.tf[h]], c);
                        acc_pairs += c;
                    }
                } else if (h >= T.nleaves) {
                    // pairs of a node pair inside one bin that are tiled only
                    // because a side holds several fields (a per-field accept
                    // would take them without distances)
                    if (FILL && whole && elo == ehi)
                        blocked_pairs += (unsigned long long)alen * (unsigned long long)T.count[h];
                    act = 2;
                    leaf = h - T.nleaves;
                    const int r0 = T.leaf_run[leaf], r1 = T.leaf_run[leaf + 1];
                    if (!sym) {
                        nr = r1 - r0;
                    } else {
                        for (int r = r0; r < r1; r++) {
                            const int a = T.run_start[r], e = a + T.run_len[r];
                            nr += (max(a, qb0) < min(e, qb1)) + (max(a, qb1) < e);
                        }
                    }
                } else {
                    act = 1;
                }
            }
        }
        int ps = act == 1 ? 2 : 0;
        for (int off = 1; off < 32; off <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, ps, off);
            if (lane >= off) ps += v;
        }
        const int ptot = __shfl_sync(0xffffffffu, ps, 31);
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
            const int v = __shfl_up_sync(0xffffffffu, es, off);
            if (lane >= off) es += v;
        }
        const int etot = __shfl_sync(0xffffffffu, es, 31);
        if (FILL && act == 2) {
            const unsigned code = (unsigned)elo | ((unsigned)(ehi - elo) << 8);
            const int r0 = T.leaf_run[leaf], r1 = T.leaf_run[leaf + 1];
            long long idx = base + emitted + es - nr;
            // record: start, leaf, length | tree field << 8 | edges << 16, and
            // w = 1 for the once-counted (H2) part of a symmetric job
            auto put = [&](int a, int len, int tf, unsigned once) {
                o.rec[idx++] = make_uint4((unsigned)a, (unsigned)leaf,
                                          (unsigned)len | ((unsigned)tf << 8) | (code << 16), once);
            };
            for (int r = r0; r < r1; r++) {
                const int a = T.run_start[r], e = a + T.run_len[r];
                if (!sym) {
                    put(a, e - a, T.run_tf[r], 0u);
                } else {
                    const int ia = max(a, qb0), ib = min(e, qb1), aa = max(a, qb1);
                    if (ia < ib) put(ia, ib - ia, T.run_tf[r], 0u);
                    if (aa < e) put(aa, e - aa, T.run_tf[r], 1u);
                }
            }
        }
        emitted += etot;
        __syncwarp();
    }
    if (!FILL && lane == 0) o.count[li - g0] = (int)emitted;
    if (FILL) {
        for (int off = 16; off; off >>= 1) {
            acc_pairs += __shfl_xor_sync(0xffffffffu, acc_pairs, off);
            blocked_pairs += __shfl_xor_sync(0xffffffffu, blocked_pairs, off);
        }
        if (lane == 0 && acc_pairs) atomicAdd(o.accepted, acc_pairs);
        if (lane == 0 && blocked_pairs) atomicAdd(o.accepted + 4, blocked_pairs);
    }
}

// Rigorous half-width E of the uncertain band around edge R.
// Geometry of a tile: query points within Rq of the block centre o; a tree
// point t is stored as t_r = fl32(t - c) (c: its leaf's centre, |t - c| <= hT)
// and staged as t' = fl32(t_r + fl32(c - o)); the query as q' = fl32(q - o);
//   T = |t'|^2 (FP32 FMA chain),  s = T - 2 q'.t' (FP32 FMA chain),
//   thr = R - |q'|^2,  c = sat(a - s/4E) with a = fl(A - |q'|^2/4E),
//   A = fl(1/2 + R/4E).
// c is exactly 1 when s is more than 2E below thr and 0 when more than 2E
// above.  Every pair that is counted or lies within E of the edge has
// d2 <= 2R, so |t - o| <= P = sqrt(2R) + Rq, and for such pairs
//   |(s - thr) - (d2 - R)| <= u32 [2 (P + Rq)(2P + 2hT + Rq) + 6 P (P + Rq)
//                                  + 3 (R + Rq^2)]
// (coordinate rounding 2 sqrt(d2) eta with eta <= u32 (2P + 2hT + Rq), the
// roundings of T and of the FMA chain for s, and those of the threshold).
// E adds 25% and a term for the FP64 reference's own rounding, and is rounded
// up to a power of two so that 1/(4E) is exact in FP32.  Pairs with d2 > 2R
// sit far above the band: their FP32 error grows only like 10 u32 d2.
__device__ __forceinline__ double band_halfwidth(double R, double Rq, double hT)
{
    const double u32 = 5.9604644775390625e-08;  // 2^-24
    const double P = sqrt(2.0 * R) + Rq;
    const double e = 2.0 * (P + Rq) * (2.0 * P + 2.0 * hT + Rq) + 6.0 * P * (P + Rq) +
                     3.0 * (R + Rq * Rq);
    const double E = 1.25 * u32 * e + 1e-15 * R + 1e-30;
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

// FP32 pass of a lane's four queries over a staged run and K (<= 4) edges.
// Each pair gives c = sat(a_k + s * nsl_k): exactly 0 or 1 outside the band,
// in [1/4, 3/4] inside it.  Per query, sum_k acc_k equals acc2 = sum c^2 bit
// for bit when every c is 0 or 1; a band pair makes them differ by at least
// 3/16, far above the FP32 rounding of these short sums (at most
// 4 * kStageMax <= 512 terms in [0, 1]: each sum is off by at most
// 512 * 512 * 2^-24 = 1/64).
// Queries travel in pairs through the packed FP32 pipe (FFMA2/FADD2: two
// independent round-to-nearest operations per instruction, the same values
// as the scalar chain); the saturating ramp has no packed form and stays
// scalar.  A staged point is (X, X, Y, Y), (Z, Z, N, N): each coordinate
// twice, so one 16-byte shared load feeds both halves of a pair.
// Returns a bit mask of the queries with a band pair.
template <int K>
__device__ __forceinline__ unsigned fp32_run(const float4 *__restrict__ ts, int rl,
                                             const float2 (&qx)[kQ / 2],
                                             const float2 (&qy)[kQ / 2],
                                             const float2 (&qz)[kQ / 2],
                                             const float (&a)[kQ][kPass32],
                                             const float (&nsl)[kPass32],
                                             unsigned (&pc)[kQ / 2][4])
{
    float2 acc[kQ / 2][K], acc2[kQ / 2];
#pragma unroll
    for (int h = 0; h < kQ / 2; h++) {
        acc2[h] = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int k = 0; k < K; k++) acc[h][k] = make_float2(0.0f, 0.0f);
    }
    auto point = [&](const float4 xy, const float4 zn) {
        const float2 X = make_float2(xy.x, xy.y), Y = make_float2(xy.z, xy.w);
        const float2 Z = make_float2(zn.x, zn.y), N = make_float2(zn.z, zn.w);
#pragma unroll
        for (int h = 0; h < kQ / 2; h++) {
            const float2 s = __ffma2_rn(qz[h], Z, __ffma2_rn(qy[h], Y, __ffma2_rn(qx[h], X, N)));
#pragma unroll
            for (int k = 0; k < K; k++) {
                const float2 c = make_float2(fma_sat(s.x, nsl[k], a[2 * h][k]),
                                             fma_sat(s.y, nsl[k], a[2 * h + 1][k]));
                acc[h][k] = __fadd2_rn(acc[h][k], c);
                acc2[h] = __ffma2_rn(c, c, acc2[h]);
            }
        }
    };
    int j = 0;
    for (; j + 4 <= rl; j += 4) {
        const float4 t0 = ts[2 * j], t1 = ts[2 * j + 1], t2 = ts[2 * j + 2], t3 = ts[2 * j + 3];
        const float4 t4 = ts[2 * j + 4], t5 = ts[2 * j + 5], t6 = ts[2 * j + 6], t7 = ts[2 * j + 7];
        point(t0, t1);
        point(t2, t3);
        point(t4, t5);
        point(t6, t7);
    }
    for (; j < rl; j++) point(ts[2 * j], ts[2 * j + 1]);
    // Counts without the conversion unit: v + 1.5 * 2^23 lands on the integer
    // grid of that binade, so the low 16 bits of its pattern are round(v)
    // (0 <= v <= 256; the bias 0x4B400000 has zero low half).  The two
    // queries of a pair are packed as (query 2h) | (query 2h + 1) << 16.
    const float2 bias = make_float2(12582912.0f, 12582912.0f);
    unsigned band = 0;
#pragma unroll
    for (int h = 0; h < kQ / 2; h++) {
        float2 tot = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int k = 0; k < K; k++) {
            tot = __fadd2_rn(tot, acc[h][k]);
            const float2 b = __fadd2_rn(acc[h][k], bias);
            pc[h][k] = __byte_perm(__float_as_uint(b.x), __float_as_uint(b.y), 0x5410);
        }
        if (tot.x != acc2[h].x) band |= 1u << (2 * h);
        if (tot.y != acc2[h].y) band |= 2u << (2 * h);
    }
    return band;
}

// reference-order FP64 distance (kdquery.c:39-47 as compiled)
__device__ __forceinline__ double d2_ref(double tx, double ty, double tz, double qx, double qy,
                                         double qz)
{
    const double dx = __dsub_rn(tx, qx), dy = __dsub_rn(ty, qy), dz = __dsub_rn(tz, qz);
    double s = __dmul_rn(dx, dx);
    s = __fma_rn(dy, dy, s);
    return __fma_rn(dz, dz, s);
}

// FP64 pass of the four queries over a staged run (FP64 mode): cumulative
// counts for K (<= 4) edges.
template <int K>
__device__ __forceinline__ void fp64_run(const double *__restrict__ tx,
                                         const double *__restrict__ ty,
                                         const double *__restrict__ tz, int rl,
                                         const double (&qx)[kQ], const double (&qy)[kQ],
                                         const double (&qz)[kQ], const double *R,
                                         int (&cnt)[kQ][4])
{
    double r[K];
#pragma unroll
    for (int k = 0; k < K; k++) r[k] = R[k];
#pragma unroll
    for (int p = 0; p < kQ; p++)
#pragma unroll
        for (int k = 0; k < 4; k++) cnt[p][k] = 0;
    for (int j = 0; j < rl; j++) {
        const double x = tx[j], y = ty[j], z = tz[j];
#pragma unroll
        for (int p = 0; p < kQ; p++) {
            const double d2 = d2_ref(x, y, z, qx[p], qy[p], qz[p]);
#pragma unroll
            for (int k = 0; k < K; k++) cnt[p][k] += d2 < r[k];
        }
    }
}

// Warp-cooperative exact recount of one query over a run: every lane takes
// the points j = lane, lane + 32, ... (at most KD_RUN_MAX / 32, so the warp
// sum of each per-edge count is at most KD_RUN_MAX <= 128: the four
// byte-packed counts add without carries in one reduction).  Returns the
// packed counts in all lanes.
__device__ __noinline__ unsigned exact_pass_warp(const double *__restrict__ tx,
                                                 const double *__restrict__ ty,
                                                 const double *__restrict__ tz, int rl,
                                                 double qx, double qy, double qz,
                                                 const double *R, int kn, int lane)
{
    unsigned part = 0;
    for (int j = lane; j < rl; j += 32) {
        const double d2 = d2_ref(__ldg(tx + j), __ldg(ty + j), __ldg(tz + j), qx, qy, qz);
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (k < kn) part += (unsigned)(d2 < R[k]) << (8 * k);
    }
    return __reduce_add_sync(0xffffffffu, part);
}

// Exact recount of one query over a run (global FP64 coordinates), for band
// rechecks and edges FP32 cannot represent; counts packed one per byte.  Out
// of line so the FP32 loop stays small.
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
    const JobDesc *jobs;
    const int *jblk;
    int njobs;
    const double *rsq;
    int ne;
    int g0, g1;                 // shard-local block indices of this launch
    const int *gmap;            // shard-local index -> global block (NULL: identity)
    const long long *off;       // launch-relative tile offsets
    const uint4 *rec;
    int *work;
    unsigned long long *stats;  // tested, rechecked, accepted, wide, edge-pairs, warp tiles
};

// shared memory of one warp
template <int MODE> struct WarpSmem {
    JobDesc job;  // the job of the block being counted
    float Aw[KD_MAX_EDGES];
    float nsl[KD_MAX_EDGES];
    double cmax2;  // squared leaf-centre distance below which FP32 is safe
    int uq[kMaxDistinctQf];
    float4 stage[MODE == KD_MODE_MIXED ? 2 * kStageMax : 1];  // (X,X,Y,Y), (Z,Z,N,N)
    double stage64[MODE == KD_MODE_FP64 ? 3 * KD_RUN_MAX : 1];
};

template <int MODE>
__global__ void __launch_bounds__(32 * kTileWarpsPerCta, 4) k_tiles(TileArgs A)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int ne = A.ne;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *R = (double *)smem;  // ne
    WarpSmem<MODE> *ws = (WarpSmem<MODE> *)(R + KD_MAX_EDGES) + w;
    // per-query bin counters, two queries per word, 16 bits each (a flush
    // empties them before any could pass 65535): P[(e * kQ / 2 + h) * 32 + lane]
    // holds queries 2h (low half) and 2h + 1 (high half)
    unsigned *P = (unsigned *)((WarpSmem<MODE> *)(R + KD_MAX_EDGES) + kTileWarpsPerCta) +
                  (size_t)w * (ne + 1) * (kQ / 2) * 32;
    for (int k = threadIdx.x; k < ne; k += blockDim.x) R[k] = A.rsq[k];
    __syncthreads();
    unsigned long long pairs = 0, rechecked = 0, wide = 0, kpairs = 0, wtiles = 0;

    while (true) {
        int item = 0;
        if (lane == 0) item = atomicAdd(A.work, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        const int li = A.g0 + item;
        if (li >= A.g1) break;
        const int g = A.gmap ? A.gmap[li] : li;
        const int jb = job_of(A.jblk, A.njobs, g);
        {
            const unsigned long long *src = (const unsigned long long *)(A.jobs + jb);
            unsigned long long *dst = (unsigned long long *)&ws->job;
            for (int u = lane; u < (int)(sizeof(JobDesc) / 8); u += 32) dst[u] = src[u];
            __syncwarp();
        }
        const JobDesc &J = ws->job;
        const int b = g - A.jblk[jb];
        const int qlen = J.Q.blk_len[b], qs = J.Q.blk_start[b];
        const long long eoff = A.off[li - A.g0];
        const int ecnt = (int)(A.off[li - A.g0 + 1] - eoff);
        const double *bx = J.Q.blk_box + 6 * (size_t)b;
        const double ox = 0.5 * (bx[0] + bx[3]), oy = 0.5 * (bx[1] + bx[4]),
                     oz = 0.5 * (bx[2] + bx[5]);
        // queries 4*lane .. 4*lane+3 of the block; their FP64 coordinates and
        // own fields are re-read from global memory when needed (exact
        // recounts, flushes) instead of being held in registers
        const int qbase = qs + kQ * lane;
        float qx[kQ], qy[kQ], qz[kQ], qn[kQ];
        unsigned vmask = 0;
#pragma unroll
        for (int p = 0; p < kQ; p++) {
            const int j = kQ * lane + p;
            const bool v = j < qlen;
            vmask |= (unsigned)v << p;
            const double xd = v ? J.Q.x[qs + j] : ox, yd = v ? J.Q.y[qs + j] : oy,
                         zd = v ? J.Q.z[qs + j] : oz;
            qx[p] = (float)(xd - ox);
            qy[p] = (float)(yd - oy);
            qz[p] = (float)(zd - oz);
            qn[p] = (float)((double)qx[p] * qx[p] + (double)qy[p] * qy[p] + (double)qz[p] * qz[p]);
        }
        const int nvalid = __popc(vmask);
        float2 qx2[kQ / 2], qy2[kQ / 2], qz2[kQ / 2];
#pragma unroll
        for (int h = 0; h < kQ / 2; h++) {
            qx2[h] = make_float2(qx[2 * h], qx[2 * h + 1]);
            qy2[h] = make_float2(qy[2 * h], qy[2 * h + 1]);
            qz2[h] = make_float2(qz[2 * h], qz[2 * h + 1]);
        }
        // half-word masks of the valid queries of each pair (invalid add 0)
        unsigned vm[kQ / 2];
#pragma unroll
        for (int h = 0; h < kQ / 2; h++)
            vm[h] = (((vmask >> (2 * h)) & 1) ? 0xFFFFu : 0u) |
                    (((vmask >> (2 * h + 1)) & 1) ? 0xFFFF0000u : 0u);
        auto qfield = [&](int p) { return ((vmask >> p) & 1) ? J.Q.qf[qbase + p] : -1; };
        // the distinct own fields of the block (up to kMaxDistinctQf are
        // reduced per warp at a flush; beyond that, per-query atomics)
        int nuq = 0;
        {
            unsigned todo = vmask;
            for (int round = 0; round <= kQ * 32; round++) {
                int cand = -1;
#pragma unroll
                for (int p = 0; p < kQ; p++)
                    if (cand < 0 && ((todo >> p) & 1)) cand = qfield(p);
                const unsigned any = __ballot_sync(0xffffffffu, cand >= 0);
                if (!any) break;
                const int pick = __shfl_sync(0xffffffffu, cand, __ffs(any) - 1);
                if (nuq < kMaxDistinctQf && lane == 0) ws->uq[nuq] = pick;
                nuq++;
#pragma unroll
                for (int p = 0; p < kQ; p++)
                    if (((todo >> p) & 1) && qfield(p) == pick) todo &= ~(1u << p);
            }
        }
        if (MODE == KD_MODE_MIXED) {
            const double hx = 0.5 * (bx[3] - bx[0]), hy = 0.5 * (bx[4] - bx[1]),
                         hz = 0.5 * (bx[5] - bx[2]);
            const double Rq = sqrt(hx * hx + hy * hy + hz * hz) * (1.0 + 1e-12);
            if (lane == 0) {
                // |t' - o| <= |c - o| + hT and |q' - o| <= Rq must stay
                // within kFp32Span (NaN box: never)
                const double lim = kFp32Span - J.hT - Rq;
                ws->cmax2 = lim > 0 ? lim * lim : -1.0;
            }
            for (int k = lane; k < ne; k += 32) {
                if (isfinite(R[k])) {
                    const double inv4e = 0.25 / band_halfwidth(R[k], Rq, J.hT);
                    ws->nsl[k] = (float)(-inv4e);
                    ws->Aw[k] = (float)(0.5 + R[k] * inv4e);
                } else {
                    ws->nsl[k] = 0.0f;
                    ws->Aw[k] = 0.0f;
                }
            }
        }
        for (int e = 0; e <= ne; e++)
#pragma unroll
            for (int h = 0; h < kQ / 2; h++) P[(e * (kQ / 2) + h) * 32 + lane] = 0;
        __syncwarp();
        int cur_tf = -1;
        int since = 0;
        int tlo = ne, thi = -1;  // bins written since the last flush

        // flush key: tree field | 256 for the once-counted part of a symmetric job
        auto flush = [&](int key) {
            const int tf = key & 0xFF;
            unsigned long long *const Hd = (key >> 8) ? J.H2 : J.H;
            int qf[kQ];
#pragma unroll
            for (int p = 0; p < kQ; p++) qf[p] = qfield(p);
            const int ehi = min(thi, ne - 1);
            for (int e = tlo; e <= ehi; e++) {
                int v[kQ];
#pragma unroll
                for (int h = 0; h < kQ / 2; h++) {
                    const unsigned wv = P[(e * (kQ / 2) + h) * 32 + lane];
                    P[(e * (kQ / 2) + h) * 32 + lane] = 0;
                    v[2 * h] = (int)(wv & 0xFFFFu);
                    v[2 * h + 1] = (int)(wv >> 16);
                }
                if (nuq <= kMaxDistinctQf) {
                    for (int u = 0; u < nuq; u++) {
                        const int uf = ws->uq[u];
                        int sum = 0;
#pragma unroll
                        for (int p = 0; p < kQ; p++) sum += qf[p] == uf ? v[p] : 0;
                        for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
                        if (lane == 0 && sum)
                            atomicAdd(&Hd[((size_t)e * J.Fqe + uf) * J.Fte + tf],
                                      (unsigned long long)sum);
                    }
                } else {
#pragma unroll
                    for (int p = 0; p < kQ; p++)
                        if (((vmask >> p) & 1) && v[p])
                            atomicAdd(&Hd[((size_t)e * J.Fqe + qf[p]) * J.Fte + tf],
                                      (unsigned long long)v[p]);
                }
            }
            if (thi == ne) {
#pragma unroll
                for (int h = 0; h < kQ / 2; h++) P[(ne * (kQ / 2) + h) * 32 + lane] = 0;
            }
            tlo = ne;
            thi = -1;
        };

        // the next record's loads, held in registers while the current run
        // is counted
        uint4 nrec = make_uint4(0, 0, 0, 0);
        float4 npt[kRunPerLane];
#pragma unroll
        for (int h = 0; h < kRunPerLane; h++) npt[h] = make_float4(0, 0, 0, 0);
        double ncx = 0, ncy = 0, ncz = 0;
        auto issue = [&](int i) {
            nrec = A.rec[eoff + i];
            const int rl = nrec.z & 0xFF, K = nrec.z >> 24;
            if (K == 0) return;
            if (MODE == KD_MODE_MIXED) {
                const unsigned rs = nrec.x, leaf = nrec.y;
                ncx = J.leaf_c[3 * (size_t)leaf];
                ncy = J.leaf_c[3 * (size_t)leaf + 1];
                ncz = J.leaf_c[3 * (size_t)leaf + 2];
#pragma unroll
                for (int h = 0; h < kRunPerLane; h++)
                    if (lane + 32 * h < rl) npt[h] = J.t4[rs + lane + 32 * h];
            } else {
                const unsigned rs = nrec.x;
                if (lane < rl) {
                    ncx = J.tx[rs + lane];
                    ncy = J.ty[rs + lane];
                    ncz = J.tz[rs + lane];
                }
            }
        };

        // stage the prefetched run (mixed mode); returns whether its leaf
        // lies in FP32 range of the block centre
        auto stage_run = [&](int rl_) {
            const double ex = ncx - ox, ey = ncy - oy, ez = ncz - oz;
            const bool in_range = ex * ex + ey * ey + ez * ez < ws->cmax2;
            const float dx = (float)ex, dy = (float)ey, dz = (float)ez;
#pragma unroll
            for (int h = 0; h < kRunPerLane; h++) {
                const int j = lane + 32 * h;
                if (j < rl_) {
                    // t' = t_r + (c - o); -0.5 * (-2 t_r) is exact
                    const float lx = fmaf(-0.5f, npt[h].x, dx);
                    const float ly = fmaf(-0.5f, npt[h].y, dy);
                    const float lz = fmaf(-0.5f, npt[h].z, dz);
                    const float X = -2.0f * lx, Y = -2.0f * ly, Z = -2.0f * lz;
                    const float N = fmaf(lz, lz, fmaf(ly, ly, lx * lx));
                    ws->stage[2 * j] = make_float4(X, X, Y, Y);
                    ws->stage[2 * j + 1] = make_float4(Z, Z, N, N);
                }
            }
            return in_range;
        };

        if (ecnt > 0) issue(0);
        for (int i = 0; i < ecnt; i++) {
            const uint4 rec = nrec;
            const int rs = (int)rec.x, rl1 = rec.z & 0xFF, tf = (rec.z >> 8) & 0xFF;
            const int k0 = (rec.z >> 16) & 0xFF, K = rec.z >> 24;
            // commit the staged run
            bool fp32_range = false;
            if (K != 0) {
                if (MODE == KD_MODE_MIXED) {
                    fp32_range = stage_run(rl1);
                } else {
                    const int rl = rl1;
                    if (lane < rl) {
                        ws->stage64[lane] = ncx;
                        ws->stage64[KD_RUN_MAX + lane] = ncy;
                        ws->stage64[2 * KD_RUN_MAX + lane] = ncz;
                    }
                    for (int j = lane + 32; j < rl; j += 32) {
                        ws->stage64[j] = J.tx[rs + j];
                        ws->stage64[KD_RUN_MAX + j] = J.ty[rs + j];
                        ws->stage64[2 * KD_RUN_MAX + j] = J.tz[rs + j];
                    }
                }
            }
            __syncwarp();
            if (i + 1 < ecnt) issue(i + 1);
            const int rl = rl1;

            const int key = tf | (int)(rec.w << 8);
            if (key != cur_tf || since + rl > 0xFFFF) {
                if (cur_tf >= 0) flush(cur_tf);
                cur_tf = key;
                since = 0;
            }
            since += rl;
            tlo = min(tlo, k0);
            thi = max(thi, k0 + K);
            if (K == 0) {
#pragma unroll
                for (int h = 0; h < kQ / 2; h++)
                    P[(k0 * (kQ / 2) + h) * 32 + lane] += (((unsigned)rl | ((unsigned)rl << 16)) & vm[h]);
                __syncwarp();
                continue;
            }
            wtiles++;
            const bool fp32 = MODE == KD_MODE_MIXED && fp32_range && R[k0 + K - 1] < kFp32MaxR;
            // packed cumulative count of the previous edge, per query pair
            unsigned prev[kQ / 2];
#pragma unroll
            for (int h = 0; h < kQ / 2; h++) prev[h] = 0;
            const int pw = MODE == KD_MODE_MIXED && fp32 ? kPass32 : 4;
            for (int kb = 0; kb < K; kb += pw) {
                const int kn = min(pw, K - kb);
                unsigned pc[kQ / 2][4];
#pragma unroll
                for (int h = 0; h < kQ / 2; h++)
#pragma unroll
                    for (int k = 0; k < 4; k++) pc[h][k] = 0;
                unsigned redo = vmask;
                if (fp32) {
                    float a[kQ][kPass32], sl[kPass32];
#pragma unroll
                    for (int k = 0; k < kPass32; k++) {
                        sl[k] = k < kn ? ws->nsl[k0 + kb + k] : 0.0f;
                        const float Ak = k < kn ? ws->Aw[k0 + kb + k] : 0.0f;
#pragma unroll
                        for (int p = 0; p < kQ; p++) a[p][k] = fmaf(qn[p], sl[k], Ak);
                    }
                    unsigned band;
                    switch (kn) {
                    case 1: band = fp32_run<1>(ws->stage, rl, qx2, qy2, qz2, a, sl, pc); break;
                    case 2: band = fp32_run<2>(ws->stage, rl, qx2, qy2, qz2, a, sl, pc); break;
                    case 3: band = fp32_run<3>(ws->stage, rl, qx2, qy2, qz2, a, sl, pc); break;
                    default: band = fp32_run<4>(ws->stage, rl, qx2, qy2, qz2, a, sl, pc); break;
                    }
                    redo = band & vmask;
                    rechecked += (unsigned long long)__popc(redo) * rl;
                } else if (MODE == KD_MODE_FP64) {
                    double qxd[kQ], qyd[kQ], qzd[kQ];
#pragma unroll
                    for (int p = 0; p < kQ; p++) {
                        const bool v = (vmask >> p) & 1;
                        qxd[p] = v ? J.Q.x[qbase + p] : ox;
                        qyd[p] = v ? J.Q.y[qbase + p] : oy;
                        qzd[p] = v ? J.Q.z[qbase + p] : oz;
                    }
                    const double *s64 = ws->stage64;
                    int cnt[kQ][4];
                    switch (kn) {
                    case 1: fp64_run<1>(s64, s64 + KD_RUN_MAX, s64 + 2 * KD_RUN_MAX, rl, qxd, qyd, qzd, R + k0 + kb, cnt); break;
                    case 2: fp64_run<2>(s64, s64 + KD_RUN_MAX, s64 + 2 * KD_RUN_MAX, rl, qxd, qyd, qzd, R + k0 + kb, cnt); break;
                    case 3: fp64_run<3>(s64, s64 + KD_RUN_MAX, s64 + 2 * KD_RUN_MAX, rl, qxd, qyd, qzd, R + k0 + kb, cnt); break;
                    default: fp64_run<4>(s64, s64 + KD_RUN_MAX, s64 + 2 * KD_RUN_MAX, rl, qxd, qyd, qzd, R + k0 + kb, cnt); break;
                    }
#pragma unroll
                    for (int h = 0; h < kQ / 2; h++)
#pragma unroll
                        for (int k = 0; k < 4; k++)
                            pc[h][k] = (unsigned)cnt[2 * h][k] | ((unsigned)cnt[2 * h + 1][k] << 16);
                    redo = 0;
                }
                // exact FP64 recount of the queries FP32 could not decide: a
                // few of them (band pairs) by the whole warp, one after the
                // other; many (edges FP32 cannot represent) lane by lane
                const unsigned nre = __reduce_add_sync(0xffffffffu, (unsigned)__popc(redo));
                if (nre <= kCoopMax) {
                    for (unsigned it = 0; it < nre; it++) {
                        const unsigned has = __ballot_sync(0xffffffffu, redo != 0);
                        const int src = __ffs(has) - 1;
                        const int pq = __shfl_sync(0xffffffffu, __ffs(redo) - 1, src);
                        const int qi = qs + kQ * src + pq;
                        const unsigned pk =
                            exact_pass_warp(J.tx + rs, J.ty + rs, J.tz + rs, rl, J.Q.x[qi],
                                            J.Q.y[qi], J.Q.z[qi], R + k0 + kb, kn, lane);
                        if (lane == src) {
                            // replace query pq's half-word (selects, no indexing)
#pragma unroll
                            for (int h = 0; h < kQ / 2; h++) {
                                const bool lo = pq == 2 * h, hi = pq == 2 * h + 1;
#pragma unroll
                                for (int k = 0; k < 4; k++) {
                                    const unsigned v = (pk >> (8 * k)) & 0xFFu;
                                    pc[h][k] = lo ? ((pc[h][k] & 0xFFFF0000u) | v)
                                                  : hi ? ((pc[h][k] & 0xFFFFu) | (v << 16)) : pc[h][k];
                                }
                            }
                            redo &= ~(1u << pq);
                        }
                    }
                }
#pragma unroll
                for (int p = 0; p < kQ; p++)
                    if ((redo >> p) & 1) {
                        const unsigned pk =
                            exact_pass(J.tx + rs, J.ty + rs, J.tz + rs, rl, J.Q.x[qbase + p],
                                       J.Q.y[qbase + p], J.Q.z[qbase + p], R + k0 + kb, kn);
                        const int sh = 16 * (p & 1);
#pragma unroll
                        for (int k = 0; k < 4; k++)
                            pc[p >> 1][k] = (pc[p >> 1][k] & ~(0xFFFFu << sh)) |
                                            (((pk >> (8 * k)) & 0xFFu) << sh);
                    }
                // bin increments: packed cumulative counts minus the previous
                // edge's (no borrow between the halves: counts grow with k)
#pragma unroll
                for (int h = 0; h < kQ / 2; h++)
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        if (k < kn) {
                            P[((k0 + kb + k) * (kQ / 2) + h) * 32 + lane] += (pc[h][k] - prev[h]) & vm[h];
                            prev[h] = pc[h][k];
                        }
            }
            const unsigned rl2 = (unsigned)rl | ((unsigned)rl << 16);
#pragma unroll
            for (int h = 0; h < kQ / 2; h++)
                P[((k0 + K) * (kQ / 2) + h) * 32 + lane] += (rl2 - prev[h]) & vm[h];
            const unsigned long long tp = (unsigned long long)nvalid * rl;
            pairs += tp;
            kpairs += tp * K;
            if (K > 4) wide += tp;
            __syncwarp();
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
    const size_t ws = mode == KD_MODE_MIXED ? sizeof(WarpSmem<KD_MODE_MIXED>)
                                            : sizeof(WarpSmem<KD_MODE_FP64>);
    return sizeof(double) * KD_MAX_EDGES + ws * kTileWarpsPerCta +
           sizeof(unsigned) * (size_t)(ne + 1) * (kQ / 2) * 32 * kTileWarpsPerCta;
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

// the traversal and tile views of one (tree, query tree) job
static JobDesc job_desc(const kd_catalog *tc, const kd_catalog *qc, unsigned long long *H)
{
    JobDesc d;
    memset(&d, 0, sizeof d);
    d.T.box = tc->d_box;
    d.T.count = tc->d_ncount;
    d.T.tf = tc->d_ntf;
    d.T.leaf_run = tc->d_leaf_run;
    d.T.leaf_pos = tc->d_leaf_pos;
    d.T.run_start = tc->d_run_start;
    d.T.run_len = tc->d_run_len;
    d.T.run_tf = tc->d_run_tf;
    d.T.D = tc->depth;
    d.T.nleaves = tc->nleaves;
    d.Q.x = qc->d_x;
    d.Q.y = qc->d_y;
    d.Q.z = qc->d_z;
    d.Q.qf = qc->d_qf;
    d.Q.blk_start = qc->d_blk_start;
    d.Q.blk_len = qc->d_blk_len;
    d.Q.blk_qf = qc->d_blk_qf;
    d.Q.blk_box = qc->d_blk_box;
    d.tx = tc->d_x;
    d.ty = tc->d_y;
    d.tz = tc->d_z;
    d.t4 = (const float4 *)tc->d_t4;
    d.leaf_c = tc->d_leaf_c;
    d.hT = tc->leaf_hdiag * (1.0 + 1e-12);
    d.H = H;
    d.H2 = nullptr;
    d.Fqe = qc->max_qf + 1;
    d.Fte = tc->max_tf + 1;
    d.sym = 0;
    return d;
}

// An autocorrelation count (one catalog on both sides) whose points all keep
// their own field on the tree side can count each unordered pair once: the
// distance of (q, t) and of (t, q) is the same double (t - q and q - t differ
// only in sign, so every square, product and FMA is identical), and the pair's
// second orientation lands in the transposed field cell.
static bool symmetric_job(const kd_catalog *tc, const kd_catalog *qc)
{
    return tc == qc && !tc->fields_split && tc->max_qf == tc->max_tf;
}

static size_t hist_size(const kd_catalog *tc, const kd_catalog *qc, int ne)
{
    return (size_t)(ne + 1) * (size_t)(qc->max_qf + 1) * (size_t)(tc->max_tf + 1);
}

// Every job's query blocks (this shard's share of them) in one traversal and
// one persistent tile launch per record batch, over a shared work counter.
static void count_batch_impl(const kd_catalog *const *tcs, const kd_catalog *const *qcs,
                             int njobs, const double *h_rsq, int ne, int mode, int shard,
                             int nshards, long long *const *hists, kd_count_stats *stats)
{
    const int device = tcs[0]->device;
    for (int j = 0; j < njobs; j++)
        if (tcs[j]->device != device || qcs[j]->device != device)
            raise(KD_EINVAL, "the catalogs of a count are on different devices");
    check(cudaSetDevice(device), "cudaSetDevice");
    init_device();
    Stream st;
    cudaStream_t s = st.s;
    Pool pool(s);
    Events ev;
    int launches = 0, tile_launches = 0;

    // job table, histogram offsets, global block numbering
    std::vector<size_t> hoff(njobs + 1, 0);
    std::vector<int> hblk(njobs + 1, 0);
    std::vector<char> sym(njobs);
    for (int j = 0; j < njobs; j++) {
        sym[j] = symmetric_job(tcs[j], qcs[j]);
        // a symmetric job has its once-counted histogram H2 right after H
        hoff[j + 1] = hoff[j] + (sym[j] ? 2 : 1) * hist_size(tcs[j], qcs[j], ne);
        if ((long long)hblk[j] + qcs[j]->nblocks > INT_MAX) raise(KD_EINVAL, "too many query blocks in one count");
        hblk[j + 1] = hblk[j] + qcs[j]->nblocks;
    }
    const size_t hsz = hoff[njobs];
    unsigned long long *H = pool.alloc<unsigned long long>(hsz);
    std::vector<JobDesc> hj(njobs);
    for (int j = 0; j < njobs; j++) {
        hj[j] = job_desc(tcs[j], qcs[j], H + hoff[j]);
        if (sym[j]) {
            hj[j].sym = 1;
            hj[j].H2 = H + hoff[j] + hist_size(tcs[j], qcs[j], ne);
        }
    }
    JobDesc *jobs = pool.alloc<JobDesc>(njobs);
    int *jblk = pool.alloc<int>(njobs + 1);
    unsigned long long *dstats = pool.alloc<unsigned long long>(8);
    int *err = pool.alloc<int>(1);
    int *work = pool.alloc<int>(1);
    double *rsq = pool.alloc<double>(std::max(ne, 1));
    check(cudaEventRecord(ev.e[0], s), "event");
    check(cudaMemsetAsync(H, 0, sizeof(unsigned long long) * hsz, s), "memset");
    check(cudaMemsetAsync(dstats, 0, sizeof(unsigned long long) * 8, s), "memset");
    check(cudaMemsetAsync(err, 0, sizeof(int), s), "memset");
    check(cudaMemcpyAsync(rsq, h_rsq, sizeof(double) * ne, cudaMemcpyHostToDevice, s), "H2D");
    check(cudaMemcpyAsync(jobs, hj.data(), sizeof(JobDesc) * njobs, cudaMemcpyHostToDevice, s), "H2D");
    check(cudaMemcpyAsync(jblk, hblk.data(), sizeof(int) * (njobs + 1), cudaMemcpyHostToDevice, s),
          "H2D");

    // this shard's global blocks
    const int NB = hblk[njobs];
    // this shard's blocks: interleaved chunks of kShardChunk global blocks
    // (chunk c belongs to shard c mod nshards), so that every shard gets an
    // even mix of early and late blocks (a symmetric job's block only counts
    // tree points after its own, so early blocks carry more work)
    std::vector<int> gl;
    if (nshards > 1)
        for (int c = shard * kShardChunk; c < NB; c += nshards * kShardChunk)
            for (int g = c; g < std::min(NB, c + kShardChunk); g++) gl.push_back(g);
    const int G0 = 0;
    const int G1 = nshards > 1 ? (int)gl.size() : NB;
    const int nb = G1 - G0;
    int *gmap = nullptr;
    if (nshards > 1 && nb > 0) {
        gmap = pool.alloc<int>(nb);
        check(cudaMemcpyAsync(gmap, gl.data(), sizeof(int) * (size_t)nb, cudaMemcpyHostToDevice, s),
              "H2D");
    }
    int *cnt = pool.alloc<int>(std::max(nb, 1));
    TravOut to;
    memset(&to, 0, sizeof to);
    to.gmap = gmap;
    to.count = cnt;
    to.accepted = dstats + 2;
    to.err = err;
    if (nb > 0) {
        k_traverse<false><<<blocks_for(nb, kTravWarps), 32 * kTravWarps, 0, s>>>(jobs, jblk, njobs,
                                                                                  rsq, ne, G0, G1, to);
        launches++;
    }
    KD_LAUNCH_CHECK("k_traverse(count)");
    std::vector<int> hcnt(std::max(nb, 1));
    check(cudaMemcpyAsync(hcnt.data(), cnt, sizeof(int) * (size_t)nb, cudaMemcpyDeviceToHost, s),
          "D2H");
    int herr = 0;
    check(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    st.sync();
    if (herr) raise(herr, "node-pair traversal exceeded its stack");

    // batches of global blocks whose tile records fit the buffer: up to 2^30
    // records (16 GiB) or a quarter of the free memory, so that on a B200 a
    // full DD + DR + RR batch of 20M-point catalogs runs as one launch
    long long total = 0, maxblk = 0;
    for (int i = 0; i < nb; i++) {
        total += hcnt[i];
        maxblk = std::max<long long>(maxblk, hcnt[i]);
    }
    // free memory: the driver's, plus what the record pool and the default
    // pool hold cached (reusable without asking the driver)
    const cudaMemPool_t rpool = side_pool(kPoolRecords);
    size_t freeb = 0, totb = 0;
    cudaMemGetInfo(&freeb, &totb);
    freeb += pool_idle_bytes(rpool);
    {
        cudaMemPool_t dpool = nullptr;
        if (cudaDeviceGetDefaultMemPool(&dpool, device) == cudaSuccess && dpool != rpool)
            freeb += pool_idle_bytes(dpool);
        cudaGetLastError();
    }
    long long cap = std::max<long long>(
        1 << 20, std::min<long long>(1LL << 30, (long long)(freeb / 4 / sizeof(uint4))));
    // KD_TILE_RECORD_CAP (records, > 0) lowers the batch size: it exercises
    // the multi-batch path on small counts
    if (const char *env = getenv("KD_TILE_RECORD_CAP")) {
        const long long v = atoll(env);
        if (v > 0) cap = v;
    }
    // every batch holds at least one whole block: the buffer must take the
    // largest block's records (a failed allocation is reported, not overrun)
    cap = std::max(cap, maxblk);
    cap = std::min<long long>(cap, std::max<long long>(total, 1));
    uint4 *rec = pool.alloc_from<uint4>(rpool, cap);
    long long *off = pool.alloc<long long>(nb + 1);
    std::vector<long long> hoffs(nb + 1);

    const size_t smem = tile_smem(ne, mode);
    auto kern = mode == KD_MODE_MIXED ? k_tiles<KD_MODE_MIXED> : k_tiles<KD_MODE_FP64>;
    check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
          "smem attribute");
    int nsm = 148, occ = 1;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 32 * kTileWarpsPerCta, smem),
          "occupancy");
    occ = std::max(occ, 1);

    float ms_trav = 0, ms_tiles = 0;
    int b0 = 0;  // shard-relative
    while (b0 < nb) {
        long long acc = 0;
        int b1 = b0;
        hoffs[0] = 0;
        while (b1 < nb && (b1 == b0 || acc + hcnt[b1] <= cap)) {
            acc += hcnt[b1];
            b1++;
            hoffs[b1 - b0] = acc;
        }
        check(cudaMemcpyAsync(off, hoffs.data(), sizeof(long long) * (size_t)(b1 - b0 + 1),
                              cudaMemcpyHostToDevice, s), "H2D");
        TravOut tf = to;
        tf.count = nullptr;
        tf.off = off;
        tf.rec = rec;
        check(cudaEventRecord(ev.e[1], s), "event");
        k_traverse<true><<<blocks_for(b1 - b0, kTravWarps), 32 * kTravWarps, 0, s>>>(
            jobs, jblk, njobs, rsq, ne, G0 + b0, G0 + b1, tf);
        launches++;
        KD_LAUNCH_CHECK("k_traverse(fill)");
        check(cudaEventRecord(ev.e[2], s), "event");
        TileArgs ta;
        ta.jobs = jobs;
        ta.jblk = jblk;
        ta.njobs = njobs;
        ta.rsq = rsq;
        ta.ne = ne;
        ta.g0 = G0 + b0;
        ta.g1 = G0 + b1;
        ta.gmap = gmap;
        ta.off = off;
        ta.rec = rec;
        ta.work = work;
        ta.stats = dstats;
        check(cudaMemsetAsync(work, 0, sizeof(int), s), "memset");
        const int grid = (int)std::min<long long>(
            ((long long)(b1 - b0) + kTileWarpsPerCta - 1) / kTileWarpsPerCta, (long long)nsm * occ);
        kern<<<grid, 32 * kTileWarpsPerCta, smem, s>>>(ta);
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
    std::vector<unsigned long long> hh(std::max<size_t>(hsz, 1));
    unsigned long long hs[8];
    check(cudaMemcpyAsync(hh.data(), H, sizeof(unsigned long long) * hsz, cudaMemcpyDeviceToHost, s),
          "D2H");
    check(cudaMemcpyAsync(hs, dstats, sizeof hs, cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    st.sync();
    if (herr) raise(herr, "node-pair traversal exceeded its stack");
    for (int j = 0; j < njobs; j++) {
        const size_t n1 = hist_size(tcs[j], qcs[j], ne);
        const unsigned long long *h1 = hh.data() + hoff[j];
        for (size_t i = 0; i < n1; i++) hists[j][i] = (long long)h1[i];
        if (sym[j]) {  // both orientations of the once-counted pairs
            const unsigned long long *h2 = h1 + n1;
            const size_t F = (size_t)hj[j].Fqe;
            for (int e = 0; e <= ne; e++)
                for (size_t a = 0; a < F; a++)
                    for (size_t c = 0; c < F; c++)
                        hists[j][((size_t)e * F + a) * F + c] +=
                            (long long)(h2[((size_t)e * F + a) * F + c] +
                                        h2[((size_t)e * F + c) * F + a]);
        }
    }
    if (stats) {
        stats->pairs_tested = (long long)hs[0];
        stats->pairs_rechecked = (long long)hs[1];
        stats->pairs_accepted = (long long)hs[2];
        stats->pairs_one_bin_multifield = (long long)hs[6];
        stats->pairs_wide = (long long)hs[3];
        stats->edge_pairs = (long long)hs[4];
        stats->warp_tiles = (long long)hs[5];
        stats->entries = total;
        stats->ms_traverse = ms_trav;
        stats->ms_tiles = ms_tiles;
        stats->ms_total = elapsed(ev.e[0], ev.e[4]);
        stats->tile_launches = tile_launches;
        stats->launches = launches;
    }
}

// ------------------------------------------------------------------------
// Count without any allocation (kd_count_radii_static).
//
// For callers that cannot allocate device memory at count time: every
// per-call buffer of a count (bin histogram, tile records, block offsets,
// scan workspace, counters, the final per-radius matrices) is carved out of
// one file-scope device array.  Every GPU that loads the library holds this
// array until the process exits.  All calls on a device share it and it keeps
// the previous call's contents, so everything that must start at zero is
// cleared at the start of a call, and two calls that overlap on the same GPU
// race.  Jobs whose tile records do not fit are counted in as many batches as
// it takes.

constexpr size_t kStaticScratchBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
void *g_static_ptr[kMaxDevices];  // device address of g_static_scratch, per device
}  // namespace

// Device address of the scratch array on the current device.  Host code
// cannot use the symbol itself (on the host it names a host-side stand-in),
// so the address is looked up once per device with that device current and
// kept for the life of the process (a device reset through this library's
// runtime would invalidate it; the entry point's contract excludes that).
static unsigned char *static_scratch(int device)
{
    if (device < 0 || device >= kMaxDevices) raise(KD_ENODEV, "device index out of range");
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_ptr[device]) {
        void *ptr = nullptr;
        check(cudaGetSymbolAddress(&ptr, g_static_scratch), "cudaGetSymbolAddress(scratch)");
        g_static_ptr[device] = ptr;
    }
    return (unsigned char *)g_static_ptr[device];
}

// last block b1 > b0 such that blocks [b0, b1) have at most cap tile records
// (at least one block); records of block b0 alone above cap: b1 = -1
__global__ void k_static_batch(const long long *off, int nb, int b0, long long cap, int *b1_out,
                               long long *rel, int rel_cap)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        int lo = b0 + 1, hi = nb;
        if (off[b0 + 1] - off[b0] > cap) {
            *b1_out = -1;
            return;
        }
        while (lo < hi) {  // largest b1 in [b0+1, nb] with off[b1] - off[b0] <= cap
            const int mid = (lo + hi + 1) / 2;
            if (off[mid] - off[b0] <= cap) lo = mid;
            else hi = mid - 1;
        }
        *b1_out = min(lo, b0 + rel_cap - 1);
    }
    __syncthreads();
    const int b1 = *b1_out;
    for (int i = threadIdx.x; b1 > b0 && i <= b1 - b0; i += blockDim.x)
        rel[i] = off[b0 + i] - off[b0];
}

// hist[e][qf][tf] -> out[k][qf*Fq + tf]: the pairs with d2 < rsq of radius k
// (cumulative over sorted edges), in the reference's counter layout.  out is
// zeroed on the stream before the launch (several (qf, tf) can share a slot
// of that layout, so the slots are accumulated atomically): any grid works.
__global__ void k_static_out(const unsigned long long *H, int ne, int Fqe, int Fte,
                             const int *edge_of, int nradii, int Fq, int Ft, long long *out)
{
    const int nrow = Fq * Ft;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nradii * Fqe * Fte;
         i += gridDim.x * blockDim.x) {
        const int k = i / (Fqe * Fte), qf = (i / Fte) % Fqe, tf = i % Fte;
        const int e = edge_of[k];
        if (e < 0) continue;
        unsigned long long v = 0;
        for (int j = 0; j <= e; j++) v += H[((size_t)j * Fqe + qf) * Fte + tf];
        atomicAdd((unsigned long long *)&out[(size_t)k * nrow + qf * Fq + tf], v);
    }
}

// int tile counts per block (staged in the offsets' storage) widened to int64
__global__ void k_gather_widen(const int *in, int n, long long *out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = in[i];
}

static size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

static void count_static_impl(const kd_catalog *tc, int Ft, const kd_catalog *qc, int Fq,
                              const double *rsq_sorted, int ne, const int *edge_of, int nradii,
                              int mode, long long *h_out)
{
    if (tc->device != qc->device) raise(KD_EINVAL, "tree and query catalogs on different devices");
    check(cudaSetDevice(tc->device), "cudaSetDevice");
    unsigned char *base = static_scratch(tc->device);
    const cudaStream_t s = 0;  // legacy default stream: nothing is created

    const int nb = qc->nblocks;
    const int Fqe = qc->max_qf + 1, Fte = tc->max_tf + 1;
    const size_t hsz = (size_t)(ne + 1) * Fqe * Fte;

    // carve the scratch
    size_t at = 0;
    auto take = [&](size_t bytes) {
        unsigned char *p = base + at;
        at = align_up(at + bytes);
        return p;
    };
    auto *H = (unsigned long long *)take(sizeof(unsigned long long) * hsz);
    auto *job = (JobDesc *)take(sizeof(JobDesc));
    auto *jblk = (int *)take(sizeof(int) * 2);
    auto *misc = (unsigned long long *)take(sizeof(unsigned long long) * 8);  // stats
    auto *err = (int *)take(sizeof(int) * 4);  // err, work, b1
    auto *rsq = (double *)take(sizeof(double) * KD_MAX_EDGES);
    auto *eo = (int *)take(sizeof(int) * KD_MAX_EDGES);
    auto *out = (long long *)take(sizeof(long long) * (size_t)nradii * Fq * Ft);
    auto *cnt = (long long *)take(sizeof(long long) * ((size_t)nb + 1));
    auto *off = (long long *)take(sizeof(long long) * ((size_t)nb + 1));
    const size_t scan_bytes = sort::scan_temp_bytes<long long>(nb + 1);
    void *scan_tmp = take(scan_bytes);
    const int rel_cap = 4096;  // blocks per batch
    auto *rel = (long long *)take(sizeof(long long) * (rel_cap + 1));
    if (at + 16 * 64 > kStaticScratchBytes)
        raise(KD_EINVAL, "count too large for the static scratch (needs more than 32 MiB for "
                         "its histogram and block tables)");
    const long long cap = (long long)((kStaticScratchBytes - at) / sizeof(uint4));
    auto *rec = (uint4 *)(base + at);

    check(cudaMemsetAsync(H, 0, sizeof(unsigned long long) * hsz, s), "memset");
    check(cudaMemsetAsync(misc, 0, sizeof(unsigned long long) * 8, s), "memset");
    check(cudaMemsetAsync(err, 0, sizeof(int) * 4, s), "memset");
    check(cudaMemsetAsync(cnt, 0, sizeof(long long) * ((size_t)nb + 1), s), "memset");
    check(cudaMemcpyAsync(rsq, rsq_sorted, sizeof(double) * ne, cudaMemcpyHostToDevice, s), "H2D");
    check(cudaMemcpyAsync(eo, edge_of, sizeof(int) * nradii, cudaMemcpyHostToDevice, s), "H2D");
    const JobDesc hjob = job_desc(tc, qc, H);
    const int hjblk[2] = {0, nb};
    check(cudaMemcpyAsync(job, &hjob, sizeof hjob, cudaMemcpyHostToDevice, s), "H2D");
    check(cudaMemcpyAsync(jblk, hjblk, sizeof hjblk, cudaMemcpyHostToDevice, s), "H2D");

    // tile counts per block (the traversal writes int counts; widen in place)
    TravOut to;
    memset(&to, 0, sizeof to);
    to.count = (int *)off;  // int counts, staged in off's storage
    to.accepted = misc + 2;
    to.err = err;
    if (nb > 0)
        k_traverse<false><<<blocks_for(nb, kTravWarps), 32 * kTravWarps, 0, s>>>(job, jblk, 1, rsq,
                                                                                  ne, 0, nb, to);
    KD_LAUNCH_CHECK("k_traverse(count)");
    k_gather_widen<<<blocks_for(nb, 256), 256, 0, s>>>((const int *)off, nb, cnt);
    check(sort::scan<long long, sort::SumOp, false>(scan_tmp, cnt, off, nb + 1, sort::SumOp(), s),
          "scan");

    const size_t smem = tile_smem(ne, mode);
    auto kern = mode == KD_MODE_MIXED ? k_tiles<KD_MODE_MIXED> : k_tiles<KD_MODE_FP64>;
    check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
          "smem attribute");
    int nsm = 148, occ = 1;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, tc->device);
    check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 32 * kTileWarpsPerCta, smem),
          "occupancy");
    occ = std::max(occ, 1);
    int b0 = 0;
    while (b0 < nb) {
        k_static_batch<<<1, 256, 0, s>>>(off, nb, b0, cap, err + 2, rel, rel_cap);
        KD_LAUNCH_CHECK("k_static_batch");
        int b1 = 0;
        check(cudaMemcpyAsync(&b1, err + 2, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
        check(cudaStreamSynchronize(s), "sync");
        if (b1 < 0) raise(KD_EINVAL, "a query block has more tile records than the static scratch holds");
        TravOut tf = to;
        tf.count = nullptr;
        tf.off = rel;
        tf.rec = rec;
        k_traverse<true><<<blocks_for(b1 - b0, kTravWarps), 32 * kTravWarps, 0, s>>>(job, jblk, 1,
                                                                                      rsq, ne, b0, b1, tf);
        KD_LAUNCH_CHECK("k_traverse(fill)");
        TileArgs ta;
        ta.jobs = job;
        ta.jblk = jblk;
        ta.njobs = 1;
        ta.rsq = rsq;
        ta.ne = ne;
        ta.g0 = b0;
        ta.g1 = b1;
        ta.gmap = nullptr;
        ta.off = rel;
        ta.rec = rec;
        ta.work = err + 1;
        ta.stats = misc;
        check(cudaMemsetAsync(err + 1, 0, sizeof(int), s), "memset");
        const int grid = (int)std::min<long long>(
            ((long long)(b1 - b0) + kTileWarpsPerCta - 1) / kTileWarpsPerCta, (long long)nsm * occ);
        kern<<<grid, 32 * kTileWarpsPerCta, smem, s>>>(ta);
        KD_LAUNCH_CHECK("k_tiles");
        b0 = b1;
    }
    check(cudaMemsetAsync(out, 0, sizeof(long long) * (size_t)nradii * Fq * Ft, s), "memset");
    k_static_out<<<blocks_for((long long)nradii * Fqe * Fte, 256), 256, 0, s>>>(H, ne, Fqe, Fte, eo,
                                                                                 nradii, Fq, Ft, out);
    KD_LAUNCH_CHECK("k_static_out");
    int herr = 0;
    check(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(h_out, out, sizeof(long long) * (size_t)nradii * Fq * Ft,
                          cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaStreamSynchronize(s), "sync");
    if (herr) raise(herr, "node-pair traversal exceeded its stack");
}

}  // namespace kd

extern "C" int kdg_count_static(const kd_catalog *tree, int Ft, const kd_catalog *query, int Fq,
                                const double *rsq_sorted, int ne, const int *edge_of,
                                int nradii, int mode, long long *out)
{
    if (ne < 0 || ne > KD_MAX_EDGES || nradii < 0 || nradii > KD_MAX_EDGES) {
        kd_set_error(KD_EINVAL, "at most %d radii", KD_MAX_EDGES);
        return KD_EINVAL;
    }
    try {
        kd::count_static_impl(tree, Ft, query, Fq, rsq_sorted, ne, edge_of, nradii, mode, out);
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

extern "C" int kdg_set_device(int device)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        kd_set_error(KD_ENODEV, "no CUDA device %d (%d visible)", device, n);
        return KD_ENODEV;
    }
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        kd_set_error(KD_ECUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
        return KD_ECUDA;
    }
    return KD_OK;
}

extern "C" int kdg_count_batch(const kd_catalog *const *trees, const kd_catalog *const *queries,
                               int njobs, const double *rsq, int ne, int mode, int shard,
                               int nshards, long long *const *hists, kd_count_stats *stats)
{
    if (nshards < 1 || shard < 0 || shard >= nshards) {
        kd_set_error(KD_EINVAL, "shard %d of %d", shard, nshards);
        return KD_EINVAL;
    }
    if (ne < 1 || ne > KD_MAX_EDGES) {
        kd_set_error(KD_EINVAL, "between 1 and %d distinct radii per count", KD_MAX_EDGES);
        return KD_EINVAL;
    }
    if (njobs < 1) {
        kd_set_error(KD_EINVAL, "a batch needs at least one job");
        return KD_EINVAL;
    }
    try {
        kd::count_batch_impl(trees, queries, njobs, rsq, ne, mode, shard, nshards, hists, stats);
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

extern "C" int kdg_count(const kd_catalog *tree, const kd_catalog *query, const double *rsq,
                         int ne, int mode, int shard, int nshards, long long *hist,
                         kd_count_stats *stats)
{
    return kdg_count_batch(&tree, &query, 1, rsq, ne, mode, shard, nshards, &hist, stats);
}
