// Persistent Jacobi-preconditioned block CG on the reduced matrix S (FP64).
//
// Algorithm: core/solve.py:66-140 `_SolveMixin._pcg` and its CuPy twin
// core/gpu.py:199-253 `pcg`, step for step: one CG per column of B in
// lockstep, `zero` columns solved by X = 0, warm start X0, alpha = rz/pAp
// where active and pAp > 0, rel = ||R||/||B||, active = rel > tol, beta =
// rz_new/rz where active.  Where the reference makes one host round trip per
// iteration (gpu.py:242) and launches ~10 kernels, this is ONE cooperative
// launch: every CTA runs the whole iteration loop, grid-wide barriers
// separate the phases, and every CTA reduces the per-CTA partial sums in the
// same fixed order, so all of them take the same convergence decision.
//
// Phases per iteration (3 grid barriers):
//   A  AP = S P.  The nonzeros are split evenly over all warps of the grid
//      (chunk = ceil(nnz / warps)), so a row of 500k nonzeros (a year level)
//      and rows of 30 (firm levels) cost the same per nonzero.  A warp walks
//      the rows of its range 32 at a time: a row with at least kLong nonzeros
//      in the range takes the whole warp, shorter rows go four at a time to
//      8-lane subgroups; each lane accumulates in registers and the group
//      reduces once per row.  The vector is gathered as 16-byte pairs (P's
//      rows are padded to an even width).  Rows inside the range are written
//      to AP; a row cut by a range boundary leaves a partial sum in the
//      warp's two carry slots.  p'Ap accumulates per row (linear in the
//      partials, so cut rows need no fix-up for it).
//   B  alpha from the reduced p'Ap.  Per row: X += alpha P, R -= alpha AP and
//      the partial sums of R^2 and R^2 dinv.  A row cut across warps is
//      finished by the warp holding its last nonzero, which sums the carry
//      slots of the warps it spans in a fixed order.
//   C  rel, active and beta from the reduced sums; P = dinv R + beta P.
//
// Determinism: the grid size, the warp ranges and every reduction order are
// fixed for a given GPU and build, so repeated solves give identical bits.
#include <cstdio>
#include <type_traits>
#include <cuda_runtime.h>

#include "common.cuh"

namespace hdfe {
namespace pcg {

// One CTA per SM (fewer arrivals at each grid barrier).  Narrow blocks run
// 1024 threads (64 registers a thread: the most warps in flight); from
// HDFE_PCG_WIDE_K columns on, a thread's K-wide accumulators and gathered
// rows no longer fit in 64 registers, so those blocks run 512 threads with up
// to 128 registers each instead of spilling to local memory.
#ifndef HDFE_PCG_WIDE_K
#define HDFE_PCG_WIDE_K 3
#endif
__host__ __device__ constexpr int threads_for(int k) { return k >= HDFE_PCG_WIDE_K ? 512 : 1024; }
constexpr int kMaxWarps = 32;
constexpr unsigned kFull = 0xffffffffu;
#ifndef HDFE_PCG_LONG
#define HDFE_PCG_LONG 64
#endif
constexpr int kLong = HDFE_PCG_LONG;    // nonzeros in a warp's range that make a row "long"
// rows per thread per trip in the vector phases (their loads all issued
// before the updates), as many as fit the registers without spills
__host__ __device__ constexpr int row_batch(int k) { return k <= 3 ? 2 : 1; }

// P's row stride: even, so a row's pairs of values are 16-byte aligned
template <int K>
struct Stride {
    static constexpr int P = K == 1 ? 1 : ((K + 1) / 2) * 2;
};

// A dimension with few levels (years) meets almost every level of the others:
// its rows and columns of S are nearly dense.  When its levels are the last
// ns <= kSmall of S ("small levels" [Lb, L)), S's CSR holds only the block of
// the other ("big") levels, and the rest is dense: cross (Lb x kSmall,
// row-major, zero-padded) = S[r, Lb + j] and small (ns x ns) = S[Lb + i, Lb + j].
// A big row's product with the small levels is then its 128-byte row of
// cross, loaded beside the row's own indices and values in the SpMM's row
// walk (the same round trips), against ns values held in shared memory; the
// small rows' products are the columns of cross summed against P's big rows
// in the same walk, reduced with the p'Ap partials: no index round trips for
// the small levels, and cross is read once for both halves of the symmetric
// block.
constexpr int kSmall = HDFE_SMALL_MAX_LEVELS;

struct Params {
    const int64_t *indptr;
    const int32_t *indices;
    const double *data;
    int64_t L, nnz;
    int64_t Lb;                 // first small level (L when there is no dense block)
    int ns;                     // small levels, 0 .. kSmall
    const double *cross;        // (Lb, kSmall) S[r, Lb + j]
    const double *small;        // (ns, ns) S[Lb + i, Lb + j]
    const int64_t *wlo;     // (warps + 1) first nonzero of each warp's range
    int64_t nwarps;
    const double *dinv;
    const double *B;
    const uint8_t *zero;
    const double *X0;
    double tol;
    int64_t maxiter;
    double *X, *R, *P, *AP;
    double *carry;      // (total warps, 2, K)
    double *part;       // (quantities, gridDim.x)
    int64_t *wfirst;    // (total warps) row of each warp's first nonzero
    uint8_t *cut;       // (L) row spans two or more warps
    unsigned *bar;
    hdfe_pcg_info *info;
};

// Workspace layout in bytes: R (L*K), P (L*KP), AP (L*K), carry, part,
// wfirst, cut flags, then the barrier words.
struct Layout {
    int64_t r, p, ap, carry, part, wfirst, wlo, cut, bar, total;
};

inline Layout layout(int64_t L, int k, int64_t blocks)
{
    Layout o;
    const int kp = k == 1 ? 1 : ((k + 1) / 2) * 2;
    int64_t p = 0;
    auto take = [&](int64_t bytes) { int64_t at = p; p += (bytes + 255) / 256 * 256; return at; };
    o.r = take(L * k * 8);
    o.p = take(L * kp * 8);
    o.ap = take(L * k * 8);
    const int64_t warps = blocks * (threads_for(k) / 32);
    o.carry = take(warps * 2 * k * 8);
    // partials: p'Ap, ||R||^2, R'dinv R, ||B||^2 per column, then the dense
    // block's column sums (kSmall x k)
    o.part = take((4 + kSmall) * (int64_t)k * blocks * 8);
    o.wfirst = take(warps * 8);
    o.wlo = take((warps + 1) * 8);
    o.cut = take(L);
    o.bar = take(64);
    o.total = p;
    return o;
}

__device__ __forceinline__ int64_t upper_bound(const int64_t *a, int64_t n, int64_t x)
{   // first index i in [0, n) with a[i] > x (n if none)
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// The warp holding nonzero e: the last warp whose range starts at or before e.
__device__ __forceinline__ int64_t warp_of(const Params &a, int64_t e)
{
    return upper_bound(a.wlo, a.nwarps + 1, e) - 1;
}

// Warp ranges of S's nonzeros balanced by cost: a row costs its nonzeros plus
// kRowCost (the per-row work of a short row's setup and write-back), so warps
// of short rows take fewer nonzeros than warps inside long rows.
// The lane kernel's nonzeros are heavy (K-wide gathers), so its rows cost
// their nonzeros alone.
#ifndef HDFE_PCG_UNROLL
#define HDFE_PCG_UNROLL 6               // nonzeros per lane in flight (k = 3, 4)
#endif

#ifndef HDFE_PCG_ROW_COST
#define HDFE_PCG_ROW_COST 32
#endif
constexpr int64_t kRowCost = HDFE_PCG_ROW_COST;

__global__ void k_partition(const int64_t *indptr, int64_t L, int64_t nnz, int64_t nwarps,
                            int64_t row_cost, int64_t *wlo)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t > nwarps) return;
    const int64_t kRowCost = row_cost;
    const int64_t total = nnz + kRowCost * L;
    const int64_t T = t * total / nwarps;
    // the last row r with indptr[r] + kRowCost r <= T
    int64_t lo = 0, hi = L;
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (indptr[mid] + kRowCost * mid <= T) lo = mid; else hi = mid - 1;
    }
    const int64_t r = lo;
    int64_t at;
    if (r >= L) {
        at = nnz;
    } else {
        const int64_t first = indptr[r] + kRowCost * (r + 1);   // where the row's nonzeros start
        at = T < first ? indptr[r] : min(indptr[r] + (T - first), indptr[r + 1]);
    }
    wlo[t] = t == nwarps ? nnz : at;
}

// Sum of partial q over all CTAs, in fixed order; lane-parallel within one
// warp (lane j takes CTAs j, j+32, ...), then a fixed xor tree.
__device__ __forceinline__ double reduce_part(const double *part, int q)
{
    const int lane = threadIdx.x & 31;
    double s = 0.0;
    const double *p = part + (int64_t)q * gridDim.x;
    for (int b = lane; b < (int)gridDim.x; b += 32) s += __ldcg(p + b);
    return warp_sum(s);
}

constexpr int kRedLoads = 8;            // CTAs per lane in reduce_range: grids up to 256 CTAs

// s_red[q] = sum over CTAs of partial q, for q in [q0, q1): one warp per
// quantity, the same fixed order in every CTA
// LOADS partials a lane (grids up to 32 LOADS CTAs), QW quantities a warp at
// a time: LOADS x QW doubles in flight a lane
template <int LOADS = kRedLoads, int QW = 4>
__device__ __forceinline__ void reduce_range(const double *part, int q0, int q1, double *s_red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int nb = gridDim.x;
    for (int qb = q0 + warp; qb < q1; qb += QW * nw) {
        // QW quantities per warp at a time, every load issued before the sums
        double v[QW][LOADS];
#pragma unroll
        for (int i = 0; i < QW; i++) {
            const int q = qb + i * nw;
#pragma unroll
            for (int u = 0; u < LOADS; u++) {
                const int b = lane + 32 * u;
                v[i][u] = (q < q1 && b < nb) ? __ldcg(part + (int64_t)q * nb + b) : 0.0;
            }
        }
#pragma unroll
        for (int i = 0; i < QW; i++) {
            double t = 0.0;
#pragma unroll
            for (int u = 0; u < LOADS; u++) t += v[i][u];
            t = warp_sum(t);
            const int q = qb + i * nw;
            if (lane == 0 && q < q1) s_red[q] = t;
        }
    }
    __syncthreads();
}

// Row c of V (stride VS) into g[0..K), with vector loads of VW elements
// (4 doubles: one 32-byte load; 2 doubles; 2 or 4 floats: 8-, 16- or 32-byte
// aligned rows) or scalars.  A gather of a random row costs the L1 one
// wavefront per load instruction, so the widest load that holds the row wins.
// Plain loads: V may be written by this kernel between grid barriers.
template <int K, int VS, int VW, typename T>
__device__ __forceinline__ void gather(const T *V, int64_t c, T (&g)[K])
{
    const T *p = V + c * VS;
    if constexpr (VW == 4 && sizeof(T) == 8) {
        static_assert(VS % 4 == 0 && K <= 4, "32-byte rows");
        double t0, t1, t2, t3;
        asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];"
                     : "=d"(t0), "=d"(t1), "=d"(t2), "=d"(t3) : "l"(p));
        g[0] = t0;
        if constexpr (K > 1) g[1] = t1;
        if constexpr (K > 2) g[2] = t2;
        if constexpr (K > 3) g[3] = t3;
    } else if constexpr (VW == 4) {
#pragma unroll
        for (int k = 0; k < K; k += 4) {
            const float4 t = *reinterpret_cast<const float4 *>(p + k);
            g[k] = t.x;
            if (k + 1 < K) g[k + 1] = t.y;
            if (k + 2 < K) g[k + 2] = t.z;
            if (k + 3 < K) g[k + 3] = t.w;
        }
    } else if constexpr (VW == 2) {
        using T2 = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
#pragma unroll
        for (int k = 0; k < K; k += 2) {
            const T2 t = *reinterpret_cast<const T2 *>(p + k);
            g[k] = t.x;
            if (k + 1 < K) g[k + 1] = t.y;
        }
    } else {
#pragma unroll
        for (int k = 0; k < K; k++) g[k] = p[k];
    }
}

// acc += sum over e = e0, e0 + STEP, ... < re of vals[e] * V[indices[e]]:
// U nonzeros per lane per round, their index/value loads and then their
// gathers all issued before the multiply-adds, so U round trips overlap.
template <int K, int VS, int VW, int STEP, typename T>
__device__ __forceinline__ void row_products(const Params &a, const T *vals, const T *V,
                                             int64_t e0, int64_t re, T (&acc)[K])
{
    constexpr int U = K <= 2 ? 4 : (K <= 4 ? HDFE_PCG_UNROLL : 2);
    for (; e0 < re; e0 += STEP * U) {
        int64_t c[U];
        T d[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t e = e0 + STEP * u;
            c[u] = 0;
            d[u] = T(0);
            if (e < re) {
                // S streams through once per iteration: evict-first loads, so
                // that it does not push the vectors (P, X, R, AP) out of L2
                c[u] = __ldcs(a.indices + e);
                d[u] = __ldcs(vals + e);
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++)
            if (c[u] < 0 || c[u] >= a.L) { GridBarrier{a.bar}.fail(HDFE_ERR_BAD_CODE); c[u] = 0; }
        T g[U][K];
#pragma unroll
        for (int u = 0; u < U; u++) gather<K, VS, VW, T>(V, c[u], g[u]);
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
            for (int k = 0; k < K; k++) acc[k] += d[u] * g[u][k];
    }
}

// The small rows' products of one step of short rows (DENSE spmm_range):
// lane (subgroup, sl) holds cv[q] = cross[row, sl JPL + q] of its subgroup's
// row and that row's V; the K products per q are summed over the subgroups
// by a reduce-scatter (the two top subgroup bits halve the K <= 4 values
// between partner lanes, the rest of the subgroup bits sum the one value
// left), and one lane per (small level, column) adds the total to the warp's
// slot: 2 + 1 + (log2(32 / LPR) - 2) shuffles per q instead of K
// log2(32 / LPR).  A fixed tree, so the sums are deterministic.
template <int K, int LPR, int JPL>
__device__ __forceinline__ void col_step(const double (&cv)[JPL], const double (&vrow)[K],
                                         double *s_colw, int lane, int sl)
{
    static_assert(K <= 4 && LPR <= 8, "four columns, at least four subgroups");
    const bool h = (lane >> 4) & 1, g = (lane >> 3) & 1;
    constexpr int kLowMask = 7 & ~(LPR - 1);       // subgroup bits below bit 3
    const int vi = 2 * (int)h + (int)g;             // the value this lane ends with
#pragma unroll
    for (int q = 0; q < JPL; q++) {
        const double v0 = cv[q] * vrow[0];
        const double v1 = K > 1 ? cv[q] * vrow[K > 1 ? 1 : 0] : 0.0;
        const double v2 = K > 2 ? cv[q] * vrow[K > 2 ? 2 : 0] : 0.0;
        const double v3 = K > 3 ? cv[q] * vrow[K > 3 ? 3 : 0] : 0.0;
        // lanes with bit 4 set keep values 2, 3; the others 0, 1
        double k0 = h ? v2 : v0, k1 = h ? v3 : v1;
        k0 += __shfl_xor_sync(kFull, h ? v0 : v2, 16);
        k1 += __shfl_xor_sync(kFull, h ? v1 : v3, 16);
        // then bit 3 picks one of the two
        double b = (g ? k1 : k0) + __shfl_xor_sync(kFull, g ? k0 : k1, 8);
#pragma unroll
        for (int o = 4; o >= LPR; o >>= 1) b += __shfl_xor_sync(kFull, b, o);
        if (vi < K && (lane & kLowMask) == 0) s_colw[(sl * JPL + q) * K + vi] += b;
    }
}

// vrow: V[row, 0..K), loaded before the row's products (for p'Ap)
template <int K, typename T>
__device__ __forceinline__ void finish_row(int64_t row, const T (&acc)[K], int64_t row_st,
                                           int64_t row_en, int64_t lo, int64_t hi, int64_t gw,
                                           const T (&vrow)[K], T *out, T *carry,
                                           double (&dot)[K], bool want_dot)
{
    if (want_dot) {
#pragma unroll
        for (int k = 0; k < K; k++) dot[k] += (double)vrow[k] * (double)acc[k];
    }
    if (row_st >= lo && row_en <= hi) {
#pragma unroll
        for (int k = 0; k < K; k++) out[row * K + k] = acc[k];
    } else {
        // cut row: slot 1 in the warp where it starts, 0 elsewhere
        T *cs = carry + (gw * 2 + (row_st >= lo ? 1 : 0)) * K;
#pragma unroll
        for (int k = 0; k < K; k++) cs[k] = acc[k];
    }
}

// out = S V over this warp's range of nonzeros (rows inside the range),
// partial sums of cut rows to the carry slots, dot[k] += V[r] . (S V)[r]
// (in FP64 whatever T is).  vals are S's values in T.  Short rows go LPR
// lanes each, 32 / LPR rows side by side: a short row costs two dependent
// round trips (its indices and values, then its gathers) whatever its length
// up to LPR x the unroll, so matrices of short rows (S's big block once the
// years are split off: ~16 nonzeros a row) run with 4 lanes a row and twice
// the rows in flight.
//   DENSE (S in the split form, see kSmall): a big row's products with the
// small levels ride the same round trips -- the row's 16 values of `cross`
// (JPL a lane: one vector load) are loaded beside its indices and values,
// multiplied by the small levels' entries of V (s_ps, shared memory) into
// the row's sum, and multiplied by the row's own V into the small rows'
// products, which are summed over the subgroups of each step and added, in
// step order, to this warp's slots s_colw (kSmall x K, zeroed here).  Only
// the warp holding a row's first nonzero does this for the row.
template <int K, int VS, int VW, typename T, int LPR = 8, bool DENSE = false>
__device__ void spmm_range(const Params &a, const T *__restrict__ vals, const T *__restrict__ V,
                           T *__restrict__ out, T *carry, double (&dot)[K], bool want_dot,
                           const double *s_ps = nullptr, double *s_colw = nullptr)
{
    static_assert(LPR == 2 || LPR == 4 || LPR == 8, "short rows take 2, 4 or 8 lanes");
    static_assert(!DENSE || sizeof(T) == 8, "the dense block is FP64");
    constexpr int RPS = 32 / LPR;       // short rows per step
    constexpr int JPL = kSmall / LPR;   // a short row's small levels a lane
    const int lane = threadIdx.x & 31, sub = lane / LPR, sl = lane % LPR;
    const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int64_t lo = a.wlo[gw];
    const int64_t hi = a.wlo[gw + 1];
    if constexpr (DENSE) {
        for (int t = lane; t < kSmall * K; t += 32) s_colw[t] = 0.0;
        __syncwarp();
    }
    if (lo >= hi) return;
    int64_t r0 = a.wfirst[gw];
    for (;;) {
        // bounds of rows r0 .. r0+31 (lane j: row r0+j)
        const int64_t q = r0 + lane;
        const int64_t st = q < a.L ? __ldg(a.indptr + q) : INT64_MAX;
        const int64_t en = q < a.L ? __ldg(a.indptr + q + 1) : INT64_MAX;
        const bool inr = st < hi;
        const unsigned inmask = __ballot_sync(kFull, inr);
        const int nrows = __popc(inmask);           // a prefix of the lanes: starts increase
        if (nrows == 0) break;
        const int64_t cs = max(st, lo), ce = min(en, hi);
        const int len = inr ? (int)(ce - cs) : 0;
        const unsigned longmask = __ballot_sync(kFull, inr && len >= kLong);
        int j = 0;
        while (j < nrows) {
            if ((longmask >> j) & 1u) {
                // one long row, the whole warp
                const int64_t rs = __shfl_sync(kFull, cs, j), re = __shfl_sync(kFull, ce, j);
                const int64_t row_st = __shfl_sync(kFull, st, j), row_en = __shfl_sync(kFull, en, j);
                // DENSE: lanes 0..15 take one small level each
                const bool dense = DENSE && r0 + j < a.Lb && row_st >= lo && lane < kSmall;
                T vrow[K];
#pragma unroll
                for (int k = 0; k < K; k++)
                    vrow[k] = ((want_dot && lane == 0) || dense) ? V[(r0 + j) * VS + k] : T(0);
                const double cv1 = dense ? __ldcs(a.cross + (r0 + j) * kSmall + lane) : 0.0;
                T acc[K];
#pragma unroll
                for (int k = 0; k < K; k++) acc[k] = T(0);
                row_products<K, VS, VW, 32, T>(a, vals, V, rs + lane, re, acc);
                if constexpr (DENSE) {
                    if (dense) {
#pragma unroll
                        for (int k = 0; k < K; k++) {
                            acc[k] += cv1 * s_ps[lane * K + k];
                            s_colw[lane * K + k] += cv1 * vrow[k];
                        }
                    }
                    __syncwarp();
                }
#pragma unroll
                for (int k = 0; k < K; k++) acc[k] = warp_sum(acc[k]);
                if (lane == 0)
                    finish_row<K, T>(r0 + j, acc, row_st, row_en, lo, hi, gw, vrow, out, carry,
                                     dot, want_dot);
                j++;
            } else {
                // up to RPS short rows, one per LPR-lane subgroup, up to the next long row
                const unsigned ahead = longmask & (0xffffffffu << j);
                int batch = ahead ? (__ffs(ahead) - 1 - j) : RPS;
                batch = min(min(batch, RPS), nrows - j);
                const int src = min(j + sub, 31);
                const bool mine = sub < batch;
                const int64_t rs = __shfl_sync(kFull, cs, src), re = __shfl_sync(kFull, ce, src);
                const int64_t row_st = __shfl_sync(kFull, st, src);
                const int64_t row_en = __shfl_sync(kFull, en, src);
                const int64_t row = r0 + j + sub;
                // DENSE: this lane's JPL small levels of the row, loaded with
                // its indices and values
                const bool dense = DENSE && mine && row < a.Lb && row_st >= lo;
                T vrow[K];
#pragma unroll
                for (int k = 0; k < K; k++)
                    vrow[k] = ((want_dot && mine && sl == 0) || dense) ? V[row * VS + k] : T(0);
                double cv[DENSE ? JPL : 1];
                if constexpr (DENSE) {
                    const double2 *cp =
                        reinterpret_cast<const double2 *>(a.cross + row * kSmall + sl * JPL);
#pragma unroll
                    for (int q = 0; q < JPL / 2; q++) {
                        const double2 t2 = dense ? __ldcs(cp + q) : make_double2(0.0, 0.0);
                        cv[2 * q] = t2.x;
                        cv[2 * q + 1] = t2.y;
                    }
                }
                T acc[K];
#pragma unroll
                for (int k = 0; k < K; k++) acc[k] = T(0);
                if (mine) row_products<K, VS, VW, LPR, T>(a, vals, V, rs + sl, re, acc);
                if constexpr (DENSE) {
#pragma unroll
                    for (int q = 0; q < JPL; q++)
#pragma unroll
                        for (int k = 0; k < K; k++) acc[k] += cv[q] * s_ps[(sl * JPL + q) * K + k];
                    // the small rows' products: this step's rows summed over the
                    // subgroups and added to the warp's slots
                    if constexpr (K <= 4) col_step<K, LPR, JPL>(cv, vrow, s_colw, lane, sl);
                    __syncwarp();
                }
#pragma unroll
                for (int k = 0; k < K; k++)
#pragma unroll
                    for (int o = LPR / 2; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(kFull, acc[k], o);
                if (mine && sl == 0 && re > rs)
                    finish_row<K, T>(r0 + j + sub, acc, row_st, row_en, lo, hi, gw, vrow, out,
                                     carry, dot, want_dot);
                j += batch;
            }
        }
        if (nrows < 32) break;
        r0 += 32;
    }
}

// AP[r] for a row whose nonzeros span several warps: summed from their carry
// slots in a fixed order by the warp holding the row's last nonzero.  Returns
// true (in all lanes) when this warp finishes such a row, with its AP in ap[].
template <int K, typename T>
__device__ bool finish_cut_row(const Params &a, const T *carry, int64_t &row, T (&ap)[K])
{
    const int lane = threadIdx.x & 31;
    const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int64_t lo = a.wlo[gw];
    const int64_t hi = a.wlo[gw + 1];
    if (lo >= hi) return false;
    const int64_t r = a.wfirst[gw];
    const int64_t rs = a.indptr[r], re = a.indptr[r + 1];
    if (!(rs < lo && re <= hi)) return false;
    const int64_t w0 = warp_of(a, rs);
    T s[K];
#pragma unroll
    for (int k = 0; k < K; k++) s[k] = T(0);
    for (int64_t w = w0 + lane; w <= gw; w += 32) {
        if (a.wlo[w] == a.wlo[w + 1]) continue;         // an empty range wrote no slots
        const T *cs = carry + (w * 2 + (w == w0 ? 1 : 0)) * K;
#pragma unroll
        for (int k = 0; k < K; k++) s[k] += __ldcg(cs + k);
    }
#pragma unroll
    for (int k = 0; k < K; k++) ap[k] = warp_sum(s[k]);
    row = r;
    return true;
}

// Per-CTA sums of N values per thread, written as partials q0 .. q0+N-1 of
// this CTA: warp trees, then one thread per value over the warps in order.
// One pair of __syncthreads for all N values.
template <int N>
__device__ __forceinline__ void block_partials(double (&v)[N], double *scratch, double *part,
                                               int q0, int nb)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < N; i++) v[i] = warp_sum(v[i]);
    if (lane == 0) {
#pragma unroll
        for (int i = 0; i < N; i++) scratch[warp * N + i] = v[i];
    }
    __syncthreads();
    if (threadIdx.x < N) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += scratch[w * N + threadIdx.x];
        part[(int64_t)(q0 + threadIdx.x) * nb + blockIdx.x] = t;
    }
    __syncthreads();
}

// ---- the dense small block (see kSmall)
//
// s_ps[j * K + k] = V[Lb + j, k]: the small levels' entries of the vector
// being multiplied, one copy per CTA.
template <int K, int VS>
__device__ __forceinline__ void load_small(const Params &a, const double *V, double *s_ps)
{
    if ((int)threadIdx.x < kSmall * K) {        // zeros past the small levels
        const int j = threadIdx.x / K, k = threadIdx.x % K;
        s_ps[threadIdx.x] = j < a.ns ? V[(a.Lb + j) * VS + k] : 0.0;
    }
    __syncthreads();
}

// This CTA's column sums (over its warps, in order) to partials qc .. qc +
// ns K - 1; with want_dot, thread k adds this CTA's share of the small rows'
// p'Ap, ps . (its column sums) (CTA 0: also ps . small ps), to dot[k].
template <int K>
__device__ __forceinline__ void dense_partials(const Params &a, const double *s_ps,
                                               double *s_col, double *s_cta, int qc, int nb,
                                               double (&dot)[K], bool want_dot)
{
    __syncthreads();
    const int t = threadIdx.x, nw = blockDim.x >> 5;
    if (t < a.ns * K) {
        double c = 0.0;
        for (int w = 0; w < nw; w++) c += s_col[w * kSmall * K + t];
        s_cta[t] = c;
        a.part[(int64_t)(qc + t) * nb + blockIdx.x] = c;
    }
    __syncthreads();
    if (want_dot && t < K) {
        double e = 0.0;
        for (int j = 0; j < a.ns; j++) e += s_ps[j * K + t] * s_cta[j * K + t];
        if (blockIdx.x == 0) {
            for (int j = 0; j < a.ns; j++) {
                double q = 0.0;
                for (int i = 0; i < a.ns; i++) q += a.small[j * a.ns + i] * s_ps[i * K + t];
                e += s_ps[j * K + t] * q;
            }
        }
#pragma unroll
        for (int k = 0; k < K; k++)
            if (t == k) dot[k] += e;
    }
}

// After the grid barrier: s_aps[j * K + k] = (S V)[Lb + j, k], the column
// sums over all CTAs (fixed order) plus small . ps, in every CTA.
template <int K>
__device__ __forceinline__ void dense_small_rows(const Params &a, const double *s_ps, int qc,
                                                 double *s_aps)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int t = warp; t < a.ns * K; t += nw) {
        const double v = reduce_part(a.part, qc + t);
        if (lane == 0) s_aps[t] = v;
    }
    __syncthreads();
    if ((int)threadIdx.x < a.ns * K) {
        const int j = threadIdx.x / K, k = threadIdx.x % K;
        double q = 0.0;
        for (int i = 0; i < a.ns; i++) q += a.small[j * a.ns + i] * s_ps[i * K + k];
        s_aps[threadIdx.x] += q;
    }
    __syncthreads();
}

// SPLIT: S in the split form (a.ns > 0); the kernels for the whole CSR carry
// none of its code (and none of its registers)
template <int K, int LPR = 8, bool SPLIT = false>
__global__ void __launch_bounds__(threads_for(K), 1) pcg_kernel(Params a)
{
    constexpr int KP = Stride<K>::P;
    __shared__ double s_red[4 * K];
    __shared__ double s_scratch[kMaxWarps * 3 * K];
    // the dense small block: its vector entries, this CTA's column sums, the
    // small rows' products, and the warps' column sums
    __shared__ double s_ps[kSmall * K], s_cta[kSmall * K], s_aps[kSmall * K];
    __shared__ double s_col[kMaxWarps * kSmall * K];
    constexpr int kQc = 4 * K;          // first partial of the column sums
    GridBarrier gb{a.bar};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t gstride = (int64_t)gridDim.x * blockDim.x;
    const int64_t L = a.L;
    const int nb = gridDim.x;

    double bnorm[K], rz[K], rel[K];
    bool active[K], zero[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
        zero[k] = a.zero != nullptr && a.zero[k] != 0;
        active[k] = !zero[k];
        rel[k] = 0.0;
    }

    // ---- set-up: each warp's first row and the cut flags (used by the same
    // warps / threads later, so no barrier is needed for them)
    {
        const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
        const int64_t lo = a.wlo[gw];
        if (lane == 0 && lo < a.nnz) a.wfirst[gw] = upper_bound(a.indptr, L + 1, lo) - 1;
        __syncwarp();
        for (int64_t r = gtid; r < L; r += gstride) {
            const int64_t rs = a.indptr[r], re = a.indptr[r + 1];
            // bit 0: the row is cut across warps; bit 1: it has no nonzeros
            a.cut[r] = ((re > rs && warp_of(a, rs) != warp_of(a, re - 1)) ? 1 : 0) |
                       (re == rs ? 2 : 0);
        }
    }
    // ---- R = B - S X0 (or B), the zero columns, ||B||, rz
    double dot[K];
#pragma unroll
    for (int k = 0; k < K; k++) dot[k] = 0.0;
    if (a.X0 != nullptr) {
        if ((SPLIT && a.ns > 0)) {
            load_small<K, K>(a, a.X0, s_ps);
            spmm_range<K, K, 1, double, LPR, true>(a, a.data, a.X0, a.AP, a.carry, dot, false,
                                                   s_ps, s_col + warp * kSmall * K);
            dense_partials<K>(a, s_ps, s_col, s_cta, kQc, nb, dot, false);
        } else {
            spmm_range<K, K, 1, double, LPR>(a, a.data, a.X0, a.AP, a.carry, dot, false);
        }
        if (!gb.sync()) return;
        if ((SPLIT && a.ns > 0)) dense_small_rows<K>(a, s_ps, kQc, s_aps);
    }
    {
        double sb[K], sr[K], sz[K];
#pragma unroll
        for (int k = 0; k < K; k++) sb[k] = sr[k] = sz[k] = 0.0;
        auto setup_row = [&](int64_t r, const double (&ap)[K]) {
            const double di = a.dinv[r];
#pragma unroll
            for (int k = 0; k < K; k++) {
                const double b = a.B[r * K + k];
                double x = 0.0, res = b;
                if (a.X0 != nullptr) { x = a.X0[r * K + k]; res = b - ap[k]; }
                if (zero[k]) { x = 0.0; res = 0.0; }
                a.X[r * K + k] = x;
                a.R[r * K + k] = res;
                a.P[r * KP + k] = res * di;
                sb[k] += b * b;
                sr[k] += res * res;
                sz[k] += res * res * di;
            }
#pragma unroll
            for (int k = K; k < KP; k++) a.P[r * KP + k] = 0.0;
        };
        for (int64_t r = gtid; r < L; r += gstride) {
            double ap[K];
            if (a.X0 != nullptr && (a.cut[r] & 1)) continue;
            const bool empty = (a.cut[r] & 2) != 0;
#pragma unroll
            for (int k = 0; k < K; k++) {
                ap[k] = (a.X0 != nullptr && !empty) ? a.AP[r * K + k] : 0.0;
                if (a.X0 != nullptr && (SPLIT && a.ns > 0) && r >= a.Lb) ap[k] = s_aps[(r - a.Lb) * K + k];
            }
            setup_row(r, ap);
        }
        if (a.X0 != nullptr) {
            int64_t r;
            double ap[K];
            if (finish_cut_row<K, double>(a, a.carry, r, ap) && lane == 0) setup_row(r, ap);
        }
        {
            double v[3 * K];
#pragma unroll
            for (int k = 0; k < K; k++) { v[k] = sb[k]; v[K + k] = sr[k]; v[2 * K + k] = sz[k]; }
            block_partials<3 * K>(v, s_scratch, a.part, 0, nb);
        }
        if (!gb.sync()) return;
        if (warp < 3) {
            for (int k = 0; k < K; k++) {
                double t = reduce_part(a.part, warp * K + k);
                if (lane == 0) s_red[warp * K + k] = t;
            }
        }
        __syncthreads();
    }
    bool any_active = false, all_zero = true;
#pragma unroll
    for (int k = 0; k < K; k++) {
        double bn = sqrt(s_red[k]);
        bnorm[k] = bn == 0.0 ? 1.0 : bn;
        rz[k] = s_red[2 * K + k];
        all_zero &= zero[k];
        if (a.X0 != nullptr) {
            rel[k] = sqrt(s_red[K + k]) / bnorm[k];
            active[k] = active[k] && rel[k] > a.tol;
        }
        any_active |= active[k];
    }
    int64_t it = 0;
    bool done = all_zero || (a.X0 != nullptr && !any_active);
    __syncthreads();
    if (!done) {
        if (!gb.sync()) return;     // the set-up partials are read before phase A reuses them
        for (it = 1; it <= a.maxiter; it++) {
            // ---- A: AP = S P, p'Ap
#pragma unroll
            for (int k = 0; k < K; k++) dot[k] = 0.0;
            // P's rows are KP wide from a 256-byte aligned workspace: 32-byte
            // rows for k = 3, 4
            constexpr int VWP = (KP == 4) ? 4 : ((KP % 2 == 0) ? 2 : 1);
            if ((SPLIT && a.ns > 0)) {
                load_small<K, KP>(a, a.P, s_ps);
                spmm_range<K, KP, VWP, double, LPR, true>(a, a.data, a.P, a.AP, a.carry, dot,
                                                          true, s_ps, s_col + warp * kSmall * K);
                dense_partials<K>(a, s_ps, s_col, s_cta, kQc, nb, dot, true);
            } else {
                spmm_range<K, KP, VWP, double, LPR>(a, a.data, a.P, a.AP, a.carry, dot, true);
            }
            block_partials<K>(dot, s_scratch, a.part, 0, nb);
            if (!gb.sync()) return;
            if (warp == 0) {
                for (int k = 0; k < K; k++) {
                    double t = reduce_part(a.part, k);
                    if (lane == 0) s_red[k] = t;
                }
            }
            __syncthreads();
            if ((SPLIT && a.ns > 0)) dense_small_rows<K>(a, s_ps, kQc, s_aps);
            double alpha[K];
#pragma unroll
            for (int k = 0; k < K; k++) {
                const double pap = s_red[k];
                alpha[k] = (active[k] && pap > 0.0) ? rz[k] / pap : 0.0;
            }
            __syncthreads();
            // ---- B: X += alpha P, R -= alpha AP, sums of R^2, R^2 dinv
            double sr[K], sz[K];
#pragma unroll
            for (int k = 0; k < K; k++) sr[k] = sz[k] = 0.0;
            auto step_row = [&](int64_t r, const double (&ap)[K]) {
                const double di = a.dinv[r];
#pragma unroll
                for (int k = 0; k < K; k++) {
                    const double p = a.P[r * KP + k];
                    a.X[r * K + k] += alpha[k] * p;
                    const double res = a.R[r * K + k] - alpha[k] * ap[k];
                    a.R[r * K + k] = res;
                    sr[k] += res * res;
                    sz[k] += res * res * di;
                }
            };
            // kRowBatch rows per thread per trip, every load issued before the
            // updates; the rows are summed in the same order as one at a time
            constexpr int kRowBatch = row_batch(K);
            for (int64_t r0 = gtid; r0 < L; r0 += kRowBatch * gstride) {
                uint8_t f[kRowBatch];
                double di[kRowBatch], p[kRowBatch][K], ap[kRowBatch][K], x[kRowBatch][K],
                    rr[kRowBatch][K];
#pragma unroll
                for (int u = 0; u < kRowBatch; u++) {
                    const int64_t r = r0 + u * gstride;
                    f[u] = r < L ? a.cut[r] : 1;
                    const bool use = (f[u] & 1) == 0;
                    const bool empty = (f[u] & 2) != 0;
                    di[u] = use ? a.dinv[r] : 0.0;
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        p[u][k] = use ? a.P[r * KP + k] : 0.0;
                        ap[u][k] = (use && !empty) ? a.AP[r * K + k] : 0.0;
                        if (use && (SPLIT && a.ns > 0) && r >= a.Lb) ap[u][k] = s_aps[(r - a.Lb) * K + k];
                        x[u][k] = use ? a.X[r * K + k] : 0.0;
                        rr[u][k] = use ? a.R[r * K + k] : 0.0;
                    }
                }
#pragma unroll
                for (int u = 0; u < kRowBatch; u++) {
                    if (f[u] & 1) continue;
                    const int64_t r = r0 + u * gstride;
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        a.X[r * K + k] = x[u][k] + alpha[k] * p[u][k];
                        const double res = rr[u][k] - alpha[k] * ap[u][k];
                        a.R[r * K + k] = res;
                        sr[k] += res * res;
                        sz[k] += res * res * di[u];
                    }
                }
            }
            {
                int64_t r;
                double ap[K];
                if (finish_cut_row<K, double>(a, a.carry, r, ap) && lane == 0) step_row(r, ap);
            }
            {
                double v[2 * K];
#pragma unroll
                for (int k = 0; k < K; k++) { v[k] = sr[k]; v[K + k] = sz[k]; }
                block_partials<2 * K>(v, s_scratch, a.part, K, nb);
            }
            if (!gb.sync()) return;
            if (warp < 2) {
                for (int k = 0; k < K; k++) {
                    double t = reduce_part(a.part, (warp + 1) * K + k);
                    if (lane == 0) s_red[(warp + 1) * K + k] = t;
                }
            }
            __syncthreads();
            // ---- C: convergence, beta, P = dinv R + beta P
            any_active = false;
            double beta[K];
#pragma unroll
            for (int k = 0; k < K; k++) {
                rel[k] = sqrt(s_red[K + k]) / bnorm[k];
                active[k] = rel[k] > a.tol;
                any_active |= active[k];
            }
            if (!any_active) break;
#pragma unroll
            for (int k = 0; k < K; k++) {
                const double rzn = s_red[2 * K + k];
                beta[k] = active[k] ? rzn / (rz[k] != 0.0 ? rz[k] : 1.0) : 0.0;
                rz[k] = rzn;
            }
            __syncthreads();
            for (int64_t r0 = gtid; r0 < L; r0 += row_batch(K) * gstride) {
                constexpr int kRowBatch = row_batch(K);
                double di[kRowBatch], rr[kRowBatch][K], p[kRowBatch][K];
#pragma unroll
                for (int u = 0; u < kRowBatch; u++) {
                    const int64_t r = r0 + u * gstride;
                    const bool in = r < L;
                    di[u] = in ? a.dinv[r] : 0.0;
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        rr[u][k] = in ? a.R[r * K + k] : 0.0;
                        p[u][k] = in ? a.P[r * KP + k] : 0.0;
                    }
                }
#pragma unroll
                for (int u = 0; u < kRowBatch; u++) {
                    const int64_t r = r0 + u * gstride;
                    if (r >= L) continue;
#pragma unroll
                    for (int k = 0; k < K; k++) a.P[r * KP + k] = rr[u][k] * di[u] + beta[k] * p[u][k];
                }
            }
            if (!gb.sync()) return;
        }
        if (it > a.maxiter) it = a.maxiter;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double mx = 0.0;
        bool conv = true;
#pragma unroll
        for (int k = 0; k < K; k++) {
            mx = fmax(mx, rel[k]);
            conv &= !active[k];
        }
        if (all_zero) { conv = true; mx = 0.0; }
        a.info->iterations = it;
        a.info->converged = conv ? 1 : 0;
        a.info->status = HDFE_OK;
        a.info->max_rel = mx;
    }
}

// Writes the barrier's error code (if any) into info after the persistent
// kernel, so a caller reading info sees a solve that stopped early.
__global__ void pcg_status_kernel(const unsigned *bar, hdfe_pcg_info *info)
{
    if (threadIdx.x == 0 && bar[2] != 0) {
        info->iterations = -1;
        info->converged = 0;
        info->status = (int32_t)bar[2];
        info->max_rel = __longlong_as_double(0x7ff8000000000000ll);
    }
}

template <int K>
int grid_blocks()
{
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel<K>, threads_for(K), 0) !=
        cudaSuccess)
        return -1;
    if (per_sm < 1) return -1;
    return sms * (per_sm < 1 ? per_sm : 1);
}

int grid_blocks_for_uncached(int k)
{
    switch (k) {
    case 1: return grid_blocks<1>();
    case 2: return grid_blocks<2>();
    case 3: return grid_blocks<3>();
    case 4: return grid_blocks<4>();
    case 5: return grid_blocks<5>();
    case 6: return grid_blocks<6>();
    case 7: return grid_blocks<7>();
    case 8: return grid_blocks<8>();
    }
    return -1;
}

// occupancy per (device, k), computed once
int grid_blocks_for(int k)
{
    static int cache[64][9] = {};
    int dev = 0;
    if (k < 1 || k > 8) return -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return grid_blocks_for_uncached(k);
    if (cache[dev][k] == 0) cache[dev][k] = grid_blocks_for_uncached(k);
    return cache[dev][k];
}

template <int K, int LPR = 8>
cudaError_t launch(Params p, int blocks, cudaStream_t s)
{
    void *args[] = {&p};
    const void *fn = (const void *)pcg_kernel<K, LPR, false>;
    if constexpr (K <= HDFE_PCG_SMALL_MAX_K) {
        if (p.ns > 0) fn = (const void *)pcg_kernel<K, LPR, true>;
    }
    return cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(threads_for(K)), args, 0, s);
}

// HDFE_PCG_SHORT_LPR lanes a short row when S's rows average at most this
// many nonzeros (8 otherwise)
#ifndef HDFE_PCG_SHORT_ROW_NNZ
#define HDFE_PCG_SHORT_ROW_NNZ 24
#endif
#ifndef HDFE_PCG_SHORT_LPR
#define HDFE_PCG_SHORT_LPR 4
#endif
constexpr int64_t kShortRowNnz = HDFE_PCG_SHORT_ROW_NNZ;
constexpr int kShortLpr = HDFE_PCG_SHORT_LPR;

// ------------------------------------------------ one column per lane
//
// Wide blocks (the JLA's blocks of probe vectors: up to 32 columns) run with
// one column per lane instead of K accumulators per thread.  The block is
// padded to K = 8, 16 or 32 columns (padding columns are zero columns); a
// row of a vector is then one coalesced load of 8K bytes, a thread holds one
// accumulator, and all columns share one pass over S's indices and values
// and one set of grid barriers per iteration.
//   SpMM: a warp streams its range of nonzeros 32 at a time, H = 32 / K
//   nonzeros side by side (one per group of K lanes), the rows of V it needs
//   staged in shared memory by asynchronous copies, several windows ahead.  Row
//   boundaries are the same in every lane, so the row walk is warp-uniform;
//   the row ends come 32 at a time from one coalesced load.  A row finishing
//   inside the range is summed over the H groups and written; a row cut by the
//   range boundary goes to the warp's carry slots as in pcg_kernel.
//   Vector phases: one thread per (row, column) element; a thread's column is
//   fixed (the grid stride is a multiple of 32), so each thread keeps its
//   column's alpha, beta and partial sums in registers, and the per-column
//   sums reduce over the lanes of that column, then over warps and CTAs in a
//   fixed order.
#ifndef HDFE_PCG_LANE_FROM
#define HDFE_PCG_LANE_FROM 5            // blocks of at least this many columns
#endif
// CTA size per block width: the K = 32 kernel stages 24 KB of gathers per
// warp, so it runs 8 warps per CTA; narrower ones run 16.
__host__ __device__ constexpr int lane_threads(int K) { return K >= 32 ? 256 : 512; }
__host__ __device__ constexpr int lane_ru(int K) { return K >= 32 ? 4 : 2; }  // vector elements per trip
constexpr int kLaneStages = 3;          // windows of 32 nonzeros in flight per warp
// The FP64 block of 32 columns keeps one window in flight: its CTAs (8 warps,
// at most 128 registers a thread) then fit two to an SM, which hides more of
// the gathers' latency than two more windows do (the 32-probe block solve of
// the KSS call: 103 -> 92 ms on the 1M-worker panel).
__host__ __device__ constexpr int lane_stages(int K) { return K >= 32 ? 1 : kLaneStages; }
__host__ __device__ constexpr int lane_ctas(int K) { return K >= 32 ? 2 : 1; }
// its reduce_range: partials a lane (grids up to 32 x this CTAs), quantities
// a warp at a time
__host__ __device__ constexpr int lane_red_loads(int K) { return K >= 32 ? 16 : kRedLoads; }
__host__ __device__ constexpr int lane_red_qw(int K) { return K >= 32 ? 2 : 4; }
constexpr uint8_t kRowCut = 1, kRowEmpty = 2;   // per-row flags
// dynamic shared memory: per warp, kLaneStages x 32 gathered rows of K values
// and their 32 matrix values
inline int lane_smem_bytes(int K, int ns = kLaneStages)
{
    return (lane_threads(K) / 32) * ns * 32 * (K + 1) * 8;
}

inline bool use_lanes(int k) { return k >= HDFE_PCG_LANE_FROM || k > 8; }
inline int lane_width(int k) { return k <= 8 ? 8 : (k <= 16 ? 16 : 32); }

struct LaneLayout {
    int64_t r, p, ap, x, carry, part, wfirst, wlo, cut, bar, total;
};

// R, P, AP (L, K); X (L, K) unless the caller's X has K columns already
inline LaneLayout lane_layout(int64_t L, int k, int64_t blocks)
{
    LaneLayout o;
    const int kw = lane_width(k);
    const int64_t warps = blocks * (lane_threads(kw) / 32);
    int64_t p = 0;
    auto take = [&](int64_t bytes) { int64_t at = p; p += (bytes + 255) / 256 * 256; return at; };
    o.r = take(L * kw * 8);
    o.p = take(L * kw * 8);
    o.ap = take(L * kw * 8);
    o.x = k == kw ? -1 : take(L * kw * 8);
    o.carry = take(warps * 2 * kw * 8);
    o.part = take(3 * (int64_t)kw * blocks * 8);
    o.wfirst = take(warps * 8);
    o.wlo = take((warps + 1) * 8);
    o.cut = take(L);
    o.bar = take(64);
    o.total = p;
    return o;
}

struct LaneArgs {
    double *Xw;     // (L, K): the iterate (the caller's X when k == K)
    int32_t k;      // the caller's columns (B, X0, X have stride k)
};

// vr = V[r, lane] (lanes < K), loaded when row r began; p'Ap in FP64
template <int K, typename T>
__device__ __forceinline__ void lane_flush(int64_t r, int64_t st, int64_t en, int64_t lo,
                                           int64_t hi, int64_t gw, T acc, T vr, T *out, T *carry,
                                           double &dot, bool want_dot)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = K; o < 32; o <<= 1) acc += __shfl_xor_sync(kFull, acc, o);
    if (lane < K) {
        if (want_dot) dot += (double)vr * (double)acc;
        if (st >= lo && en <= hi)
            out[r * K + lane] = acc;
        else    // cut row: slot 1 in the warp where it starts, 0 elsewhere
            carry[(gw * 2 + (st >= lo ? 1 : 0)) * K + lane] = acc;
    }
}

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
// one element of T (8-byte double or 4-byte float) from global to shared memory
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *smem, const T *gmem)
{
    if constexpr (sizeof(T) == 8) cp_async8(smem, gmem);
    else cp_async4(smem, gmem);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// out = S V over this warp's range of nonzeros (rows inside the range); cut
// rows to the carry slots; dot += V[r, col] (S V)[r, col] in lanes < K.  T is
// the arithmetic of the product: FP64 (S's values `mvals`, V, out, carry and
// the accumulators in double) or FP32 (S's values as floats and FP32
// vectors, the accumulators in float); dot is FP64 either way.
// The gathers go through shared memory: for each window of 32 nonzeros the
// warp issues asynchronous copies (cp.async) of the 32 rows of V it needs,
// lane (sub, col) copying column col of the rows it will itself multiply,
// plus the window's matrix values, and keeps kLaneStages windows in flight,
// so the bytes in flight per SM do not depend on registers.  Row walk and
// flushes as described above; V[r] for p'Ap is loaded as row r begins.
template <int K, typename T, int NS = kLaneStages>
__device__ void lane_spmm(const Params &a, const T *__restrict__ mvals, const T *__restrict__ V,
                          T *__restrict__ out, T *carry, double &dot, bool want_dot, T *stage)
{
    constexpr int H = 32 / K;
    const int lane = threadIdx.x & 31, col = lane % K, sub = lane / K;
    const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int64_t lo = a.wlo[gw];
    const int64_t hi = a.wlo[gw + 1];
    if (lo >= hi) return;
    T *vals = stage;                        // [NS][32][K]
    T *wts = stage + NS * 32 * K;           // [NS][32]
    const int64_t nwin = (hi - lo + 31) / 32;
    auto load_idx = [&](int64_t w) -> int32_t {
        const int64_t e = lo + w * 32 + lane;
        int32_t c = 0;
        if (w < nwin && e < hi) {
            c = __ldg(a.indices + e);
            if (c < 0 || c >= a.L) { GridBarrier{a.bar}.fail(HDFE_ERR_BAD_CODE); c = 0; }
        }
        return c;
    };
    auto issue = [&](int64_t w, int32_t c) {    // window w's rows and values into its stage
        if (w < nwin) {
            const int sgi = (int)(w % NS);
            const int64_t base = lo + w * 32;
            const int n = (int)min((int64_t)32, hi - base);
            T *vs = vals + sgi * 32 * K;
#pragma unroll
            for (int u = 0; u < K; u++) {
                const int t = u * H + sub;
                const int cc = __shfl_sync(kFull, c, t);
                if (t < n) cp_async_elem<T>(vs + t * K + col, V + (int64_t)cc * K + col);
            }
            if (lane < n) cp_async_elem<T>(wts + sgi * 32 + lane, mvals + base + lane);
        }
        cp_async_commit();                      // one group per window, empty past the end
    };
    int32_t cnext = load_idx(0);
#pragma unroll
    for (int w = 0; w < NS - 1; w++) {
        const int32_t c = cnext;
        cnext = load_idx(w + 1);
        issue(w, c);
    }
    int64_t r = a.wfirst[gw];
    int64_t st = a.indptr[r];
    int64_t rw = r;     // row-end window: lane i holds indptr[rw + 1 + i]
    int64_t rend = rw + 1 + lane <= a.L ? a.indptr[rw + 1 + lane] : INT64_MAX;
    int64_t en = __shfl_sync(kFull, rend, 0);
    T vr = want_dot ? V[r * K + col] : T(0);
    T acc = T(0);
    for (int64_t w = 0; w < nwin; w++) {
        {
            const int32_t c = cnext;
            cnext = load_idx(w + NS);
            issue(w + NS - 1, c);
        }
        cp_async_wait<NS - 1>();        // window w has landed (this lane's copies) ...
        __syncwarp();                   // ... and every lane's (the values)
        const int sgi = (int)(w % NS);
        const int64_t base = lo + w * 32;
        const T *vs = vals + sgi * 32 * K;
        const T *ws = wts + sgi * 32;
#pragma unroll 8
        for (int u = 0; u < K; u++) {
            const int64_t sb = base + u * H;             // this step's first nonzero
            if (sb >= hi) break;
            const int t = u * H + sub;
            const bool valid = sb + sub < hi;
            const T g = valid ? vs[t * K + col] : T(0);
            const T wv = valid ? ws[t] : T(0);
            if (sb + H <= en) {                          // the whole step in row r
                acc += wv * g;
                continue;
            }
            for (int h = 0; h < H; h++) {
                const int64_t el = sb + h;
                if (el >= hi) break;
                while (el >= en) {                       // rows ending before el (empty ones too)
                    lane_flush<K, T>(r, st, en, lo, hi, gw, acc, vr, out, carry, dot, want_dot);
                    acc = T(0);
                    r++;
                    st = en;
                    if (want_dot) vr = V[r * K + col];
                    if (r - rw >= 32) {
                        rw = r;
                        rend = rw + 1 + lane <= a.L ? a.indptr[rw + 1 + lane] : INT64_MAX;
                    }
                    en = __shfl_sync(kFull, rend, (int)(r - rw));
                }
                if (sub == h) acc += wv * g;
            }
        }
        __syncwarp();                   // every lane is done with this stage before it is refilled
    }
    cp_async_wait<0>();
    lane_flush<K, T>(r, st, en, lo, hi, gw, acc, vr, out, carry, dot, want_dot);
}

// The cut row this warp finishes (its first row, when that row started in an
// earlier warp and ends in this one): the carry slots of the warps it spans
// summed in warp order, lane col holding column col.
template <int K, typename T = double>
__device__ bool lane_finish_cut(const Params &a, const T *carry, int64_t &row, T &ap)
{
    const int col = (threadIdx.x & 31) % K;
    const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int64_t lo = a.wlo[gw];
    const int64_t hi = a.wlo[gw + 1];
    if (lo >= hi) return false;
    const int64_t r = a.wfirst[gw];
    const int64_t rs = a.indptr[r], re = a.indptr[r + 1];
    if (!(rs < lo && re <= hi)) return false;
    const int64_t w0 = warp_of(a, rs);
    T s = T(0);
    for (int64_t w = w0; w <= gw; w++)
        if (a.wlo[w] != a.wlo[w + 1]) s += __ldcg(carry + (w * 2 + (w == w0 ? 1 : 0)) * K + col);
    ap = s;
    row = r;
    return true;
}

// Per-CTA sums of N quantities per column: v[i] is this thread's partial of
// quantity i for its column (lane % K); written as partials (q0 + i) * K + col.
template <int K, int N>
__device__ __forceinline__ void column_partials(double (&v)[N], double *scratch, double *part,
                                                int q0, int nb)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int o = K; o < 32; o <<= 1) v[i] += __shfl_xor_sync(kFull, v[i], o);
    if (lane < K) {
#pragma unroll
        for (int i = 0; i < N; i++) scratch[(i * nw + warp) * K + lane] = v[i];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < N * K; t += blockDim.x) {
        const int i = t / K, c = t % K;
        double s = 0.0;
        for (int w = 0; w < nw; w++) s += scratch[(i * nw + w) * K + c];
        part[(int64_t)(q0 * K + t) * nb + blockIdx.x] = s;
    }
    __syncthreads();
}

template <int K>
__global__ void __launch_bounds__(lane_threads(K), lane_ctas(K)) lane_kernel(Params a, LaneArgs x)
{
    constexpr int RU = lane_ru(K);
    extern __shared__ double s_stage[];
    __shared__ double s_red[3 * K];
    __shared__ double s_scratch[(lane_threads(K) / 32) * 3 * K];
    __shared__ double s_bnorm[K], s_rel[K];
    __shared__ int s_active[K];
    GridBarrier gb{a.bar};
    const int lane = threadIdx.x & 31, col = lane % K;
    const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t gstride = (int64_t)gridDim.x * blockDim.x;
    const int64_t L = a.L, LK = a.L * K;
    const int nb = gridDim.x;
    const int kc = x.k;
    double *Xw = x.Xw;
    const bool zero_c = col >= kc || (a.zero != nullptr && a.zero[col] != 0);
    double *stage = s_stage + (threadIdx.x >> 5) * lane_stages(K) * 32 * (K + 1);

    // ---- set-up: each warp's first row and the cut flags
    {
        const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
        const int64_t lo = a.wlo[gw];
        if (lane == 0 && lo < a.nnz) a.wfirst[gw] = upper_bound(a.indptr, L + 1, lo) - 1;
        __syncwarp();
        for (int64_t r = gtid; r < L; r += gstride) {
            const int64_t rs = a.indptr[r], re = a.indptr[r + 1];
            a.cut[r] = (re > rs && warp_of(a, rs) != warp_of(a, re - 1) ? kRowCut : 0) |
                       (re == rs ? kRowEmpty : 0);
        }
    }
    // ---- R = B - S X0 (or B), the zero and padding columns, ||B||, rz
    double dot = 0.0;
    if (a.X0 != nullptr) {
        for (int64_t t = gtid; t < LK; t += gstride)
            Xw[t] = zero_c ? 0.0 : a.X0[(t / K) * kc + col];
        if (!gb.sync()) return;
        lane_spmm<K, double, lane_stages(K)>(a, a.data, Xw, a.AP, a.carry, dot, false, stage);
        if (!gb.sync()) return;
    }
    double rel_c = 0.0, rz_c, bnorm_c;
    bool active_c = !zero_c;
    {
        double v[3] = {0.0, 0.0, 0.0};      // b^2, r^2, r^2 dinv
        auto setup_row = [&](int64_t r, double ap) {
            const double di = a.dinv[r];
            const double b = col < kc ? a.B[r * kc + col] : 0.0;
            double xv = 0.0, res = b;
            if (a.X0 != nullptr) { xv = Xw[r * K + col]; res = b - ap; }
            if (zero_c) { xv = 0.0; res = 0.0; }
            Xw[r * K + col] = xv;
            a.R[r * K + col] = res;
            a.P[r * K + col] = res * di;
            v[0] += b * b;
            v[1] += res * res;
            v[2] += res * res * di;
        };
        for (int64_t t = gtid; t < LK; t += gstride) {
            const int64_t r = t / K;
            const uint8_t f = a.cut[r];
            if (a.X0 != nullptr && (f & kRowCut)) continue;
            setup_row(r, (a.X0 != nullptr && !(f & kRowEmpty)) ? a.AP[t] : 0.0);
        }
        if (a.X0 != nullptr) {
            int64_t r;
            double ap;
            if (lane_finish_cut<K>(a, a.carry, r, ap) && lane < K) setup_row(r, ap);
        }
        column_partials<K, 3>(v, s_scratch, a.part, 0, nb);
        if (!gb.sync()) return;
        reduce_range<lane_red_loads(K), lane_red_qw(K)>(a.part, 0, 3 * K, s_red);
        const double bn = sqrt(s_red[col]);
        bnorm_c = bn == 0.0 ? 1.0 : bn;
        rz_c = s_red[2 * K + col];
        if (a.X0 != nullptr) {
            rel_c = sqrt(s_red[K + col]) / bnorm_c;
            active_c = active_c && rel_c > a.tol;
        }
        if (threadIdx.x < K) {
            s_bnorm[col] = bnorm_c;
            s_rel[col] = rel_c;
            s_active[col] = active_c ? 1 : 0;
        }
    }
    const bool all_zero = __syncthreads_and(zero_c) != 0;
    const bool any_active0 = __syncthreads_or(active_c) != 0;
    int64_t it = 0;
    const bool done = all_zero || (a.X0 != nullptr && !any_active0);
    if (!done) {
        if (!gb.sync()) return;     // the set-up partials are read before phase A reuses them
        for (it = 1; it <= a.maxiter; it++) {
            // ---- A: AP = S P, p'Ap
            dot = 0.0;
            lane_spmm<K, double, lane_stages(K)>(a, a.data, a.P, a.AP, a.carry, dot, true, stage);
            {
                double v[1] = {dot};
                column_partials<K, 1>(v, s_scratch, a.part, 0, nb);
            }
            if (!gb.sync()) return;
            reduce_range<lane_red_loads(K), lane_red_qw(K)>(a.part, 0, K, s_red);
            const double pap = s_red[col];
            const double alpha = (active_c && pap > 0.0) ? rz_c / pap : 0.0;
            // ---- B: X += alpha P, R -= alpha AP, sums of R^2, R^2 dinv
            double v[2] = {0.0, 0.0};
            auto step_row = [&](int64_t r, double ap) {
                const double di = a.dinv[r];
                const int64_t t = r * K + col;
                Xw[t] += alpha * a.P[t];
                const double res = a.R[t] - alpha * ap;
                a.R[t] = res;
                v[0] += res * res;
                v[1] += res * res * di;
            };
            // RU elements per thread per trip, all loads first
            for (int64_t t0 = gtid; t0 < LK; t0 += RU * gstride) {
                uint8_t f[RU];
                double ap[RU], pv[RU], xv[RU], rv[RU], di[RU];
#pragma unroll
                for (int u = 0; u < RU; u++) {
                    const int64_t t = t0 + u * gstride;
                    f[u] = kRowCut;
                    if (t < LK) {
                        const int64_t r = t / K;
                        f[u] = a.cut[r];
                        ap[u] = a.AP[t];
                        pv[u] = a.P[t];
                        xv[u] = Xw[t];
                        rv[u] = a.R[t];
                        di[u] = a.dinv[r];
                    }
                }
#pragma unroll
                for (int u = 0; u < RU; u++) {
                    if (f[u] & kRowCut) continue;       // also the slots past the end
                    const int64_t t = t0 + u * gstride;
                    Xw[t] = xv[u] + alpha * pv[u];
                    const double res = rv[u] - alpha * ((f[u] & kRowEmpty) ? 0.0 : ap[u]);
                    a.R[t] = res;
                    v[0] += res * res;
                    v[1] += res * res * di[u];
                }
            }
            {
                int64_t r;
                double ap;
                if (lane_finish_cut<K>(a, a.carry, r, ap) && lane < K) step_row(r, ap);
            }
            column_partials<K, 2>(v, s_scratch, a.part, 1, nb);
            if (!gb.sync()) return;
            reduce_range<lane_red_loads(K), lane_red_qw(K)>(a.part, K, 3 * K, s_red);
            // ---- C: convergence, beta, P = dinv R + beta P
            rel_c = sqrt(s_red[K + col]) / bnorm_c;
            active_c = rel_c > a.tol;
            if (threadIdx.x < K) {
                s_rel[col] = rel_c;
                s_active[col] = active_c ? 1 : 0;
            }
            if (!__syncthreads_or(active_c)) break;
            const double rzn = s_red[2 * K + col];
            const double beta = active_c ? rzn / (rz_c != 0.0 ? rz_c : 1.0) : 0.0;
            rz_c = rzn;
            for (int64_t t0 = gtid; t0 < LK; t0 += RU * gstride) {
                double rv[RU], pv[RU], di[RU];
#pragma unroll
                for (int u = 0; u < RU; u++) {
                    const int64_t t = t0 + u * gstride;
                    if (t < LK) {
                        rv[u] = a.R[t];
                        pv[u] = a.P[t];
                        di[u] = a.dinv[t / K];
                    }
                }
#pragma unroll
                for (int u = 0; u < RU; u++) {
                    const int64_t t = t0 + u * gstride;
                    if (t < LK) a.P[t] = rv[u] * di[u] + beta * pv[u];
                }
            }
            if (!gb.sync()) return;
        }
        if (it > a.maxiter) it = a.maxiter;
    }
    // ---- the iterate to the caller's X (stride k)
    if (Xw != a.X) {
        for (int64_t t = gtid; t < LK; t += gstride)
            if (col < kc) a.X[(t / K) * kc + col] = Xw[t];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double mx = 0.0;
        bool conv = true;
        for (int c = 0; c < kc; c++) {
            mx = fmax(mx, s_rel[c]);
            conv &= s_active[c] == 0;
        }
        if (all_zero) { conv = true; mx = 0.0; }
        a.info->iterations = it;
        a.info->converged = conv ? 1 : 0;
        a.info->status = HDFE_OK;
        a.info->max_rel = mx;
    }
}

template <int K>
int lane_grid()
{
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    if (cudaFuncSetAttribute(lane_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             lane_smem_bytes(K, lane_stages(K))) != cudaSuccess)
        return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lane_kernel<K>, lane_threads(K),
                                                      lane_smem_bytes(K, lane_stages(K))) !=
        cudaSuccess)
        return -1;
    // lane_ctas(K) CTAs per SM (fewer if they do not fit), at most as many as
    // reduce_range sums (32 lanes x lane_red_loads(K) partials each)
    const int want = sms * (per_sm < lane_ctas(K) ? per_sm : lane_ctas(K));
    const int most = 32 * lane_red_loads(K);
    return per_sm < 1 ? -1 : (want < most ? want : most);
}

int lane_grid_for(int kw)
{
    static int cache[64][3] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -1;
    const int i = kw == 8 ? 0 : (kw == 16 ? 1 : 2);
    if (cache[dev][i] == 0)
        cache[dev][i] = kw == 8 ? lane_grid<8>() : (kw == 16 ? lane_grid<16>() : lane_grid<32>());
    return cache[dev][i];
}

template <int K>
cudaError_t launch_lanes(Params p, LaneArgs x, int blocks, cudaStream_t s)
{
    void *args[] = {&p, &x};
    return cudaLaunchCooperativeKernel((const void *)lane_kernel<K>, dim3(blocks),
                                       dim3(lane_threads(K)), args,
                                       lane_smem_bytes(K, lane_stages(K)), s);
}

int solve_lanes(const int64_t *indptr, const int32_t *indices, const double *data, int64_t L,
                int64_t nnz, const double *dinv, const double *B, int32_t k, const uint8_t *zero,
                const double *X0, double tol, int64_t maxiter, double *X, void *workspace,
                int64_t workspace_bytes, hdfe_pcg_info *info, cudaStream_t s)
{
    const int kw = lane_width(k);
    const int blocks = lane_grid_for(kw);
    if (blocks < 1) return hdfe_set_cuda_error(cudaGetLastError());
    const LaneLayout lay = lane_layout(L, k, blocks);
    if (workspace_bytes < lay.total)
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_pcg_solve: workspace too small");
    char *ws = (char *)workspace;
    Params p{};
    p.indptr = indptr;
    p.indices = indices;
    p.data = data;
    p.L = L;
    p.nnz = nnz;
    const int64_t warps = (int64_t)blocks * (lane_threads(kw) / 32);
    p.nwarps = warps;
    p.dinv = dinv;
    p.B = B;
    p.zero = zero;
    p.X0 = X0;
    p.tol = tol;
    p.maxiter = maxiter;
    p.X = X;
    p.R = (double *)(ws + lay.r);
    p.P = (double *)(ws + lay.p);
    p.AP = (double *)(ws + lay.ap);
    p.carry = (double *)(ws + lay.carry);
    p.part = (double *)(ws + lay.part);
    p.wfirst = (int64_t *)(ws + lay.wfirst);
    p.wlo = (int64_t *)(ws + lay.wlo);
    p.cut = (uint8_t *)(ws + lay.cut);
    p.bar = (unsigned *)(ws + lay.bar);
    p.info = info;
    LaneArgs x;
    x.Xw = lay.x < 0 ? X : (double *)(ws + lay.x);
    x.k = k;
    HDFE_CUDA_TRY(cudaMemsetAsync(p.bar, 0, 16, s));
    pcg::k_partition<<<(unsigned)((p.nwarps + 256) / 256), 256, 0, s>>>(indptr, L, nnz, p.nwarps,
                                                                      0, (int64_t *)p.wlo);
    cudaError_t e = kw == 8 ? launch_lanes<8>(p, x, blocks, s)
                  : kw == 16 ? launch_lanes<16>(p, x, blocks, s)
                             : launch_lanes<32>(p, x, blocks, s);
    HDFE_CUDA_TRY(e);
    pcg_status_kernel<<<1, 32, 0, s>>>(p.bar, info);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(3);
    return HDFE_OK;
}

}  // namespace pcg
}  // namespace hdfe

using namespace hdfe;

extern "C" int64_t hdfe_pcg_workspace_bytes(int64_t L, int64_t nnz, int32_t k)
{
    (void)nnz;
    if (k < 1 || k > HDFE_PCG_MAX_K || L < 0) return -1;
    if (pcg::use_lanes(k)) {
        const int blocks = pcg::lane_grid_for(pcg::lane_width(k));
        return blocks < 1 ? -1 : pcg::lane_layout(L, k, blocks).total;
    }
    int blocks = pcg::grid_blocks_for(k);
    if (blocks < 1) return -1;
    return pcg::layout(L, k, blocks).total;
}

namespace {

int solve_registers(const int64_t *indptr, const int32_t *indices, const double *data, int64_t L,
                    int64_t nnz, int64_t small_first, int32_t small_count, const double *cross,
                    const double *small, const double *dinv, const double *B, int32_t k,
                    const uint8_t *zero, const double *X0, double tol, int64_t maxiter, double *X,
                    void *workspace, int64_t workspace_bytes, hdfe_pcg_info *info,
                    cudaStream_t s)
{
    int blocks = pcg::grid_blocks_for(k);
    if (blocks < 1) return hdfe_set_cuda_error(cudaGetLastError());
    pcg::Layout lay = pcg::layout(L, k, blocks);
    if (workspace_bytes < lay.total)
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_pcg_solve: workspace too small");
    char *ws = (char *)workspace;
    pcg::Params p{};
    p.indptr = indptr;
    p.indices = indices;
    p.data = data;
    p.L = L;
    p.nnz = nnz;
    p.Lb = small_count > 0 ? small_first : L;
    p.ns = small_count;
    p.cross = cross;
    p.small = small;
    const int64_t warps = (int64_t)blocks * (pcg::threads_for(k) / 32);
    p.nwarps = warps;
    p.dinv = dinv;
    p.B = B;
    p.zero = zero;
    p.X0 = X0;
    p.tol = tol;
    p.maxiter = maxiter;
    p.X = X;
    p.R = (double *)(ws + lay.r);
    p.P = (double *)(ws + lay.p);
    p.AP = (double *)(ws + lay.ap);
    p.carry = (double *)(ws + lay.carry);
    p.part = (double *)(ws + lay.part);
    p.wfirst = (int64_t *)(ws + lay.wfirst);
    p.wlo = (int64_t *)(ws + lay.wlo);
    p.cut = (uint8_t *)(ws + lay.cut);
    p.bar = (unsigned *)(ws + lay.bar);
    p.info = info;
    HDFE_CUDA_TRY(cudaMemsetAsync(p.bar, 0, 16, s));
    pcg::k_partition<<<(unsigned)((p.nwarps + 256) / 256), 256, 0, s>>>(indptr, L, nnz, p.nwarps,
                                                                      pcg::kRowCost, (int64_t *)p.wlo);
    cudaError_t e = cudaErrorInvalidValue;
    const bool short_rows = nnz <= pcg::kShortRowNnz * L;
    switch (k) {
    case 1: e = short_rows ? pcg::launch<1, pcg::kShortLpr>(p, blocks, s) : pcg::launch<1>(p, blocks, s); break;
    case 2: e = short_rows ? pcg::launch<2, pcg::kShortLpr>(p, blocks, s) : pcg::launch<2>(p, blocks, s); break;
    case 3: e = short_rows ? pcg::launch<3, pcg::kShortLpr>(p, blocks, s) : pcg::launch<3>(p, blocks, s); break;
    case 4: e = short_rows ? pcg::launch<4, pcg::kShortLpr>(p, blocks, s) : pcg::launch<4>(p, blocks, s); break;
    case 5: e = pcg::launch<5>(p, blocks, s); break;
    case 6: e = pcg::launch<6>(p, blocks, s); break;
    case 7: e = pcg::launch<7>(p, blocks, s); break;
    case 8: e = pcg::launch<8>(p, blocks, s); break;
    }
    HDFE_CUDA_TRY(e);
    pcg::pcg_status_kernel<<<1, 32, 0, s>>>(p.bar, info);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(3);
    return HDFE_OK;
}

}  // namespace

extern "C" int hdfe_pcg_solve(const int64_t *indptr, const int32_t *indices, const double *data,
                              int64_t L, int64_t nnz, const double *dinv, const double *B,
                              int32_t k, const uint8_t *zero, const double *X0, double tol,
                              int64_t maxiter, double *X, void *workspace,
                              int64_t workspace_bytes, hdfe_pcg_info *info, void *stream)
{
    if (k < 1 || k > HDFE_PCG_MAX_K || L < 1 || nnz < 0 || !indptr || !dinv || !B || !X ||
        !info || !workspace || maxiter < 0 || (nnz > 0 && (!indices || !data)))
        return hdfe_set_arg_error("hdfe_pcg_solve: bad argument");
    if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
        return hdfe_set_arg_error("hdfe_pcg_solve: workspace must be 256-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    if (pcg::use_lanes(k)) return pcg::solve_lanes(indptr, indices, data, L, nnz, dinv, B, k, zero,
                                                   X0, tol, maxiter, X, workspace,
                                                   workspace_bytes, info, s);
    return solve_registers(indptr, indices, data, L, nnz, L, 0, nullptr, nullptr, dinv, B, k, zero,
                           X0, tol, maxiter, X, workspace, workspace_bytes, info, s);
}

extern "C" int hdfe_pcg_solve_small(const int64_t *indptr, const int32_t *indices,
                                    const double *data, int64_t L, int64_t nnz,
                                    int64_t small_first, int32_t small_count,
                                    const double *cross, const double *small, const double *dinv,
                                    const double *B, int32_t k, const uint8_t *zero,
                                    const double *X0, double tol, int64_t maxiter, double *X,
                                    void *workspace, int64_t workspace_bytes,
                                    hdfe_pcg_info *info, void *stream)
{
    if (k < 1 || k > HDFE_PCG_SMALL_MAX_K || L < 1 || nnz < 0 || !indptr || !dinv || !B || !X ||
        !info || !workspace || maxiter < 0 || (nnz > 0 && (!indices || !data)) ||
        small_count < 1 || small_count > HDFE_SMALL_MAX_LEVELS || small_first < 0 ||
        small_first + small_count != L || !cross || !small)
        return hdfe_set_arg_error("hdfe_pcg_solve_small: bad argument");
    if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
        return hdfe_set_arg_error("hdfe_pcg_solve_small: workspace must be 256-byte aligned");
    return solve_registers(indptr, indices, data, L, nnz, small_first, small_count, cross, small,
                           dinv, B, k, zero, X0, tol, maxiter, X, workspace, workspace_bytes,
                           info, (cudaStream_t)stream);
}

// ------------------------------------------------ allocation-free variant
//
// Some callers cannot allocate device memory for the solver's scratch: a
// host binding that has no CUDA allocator of its own (a thin FFI layer from
// another language runtime), or code that must not call cudaMalloc because
// it synchronises the device and would stall other work in flight.  For
// them hdfe_pcg_solve_noalloc keeps the scratch in this file-scope device
// array instead of a caller-provided workspace.  Every GPU that loads the
// library holds the array until the process exits.

static __device__ __align__(256) unsigned char g_pcg_scratch[HDFE_PCG_NOALLOC_BYTES];

namespace {
// the array's device address, looked up once per device (with that device
// current): in host code the symbol is only a host-side stand-in
void *g_scratch_addr[64] = {};
}

extern "C" int hdfe_pcg_solve_noalloc(const int64_t *indptr, const int32_t *indices,
                                      const double *data, int64_t L, int64_t nnz,
                                      const double *dinv, const double *B, int32_t k,
                                      const uint8_t *zero, const double *X0, double tol,
                                      int64_t maxiter, double *X, hdfe_pcg_info *info,
                                      void *stream)
{
    if (k < 1 || k > HDFE_PCG_MAX_K || L < 1)
        return hdfe_set_arg_error("hdfe_pcg_solve_noalloc: bad argument");
    const int64_t need = hdfe_pcg_workspace_bytes(L, nnz, k);
    if (need < 0) return hdfe_set_cuda_error(cudaGetLastError());
    if (need > (int64_t)HDFE_PCG_NOALLOC_BYTES)
        return hdfe_set_error(HDFE_ERR_WORKSPACE,
                              "hdfe_pcg_solve_noalloc: L x k too large for the built-in scratch "
                              "(HDFE_PCG_NOALLOC_BYTES); use hdfe_pcg_solve with a workspace");
    int dev = 0;
    HDFE_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return hdfe_set_arg_error("hdfe_pcg_solve_noalloc: device index");
    if (g_scratch_addr[dev] == nullptr) {
        void *ptr = nullptr;
        HDFE_CUDA_TRY(cudaGetSymbolAddress(&ptr, g_pcg_scratch));
        g_scratch_addr[dev] = ptr;
    }
    return hdfe_pcg_solve(indptr, indices, data, L, nnz, dinv, B, k, zero, X0, tol, maxiter, X,
                          g_scratch_addr[dev], (int64_t)HDFE_PCG_NOALLOC_BYTES, info, stream);
}

// ---------------------------------------------- mixed precision (refined)
//
// The same solve with the inner CG in FP32 and iterative refinement in FP64:
//   outer:  R = B - S X in FP64 (S's FP64 values); rel = ||R|| / ||B||; stop
//           when every column meets tol;
//   inner:  Jacobi PCG on S D = R with S's values, the vectors and the
//           products in FP32 (half the bytes per iteration), its dot products
//           and norms accumulated in FP64, until ||R_inner|| <= inner_tol ||R||;
//   update: X += D in FP64.
// Columns, zero columns, warm starts and the reported relative residual follow
// hdfe_pcg_solve; `iterations` counts inner iterations, bounded by maxiter.
namespace hdfe {
namespace pcg {

template <int K>
struct FStride {     // FP32 P's row stride: 1, 2, or a multiple of 4 (16-byte rows)
    static constexpr int P = K == 1 ? 1 : (K == 2 ? 2 : ((K + 3) / 4) * 4);
    static constexpr int VW = P % 4 == 0 ? 4 : (P % 2 == 0 ? 2 : 1);
};

struct Mixed {
    const float *data32;
    float *R, *P, *AP, *D;      // inner vectors
    double *AX;                 // FP64 S X, then the FP64 residual
    double inner_tol;
};

struct MixedLayout {
    int64_t r, p, ap, d, ax, carry, part, wfirst, wlo, cut, bar, total;
};

inline MixedLayout mixed_layout(int64_t L, int k, int64_t blocks)
{
    MixedLayout o;
    const int kf = k == 1 ? 1 : (k == 2 ? 2 : ((k + 3) / 4) * 4);
    int64_t p = 0;
    auto take = [&](int64_t bytes) { int64_t at = p; p += (bytes + 255) / 256 * 256; return at; };
    o.r = take(L * k * 4);
    o.p = take(L * kf * 4);
    o.ap = take(L * k * 4);
    o.d = take(L * k * 4);
    o.ax = take(L * k * 8);
    const int64_t warps = blocks * (threads_for(k) / 32);
    o.carry = take(warps * 2 * k * 8);
    o.part = take(4 * (int64_t)k * blocks * 8);
    o.wfirst = take(warps * 8);
    o.wlo = take((warps + 1) * 8);
    o.cut = take(L);
    o.bar = take(64);
    o.total = p;
    return o;
}

template <int K>
__global__ void __launch_bounds__(threads_for(K), 1) mixed_kernel(Params a, Mixed f)
{
    constexpr int KF = FStride<K>::P;
    constexpr int VWF = FStride<K>::VW;
    __shared__ double s_red[4 * K];
    __shared__ double s_scratch[kMaxWarps * 3 * K];
    GridBarrier gb{a.bar};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t gstride = (int64_t)gridDim.x * blockDim.x;
    const int64_t L = a.L;
    const int nb = gridDim.x;
    float *carry32 = reinterpret_cast<float *>(a.carry);

    double bnorm[K], rel[K];
    bool active[K], zero[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
        zero[k] = a.zero != nullptr && a.zero[k] != 0;
        active[k] = !zero[k];
        rel[k] = 0.0;
    }
    // each warp's first row and the cut flags, X = X0 (or 0), ||B||
    {
        const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
        const int64_t lo = a.wlo[gw];
        if (lane == 0 && lo < a.nnz) a.wfirst[gw] = upper_bound(a.indptr, L + 1, lo) - 1;
        __syncwarp();
        double sb[K];
#pragma unroll
        for (int k = 0; k < K; k++) sb[k] = 0.0;
        for (int64_t r = gtid; r < L; r += gstride) {
            const int64_t rs = a.indptr[r], re = a.indptr[r + 1];
            a.cut[r] = (re > rs && warp_of(a, rs) != warp_of(a, re - 1)) ? 1 : 0;
#pragma unroll
            for (int k = 0; k < K; k++) {
                const double b = a.B[r * K + k];
                sb[k] += b * b;
                a.X[r * K + k] = (a.X0 != nullptr && !zero[k]) ? a.X0[r * K + k] : 0.0;
            }
        }
        block_partials<K>(sb, s_scratch, a.part, 0, nb);
        if (!gb.sync()) return;
        if (warp == 0) {
            for (int k = 0; k < K; k++) {
                const double t = reduce_part(a.part, k);
                if (lane == 0) s_red[k] = t;
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < K; k++) {
            const double bn = sqrt(s_red[k]);
            bnorm[k] = bn == 0.0 ? 1.0 : bn;
        }
    }
    int64_t total = 0;
    bool any_active = false;
    double dot[K];
    for (int64_t outer = 0;; outer++) {
        // ---- FP64 residual R = B - S X (into AX)
        const bool have_x = outer > 0 || a.X0 != nullptr;
        if (have_x) {
#pragma unroll
            for (int k = 0; k < K; k++) dot[k] = 0.0;
            spmm_range<K, K, 1, double>(a, a.data, a.X, f.AX, a.carry, dot, false);
            if (!gb.sync()) return;
        }
        double sr[K];
#pragma unroll
        for (int k = 0; k < K; k++) sr[k] = 0.0;
        auto resid_row = [&](int64_t r, const double (&ax)[K]) {
#pragma unroll
            for (int k = 0; k < K; k++) {
                const double res = zero[k] ? 0.0 : a.B[r * K + k] - ax[k];
                f.AX[r * K + k] = res;
                sr[k] += res * res;
            }
        };
        for (int64_t r = gtid; r < L; r += gstride) {
            if (have_x && a.cut[r]) continue;
            const bool empty = a.indptr[r + 1] == a.indptr[r];
            double ax[K];
#pragma unroll
            for (int k = 0; k < K; k++) ax[k] = (have_x && !empty) ? f.AX[r * K + k] : 0.0;
            resid_row(r, ax);
        }
        if (have_x) {
            int64_t r;
            double ax[K];
            if (finish_cut_row<K, double>(a, a.carry, r, ax) && lane == 0) resid_row(r, ax);
        }
        block_partials<K>(sr, s_scratch, a.part, K, nb);
        if (!gb.sync()) return;
        if (warp == 0) {
            for (int k = 0; k < K; k++) {
                const double t = reduce_part(a.part, K + k);
                if (lane == 0) s_red[K + k] = t;
            }
        }
        __syncthreads();
        any_active = false;
        double rnorm[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            rnorm[k] = sqrt(s_red[K + k]);
            rel[k] = rnorm[k] / bnorm[k];
            active[k] = !zero[k] && rel[k] > a.tol;
            any_active |= active[k];
        }
        if (!any_active || total >= a.maxiter) break;
        // ---- inner FP32 PCG on S D = R
        double rz[K];
        {
            double sz[K];
#pragma unroll
            for (int k = 0; k < K; k++) sz[k] = 0.0;
            for (int64_t r = gtid; r < L; r += gstride) {
                const float di = (float)a.dinv[r];
#pragma unroll
                for (int k = 0; k < K; k++) {
                    const float res = active[k] ? (float)f.AX[r * K + k] : 0.0f;
                    f.R[r * K + k] = res;
                    f.D[r * K + k] = 0.0f;
                    const float z = res * di;
                    f.P[r * KF + k] = z;
                    sz[k] += (double)res * (double)z;
                }
#pragma unroll
                for (int k = K; k < KF; k++) f.P[r * KF + k] = 0.0f;
            }
            block_partials<K>(sz, s_scratch, a.part, 2 * K, nb);
            if (!gb.sync()) return;
            if (warp == 0) {
                for (int k = 0; k < K; k++) {
                    const double t = reduce_part(a.part, 2 * K + k);
                    if (lane == 0) s_red[2 * K + k] = t;
                }
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < K; k++) rz[k] = s_red[2 * K + k];
        }
        bool inner_active[K];
#pragma unroll
        for (int k = 0; k < K; k++) inner_active[k] = active[k];
        while (total < a.maxiter) {
            total++;
            // A: AP = S P (FP32), p'Ap in FP64
#pragma unroll
            for (int k = 0; k < K; k++) dot[k] = 0.0;
            spmm_range<K, KF, VWF, float>(a, f.data32, f.P, f.AP, carry32, dot, true);
            block_partials<K>(dot, s_scratch, a.part, 0, nb);
            if (!gb.sync()) return;
            if (warp == 0) {
                for (int k = 0; k < K; k++) {
                    const double t = reduce_part(a.part, k);
                    if (lane == 0) s_red[k] = t;
                }
            }
            __syncthreads();
            float alpha[K];
#pragma unroll
            for (int k = 0; k < K; k++) {
                const double pap = s_red[k];
                alpha[k] = (inner_active[k] && pap > 0.0) ? (float)(rz[k] / pap) : 0.0f;
            }
            __syncthreads();
            // B: D += alpha P, R -= alpha AP; sums of R^2 and R^2 dinv in FP64
            double s1[K], s2[K];
#pragma unroll
            for (int k = 0; k < K; k++) s1[k] = s2[k] = 0.0;
            auto step_row = [&](int64_t r, const float (&ap)[K]) {
                const double di = a.dinv[r];
#pragma unroll
                for (int k = 0; k < K; k++) {
                    f.D[r * K + k] += alpha[k] * f.P[r * KF + k];
                    const float res = f.R[r * K + k] - alpha[k] * ap[k];
                    f.R[r * K + k] = res;
                    const double rd = (double)res;
                    s1[k] += rd * rd;
                    s2[k] += rd * rd * di;
                }
            };
            for (int64_t r = gtid; r < L; r += gstride) {
                if (a.cut[r]) continue;
                float ap[K];
                const bool empty = a.indptr[r + 1] == a.indptr[r];
#pragma unroll
                for (int k = 0; k < K; k++) ap[k] = empty ? 0.0f : f.AP[r * K + k];
                step_row(r, ap);
            }
            {
                int64_t r;
                float ap[K];
                if (finish_cut_row<K, float>(a, carry32, r, ap) && lane == 0) step_row(r, ap);
            }
            {
                double v[2 * K];
#pragma unroll
                for (int k = 0; k < K; k++) { v[k] = s1[k]; v[K + k] = s2[k]; }
                block_partials<2 * K>(v, s_scratch, a.part, K, nb);
            }
            if (!gb.sync()) return;
            if (warp < 2) {
                for (int k = 0; k < K; k++) {
                    const double t = reduce_part(a.part, (warp + 1) * K + k);
                    if (lane == 0) s_red[(warp + 1) * K + k] = t;
                }
            }
            __syncthreads();
            // C: inner convergence, beta, P = dinv R + beta P
            bool any_inner = false;
            float beta[K];
#pragma unroll
            for (int k = 0; k < K; k++) {
                inner_active[k] = inner_active[k] && sqrt(s_red[K + k]) > f.inner_tol * rnorm[k];
                any_inner |= inner_active[k];
            }
            if (!any_inner) break;
#pragma unroll
            for (int k = 0; k < K; k++) {
                const double rzn = s_red[2 * K + k];
                beta[k] = inner_active[k] ? (float)(rzn / (rz[k] != 0.0 ? rz[k] : 1.0)) : 0.0f;
                rz[k] = rzn;
            }
            __syncthreads();
            for (int64_t r = gtid; r < L; r += gstride) {
                const float di = (float)a.dinv[r];
#pragma unroll
                for (int k = 0; k < K; k++)
                    f.P[r * KF + k] = f.R[r * K + k] * di + beta[k] * f.P[r * KF + k];
            }
            if (!gb.sync()) return;
        }
        // ---- X += D in FP64, then a barrier before the next product reads X
        for (int64_t r = gtid; r < L; r += gstride) {
#pragma unroll
            for (int k = 0; k < K; k++)
                if (active[k]) a.X[r * K + k] += (double)f.D[r * K + k];
        }
        if (!gb.sync()) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double mx = 0.0;
#pragma unroll
        for (int k = 0; k < K; k++) mx = fmax(mx, rel[k]);
        a.info->iterations = total;
        a.info->converged = any_active ? 0 : 1;
        a.info->status = HDFE_OK;
        a.info->max_rel = mx;
    }
}

// ------------------------------------------- mixed precision, wide blocks
//
// The refined solve for blocks of 5 to 32 columns (the JLA's probe blocks),
// one column per lane as in lane_kernel: the FP64 residual B - S X uses S's
// FP64 values and the FP64 iterate; the inner PCG runs on S's FP32 values and
// FP32 vectors R, P, AP, D with FP32 products and updates (p'Ap, the norms and
// r'z accumulated in FP64); X += D in FP64.  Per inner iteration the bytes are
// S's 8 per nonzero and 4 per vector element instead of 12 and 8.
struct MixedLane {
    const float *data32;
    float *R, *P, *AP, *D;
    double *AX;                 // S X, then the FP64 residual
    double inner_tol;
};

struct MixedLaneLayout {
    int64_t r, p, ap, d, ax, x, carry, part, wfirst, wlo, cut, bar, total;
};

inline MixedLaneLayout mixed_lane_layout(int64_t L, int k, int64_t blocks)
{
    MixedLaneLayout o;
    const int kw = lane_width(k);
    const int64_t warps = blocks * (lane_threads(kw) / 32);
    int64_t p = 0;
    auto take = [&](int64_t bytes) { int64_t at = p; p += (bytes + 255) / 256 * 256; return at; };
    o.r = take(L * kw * 4);
    o.p = take(L * kw * 4);
    o.ap = take(L * kw * 4);
    o.d = take(L * kw * 4);
    o.ax = take(L * kw * 8);
    o.x = k == kw ? -1 : take(L * kw * 8);
    o.carry = take(warps * 2 * kw * 8);
    o.part = take(3 * (int64_t)kw * blocks * 8);
    o.wfirst = take(warps * 8);
    o.wlo = take((warps + 1) * 8);
    o.cut = take(L);
    o.bar = take(64);
    o.total = p;
    return o;
}

template <int K>
__global__ void __launch_bounds__(lane_threads(K), 1) mixed_lane_kernel(Params a, LaneArgs x,
                                                                        MixedLane f)
{
    constexpr int RU = lane_ru(K);
    extern __shared__ double s_stage[];
    __shared__ double s_red[3 * K];
    __shared__ double s_scratch[(lane_threads(K) / 32) * 3 * K];
    __shared__ double s_rel[K];
    __shared__ int s_active[K];
    GridBarrier gb{a.bar};
    const int lane = threadIdx.x & 31, col = lane % K;
    const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t gstride = (int64_t)gridDim.x * blockDim.x;
    const int64_t L = a.L, LK = a.L * K;
    const int nb = gridDim.x;
    const int kc = x.k;
    double *Xw = x.Xw;
    const bool zero_c = col >= kc || (a.zero != nullptr && a.zero[col] != 0);
    double *stage = s_stage + (threadIdx.x >> 5) * kLaneStages * 32 * (K + 1);
    float *stage32 = reinterpret_cast<float *>(stage);
    float *carry32 = reinterpret_cast<float *>(a.carry);

    // ---- set-up: each warp's first row, the cut flags, X = X0 (or 0), ||B||
    {
        const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
        const int64_t lo = a.wlo[gw];
        if (lane == 0 && lo < a.nnz) a.wfirst[gw] = upper_bound(a.indptr, L + 1, lo) - 1;
        __syncwarp();
        for (int64_t r = gtid; r < L; r += gstride) {
            const int64_t rs = a.indptr[r], re = a.indptr[r + 1];
            a.cut[r] = (re > rs && warp_of(a, rs) != warp_of(a, re - 1) ? kRowCut : 0) |
                       (re == rs ? kRowEmpty : 0);
        }
    }
    double bnorm_c;
    {
        double v[1] = {0.0};
        for (int64_t t = gtid; t < LK; t += gstride) {
            const int64_t r = t / K;
            const double b = col < kc ? a.B[r * kc + col] : 0.0;
            v[0] += b * b;
            Xw[t] = (a.X0 != nullptr && !zero_c) ? a.X0[r * kc + col] : 0.0;
        }
        column_partials<K, 1>(v, s_scratch, a.part, 0, nb);
        if (!gb.sync()) return;
        reduce_range(a.part, 0, K, s_red);
        const double bn = sqrt(s_red[col]);
        bnorm_c = bn == 0.0 ? 1.0 : bn;
    }
    int64_t total = 0;
    double rel_c = 0.0;
    bool active_c = false;
    for (int64_t outer = 0;; outer++) {
        // ---- the FP64 residual B - S X (into AX), its norm
        const bool have_x = outer > 0 || a.X0 != nullptr;
        double dot = 0.0;
        if (have_x) {
            lane_spmm<K, double>(a, a.data, Xw, f.AX, a.carry, dot, false, stage);
            if (!gb.sync()) return;
        }
        double v1[1] = {0.0};
        auto resid = [&](int64_t r, double ax) {
            const int64_t t = r * K + col;
            const double res = zero_c ? 0.0 : a.B[r * kc + col] - ax;
            f.AX[t] = res;
            v1[0] += res * res;
        };
        for (int64_t t = gtid; t < LK; t += gstride) {
            const int64_t r = t / K;
            const uint8_t fl = a.cut[r];
            if (have_x && (fl & kRowCut)) continue;
            resid(r, (have_x && !(fl & kRowEmpty)) ? f.AX[t] : 0.0);
        }
        if (have_x) {
            int64_t r;
            double ap;
            if (lane_finish_cut<K, double>(a, a.carry, r, ap) && lane < K) resid(r, ap);
        }
        column_partials<K, 1>(v1, s_scratch, a.part, 1, nb);
        if (!gb.sync()) return;
        reduce_range(a.part, K, 2 * K, s_red);
        const double rnorm_c = sqrt(s_red[K + col]);
        rel_c = rnorm_c / bnorm_c;
        active_c = !zero_c && rel_c > a.tol;
        if (threadIdx.x < K) {
            s_rel[col] = zero_c ? 0.0 : rel_c;
            s_active[col] = active_c ? 1 : 0;
        }
        if (!__syncthreads_or(active_c) || total >= a.maxiter) break;
        // ---- inner FP32 PCG on S D = R: R, D = 0, P = dinv R, r'z
        double rz_c;
        {
            double v[1] = {0.0};
            for (int64_t t = gtid; t < LK; t += gstride) {
                const float di = (float)a.dinv[t / K];
                const float res = active_c ? (float)f.AX[t] : 0.0f;
                f.R[t] = res;
                f.D[t] = 0.0f;
                const float z = res * di;
                f.P[t] = z;
                v[0] += (double)res * (double)z;
            }
            column_partials<K, 1>(v, s_scratch, a.part, 2, nb);
            if (!gb.sync()) return;
            reduce_range(a.part, 2 * K, 3 * K, s_red);
            rz_c = s_red[2 * K + col];
        }
        bool inner_c = active_c;
        while (total < a.maxiter) {
            total++;
            // A: AP = S P in FP32, p'Ap in FP64
            dot = 0.0;
            lane_spmm<K, float>(a, f.data32, f.P, f.AP, carry32, dot, true, stage32);
            {
                double v[1] = {dot};
                column_partials<K, 1>(v, s_scratch, a.part, 0, nb);
            }
            if (!gb.sync()) return;
            reduce_range(a.part, 0, K, s_red);
            const double pap = s_red[col];
            const float alpha = (inner_c && pap > 0.0) ? (float)(rz_c / pap) : 0.0f;
            // B: D += alpha P, R -= alpha AP; sums of R^2 and R^2 dinv in FP64
            double v[2] = {0.0, 0.0};
            auto step = [&](int64_t r, float ap) {
                const double di = a.dinv[r];
                const int64_t t = r * K + col;
                f.D[t] += alpha * f.P[t];
                const float res = f.R[t] - alpha * ap;
                f.R[t] = res;
                const double rd = (double)res;
                v[0] += rd * rd;
                v[1] += rd * rd * di;
            };
            for (int64_t t0 = gtid; t0 < LK; t0 += RU * gstride) {
                uint8_t fl[RU];
                float ap[RU], pv[RU], dv[RU], rv[RU];
                double di[RU];
#pragma unroll
                for (int u = 0; u < RU; u++) {
                    const int64_t t = t0 + u * gstride;
                    fl[u] = kRowCut;
                    if (t < LK) {
                        const int64_t r = t / K;
                        fl[u] = a.cut[r];
                        ap[u] = f.AP[t];
                        pv[u] = f.P[t];
                        dv[u] = f.D[t];
                        rv[u] = f.R[t];
                        di[u] = a.dinv[r];
                    }
                }
#pragma unroll
                for (int u = 0; u < RU; u++) {
                    if (fl[u] & kRowCut) continue;      // also the slots past the end
                    const int64_t t = t0 + u * gstride;
                    f.D[t] = dv[u] + alpha * pv[u];
                    const float res = rv[u] - alpha * ((fl[u] & kRowEmpty) ? 0.0f : ap[u]);
                    f.R[t] = res;
                    const double rd = (double)res;
                    v[0] += rd * rd;
                    v[1] += rd * rd * di[u];
                }
            }
            {
                int64_t r;
                float ap;
                if (lane_finish_cut<K, float>(a, carry32, r, ap) && lane < K) step(r, ap);
            }
            column_partials<K, 2>(v, s_scratch, a.part, 1, nb);
            if (!gb.sync()) return;
            reduce_range(a.part, K, 3 * K, s_red);
            // C: inner convergence, beta, P = dinv R + beta P
            inner_c = inner_c && sqrt(s_red[K + col]) > f.inner_tol * rnorm_c;
            if (!__syncthreads_or(inner_c)) break;
            const double rzn = s_red[2 * K + col];
            const float beta = inner_c ? (float)(rzn / (rz_c != 0.0 ? rz_c : 1.0)) : 0.0f;
            rz_c = rzn;
            for (int64_t t0 = gtid; t0 < LK; t0 += RU * gstride) {
                float rv[RU], pv[RU], di[RU];
#pragma unroll
                for (int u = 0; u < RU; u++) {
                    const int64_t t = t0 + u * gstride;
                    if (t < LK) {
                        rv[u] = f.R[t];
                        pv[u] = f.P[t];
                        di[u] = (float)a.dinv[t / K];
                    }
                }
#pragma unroll
                for (int u = 0; u < RU; u++) {
                    const int64_t t = t0 + u * gstride;
                    if (t < LK) f.P[t] = rv[u] * di[u] + beta * pv[u];
                }
            }
            if (!gb.sync()) return;
        }
        // ---- X += D in FP64, then a barrier before the next product reads X
        for (int64_t t = gtid; t < LK; t += gstride)
            if (active_c) Xw[t] += (double)f.D[t];
        if (!gb.sync()) return;
    }
    // ---- the iterate to the caller's X (stride k)
    if (Xw != a.X) {
        for (int64_t t = gtid; t < LK; t += gstride)
            if (col < kc) a.X[(t / K) * kc + col] = Xw[t];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double mx = 0.0;
        bool conv = true;
        for (int c = 0; c < kc; c++) {
            mx = fmax(mx, s_rel[c]);
            conv &= s_active[c] == 0;
        }
        a.info->iterations = total;
        a.info->converged = conv ? 1 : 0;
        a.info->status = HDFE_OK;
        a.info->max_rel = mx;
    }
}

template <int K>
int mixed_lane_grid()
{
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    if (cudaFuncSetAttribute(mixed_lane_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             lane_smem_bytes(K)) != cudaSuccess)
        return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mixed_lane_kernel<K>,
                                                      lane_threads(K), lane_smem_bytes(K)) !=
        cudaSuccess)
        return -1;
    return per_sm < 1 ? -1 : (sms < 32 * kRedLoads ? sms : 32 * kRedLoads);
}

int mixed_lane_grid_for(int kw)
{
    static int cache[64][3] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -1;
    const int i = kw == 8 ? 0 : (kw == 16 ? 1 : 2);
    if (cache[dev][i] == 0)
        cache[dev][i] = kw == 8 ? mixed_lane_grid<8>()
                                : (kw == 16 ? mixed_lane_grid<16>() : mixed_lane_grid<32>());
    return cache[dev][i];
}

template <int K>
cudaError_t launch_mixed_lanes(Params p, LaneArgs x, MixedLane m, int blocks, cudaStream_t s)
{
    void *args[] = {&p, &x, &m};
    return cudaLaunchCooperativeKernel((const void *)mixed_lane_kernel<K>, dim3(blocks),
                                       dim3(lane_threads(K)), args, lane_smem_bytes(K), s);
}

template <int K>
int mixed_grid()
{
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mixed_kernel<K>, threads_for(K), 0) !=
        cudaSuccess)
        return -1;
    return per_sm < 1 ? -1 : sms;
}

int mixed_grid_for(int k)
{
    static int cache[64][5] = {};
    int dev = 0;
    if (k < 1 || k > 4) return -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -1;
    if (cache[dev][k] == 0) {
        switch (k) {
        case 1: cache[dev][k] = mixed_grid<1>(); break;
        case 2: cache[dev][k] = mixed_grid<2>(); break;
        case 3: cache[dev][k] = mixed_grid<3>(); break;
        case 4: cache[dev][k] = mixed_grid<4>(); break;
        default: return -1;
        }
    }
    return cache[dev][k];
}

template <int K>
cudaError_t launch_mixed(Params p, Mixed m, int blocks, cudaStream_t s)
{
    void *args[] = {&p, &m};
    return cudaLaunchCooperativeKernel((const void *)mixed_kernel<K>, dim3(blocks),
                                       dim3(threads_for(K)), args, 0, s);
}

}  // namespace pcg
}  // namespace hdfe

extern "C" int64_t hdfe_pcg_mixed_workspace_bytes(int64_t L, int64_t nnz, int32_t k)
{
    (void)nnz;
    if (k < 1 || k > HDFE_PCG_MIXED_MAX_K || L < 0) return -1;
    if (pcg::use_lanes(k)) {
        const int blocks = pcg::mixed_lane_grid_for(pcg::lane_width(k));
        return blocks < 1 ? -1 : pcg::mixed_lane_layout(L, k, blocks).total;
    }
    const int blocks = pcg::mixed_grid_for(k);
    if (blocks < 1) return -1;
    return pcg::mixed_layout(L, k, blocks).total;
}

namespace hdfe {
namespace pcg {

int solve_mixed_lanes(const int64_t *indptr, const int32_t *indices, const double *data,
                      const float *data32, int64_t L, int64_t nnz, const double *dinv,
                      const double *B, int32_t k, const uint8_t *zero, const double *X0,
                      double tol, double inner_tol, int64_t maxiter, double *X, void *workspace,
                      int64_t workspace_bytes, hdfe_pcg_info *info, cudaStream_t s)
{
    const int kw = lane_width(k);
    const int blocks = mixed_lane_grid_for(kw);
    if (blocks < 1) return hdfe_set_cuda_error(cudaGetLastError());
    const MixedLaneLayout lay = mixed_lane_layout(L, k, blocks);
    if (workspace_bytes < lay.total)
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_pcg_solve_mixed: workspace too small");
    char *ws = (char *)workspace;
    Params p{};
    p.indptr = indptr;
    p.indices = indices;
    p.data = data;
    p.L = L;
    p.nnz = nnz;
    p.nwarps = (int64_t)blocks * (lane_threads(kw) / 32);
    p.dinv = dinv;
    p.B = B;
    p.zero = zero;
    p.X0 = X0;
    p.tol = tol;
    p.maxiter = maxiter;
    p.X = X;
    p.carry = (double *)(ws + lay.carry);
    p.part = (double *)(ws + lay.part);
    p.wfirst = (int64_t *)(ws + lay.wfirst);
    p.wlo = (int64_t *)(ws + lay.wlo);
    p.cut = (uint8_t *)(ws + lay.cut);
    p.bar = (unsigned *)(ws + lay.bar);
    p.info = info;
    LaneArgs x;
    x.Xw = lay.x < 0 ? X : (double *)(ws + lay.x);
    x.k = k;
    MixedLane m;
    m.data32 = data32;
    m.R = (float *)(ws + lay.r);
    m.P = (float *)(ws + lay.p);
    m.AP = (float *)(ws + lay.ap);
    m.D = (float *)(ws + lay.d);
    m.AX = (double *)(ws + lay.ax);
    m.inner_tol = inner_tol;
    HDFE_CUDA_TRY(cudaMemsetAsync(p.bar, 0, 16, s));
    k_partition<<<(unsigned)((p.nwarps + 256) / 256), 256, 0, s>>>(indptr, L, nnz, p.nwarps, 0,
                                                                   (int64_t *)p.wlo);
    cudaError_t e = kw == 8 ? launch_mixed_lanes<8>(p, x, m, blocks, s)
                  : kw == 16 ? launch_mixed_lanes<16>(p, x, m, blocks, s)
                             : launch_mixed_lanes<32>(p, x, m, blocks, s);
    HDFE_CUDA_TRY(e);
    pcg_status_kernel<<<1, 32, 0, s>>>(p.bar, info);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(3);
    return HDFE_OK;
}

}  // namespace pcg
}  // namespace hdfe

extern "C" int hdfe_pcg_solve_mixed(const int64_t *indptr, const int32_t *indices,
                                    const double *data, const float *data32, int64_t L,
                                    int64_t nnz, const double *dinv, const double *B, int32_t k,
                                    const uint8_t *zero, const double *X0, double tol,
                                    double inner_tol, int64_t maxiter, double *X,
                                    void *workspace, int64_t workspace_bytes,
                                    hdfe_pcg_info *info, void *stream)
{
    if (k < 1 || k > HDFE_PCG_MIXED_MAX_K || L < 1 || nnz < 0 || !indptr || !dinv || !B || !X ||
        !info || !workspace || maxiter < 0 || !(inner_tol > 0.0 && inner_tol < 1.0) ||
        (nnz > 0 && (!indices || !data || !data32)))
        return hdfe_set_arg_error("hdfe_pcg_solve_mixed: bad argument");
    if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
        return hdfe_set_arg_error("hdfe_pcg_solve_mixed: workspace must be 256-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    if (pcg::use_lanes(k))
        return pcg::solve_mixed_lanes(indptr, indices, data, data32, L, nnz, dinv, B, k, zero, X0,
                                      tol, inner_tol, maxiter, X, workspace, workspace_bytes, info,
                                      s);
    const int blocks = pcg::mixed_grid_for(k);
    if (blocks < 1) return hdfe_set_cuda_error(cudaGetLastError());
    const pcg::MixedLayout lay = pcg::mixed_layout(L, k, blocks);
    if (workspace_bytes < lay.total)
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_pcg_solve_mixed: workspace too small");
    char *ws = (char *)workspace;
    pcg::Params p{};
    p.indptr = indptr;
    p.indices = indices;
    p.data = data;
    p.L = L;
    p.nnz = nnz;
    const int64_t warps = (int64_t)blocks * (pcg::threads_for(k) / 32);
    p.nwarps = warps;
    p.dinv = dinv;
    p.B = B;
    p.zero = zero;
    p.X0 = X0;
    p.tol = tol;
    p.maxiter = maxiter;
    p.X = X;
    p.carry = (double *)(ws + lay.carry);
    p.part = (double *)(ws + lay.part);
    p.wfirst = (int64_t *)(ws + lay.wfirst);
    p.wlo = (int64_t *)(ws + lay.wlo);
    p.cut = (uint8_t *)(ws + lay.cut);
    p.bar = (unsigned *)(ws + lay.bar);
    p.info = info;
    pcg::Mixed m;
    m.data32 = data32;
    m.R = (float *)(ws + lay.r);
    m.P = (float *)(ws + lay.p);
    m.AP = (float *)(ws + lay.ap);
    m.D = (float *)(ws + lay.d);
    m.AX = (double *)(ws + lay.ax);
    m.inner_tol = inner_tol;
    HDFE_CUDA_TRY(cudaMemsetAsync(p.bar, 0, 16, s));
    pcg::k_partition<<<(unsigned)((p.nwarps + 256) / 256), 256, 0, s>>>(indptr, L, nnz, p.nwarps,
                                                                      pcg::kRowCost, (int64_t *)p.wlo);
    cudaError_t e = cudaErrorInvalidValue;
    switch (k) {
    case 1: e = pcg::launch_mixed<1>(p, m, blocks, s); break;
    case 2: e = pcg::launch_mixed<2>(p, m, blocks, s); break;
    case 3: e = pcg::launch_mixed<3>(p, m, blocks, s); break;
    case 4: e = pcg::launch_mixed<4>(p, m, blocks, s); break;
    }
    HDFE_CUDA_TRY(e);
    pcg::pcg_status_kernel<<<1, 32, 0, s>>>(p.bar, info);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(3);
    return HDFE_OK;
}
