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

constexpr int kThreads = 1024;    // one CTA per SM: fewer arrivals at each grid barrier
constexpr int kWarps = kThreads / 32;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kLong = 64;           // nonzeros in a warp's range that make a row "long"

// P's row stride: even, so a row's pairs of values are 16-byte aligned
template <int K>
struct Stride {
    static constexpr int P = K == 1 ? 1 : ((K + 1) / 2) * 2;
};

struct Params {
    const int64_t *indptr;
    const int32_t *indices;
    const double *data;
    int64_t L, nnz, chunk;
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
    int64_t r, p, ap, carry, part, wfirst, cut, bar, total;
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
    o.carry = take(blocks * kWarps * 2 * k * 8);
    o.part = take(4 * (int64_t)k * blocks * 8);
    o.wfirst = take(blocks * kWarps * 8);
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

// Row c of V (stride VS) into g[0..K), with vector loads of VW elements
// (2 doubles, or 2 or 4 floats: 8- or 16-byte aligned rows) or scalars.
// Plain loads: V may be written by this kernel between grid barriers.
template <int K, int VS, int VW, typename T>
__device__ __forceinline__ void gather(const T *V, int64_t c, T (&g)[K])
{
    const T *p = V + c * VS;
    if constexpr (VW == 4) {
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
    constexpr int U = K <= 4 ? 4 : 2;
    for (; e0 < re; e0 += STEP * U) {
        int64_t c[U];
        T d[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t e = e0 + STEP * u;
            c[u] = 0;
            d[u] = T(0);
            if (e < re) {
                c[u] = __ldg(a.indices + e);
                d[u] = __ldg(vals + e);
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

template <int K, int VS, typename T>
__device__ __forceinline__ void finish_row(int64_t row, const T (&acc)[K], int64_t row_st,
                                           int64_t row_en, int64_t lo, int64_t hi, int64_t gw,
                                           const T *V, T *out, T *carry, double (&dot)[K],
                                           bool want_dot)
{
    if (want_dot) {
#pragma unroll
        for (int k = 0; k < K; k++) dot[k] += (double)V[row * VS + k] * (double)acc[k];
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
// (in FP64 whatever T is).  vals are S's values in T.
template <int K, int VS, int VW, typename T>
__device__ void spmm_range(const Params &a, const T *__restrict__ vals, const T *__restrict__ V,
                           T *__restrict__ out, T *carry, double (&dot)[K], bool want_dot)
{
    const int lane = threadIdx.x & 31, sub = lane >> 3, sl = lane & 7;
    const int64_t gw = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
    const int64_t lo = gw * a.chunk;
    const int64_t hi = min(lo + a.chunk, a.nnz);
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
                T acc[K];
#pragma unroll
                for (int k = 0; k < K; k++) acc[k] = T(0);
                row_products<K, VS, VW, 32, T>(a, vals, V, rs + lane, re, acc);
#pragma unroll
                for (int k = 0; k < K; k++) acc[k] = warp_sum(acc[k]);
                const int64_t row_st = __shfl_sync(kFull, st, j), row_en = __shfl_sync(kFull, en, j);
                if (lane == 0)
                    finish_row<K, VS, T>(r0 + j, acc, row_st, row_en, lo, hi, gw, V, out, carry,
                                         dot, want_dot);
                j++;
            } else {
                // up to four short rows, one per 8-lane subgroup, up to the next long row
                const unsigned ahead = longmask & (0xffffffffu << j);
                int batch = ahead ? (__ffs(ahead) - 1 - j) : 4;
                batch = min(min(batch, 4), nrows - j);
                const int src = min(j + sub, 31);
                const bool mine = sub < batch;
                const int64_t rs = __shfl_sync(kFull, cs, src), re = __shfl_sync(kFull, ce, src);
                const int64_t row_st = __shfl_sync(kFull, st, src);
                const int64_t row_en = __shfl_sync(kFull, en, src);
                T acc[K];
#pragma unroll
                for (int k = 0; k < K; k++) acc[k] = T(0);
                if (mine) row_products<K, VS, VW, 8, T>(a, vals, V, rs + sl, re, acc);
#pragma unroll
                for (int k = 0; k < K; k++) {
                    acc[k] += __shfl_xor_sync(kFull, acc[k], 4);
                    acc[k] += __shfl_xor_sync(kFull, acc[k], 2);
                    acc[k] += __shfl_xor_sync(kFull, acc[k], 1);
                }
                if (mine && sl == 0 && re > rs)
                    finish_row<K, VS, T>(r0 + j + sub, acc, row_st, row_en, lo, hi, gw, V, out,
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
    const int64_t gw = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
    const int64_t lo = gw * a.chunk;
    const int64_t hi = min(lo + a.chunk, a.nnz);
    if (lo >= hi) return false;
    const int64_t r = a.wfirst[gw];
    const int64_t rs = a.indptr[r], re = a.indptr[r + 1];
    if (!(rs < lo && re <= hi)) return false;
    const int64_t w0 = rs / a.chunk;
    T s[K];
#pragma unroll
    for (int k = 0; k < K; k++) s[k] = T(0);
    for (int64_t w = w0 + lane; w <= gw; w += 32) {
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
        for (int w = 0; w < kWarps; w++) t += scratch[w * N + threadIdx.x];
        part[(int64_t)(q0 + threadIdx.x) * nb + blockIdx.x] = t;
    }
    __syncthreads();
}

template <int K>
__global__ void __launch_bounds__(kThreads, 1) pcg_kernel(Params a)
{
    constexpr int KP = Stride<K>::P;
    __shared__ double s_red[4 * K];
    __shared__ double s_scratch[kWarps * 3 * K];
    GridBarrier gb{a.bar};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t gtid = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    const int64_t gstride = (int64_t)gridDim.x * kThreads;
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
        const int64_t gw = (int64_t)blockIdx.x * kWarps + warp;
        const int64_t lo = gw * a.chunk;
        if (lane == 0 && lo < a.nnz) a.wfirst[gw] = upper_bound(a.indptr, L + 1, lo) - 1;
        __syncwarp();
        for (int64_t r = gtid; r < L; r += gstride) {
            const int64_t rs = a.indptr[r], re = a.indptr[r + 1];
            a.cut[r] = (re > rs && (rs / a.chunk) != ((re - 1) / a.chunk)) ? 1 : 0;
        }
    }
    // ---- R = B - S X0 (or B), the zero columns, ||B||, rz
    double dot[K];
#pragma unroll
    for (int k = 0; k < K; k++) dot[k] = 0.0;
    if (a.X0 != nullptr) {
        spmm_range<K, K, 1, double>(a, a.data, a.X0, a.AP, a.carry, dot, false);
        if (!gb.sync()) return;
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
            if (a.X0 != nullptr && a.cut[r]) continue;
            const bool empty = a.indptr[r + 1] == a.indptr[r];
#pragma unroll
            for (int k = 0; k < K; k++) ap[k] = (a.X0 != nullptr && !empty) ? a.AP[r * K + k] : 0.0;
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
            spmm_range<K, KP, (KP % 2 == 0) ? 2 : 1, double>(a, a.data, a.P, a.AP, a.carry, dot, true);
            block_partials<K>(dot, s_scratch, a.part, 0, nb);
            if (!gb.sync()) return;
            if (warp == 0) {
                for (int k = 0; k < K; k++) {
                    double t = reduce_part(a.part, k);
                    if (lane == 0) s_red[k] = t;
                }
            }
            __syncthreads();
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
            for (int64_t r = gtid; r < L; r += gstride) {
                if (a.cut[r]) continue;
                double ap[K];
                const bool empty = a.indptr[r + 1] == a.indptr[r];
#pragma unroll
                for (int k = 0; k < K; k++) ap[k] = empty ? 0.0 : a.AP[r * K + k];
                step_row(r, ap);
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
            for (int64_t r = gtid; r < L; r += gstride) {
                const double di = a.dinv[r];
#pragma unroll
                for (int k = 0; k < K; k++)
                    a.P[r * KP + k] = a.R[r * K + k] * di + beta[k] * a.P[r * KP + k];
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
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel<K>, kThreads, 0) !=
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
    static int cache[64][HDFE_PCG_MAX_K + 1] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return grid_blocks_for_uncached(k);
    if (cache[dev][k] == 0) cache[dev][k] = grid_blocks_for_uncached(k);
    return cache[dev][k];
}

template <int K>
cudaError_t launch(Params p, int blocks, cudaStream_t s)
{
    void *args[] = {&p};
    return cudaLaunchCooperativeKernel((const void *)pcg_kernel<K>, dim3(blocks), dim3(kThreads),
                                       args, 0, s);
}

}  // namespace pcg
}  // namespace hdfe

using namespace hdfe;

extern "C" int64_t hdfe_pcg_workspace_bytes(int64_t L, int64_t nnz, int32_t k)
{
    (void)nnz;
    if (k < 1 || k > HDFE_PCG_MAX_K || L < 0) return -1;
    int blocks = pcg::grid_blocks_for(k);
    if (blocks < 1) return -1;
    return pcg::layout(L, k, blocks).total;
}

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
    int blocks = pcg::grid_blocks_for(k);
    if (blocks < 1) return hdfe_set_cuda_error(cudaGetLastError());
    pcg::Layout lay = pcg::layout(L, k, blocks);
    if (workspace_bytes < lay.total)
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_pcg_solve: workspace too small");
    char *ws = (char *)workspace;
    pcg::Params p;
    p.indptr = indptr;
    p.indices = indices;
    p.data = data;
    p.L = L;
    p.nnz = nnz;
    const int64_t warps = (int64_t)blocks * pcg::kWarps;
    p.chunk = nnz > 0 ? (nnz + warps - 1) / warps : 1;
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
    p.cut = (uint8_t *)(ws + lay.cut);
    p.bar = (unsigned *)(ws + lay.bar);
    p.info = info;
    HDFE_CUDA_TRY(cudaMemsetAsync(p.bar, 0, 16, s));
    cudaError_t e = cudaErrorInvalidValue;
    switch (k) {
    case 1: e = pcg::launch<1>(p, blocks, s); break;
    case 2: e = pcg::launch<2>(p, blocks, s); break;
    case 3: e = pcg::launch<3>(p, blocks, s); break;
    case 4: e = pcg::launch<4>(p, blocks, s); break;
    case 5: e = pcg::launch<5>(p, blocks, s); break;
    case 6: e = pcg::launch<6>(p, blocks, s); break;
    case 7: e = pcg::launch<7>(p, blocks, s); break;
    case 8: e = pcg::launch<8>(p, blocks, s); break;
    }
    HDFE_CUDA_TRY(e);
    pcg::pcg_status_kernel<<<1, 32, 0, s>>>(p.bar, info);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(2);
    return HDFE_OK;
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
    int64_t r, p, ap, d, ax, carry, part, wfirst, cut, bar, total;
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
    o.carry = take(blocks * kWarps * 2 * k * 8);
    o.part = take(4 * (int64_t)k * blocks * 8);
    o.wfirst = take(blocks * kWarps * 8);
    o.cut = take(L);
    o.bar = take(64);
    o.total = p;
    return o;
}

template <int K>
__global__ void __launch_bounds__(kThreads, 1) mixed_kernel(Params a, Mixed f)
{
    constexpr int KF = FStride<K>::P;
    constexpr int VWF = FStride<K>::VW;
    __shared__ double s_red[4 * K];
    __shared__ double s_scratch[kWarps * 3 * K];
    GridBarrier gb{a.bar};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t gtid = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    const int64_t gstride = (int64_t)gridDim.x * kThreads;
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
        const int64_t gw = (int64_t)blockIdx.x * kWarps + warp;
        const int64_t lo = gw * a.chunk;
        if (lane == 0 && lo < a.nnz) a.wfirst[gw] = upper_bound(a.indptr, L + 1, lo) - 1;
        __syncwarp();
        double sb[K];
#pragma unroll
        for (int k = 0; k < K; k++) sb[k] = 0.0;
        for (int64_t r = gtid; r < L; r += gstride) {
            const int64_t rs = a.indptr[r], re = a.indptr[r + 1];
            a.cut[r] = (re > rs && (rs / a.chunk) != ((re - 1) / a.chunk)) ? 1 : 0;
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

template <int K>
int mixed_grid()
{
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mixed_kernel<K>, kThreads, 0) !=
        cudaSuccess)
        return -1;
    return per_sm < 1 ? -1 : sms;
}

int mixed_grid_for(int k)
{
    static int cache[64][HDFE_PCG_MAX_K + 1] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -1;
    if (cache[dev][k] == 0) {
        switch (k) {
        case 1: cache[dev][k] = mixed_grid<1>(); break;
        case 2: cache[dev][k] = mixed_grid<2>(); break;
        case 3: cache[dev][k] = mixed_grid<3>(); break;
        case 4: cache[dev][k] = mixed_grid<4>(); break;
        case 5: cache[dev][k] = mixed_grid<5>(); break;
        case 6: cache[dev][k] = mixed_grid<6>(); break;
        case 7: cache[dev][k] = mixed_grid<7>(); break;
        case 8: cache[dev][k] = mixed_grid<8>(); break;
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
                                       dim3(kThreads), args, 0, s);
}

}  // namespace pcg
}  // namespace hdfe

extern "C" int64_t hdfe_pcg_mixed_workspace_bytes(int64_t L, int64_t nnz, int32_t k)
{
    (void)nnz;
    if (k < 1 || k > HDFE_PCG_MAX_K || L < 0) return -1;
    const int blocks = pcg::mixed_grid_for(k);
    if (blocks < 1) return -1;
    return pcg::mixed_layout(L, k, blocks).total;
}

extern "C" int hdfe_pcg_solve_mixed(const int64_t *indptr, const int32_t *indices,
                                    const double *data, const float *data32, int64_t L,
                                    int64_t nnz, const double *dinv, const double *B, int32_t k,
                                    const uint8_t *zero, const double *X0, double tol,
                                    double inner_tol, int64_t maxiter, double *X,
                                    void *workspace, int64_t workspace_bytes,
                                    hdfe_pcg_info *info, void *stream)
{
    if (k < 1 || k > HDFE_PCG_MAX_K || L < 1 || nnz < 0 || !indptr || !dinv || !B || !X ||
        !info || !workspace || maxiter < 0 || !(inner_tol > 0.0 && inner_tol < 1.0) ||
        (nnz > 0 && (!indices || !data || !data32)))
        return hdfe_set_arg_error("hdfe_pcg_solve_mixed: bad argument");
    if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
        return hdfe_set_arg_error("hdfe_pcg_solve_mixed: workspace must be 256-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
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
    const int64_t warps = (int64_t)blocks * pcg::kWarps;
    p.chunk = nnz > 0 ? (nnz + warps - 1) / warps : 1;
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
    cudaError_t e = cudaErrorInvalidValue;
    switch (k) {
    case 1: e = pcg::launch_mixed<1>(p, m, blocks, s); break;
    case 2: e = pcg::launch_mixed<2>(p, m, blocks, s); break;
    case 3: e = pcg::launch_mixed<3>(p, m, blocks, s); break;
    case 4: e = pcg::launch_mixed<4>(p, m, blocks, s); break;
    case 5: e = pcg::launch_mixed<5>(p, m, blocks, s); break;
    case 6: e = pcg::launch_mixed<6>(p, m, blocks, s); break;
    case 7: e = pcg::launch_mixed<7>(p, m, blocks, s); break;
    case 8: e = pcg::launch_mixed<8>(p, m, blocks, s); break;
    }
    HDFE_CUDA_TRY(e);
    pcg::pcg_status_kernel<<<1, 32, 0, s>>>(p.bar, info);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(2);
    return HDFE_OK;
}
