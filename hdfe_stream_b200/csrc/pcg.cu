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
//      and rows of 10 (firm levels) cost the same per nonzero.  A warp walks
//      its range 32 nonzeros at a time with coalesced index/value loads,
//      finds each lane's row by a shuffle binary search over the row ends,
//      and reduces by row with a segmented shuffle scan.  Rows inside the
//      warp's range are written to AP; a row cut by a range boundary leaves a
//      partial sum in the warp's two carry slots.  p'Ap accumulates per warp
//      (linear in the partials, so cut rows need no fix-up for it).
//   B  alpha from the reduced p'Ap.  Per row: X += alpha P, R -= alpha AP and
//      the partial sums of R^2 and R^2 dinv.  A row cut across warps is
//      finished by the warp holding its last nonzero, which sums the carry
//      slots of the warps it spans in a fixed order.
//   C  rel, active and beta from the reduced sums; P = dinv R + beta P.
//
// Determinism: the grid size, the warp ranges and every reduction order are
// fixed for a given GPU and build, so repeated solves give identical bits.
#include <cstdio>
#include <cuda_runtime.h>

#include "common.cuh"

namespace hdfe {
namespace pcg {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr unsigned kFull = 0xffffffffu;

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
    unsigned *bar;
    hdfe_pcg_info *info;
};

// Workspace layout, in doubles: R, P, AP (L*K each), carry (warps*2*K),
// part (4*K*blocks), then the barrier words.
struct Layout {
    int64_t r, p, ap, carry, part, bar_bytes_off, total_bytes;
};

__host__ __device__ inline Layout layout(int64_t L, int k, int64_t blocks)
{
    Layout o;
    int64_t lk = L * k;
    o.r = 0;
    o.p = lk;
    o.ap = 2 * lk;
    o.carry = 3 * lk;
    o.part = o.carry + blocks * kWarps * 2 * k;
    int64_t doubles = o.part + 4 * (int64_t)k * blocks;
    o.bar_bytes_off = ((doubles * 8 + 255) / 256) * 256;
    o.total_bytes = o.bar_bytes_off + 256;
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

// AP-type product of the nonzeros in this warp's range: out = S * V for
// rows inside the range, partial sums of cut rows to the carry slots, and
// dot[k] += V[r] . (S V)[r] over the range when want_dot.
template <int K>
__device__ void spmm_range(const Params &a, const double *__restrict__ V, double *__restrict__ out,
                           double (&dot)[K], bool want_dot)
{
    const int lane = threadIdx.x & 31;
    const int64_t gw = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
    const int64_t lo = gw * a.chunk;
    const int64_t hi = min(lo + a.chunk, a.nnz);
    if (lo >= hi) return;
    const int64_t *__restrict__ indptr = a.indptr;
    int64_t r_cur = upper_bound(indptr, a.L + 1, lo) - 1;    // row of nonzero `lo`
    int64_t rcur_start = __ldg(indptr + r_cur);              // its first nonzero
    int64_t row_open = -1;                                   // row continued from the last chunk
    double carry[K];
#pragma unroll
    for (int k = 0; k < K; k++) carry[k] = 0.0;
    // the next chunk's indices and values are loaded one chunk ahead
    int64_t c_nx = 0;
    double d_nx = 0.0;
    if (lo + lane < hi) {
        c_nx = __ldg(a.indices + lo + lane);
        d_nx = __ldg(a.data + lo + lane);
    }
    for (int64_t base = lo; base < hi; base += 32) {
        const int64_t e = base + lane;
        const bool valid = e < hi;
        int64_t c = c_nx;
        const double d = d_nx;
        double g[K];
        if (valid) {
            if (c < 0 || c >= a.L) {            // not a CSR of this size: record, skip
                GridBarrier{a.bar}.fail(HDFE_ERR_BAD_CODE);
                c = 0;
            }
#pragma unroll
            for (int k = 0; k < K; k++) g[k] = V[c * K + k];
        }
        if (e + 32 < hi) {
            c_nx = __ldg(a.indices + e + 32);
            d_nx = __ldg(a.data + e + 32);
        }
        // the row of nonzero e, as an offset from r_cur: #(row ends <= e),
        // row ends taken relative to `base` in windows of 32 rows
        int rr = -1;
        int64_t Eq_last = 0;
        int nwin = 0;
        for (int64_t ws = r_cur;; ws += 32) {
            const int64_t q = ws + 1 + lane;
            const int64_t Eq = q <= a.L ? __ldg(indptr + q) : INT64_MAX;
            Eq_last = Eq;
            nwin++;
            const int Er = (int)min(Eq - base, (int64_t)INT32_MAX);
            int pos = 0;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1) {
                const int v = __shfl_sync(kFull, Er, pos + step - 1);
                if (v <= lane) pos += step;
            }
            if (__shfl_sync(kFull, Er, 31) <= lane) pos = 32;
            if (rr < 0 && pos < 32) rr = (int)(ws - r_cur) + pos;
            if (!__any_sync(kFull, valid && rr < 0)) break;
        }
        double v[K];
        if (valid) {
#pragma unroll
            for (int k = 0; k < K; k++) v[k] = d * g[k];
        } else {
            rr = INT32_MAX;
#pragma unroll
            for (int k = 0; k < K; k++) v[k] = 0.0;
        }
        // segmented inclusive scan over lanes of equal row
#pragma unroll
        for (int s = 1; s < 32; s <<= 1) {
            const int ro = __shfl_up_sync(kFull, rr, s);
#pragma unroll
            for (int k = 0; k < K; k++) {
                const double o = __shfl_up_sync(kFull, v[k], s);
                if (lane >= s && ro == rr) v[k] += o;
            }
        }
        const int rnext = __shfl_down_sync(kFull, rr, 1);
        const bool tail = valid && (lane == 31 || rnext != rr);
        const int64_t row = r_cur + rr;
        // with one window (the usual case) lane q holds the end of row r_cur + q,
        // so a row's bounds come from shuffles instead of loads
        const bool single = nwin == 1;
        const int64_t re_w = __shfl_sync(kFull, Eq_last, min(max(rr, 0), 31));
        int64_t rs_w = __shfl_sync(kFull, Eq_last, min(max(rr - 1, 0), 31));
        if (rr == 0) rs_w = rcur_start;
        if (tail && row == row_open) {
#pragma unroll
            for (int k = 0; k < K; k++) v[k] += carry[k];
        }
        // the last lane's row and sum carry into the next chunk when it goes on
        const int r31 = __shfl_sync(kFull, rr, 31);
        bool goes_on = false;
        if (tail) {
            const int64_t rs = single ? rs_w : __ldg(indptr + row);
            const int64_t re = single ? re_w : __ldg(indptr + row + 1);
            const bool ends_here = re == e + 1;
            goes_on = !ends_here && e + 1 < hi;                 // into the next chunk
            if (!goes_on) {
                if (want_dot) {
#pragma unroll
                    for (int k = 0; k < K; k++) dot[k] += V[row * K + k] * v[k];
                }
                if (ends_here && rs >= lo) {
#pragma unroll
                    for (int k = 0; k < K; k++) out[row * K + k] = v[k];
                } else {
                    // cut row: slot 1 in the warp where it starts, 0 elsewhere
                    const int slot = rs >= lo ? 1 : 0;
                    double *cs = a.carry + (gw * 2 + slot) * K;
#pragma unroll
                    for (int k = 0; k < K; k++) cs[k] = v[k];
                }
            }
        }
        if (__shfl_sync(kFull, (int)goes_on, 31)) {
            row_open = r_cur + r31;
#pragma unroll
            for (int k = 0; k < K; k++) carry[k] = __shfl_sync(kFull, v[k], 31);
        } else {
            row_open = -1;
        }
        if (r31 != INT32_MAX) {
            const int64_t next_start = __shfl_sync(kFull, Eq_last, min(max(r31 - 1, 0), 31));
            if (r31 > 0) rcur_start = single ? next_start : __ldg(indptr + r_cur + r31);
            r_cur += r31;
        }
    }
}

// AP[r] for a row whose nonzeros span several warps: summed from their carry
// slots in a fixed order by the warp holding the row's last nonzero.  Returns
// true (in all lanes) when this warp finishes such a row, with its AP in ap[].
template <int K>
__device__ bool finish_cut_row(const Params &a, int64_t &row, double (&ap)[K])
{
    const int lane = threadIdx.x & 31;
    const int64_t gw = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
    const int64_t lo = gw * a.chunk;
    const int64_t hi = min(lo + a.chunk, a.nnz);
    if (lo >= hi) return false;
    const int64_t r = upper_bound(a.indptr, a.L + 1, lo) - 1;
    const int64_t rs = a.indptr[r], re = a.indptr[r + 1];
    if (!(rs < lo && re <= hi)) return false;
    const int64_t w0 = rs / a.chunk;
    double s[K];
#pragma unroll
    for (int k = 0; k < K; k++) s[k] = 0.0;
    for (int64_t w = w0 + lane; w <= gw; w += 32) {
        const double *cs = a.carry + (w * 2 + (w == w0 ? 1 : 0)) * K;
#pragma unroll
        for (int k = 0; k < K; k++) s[k] += __ldcg(cs + k);
    }
#pragma unroll
    for (int k = 0; k < K; k++) ap[k] = warp_sum(s[k]);
    row = r;
    return true;
}

__device__ __forceinline__ bool row_is_cut(const int64_t *indptr, int64_t r, int64_t chunk)
{
    const int64_t rs = indptr[r], re = indptr[r + 1];
    return re > rs && (rs / chunk) != ((re - 1) / chunk);
}

template <int K>
__global__ void __launch_bounds__(kThreads, 4) pcg_kernel(Params a)
{
    __shared__ double s_red[4 * K];
    __shared__ double s_scratch[kWarps];
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

    // ---- set-up: R = B - S X0 (or B), the zero columns, ||B||, rz
    double dot[K];
#pragma unroll
    for (int k = 0; k < K; k++) dot[k] = 0.0;
    if (a.X0 != nullptr) {
        spmm_range<K>(a, a.X0, a.AP, dot, false);
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
                a.P[r * K + k] = res * di;
                sb[k] += b * b;
                sr[k] += res * res;
                sz[k] += res * res * di;
            }
        };
        for (int64_t r = gtid; r < L; r += gstride) {
            double ap[K];
            const bool cut = a.X0 != nullptr && row_is_cut(a.indptr, r, a.chunk);
            if (cut) continue;
            const bool empty = a.indptr[r + 1] == a.indptr[r];
#pragma unroll
            for (int k = 0; k < K; k++) ap[k] = (a.X0 != nullptr && !empty) ? a.AP[r * K + k] : 0.0;
            setup_row(r, ap);
        }
        if (a.X0 != nullptr) {
            int64_t r;
            double ap[K];
            if (finish_cut_row<K>(a, r, ap) && lane == 0) setup_row(r, ap);
        }
#pragma unroll
        for (int k = 0; k < K; k++) {
            double t0 = block_sum(sb[k], s_scratch);
            double t1 = block_sum(sr[k], s_scratch);
            double t2 = block_sum(sz[k], s_scratch);
            if (threadIdx.x == 0) {
                a.part[(int64_t)(0 * K + k) * nb + blockIdx.x] = t0;
                a.part[(int64_t)(1 * K + k) * nb + blockIdx.x] = t1;
                a.part[(int64_t)(2 * K + k) * nb + blockIdx.x] = t2;
            }
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
        if (!gb.sync()) return;     // P complete before the first SpMM
        for (it = 1; it <= a.maxiter; it++) {
            // ---- A: AP = S P, p'Ap
#pragma unroll
            for (int k = 0; k < K; k++) dot[k] = 0.0;
            spmm_range<K>(a, a.P, a.AP, dot, true);
#pragma unroll
            for (int k = 0; k < K; k++) {
                double t = block_sum(dot[k], s_scratch);
                if (threadIdx.x == 0) a.part[(int64_t)k * nb + blockIdx.x] = t;
            }
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
                    const double p = a.P[r * K + k];
                    a.X[r * K + k] += alpha[k] * p;
                    const double res = a.R[r * K + k] - alpha[k] * ap[k];
                    a.R[r * K + k] = res;
                    sr[k] += res * res;
                    sz[k] += res * res * di;
                }
            };
            for (int64_t r = gtid; r < L; r += gstride) {
                if (row_is_cut(a.indptr, r, a.chunk)) continue;
                double ap[K];
                const bool empty = a.indptr[r + 1] == a.indptr[r];
#pragma unroll
                for (int k = 0; k < K; k++) ap[k] = empty ? 0.0 : a.AP[r * K + k];
                step_row(r, ap);
            }
            {
                int64_t r;
                double ap[K];
                if (finish_cut_row<K>(a, r, ap) && lane == 0) step_row(r, ap);
            }
#pragma unroll
            for (int k = 0; k < K; k++) {
                double t1 = block_sum(sr[k], s_scratch);
                double t2 = block_sum(sz[k], s_scratch);
                if (threadIdx.x == 0) {
                    a.part[(int64_t)(1 * K + k) * nb + blockIdx.x] = t1;
                    a.part[(int64_t)(2 * K + k) * nb + blockIdx.x] = t2;
                }
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
                    a.P[r * K + k] = a.R[r * K + k] * di + beta[k] * a.P[r * K + k];
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

// Writes the barrier's error code (if any) into info->status after the
// persistent kernel, so a caller reading info sees a timed-out solve.
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
    return sms * (per_sm < 4 ? per_sm : 4);
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
    return pcg::layout(L, k, blocks).total_bytes;
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
    cudaStream_t s = (cudaStream_t)stream;
    int blocks = pcg::grid_blocks_for(k);
    if (blocks < 1) return hdfe_set_cuda_error(cudaGetLastError());
    pcg::Layout lay = pcg::layout(L, k, blocks);
    if (workspace_bytes < lay.total_bytes)
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_pcg_solve: workspace too small");
    double *ws = (double *)workspace;
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
    p.R = ws + lay.r;
    p.P = ws + lay.p;
    p.AP = ws + lay.ap;
    p.carry = ws + lay.carry;
    p.part = ws + lay.part;
    p.bar = (unsigned *)((char *)workspace + lay.bar_bytes_off);
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
