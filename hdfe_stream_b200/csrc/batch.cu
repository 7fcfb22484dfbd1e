// Many independent fixed-effects systems in one persistent launch.
//
// The systems' reduced matrices sit on the diagonal of one CSR matrix, each
// system's levels a contiguous range of rows.  Every warp of the cooperative
// grid owns a contiguous range of rows inside ONE system (the host splits the
// systems' rows over the warps by cost, at least one warp per system), so the
// Jacobi block PCG of core/solve.py:66-140 runs per system with its own
// scalars: per (system, column) alpha, beta, the active flag and the relative
// residual, exactly the algorithm of the single-system kernel (pcg.cu).  The
// dot products are summed per warp, then per CTA and system (a CTA's warps
// cover at most kWarps systems) into a global slot; after a grid barrier one
// warp per (CTA, system) sums that system's CTA slots (lanes over the CTAs,
// then a warp sum) and shares the totals through shared memory.  The order is
// fixed, so every warp of a system holds the same scalars and the result does
// not depend on scheduling; each phase has its own slots, so a phase's
// writes never meet the previous phase's reads.  The loop ends when no system has an active
// column: a flag per iteration parity, set by the warps whose system is still
// active and cleared two phases before its next use.
//
// The SpMV gives each row LPR lanes (4, 8, 16 or 32: the caller's tuner picks
// it for the batch), LPR nonzeros in flight per row, reduced by shuffles.
// Long rows (the small dimensions' levels, whose rows hold a nonzero per
// level they meet) are cut by the host into chunks that any warps of the
// system take, a whole warp per chunk: each chunk's partial sums go to its
// own slot and its share of p'Ap is taken there, and the row's owner adds
// the slots in chunk order when it needs the row of AP, so no row holds one
// warp for long and the sums keep a fixed order.
#include <climits>
#include <cuda_runtime.h>

#include "common.cuh"

namespace hdfe {
namespace batch {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxK = 8;

// P's row stride: 3 columns padded to 4, so that a row is one aligned
// 32-byte load (a random gather costs the L1 a wavefront per load instruction)
__host__ __device__ constexpr int p_stride(int k) { return k == 3 ? 4 : k; }

// Row c of P (stride PS) into g[0..K)
template <int K, int PS>
__device__ __forceinline__ void gather_p(const double *P, int64_t c, double (&g)[K])
{
    const double *p = P + c * PS;
    if constexpr (PS == 4) {
        double t0, t1, t2, t3;
        asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];"
                     : "=d"(t0), "=d"(t1), "=d"(t2), "=d"(t3) : "l"(p));
        g[0] = t0;
        if constexpr (K > 1) g[1] = t1;
        if constexpr (K > 2) g[2] = t2;
        if constexpr (K > 3) g[3] = t3;
    } else {
#pragma unroll
        for (int k = 0; k < K; k++) g[k] = p[k];
    }
}

struct Args {
    const int64_t *indptr;
    const int32_t *indices;
    const double *data;
    int64_t L;
    const double *dinv;
    const double *B;            // (L, K)
    const uint8_t *zero;        // (systems, K) or null
    double tol;
    int64_t maxiter;
    double *X, *R, *P, *AP;     // (L, K)
    const int64_t *wrow;        // (warps + 1) first row of each warp
    const int32_t *wsys;        // (warps) system of each warp
    const int32_t *swarp;       // (systems + 1) first warp of each system
    const int32_t *wchunk;      // (warps + 1) first chunk of each warp
    const int32_t *chunk_row;   // (chunks) row of each chunk
    const int64_t *chunk_lo;    // (chunks) first nonzero of each chunk
    const int64_t *chunk_hi;    // (chunks) one past its last
    const int32_t *row_chunk;   // (L) a long row's first chunk, -1 for the others
    double *cp;                 // (chunks, K) chunk partial sums
    double *cpart;              // (blocks, kWarps, 5 K): per CTA and local system
    unsigned *flag;             // [2]
    unsigned *bar;
    int64_t *iterations;        // (systems)
    double *max_rel;            // (systems)
    int32_t *converged;         // (systems)
    int64_t nwarps;
};

// Totals over each warp's system of N per-warp values v (already summed over
// the warp, the same in every lane), through slots [q0, q0 + N) of cpart;
// S the slots per entry.  One grid barrier.  Returns false when the kernel
// must stop.
template <int N, int S>
__device__ __forceinline__ bool system_totals(const Args &a, const GridBarrier &gb, double (&v)[N],
                                              int q0, double *s_w, double *s_sys, int first,
                                              int nsys, int local)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < N; q++) s_w[warp * N + q] = v[q];
    }
    __syncthreads();
    if (warp < nsys) {
        for (int q = lane; q < N; q += 32) {
            double t = 0.0;
            for (int w = 0; w < kWarps; w++)
                if (a.wsys[blockIdx.x * kWarps + w] == first + warp) t += s_w[w * N + q];
            a.cpart[((int64_t)blockIdx.x * kWarps + warp) * S + q0 + q] = t;
        }
    }
    if (!gb.sync()) return false;
    if (warp < nsys) {
        const int sys = first + warp;
        const int bf = a.swarp[sys] / kWarps, bl = (a.swarp[sys + 1] - 1) / kWarps;
#pragma unroll
        for (int q = 0; q < N; q++) {
            double t = 0.0;
            for (int b = bf + lane; b <= bl; b += 32) {
                const int j = sys - a.wsys[b * kWarps];
                t += a.cpart[((int64_t)b * kWarps + j) * S + q0 + q];
            }
            t = warp_sum(t);
            if (lane == 0) s_sys[warp * N + q] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < N; q++) v[q] = s_sys[local * N + q];
    __syncthreads();
    return true;
}

template <int K, int LPR>
__global__ void __launch_bounds__(kThreads) k_batch_pcg(Args a)
{
    __shared__ double s_w[kWarps * 2 * K], s_sys[kWarps * 2 * K];
    GridBarrier gb{a.bar};
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
    const int64_t r0 = a.wrow[gw], r1 = a.wrow[gw + 1];
    const int sys = a.wsys[gw];
    const int w0 = a.swarp[sys];
    const int first = a.wsys[blockIdx.x * kWarps];
    const int nsys = a.wsys[blockIdx.x * kWarps + kWarps - 1] - first + 1;
    const int local = sys - first;
    constexpr int S5 = 5 * K;       // slots: set-up 2K, phase A K, phase B 2K
    constexpr int PS = p_stride(K);

    bool zero[K], active[K];
    double bnorm[K], rz[K], rel[K];
    // ---- set-up: R = B, P = dinv R, ||B||^2, R'dinv R
    double sb[K], sz[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
        zero[k] = a.zero != nullptr && a.zero[sys * K + k] != 0;
        sb[k] = sz[k] = 0.0;
        rel[k] = 0.0;
    }
    for (int64_t r = r0 + lane; r < r1; r += 32) {
        const double di = a.dinv[r];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const double b = a.B[r * K + k];
            const double res = zero[k] ? 0.0 : b;
            a.X[r * K + k] = 0.0;
            a.R[r * K + k] = res;
            a.P[r * PS + k] = res * di;
            sb[k] += b * b;
            sz[k] += res * res * di;
        }
    }
    {
        double v[2 * K];
#pragma unroll
        for (int k = 0; k < K; k++) { v[k] = warp_sum(sb[k]); v[K + k] = warp_sum(sz[k]); }
        if (blockIdx.x == 0 && threadIdx.x == 0) { a.flag[0] = 0; a.flag[1] = 0; }
        if (!system_totals<2 * K, S5>(a, gb, v, 0, s_w, s_sys, first, nsys, local)) return;
#pragma unroll
        for (int k = 0; k < K; k++) { sb[k] = v[k]; sz[k] = v[K + k]; }
    }
    bool any = false;
#pragma unroll
    for (int k = 0; k < K; k++) {
        const double bn = sqrt(sb[k]);
        bnorm[k] = bn == 0.0 ? 1.0 : bn;
        rz[k] = sz[k];
        active[k] = !zero[k];
        any |= active[k];
    }
    int64_t done_at = any ? -1 : 0;
    int64_t it;
    for (it = 1; it <= a.maxiter; it++) {
        // ---- A: AP = S P for the warp's rows, p'Ap
        double dot[K];
#pragma unroll
        for (int k = 0; k < K; k++) dot[k] = 0.0;
        {
            constexpr int RPW = 32 / LPR;           // rows per warp step
            const int sub = lane / LPR, sl = lane % LPR;
            for (int64_t base = r0; base < r1; base += RPW) {
                const int64_t r = base + sub;
                double acc[K];
#pragma unroll
                for (int k = 0; k < K; k++) acc[k] = 0.0;
                if (r < r1 && a.row_chunk[r] < 0) {
                    const int64_t e = a.indptr[r + 1];
                    for (int64_t j = a.indptr[r] + sl; j < e; j += LPR) {
                        const int32_t c = a.indices[j];
                        const double v = a.data[j];
                        if (c < 0 || c >= a.L) { gb.fail(HDFE_ERR_BAD_CODE); continue; }
                        double g[K];
                        gather_p<K, PS>(a.P, c, g);
#pragma unroll
                        for (int k = 0; k < K; k++) acc[k] += v * g[k];
                    }
                }
#pragma unroll
                for (int k = 0; k < K; k++)
#pragma unroll
                    for (int o = LPR / 2; o > 0; o >>= 1)
                        acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
                if (sl == 0 && r < r1 && a.row_chunk[r] < 0) {
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        a.AP[r * K + k] = acc[k];
                        dot[k] += acc[k] * a.P[r * PS + k];
                    }
                }
            }
            // the warp's chunks of long rows: partial sums and their p'Ap
            const int c1 = a.wchunk[gw + 1];
            for (int c = a.wchunk[gw]; c < c1; c++) {
                const int64_t r = a.chunk_row[c];
                const int64_t e = a.chunk_hi[c];
                double acc[K];
#pragma unroll
                for (int k = 0; k < K; k++) acc[k] = 0.0;
                for (int64_t j = a.chunk_lo[c] + lane; j < e; j += 32) {
                    const int32_t col = a.indices[j];
                    const double v = a.data[j];
                    if (col < 0 || col >= a.L) { gb.fail(HDFE_ERR_BAD_CODE); continue; }
                    double g[K];
                    gather_p<K, PS>(a.P, col, g);
#pragma unroll
                    for (int k = 0; k < K; k++) acc[k] += v * g[k];
                }
#pragma unroll
                for (int k = 0; k < K; k++) {
                    const double t = warp_sum(acc[k]);
                    if (lane == 0) {
                        a.cp[(int64_t)c * K + k] = t;
                        dot[k] += t * a.P[r * PS + k];
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < K; k++) dot[k] = warp_sum(dot[k]);
        if (!system_totals<K, S5>(a, gb, dot, 2 * K, s_w, s_sys, first, nsys, local)) return;
        // the parity-(it + 1) flag was read by everyone before that barrier
        if (blockIdx.x == 0 && threadIdx.x == 0) a.flag[(it + 1) & 1] = 0;
        double alpha[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const double pap = dot[k];
            alpha[k] = (active[k] && pap > 0.0) ? rz[k] / pap : 0.0;
        }
        // ---- B: X += alpha P, R -= alpha AP; ||R||^2, R'dinv R
        double sr[K], s2[K];
#pragma unroll
        for (int k = 0; k < K; k++) sr[k] = s2[k] = 0.0;
        for (int64_t r = r0 + lane; r < r1; r += 32) {
            const double di = a.dinv[r];
            double ap[K];
            const int32_t c0 = a.row_chunk[r];
            if (c0 < 0) {
#pragma unroll
                for (int k = 0; k < K; k++) ap[k] = a.AP[r * K + k];
            } else {
#pragma unroll
                for (int k = 0; k < K; k++) ap[k] = 0.0;
                for (int c = c0; a.chunk_row[c] == (int32_t)r; c++) {
#pragma unroll
                    for (int k = 0; k < K; k++) ap[k] += a.cp[(int64_t)c * K + k];
                    if (c + 1 >= a.wchunk[a.nwarps]) break;
                }
            }
#pragma unroll
            for (int k = 0; k < K; k++) {
                a.X[r * K + k] += alpha[k] * a.P[r * PS + k];
                const double res = a.R[r * K + k] - alpha[k] * ap[k];
                a.R[r * K + k] = res;
                sr[k] += res * res;
                s2[k] += res * res * di;
            }
        }
        double v[2 * K];
#pragma unroll
        for (int k = 0; k < K; k++) { v[k] = warp_sum(sr[k]); v[K + k] = warp_sum(s2[k]); }
        if (!system_totals<2 * K, S5>(a, gb, v, 3 * K, s_w, s_sys, first, nsys, local)) return;
        // ---- C: convergence, beta, P = dinv R + beta P
        bool sys_active = false;
        double beta[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const double rr = v[k];
            const double rzn = v[K + k];
            rel[k] = sqrt(rr) / bnorm[k];
            active[k] = rel[k] > a.tol;
            sys_active |= active[k];
            beta[k] = active[k] ? rzn / (rz[k] != 0.0 ? rz[k] : 1.0) : 0.0;
            rz[k] = rzn;
        }
        if (!sys_active && done_at < 0) done_at = it;
        if (sys_active) {
            for (int64_t r = r0 + lane; r < r1; r += 32) {
                const double di = a.dinv[r];
#pragma unroll
                for (int k = 0; k < K; k++)
                    a.P[r * PS + k] = a.R[r * K + k] * di + beta[k] * a.P[r * PS + k];
            }
            if (lane == 0) atomicOr(a.flag + (it & 1), 1u);
        }
        if (!gb.sync()) return;
        if (*(volatile unsigned *)(a.flag + (it & 1)) == 0) break;
    }
    if (gw == w0 && lane == 0) {
        double mx = 0.0;
        bool conv = true;
#pragma unroll
        for (int k = 0; k < K; k++) {
            if (zero[k]) continue;
            mx = fmax(mx, rel[k]);
            conv &= !active[k];
        }
        a.iterations[sys] = done_at >= 0 ? done_at : (it > a.maxiter ? a.maxiter : it);
        a.converged[sys] = conv ? 1 : 0;
        a.max_rel[sys] = mx;
    }
}

template <int K, int LPR>
int blocks_per_sm()
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_pcg<K, LPR>, kThreads, 0) !=
        cudaSuccess)
        return -1;
    return per_sm;
}

template <int K>
int per_sm_for(int lpr)
{
    switch (lpr) {
    case 4: return blocks_per_sm<K, 4>();
    case 8: return blocks_per_sm<K, 8>();
    case 16: return blocks_per_sm<K, 16>();
    case 32: return blocks_per_sm<K, 32>();
    }
    return -1;
}

int per_sm(int k, int lpr)
{
    switch (k) {
    case 1: return per_sm_for<1>(lpr);
    case 2: return per_sm_for<2>(lpr);
    case 3: return per_sm_for<3>(lpr);
    case 4: return per_sm_for<4>(lpr);
    case 5: return per_sm_for<5>(lpr);
    case 6: return per_sm_for<6>(lpr);
    case 7: return per_sm_for<7>(lpr);
    case 8: return per_sm_for<8>(lpr);
    }
    return -1;
}

template <int K, int LPR>
cudaError_t launch(Args a, int blocks, cudaStream_t s)
{
    void *args[] = {&a};
    return cudaLaunchCooperativeKernel((const void *)k_batch_pcg<K, LPR>, dim3(blocks),
                                       dim3(kThreads), args, 0, s);
}

template <int K>
cudaError_t launch_k(Args a, int lpr, int blocks, cudaStream_t s)
{
    switch (lpr) {
    case 4: return launch<K, 4>(a, blocks, s);
    case 8: return launch<K, 8>(a, blocks, s);
    case 16: return launch<K, 16>(a, blocks, s);
    default: return launch<K, 32>(a, blocks, s);
    }
}

cudaError_t launch_any(Args a, int k, int lpr, int blocks, cudaStream_t s)
{
    switch (k) {
    case 1: return launch_k<1>(a, lpr, blocks, s);
    case 2: return launch_k<2>(a, lpr, blocks, s);
    case 3: return launch_k<3>(a, lpr, blocks, s);
    case 4: return launch_k<4>(a, lpr, blocks, s);
    case 5: return launch_k<5>(a, lpr, blocks, s);
    case 6: return launch_k<6>(a, lpr, blocks, s);
    case 7: return launch_k<7>(a, lpr, blocks, s);
    default: return launch_k<8>(a, lpr, blocks, s);
    }
}

__global__ void k_status(const unsigned *bar, int32_t *status)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *status = (int32_t)bar[2];
}

}  // namespace batch
}  // namespace hdfe

using namespace hdfe;

extern "C" int hdfe_batch_pcg_grid(int32_t k, int32_t lanes_per_row, int32_t *blocks,
                                   int32_t *warps_per_block)
{
    if (k < 1 || k > batch::kMaxK || !(lanes_per_row == 4 || lanes_per_row == 8 ||
                                       lanes_per_row == 16 || lanes_per_row == 32) ||
        !blocks || !warps_per_block)
        return hdfe_set_arg_error("hdfe_batch_pcg_grid: bad argument (k <= 8, lanes 4/8/16/32)");
    int dev = 0, sms = 0;
    HDFE_CUDA_TRY(cudaGetDevice(&dev));
    HDFE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int per = batch::per_sm(k, lanes_per_row);
    if (per < 1) return hdfe_set_error(HDFE_ERR_CUDA, "hdfe_batch_pcg_grid: no occupancy");
    *blocks = sms * per;
    *warps_per_block = batch::kWarps;
    return HDFE_OK;
}

extern "C" int64_t hdfe_batch_pcg_workspace_bytes(int64_t L, int32_t k, int64_t warps,
                                                  int64_t n_chunks)
{
    if (L < 1 || k < 1 || k > batch::kMaxK || warps < 1 || n_chunks < 0) return -1;
    auto up = [](int64_t b) { return (b + 255) / 256 * 256; };
    return 2 * up(L * k * 8) + up(L * batch::p_stride(k) * 8) + up(warps * 5 * k * 8) +
           up((n_chunks + 1) * k * 8) + 256;
}

extern "C" int hdfe_batch_pcg_solve(const int64_t *indptr, const int32_t *indices,
                                    const double *data, int64_t L, const double *dinv,
                                    const double *B, int32_t k, const uint8_t *zero,
                                    int64_t n_systems, const int64_t *warp_rows,
                                    const int32_t *warp_system, const int32_t *system_warps,
                                    const int32_t *warp_chunks, const int32_t *chunk_row,
                                    const int64_t *chunk_lo, const int64_t *chunk_hi,
                                    const int32_t *row_chunk,
                                    int64_t n_chunks, int32_t blocks, int32_t lanes_per_row,
                                    double tol,
                                    int64_t maxiter, double *X, int64_t *iterations,
                                    double *max_rel, int32_t *converged, int32_t *status,
                                    void *workspace, int64_t workspace_bytes, void *stream)
{
    if (!indptr || !indices || !data || L < 1 || !dinv || !B || k < 1 || k > batch::kMaxK ||
        n_systems < 1 || !warp_rows || !warp_system || !system_warps || !warp_chunks ||
        !row_chunk || n_chunks < 0 || (n_chunks > 0 && (!chunk_row || !chunk_lo || !chunk_hi)) ||
        blocks < 1 ||
        !(lanes_per_row == 4 || lanes_per_row == 8 || lanes_per_row == 16 ||
          lanes_per_row == 32) ||
        !(tol > 0.0) || maxiter < 1 || !X || !iterations || !max_rel || !converged || !status ||
        !workspace)
        return hdfe_set_arg_error("hdfe_batch_pcg_solve: bad argument");
    if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
        return hdfe_set_arg_error("hdfe_batch_pcg_solve: workspace must be 256-byte aligned");
    const int64_t warps = (int64_t)blocks * batch::kWarps;
    if (workspace_bytes < hdfe_batch_pcg_workspace_bytes(L, k, warps, n_chunks))
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_batch_pcg_solve: workspace too small");
    int dev = 0, sms = 0;
    HDFE_CUDA_TRY(cudaGetDevice(&dev));
    HDFE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int per = batch::per_sm(k, lanes_per_row);
    if (per < 1 || blocks > sms * per)
        return hdfe_set_arg_error("hdfe_batch_pcg_solve: more blocks than can be resident");
    cudaStream_t s = (cudaStream_t)stream;
    auto up = [](int64_t b) { return (b + 255) / 256 * 256; };
    char *ws = (char *)workspace;
    batch::Args a{};
    a.indptr = indptr;
    a.indices = indices;
    a.data = data;
    a.L = L;
    a.dinv = dinv;
    a.B = B;
    a.zero = zero;
    a.tol = tol;
    a.maxiter = maxiter;
    a.X = X;
    const int64_t vec = up(L * k * 8), pvec = up(L * batch::p_stride(k) * 8);
    a.R = (double *)ws;
    a.P = (double *)(ws + vec);
    a.AP = (double *)(ws + vec + pvec);
    a.cpart = (double *)(ws + 2 * vec + pvec);
    a.cp = (double *)(ws + 2 * vec + pvec + up(warps * 5 * k * 8));
    unsigned *words = (unsigned *)(ws + 2 * vec + pvec + up(warps * 5 * k * 8) +
                                   up((n_chunks + 1) * k * 8));
    a.bar = words;          // [0..2] barrier
    a.flag = words + 4;     // [2]
    a.wrow = warp_rows;
    a.wsys = warp_system;
    a.swarp = system_warps;
    a.wchunk = warp_chunks;
    a.chunk_row = chunk_row;
    a.chunk_lo = chunk_lo;
    a.chunk_hi = chunk_hi;
    a.row_chunk = row_chunk;
    a.nwarps = warps;
    a.iterations = iterations;
    a.max_rel = max_rel;
    a.converged = converged;
    HDFE_CUDA_TRY(cudaMemsetAsync(words, 0, 64, s));
    HDFE_CUDA_TRY(batch::launch_any(a, k, lanes_per_row, blocks, s));
    batch::k_status<<<1, 32, 0, s>>>(a.bar, status);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(2);
    return HDFE_OK;
}
