// Row passes of the KSS standard errors (leaveout_se.py, kernels_se.py).
//
//   k_readout       (A u)_i = u_g(i) + sum_d u_levels[level_d(i)] + x_i' u_cov,
//                   optionally times sqrt(w_i): kernels_se.py:19-43
//                   `_nb_readout`.  A warp takes a group; its rows' B values are
//                   one contiguous stretch of the output, which the lanes walk
//                   flat (row, column), so stores are coalesced and each
//                   row's gathers of U touch B consecutive values.
//   k_cov_cross     kernels_se.py:46-77 `_nb_cov_cross`: per psi level the sum
//                   of w_i u_streamed[g(i)] (atomic), per group the sum of
//                   w_i u_levels[psi(i)]; a warp per group, a lane per column.
//   k_bii_moments   kernels_se.py:80-98 `_nb_bii_moments`, thread per row.
//   k_c_sums        the assembly of C v = B v - (b .* M v + M (b .* v)) / 2
//                   from the readouts (leaveout_se.py:579-596) fused with the
//                   sums the first term, theta and the trace term take of it
//                   (:718-726, :918-925); per-CTA sums in a fixed order, then
//                   over CTAs in a fixed order.
//   k_smooth_cells  / k_smooth_eval: the sigma2 smoother (leaveout_se.py:
//                   982-1054): a row's cell in the grid of empirical quantiles
//                   of (P_ii, B_ii), cell sums, and the bilinear evaluation
//                   between cell centres.  The rank map is numpy's `interp`
//                   through the knots, evaluated in the same order of
//                   operations (no fused multiply-add).
#include <cuda_runtime.h>

#include "common.cuh"

namespace hdfe {
namespace se {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxCov = 8;
constexpr int kMaxKnots = 1024;
constexpr int kSumGrid = 148 * 4;

struct Rows {
    const int64_t *starts;
    int64_t G;
    const uint32_t *codes;
    int D;
    int64_t offs[HDFE_MAX_DIMS];
    int64_t nlev[HDFE_MAX_DIMS];
    const double *X;
    int c;
    unsigned *status;
};

__device__ __forceinline__ int64_t level_of(const Rows &r, int64_t i, int d)
{
    uint32_t code = r.codes[i * r.D + d];
    if ((int64_t)code >= r.nlev[d]) {
        if (r.status) atomicCAS(r.status, 0u, (unsigned)HDFE_ERR_BAD_CODE);
        code = 0;
    }
    return r.offs[d] + code;
}

__global__ void __launch_bounds__(kThreads) k_readout(Rows r, const double *Ul, const double *Uc,
                                                      const double *Ug, int B, const double *w,
                                                      double *out)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * kThreads) >> 5;
    for (int64_t g = warp; g < r.G; g += nw) {
        const int64_t s = r.starts[g], e = r.starts[g + 1];
        const int64_t n = (e - s) * B;
        for (int64_t t = lane; t < n; t += 32) {
            const int64_t i = s + t / B;
            const int j = (int)(t % B);
            double h = Ug[g * B + j];
            for (int d = 0; d < r.D; d++) h += Ul[level_of(r, i, d) * B + j];
            for (int k = 0; k < r.c; k++) h += r.X[i * r.c + k] * Uc[k * B + j];
            if (w) h *= sqrt(w[i]);
            out[s * B + t] = h;
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_cov_cross(Rows r, int psi, const double *w,
                                                        const double *Ul, const double *Ug,
                                                        int B, double *acc, double *out_groups)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * kThreads) >> 5;
    for (int64_t g = warp; g < r.G; g += nw) {
        if (lane >= B) continue;
        const int64_t s = r.starts[g], e = r.starts[g + 1];
        const double ug = Ug[g * B + lane];
        double total = 0.0;
        for (int64_t i = s; i < e; i++) {
            const double wi = w ? w[i] : 1.0;
            const int64_t l = level_of(r, i, psi);
            atomicAdd(acc + l * B + lane, wi * ug);
            total += wi * Ul[l * B + lane];
        }
        out_groups[g * B + lane] = total;
    }
}

// out (3, N) += per row: sum_j (root r1_j)^2, (root r2_j)^2, root^2 r1_j r2_j;
// rows (N, 2 * size) holds r1 then r2
__global__ void __launch_bounds__(kThreads) k_bii_moments(const double *rows, int size,
                                                          const double *w, int64_t N,
                                                          double *out)
{
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < N;
         i += (int64_t)gridDim.x * kThreads) {
        const double root = w ? sqrt(w[i]) : 1.0;
        const double *r = rows + i * 2 * size;
        double a = 0.0, b = 0.0, c = 0.0;
        for (int j = 0; j < size; j++) {
            const double x = root * r[j], y = root * r[size + j];
            a += x * x;
            b += y * y;
            c += x * y;
        }
        out[i] += a;
        out[N + i] += b;
        out[2 * N + i] += c;
    }
}

// C v per component from the readouts, and its sums.
//   v: (N, nv) with nv = size (shared input) or the draws z (N, size) scaled
//   per component by scale_k = sqrt(max(s_k, 0)) (per_component);
//   base (N, (n_in + 3) size) = sqrt(w) A U0, through_q (N, 3 size) = sqrt(w)
//   A U1 (both already scaled by the root);
//   part[blockIdx][q] (kSums values): q = k: sum_i s_k,i sum_j cv_kij^2;
//   q = 3 + k: sum_i y_i cv_ki0 (y NULL: 0); q = 6 + k: see g below.
// n_vec row vectors u (n_vec, 3, N) with coef (3, 1 + n_vec, size), when
// given, add low-rank terms: cv_kij += coef[k][0][j] + sum_r u_rki
// coef[k][1 + r][j] -- the rank-two term of the reference-centred kernel
// (leaveout_se.py:591-595) and the deflation of C2 (:580-582).  g (3, N), when
// given, adds sums[6 + k] = sum_i g_ki cv_ki0 (the covariance of b1 and theta1).
constexpr int kMaxVec = 4;
constexpr int kSums = 9;

__global__ void __launch_bounds__(kThreads) k_c_sums(const double *v, int size, int per_component,
                                                     const double *b, const double *s,
                                                     const double *base, const double *thq,
                                                     const double *y, int n_vec, const double *u,
                                                     const double *coef, const double *g,
                                                     int64_t N, double *part)
{
    __shared__ double s_red[kWarps][kSums];
    const int n_in = per_component ? 3 : 1;
    const int wide = (n_in + 3) * size;
    double acc[kSums] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < N;
         i += (int64_t)gridDim.x * kThreads) {
        const double *bs = base + i * wide;
        const double *tq = thq + i * 3 * size;
        for (int k = 0; k < 3; k++) {
            const double bk = b[k * N + i];
            const double sk = s[k * N + i];
            const double scale = per_component ? sqrt(fmax(sk, 0.0)) : 1.0;
            const int in0 = (per_component ? k : 0) * size;
            const int bc0 = (n_in + k) * size;
            double uk[kMaxVec];
            for (int r = 0; r < n_vec; r++) uk[r] = u[((int64_t)r * 3 + k) * N + i];
            const double *ck = coef ? coef + (int64_t)k * (1 + n_vec) * size : nullptr;
            double sq = 0.0;
            for (int j = 0; j < size; j++) {
                const double vk = v[i * size + j] * scale;
                const double Mv = vk - bs[in0 + j];
                const double Bv = tq[k * size + j];
                const double M_bv = vk * bk - bs[bc0 + j];
                double cv = Bv - 0.5 * (bk * Mv + M_bv);
                if (ck) {
                    double low = ck[j];
                    for (int r = 0; r < n_vec; r++) low += uk[r] * ck[(1 + r) * size + j];
                    cv += low;
                }
                sq += cv * cv;
                if (j == 0) {
                    if (y) acc[3 + k] += y[i] * cv;
                    if (g) acc[6 + k] += g[k * N + i] * cv;
                }
            }
            acc[k] += sk * sq;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < kSums; q++) {
        const double t = warp_sum(acc[q]);
        if (lane == 0) s_red[warp][q] = t;
    }
    __syncthreads();
    if (threadIdx.x < kSums) {
        double t = 0.0;
        for (int wv = 0; wv < kWarps; wv++) t += s_red[wv][threadIdx.x];
        part[(int64_t)blockIdx.x * kSums + threadIdx.x] = t;
    }
}

// out[q] for q < n = the sum over blocks of part[block * stride + q], one warp
// per q, in a fixed order
__global__ void __launch_bounds__(kThreads) k_sum_parts(const double *part, int blocks, int n,
                                                        int stride, double *out)
{
    const int lane = threadIdx.x & 31;
    const int q = (int)(((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5);
    if (q >= n) return;
    double t = 0.0;
    for (int bl = lane; bl < blocks; bl += 32) t += part[(int64_t)bl * stride + q];
    t = warp_sum(t);
    if (lane == 0) out[q] = t;
}

// numpy.interp(x, xp, fp) with xp increasing (n points), left/right clamped
__device__ __forceinline__ double interp(double x, const double *xp, const double *fp, int n)
{
    if (x <= xp[0]) return fp[0];            // numpy: x < xp[0] -> left = fp[0]
    if (x >= xp[n - 1]) return fp[n - 1];
    int lo = 0, hi = n - 1;                  // xp[lo] <= x < xp[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (xp[mid] <= x) lo = mid;
        else hi = mid;
    }
    const double slope = __ddiv_rn(__dsub_rn(fp[lo + 1], fp[lo]), __dsub_rn(xp[lo + 1], xp[lo]));
    return __dadd_rn(__dmul_rn(slope, __dsub_rn(x, xp[lo])), fp[lo]);
}

struct Smooth {
    const double *knots0, *knots1, *fp;     // n_bins + 1 each; knots1 NULL: one axis
    int n_bins;
};

__device__ __forceinline__ void load_knots(const Smooth &sm, double *s0, double *s1, double *sf)
{
    for (int t = threadIdx.x; t <= sm.n_bins; t += kThreads) {
        s0[t] = sm.knots0[t];
        if (sm.knots1) s1[t] = sm.knots1[t];
        sf[t] = sm.fp[t];
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kThreads) k_smooth_cells(Smooth sm, const double *lev,
                                                           const double *bii,
                                                           const double *sigma2, int64_t N,
                                                           double *totals, double *counts)
{
    __shared__ double s0[kMaxKnots + 1], s1[kMaxKnots + 1], sf[kMaxKnots + 1];
    load_knots(sm, s0, s1, sf);
    const int nk = sm.n_bins + 1;
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < N;
         i += (int64_t)gridDim.x * kThreads) {
        int64_t c0 = (int64_t)__dmul_rn(interp(lev[i], s0, sf, nk), (double)sm.n_bins);
        if (c0 > sm.n_bins - 1) c0 = sm.n_bins - 1;
        int64_t cell = c0;
        if (sm.knots1) {
            int64_t c1 = (int64_t)__dmul_rn(interp(bii[i], s1, sf, nk), (double)sm.n_bins);
            if (c1 > sm.n_bins - 1) c1 = sm.n_bins - 1;
            cell = c0 * sm.n_bins + c1;
        }
        atomicAdd(totals + cell, sigma2[i]);
        atomicAdd(counts + cell, 1.0);
    }
}

__device__ __forceinline__ void cell_weights(double rank, int n_bins, int64_t &j0, double &a)
{
    const double f = __dsub_rn(__dmul_rn(rank, (double)n_bins), 0.5);
    int64_t j = (int64_t)floor(f);
    if (j < 0) j = 0;
    if (j > n_bins - 2) j = n_bins - 2;
    j0 = j;
    a = fmin(fmax(__dsub_rn(f, (double)j), 0.0), 1.0);
}

__global__ void __launch_bounds__(kThreads) k_smooth_eval(Smooth sm, const double *means,
                                                          const double *lev,
                                                          const double *bii, int64_t N,
                                                          double *out)
{
    __shared__ double s0[kMaxKnots + 1], s1[kMaxKnots + 1], sf[kMaxKnots + 1];
    load_knots(sm, s0, s1, sf);
    const int nk = sm.n_bins + 1, nb = sm.n_bins;
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < N;
         i += (int64_t)gridDim.x * kThreads) {
        int64_t i0;
        double a;
        cell_weights(interp(lev[i], s0, sf, nk), nb, i0, a);
        const double ca = __dsub_rn(1.0, a);
        if (!sm.knots1) {
            out[i] = __dadd_rn(__dmul_rn(ca, means[i0]), __dmul_rn(a, means[i0 + 1]));
            continue;
        }
        int64_t j0;
        double b;
        cell_weights(interp(bii[i], s1, sf, nk), nb, j0, b);
        const double cb = __dsub_rn(1.0, b);
        double t = __dmul_rn(__dmul_rn(ca, cb), means[i0 * nb + j0]);
        t = __dadd_rn(t, __dmul_rn(__dmul_rn(a, cb), means[(i0 + 1) * nb + j0]));
        t = __dadd_rn(t, __dmul_rn(__dmul_rn(ca, b), means[i0 * nb + j0 + 1]));
        t = __dadd_rn(t, __dmul_rn(__dmul_rn(a, b), means[(i0 + 1) * nb + j0 + 1]));
        out[i] = t;
    }
}

int fill(Rows &r, const int64_t *starts, int64_t G, const uint32_t *codes, int32_t D,
         const int64_t *n_levels, const double *X, int32_t c, void *status)
{
    if (!starts || G < 0 || !codes || D < 1 || D > HDFE_MAX_DIMS || !n_levels || c < 0 ||
        c > kMaxCov || (c > 0 && !X))
        return hdfe_set_arg_error("standard-error row pass: bad argument");
    r = Rows{};
    r.starts = starts;
    r.G = G;
    r.codes = codes;
    r.D = D;
    int64_t off = 0;
    for (int d = 0; d < D; d++) {
        r.offs[d] = off;
        r.nlev[d] = n_levels[d];
        off += n_levels[d];
    }
    r.X = X;
    r.c = c;
    r.status = (unsigned *)status;
    return HDFE_OK;
}

inline unsigned grid_for(int64_t items, int per_block, int64_t cap = 148 * 32)
{
    int64_t b = (items + per_block - 1) / per_block;
    if (b > cap) b = cap;
    return (unsigned)(b > 0 ? b : 1);
}

}  // namespace se
}  // namespace hdfe

using namespace hdfe;

extern "C" int hdfe_rows_readout(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                                 int32_t D, const int64_t *n_levels, const double *X, int32_t c,
                                 const double *U_levels, const double *U_cov,
                                 const double *U_groups, int32_t B, const double *w,
                                 double *out, void *status, void *stream)
{
    se::Rows r;
    int st = se::fill(r, starts, n_groups, codes, D, n_levels, X, c, status);
    if (st != HDFE_OK) return st;
    if (B < 1 || !U_levels || !U_groups || !out || (c > 0 && !U_cov))
        return hdfe_set_arg_error("hdfe_rows_readout: bad argument");
    se::k_readout<<<se::grid_for(n_groups, se::kWarps), se::kThreads, 0, (cudaStream_t)stream>>>(
        r, U_levels, U_cov, U_groups, B, w, out);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(1);
    return HDFE_OK;
}

extern "C" int hdfe_cov_cross(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                              int32_t D, const int64_t *n_levels, int32_t psi_column,
                              const double *w, const double *U_levels, const double *U_groups,
                              int32_t B, double *acc, double *out_groups, void *status,
                              void *stream)
{
    se::Rows r;
    int st = se::fill(r, starts, n_groups, codes, D, n_levels, nullptr, 0, status);
    if (st != HDFE_OK) return st;
    if (B < 1 || B > 32 || psi_column < 0 || psi_column >= D || !U_levels || !U_groups || !acc ||
        !out_groups)
        return hdfe_set_arg_error("hdfe_cov_cross: bad argument (B <= 32)");
    se::k_cov_cross<<<se::grid_for(n_groups, se::kWarps), se::kThreads, 0,
                      (cudaStream_t)stream>>>(r, psi_column, w, U_levels, U_groups, B, acc,
                                              out_groups);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(1);
    return HDFE_OK;
}

extern "C" int hdfe_bii_moments(const double *rows, int32_t size, const double *w, int64_t n_rows,
                                double *out, void *stream)
{
    if (!rows || size < 1 || n_rows < 0 || !out)
        return hdfe_set_arg_error("hdfe_bii_moments: bad argument");
    if (n_rows == 0) return HDFE_OK;
    se::k_bii_moments<<<se::grid_for(n_rows, se::kThreads), se::kThreads, 0,
                        (cudaStream_t)stream>>>(rows, size, w, n_rows, out);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(1);
    return HDFE_OK;
}

extern "C" int64_t hdfe_c_sums_workspace_bytes(void)
{
    return (int64_t)se::kSumGrid * se::kSums * 8;
}

extern "C" int hdfe_c_sums_ext(const double *v, int32_t size, int32_t per_component,
                               const double *b, const double *s, const double *base,
                               const double *through_q, const double *y, int32_t n_vec,
                               const double *u, const double *coef, const double *g,
                               int64_t n_rows, double *sums, void *workspace,
                               int64_t workspace_bytes, void *stream)
{
    if (!v || size < 1 || !b || !s || !base || !through_q || n_rows < 1 || !sums || !workspace ||
        workspace_bytes < hdfe_c_sums_workspace_bytes() || n_vec < 0 || n_vec > se::kMaxVec ||
        (n_vec > 0 && !u))
        return hdfe_set_arg_error("hdfe_c_sums: bad argument (0 <= n_vec <= 4)");
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned grid = se::grid_for(n_rows, se::kThreads, se::kSumGrid);
    double *part = (double *)workspace;
    se::k_c_sums<<<grid, se::kThreads, 0, st>>>(v, size, per_component, b, s, base, through_q, y,
                                                coef ? n_vec : 0, u, coef, g, n_rows, part);
    const int n_sums = g ? se::kSums : 6;
    se::k_sum_parts<<<(n_sums + se::kWarps - 1) / se::kWarps, se::kThreads, 0, st>>>(
        part, (int)grid, n_sums, se::kSums, sums);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(2);
    return HDFE_OK;
}

extern "C" int hdfe_c_sums(const double *v, int32_t size, int32_t per_component, const double *b,
                           const double *s, const double *base, const double *through_q,
                           const double *y, int64_t n_rows, double *sums, void *workspace,
                           int64_t workspace_bytes, void *stream)
{
    return hdfe_c_sums_ext(v, size, per_component, b, s, base, through_q, y, 0, nullptr, nullptr,
                           nullptr, n_rows, sums, workspace, workspace_bytes, stream);
}

extern "C" int hdfe_smooth_cells(const double *knots0, const double *knots1, const double *fp,
                                 int32_t n_bins, const double *leverage, const double *b_ii,
                                 const double *sigma2, int64_t n_rows, double *totals,
                                 double *counts, void *stream)
{
    if (!knots0 || !fp || n_bins < 2 || n_bins > se::kMaxKnots || !leverage ||
        (knots1 && !b_ii) || !sigma2 || n_rows < 0 || !totals || !counts)
        return hdfe_set_arg_error("hdfe_smooth_cells: bad argument (2 <= n_bins <= 1024)");
    if (n_rows == 0) return HDFE_OK;
    se::Smooth sm{knots0, knots1, fp, n_bins};
    se::k_smooth_cells<<<se::grid_for(n_rows, se::kThreads, 148 * 8), se::kThreads, 0,
                         (cudaStream_t)stream>>>(sm, leverage, b_ii, sigma2, n_rows, totals,
                                                 counts);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(1);
    return HDFE_OK;
}

extern "C" int hdfe_smooth_eval(const double *knots0, const double *knots1, const double *fp,
                                int32_t n_bins, const double *means, const double *leverage,
                                const double *b_ii, int64_t n_rows, double *out, void *stream)
{
    if (!knots0 || !fp || n_bins < 2 || n_bins > se::kMaxKnots || !means || !leverage ||
        (knots1 && !b_ii) || n_rows < 0 || !out)
        return hdfe_set_arg_error("hdfe_smooth_eval: bad argument (2 <= n_bins <= 1024)");
    if (n_rows == 0) return HDFE_OK;
    se::Smooth sm{knots0, knots1, fp, n_bins};
    se::k_smooth_eval<<<se::grid_for(n_rows, se::kThreads, 148 * 8), se::kThreads, 0,
                        (cudaStream_t)stream>>>(sm, means, leverage, b_ii, n_rows, out);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(1);
    return HDFE_OK;
}
