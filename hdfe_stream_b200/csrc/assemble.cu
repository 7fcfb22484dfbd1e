// Steps 3-4 of a fit, as far as the KSS components read them.
//
// Reference: core/kernels_base.py:114-146 `_nb_residualize_rows` with
// core/inference.py:109-135 `_assemble` (V' W V of the fully residualised
// variables), core/kernels_base.py:544-615 `_nb_pass2` (residuals and the
// streamed effect, with gam_y = Gamma_y - Gamma_x beta, core/inference.py:
// 454-456) and the KSS pieces of leaveout.py: the plug-in moments' sums
// (:807-833) and sigma2 (:949-1016, stayers "own", weighted centring).
//
// One thread per group of rows (the groups are short, ~10 rows): the group's
// rows are read twice, once for its weighted means and once for the sums.
// Per-thread sums are combined per CTA in a fixed order and then over CTAs in
// a fixed order, so both results are deterministic.
#include <cuda_runtime.h>

#include "common.cuh"

namespace hdfe {
namespace assemble {

constexpr int kThreads = 256;
constexpr int kGrid = 148 * 4;
constexpr int kMaxM = 8;

struct Args {
    const int64_t *starts;
    int64_t G;
    const uint32_t *codes;
    int D;
    int64_t offs[HDFE_MAX_DIMS];
    int64_t nlev[HDFE_MAX_DIMS];
    const double *w;
    const double *V;        // (m, N): one row per variable
    int m;
    int64_t N;
    unsigned *status;
};

__device__ __forceinline__ int64_t level(const Args &a, int64_t i, int d)
{
    uint32_t c = a.codes[i * a.D + d];
    if ((int64_t)c >= a.nlev[d]) {
        if (a.status) atomicCAS(a.status, 0u, (unsigned)HDFE_ERR_BAD_CODE);
        c = 0;
    }
    return a.offs[d] + c;
}

// per CTA: thread values v[0..n) summed over the CTA in thread order
__device__ __forceinline__ void cta_sums(const double *v, int n, double *s_part, double *out)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < n; q++) {
        const double t = warp_sum(v[q]);
        if (lane == 0) s_part[warp * n + q] = t;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < n; q += kThreads) {
        double s = 0.0;
        for (int wv = 0; wv < kThreads / 32; wv++) s += s_part[wv * n + q];
        out[(int64_t)blockIdx.x * n + q] = s;
    }
}

// V' W V of the residualised variables: per-CTA partials (gridDim, m, m)
template <int M>
__global__ void __launch_bounds__(kThreads) k_moments(Args a, const double *Gamma, double *part)
{
    __shared__ double s_part[(kThreads / 32) * kMaxM * kMaxM];
    double acc[M * M];
#pragma unroll
    for (int q = 0; q < M * M; q++) acc[q] = 0.0;
    for (int64_t g = (int64_t)blockIdx.x * kThreads + threadIdx.x; g < a.G;
         g += (int64_t)gridDim.x * kThreads) {
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        double q[M], Wg = 0.0;
#pragma unroll
        for (int j = 0; j < M; j++) q[j] = 0.0;
        for (int64_t i = s; i < e; i++) {
            const double wi = a.w ? a.w[i] : 1.0;
            Wg += wi;
#pragma unroll
            for (int j = 0; j < M; j++) {
                double v = a.V[(int64_t)j * a.N + i];
                for (int d = 0; d < a.D; d++) v -= Gamma[level(a, i, d) * M + j];
                q[j] += wi * v;
            }
        }
#pragma unroll
        for (int j = 0; j < M; j++) q[j] = Wg > 0.0 ? q[j] / Wg : 0.0;
        for (int64_t i = s; i < e; i++) {
            const double wi = a.w ? a.w[i] : 1.0;
            double v[M];
#pragma unroll
            for (int j = 0; j < M; j++) {
                double x = a.V[(int64_t)j * a.N + i];
                for (int d = 0; d < a.D; d++) x -= Gamma[level(a, i, d) * M + j];
                v[j] = x - q[j];
            }
#pragma unroll
            for (int j = 0; j < M; j++)
#pragma unroll
                for (int k = 0; k < M; k++) acc[j * M + k] += wi * v[j] * v[k];
        }
    }
    cta_sums(acc, M * M, s_part, part);
}

// The y-equation's residuals and streamed effect, and the sums the plug-in
// moments and the centring of sigma2 need: w, w y, w a, w b, w a^2, w b^2,
// w a b (a = the psi dimension's effect, b = the streamed effect).
template <int M>
__global__ void __launch_bounds__(kThreads) k_effects(Args a, int psi, const double *beta,
                                                      const double *gam_y, double *resid,
                                                      double *alpha, double *part)
{
    __shared__ double s_part[(kThreads / 32) * 7];
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    double b[M > 1 ? M - 1 : 1];
#pragma unroll
    for (int j = 0; j + 1 < M; j++) b[j] = beta[j];
    for (int64_t g = (int64_t)blockIdx.x * kThreads + threadIdx.x; g < a.G;
         g += (int64_t)gridDim.x * kThreads) {
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        auto u_of = [&](int64_t i) {
            double u = a.V[i];
#pragma unroll
            for (int j = 0; j + 1 < M; j++) u -= a.V[(int64_t)(j + 1) * a.N + i] * b[j];
            for (int d = 0; d < a.D; d++) u -= gam_y[level(a, i, d)];
            return u;
        };
        double Wg = 0.0, mu = 0.0;
        for (int64_t i = s; i < e; i++) {
            const double wi = a.w ? a.w[i] : 1.0;
            Wg += wi;
            mu += wi * u_of(i);
        }
        mu = Wg > 0.0 ? mu / Wg : 0.0;
        if (alpha) alpha[g] = mu;
        for (int64_t i = s; i < e; i++) {
            const double wi = a.w ? a.w[i] : 1.0;
            const double ei = u_of(i) - mu;
            if (resid) resid[i] = ei;
            const double ap = gam_y[level(a, i, psi)];
            acc[0] += wi;
            acc[1] += wi * a.V[i];
            acc[2] += wi * ap;
            acc[3] += wi * mu;
            acc[4] += wi * ap * ap;
            acc[5] += wi * mu * mu;
            acc[6] += wi * ap * mu;
        }
    }
    cta_sums(acc, 7, s_part, part);
}

// The sums of the variances of beta (core/inference.py:566-578, OLS with
// analytic weights): with h the residualised covariates (x less Gamma_x's
// projection and its weighted group mean) and e the residuals (the y
// equation's, as k_effects), per CTA: the bread sum w h h', the meat sum
// (w e)^2 h h', the streamed groups' meat sum_g s_g s_g' (s_g the group's
// sum of w e h) -- each as its upper triangle, row by row -- and sum w e^2.
template <int M>
__global__ void __launch_bounds__(kThreads) k_variance(Args a, const double *Gamma,
                                                       const double *beta, double *part)
{
    constexpr int KX = M - 1;
    constexpr int T = KX * (KX + 1) / 2;
    constexpr int NQ = 3 * T + 1;
    __shared__ double s_part[(kThreads / 32) * NQ];
    double acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) acc[q] = 0.0;
    double b[KX];
#pragma unroll
    for (int j = 0; j < KX; j++) b[j] = beta[j];
    for (int64_t g = (int64_t)blockIdx.x * kThreads + threadIdx.x; g < a.G;
         g += (int64_t)gridDim.x * kThreads) {
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        // row i's y and covariates less their fixed-effect projections
        auto raw = [&](int64_t i, double &yr, double (&hr)[KX]) {
            yr = a.V[i];
#pragma unroll
            for (int j = 0; j < KX; j++) hr[j] = a.V[(int64_t)(j + 1) * a.N + i];
            for (int d = 0; d < a.D; d++) {
                const int64_t l = level(a, i, d);
                yr -= Gamma[l * M];
#pragma unroll
                for (int j = 0; j < KX; j++) hr[j] -= Gamma[l * M + j + 1];
            }
        };
        double Wg = 0.0, mu = 0.0, mh[KX];
#pragma unroll
        for (int j = 0; j < KX; j++) mh[j] = 0.0;
        for (int64_t i = s; i < e; i++) {
            const double wi = a.w ? a.w[i] : 1.0;
            double yr, hr[KX];
            raw(i, yr, hr);
            double u = yr;
#pragma unroll
            for (int j = 0; j < KX; j++) { u -= b[j] * hr[j]; mh[j] += wi * hr[j]; }
            Wg += wi;
            mu += wi * u;
        }
        const double inv = Wg > 0.0 ? 1.0 / Wg : 0.0;
        mu *= inv;
#pragma unroll
        for (int j = 0; j < KX; j++) mh[j] *= inv;
        double sg[KX];
#pragma unroll
        for (int j = 0; j < KX; j++) sg[j] = 0.0;
        for (int64_t i = s; i < e; i++) {
            const double wi = a.w ? a.w[i] : 1.0;
            double yr, h[KX];
            raw(i, yr, h);
            double u = yr;
#pragma unroll
            for (int j = 0; j < KX; j++) { u -= b[j] * h[j]; h[j] -= mh[j]; }
            const double ei = u - mu, we = wi * ei;
            int t = 0;
#pragma unroll
            for (int j1 = 0; j1 < KX; j1++)
#pragma unroll
                for (int j2 = j1; j2 < KX; j2++, t++) {
                    acc[t] += wi * h[j1] * h[j2];
                    acc[T + t] += we * we * h[j1] * h[j2];
                }
#pragma unroll
            for (int j = 0; j < KX; j++) sg[j] += we * h[j];
            acc[3 * T] += wi * ei * ei;
        }
        int t = 0;
#pragma unroll
        for (int j1 = 0; j1 < KX; j1++)
#pragma unroll
            for (int j2 = j1; j2 < KX; j2++, t++) acc[2 * T + t] += sg[j1] * sg[j2];
    }
    cta_sums(acc, NQ, s_part, part);
}

// The per-row scores w e h (out (N, m - 1) row-major) from the same row pass
// as k_variance: core/inference.py:594-603, the rows that pass 2 scatters
// into the clusters of a CRV1 term that is not the streamed dimension.
template <int M>
__global__ void __launch_bounds__(kThreads) k_scores(Args a, const double *Gamma,
                                                     const double *beta, double *out,
                                                     double *h_out)
{
    constexpr int KX = M - 1;
    double b[KX];
#pragma unroll
    for (int j = 0; j < KX; j++) b[j] = beta[j];
    for (int64_t g = (int64_t)blockIdx.x * kThreads + threadIdx.x; g < a.G;
         g += (int64_t)gridDim.x * kThreads) {
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        auto raw = [&](int64_t i, double &yr, double (&hr)[KX]) {
            yr = a.V[i];
#pragma unroll
            for (int j = 0; j < KX; j++) hr[j] = a.V[(int64_t)(j + 1) * a.N + i];
            for (int d = 0; d < a.D; d++) {
                const int64_t l = level(a, i, d);
                yr -= Gamma[l * M];
#pragma unroll
                for (int j = 0; j < KX; j++) hr[j] -= Gamma[l * M + j + 1];
            }
        };
        double Wg = 0.0, mu = 0.0, mh[KX];
#pragma unroll
        for (int j = 0; j < KX; j++) mh[j] = 0.0;
        for (int64_t i = s; i < e; i++) {
            const double wi = a.w ? a.w[i] : 1.0;
            double yr, hr[KX];
            raw(i, yr, hr);
            double u = yr;
#pragma unroll
            for (int j = 0; j < KX; j++) { u -= b[j] * hr[j]; mh[j] += wi * hr[j]; }
            Wg += wi;
            mu += wi * u;
        }
        const double inv = Wg > 0.0 ? 1.0 / Wg : 0.0;
        mu *= inv;
#pragma unroll
        for (int j = 0; j < KX; j++) mh[j] *= inv;
        for (int64_t i = s; i < e; i++) {
            const double wi = a.w ? a.w[i] : 1.0;
            double yr, h[KX];
            raw(i, yr, h);
            double u = yr;
#pragma unroll
            for (int j = 0; j < KX; j++) { u -= b[j] * h[j]; h[j] -= mh[j]; }
            const double we = wi * (u - mu);
#pragma unroll
            for (int j = 0; j < KX; j++) out[i * KX + j] = we * h[j];
            if (h_out) {
#pragma unroll
                for (int j = 0; j < KX; j++) h_out[i * KX + j] = h[j];
            }
        }
    }
}

// out[q] = sum over CTAs of part[., q], one warp per entry, fixed order
__global__ void __launch_bounds__(kThreads) k_sum_parts(const double *part, int blocks, int n,
                                                        double *out)
{
    const int lane = threadIdx.x & 31;
    const int q = (int)(((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5);
    if (q >= n) return;
    double s = 0.0;
    for (int b = lane; b < blocks; b += 32) s += part[(int64_t)b * n + q];
    s = warp_sum(s);
    if (lane == 0) out[q] = s;
}

// sigma2_i = w_i (y_i - ybar) e_i / M_ii * factor_i (leaveout.py:1000-1003)
__global__ void __launch_bounds__(kThreads) k_sigma2(const double *y, const double *w,
                                                     const double *e, const double *comp,
                                                     const double *factor, double ybar,
                                                     int64_t N, double *out)
{
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < N;
         i += (int64_t)gridDim.x * kThreads) {
        const double wi = w ? w[i] : 1.0;
        out[i] = wi * (y[i] - ybar) * e[i] / comp[i] * factor[i];
    }
}

int fill(Args &a, const int64_t *starts, int64_t G, const uint32_t *codes, int32_t D,
         const int64_t *n_levels, const double *w, const double *V, int32_t m, int64_t N,
         unsigned *status)
{
    if (D < 1 || D > HDFE_MAX_DIMS || G < 0 || !starts || !codes || !n_levels || !V || m < 1 ||
        m > kMaxM || N < 1)
        return hdfe_set_arg_error("hdfe_resid_moments/row_effects: bad argument (m <= 8)");
    a = Args{};
    a.starts = starts;
    a.G = G;
    a.codes = codes;
    a.D = D;
    int64_t L = 0;
    for (int d = 0; d < D; d++) {
        a.offs[d] = L;
        a.nlev[d] = n_levels[d];
        L += n_levels[d];
    }
    a.w = w;
    a.V = V;
    a.m = m;
    a.N = N;
    a.status = status;
    return HDFE_OK;
}

inline unsigned grid_for(int64_t G)
{
    int64_t b = (G + kThreads - 1) / kThreads;
    if (b > kGrid) b = kGrid;
    return (unsigned)(b > 0 ? b : 1);
}

}  // namespace assemble
}  // namespace hdfe

using namespace hdfe;

extern "C" int64_t hdfe_assemble_workspace_bytes(int32_t m)
{
    if (m < 1 || m > assemble::kMaxM) return -1;
    return (int64_t)assemble::kGrid * (m * m > 7 ? m * m : 7) * 8;
}

extern "C" int hdfe_resid_moments(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                                  int32_t D, const int64_t *n_levels, const double *w,
                                  const double *V, int32_t m, int64_t n_rows,
                                  const double *Gamma, double *out, void *workspace,
                                  int64_t workspace_bytes, void *status, void *stream)
{
    assemble::Args a;
    int st = assemble::fill(a, starts, n_groups, codes, D, n_levels, w, V, m, n_rows,
                            (unsigned *)status);
    if (st != HDFE_OK) return st;
    if (!Gamma || !out || !workspace || workspace_bytes < hdfe_assemble_workspace_bytes(m))
        return hdfe_set_arg_error("hdfe_resid_moments: bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned grid = assemble::grid_for(n_groups);
    double *part = (double *)workspace;
    switch (m) {
    case 1: assemble::k_moments<1><<<grid, assemble::kThreads, 0, s>>>(a, Gamma, part); break;
    case 2: assemble::k_moments<2><<<grid, assemble::kThreads, 0, s>>>(a, Gamma, part); break;
    case 3: assemble::k_moments<3><<<grid, assemble::kThreads, 0, s>>>(a, Gamma, part); break;
    case 4: assemble::k_moments<4><<<grid, assemble::kThreads, 0, s>>>(a, Gamma, part); break;
    case 5: assemble::k_moments<5><<<grid, assemble::kThreads, 0, s>>>(a, Gamma, part); break;
    case 6: assemble::k_moments<6><<<grid, assemble::kThreads, 0, s>>>(a, Gamma, part); break;
    case 7: assemble::k_moments<7><<<grid, assemble::kThreads, 0, s>>>(a, Gamma, part); break;
    default: assemble::k_moments<8><<<grid, assemble::kThreads, 0, s>>>(a, Gamma, part); break;
    }
    assemble::k_sum_parts<<<(unsigned)((m * m * 32 + assemble::kThreads - 1) / assemble::kThreads),
                            assemble::kThreads, 0, s>>>(part, (int)grid, m * m, out);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(2);
    return HDFE_OK;
}

extern "C" int hdfe_row_effects(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                                int32_t D, const int64_t *n_levels, int32_t psi_column,
                                const double *w, const double *V, int32_t m, int64_t n_rows,
                                const double *beta, const double *gam_y, double *resid,
                                double *alpha, double *sums, void *workspace,
                                int64_t workspace_bytes, void *status, void *stream)
{
    assemble::Args a;
    int st = assemble::fill(a, starts, n_groups, codes, D, n_levels, w, V, m, n_rows,
                            (unsigned *)status);
    if (st != HDFE_OK) return st;
    if (psi_column < 0 || psi_column >= D || (m > 1 && !beta) || !gam_y || !sums ||
        !workspace || workspace_bytes < hdfe_assemble_workspace_bytes(m))
        return hdfe_set_arg_error("hdfe_row_effects: bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned grid = assemble::grid_for(n_groups);
    double *part = (double *)workspace;
#define HDFE_EFFECTS(M) assemble::k_effects<M><<<grid, assemble::kThreads, 0, s>>>( \
        a, psi_column, beta, gam_y, resid, alpha, part)
    switch (m) {
    case 1: HDFE_EFFECTS(1); break;
    case 2: HDFE_EFFECTS(2); break;
    case 3: HDFE_EFFECTS(3); break;
    case 4: HDFE_EFFECTS(4); break;
    case 5: HDFE_EFFECTS(5); break;
    case 6: HDFE_EFFECTS(6); break;
    case 7: HDFE_EFFECTS(7); break;
    default: HDFE_EFFECTS(8); break;
    }
#undef HDFE_EFFECTS
    assemble::k_sum_parts<<<(unsigned)((7 * 32 + assemble::kThreads - 1) / assemble::kThreads),
                            assemble::kThreads, 0, s>>>(part, (int)grid, 7, sums);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(2);
    return HDFE_OK;
}

extern "C" int hdfe_kss_sigma2(const double *y, const double *w, const double *resid,
                               const double *complement, const double *factor, double ybar,
                               int64_t n_rows, double *out, void *stream)
{
    if (!y || !resid || !complement || !factor || !out || n_rows < 0)
        return hdfe_set_arg_error("hdfe_kss_sigma2: bad argument");
    if (n_rows == 0) return HDFE_OK;
    int64_t b = (n_rows + assemble::kThreads - 1) / assemble::kThreads;
    if (b > 148 * 16) b = 148 * 16;
    assemble::k_sigma2<<<(unsigned)b, assemble::kThreads, 0, (cudaStream_t)stream>>>(
        y, w, resid, complement, factor, ybar, n_rows, out);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(1);
    return HDFE_OK;
}

extern "C" int64_t hdfe_variance_sums_workspace_bytes(int32_t m)
{
    if (m < 2 || m > assemble::kMaxM) return -1;
    const int kx = m - 1, nq = 3 * kx * (kx + 1) / 2 + 1;
    return (int64_t)assemble::kGrid * nq * 8;
}

extern "C" int hdfe_variance_sums(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                                  int32_t D, const int64_t *n_levels, const double *w,
                                  const double *V, int32_t m, int64_t n_rows,
                                  const double *Gamma, const double *beta, double *out,
                                  void *workspace, int64_t workspace_bytes, void *status,
                                  void *stream)
{
    assemble::Args a;
    int st = assemble::fill(a, starts, n_groups, codes, D, n_levels, w, V, m, n_rows,
                            (unsigned *)status);
    if (st != HDFE_OK) return st;
    if (m < 2 || !Gamma || !beta || !out || !workspace ||
        workspace_bytes < hdfe_variance_sums_workspace_bytes(m))
        return hdfe_set_arg_error("hdfe_variance_sums: bad argument (2 <= m <= 8)");
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned grid = assemble::grid_for(n_groups);
    double *part = (double *)workspace;
    const int kx = m - 1, nq = 3 * kx * (kx + 1) / 2 + 1;
#define HDFE_VARIANCE(M) assemble::k_variance<M><<<grid, assemble::kThreads, 0, s>>>( \
        a, Gamma, beta, part)
    switch (m) {
    case 2: HDFE_VARIANCE(2); break;
    case 3: HDFE_VARIANCE(3); break;
    case 4: HDFE_VARIANCE(4); break;
    case 5: HDFE_VARIANCE(5); break;
    case 6: HDFE_VARIANCE(6); break;
    case 7: HDFE_VARIANCE(7); break;
    default: HDFE_VARIANCE(8); break;
    }
#undef HDFE_VARIANCE
    assemble::k_sum_parts<<<(unsigned)((nq * 32 + assemble::kThreads - 1) / assemble::kThreads),
                            assemble::kThreads, 0, s>>>(part, (int)grid, nq, out);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(2);
    return HDFE_OK;
}

extern "C" int hdfe_row_scores(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                               int32_t D, const int64_t *n_levels, const double *w,
                               const double *V, int32_t m, int64_t n_rows, const double *Gamma,
                               const double *beta, double *out, double *h_out, void *status,
                               void *stream)
{
    assemble::Args a;
    int st = assemble::fill(a, starts, n_groups, codes, D, n_levels, w, V, m, n_rows,
                            (unsigned *)status);
    if (st != HDFE_OK) return st;
    if (m < 2 || !Gamma || !beta || !out)
        return hdfe_set_arg_error("hdfe_row_scores: bad argument (2 <= m <= 8)");
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned grid = assemble::grid_for(n_groups);
#define HDFE_SCORES(M) assemble::k_scores<M><<<grid, assemble::kThreads, 0, s>>>(a, Gamma, beta, out, \
                                                                                h_out)
    switch (m) {
    case 2: HDFE_SCORES(2); break;
    case 3: HDFE_SCORES(3); break;
    case 4: HDFE_SCORES(4); break;
    case 5: HDFE_SCORES(5); break;
    case 6: HDFE_SCORES(6); break;
    case 7: HDFE_SCORES(7); break;
    default: HDFE_SCORES(8); break;
    }
#undef HDFE_SCORES
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(1);
    return HDFE_OK;
}
