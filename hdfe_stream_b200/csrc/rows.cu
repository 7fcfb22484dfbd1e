// Row passes of the inverse operator A S^- A' (the leave-out machinery).
//
// Reference: inverse.py:240-309 `project_rows` with kernels_inverse.py:35-71
// `_nb_center_rows` and :75-107 `_nb_project_rows`, the counter-based draws
// of core/kernels_groups.py:53-76 `_nb_rademacher`, and the JLA sink and
// moment combination of leaveout.py:181-190 and :210-282.
//
// The vectors being projected are Rademacher draws regenerated from (seed,
// row ordinal, draw index) by splitmix64 in registers -- bit-identical to
// `_nb_rademacher`, never stored -- or explicit row vectors (the covariates
// themselves, for the Schur border).  Rows come grouped by the streamed
// dimension; a sub-warp of Bp lanes (Bp = the draw count rounded up to 8, 16
// or 32) takes one group, lane j one draw, so every group mean and scatter is
// a per-lane loop over the group's rows:
//   center   acc[level, j] += w_i (R_ij - Rbar_gj)  over the group's rows, for
//            each non-streamed dimension; acc_x[c, j] += X_ic w_i (R_ij -
//            Rbar_gj); sum w R^2 per draw.  Levels of small dimensions are
//            accumulated in shared memory per CTA.
//   project  h_ij = sum_d U[level_d(i), j] + X_i . C[:, j]; Ubar = weighted
//            group mean of (R - h); out_ij = h_ij + Ubar (times sqrt(w_i) in
//            the square-root weight metric), and the JLA sink's five running
//            sums per row: P = out^2, M = (r - out)^2, P^2, M^2, P M, summed
//            over the block's draws in draw order.
#include <cuda_runtime.h>

#include "common.cuh"

namespace hdfe {
namespace rows {

constexpr int kThreads = 256;
constexpr int kMaxCov = 8;

__device__ __forceinline__ double rademacher(uint64_t seed, int64_t row, int64_t draw)
{
    uint64_t x = seed ^ ((uint64_t)row * 0x9E3779B97F4A7C15ull) ^
                 ((uint64_t)draw * 0xBF58476D1CE4E5B9ull);
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    x = x ^ (x >> 31);
    return (x >> 63) == 0 ? 1.0 : -1.0;
}

struct Args {
    const int64_t *starts;      // (G+1) row boundaries of the groups
    int64_t G;
    const uint32_t *codes;      // (N, D)
    int D;
    int64_t offs[HDFE_MAX_DIMS];
    int64_t nlev[HDFE_MAX_DIMS];
    int small[HDFE_MAX_DIMS];
    int64_t soff[HDFE_MAX_DIMS];
    int64_t n_small;
    int64_t L;
    const double *w;            // (N) or null (ones)
    const double *X;            // (N, c) covariates or null
    int c;
    const double *R;            // (N, B) explicit vectors, or null: Rademacher
    uint64_t seed;
    int64_t first_draw, ordinal0;
    int B, Bp;
    int sqrt_weights;
    // center
    double *acc, *acc_x, *squares;
    // project
    const double *U, *C;        // (L, B), (c, B)
    double *out;                // (N, B) or null
    double *moments;            // (5, N) or null
    int64_t N;
    unsigned *status;
};

__device__ __forceinline__ double row_vec(const Args &a, int64_t i, int j)
{
    if (a.R) return a.R[i * a.B + j];
    return rademacher(a.seed, a.ordinal0 + i, a.first_draw + j);
}

// the weight metric: the vectors enter scaled by w^(-1/2) (inverse.py:280-281)
__device__ __forceinline__ double inv_root(const Args &a, double wi)
{
    if (!a.sqrt_weights) return 1.0;
    const double r = sqrt(wi);
    return r > 0.0 ? 1.0 / r : 0.0;
}

__global__ void __launch_bounds__(kThreads) k_center(Args a)
{
    extern __shared__ double s_acc[];
    const int lane = threadIdx.x & 31;
    const int j = lane % a.Bp, sub = lane / a.Bp, per_warp = 32 / a.Bp;
    const int64_t nsm = a.n_small * a.B;
    for (int64_t k = threadIdx.x; k < nsm; k += kThreads) s_acc[k] = 0.0;
    __syncthreads();
    const bool on = j < a.B;
    double sq = 0.0;
    double ax[kMaxCov];
    for (int c = 0; c < a.c; c++) ax[c] = 0.0;
    const int64_t gsub = ((int64_t)blockIdx.x * kThreads + threadIdx.x) / 32 * per_warp + sub;
    const int64_t nsub = (int64_t)gridDim.x * kThreads / 32 * per_warp;
    for (int64_t g = gsub; g < a.G; g += nsub) {
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        double sw = 0.0, tot = 0.0;
        for (int64_t i = s; i < e; i++) {
            const double wi = a.w ? a.w[i] : 1.0;
            sw += wi;
            if (on) {
                const double r = row_vec(a, i, j) * inv_root(a, wi);
                tot += wi * r;
                sq += wi * r * r;
            }
        }
        if (!(sw > 0.0) || !on) continue;
        const double mean = tot / sw;
        for (int64_t i = s; i < e; i++) {
            const double wi = a.w ? a.w[i] : 1.0;
            const double r = row_vec(a, i, j) * inv_root(a, wi);
            const double v = wi * (r - mean);
            for (int d = 0; d < a.D; d++) {
                uint32_t code = a.codes[i * a.D + d];
                if ((int64_t)code >= a.nlev[d]) { atomicCAS(a.status, 0u, (unsigned)HDFE_ERR_BAD_CODE); code = 0; }
                if (a.small[d]) atomicAdd(s_acc + (a.soff[d] + code) * a.B + j, v);
                else atomicAdd(a.acc + (a.offs[d] + code) * a.B + j, v);
            }
            for (int c = 0; c < a.c; c++) ax[c] += a.X[i * a.c + c] * v;
        }
    }
    // the covariate block and the sums of squares: per lane, then per CTA
    if (a.acc_x && j < a.B)
        for (int c = 0; c < a.c; c++) atomicAdd(a.acc_x + c * a.B + j, ax[c]);
    if (a.squares && j < a.B) atomicAdd(a.squares + j, sq);
    __syncthreads();
    for (int d = 0; d < a.D; d++) {
        if (!a.small[d]) continue;
        for (int64_t q = threadIdx.x; q < a.nlev[d] * a.B; q += kThreads) {
            const double v = s_acc[a.soff[d] * a.B + q];
            if (v != 0.0) atomicAdd(a.acc + a.offs[d] * a.B + q, v);
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_project(Args a)
{
    const int lane = threadIdx.x & 31;
    const int j = lane % a.Bp, sub = lane / a.Bp, per_warp = 32 / a.Bp;
    const bool on = j < a.B;
    const unsigned smask = a.Bp == 32 ? 0xffffffffu : (((1u << a.Bp) - 1u) << (sub * a.Bp));
    double Cj[kMaxCov];
    for (int c = 0; c < a.c; c++) Cj[c] = on ? a.C[c * a.B + j] : 0.0;
    const int64_t gsub = ((int64_t)blockIdx.x * kThreads + threadIdx.x) / 32 * per_warp + sub;
    const int64_t nsub = (int64_t)gridDim.x * kThreads / 32 * per_warp;
    // the sub-warp loops over groups; per_warp sub-warps of a warp run the same
    // trip count so their shuffles stay converged (idle ones take g = -1)
    const int64_t rounds = (a.G + nsub - 1) / nsub;
    for (int64_t t = 0; t < rounds; t++) {
        const int64_t g = gsub + t * nsub;
        const bool live = g < a.G;
        const int64_t s = live ? a.starts[g] : 0, e = live ? a.starts[g + 1] : 0;
        double sw = 0.0, tot = 0.0;
        for (int64_t i = s; i < e; i++) {
            const double wi = a.w ? a.w[i] : 1.0;
            sw += wi;
            if (!on) continue;
            double h = 0.0;
            for (int d = 0; d < a.D; d++) {
                uint32_t code = a.codes[i * a.D + d];
                if ((int64_t)code >= a.nlev[d]) code = 0;
                h += a.U[(a.offs[d] + code) * a.B + j];
            }
            for (int c = 0; c < a.c; c++) h += a.X[i * a.c + c] * Cj[c];
            const double r = row_vec(a, i, j) * inv_root(a, wi);
            tot += wi * (r - h);
        }
        const double mean = sw > 0.0 ? tot / sw : 0.0;
        // the group's rows again: the projection, and the sink
        const int64_t n = e - s;
        for (int64_t ii = 0; ii < n; ii++) {
            const int64_t i = s + ii;
            const double wi = a.w ? a.w[i] : 1.0;
            double o = 0.0, pp = 0.0, mm = 0.0;
            if (on) {
                double h = 0.0;
                for (int d = 0; d < a.D; d++) {
                    uint32_t code = a.codes[i * a.D + d];
                    if ((int64_t)code >= a.nlev[d]) code = 0;
                    h += a.U[(a.offs[d] + code) * a.B + j];
                }
                for (int c = 0; c < a.c; c++) h += a.X[i * a.c + c] * Cj[c];
                o = h + mean;
                if (a.sqrt_weights) o *= sqrt(wi);
                if (a.out) a.out[i * a.B + j] = o;
                const double rr = row_vec(a, i, j);     // the sink's unscaled draw
                pp = o * o;
                mm = (rr - o) * (rr - o);
            }
            if (a.moments) {
                // the five sums over the block's draws, in draw order
                double m0 = pp, m1 = mm, m2 = pp * pp, m3 = mm * mm, m4 = pp * mm;
                for (int q = 1; q < a.Bp; q <<= 1) {
                    m0 += __shfl_down_sync(smask, m0, q, a.Bp);
                    m1 += __shfl_down_sync(smask, m1, q, a.Bp);
                    m2 += __shfl_down_sync(smask, m2, q, a.Bp);
                    m3 += __shfl_down_sync(smask, m3, q, a.Bp);
                    m4 += __shfl_down_sync(smask, m4, q, a.Bp);
                }
                if (j == 0) {
                    a.moments[0 * a.N + i] += m0;
                    a.moments[1 * a.N + i] += m1;
                    a.moments[2 * a.N + i] += m2;
                    a.moments[3 * a.N + i] += m3;
                    a.moments[4 * a.N + i] += m4;
                }
            }
        }
    }
}

// JLA leverages from the five running sums (leaveout.py:210-282), in place:
// slot 0 <- Pbar, slot 1 <- Mbar = 1 - Pbar, slot 2 <- the factor.
__global__ void __launch_bounds__(kThreads) k_jla_combine(double *mom, int64_t N, double n_draws)
{
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < N;
         i += (int64_t)gridDim.x * kThreads) {
        const double P = mom[i] / n_draws, M = mom[N + i] / n_draws;
        const double mPP = mom[2 * N + i] / n_draws, mMM = mom[3 * N + i] / n_draws;
        const double mPM = mom[4 * N + i] / n_draws;
        const double total = P + M;
        const double Pb = total > 0.0 ? P / total : 0.0;
        const double Mb = 1.0 - Pb;
        const double V = (Mb * Mb * mPP + Pb * Pb * mMM - 2.0 * Pb * Mb * mPM) / n_draws;
        const double Bb = (Mb * mPP - Pb * mMM + (Mb - Pb) * mPM) / n_draws;
        double factor = 1.0;
        if (Mb > 0.0) factor = 1.0 - V / (Mb * Mb) + Bb / Mb;
        mom[i] = Pb;
        mom[N + i] = Mb;
        mom[2 * N + i] = factor;
    }
}

// group boundaries of rows sorted by gcode: flags, then compaction by tiles
constexpr int kTile = 4096;

__global__ void __launch_bounds__(kThreads) k_group_count(const uint32_t *gcode, int64_t N,
                                                          int64_t *tiles)
{
    __shared__ double s_red[kThreads / 32];
    const int64_t t0 = (int64_t)blockIdx.x * kTile, t1 = min(t0 + kTile, N);
    int c = 0;
    for (int64_t i = t0 + threadIdx.x; i < t1; i += kThreads)
        c += (i == 0 || gcode[i] != gcode[i - 1]);
    const double t = block_sum((double)c, s_red);
    if (threadIdx.x == 0) tiles[blockIdx.x] = (int64_t)t;
}

__global__ void k_group_scan(int64_t *tiles, int64_t nt, int64_t *total)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int64_t run = 0;
    for (int64_t b = 0; b < nt; b++) { const int64_t v = tiles[b]; tiles[b] = run; run += v; }
    *total = run;
}

__global__ void __launch_bounds__(kThreads) k_group_write(const uint32_t *gcode, int64_t N,
                                                          const int64_t *tiles, int64_t *starts,
                                                          const int64_t *total)
{
    __shared__ int s_w[kThreads / 32 + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t t0 = (int64_t)blockIdx.x * kTile, t1 = min(t0 + kTile, N);
    int64_t run = tiles[blockIdx.x];
    for (int64_t base = t0; base < t1; base += kThreads) {
        const int64_t i = base + threadIdx.x;
        const bool f = i < t1 && (i == 0 || gcode[i] != gcode[i - 1]);
        const unsigned m = __ballot_sync(0xffffffffu, f);
        if (lane == 0) s_w[warp] = __popc(m);
        __syncthreads();
        if (threadIdx.x == 0) {
            int r = 0;
            for (int k = 0; k < kThreads / 32; k++) { const int t = s_w[k]; s_w[k] = r; r += t; }
            s_w[kThreads / 32] = r;
        }
        __syncthreads();
        if (f) starts[run + s_w[warp] + __popc(m & ((1u << lane) - 1))] = i;
        run += s_w[kThreads / 32];
        __syncthreads();
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) starts[*total] = N;
}

int fill_args(Args &a, const int64_t *starts, int64_t G, const uint32_t *codes, int32_t D,
              const int64_t *n_levels, const double *w, const double *X, int32_t c,
              const double *R, int32_t B, uint64_t seed, int64_t first_draw, int64_t ordinal0,
              int32_t sqrt_weights, unsigned *status)
{
    if (D < 1 || D > HDFE_MAX_DIMS || G < 0 || !starts || !codes || !n_levels || B < 1 || B > 32 ||
        c < 0 || c > kMaxCov || (c > 0 && !X))
        return hdfe_set_arg_error("hdfe_rows: bad argument");
    a = Args{};
    a.starts = starts;
    a.G = G;
    a.codes = codes;
    a.D = D;
    int64_t L = 0;
    for (int d = 0; d < D; d++) {
        if (n_levels[d] < 1) return hdfe_set_arg_error("hdfe_rows: n_levels must be >= 1");
        a.offs[d] = L;
        a.nlev[d] = n_levels[d];
        L += n_levels[d];
    }
    a.L = L;
    a.w = w;
    a.X = X;
    a.c = c;
    a.R = R;
    a.seed = seed;
    a.first_draw = first_draw;
    a.ordinal0 = ordinal0;
    a.B = B;
    a.Bp = B <= 8 ? 8 : (B <= 16 ? 16 : 32);
    a.sqrt_weights = sqrt_weights;
    a.status = status;
    return HDFE_OK;
}

inline unsigned grid_for(int64_t G, int Bp)
{
    const int64_t groups_per_cta = (int64_t)kThreads / 32 * (32 / Bp);
    int64_t b = (G + groups_per_cta - 1) / groups_per_cta;
    if (b > 148 * 16) b = 148 * 16;
    return (unsigned)(b > 0 ? b : 1);
}

}  // namespace rows
}  // namespace hdfe

using namespace hdfe;

extern "C" int64_t hdfe_row_groups_workspace_bytes(int64_t n_rows)
{
    return ((n_rows + rows::kTile - 1) / rows::kTile + 2) * 8 + 256;
}

extern "C" int hdfe_row_groups(const uint32_t *gcode, int64_t n_rows, int64_t *starts,
                               int64_t *n_groups, void *workspace, int64_t workspace_bytes,
                               void *stream)
{
    if (!gcode || n_rows < 1 || !starts || !n_groups || !workspace ||
        workspace_bytes < hdfe_row_groups_workspace_bytes(n_rows))
        return hdfe_set_arg_error("hdfe_row_groups: bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t nt = (n_rows + rows::kTile - 1) / rows::kTile;
    int64_t *tiles = (int64_t *)workspace;
    rows::k_group_count<<<(unsigned)nt, rows::kThreads, 0, s>>>(gcode, n_rows, tiles);
    rows::k_group_scan<<<1, 32, 0, s>>>(tiles, nt, n_groups);
    rows::k_group_write<<<(unsigned)nt, rows::kThreads, 0, s>>>(gcode, n_rows, tiles, starts,
                                                                 n_groups);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(3);
    return HDFE_OK;
}

extern "C" int hdfe_rows_center(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                                int32_t D, const int64_t *n_levels, const double *w,
                                const double *X, int32_t c, const double *R, int32_t B,
                                uint64_t seed, int64_t first_draw, int64_t ordinal0,
                                int32_t sqrt_weights, double *acc, double *acc_x,
                                double *squares, void *workspace, int64_t workspace_bytes,
                                void *stream)
{
    rows::Args a;
    if (!workspace || workspace_bytes < 256) return hdfe_set_arg_error("hdfe_rows_center: workspace");
    int st = rows::fill_args(a, starts, n_groups, codes, D, n_levels, w, X, c, R, B, seed,
                             first_draw, ordinal0, sqrt_weights, (unsigned *)workspace);
    if (st != HDFE_OK) return st;
    if (!acc || (c > 0 && !acc_x)) return hdfe_set_arg_error("hdfe_rows_center: null output");
    a.acc = acc;
    a.acc_x = acc_x;
    a.squares = squares;
    // small dimensions in shared memory (up to 40 KB of level x draw sums)
    int64_t slots = 0;
    for (int d = 0; d < D; d++) {
        if ((slots + n_levels[d]) * B * 8 <= 40 * 1024 && n_levels[d] <= 4096) {
            a.small[d] = 1;
            a.soff[d] = slots;
            slots += n_levels[d];
        }
    }
    a.n_small = slots;
    cudaStream_t s = (cudaStream_t)stream;
    HDFE_CUDA_TRY(cudaMemsetAsync(workspace, 0, 8, s));
    HDFE_CUDA_TRY(cudaMemsetAsync(acc, 0, a.L * B * 8, s));
    if (c > 0) HDFE_CUDA_TRY(cudaMemsetAsync(acc_x, 0, (int64_t)c * B * 8, s));
    if (squares) HDFE_CUDA_TRY(cudaMemsetAsync(squares, 0, B * 8, s));
    rows::k_center<<<rows::grid_for(n_groups, a.Bp), rows::kThreads, slots * B * 8, s>>>(a);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(1);
    return HDFE_OK;
}

extern "C" int hdfe_rows_project(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                                 int32_t D, const int64_t *n_levels, const double *w,
                                 const double *X, int32_t c, const double *C, const double *U,
                                 const double *R, int32_t B, uint64_t seed, int64_t first_draw,
                                 int64_t ordinal0, int32_t sqrt_weights, int64_t n_rows,
                                 double *out, double *moments, void *stream)
{
    rows::Args a;
    int st = rows::fill_args(a, starts, n_groups, codes, D, n_levels, w, X, c, R, B, seed,
                             first_draw, ordinal0, sqrt_weights, nullptr);
    if (st != HDFE_OK) return st;
    if (!U || (c > 0 && !C) || (!out && !moments) || n_rows < 0)
        return hdfe_set_arg_error("hdfe_rows_project: bad argument");
    a.U = U;
    a.C = C;
    a.out = out;
    a.moments = moments;
    a.N = n_rows;
    cudaStream_t s = (cudaStream_t)stream;
    rows::k_project<<<rows::grid_for(n_groups, a.Bp), rows::kThreads, 0, s>>>(a);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(1);
    return HDFE_OK;
}

extern "C" int hdfe_jla_combine(double *moments, int64_t n_rows, int64_t n_draws, void *stream)
{
    if (!moments || n_rows < 0 || n_draws < 1) return hdfe_set_arg_error("hdfe_jla_combine: bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    int64_t b = (n_rows + rows::kThreads - 1) / rows::kThreads;
    if (b > 4096) b = 4096;
    rows::k_jla_combine<<<(unsigned)(b > 0 ? b : 1), rows::kThreads, 0, s>>>(moments, n_rows,
                                                                            (double)n_draws);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(1);
    return HDFE_OK;
}
