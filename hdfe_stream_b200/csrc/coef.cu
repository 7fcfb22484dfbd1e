// Coefficient-space passes of the inverse operator, and the trace moments.
//
// Reference: inverse.py:311-374 `apply_inverse` with kernels_inverse.py:
// 112-130 `_nb_reduce_rows`, :134-152 `_nb_spread_groups`, :157-188
// `_nb_project_coef`; the Hutchinson trace's collect sink (leaveout.py:
// 423-431, with core/kernels_groups.py:17-27 `_nb_group_sums`) and
// kernels_inverse.py:192-231 `_nb_trace_moments`; the coefficient-space
// Rademacher vectors of `_trace_block` (core/kernels_groups.py:53-76).
//
// One sub-warp of Bp lanes (Bp = the block width rounded up to 8, 16 or 32)
// per group of rows, lane j holding vector j:
//   reduce        acc[level, j] += w_i R_ij over the rows (no centring), where
//                 R is either explicit rows or the streamed block spread over
//                 its group (R_ij = streamed[g, j] / s_g, s_g = the group's
//                 weight); acc_x[c, j] += X_ic w_i R_ij; optionally the group
//                 sums of w_i R_ij.  Sums over a run of rows with equal codes
//                 are added once per run.
//   project_coef  h_ij = sum_d U[level_d(i), j] + X_i . C[:, j]; u0[g, j] =
//                 weighted group mean of (rho - h); rows (A u)_ij = h + u0 and
//                 the groups' u0; optionally the collect sink in the same pass:
//                 v = w_i omega_i (A u)_ij reduced like `reduce`.
//   trace         per vector j the eight weighted sums of the psi-dimension
//                 values (a) and streamed values (b) of Z and U over rows, per
//                 CTA in a fixed order and then over CTAs in a fixed order.
#include <cuda_runtime.h>

#include "common.cuh"

namespace hdfe {
namespace coef {

constexpr int kThreads = 128;
constexpr int kMaxCov = 8;
constexpr int kMaxGrid = 148 * 16;

struct Args {
    const int64_t *starts;
    int64_t G;
    const uint32_t *codes;
    int D;
    int64_t offs[HDFE_MAX_DIMS];
    int64_t nlev[HDFE_MAX_DIMS];
    int64_t L;
    const double *w;            // (N) or null (ones)
    const double *X;            // (N, c) or null
    int c;
    int B, Bp;
    const double *streamed;     // (G, B): spread over the rows, or null
    const double *R;            // (N, B) explicit rows (reduce), or null
    const double *U, *C;        // (L, B), (c, B)
    const double *omega;        // (N) or null: the collect sink's row weights (ones)
    bool collect;               // project_coef: run the collect sink
    double *rows;               // (N, B) or null
    double *groups;             // (G, B) or null
    double *acc, *acc_x;        // (L, B), (c, B): added into
    double *gsum;               // (G, B) or null
    unsigned *status;
};

template <int BP>
struct Lanes {
    int lane, j;
    unsigned mask;
    bool on;
    __device__ Lanes(int B)
    {
        lane = threadIdx.x & 31;
        j = lane % BP;
        const int sub = lane / BP;
        mask = BP == 32 ? 0xffffffffu : (((1u << BP) - 1u) << (sub * BP));
        on = j < B;
    }
};

// row i's codes, checked (an out-of-range code is reported and read as 0)
__device__ __forceinline__ void row_codes(const Args &a, int64_t i, uint32_t (&c)[HDFE_MAX_DIMS])
{
#pragma unroll
    for (int d = 0; d < HDFE_MAX_DIMS; d++) {
        if (d >= a.D) break;
        uint32_t v = __ldg(a.codes + i * a.D + d);
        if ((int64_t)v >= a.nlev[d]) {
            if (a.status) atomicCAS(a.status, 0u, (unsigned)HDFE_ERR_BAD_CODE);
            v = 0;
        }
        c[d] = v;
    }
}

__device__ __forceinline__ bool same(const Args &a, const uint32_t (&x)[HDFE_MAX_DIMS],
                                     const uint32_t (&y)[HDFE_MAX_DIMS])
{
    bool s = true;
#pragma unroll
    for (int d = 0; d < HDFE_MAX_DIMS; d++) {
        if (d >= a.D) break;
        s &= x[d] == y[d];
    }
    return s;
}

__device__ __forceinline__ double group_weight(const Args &a, int64_t s, int64_t e)
{
    double sw = 0.0;
    for (int64_t i = s; i < e; i++) sw += a.w ? __ldg(a.w + i) : 1.0;
    return sw;
}

// the run sums: v of consecutive rows with equal codes, added once per run
struct Runs {
    uint32_t codes[HDFE_MAX_DIMS];
    double v;
    bool have;
};

__device__ __forceinline__ void run_flush(const Args &a, const Runs &run, int j)
{
#pragma unroll
    for (int d = 0; d < HDFE_MAX_DIMS; d++) {
        if (d >= a.D) break;
        atomicAdd(a.acc + (a.offs[d] + run.codes[d]) * a.B + j, run.v);
    }
}

__device__ __forceinline__ void run_add(const Args &a, Runs &run, const uint32_t (&c)[HDFE_MAX_DIMS],
                                        double v, int j, bool on)
{
    if (run.have && !same(a, run.codes, c)) {
        if (on) run_flush(a, run, j);
        run.v = 0.0;
    }
#pragma unroll
    for (int d = 0; d < HDFE_MAX_DIMS; d++) {
        if (d >= a.D) break;
        run.codes[d] = c[d];
    }
    run.have = true;
    run.v += v;
}

// the covariate block: per thread, then per CTA, then one add per entry
__device__ __forceinline__ void flush_cov(const Args &a, const double (&ax)[kMaxCov], double *s_ax,
                                          int j, bool on)
{
    for (int k = threadIdx.x; k < a.c * a.B; k += kThreads) s_ax[k] = 0.0;
    __syncthreads();
    if (on) {
#pragma unroll
        for (int c = 0; c < kMaxCov; c++) {
            if (c >= a.c) break;
            atomicAdd(s_ax + c * a.B + j, ax[c]);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < a.c * a.B; k += kThreads)
        if (s_ax[k] != 0.0) atomicAdd(a.acc_x + k, s_ax[k]);
}

template <int BP>
__global__ void __launch_bounds__(kThreads) k_reduce(Args a)
{
    constexpr int SUBS = kThreads / BP;
    __shared__ double s_ax[kMaxCov * 32];
    const Lanes<BP> ln(a.B);
    const int64_t g0 = (int64_t)blockIdx.x * SUBS + threadIdx.x / BP;
    const int64_t gstep = (int64_t)gridDim.x * SUBS;
    double ax[kMaxCov];
#pragma unroll
    for (int c = 0; c < kMaxCov; c++) ax[c] = 0.0;
    for (int64_t g = g0; g < a.G; g += gstep) {
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        double rho = 0.0;
        if (a.streamed) {
            const double sw = group_weight(a, s, e);
            rho = (ln.on && sw > 0.0) ? a.streamed[g * a.B + ln.j] / sw : 0.0;
        }
        Runs run{};
        double gs = 0.0;
        for (int64_t i = s; i < e; i++) {
            uint32_t c[HDFE_MAX_DIMS];
            row_codes(a, i, c);
            const double wi = a.w ? __ldg(a.w + i) : 1.0;
            const double r = a.streamed ? rho : (ln.on ? a.R[i * a.B + ln.j] : 0.0);
            const double v = wi * r;
            run_add(a, run, c, v, ln.j, ln.on);
            gs += v;
#pragma unroll
            for (int cc = 0; cc < kMaxCov; cc++) {
                if (cc >= a.c) break;
                ax[cc] += __ldg(a.X + i * a.c + cc) * v;
            }
        }
        if (run.have && ln.on) run_flush(a, run, ln.j);
        if (a.gsum && ln.on) a.gsum[g * a.B + ln.j] = gs;
    }
    if (a.acc_x && a.c > 0) flush_cov(a, ax, s_ax, ln.j, ln.on);
}

template <int BP>
__global__ void __launch_bounds__(kThreads) k_project_coef(Args a)
{
    constexpr int SUBS = kThreads / BP;
    __shared__ double s_ax[kMaxCov * 32];
    __shared__ double s_C[kMaxCov * 32];
    const Lanes<BP> ln(a.B);
    for (int k = threadIdx.x; k < a.c * a.B; k += kThreads) s_C[k] = a.C[k];
    __syncthreads();
    const int64_t g0 = (int64_t)blockIdx.x * SUBS + threadIdx.x / BP;
    const int64_t gstep = (int64_t)gridDim.x * SUBS;
    double ax[kMaxCov];
#pragma unroll
    for (int c = 0; c < kMaxCov; c++) ax[c] = 0.0;
    auto h_of = [&](int64_t i, const uint32_t (&c)[HDFE_MAX_DIMS], double &hU, Runs &key) {
        // sum_d U[level_d(i), j], read again only when the codes change
        if (!key.have || !same(a, key.codes, c)) {
            hU = 0.0;
            if (ln.on) {
#pragma unroll
                for (int d = 0; d < HDFE_MAX_DIMS; d++) {
                    if (d >= a.D) break;
                    hU += a.U[(a.offs[d] + c[d]) * a.B + ln.j];
                }
            }
#pragma unroll
            for (int d = 0; d < HDFE_MAX_DIMS; d++) {
                if (d >= a.D) break;
                key.codes[d] = c[d];
            }
            key.have = true;
        }
        double h = hU;
        if (ln.on)
            for (int cc = 0; cc < a.c; cc++) h += __ldg(a.X + i * a.c + cc) * s_C[cc * a.B + ln.j];
        return h;
    };
    for (int64_t g = g0; g < a.G; g += gstep) {
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        const double sw = group_weight(a, s, e);
        const double rho = (a.streamed && ln.on && sw > 0.0) ? a.streamed[g * a.B + ln.j] / sw : 0.0;
        // pass 1: the group's mean of rho - h
        double tot = 0.0, hU = 0.0;
        Runs key{};
        for (int64_t i = s; i < e; i++) {
            uint32_t c[HDFE_MAX_DIMS];
            row_codes(a, i, c);
            const double wi = a.w ? __ldg(a.w + i) : 1.0;
            tot += wi * (rho - h_of(i, c, hU, key));
        }
        const double mean = sw > 0.0 ? tot / sw : 0.0;
        if (a.groups && ln.on) a.groups[g * a.B + ln.j] = mean;
        if (!a.rows && !a.collect) continue;
        // pass 2: the rows, and the collect sink
        key.have = false;
        Runs run{};
        double gs = 0.0;
        for (int64_t i = s; i < e; i++) {
            uint32_t c[HDFE_MAX_DIMS];
            row_codes(a, i, c);
            const double o = h_of(i, c, hU, key) + mean;
            if (a.rows && ln.on) a.rows[i * a.B + ln.j] = o;
            if (a.collect) {
                const double wi = a.w ? __ldg(a.w + i) : 1.0;
                const double v = wi * (a.omega ? __ldg(a.omega + i) : 1.0) * o;
                run_add(a, run, c, v, ln.j, ln.on);
                gs += v;
#pragma unroll
                for (int cc = 0; cc < kMaxCov; cc++) {
                    if (cc >= a.c) break;
                    ax[cc] += __ldg(a.X + i * a.c + cc) * v;
                }
            }
        }
        if (a.collect) {
            if (run.have && ln.on) run_flush(a, run, ln.j);
            if (a.gsum && ln.on) a.gsum[g * a.B + ln.j] = gs;
        }
    }
    if (a.collect && a.acc_x && a.c > 0) flush_cov(a, ax, s_ax, ln.j, ln.on);
}

// ---------------------------------------------------------- trace moments

struct TraceArgs {
    const int64_t *starts;
    int64_t G;
    const uint32_t *codes;
    int D, psi_column;
    int64_t psi_offset, psi_levels;
    const double *w;
    const double *Zl, *Zg, *Ul, *Ug;     // (L, B), (G, B), (L, B), (G, B)
    int B;
    double *partial;                     // (gridDim, B, 8)
    unsigned *status;
};

template <int BP>
__global__ void __launch_bounds__(kThreads) k_trace(TraceArgs a)
{
    constexpr int SUBS = kThreads / BP;
    __shared__ double s_m[SUBS][BP][8];
    const Lanes<BP> ln(a.B);
    const int sub = threadIdx.x / BP;
    const int64_t g0 = (int64_t)blockIdx.x * SUBS + sub;
    const int64_t gstep = (int64_t)gridDim.x * SUBS;
    double m[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t g = g0; g < a.G; g += gstep) {
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        const double b1 = ln.on ? a.Zg[g * a.B + ln.j] : 0.0;
        const double b2 = ln.on ? a.Ug[g * a.B + ln.j] : 0.0;
        uint32_t prev = 0xffffffffu;
        double a1 = 0.0, a2 = 0.0;
        for (int64_t i = s; i < e; i++) {
            uint32_t code = __ldg(a.codes + i * a.D + a.psi_column);
            if ((int64_t)code >= a.psi_levels) {
                if (a.status) atomicCAS(a.status, 0u, (unsigned)HDFE_ERR_BAD_CODE);
                code = 0;
            }
            if (code != prev) {
                prev = code;
                const int64_t lv = a.psi_offset + code;
                a1 = ln.on ? a.Zl[lv * a.B + ln.j] : 0.0;
                a2 = ln.on ? a.Ul[lv * a.B + ln.j] : 0.0;
            }
            const double wt = a.w ? __ldg(a.w + i) : 1.0;
            m[0] += wt;
            m[1] += wt * a1 * a2;
            m[2] += wt * b1 * b2;
            m[3] += wt * (a1 * b2 + b1 * a2);
            m[4] += wt * a1;
            m[5] += wt * a2;
            m[6] += wt * b1;
            m[7] += wt * b2;
        }
    }
#pragma unroll
    for (int k = 0; k < 8; k++) s_m[sub][ln.j][k] = m[k];
    __syncthreads();
    for (int t = threadIdx.x; t < a.B * 8; t += kThreads) {
        const int j = t / 8, k = t % 8;
        double sum = 0.0;
        for (int q = 0; q < SUBS; q++) sum += s_m[q][j][k];
        a.partial[((int64_t)blockIdx.x * a.B + j) * 8 + k] = sum;
    }
}

// out[j, k] = sum over CTAs of partial, one warp per entry, fixed order
__global__ void __launch_bounds__(kThreads) k_trace_reduce(const double *partial, int64_t blocks,
                                                           int B, double *out)
{
    const int lane = threadIdx.x & 31;
    const int64_t q = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
    if (q >= (int64_t)B * 8) return;
    double s = 0.0;
    for (int64_t b = lane; b < blocks; b += 32) s += partial[b * B * 8 + q];
    s = warp_sum(s);
    if (lane == 0) out[q] = s;
}

// ------------------------------------------------------- Rademacher draws

__global__ void __launch_bounds__(256) k_rademacher(double *out, int64_t n_rows, int64_t ordinal0,
                                                    int B, uint64_t seed, int64_t first_draw)
{
    const int64_t total = n_rows * B;
    for (int64_t t = (int64_t)blockIdx.x * 256 + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * 256) {
        const int64_t i = t / B, j = t % B;
        uint64_t x = seed ^ ((uint64_t)(ordinal0 + i) * 0x9E3779B97F4A7C15ull) ^
                     ((uint64_t)(first_draw + j) * 0xBF58476D1CE4E5B9ull);
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        x = x ^ (x >> 31);
        out[t] = (x >> 63) == 0 ? 1.0 : -1.0;
    }
}

int fill(Args &a, const int64_t *starts, int64_t G, const uint32_t *codes, int32_t D,
         const int64_t *n_levels, const double *w, const double *X, int32_t c, int32_t B,
         unsigned *status)
{
    if (D < 1 || D > HDFE_MAX_DIMS || G < 0 || !starts || !codes || !n_levels || B < 1 ||
        B > 32 || c < 0 || c > kMaxCov || (c > 0 && !X))
        return hdfe_set_arg_error("hdfe_rows_reduce/project_coef: bad argument");
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
    a.B = B;
    a.Bp = B <= 8 ? 8 : (B <= 16 ? 16 : 32);
    a.status = status;
    return HDFE_OK;
}

inline unsigned grid_for(int64_t G, int Bp)
{
    const int64_t per = kThreads / Bp;
    int64_t b = (G + per - 1) / per;
    if (b > kMaxGrid) b = kMaxGrid;
    return (unsigned)(b > 0 ? b : 1);
}

}  // namespace coef
}  // namespace hdfe

using namespace hdfe;

extern "C" int hdfe_rows_reduce(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                                int32_t D, const int64_t *n_levels, const double *w,
                                const double *X, int32_t c, const double *streamed,
                                const double *R, int32_t B, double *acc, double *acc_x,
                                double *group_sums, void *status, void *stream)
{
    coef::Args a;
    int st = coef::fill(a, starts, n_groups, codes, D, n_levels, w, X, c, B, (unsigned *)status);
    if (st != HDFE_OK) return st;
    if ((streamed == nullptr) == (R == nullptr) || !acc || (c > 0 && !acc_x) ||
        (group_sums && streamed))
        return hdfe_set_arg_error("hdfe_rows_reduce: give exactly one of streamed and R "
                                  "(group sums with R only)");
    a.streamed = streamed;
    a.R = R;
    a.acc = acc;
    a.acc_x = acc_x;
    a.gsum = group_sums;
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned grid = coef::grid_for(n_groups, a.Bp);
    if (a.Bp == 8) coef::k_reduce<8><<<grid, coef::kThreads, 0, s>>>(a);
    else if (a.Bp == 16) coef::k_reduce<16><<<grid, coef::kThreads, 0, s>>>(a);
    else coef::k_reduce<32><<<grid, coef::kThreads, 0, s>>>(a);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(1);
    return HDFE_OK;
}

extern "C" int hdfe_rows_project_coef(const int64_t *starts, int64_t n_groups,
                                      const uint32_t *codes, int32_t D, const int64_t *n_levels,
                                      const double *w, const double *X, int32_t c,
                                      const double *C, const double *U, const double *streamed,
                                      int32_t B, double *rows, double *groups,
                                      const double *omega, double *acc, double *acc_x,
                                      double *group_sums, void *status, void *stream)
{
    coef::Args a;
    int st = coef::fill(a, starts, n_groups, codes, D, n_levels, w, X, c, B, (unsigned *)status);
    if (st != HDFE_OK) return st;
    if (!U || (c > 0 && !C) || (omega && (!acc || (c > 0 && !acc_x))))
        return hdfe_set_arg_error("hdfe_rows_project_coef: bad argument");
    a.U = U;
    a.C = C;
    a.streamed = streamed;
    a.rows = rows;
    a.groups = groups;
    a.omega = omega;
    a.collect = omega != nullptr;
    a.acc = acc;
    a.acc_x = acc_x;
    a.gsum = group_sums;
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned grid = coef::grid_for(n_groups, a.Bp);
    if (a.Bp == 8) coef::k_project_coef<8><<<grid, coef::kThreads, 0, s>>>(a);
    else if (a.Bp == 16) coef::k_project_coef<16><<<grid, coef::kThreads, 0, s>>>(a);
    else coef::k_project_coef<32><<<grid, coef::kThreads, 0, s>>>(a);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(1);
    return HDFE_OK;
}

extern "C" int64_t hdfe_trace_moments_workspace_bytes(int32_t B)
{
    if (B < 1 || B > 32) return -1;
    return (int64_t)coef::kMaxGrid * B * 8 * 8;
}

extern "C" int hdfe_trace_moments(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                                  int32_t D, const int64_t *n_levels, int32_t psi_column,
                                  const double *w, const double *Z_levels,
                                  const double *Z_groups, const double *U_levels,
                                  const double *U_groups, int32_t B, double *out,
                                  void *workspace, int64_t workspace_bytes, void *status,
                                  void *stream)
{
    if (D < 1 || D > HDFE_MAX_DIMS || psi_column < 0 || psi_column >= D || n_groups < 0 ||
        !starts || !codes || !n_levels || !Z_levels || !Z_groups || !U_levels || !U_groups ||
        !out || B < 1 || B > 32 || !workspace)
        return hdfe_set_arg_error("hdfe_trace_moments: bad argument");
    if (workspace_bytes < hdfe_trace_moments_workspace_bytes(B))
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_trace_moments: workspace too small");
    coef::TraceArgs a{};
    a.starts = starts;
    a.G = n_groups;
    a.codes = codes;
    a.D = D;
    a.psi_column = psi_column;
    int64_t off = 0;
    for (int d = 0; d < psi_column; d++) off += n_levels[d];
    a.psi_offset = off;
    a.psi_levels = n_levels[psi_column];
    a.w = w;
    a.Zl = Z_levels;
    a.Zg = Z_groups;
    a.Ul = U_levels;
    a.Ug = U_groups;
    a.B = B;
    a.partial = (double *)workspace;
    a.status = (unsigned *)status;
    cudaStream_t s = (cudaStream_t)stream;
    const int Bp = B <= 8 ? 8 : (B <= 16 ? 16 : 32);
    const unsigned grid = coef::grid_for(n_groups, Bp);
    if (Bp == 8) coef::k_trace<8><<<grid, coef::kThreads, 0, s>>>(a);
    else if (Bp == 16) coef::k_trace<16><<<grid, coef::kThreads, 0, s>>>(a);
    else coef::k_trace<32><<<grid, coef::kThreads, 0, s>>>(a);
    coef::k_trace_reduce<<<(unsigned)((B * 8 * 32 + coef::kThreads - 1) / coef::kThreads),
                           coef::kThreads, 0, s>>>(a.partial, grid, B, out);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(2);
    return HDFE_OK;
}

extern "C" int hdfe_rademacher(double *out, int64_t n_rows, int64_t ordinal0, int32_t B,
                               uint64_t seed, int64_t first_draw, void *stream)
{
    if (!out || n_rows < 0 || B < 1) return hdfe_set_arg_error("hdfe_rademacher: bad argument");
    if (n_rows == 0) return HDFE_OK;
    int64_t blocks = (n_rows * B + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    coef::k_rademacher<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(out, n_rows, ordinal0,
                                                                          B, seed, first_draw);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(1);
    return HDFE_OK;
}

// (D_o' M_0 D_o) P from the identifying cells, without S: per group the
// n-weighted mean of h_i = sum_d P[level_d(i)] is taken off, and
// n_i (h_i - mean) is added to each of cell i's levels -- the projection pass
// with U = P, no streamed block, weights n and the collect sink's unit weights
// (core/kernels_base.py:478-507 `_nb_stream_matvec`).
extern "C" int hdfe_stream_matvec(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                                  int32_t D, const int64_t *n_levels, const double *n,
                                  const double *P, int32_t k, double *out, void *status,
                                  void *stream)
{
    coef::Args a;
    int st = coef::fill(a, starts, n_groups, codes, D, n_levels, n, nullptr, 0, k,
                        (unsigned *)status);
    if (st != HDFE_OK) return st;
    if (!n || !P || !out) return hdfe_set_arg_error("hdfe_stream_matvec: bad argument");
    a.U = P;
    a.collect = true;
    a.acc = out;
    cudaStream_t s = (cudaStream_t)stream;
    HDFE_CUDA_TRY(cudaMemsetAsync(out, 0, a.L * k * 8, s));
    const unsigned grid = coef::grid_for(n_groups, a.Bp);
    if (a.Bp == 8) coef::k_project_coef<8><<<grid, coef::kThreads, 0, s>>>(a);
    else if (a.Bp == 16) coef::k_project_coef<16><<<grid, coef::kThreads, 0, s>>>(a);
    else coef::k_project_coef<32><<<grid, coef::kThreads, 0, s>>>(a);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(1);
    return HDFE_OK;
}
