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
// or 32) takes one group, lane j one draw.  The group's rows are staged 32 at
// a time in shared memory (codes, covariates; weights in registers), loaded
// lane-parallel; the draws' signs of a group's first chunk are kept as bits
// between its two passes.
//   center   acc[level, j] += w_i (R_ij - Rbar_gj)  over the group's rows, for
//            each non-streamed dimension, summed over each run of rows with
//            equal codes and added once per run; acc_x[c, j] += X_ic w_i (R_ij
//            - Rbar_gj); sum w R^2 per draw.  Levels of small dimensions are
//            accumulated in shared memory per CTA.
//   project  h_ij = sum_d U[level_d(i), j] (read once per run) + X_i . C[:, j];
//            Ubar = weighted group mean of (R - h); out_ij = h_ij + Ubar
//            (times sqrt(w_i) in the square-root weight metric), and the JLA
//            sink's five running sums per row: P = out^2, M = (r - out)^2, P^2,
//            M^2, P M, summed over the block's draws in draw order (through a
//            shared-memory transpose: lane t sums row t).
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

// The sign of `rademacher` from precomputed row and draw terms: the last
// step of splitmix64 (x ^= x >> 31) leaves bit 63 alone, so the draw is -1
// exactly when bit 63 is set before it.
__device__ __forceinline__ bool rad_negative(uint64_t seed, uint64_t rterm, uint64_t dterm)
{
    uint64_t x = seed ^ rterm ^ dterm;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return (x >> 63) != 0;
}

constexpr uint64_t kRowMul = 0x9E3779B97F4A7C15ull, kDrawMul = 0xBF58476D1CE4E5B9ull;
constexpr int kPassThreads = 128;

// Per sub-warp staging of a chunk of up to BP rows: codes (BP x D) and
// covariates (BP x c), loaded lane-parallel (lane t: row i0 + t) and read by
// every lane from shared memory; the weights stay in registers (shuffled).
template <int BP>
struct Chunk {
    static constexpr int kBytes = BP * (HDFE_MAX_DIMS * 4 + kMaxCov * 8);
    uint32_t *codes;    // [BP][D]
    double *x;          // [BP][c]
};

// a sub-warp of BP lanes: lane j holds draw j of the block (on: j < B)
template <int BP>
struct Lanes {
    int lane, j, sub;
    unsigned mask;
    bool on;
    __device__ Lanes(int B)
    {
        lane = threadIdx.x & 31;
        j = lane % BP;
        sub = lane / BP;
        mask = BP == 32 ? 0xffffffffu : (((1u << BP) - 1u) << (sub * BP));
        on = j < B;
    }
};

// Load rows [i0, i0 + n) of the group into the chunk (lane t: row i0 + t):
// codes (checked: an out-of-range code is reported and read as 0) and
// covariates; returns this lane's row weight (1 without weights).
template <int BP>
__device__ __forceinline__ double load_chunk(const Args &a, const Lanes<BP> &ln, Chunk<BP> &ch,
                                             int64_t i0, int n)
{
    double w = 1.0;
    if (ln.j < n) {
        const int64_t i = i0 + ln.j;
        if (a.w) w = a.w[i];
        for (int d = 0; d < a.D; d++) {
            uint32_t code = a.codes[i * a.D + d];
            if ((int64_t)code >= a.nlev[d]) {
                if (a.status) atomicCAS(a.status, 0u, (unsigned)HDFE_ERR_BAD_CODE);
                code = 0;
            }
            ch.codes[ln.j * a.D + d] = code;
        }
        for (int c = 0; c < a.c; c++) ch.x[ln.j * a.c + c] = a.X[i * a.c + c];
    }
    __syncwarp(ln.mask);
    return w;
}

// codes of chunk row q equal to the previous row's (prev)
__device__ __forceinline__ bool same_codes(const Args &a, const uint32_t *codes, int q,
                                           const uint32_t (&prev)[HDFE_MAX_DIMS])
{
    bool same = true;
#pragma unroll
    for (int d = 0; d < HDFE_MAX_DIMS; d++) {
        if (d >= a.D) break;
        same &= codes[q * a.D + d] == prev[d];
    }
    return same;
}

__device__ __forceinline__ void take_codes(const Args &a, const uint32_t *codes, int q,
                                           uint32_t (&prev)[HDFE_MAX_DIMS])
{
#pragma unroll
    for (int d = 0; d < HDFE_MAX_DIMS; d++) {
        if (d >= a.D) break;
        prev[d] = codes[q * a.D + d];
    }
}

__device__ __forceinline__ double inv_root(const Args &a, double w)
{
    return a.sqrt_weights ? (w > 0.0 ? 1.0 / sqrt(w) : 0.0) : 1.0;
}

// `_nb_center_rows` for one sub-warp of BP lanes per group (lane j: draw j).
// Pass 1 over the group's rows: sum w, sum w r, sum w r^2, with the draws'
// signs kept as bits for the group's first chunk; pass 2: v = w (r - mean)
// summed over each run of rows with equal codes and added once per run to
// every dimension's level (shared-memory copies for small dimensions), and
// the covariate block per row.
template <int BP>
__global__ void __launch_bounds__(kPassThreads) k_center(Args a)
{
    extern __shared__ double s_dyn[];
    constexpr int SUBS = kPassThreads / BP;
    double *s_acc = s_dyn;                                          // small dimensions
    char *s_chunks = reinterpret_cast<char *>(s_dyn + a.n_small * a.B);
    const Lanes<BP> ln(a.B);
    const int subw = threadIdx.x / BP;
    Chunk<BP> ch;
    ch.codes = reinterpret_cast<uint32_t *>(s_chunks + subw * Chunk<BP>::kBytes);
    ch.x = reinterpret_cast<double *>(s_chunks + subw * Chunk<BP>::kBytes + BP * HDFE_MAX_DIMS * 4);
    for (int64_t k = threadIdx.x; k < a.n_small * a.B; k += kPassThreads) s_acc[k] = 0.0;
    __syncthreads();
    const uint64_t dterm = (uint64_t)(a.first_draw + ln.j) * kDrawMul;
    double sq = 0.0;
    double ax[kMaxCov];
#pragma unroll
    for (int c = 0; c < kMaxCov; c++) ax[c] = 0.0;
    auto flush = [&](const uint32_t (&codes)[HDFE_MAX_DIMS], double v) {
        if (!ln.on) return;
#pragma unroll
        for (int d = 0; d < HDFE_MAX_DIMS; d++) {
            if (d >= a.D) break;
            if (a.small[d]) atomicAdd(s_acc + (a.soff[d] + codes[d]) * a.B + ln.j, v);
            else atomicAdd(a.acc + (a.offs[d] + codes[d]) * a.B + ln.j, v);
        }
    };
    const int64_t g0 = (int64_t)blockIdx.x * SUBS + subw, gstep = (int64_t)gridDim.x * SUBS;
    for (int64_t g = g0; g < a.G; g += gstep) {
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        const int n = (int)(e - s);
        // pass 1
        double sw = 0.0, tot = 0.0;
        uint32_t bits = 0;
        double wl = 1.0, irl = 1.0;
        for (int c0 = 0; c0 < n; c0 += BP) {
            const int m = min(BP, n - c0);
            wl = load_chunk<BP>(a, ln, ch, s + c0, m);
            irl = inv_root(a, wl);
            for (int q = 0; q < m; q++) {
                const double wi = __shfl_sync(ln.mask, wl, q, BP);
                const double ir = __shfl_sync(ln.mask, irl, q, BP);
                sw += wi;
                if (ln.on) {
                    double r;
                    const int64_t i = s + c0 + q;
                    if (a.R) {
                        r = a.R[i * a.B + ln.j] * ir;
                    } else {
                        const bool neg =
                            rad_negative(a.seed, (uint64_t)(a.ordinal0 + i) * kRowMul, dterm);
                        if (c0 == 0 && neg) bits |= 1u << q;
                        r = neg ? -ir : ir;
                    }
                    tot += wi * r;
                    sq += wi * r * r;
                }
            }
            if (c0 + BP < n) __syncwarp(ln.mask);     // the next chunk reuses the staging
        }
        if (!(sw > 0.0)) continue;
        const double mean = tot / sw;
        // pass 2 (a group of one chunk keeps its staged rows and weights)
        uint32_t prev[HDFE_MAX_DIMS] = {0, 0, 0, 0};
        double run = 0.0;
        bool have = false;
        for (int c0 = 0; c0 < n; c0 += BP) {
            const int m = min(BP, n - c0);
            if (n > BP) {
                __syncwarp(ln.mask);
                wl = load_chunk<BP>(a, ln, ch, s + c0, m);
                irl = inv_root(a, wl);
            }
            for (int q = 0; q < m; q++) {
                const double wi = __shfl_sync(ln.mask, wl, q, BP);
                const double ir = __shfl_sync(ln.mask, irl, q, BP);
                if (have && !same_codes(a, ch.codes, q, prev)) {
                    flush(prev, run);
                    run = 0.0;
                }
                take_codes(a, ch.codes, q, prev);
                have = true;
                if (!ln.on) continue;
                const int64_t i = s + c0 + q;
                double r;
                if (a.R) {
                    r = a.R[i * a.B + ln.j] * ir;
                } else {
                    const bool neg =
                        c0 == 0 ? ((bits >> q) & 1u) != 0
                                : rad_negative(a.seed, (uint64_t)(a.ordinal0 + i) * kRowMul, dterm);
                    r = neg ? -ir : ir;
                }
                const double v = wi * (r - mean);
                run += v;
#pragma unroll
                for (int c = 0; c < kMaxCov; c++) {
                    if (c >= a.c) break;
                    ax[c] += ch.x[q * a.c + c] * v;
                }
            }
        }
        if (have) flush(prev, run);
        __syncwarp(ln.mask);
    }
    // the covariate block and the sums of squares: per lane, then per CTA
    if (a.acc_x && ln.on) {
#pragma unroll
        for (int c = 0; c < kMaxCov; c++) {
            if (c >= a.c) break;
            atomicAdd(a.acc_x + c * a.B + ln.j, ax[c]);
        }
    }
    if (a.squares && ln.on) atomicAdd(a.squares + ln.j, sq);
    __syncthreads();
    for (int d = 0; d < a.D; d++) {
        if (!a.small[d]) continue;
        for (int64_t q = threadIdx.x; q < a.nlev[d] * a.B; q += kPassThreads) {
            const double v = s_acc[a.soff[d] * a.B + q];
            if (v != 0.0) atomicAdd(a.acc + a.offs[d] * a.B + q, v);
        }
    }
}

// `_nb_project_rows` and the JLA sink, one sub-warp of BP lanes per group
// (lane j: draw j).  h_ij = sum_d U[level_d(i), j] + X_i . C[:, j]; pass 1:
// the weighted group mean of r - h; pass 2: the projection o_ij (times
// sqrt(w_i) in the square-root weight metric), written to out and/or turned
// into the sink's P = o^2 and M = (r - o)^2.
//   The group's rows are staged BP at a time (lane t loads row t: codes and
// covariates to shared memory, the weight to a register) and walked in windows
// of kWin rows: the window's U gathers (one coalesced BP-wide row of U each)
// are all issued before any is used, so a sub-warp has kWin gathers in flight
// instead of one dependent gather per row; their sums are parked in the
// window's shared-memory slots (each lane its own), so the loop over the
// window's rows runs without unrolling (the unrolled body did not fit the
// instruction cache: most issue slots were lost waiting for instructions).
// The JLA sums go through a
// shared-memory transpose per window: each lane stores its P and M for the
// window's rows, then lane t sums row t's values over the draws in draw order
// and adds them to the running moments, whose old values it loaded when the
// window began.
constexpr int kProjThreads = 256;
constexpr int kWin = 8;

struct ProjLayout {     // dynamic shared memory of k_project, in doubles
    int chunk;          // per sub-warp: staged codes (BP x D u32) and covariates (BP x c)
    int win;            // per sub-warp: P and M of one window, [2][kWin][BP + 1]
    int c_off;          // C (c x B) first, then the sub-warps' areas
    int total_bytes;
};

template <int BP>
__host__ __device__ inline ProjLayout proj_layout(int D, int c)
{
    ProjLayout o;
    o.chunk = (BP * D + 1) / 2 + BP * c;
    o.win = 2 * kWin * (BP + 1);
    o.c_off = kMaxCov * 32;
    o.total_bytes = (o.c_off + (kProjThreads / BP) * (o.chunk + o.win)) * 8;
    return o;
}

template <int BP>
__global__ void __launch_bounds__(kProjThreads, 4) k_project(Args a)
{
    constexpr int SUBS = kProjThreads / BP;
    extern __shared__ double s_dyn[];
    const Lanes<BP> ln(a.B);
    const int subw = threadIdx.x / BP;
    const ProjLayout lay = proj_layout<BP>(a.D, a.c);
    double *s_C = s_dyn;
    double *area = s_dyn + lay.c_off + subw * (lay.chunk + lay.win);
    uint32_t *s_codes = reinterpret_cast<uint32_t *>(area);          // [BP][D]
    double *s_x = area + (BP * a.D + 1) / 2;                          // [BP][c]
    double *s_P = area + lay.chunk;                                   // [kWin][BP + 1]
    double *s_M = s_P + kWin * (BP + 1);
    for (int k = threadIdx.x; k < a.c * a.B; k += kProjThreads) s_C[k] = a.C[k];
    __syncthreads();
    const uint64_t dterm = (uint64_t)(a.first_draw + ln.j) * kDrawMul;

    // stage rows i0 .. i0 + m - 1 (lane t: row i0 + t); returns the lane's weight
    auto stage = [&](int64_t i0, int m) -> double {
        double w = 1.0;
        if (ln.j < m) {
            const int64_t i = i0 + ln.j;
            if (a.w) w = __ldg(a.w + i);
            for (int d = 0; d < a.D; d++) {
                uint32_t code = __ldg(a.codes + i * a.D + d);
                if ((int64_t)code >= a.nlev[d]) {
                    if (a.status) atomicCAS(a.status, 0u, (unsigned)HDFE_ERR_BAD_CODE);
                    code = 0;
                }
                s_codes[ln.j * a.D + d] = code;
            }
            for (int c = 0; c < a.c; c++) s_x[ln.j * a.c + c] = __ldg(a.X + i * a.c + c);
        }
        __syncwarp(ln.mask);
        return w;
    };
    // sum_d U[level_d(q), j] for the window's rows q0 .. q0 + kWin - 1 (< m)
    // into slot u of hs (this lane's column), every gather issued before the
    // first is used
    auto gather = [&](int q0, int m, double *hs) {
        double hU[kWin];
#pragma unroll
        for (int u = 0; u < kWin; u++) {
            const int q = q0 + u;
            double h = 0.0;
            if (q < m && ln.on) {
                for (int d = 0; d < a.D; d++)
                    h += __ldg(a.U + (a.offs[d] + s_codes[q * a.D + d]) * a.B + ln.j);
            }
            hU[u] = h;
        }
#pragma unroll
        for (int u = 0; u < kWin; u++) hs[u * (BP + 1) + ln.j] = hU[u];
    };
    auto h_cov = [&](int q) {
        double h = 0.0;
        for (int c = 0; c < a.c; c++) h += s_x[q * a.c + c] * s_C[c * a.B + ln.j];
        return h;
    };
    // the draw of row i (unscaled +-1, or the explicit vector)
    auto draw = [&](int64_t i) -> double {
        if (a.R) return ln.on ? __ldg(a.R + i * a.B + ln.j) : 0.0;
        return rad_negative(a.seed, (uint64_t)(a.ordinal0 + i) * kRowMul, dterm) ? -1.0 : 1.0;
    };

    const int64_t g0 = (int64_t)blockIdx.x * SUBS + subw, gstep = (int64_t)gridDim.x * SUBS;
    for (int64_t g = g0; g < a.G; g += gstep) {
        const int64_t s = __ldg(a.starts + g), e = __ldg(a.starts + g + 1);
        const int n = (int)(e - s);
        // pass 1: the weighted group mean of r - h
        double sw = 0.0, tot = 0.0;
        for (int c0 = 0; c0 < n; c0 += BP) {
            const int m = min(BP, n - c0);
            const double wl = stage(s + c0, m);
            const double irl = inv_root(a, wl);
            for (int q0 = 0; q0 < m; q0 += kWin) {
                gather(q0, m, s_P);
                const int nw = min(kWin, m - q0);
#pragma unroll 1
                for (int u = 0; u < nw; u++) {
                    const int q = q0 + u;
                    const double wi = __shfl_sync(ln.mask, wl, q, BP);
                    const double ir = __shfl_sync(ln.mask, irl, q, BP);
                    sw += wi;
                    if (ln.on)
                        tot += wi * (draw(s + c0 + q) * ir -
                                     (s_P[u * (BP + 1) + ln.j] + h_cov(q)));
                }
            }
            if (c0 + BP < n) __syncwarp(ln.mask);   // the next chunk reuses the staging
        }
        const double mean = sw > 0.0 ? tot / sw : 0.0;
        // pass 2: the projection and the JLA sums (a group of one chunk keeps
        // its staged rows)
        for (int c0 = 0; c0 < n; c0 += BP) {
            const int m = min(BP, n - c0);
            double wl = 1.0;
            if (n > BP) {
                __syncwarp(ln.mask);
                wl = stage(s + c0, m);
            } else if (ln.j < m && a.w) {
                wl = __ldg(a.w + s + ln.j);
            }
            for (int q0 = 0; q0 < m; q0 += kWin) {
                const int nw = min(kWin, m - q0);
                double mom[5] = {0, 0, 0, 0, 0};
                const int64_t ir = s + c0 + q0 + ln.j;          // the row this lane sums
                if (a.moments && ln.j < nw) {
#pragma unroll
                    for (int k = 0; k < 5; k++) mom[k] = a.moments[k * a.N + ir];
                }
                gather(q0, m, s_P);
#pragma unroll 1
                for (int u = 0; u < nw; u++) {
                    const int q = q0 + u;
                    const double wi = __shfl_sync(ln.mask, wl, q, BP);
                    if (!ln.on) continue;
                    const int64_t i = s + c0 + q;
                    double o = s_P[u * (BP + 1) + ln.j] + h_cov(q) + mean;
                    if (a.sqrt_weights) o *= sqrt(wi);
                    if (a.out) a.out[i * a.B + ln.j] = o;
                    if (a.moments) {
                        const double rr = draw(i);
                        s_P[u * (BP + 1) + ln.j] = o * o;
                        s_M[u * (BP + 1) + ln.j] = (rr - o) * (rr - o);
                    }
                }
                if (a.moments) {
                    __syncwarp(ln.mask);
                    if (ln.j < nw) {
                        const double *pr = s_P + ln.j * (BP + 1), *mr = s_M + ln.j * (BP + 1);
                        for (int k = 0; k < a.B; k++) {
                            const double P = pr[k], M = mr[k];
                            mom[0] += P;
                            mom[1] += M;
                            mom[2] += P * P;
                            mom[3] += M * M;
                            mom[4] += P * M;
                        }
#pragma unroll
                        for (int k = 0; k < 5; k++) a.moments[k * a.N + ir] = mom[k];
                    }
                    __syncwarp(ln.mask);
                }
            }
        }
        __syncwarp(ln.mask);
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
    const int64_t groups_per_cta = kPassThreads / Bp;
    int64_t b = (G + groups_per_cta - 1) / groups_per_cta;
    if (b > 148 * 16) b = 148 * 16;
    return (unsigned)(b > 0 ? b : 1);
}

template <int BP>
constexpr int project_smem_max()
{
    return (kMaxCov * 32 + (kProjThreads / BP) * ((BP * HDFE_MAX_DIMS + 1) / 2 + BP * kMaxCov +
                                                   2 * kWin * (BP + 1))) * 8;
}

// k_project's grid: its groups spread over every SM, two waves of its four
// resident CTAs per SM at most (the rest grid-stride)
inline unsigned project_grid(int64_t G, int Bp)
{
    const int64_t groups_per_cta = kProjThreads / Bp;
    int64_t b = (G + groups_per_cta - 1) / groups_per_cta;
    if (b > 148 * 8) b = 148 * 8;
    return (unsigned)(b > 0 ? b : 1);
}

template <int BP>
constexpr int center_chunk_smem() { return (kPassThreads / BP) * Chunk<BP>::kBytes; }

constexpr int kSmallBytes = 40 * 1024;    // small dimensions' level x draw sums per CTA

// the dynamic shared memory limits, raised once per device
bool set_smem_limits()
{
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    if (done[dev]) return true;
    const cudaFuncAttribute at = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if (cudaFuncSetAttribute(k_center<8>, at, kSmallBytes + center_chunk_smem<8>()) != cudaSuccess ||
        cudaFuncSetAttribute(k_center<16>, at, kSmallBytes + center_chunk_smem<16>()) != cudaSuccess ||
        cudaFuncSetAttribute(k_center<32>, at, kSmallBytes + center_chunk_smem<32>()) != cudaSuccess ||
        cudaFuncSetAttribute(k_project<8>, at, project_smem_max<8>()) != cudaSuccess ||
        cudaFuncSetAttribute(k_project<16>, at, project_smem_max<16>()) != cudaSuccess ||
        cudaFuncSetAttribute(k_project<32>, at, project_smem_max<32>()) != cudaSuccess)
        return false;
    done[dev] = true;
    return true;
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
        if ((slots + n_levels[d]) * B * 8 <= rows::kSmallBytes && n_levels[d] <= 4096) {
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
    if (!rows::set_smem_limits()) return hdfe_set_cuda_error(cudaGetLastError());
    const unsigned grid = rows::grid_for(n_groups, a.Bp);
    if (a.Bp == 8)
        rows::k_center<8><<<grid, rows::kPassThreads, slots * B * 8 + rows::center_chunk_smem<8>(), s>>>(a);
    else if (a.Bp == 16)
        rows::k_center<16><<<grid, rows::kPassThreads, slots * B * 8 + rows::center_chunk_smem<16>(), s>>>(a);
    else
        rows::k_center<32><<<grid, rows::kPassThreads, slots * B * 8 + rows::center_chunk_smem<32>(), s>>>(a);
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
    if (!rows::set_smem_limits()) return hdfe_set_cuda_error(cudaGetLastError());
    const unsigned grid = rows::project_grid(n_groups, a.Bp);
    if (a.Bp == 8)
        rows::k_project<8><<<grid, rows::kProjThreads,
                             rows::proj_layout<8>(D, c).total_bytes, s>>>(a);
    else if (a.Bp == 16)
        rows::k_project<16><<<grid, rows::kProjThreads,
                              rows::proj_layout<16>(D, c).total_bytes, s>>>(a);
    else
        rows::k_project<32><<<grid, rows::kProjThreads,
                              rows::proj_layout<32>(D, c).total_bytes, s>>>(a);
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
