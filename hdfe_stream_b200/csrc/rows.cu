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

// `_nb_project_rows` and the JLA sink, one sub-warp of BP lanes per group.
// h_ij = sum_d U[level_d(i), j] (loaded once per run of equal codes) +
// X_i . C[:, j]; pass 1: the weighted group mean of r - h; pass 2: the
// projection o_ij (times sqrt(w_i) in the square-root weight metric), written
// to out and/or turned into the sink's P = o^2 and M = (r - o)^2.  The five
// per-row sums over the block's draws go through shared memory: each lane
// stores its P and M for up to MR rows, then lane t sums row t's values in
// draw order and adds them to the running moments.
template <int BP>
__global__ void __launch_bounds__(kPassThreads) k_project(Args a)
{
    constexpr int SUBS = kPassThreads / BP;
    constexpr int MR = BP < 16 ? BP : 16;                 // rows per moment flush
    extern __shared__ double s_dyn[];
    const Lanes<BP> ln(a.B);
    const int subw = threadIdx.x / BP;
    double *s_C = s_dyn;                                   // (c, B)
    double *s_mom = s_dyn + kMaxCov * 32 + subw * (MR * (BP + 1) * 2);   // [2][MR][BP+1]
    char *s_chunks = reinterpret_cast<char *>(s_dyn + kMaxCov * 32 + SUBS * MR * (BP + 1) * 2);
    Chunk<BP> ch;
    ch.codes = reinterpret_cast<uint32_t *>(s_chunks + subw * Chunk<BP>::kBytes);
    ch.x = reinterpret_cast<double *>(s_chunks + subw * Chunk<BP>::kBytes + BP * HDFE_MAX_DIMS * 4);
    for (int k = threadIdx.x; k < a.c * a.B; k += kPassThreads) s_C[k] = a.C[k];
    __syncthreads();
    const uint64_t dterm = (uint64_t)(a.first_draw + ln.j) * kDrawMul;
    double *pp_buf = s_mom, *mm_buf = s_mom + MR * (BP + 1);
    auto hU_of = [&](const uint32_t (&codes)[HDFE_MAX_DIMS]) {
        double h = 0.0;
        if (ln.on) {
#pragma unroll
            for (int d = 0; d < HDFE_MAX_DIMS; d++) {
                if (d >= a.D) break;
                h += a.U[(a.offs[d] + codes[d]) * a.B + ln.j];
            }
        }
        return h;
    };
    auto h_cov = [&](int q) {
        double h = 0.0;
        for (int c = 0; c < a.c; c++) h += ch.x[q * a.c + c] * s_C[c * a.B + ln.j];
        return h;
    };
    // lane t < nrow adds the sums of row i0 + t to the moments
    auto flush_moments = [&](int64_t i0, int nrow) {
        __syncwarp(ln.mask);
        if (ln.j < nrow) {
            double m0 = 0.0, m1 = 0.0, m2 = 0.0, m3 = 0.0, m4 = 0.0;
            const double *pr = pp_buf + ln.j * (BP + 1), *mr = mm_buf + ln.j * (BP + 1);
            for (int k = 0; k < a.B; k++) {
                const double P = pr[k], M = mr[k];
                m0 += P;
                m1 += M;
                m2 += P * P;
                m3 += M * M;
                m4 += P * M;
            }
            const int64_t i = i0 + ln.j;
            a.moments[0 * a.N + i] += m0;
            a.moments[1 * a.N + i] += m1;
            a.moments[2 * a.N + i] += m2;
            a.moments[3 * a.N + i] += m3;
            a.moments[4 * a.N + i] += m4;
        }
        __syncwarp(ln.mask);
    };
    const int64_t g0 = (int64_t)blockIdx.x * SUBS + subw, gstep = (int64_t)gridDim.x * SUBS;
    for (int64_t g = g0; g < a.G; g += gstep) {
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        const int n = (int)(e - s);
        // pass 1
        double sw = 0.0, tot = 0.0;
        uint32_t bits = 0;
        double wl = 1.0, irl = 1.0;
        uint32_t prev[HDFE_MAX_DIMS] = {0, 0, 0, 0};
        bool have = false;
        double hU = 0.0;
        for (int c0 = 0; c0 < n; c0 += BP) {
            const int m = min(BP, n - c0);
            wl = load_chunk<BP>(a, ln, ch, s + c0, m);
            irl = inv_root(a, wl);
            for (int q = 0; q < m; q++) {
                const double wi = __shfl_sync(ln.mask, wl, q, BP);
                const double ir = __shfl_sync(ln.mask, irl, q, BP);
                sw += wi;
                if (!have || !same_codes(a, ch.codes, q, prev)) {
                    take_codes(a, ch.codes, q, prev);
                    hU = hU_of(prev);
                    have = true;
                }
                if (!ln.on) continue;
                const int64_t i = s + c0 + q;
                double r;
                if (a.R) {
                    r = a.R[i * a.B + ln.j] * ir;
                } else {
                    const bool neg = rad_negative(a.seed, (uint64_t)(a.ordinal0 + i) * kRowMul, dterm);
                    if (c0 == 0 && neg) bits |= 1u << q;
                    r = neg ? -ir : ir;
                }
                tot += wi * (r - (hU + h_cov(q)));
            }
            if (c0 + BP < n) __syncwarp(ln.mask);
        }
        const double mean = sw > 0.0 ? tot / sw : 0.0;
        // pass 2
        have = false;
        int nbuf = 0;               // rows in the moment buffer
        int64_t buf0 = s;           // the first of them
        for (int c0 = 0; c0 < n; c0 += BP) {
            const int m = min(BP, n - c0);
            if (n > BP) {
                __syncwarp(ln.mask);
                wl = load_chunk<BP>(a, ln, ch, s + c0, m);
            }
            for (int q = 0; q < m; q++) {
                const double wi = __shfl_sync(ln.mask, wl, q, BP);
                if (!have || !same_codes(a, ch.codes, q, prev)) {
                    take_codes(a, ch.codes, q, prev);
                    hU = hU_of(prev);
                    have = true;
                }
                const int64_t i = s + c0 + q;
                double P = 0.0, M = 0.0;
                if (ln.on) {
                    double o = hU + h_cov(q) + mean;
                    if (a.sqrt_weights) o *= sqrt(wi);
                    if (a.out) a.out[i * a.B + ln.j] = o;
                    double rr;       // the sink's unscaled draw
                    if (a.R) {
                        rr = a.R[i * a.B + ln.j];
                    } else {
                        const bool neg =
                            c0 == 0 ? ((bits >> q) & 1u) != 0
                                    : rad_negative(a.seed, (uint64_t)(a.ordinal0 + i) * kRowMul, dterm);
                        rr = neg ? -1.0 : 1.0;
                    }
                    P = o * o;
                    M = (rr - o) * (rr - o);
                }
                if (a.moments) {
                    pp_buf[nbuf * (BP + 1) + ln.j] = P;
                    mm_buf[nbuf * (BP + 1) + ln.j] = M;
                    if (++nbuf == MR) {
                        flush_moments(buf0, nbuf);
                        nbuf = 0;
                        buf0 = i + 1;
                    }
                }
            }
        }
        if (a.moments && nbuf > 0) flush_moments(buf0, nbuf);
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
constexpr int project_smem()
{
    constexpr int subs = kPassThreads / BP, mr = BP < 16 ? BP : 16;
    return (kMaxCov * 32 + subs * mr * (BP + 1) * 2) * 8 + subs * Chunk<BP>::kBytes;
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
        cudaFuncSetAttribute(k_project<8>, at, project_smem<8>()) != cudaSuccess ||
        cudaFuncSetAttribute(k_project<16>, at, project_smem<16>()) != cudaSuccess ||
        cudaFuncSetAttribute(k_project<32>, at, project_smem<32>()) != cudaSuccess)
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
    const unsigned grid = rows::grid_for(n_groups, a.Bp);
    if (a.Bp == 8)
        rows::k_project<8><<<grid, rows::kPassThreads, rows::project_smem<8>(), s>>>(a);
    else if (a.Bp == 16)
        rows::k_project<16><<<grid, rows::kPassThreads, rows::project_smem<16>(), s>>>(a);
    else
        rows::k_project<32><<<grid, rows::kPassThreads, rows::project_smem<32>(), s>>>(a);
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
