// Pass 1 on the device: rows -> cells -> identifying cells, with the level
// bookkeeping built on the way.
//
// Reference: core/passes.py:397-531 `_pass1_cells` and :533-589
// `_cell_chunks` (cells = runs of rows with equal group and codes; cnt, n and
// the sums of the centred variables, `_nb_run_sums` core/kernels_base.py:
// 375-422); obs/cnt per level over all cells; identifying cells = those of
// groups with more than one cell; the Jacobi diagonal (`_nb_diag`,
// core/kernels_base.py:87-110) and the right-hand side D_o' M_0 V (`_nb_rhs`,
// :65-83) over the identifying cells.  The means the variables are centred by
// are the pass-0 scan's (core/passes.py:178-187), computed here from V.
//
// Kernels (rows in fixed tiles of kRowTile, groups in tiles of kGroupTile):
//   rows_count   per tile: group starts, cell starts, sum v, sum v^2
//   scan_tiles   one CTA: exclusive offsets of the tile counts; means, ss
//   rows_index   per tile: each group's first row and first cell
//   groups_count per tile of groups: identifying groups and their cells
//   scan_tiles   offsets of those
//   groups_work  persistent over tiles of groups: each warp walks its groups
//                in windows of whole groups (one row per lane), forms cells and
//                group sums by segmented warp scans, writes the identifying
//                cells and aggregates the level statistics per level before
//                updating them (years in per-warp shared slots).
// Integer-valued sums (cnt; obs without weights) are exact in any order;
// other sums are FP64 in atomic order (well inside the 1e-8 bar).
#include <cuda_runtime.h>

#include "common.cuh"

namespace hdfe {
namespace cells {

constexpr int kThreads = 256;
constexpr int kRowTile = 4096;          // rows per tile (16 per thread)
constexpr int kGroupTile = 1024;        // groups per tile (4 per thread)
constexpr int kMaxDims = HDFE_MAX_DIMS;
constexpr int kMaxVars = HDFE_MAX_VARS;
constexpr int kSmemLevelBudget = 64 * 1024;   // bytes of level accumulators per CTA (all warps)
// a shared level slot: obs, cnt, diag, groups (lcount), work, then rhs[m]
constexpr int kSlotFixed = 5;

struct Dims {
    int D, m;
    int64_t offs[kMaxDims];
    int64_t nlev[kMaxDims];
    int small[kMaxDims];        // dimension accumulates in shared memory
    int64_t soff[kMaxDims];     // its first slot there
    int64_t n_small;            // shared slots in use (levels)
};

// ---------------------------------------------------------------- helpers

template <int D>
__device__ __forceinline__ void load_codes(const uint32_t *codes, int64_t i, uint32_t (&c)[D])
{
    if constexpr (D == 2) {
        uint2 v = __ldg(reinterpret_cast<const uint2 *>(codes) + i);
        c[0] = v.x;
        c[1] = v.y;
    } else {
#pragma unroll
        for (int d = 0; d < D; d++) c[d] = __ldg(codes + i * D + d);
    }
}

// Exclusive prefix of a per-thread count over the CTA (thread order), and the
// CTA total.  scratch: kThreads/32 ints.
__device__ __forceinline__ int block_exclusive(int v, int *scratch, int &total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) scratch[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int w = 0; w < kThreads / 32; w++) {
            int t = scratch[w];
            scratch[w] = run;
            run += t;
        }
        scratch[kThreads / 32] = run;
    }
    __syncthreads();
    int excl = scratch[warp] + x - v;
    total = scratch[kThreads / 32];
    __syncthreads();
    return excl;
}

// ------------------------------------------------------------ row kernels

struct RowArgs {
    const uint32_t *gcode;
    const uint32_t *codes;
    const double *V;        // (m, N): one contiguous row per variable
    int64_t N;
    int m;
    int64_t *tile_cnt;      // (tiles, 2): group starts, cell starts
    double *tile_mom;       // (tiles, 2m): sum v, sum v^2
    unsigned *status;
};

template <int D>
__device__ __forceinline__ void row_flags(const RowArgs &a, int64_t i, bool &gs, bool &cs)
{
    uint32_t c[D], p[D];
    const uint32_t g = __ldg(a.gcode + i);
    if (i == 0) { gs = cs = true; return; }
    const uint32_t gp = __ldg(a.gcode + i - 1);
    gs = g != gp;
    load_codes<D>(a.codes, i, c);
    load_codes<D>(a.codes, i - 1, p);
    bool same = !gs;
#pragma unroll
    for (int d = 0; d < D; d++) same &= c[d] == p[d];
    cs = !same;
}

template <int D>
__global__ void __launch_bounds__(kThreads) rows_count(RowArgs a)
{
    __shared__ double s_red[kThreads / 32];
    const int64_t t0 = (int64_t)blockIdx.x * kRowTile;
    const int64_t t1 = min(t0 + kRowTile, a.N);
    int ng = 0, nc = 0;
    for (int64_t i = t0 + threadIdx.x; i < t1; i += kThreads) {
        bool gs, cs;
        row_flags<D>(a, i, gs, cs);
        ng += gs;
        nc += cs;
    }
    double tg = block_sum((double)ng, s_red);
    double tc = block_sum((double)nc, s_red);
    if (threadIdx.x == 0) {
        a.tile_cnt[blockIdx.x * 2 + 0] = (int64_t)tg;
        a.tile_cnt[blockIdx.x * 2 + 1] = (int64_t)tc;
    }
    for (int j = 0; j < a.m; j++) {
        const double *v = a.V + (int64_t)j * a.N;
        double s1 = 0.0, s2 = 0.0;
        for (int64_t i = t0 + threadIdx.x; i < t1; i += kThreads) {
            const double x = __ldg(v + i);
            s1 += x;
            s2 += x * x;
        }
        s1 = block_sum(s1, s_red);
        s2 = block_sum(s2, s_red);
        if (threadIdx.x == 0) {
            a.tile_mom[blockIdx.x * 2 * a.m + j] = s1;
            a.tile_mom[blockIdx.x * 2 * a.m + a.m + j] = s2;
        }
    }
}

// Exclusive scan of `ncols` int64 columns of (tiles, ncols) in place, fixed
// order, one CTA of 1024 threads (each a contiguous run of tiles, combined by
// warp scans); totals to out_totals.  Optionally reduces the moment columns
// into means and sums of squared deviations (fixed-order tree sums).
__global__ void __launch_bounds__(1024) scan_tiles(int64_t *cnt, int64_t tiles, int ncols,
                                                   int64_t *out_totals, const double *mom, int m,
                                                   int64_t N, double *means, double *ss)
{
    __shared__ int64_t s_w[32];
    __shared__ double s_d[32];
    const int T = blockDim.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t per = (tiles + T - 1) / T;
    const int64_t b0 = threadIdx.x * per, b1 = min(b0 + per, tiles);
    for (int c = 0; c < ncols; c++) {
        int64_t s = 0;
        for (int64_t b = b0; b < b1; b++) s += cnt[b * ncols + c];
        // exclusive prefix over threads: warp scans, then the warps' totals
        int64_t x = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_w[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int64_t t = s_w[lane], u = t;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t y = __shfl_up_sync(0xffffffffu, u, o);
                if (lane >= o) u += y;
            }
            s_w[lane] = u - t;
            if (lane == 31) out_totals[c] = u;
        }
        __syncthreads();
        int64_t run = s_w[warp] + x - s;
        for (int64_t b = b0; b < b1; b++) {
            const int64_t v = cnt[b * ncols + c];
            cnt[b * ncols + c] = run;
            run += v;
        }
        __syncthreads();
    }
    if (mom == nullptr) return;
    for (int j = 0; j < 2 * m; j++) {
        double s = 0.0;
        for (int64_t b = b0; b < b1; b++) s += mom[b * 2 * m + j];
        s = warp_sum(s);
        if (lane == 0) s_d[warp] = s;
        __syncthreads();
        if (warp == 0) {
            const double tot = warp_sum(lane < (T >> 5) ? s_d[lane] : 0.0);
            if (lane == 0) {
                if (j < m) means[j] = N > 0 ? tot / (double)N : 0.0;
                else {
                    const double mu = N > 0 ? means[j - m] : 0.0;
                    ss[j - m] = fmax(tot - (double)N * mu * mu, 0.0);
                }
            }
        }
        __syncthreads();
    }
}

template <int D>
__global__ void __launch_bounds__(kThreads) rows_index(RowArgs a, const int64_t *tile_off,
                                                       int64_t *grow, int64_t *gcell,
                                                       const int64_t *totals)
{
    __shared__ int s_scr[2][kThreads / 32 + 1];
    const int64_t t0 = (int64_t)blockIdx.x * kRowTile;
    const int64_t t1 = min(t0 + kRowTile, a.N);
    int64_t g_run = tile_off[blockIdx.x * 2 + 0];
    int64_t c_run = tile_off[blockIdx.x * 2 + 1];
    for (int64_t base = t0; base < t1; base += kThreads) {
        const int64_t i = base + threadIdx.x;
        bool gs = false, cs = false;
        if (i < t1) row_flags<D>(a, i, gs, cs);
        int tg, tc;
        const int eg = block_exclusive(gs ? 1 : 0, s_scr[0], tg);
        const int ec = block_exclusive(cs ? 1 : 0, s_scr[1], tc);
        if (gs) {
            grow[g_run + eg] = i;
            gcell[g_run + eg] = c_run + ec;
        }
        g_run += tg;
        c_run += tc;
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
        grow[totals[0]] = a.N;
        gcell[totals[0]] = totals[1];
    }
}

// ---------------------------------------------------------- group kernels

__global__ void __launch_bounds__(kThreads) groups_count(const int64_t *gcell,
                                                         const int64_t *totals,
                                                         int64_t *tile_cnt)
{
    __shared__ double s_red[kThreads / 32];
    const int64_t G = totals[0];
    const int64_t t0 = (int64_t)blockIdx.x * kGroupTile;
    const int64_t t1 = min(t0 + kGroupTile, G);
    int64_t kg = 0, kc = 0;
    for (int64_t g = t0 + threadIdx.x; g < t1; g += kThreads) {
        const int64_t nc = gcell[g + 1] - gcell[g];
        if (nc > 1) { kg++; kc += nc; }
    }
    double a = block_sum((double)kg, s_red);
    double b = block_sum((double)kc, s_red);
    if (threadIdx.x == 0) {
        tile_cnt[blockIdx.x * 2 + 0] = (int64_t)a;
        tile_cnt[blockIdx.x * 2 + 1] = (int64_t)b;
    }
}

struct GroupArgs {
    Dims dims;
    const uint32_t *codes;
    const double *V;
    const double *w;
    int64_t N;
    const int64_t *grow, *gcell, *tile_off, *totals;
    const double *means;
    int64_t *starts;            // identifying group boundaries (G'+1)
    uint32_t *cell_codes;       // (M, D)
    double *cell_n;             // (M)
    double *cell_sums;          // (M, m) or null: then a scratch buffer is used
    double *group_n;            // (G') sum of n over the group's cells
    double *obs, *cnt, *diag, *rhs;
    int32_t *lcount;            // identifying groups per level (or null)
    int64_t *work;              // cells of those groups per level
    unsigned *status;
};

// One group: cells from its rows, level scatter, identifying-cell output.
// MV > 0 fixes the number of variables at compile time (registers, unrolled
// loops); MV == 0 takes it from the arguments; MV < 0 is the structure-only
// pass (no variables: cells, counts and diag alone).
template <int D, int MV>
__device__ void do_group(const GroupArgs &a, int64_t g, bool keep, int64_t gi, int64_t co,
                         double *s_acc, double *sums_buf)
{
    const Dims &dm = a.dims;
    const int m = MV > 0 ? MV : (MV < 0 ? 0 : dm.m);
    constexpr int kV = MV > 0 ? MV : (MV < 0 ? 1 : kMaxVars);
    const int64_t r0 = a.grow[g], r1 = a.grow[g + 1];
    double Ng = 0.0, vsum[kV];
    for (int j = 0; j < m; j++) vsum[j] = 0.0;
    int64_t q = co;     // next identifying cell slot
    // the cells are runs of rows with equal codes
    int64_t i = r0;
    while (i < r1) {
        uint32_t c[D];
        load_codes<D>(a.codes, i, c);
        int64_t j = i + 1;
        double n = a.w ? a.w[i] : 1.0;
        double s[kV];
#pragma unroll
        for (int v = 0; v < m; v++) s[v] = a.w ? a.w[i] * (a.V[(int64_t)v * a.N + i] - a.means[v])
                                              : (a.V[(int64_t)v * a.N + i] - a.means[v]);
        while (j < r1) {
            uint32_t cj[D];
            load_codes<D>(a.codes, j, cj);
            bool same = true;
#pragma unroll
            for (int d = 0; d < D; d++) same &= cj[d] == c[d];
            if (!same) break;
            const double wj = a.w ? a.w[j] : 1.0;
            if (a.w) n += wj;
            for (int v = 0; v < m; v++) {
                const double z = a.V[(int64_t)v * a.N + j] - a.means[v];
                s[v] += a.w ? wj * z : z;
            }
            j++;
        }
        const double cntv = (double)(j - i);
        if (!a.w) n = cntv;
        // obs / cnt over all cells
#pragma unroll
        for (int d = 0; d < D; d++) {
            if ((int64_t)c[d] >= dm.nlev[d]) {
                atomicCAS(a.status, 0u, (unsigned)HDFE_ERR_BAD_CODE);
                c[d] = 0;
            }
            if (dm.small[d]) {
                double *slot = s_acc + (dm.soff[d] + c[d]) * (kSlotFixed + m);
                atomicAdd(slot + 0, n);
                atomicAdd(slot + 1, cntv);
            } else {
                const int64_t lv = dm.offs[d] + c[d];
                atomicAdd(a.obs + lv, n);
                atomicAdd(a.cnt + lv, cntv);
            }
        }
        if (keep) {
#pragma unroll
            for (int d = 0; d < D; d++) a.cell_codes[q * D + d] = c[d];
            a.cell_n[q] = n;
            for (int v = 0; v < m; v++) sums_buf[q * m + v] = s[v];
            Ng += n;
            for (int v = 0; v < m; v++) vsum[v] += s[v];
            q++;
        }
        i = j;
    }
    if (!keep) return;
    a.starts[gi] = co;
    a.group_n[gi] = Ng;
    double vbar[kV];
    for (int v = 0; v < m; v++) vbar[v] = vsum[v] / Ng;
    // rhs and the diagonal's n over the identifying cells (_nb_rhs, _nb_diag)
    for (int64_t k = co; k < q; k++) {
        uint32_t c[D];
        load_codes<D>(a.cell_codes, k, c);
        const double n = a.cell_n[k];
#pragma unroll
        for (int d = 0; d < D; d++) {
            double *sl = dm.small[d] ? s_acc + (dm.soff[d] + c[d]) * (kSlotFixed + m) : nullptr;
            const int64_t lv = dm.offs[d] + c[d];
            if (sl) atomicAdd(sl + 2, n); else atomicAdd(a.diag + lv, n);
            for (int v = 0; v < m; v++) {
                const double r = sums_buf[k * m + v] - n * vbar[v];
                if (sl) atomicAdd(sl + kSlotFixed + v, r); else atomicAdd(a.rhs + lv * m + v, r);
            }
        }
    }
    // diag -= u_a^2 / N_g over the group's distinct levels (first occurrences)
#pragma unroll
    for (int d = 0; d < D; d++) {
        for (int64_t k = co; k < q; k++) {
            const uint32_t ck = a.cell_codes[k * D + d];
            bool first = true;
            for (int64_t k2 = co; k2 < k; k2++)
                if (a.cell_codes[k2 * D + d] == ck) { first = false; break; }
            if (!first) continue;
            double u = 0.0;
            for (int64_t k2 = k; k2 < q; k2++)
                if (a.cell_codes[k2 * D + d] == ck) u += a.cell_n[k2];
            const double corr = -(u * u / Ng);
            if (dm.small[d]) {
                double *sl = s_acc + (dm.soff[d] + ck) * (kSlotFixed + m);
                atomicAdd(sl + 2, corr);
                if (a.lcount) { atomicAdd(sl + 3, 1.0); atomicAdd(sl + 4, (double)(q - co)); }
            } else {
                atomicAdd(a.diag + dm.offs[d] + ck, corr);
                if (a.lcount) {
                    atomicAdd(a.lcount + dm.offs[d] + ck, 1);
                    atomicAdd(reinterpret_cast<unsigned long long *>(a.work) + dm.offs[d] + ck,
                              (unsigned long long)(q - co));
                }
            }
        }
    }
}

// ------------------------------------------------- warp-cooperative groups
//
// groups_work processes a tile of kGroupTile groups per CTA iteration: the
// tile's identifying-group and identifying-cell offsets are scanned into
// shared memory, then each warp takes kGroupsPerWarp consecutive groups and
// walks them in windows of whole groups of at most 32 rows, one row per lane
// (coalesced loads of codes, weights and variables).  Within a window:
//   - group and cell sums are segmented warp scans (lanes = rows);
//   - identifying cells are written by the lane ending each cell;
//   - the level statistics (obs, cnt, diag with its -u^2/N_g correction, rhs,
//     lcount, work) are aggregated first per (group, level) and then per level
//     with __match_any_sync, so each distinct level of the window is updated
//     once: small dimensions in this warp's own shared slots (plain adds, no
//     contention), the others by global atomics.
// A group longer than 32 rows is processed by one lane with do_group.
constexpr int kWarpsPerCta = kThreads / 32;
constexpr int kGroupsPerWarp = kGroupTile / kWarpsPerCta;

// inclusive segmented sums of x over lanes; seg: first lane of this lane's segment
template <int NV>
__device__ __forceinline__ void seg_scan(double (&x)[NV], int nv, int seg, int lane)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            if (k >= nv) break;
            const double y = __shfl_up_sync(0xffffffffu, x[k], o);
            if (lane - o >= seg) x[k] += y;
        }
    }
}

// first lane of the segment holding `lane`, and its last lane (< n)
__device__ __forceinline__ void segment(unsigned heads, int lane, int n, int &first, int &last)
{
    const unsigned upto = (2u << lane) - 1u;        // lanes 0..lane (all 32 when lane = 31)
    first = 31 - __clz(heads & upto);
    const unsigned after = heads & ~upto;
    last = after ? __ffs(after) - 2 : n - 1;
}

template <int D, int MV>
__global__ void __launch_bounds__(kThreads) groups_work(GroupArgs a, double *sums_scratch)
{
    extern __shared__ double s_dyn[];
    __shared__ int64_t s_gi[kGroupTile], s_co[kGroupTile];
    __shared__ int s_nc[kGroupTile];
    __shared__ int s_scr[2][kThreads / 32 + 1];
    const Dims &dm = a.dims;
    const int m = MV > 0 ? MV : (MV < 0 ? 0 : dm.m);
    constexpr int kV = MV > 0 ? MV : (MV < 0 ? 1 : kMaxVars);
    const int NS = kSlotFixed + m;                  // values per level slot
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *w_slots = s_dyn + (int64_t)warp * dm.n_small * NS;           // this warp's small levels
    const int NSP = NS | 1;                         // scratch row stride: odd, no bank conflicts
    double *w_scr = s_dyn + (int64_t)kWarpsPerCta * dm.n_small * NS + warp * 32 * NSP;
    for (int64_t k = threadIdx.x; k < (int64_t)kWarpsPerCta * dm.n_small * NS; k += kThreads)
        s_dyn[k] = 0.0;
    __syncthreads();
    const int64_t G = a.totals[0];
    const int64_t tiles = (G + kGroupTile - 1) / kGroupTile;
    double *sums_buf = a.cell_sums ? a.cell_sums : sums_scratch;
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int64_t t0 = t * kGroupTile, t1 = min(t0 + kGroupTile, G);
        {
            int64_t gi_run = a.tile_off[t * 2 + 0];
            int64_t co_run = a.tile_off[t * 2 + 1];
            for (int64_t base = t0; base < t1; base += kThreads) {
                const int64_t g = base + threadIdx.x;
                int64_t nc = 0;
                if (g < t1) nc = a.gcell[g + 1] - a.gcell[g];
                const bool keep = nc > 1;
                int tg, tc;
                const int eg = block_exclusive(keep ? 1 : 0, s_scr[0], tg);
                const int ec = block_exclusive(keep ? (int)nc : 0, s_scr[1], tc);
                if (g < t1) {
                    s_gi[g - t0] = keep ? gi_run + eg : -1;
                    s_co[g - t0] = co_run + ec;
                    s_nc[g - t0] = (int)nc;
                }
                gi_run += tg;
                co_run += tc;
            }
        }
        __syncthreads();
        const int64_t gb = t0 + (int64_t)warp * kGroupsPerWarp;
        const int64_t ge = min(gb + kGroupsPerWarp, t1);
        int64_t g = gb;
        while (g < ge) {
            const int64_t r = a.grow[g];
            const int64_t gl = g + 1 + lane;
            const int64_t e = gl <= ge ? a.grow[gl] : INT64_MAX;   // end of group g + lane
            const unsigned fm = __ballot_sync(0xffffffffu, e - r <= 32);
            const int k = __popc(fm);                              // whole groups in the window
            if (k == 0) {       // group g has more than 32 rows: one lane takes it
                if (lane == 0) {
                    const int64_t gloc = g - t0;
                    do_group<D, MV>(a, g, s_gi[gloc] >= 0, s_gi[gloc], s_co[gloc], w_slots, sums_buf);
                }
                __syncwarp();
                g++;
                continue;
            }
            const int n = (int)(__shfl_sync(0xffffffffu, e, k - 1) - r);
            const unsigned heads =
                __reduce_or_sync(0xffffffffu, lane < k - 1 ? (1u << (int)(e - r)) : 0u) | 1u;
            const bool act = lane < n;
            const int64_t i = r + lane;
            // the lane's row
            uint32_t c[D];
#pragma unroll
            for (int d = 0; d < D; d++) c[d] = 0;
            double x[1 + kV];                   // w, then w (v - mean) per variable
#pragma unroll
            for (int v = 0; v <= kV; v++) x[v] = 0.0;
            if (act) {
                load_codes<D>(a.codes, i, c);
                const double wv = a.w ? a.w[i] : 1.0;
                x[0] = wv;
#pragma unroll
                for (int v = 0; v < kV; v++) {
                    if (v >= m) break;
                    const double z = a.V[(int64_t)v * a.N + i] - a.means[v];
                    x[1 + v] = a.w ? wv * z : z;
                }
            }
            int gf, gla;
            segment(heads, lane, n, gf, gla);
            const int grp = __popc(heads & ((2u << lane) - 1u)) - 1;
            const int64_t gloc = g + grp - t0;
            const int64_t gi = s_gi[gloc], co = s_co[gloc];
            const int ncg = s_nc[gloc];
            const bool keep = gi >= 0;
            // cells: a new cell at a group start or where the codes change (the
            // codes as stored, as the cell counts were made); then out-of-range
            // codes are reported and read as level 0
            bool cs = lane == gf;
#pragma unroll
            for (int d = 0; d < D; d++) cs |= __shfl_up_sync(0xffffffffu, c[d], 1) != c[d];
            const unsigned cells = __ballot_sync(0xffffffffu, act && cs) | 1u;
#pragma unroll
            for (int d = 0; d < D; d++) {
                if (act && (int64_t)c[d] >= dm.nlev[d]) {
                    atomicCAS(a.status, 0u, (unsigned)HDFE_ERR_BAD_CODE);
                    c[d] = 0;
                }
            }
            // group sums
            double gsum[1 + kV];
#pragma unroll
            for (int v = 0; v <= kV; v++) gsum[v] = x[v];
            seg_scan<1 + kV>(gsum, 1 + m, gf, lane);
            const double Ng = __shfl_sync(0xffffffffu, gsum[0], gla);
            double vbar[kV];
#pragma unroll
            for (int v = 0; v < kV; v++) {
                if (v >= m) break;
                vbar[v] = __shfl_sync(0xffffffffu, gsum[1 + v], gla) / Ng;
            }
            // identifying cells and groups
            if (__any_sync(0xffffffffu, act && keep)) {
                int cf, cl;
                segment(cells, lane, n, cf, cl);
                double csum[1 + kV];
#pragma unroll
                for (int v = 0; v <= kV; v++) csum[v] = x[v];
                const unsigned actmask = n == 32 ? 0xffffffffu : ((1u << n) - 1u);
                if ((cells & actmask) != actmask) seg_scan<1 + kV>(csum, 1 + m, cf, lane);
                const int cidx = __popc(cells & ((2u << lane) - 1u) & ~((1u << gf) - 1u)) - 1;
                if (act && keep && lane == cl && cidx < ncg) {
                    const int64_t q = co + cidx;
#pragma unroll
                    for (int d = 0; d < D; d++) a.cell_codes[q * D + d] = c[d];
                    a.cell_n[q] = csum[0];
                    if (a.cell_sums) {
#pragma unroll
                        for (int v = 0; v < kV; v++) {
                            if (v >= m) break;
                            a.cell_sums[q * m + v] = csum[1 + v];
                        }
                    }
                }
                if (act && keep && lane == gf) {
                    a.starts[gi] = co;
                    a.group_n[gi] = Ng;
                }
            }
            // level statistics: per (group, level), then per level
#pragma unroll
            for (int d = 0; d < D; d++) {
                const unsigned long long key1 =
                    act ? (((unsigned long long)c[d] << 5) | (unsigned)grp) : (~0ull - lane);
                const unsigned mk1 = __match_any_sync(0xffffffffu, key1);
                const bool lead1 = act && lane == __ffs(mk1) - 1;
                if (act) {
#pragma unroll
                    for (int v = 0; v <= kV; v++) {
                        if (v > m) break;
                        w_scr[lane * NSP + v] = x[v];
                    }
                }
                __syncwarp();
                double T[kSlotFixed + kV];
#pragma unroll
                for (int q = 0; q < kSlotFixed + kV; q++) T[q] = 0.0;
                if (lead1) {
                    double u = 0.0, sv[kV];
#pragma unroll
                    for (int v = 0; v < kV; v++) sv[v] = 0.0;
                    for (unsigned b = mk1; b; b &= b - 1) {
                        const int l = __ffs(b) - 1;
                        u += w_scr[l * NSP];
#pragma unroll
                        for (int v = 0; v < kV; v++) {
                            if (v >= m) break;
                            sv[v] += w_scr[l * NSP + 1 + v];
                        }
                    }
                    T[0] = u;
                    T[1] = (double)__popc(mk1);
                    if (keep) {
                        T[2] = u - u * u / Ng;
                        T[3] = 1.0;
                        T[4] = (double)ncg;
#pragma unroll
                        for (int v = 0; v < kV; v++) {
                            if (v >= m) break;
                            T[kSlotFixed + v] = sv[v] - u * vbar[v];
                        }
                    }
                }
                __syncwarp();
                const unsigned long long key2 =
                    lead1 ? (unsigned long long)c[d] : (0xffffffff00000000ull | (unsigned)lane);
                const unsigned mk2 = __match_any_sync(0xffffffffu, key2);
                const bool lead2 = lead1 && lane == __ffs(mk2) - 1;
                if (lead1) {
#pragma unroll
                    for (int q = 0; q < kSlotFixed + kV; q++) {
                        if (q >= NS) break;
                        w_scr[lane * NSP + q] = T[q];
                    }
                }
                __syncwarp();
                if (lead2) {
                    for (unsigned b = mk2 & (mk2 - 1); b; b &= b - 1) {     // the other leaders
                        const int l = __ffs(b) - 1;
#pragma unroll
                        for (int q = 0; q < kSlotFixed + kV; q++) {
                            if (q >= NS) break;
                            T[q] += w_scr[l * NSP + q];
                        }
                    }
                    if (dm.small[d]) {
                        double *sl = w_slots + (dm.soff[d] + c[d]) * NS;
#pragma unroll
                        for (int q = 0; q < kSlotFixed + kV; q++) {
                            if (q >= NS) break;
                            sl[q] += T[q];
                        }
                    } else {
                        const int64_t lv = dm.offs[d] + c[d];
                        atomicAdd(a.obs + lv, T[0]);
                        atomicAdd(a.cnt + lv, T[1]);
                        if (T[3] > 0.0) {
                            atomicAdd(a.diag + lv, T[2]);
#pragma unroll
                            for (int v = 0; v < kV; v++) {
                                if (v >= m) break;
                                atomicAdd(a.rhs + lv * m + v, T[kSlotFixed + v]);
                            }
                            if (a.lcount) {
                                atomicAdd(a.lcount + lv, (int)T[3]);
                                atomicAdd(reinterpret_cast<unsigned long long *>(a.work) + lv,
                                          (unsigned long long)T[4]);
                            }
                        }
                    }
                }
                __syncwarp();
            }
            g += k;
        }
        __syncthreads();            // the tile's offsets are replaced next
    }
    // the warps' small-dimension slots: summed in warp order, flushed once per CTA
    for (int d = 0; d < dm.D; d++) {
        if (!dm.small[d]) continue;
        for (int64_t l = threadIdx.x; l < dm.nlev[d]; l += kThreads) {
            double sl[kSlotFixed + kV];
#pragma unroll
            for (int q = 0; q < kSlotFixed + kV; q++) sl[q] = 0.0;
            for (int wv = 0; wv < kWarpsPerCta; wv++) {
                const double *src = s_dyn + ((int64_t)wv * dm.n_small + dm.soff[d] + l) * NS;
#pragma unroll
                for (int q = 0; q < kSlotFixed + kV; q++) {
                    if (q >= NS) break;
                    sl[q] += src[q];
                }
            }
            const int64_t lv = dm.offs[d] + l;
            if (sl[0] != 0.0) atomicAdd(a.obs + lv, sl[0]);
            if (sl[1] != 0.0) atomicAdd(a.cnt + lv, sl[1]);
            if (sl[2] != 0.0) atomicAdd(a.diag + lv, sl[2]);
            if (a.lcount && sl[3] != 0.0) {
                atomicAdd(a.lcount + lv, (int)sl[3]);
                atomicAdd(reinterpret_cast<unsigned long long *>(a.work) + lv,
                          (unsigned long long)sl[4]);
            }
#pragma unroll
            for (int v = 0; v < kV; v++) {
                if (v >= m) break;
                if (sl[kSlotFixed + v] != 0.0) atomicAdd(a.rhs + lv * m + v, sl[kSlotFixed + v]);
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const int64_t Gk = a.totals[2];
        a.starts[Gk] = a.totals[3];
    }
}

__global__ void write_counts(const int64_t *tot_rows, const int64_t *tot_groups, int64_t N,
                             hdfe_pass1_counts *out, const unsigned *status)
{
    if (threadIdx.x != 0) return;
    out->n_rows = N;
    out->n_groups = tot_rows[0];
    out->n_cells = tot_rows[1];
    out->n_ident_groups = tot_groups[0];
    out->n_ident_cells = tot_groups[1];
    out->status = (int64_t)*status;
}

// workspace layout (bytes)
struct Layout {
    int64_t tile_cnt, tile_mom, gtile, grow, gcell, totals, status, sums, total;
};

inline Layout layout(int64_t N, int m, bool need_sums)
{
    Layout o;
    const int64_t rt = (N + kRowTile - 1) / kRowTile + 1;
    const int64_t gt = (N + kGroupTile - 1) / kGroupTile + 1;
    int64_t p = 0;
    auto take = [&](int64_t bytes) { int64_t at = p; p += (bytes + 255) / 256 * 256; return at; };
    o.tile_cnt = take(rt * 2 * 8);
    o.tile_mom = take(rt * 2 * (int64_t)m * 8);
    o.gtile = take(gt * 2 * 8);
    o.grow = take((N + 2) * 8);
    o.gcell = take((N + 2) * 8);
    o.totals = take(8 * 8);
    o.status = take(8);
    o.sums = need_sums ? take(N * (int64_t)m * 8) : p;
    o.total = p;
    return o;
}

template <int D>
int run(const uint32_t *gcode, const uint32_t *codes, const double *V, int m, const double *w,
        int64_t N, const int64_t *n_levels, double *means, double *raw_ss, int64_t *starts,
        uint32_t *cell_codes, double *cell_n, double *cell_sums, double *group_n, double *obs,
        double *cnt, double *diag, double *rhs, int32_t *lcount, int64_t *work,
        hdfe_pass1_counts *counts, char *ws, cudaStream_t s)
{
    Layout lay = layout(N, m, cell_sums == nullptr);
    int64_t *tile_cnt = (int64_t *)(ws + lay.tile_cnt);
    double *tile_mom = (double *)(ws + lay.tile_mom);
    int64_t *gtile = (int64_t *)(ws + lay.gtile);
    int64_t *grow = (int64_t *)(ws + lay.grow);
    int64_t *gcell = (int64_t *)(ws + lay.gcell);
    int64_t *totals = (int64_t *)(ws + lay.totals);
    unsigned *status = (unsigned *)(ws + lay.status);
    double *sums_scratch = cell_sums ? nullptr : (double *)(ws + lay.sums);

    Dims dm{};
    dm.D = D;
    dm.m = m;
    int64_t L = 0, slots = 0;
    for (int d = 0; d < D; d++) {
        dm.offs[d] = L;
        dm.nlev[d] = n_levels[d];
        L += n_levels[d];
    }
    // small dimensions: shared-memory accumulators (one copy per warp), smallest first
    const int64_t per_level = (int64_t)(kSlotFixed + m) * 8 * kWarpsPerCta;
    for (int pass = 0; pass < D; pass++) {
        int best = -1;
        for (int d = 0; d < D; d++)
            if (!dm.small[d] && (best < 0 || n_levels[d] < n_levels[best])) best = d;
        if (best < 0) break;
        if ((slots + n_levels[best]) * per_level > kSmemLevelBudget || n_levels[best] > 1024) {
            dm.small[best] = -1;        // tried; stays global
            continue;
        }
        dm.small[best] = 1;
        dm.soff[best] = slots;
        slots += n_levels[best];
    }
    for (int d = 0; d < D; d++) if (dm.small[d] < 0) dm.small[d] = 0;
    dm.n_small = slots;

    HDFE_CUDA_TRY(cudaMemsetAsync(status, 0, 8, s));
    HDFE_CUDA_TRY(cudaMemsetAsync(obs, 0, L * 8, s));
    HDFE_CUDA_TRY(cudaMemsetAsync(cnt, 0, L * 8, s));
    HDFE_CUDA_TRY(cudaMemsetAsync(diag, 0, L * 8, s));
    if (m > 0) HDFE_CUDA_TRY(cudaMemsetAsync(rhs, 0, L * m * 8, s));
    if (lcount) {
        HDFE_CUDA_TRY(cudaMemsetAsync(lcount, 0, L * 4, s));
        HDFE_CUDA_TRY(cudaMemsetAsync(work, 0, L * 8, s));
    }
    const int64_t rtiles = (N + kRowTile - 1) / kRowTile;
    RowArgs ra{gcode, codes, V, N, m, tile_cnt, tile_mom, status};
    rows_count<D><<<(unsigned)rtiles, kThreads, 0, s>>>(ra);
    HDFE_CUDA_TRY(cudaGetLastError());
    scan_tiles<<<1, 1024, 0, s>>>(tile_cnt, rtiles, 2, totals, tile_mom, m, N, means, raw_ss);
    HDFE_CUDA_TRY(cudaGetLastError());
    rows_index<D><<<(unsigned)rtiles, kThreads, 0, s>>>(ra, tile_cnt, grow, gcell, totals);
    HDFE_CUDA_TRY(cudaGetLastError());
    // group tiles: G <= N, sized on the worst case (the counts are on the device)
    const int64_t gtiles = (N + kGroupTile - 1) / kGroupTile;
    HDFE_CUDA_TRY(cudaMemsetAsync(gtile, 0, (gtiles + 1) * 2 * 8, s));
    groups_count<<<(unsigned)gtiles, kThreads, 0, s>>>(gcell, totals, gtile);
    HDFE_CUDA_TRY(cudaGetLastError());
    scan_tiles<<<1, 1024, 0, s>>>(gtile, gtiles, 2, totals + 2, nullptr, 0, 0, nullptr, nullptr);
    HDFE_CUDA_TRY(cudaGetLastError());
    GroupArgs ga;
    ga.dims = dm;
    ga.codes = codes;
    ga.V = V;
    ga.w = w;
    ga.N = N;
    ga.grow = grow;
    ga.gcell = gcell;
    ga.tile_off = gtile;
    ga.totals = totals;
    ga.means = means;
    ga.starts = starts;
    ga.cell_codes = cell_codes;
    ga.cell_n = cell_n;
    ga.cell_sums = cell_sums;
    ga.group_n = group_n;
    ga.obs = obs;
    ga.cnt = cnt;
    ga.diag = diag;
    ga.rhs = rhs;
    ga.lcount = lcount;
    ga.work = work;
    ga.status = status;
    int dev = 0, sms = 0, per_sm = 0;
    HDFE_CUDA_TRY(cudaGetDevice(&dev));
    HDFE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // the warps' small-level slots, then their 32-lane scratch rows
    const size_t smem = (size_t)(slots * per_level) + (size_t)kWarpsPerCta * 32 * ((kSlotFixed + m) | 1) * 8;
    void (*kern)(GroupArgs, double *) = m == 0 ? groups_work<D, -1>
                                       : m == 1 ? groups_work<D, 1> : m == 2 ? groups_work<D, 2>
                                       : m == 3 ? groups_work<D, 3> : m == 4 ? groups_work<D, 4>
                                       : groups_work<D, 0>;
    HDFE_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    HDFE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem));
    int64_t blocks = (int64_t)sms * (per_sm > 0 ? per_sm : 1);
    if (blocks > gtiles) blocks = gtiles > 0 ? gtiles : 1;
    kern<<<(unsigned)blocks, kThreads, smem, s>>>(ga, sums_scratch);
    HDFE_CUDA_TRY(cudaGetLastError());
    write_counts<<<1, 32, 0, s>>>(totals, totals + 2, N, counts, status);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(7);
    return HDFE_OK;
}

}  // namespace cells
}  // namespace hdfe

using namespace hdfe;

extern "C" int64_t hdfe_pass1_workspace_bytes(int64_t n_rows, int32_t m, int32_t keep_sums)
{
    if (n_rows < 0 || m < 0 || m > HDFE_MAX_VARS) return -1;
    return cells::layout(n_rows, m, keep_sums == 0).total;
}

extern "C" int hdfe_pass1(const uint32_t *gcode, const uint32_t *codes, int32_t D,
                          const double *V, int32_t m, const double *w, int64_t n_rows,
                          const int64_t *n_levels, double *means, double *raw_ss,
                          int64_t *starts, uint32_t *cell_codes, double *cell_n,
                          double *cell_sums, double *group_n, double *obs, double *cnt,
                          double *diag, double *rhs, int32_t *lcount, int64_t *work,
                          hdfe_pass1_counts *counts, void *workspace, int64_t workspace_bytes,
                          void *stream)
{
    if (D < 1 || D > HDFE_MAX_DIMS || m < 0 || m > HDFE_MAX_VARS || n_rows < 1 || !gcode ||
        !codes || (m > 0 && !V) || !n_levels || !starts || !cell_codes || !cell_n || !group_n ||
        !obs || !cnt || !diag || (m > 0 && !rhs) || !counts || !workspace || !means || !raw_ss ||
        ((lcount == nullptr) != (work == nullptr)))
        return hdfe_set_arg_error("hdfe_pass1: bad argument");
    for (int d = 0; d < D; d++)
        if (n_levels[d] < 1 || n_levels[d] > 0xffffffffll)
            return hdfe_set_arg_error("hdfe_pass1: n_levels out of range");
    if (workspace_bytes < cells::layout(n_rows, m, cell_sums == nullptr).total)
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_pass1: workspace too small");
    if ((reinterpret_cast<uintptr_t>(codes) & 7) != 0 && D == 2)
        return hdfe_set_arg_error("hdfe_pass1: codes must be 8-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    char *ws = (char *)workspace;
    switch (D) {
    case 1: return cells::run<1>(gcode, codes, V, m, w, n_rows, n_levels, means, raw_ss, starts,
                                 cell_codes, cell_n, cell_sums, group_n, obs, cnt, diag, rhs,
                                 lcount, work, counts, ws, s);
    case 2: return cells::run<2>(gcode, codes, V, m, w, n_rows, n_levels, means, raw_ss, starts,
                                 cell_codes, cell_n, cell_sums, group_n, obs, cnt, diag, rhs,
                                 lcount, work, counts, ws, s);
    case 3: return cells::run<3>(gcode, codes, V, m, w, n_rows, n_levels, means, raw_ss, starts,
                                 cell_codes, cell_n, cell_sums, group_n, obs, cnt, diag, rhs,
                                 lcount, work, counts, ws, s);
    case 4: return cells::run<4>(gcode, codes, V, m, w, n_rows, n_levels, means, raw_ss, starts,
                                 cell_codes, cell_n, cell_sums, group_n, obs, cnt, diag, rhs,
                                 lcount, work, counts, ws, s);
    }
    return hdfe_set_arg_error("hdfe_pass1: D out of range");
}
