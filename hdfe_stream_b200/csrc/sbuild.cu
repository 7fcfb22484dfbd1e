// The explicit reduced matrix S = D_o' M_0 D_o in CSR on the device.
//
// Reference: core/solve.py:148-194 `_build_explicit` with the kernels of
// core/kernels_base.py:201-358 (`_nb_level_groups`, `_nb_row_work`,
// `_nb_row_nnz`, `_nb_row_fill`).  Row r of S (level r of dimension dr)
// collects, over every identifying group g containing r and every cell i of
// g, the value  v_i = n_i [i has r] - n_i u_r / N_g  into the columns of
// cell i's levels; u_r = sum of n over g's cells with level r.  Columns come
// out sorted, and the pattern (every level of every group the row's level is
// in, explicit zeros included) is the reference's.
//
// B200 mapping (three calls: analyze, count, fill):
//   analyze   per-level group counts and work (from pass 1, or k_level_stats)
//             -> each level's class: "warp" rows (one warp, a shared hash of
//             32-512 slots), "block" rows (one CTA, up to 8192 slots), or
//             "wide" rows (levels of small dimensions such as years, present
//             in most groups); the groups of each narrow level (lists),
//             each with the pair's u_r / N_g.
//   count     narrow rows, ONE pass: a warp sorts the row's groups (fixed
//             summation order), flattens the row's (group, cell) items over
//             all 32 lanes, and adds each item's v into the hash slot of each
//             of its columns -- lanes with the same column combined first by
//             __match_any_sync in lane order, so the sums are deterministic.
//             The row is compacted, sorted (bitonic) and parked in a temp
//             buffer at a capacity bound; its entries at wide columns also go
//             to a dense (wide x L) buffer.  Wide x wide block: each warp
//             owns the W^2 entries in registers over a fixed set of groups,
//             then fixed-order sums over warps and CTAs (no atomics).  Row
//             nnz -> indptr.
//   fill      narrow rows copied from the temp buffer to their final place;
//             each wide row is the compaction of its dense row (S is
//             symmetric: the narrow rows' entries at the wide column), in
//             column segments processed in parallel.
// Split form (the *_split entry points, for hdfe_pcg_solve_small): the
// trailing small dimensions' levels [small_first, L) are the wide rows, by
// force; a narrow row adds its items at those columns into 16 direct slots
// instead of the hash (the same additions in the same order) and writes them
// as its row of `cross`; the wide x wide block goes to `small`; no wide row
// is written to the CSR, which holds the big block only.
#include <cuda_runtime.h>

#include "common.cuh"

namespace hdfe {
namespace sbuild {

constexpr int kThreads = 256;
constexpr int kSmallSlots = 256;                // hash slots per warp (small warp rows)
constexpr int kSmallListCap = 64;               // groups per small warp row
constexpr int kSmallWarpsPerCta = 8;
constexpr int kWarpSlots = 512;                 // max hash slots per warp (warp rows)
constexpr int kBlockSlots = 8192;               // max hash slots per CTA (block rows)
constexpr int kWarpListCap = 128;               // groups per warp row
constexpr int kBlockListCap = 2048;             // groups per block row
constexpr int32_t kEmptyKey = -1;
constexpr int32_t kKindEmpty = -1, kKindWarp = -2, kKindBlock = -3, kKindWide = -100;
constexpr int kWideWarp = 16;                   // wide x wide on one warp's tiles up to this W
constexpr int kScanTile = 4096;
constexpr int64_t kSeg = 16384;                 // columns per wide-row segment
constexpr int kWarpsPerCta = 4;


__host__ __device__ inline int ceil_log2(int64_t x)
{
    int b = 0;
    while ((int64_t(1) << b) < x) b++;
    return b;
}

struct Args {
    const int64_t *starts;      // (G+1) identifying groups
    int64_t G;
    const uint32_t *codes;      // (M, D)
    const double *n;            // (M)
    const double *group_n;      // (G) N_g
    int64_t M;
    int D;
    int64_t L;
    int64_t offs[HDFE_MAX_DIMS];
    int64_t nlev[HDFE_MAX_DIMS];
    // per-level statistics (pass 1's, or computed here)
    const int32_t *lcount;
    const unsigned long long *work;
    // main workspace
    int32_t *lcount_ws;
    unsigned long long *work_ws;
    int32_t *kind;              // kKind* or the wide index
    int64_t *lptr;              // (L+1)
    int32_t *fillpos;
    int32_t *lgrp;
    double *lwv;                // beside lgrp: u_r / N_g of the (level r, group g) pair
    int64_t *rnnz;              // (L+1) row nnz
    int64_t *toff;              // (L+1) temp offsets of the narrow rows
    int32_t *wide_list;         // wide index -> level
    int32_t *warp_rows, *block_rows;
    int64_t *tiles;             // scan partials
    int64_t *ctr;               // [0] W, [1] warp rows, [2] block rows, [3] lgrp len,
                                // [7] bit d: dimension d has narrow levels, bit 8 + d:
                                // wide levels,
                                // [4] nnz, [5] temp len
    unsigned *status;
    // wide workspace
    double *dval;               // (W, L)
    uint8_t *dpres;             // (W, L)
    int32_t *cell_widx;         // (M, D) wide index of each cell's level, or -1
    double *wpart;              // (CTAs, W*W) per-CTA wide x wide sums
    uint8_t *wpres;             // (CTAs, W*W)
    double *wcross;             // (W*W) n of cells with two wide levels
    int64_t *segcnt;            // (W, nseg)
    int64_t W, nseg, wide_ctas;
    // temp
    int32_t *tcol;
    double *tval;
    // output
    int64_t *indptr;
    int32_t *indices;
    double *data;
    // split form: levels >= small_first are the small levels (L: no split)
    int64_t small_first;
    int ns;
    double *cross;              // (small_first, kCross)
    double *smallb;             // (ns, ns)
};

constexpr int kCross = HDFE_SMALL_MAX_LEVELS;     // cross's row stride

__device__ __forceinline__ int level_dim(const Args &a, int64_t r)
{
    int d = 0;
    while (d + 1 < a.D && a.offs[d + 1] <= r) d++;
    return d;
}

// ------------------------------------------------------------- analyze

// per-level group counts and work, when the caller has no pass-1 statistics
__global__ void __launch_bounds__(kThreads) k_level_stats(Args a)
{
    for (int64_t g = (int64_t)blockIdx.x * kThreads + threadIdx.x; g < a.G;
         g += (int64_t)gridDim.x * kThreads) {
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        const unsigned long long size = (unsigned long long)(e - s);
        for (int d = 0; d < a.D; d++) {
            for (int64_t i = s; i < e; i++) {
                const uint32_t c = a.codes[i * a.D + d];
                bool first = true;
                for (int64_t j = s; j < i; j++)
                    if (a.codes[j * a.D + d] == c) { first = false; break; }
                if (!first) continue;
                if ((int64_t)c >= a.nlev[d]) { atomicCAS(a.status, 0u, (unsigned)HDFE_ERR_BAD_CODE); continue; }
                const int64_t lv = a.offs[d] + c;
                atomicAdd(a.lcount_ws + lv, 1);
                atomicAdd(a.work_ws + lv, size);
            }
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_classify(Args a)
{
    unsigned dims = 0;          // dimensions of this thread's narrow levels
    for (int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x; r < a.L;
         r += (int64_t)gridDim.x * kThreads) {
        const unsigned long long w = a.work[r];
        const int32_t lc = a.lcount[r];
        // distinct columns of the row: at most min(items, levels) per dimension
        int64_t cap = 0;
        for (int d = 0; d < a.D; d++) cap += (int64_t)w < a.nlev[d] ? (int64_t)w : a.nlev[d];
        if (cap > a.L) cap = a.L;
        int32_t k;
        if (w == 0) k = kKindEmpty;
        else if (cap <= kSmallSlots * 3 / 4 && lc <= kSmallListCap) k = kKindWarp;
        else if (cap <= kWarpSlots * 3 / 4 && lc <= kWarpListCap) k = kKindWarp;
        else if (cap <= kBlockSlots * 3 / 4 && lc <= kBlockListCap) k = kKindBlock;
        else k = kKindWide;
        if (r >= a.small_first) {
            k = kKindWide;                  // the split form's small levels
        } else if (k == kKindWide && a.small_first < a.L) {
            // a big row too wide for a narrow row: the split form cannot be built
            atomicCAS(a.status, 0u, (unsigned)HDFE_ERR_CAPACITY);
        }
        if (k == kKindWarp) {
            if (cap <= kSmallSlots * 3 / 4 && lc <= kSmallListCap)   // small rows from the front
                a.warp_rows[atomicAdd((unsigned long long *)(a.ctr + 1), 1ull)] = (int32_t)r;
            else                                                      // the others from the back
                a.warp_rows[a.L - 1 - (int64_t)atomicAdd((unsigned long long *)(a.ctr + 6), 1ull)] =
                    (int32_t)r;
        }
        if (k == kKindBlock) a.block_rows[atomicAdd((unsigned long long *)(a.ctr + 2), 1ull)] = (int32_t)r;
        if (k == kKindWide) {
            const int64_t wi = (int64_t)atomicAdd((unsigned long long *)a.ctr, 1ull);
            a.wide_list[wi] = (int32_t)r;
            k = (int32_t)wi;
        }
        a.kind[r] = k;
        const bool narrow = k == kKindWarp || k == kKindBlock;
        a.lptr[r] = narrow ? lc : 0;
        a.toff[r] = narrow ? cap : 0;   // capacity of the row in the temp buffer
        if (narrow) dims |= 1u << level_dim(a, r);
        if (k >= 0) dims |= 1u << (8 + level_dim(a, r));
    }
    dims = __reduce_or_sync(0xffffffffu, dims);
    if ((threadIdx.x & 31) == 0 && dims != 0)
        atomicOr(reinterpret_cast<unsigned long long *>(a.ctr + 7), (unsigned long long)dims);
}

// the wide list in level order, so wide indices do not depend on atomics
__global__ void k_sort_wide(Args a)
{
    if (threadIdx.x != 0) return;
    const int64_t W = a.ctr[0];
    for (int64_t i = 1; i < W; i++) {
        int32_t x = a.wide_list[i];
        int64_t j = i - 1;
        while (j >= 0 && a.wide_list[j] > x) { a.wide_list[j + 1] = a.wide_list[j]; j--; }
        a.wide_list[j + 1] = x;
    }
    for (int64_t i = 0; i < W; i++) a.kind[a.wide_list[i]] = (int32_t)i;
}

// ------------------------------------------------- exclusive scan (int64)

__global__ void __launch_bounds__(kThreads) k_scan_tiles(const int64_t *x, int64_t n, int64_t *tiles)
{
    __shared__ double s_red[kThreads / 32];
    const int64_t t0 = (int64_t)blockIdx.x * kScanTile, t1 = min(t0 + kScanTile, n);
    int64_t s = 0;
    for (int64_t i = t0 + threadIdx.x; i < t1; i += kThreads) s += x[i];
    double t = block_sum((double)s, s_red);     // integer sums stay exact below 2^53
    if (threadIdx.x == 0) tiles[blockIdx.x] = (int64_t)t;
}

__global__ void __launch_bounds__(1024) k_scan_top(int64_t *tiles, int64_t nt, int64_t *total)
{
    __shared__ int64_t s[1024];
    const int64_t per = (nt + blockDim.x - 1) / blockDim.x;
    const int64_t b0 = threadIdx.x * per, b1 = min(b0 + per, nt);
    int64_t acc = 0;
    for (int64_t b = b0; b < b1; b++) acc += tiles[b];
    s[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t run = 0;
        for (unsigned t = 0; t < blockDim.x; t++) { int64_t v = s[t]; s[t] = run; run += v; }
        *total = run;
    }
    __syncthreads();
    int64_t run = s[threadIdx.x];
    for (int64_t b = b0; b < b1; b++) { int64_t v = tiles[b]; tiles[b] = run; run += v; }
}

// out[i] = exclusive prefix of x (out may alias x); out[n] = total
__global__ void __launch_bounds__(kThreads) k_scan_apply(const int64_t *x, int64_t n,
                                                         const int64_t *tiles, int64_t *out,
                                                         const int64_t *total)
{
    __shared__ int64_t s_w[kThreads / 32 + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t t0 = (int64_t)blockIdx.x * kScanTile, t1 = min(t0 + kScanTile, n);
    int64_t run = tiles[blockIdx.x];
    for (int64_t base = t0; base < t1; base += kThreads) {
        const int64_t i = base + threadIdx.x;
        const int64_t v = i < t1 ? x[i] : 0;
        int64_t inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int64_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) s_w[warp] = inc;
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t r = 0;
            for (int w = 0; w < kThreads / 32; w++) { int64_t t = s_w[w]; s_w[w] = r; r += t; }
            s_w[kThreads / 32] = r;
        }
        __syncthreads();
        const int64_t excl = run + s_w[warp] + inc - v;
        const int64_t tile_total = s_w[kThreads / 32];
        __syncthreads();
        if (i < t1) out[i] = excl;
        run += tile_total;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = *total;
}

// ------------------------------------------------------- group lists

// A thread per group.  Per dimension, each level's first cell in the group
// appends the group to the level's list, with u_r / N_g beside it (u_r = n
// summed over the group's cells at the level, in cell order).  When the
// group's codes in the dimension are nondecreasing (pass 0's layout), a run
// start is its level's first cell and the run holds all of the level's
// cells; otherwise the group's cells are walked for both.  A warp takes 32
// consecutive groups at a time and first stages their cells' codes and n in
// shared memory by coalesced loads (a chunk of more than kListCap cells is
// read in place), so each cell is fetched once.
constexpr int kListWarps = 4;
constexpr int kListCap = 384;                   // cells staged per warp

inline size_t list_smem(int D) { return (size_t)kListWarps * kListCap * (8 + 4 * (size_t)D); }

__device__ __forceinline__ void list_append(const Args &a, int64_t lv, int64_t g, double u)
{
    const int32_t at = atomicAdd(a.fillpos + lv, 1);
    if (a.lptr[lv] + at < a.lptr[lv + 1]) {
        a.lgrp[a.lptr[lv] + at] = (int32_t)g;
        a.lwv[a.lptr[lv] + at] = u / a.group_n[g];
    }
}

__device__ __forceinline__ bool listed(const Args &a, int64_t lv)
{
    const int32_t k = a.kind[lv];
    return k == kKindWarp || k == kKindBlock;       // no list for wide rows
}

// the group's lists from codes cd (stride D) and weights nw, both indexed
// from the group's first cell
__device__ void group_lists(const Args &a, int64_t g, int cells, const uint32_t *cd,
                            const double *nw)
{
    const int D = a.D;
    const int64_t dims = a.ctr[7];
    const double gn = a.group_n[g];
    for (int d = 0; d < D; d++) {
        if (!((dims >> d) & 1)) continue;           // no narrow level in this dimension
        bool sorted = true;
        for (int i = 1; i < cells; i++) sorted &= cd[(i - 1) * D + d] <= cd[i * D + d];
        if (sorted) {
            // kRuns runs at a time: their levels' kinds, then their list slots,
            // each set of loads and atomics issued together
            constexpr int kRuns = 4;
            for (int i = 0; i < cells;) {
                int64_t lv[kRuns];
                double u[kRuns];
                int nr = 0;
#pragma unroll
                for (int t = 0; t < kRuns; t++) {
                    lv[t] = -1;
                    u[t] = 0.0;
                    if (i < cells) {
                        const uint32_t c = cd[i * D + d];
                        double su = nw[i];
                        int j = i + 1;
                        for (; j < cells && cd[j * D + d] == c; j++) su += nw[j];
                        if ((int64_t)c < a.nlev[d]) lv[t] = a.offs[d] + c;
                        u[t] = su;
                        i = j;
                        nr = t + 1;
                    }
                }
                int32_t kk[kRuns];
#pragma unroll
                for (int t = 0; t < kRuns; t++) kk[t] = lv[t] >= 0 ? a.kind[lv[t]] : kKindEmpty;
                int32_t at[kRuns];
                int64_t l0[kRuns], l1[kRuns];
#pragma unroll
                for (int t = 0; t < kRuns; t++) {
                    const bool on = t < nr && (kk[t] == kKindWarp || kk[t] == kKindBlock);
                    at[t] = on ? atomicAdd(a.fillpos + lv[t], 1) : -1;
                    l0[t] = on ? a.lptr[lv[t]] : 0;
                    l1[t] = on ? a.lptr[lv[t] + 1] : 0;
                }
#pragma unroll
                for (int t = 0; t < kRuns; t++) {
                    if (at[t] >= 0 && l0[t] + at[t] < l1[t]) {
                        a.lgrp[l0[t] + at[t]] = (int32_t)g;
                        a.lwv[l0[t] + at[t]] = u[t] / gn;
                    }
                }
            }
            continue;
        }
        uint32_t prev = 0xffffffffu;
        for (int i = 0; i < cells; i++) {
            const uint32_t c = cd[i * D + d];
            if (c == prev || (int64_t)c >= a.nlev[d]) continue;        // a run of one level
            prev = c;
            const int64_t lv = a.offs[d] + c;
            if (!listed(a, lv)) continue;
            bool first = true;
            for (int j = 0; j < i; j++)
                if (cd[j * D + d] == c) { first = false; break; }
            if (!first) continue;
            double u = 0.0;
            for (int j = i; j < cells; j++)
                if (cd[j * D + d] == c) u += nw[j];
            list_append(a, lv, g, u);
        }
    }
}

__global__ void __launch_bounds__(kListWarps * 32) k_fill_lists(Args a)
{
    extern __shared__ double s_list_raw[];
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    const int D = a.D;
    double *sn = s_list_raw + (size_t)wl * kListCap;
    uint32_t *sc = reinterpret_cast<uint32_t *>(s_list_raw + (size_t)kListWarps * kListCap) +
                   (size_t)wl * kListCap * D;
    const int64_t chunks = (a.G + 31) / 32;
    const int64_t wstep = (int64_t)gridDim.x * kListWarps;
    for (int64_t ch = (int64_t)blockIdx.x * kListWarps + wl; ch < chunks; ch += wstep) {
        const int64_t g0 = ch * 32;
        const int ng = (int)min((int64_t)32, a.G - g0);
        const int64_t g = g0 + lane;
        const int64_t s = lane < ng ? a.starts[g] : 0, e = lane < ng ? a.starts[g + 1] : 0;
        const int64_t c0 = __shfl_sync(0xffffffffu, s, 0);
        const int64_t c1 = __shfl_sync(0xffffffffu, e, ng - 1);
        const bool staged = c1 - c0 <= kListCap;            // warp-uniform
        if (staged) {
            for (int64_t q = lane; q < (c1 - c0) * D; q += 32) sc[q] = a.codes[c0 * D + q];
            for (int64_t q = lane; q < c1 - c0; q += 32) sn[q] = a.n[c0 + q];
        }
        __syncwarp();
        if (lane < ng) {
            if (staged) group_lists(a, g, (int)(e - s), sc + (s - c0) * D, sn + (s - c0));
            else group_lists(a, g, (int)(e - s), a.codes + s * D, a.n + s);
        }
        __syncwarp();
    }
}

// ------------------------------------------------------- narrow rows

__device__ __forceinline__ uint32_t slot_of(int32_t col, int bits)
{
    return ((uint32_t)col * 2654435761u) >> (32 - bits);
}

// Sort n int32 keys (ascending, n <= the buffer's power-of-two capacity) in
// warp-shared memory, with an optional double payload.
__device__ void warp_bitonic(int32_t *key, double *val, int n, int lane)
{
    int size = 1;
    while (size < n) size <<= 1;
    for (int i = n + lane; i < size; i += 32) key[i] = INT32_MAX;
    __syncwarp();
    for (int k = 2; k <= size; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < size; i += 32) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const bool up = (i & k) == 0;
                    const int32_t ki = key[i], kj = key[ixj];
                    if ((ki > kj) == up) {
                        key[i] = kj;
                        key[ixj] = ki;
                        if (val) { double t = val[i]; val[i] = val[ixj]; val[ixj] = t; }
                    }
                }
            }
            __syncwarp();
        }
    }
}

// Sort n <= 128 distinct int32 keys (with an optional double payload) in
// warp-shared memory by rank: each key's position is the number of keys
// below it.  Keys are distinct (columns of a row, groups of a list).
__device__ void warp_rank_sort(int32_t *key, double *val, int n, int lane)
{
    int32_t k[4];
    double v[4];
    int rank[4];
#pragma unroll
    for (int t = 0; t < 4; t++) {
        const int i = lane + 32 * t;
        k[t] = i < n ? key[i] : INT32_MAX;
        v[t] = (val && i < n) ? val[i] : 0.0;
        rank[t] = 0;
    }
    const int chunks = (n + 31) >> 5;
    for (int c = 0; c < chunks; c++) {
        // chunk c's keys, one per lane (selected without indexing the array)
        const int32_t kc = c == 0 ? k[0] : c == 1 ? k[1] : c == 2 ? k[2] : k[3];
        for (int j = 0; j < 32; j++) {
            const int32_t other = __shfl_sync(0xffffffffu, kc, j);
#pragma unroll
            for (int t = 0; t < 4; t++) rank[t] += other < k[t];
        }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < 4; t++) {
        const int i = lane + 32 * t;
        if (i < n) {
            key[rank[t]] = k[t];
            if (val) val[rank[t]] = v[t];
        }
    }
    __syncwarp();
}

// The same for n <= 32 keys: one key a lane.
__device__ void warp_rank_sort32(int32_t *key, double *val, int n, int lane)
{
    const int32_t k = lane < n ? key[lane] : INT32_MAX;
    const double v = (val && lane < n) ? val[lane] : 0.0;
    int rank = 0;
    for (int j = 0; j < n; j++) rank += __shfl_sync(0xffffffffu, k, j) < k;
    __syncwarp();
    if (lane < n) {
        key[rank] = k;
        if (val) val[rank] = v;
    }
    __syncwarp();
}

__device__ __forceinline__ void warp_sort(int32_t *key, double *val, int n, int lane)
{
    if (n <= 32) warp_rank_sort32(key, val, n, lane);
    else if (n <= 128) warp_rank_sort(key, val, n, lane);
    else warp_bitonic(key, val, n, lane);
}

struct RowSmem {
    double *xs;         // kCross direct slots: the split form's small columns
    int32_t *keys;
    double *vals;
    int32_t *list;      // the row's groups
    int32_t *loff;      // (nl+1) item offsets
    int64_t *gs;        // first cell of each listed group
    double *wv;         // u_r / N_g of each listed group
    double *stage;      // 32
    int *cnt;
};

// One narrow row by one warp: accumulate, compact, sort, park in temp.
__device__ void narrow_row(const Args &a, int64_t r, const RowSmem &sm, int max_bits)
{
    const int lane = threadIdx.x & 31;
    const int dr = level_dim(a, r);
    const uint32_t lr = (uint32_t)(r - a.offs[dr]);
    const bool split = a.small_first < a.L;
    // the table holds the row's hashed columns: all of them, or in the split
    // form the big levels' alone (the small ones go to direct slots)
    int64_t cap = a.toff[r + 1] - a.toff[r];
    if (split) {
        const int64_t w = (int64_t)a.work[r];
        int64_t cb = 0;
        for (int d = 0; d < a.D; d++)
            if (a.offs[d] < a.small_first) cb += w < a.nlev[d] ? w : a.nlev[d];
        cap = cb < cap ? cb : cap;
    }
    int bits = ceil_log2((cap * 4 + 2) / 3);
    bits = bits < 5 ? 5 : (bits > max_bits ? max_bits : bits);
    const int slots = 1 << bits;
    for (int i = lane; i < slots; i += 32) { sm.keys[i] = kEmptyKey; sm.vals[i] = 0.0; }
    if (lane < kCross) sm.xs[lane] = 0.0;
    // the row's groups, ascending
    const int64_t l0 = a.lptr[r];
    const int nl = (int)(a.lptr[r + 1] - l0);
    for (int i = lane; i < nl; i += 32) {
        sm.list[i] = a.lgrp[l0 + i];
        sm.wv[i] = a.lwv[l0 + i];
    }
    __syncwarp();
    warp_sort(sm.list, sm.wv, nl, lane);
    // per group: first cell and cell count (u_r / N_g came with the list)
    for (int k = lane; k < nl; k += 32) {
        const int64_t g = sm.list[k];
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        sm.gs[k] = s;
        sm.loff[k] = (int32_t)(e - s);
    }
    __syncwarp();
    // exclusive offsets of the groups' cells (the row's items)
    int32_t carry = 0;
    for (int base = 0; base < nl; base += 32) {
        const int k = base + lane;
        const int32_t v = k < nl ? sm.loff[k] : 0;
        int32_t inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        __syncwarp();
        if (k < nl) sm.loff[k] = carry + inc - v;
        carry += __shfl_sync(0xffffffffu, inc, 31);
        __syncwarp();
    }
    if (lane == 0) sm.loff[nl] = carry;
    __syncwarp();
    const int32_t items = carry;
    for (int32_t base = 0; base < items; base += 32) {
        const int32_t j = base + lane;
        const bool valid = j < items;
        int64_t i = 0;
        double v = 0.0;
        if (valid) {
            int lo = 0, hi = nl;            // last group with loff <= j
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (sm.loff[mid] <= j) lo = mid; else hi = mid;
            }
            i = sm.gs[lo] + (j - sm.loff[lo]);
            const double ni = a.n[i];
            v -= ni * sm.wv[lo];
            if (a.codes[i * a.D + dr] == lr) v += ni;
        }
        for (int d = 0; d < a.D; d++) {
            const int32_t col = valid ? (int32_t)(a.offs[d] + a.codes[i * a.D + d]) : -1;
            const unsigned peers = __match_any_sync(0xffffffffu, col);
            const int leader = __ffs(peers) - 1;
            sm.stage[lane] = v;
            __syncwarp();
            if (valid && lane == leader && split && col >= a.small_first) {
                double sum = 0.0;
                for (unsigned p = peers; p; p &= p - 1) sum += sm.stage[__ffs(p) - 1];
                sm.xs[col - a.small_first] += sum;      // a direct slot, not the hash
            } else if (valid && lane == leader) {
                double sum = 0.0;
                for (unsigned p = peers; p; p &= p - 1) sum += sm.stage[__ffs(p) - 1];
                // the leaders' columns are distinct, so a slot found holding col
                // is this lane's alone; an empty one is claimed by a CAS
                uint32_t h = slot_of(col, bits);
                for (int probe = 0; probe < slots; probe++) {
                    int32_t old = sm.keys[h];
                    if (old == kEmptyKey) old = atomicCAS(sm.keys + h, kEmptyKey, col);
                    if (old == kEmptyKey || old == col) {
                        sm.vals[h] += sum;
                        break;
                    }
                    h = (h + 1) & (slots - 1);
                }
            }
            __syncwarp();
        }
    }
    // compact the table to its first slots (entries never overtake unread slots)
    if (lane == 0) *sm.cnt = 0;
    __syncwarp();
    for (int base = 0; base < slots; base += 32) {
        const int i = base + lane;
        const int32_t c = sm.keys[i];
        const double v = sm.vals[i];
        const bool has = c != kEmptyKey;
        const unsigned m = __ballot_sync(0xffffffffu, has);
        const int before = __popc(m & ((1u << lane) - 1));
        const int at0 = *sm.cnt;
        __syncwarp();
        if (has) { sm.keys[at0 + before] = c; sm.vals[at0 + before] = v; }
        __syncwarp();
        if (lane == 0) *sm.cnt = at0 + __popc(m);
        __syncwarp();
    }
    const int cnt = *sm.cnt;
    warp_sort(sm.keys, sm.vals, cnt, lane);
    const int64_t t0 = a.toff[r];
    for (int i = lane; i < cnt; i += 32) {
        const int32_t c = sm.keys[i];
        a.tcol[t0 + i] = c;
        a.tval[t0 + i] = sm.vals[i];
        const int32_t k = split ? -1 : a.kind[c];     // the split form has no wide column here
        if (k >= 0) {
            a.dpres[(int64_t)k * a.L + r] = 1;
            a.dval[(int64_t)k * a.L + r] = sm.vals[i];
        }
    }
    if (split && lane < kCross) a.cross[r * kCross + lane] = sm.xs[lane];
    if (lane == 0) a.rnnz[r] = cnt;
    __syncwarp();
}

// small warp rows (the front of warp_rows): 256-slot tables, 8 warps per CTA
__global__ void __launch_bounds__(kSmallWarpsPerCta * 32) k_small_rows(Args a)
{
    __shared__ double s_xs[kSmallWarpsPerCta][kCross];
    __shared__ int32_t s_keys[kSmallWarpsPerCta][kSmallSlots];
    __shared__ double s_vals[kSmallWarpsPerCta][kSmallSlots];
    __shared__ int32_t s_list[kSmallWarpsPerCta][kSmallListCap];
    __shared__ int32_t s_loff[kSmallWarpsPerCta][kSmallListCap + 1];
    __shared__ int64_t s_gs[kSmallWarpsPerCta][kSmallListCap];
    __shared__ double s_wv[kSmallWarpsPerCta][kSmallListCap];
    __shared__ double s_stage[kSmallWarpsPerCta][32];
    __shared__ int s_cnt[kSmallWarpsPerCta];
    const int w = threadIdx.x >> 5;
    RowSmem sm{s_xs[w], s_keys[w], s_vals[w], s_list[w], s_loff[w], s_gs[w], s_wv[w], s_stage[w],
               &s_cnt[w]};
    const int64_t nrows = a.ctr[1];
    for (int64_t k = (int64_t)blockIdx.x * kSmallWarpsPerCta + w; k < nrows;
         k += (int64_t)gridDim.x * kSmallWarpsPerCta)
        narrow_row(a, a.warp_rows[k], sm, 8);
}

// the other warp rows (the back of warp_rows): 512-slot tables
__global__ void __launch_bounds__(kWarpsPerCta * 32) k_warp_rows(Args a)
{
    __shared__ double s_xs[kWarpsPerCta][kCross];
    __shared__ int32_t s_keys[kWarpsPerCta][kWarpSlots];
    __shared__ double s_vals[kWarpsPerCta][kWarpSlots];
    __shared__ int32_t s_list[kWarpsPerCta][kWarpListCap];
    __shared__ int32_t s_loff[kWarpsPerCta][kWarpListCap + 1];
    __shared__ int64_t s_gs[kWarpsPerCta][kWarpListCap];
    __shared__ double s_wv[kWarpsPerCta][kWarpListCap];
    __shared__ double s_stage[kWarpsPerCta][32];
    __shared__ int s_cnt[kWarpsPerCta];
    const int w = threadIdx.x >> 5;
    RowSmem sm{s_xs[w], s_keys[w], s_vals[w], s_list[w], s_loff[w], s_gs[w], s_wv[w], s_stage[w],
               &s_cnt[w]};
    const int64_t nrows = a.ctr[6];
    for (int64_t k = (int64_t)blockIdx.x * kWarpsPerCta + w; k < nrows;
         k += (int64_t)gridDim.x * kWarpsPerCta)
        narrow_row(a, a.warp_rows[a.L - 1 - k], sm, 9);
}

// block rows: one warp per CTA with the large table in dynamic shared memory
__global__ void __launch_bounds__(32) k_block_rows(Args a)
{
    extern __shared__ unsigned char s_raw[];
    double *vals = reinterpret_cast<double *>(s_raw);
    double *wv = vals + kBlockSlots;
    int64_t *gs = reinterpret_cast<int64_t *>(wv + kBlockListCap);
    int32_t *keys = reinterpret_cast<int32_t *>(gs + kBlockListCap);
    int32_t *list = keys + kBlockSlots;
    int32_t *loff = list + kBlockListCap;
    __shared__ double s_stage[32];
    __shared__ double s_xs[kCross];
    __shared__ int s_cnt;
    RowSmem sm{s_xs, keys, vals, list, loff, gs, wv, s_stage, &s_cnt};
    const int64_t nrows = a.ctr[2];
    for (int64_t k = blockIdx.x; k < nrows; k += gridDim.x)
        narrow_row(a, a.block_rows[k], sm, 13);
}

constexpr size_t kBlockSmem = (size_t)kBlockSlots * 12 + (size_t)kBlockListCap * (8 + 8 + 4 + 4) + 16;

// narrow rows from the temp buffer to their place in the CSR
// (kCopyLanes lanes a row, so a warp has several rows' dependent loads --
// the row, its offsets, then its entries -- in flight at once)
constexpr int kCopyLanes = 8;

__global__ void __launch_bounds__(kThreads) k_copy_narrow(Args a)
{
    const int64_t t = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    const int sl = (int)(t % kCopyLanes);
    const int64_t gs = t / kCopyLanes, ns = ((int64_t)gridDim.x * kThreads) / kCopyLanes;
    const int64_t n1 = a.ctr[1], n6 = a.ctr[6], n2 = a.ctr[2];
    for (int64_t k = gs; k < n1 + n6 + n2; k += ns) {
        const int64_t r = k < n1 ? a.warp_rows[k]
                        : k < n1 + n6 ? a.warp_rows[a.L - 1 - (k - n1)] : a.block_rows[k - n1 - n6];
        const int64_t src = a.toff[r], dst = a.indptr[r], cnt = a.rnnz[r];
        for (int64_t i = sl; i < cnt; i += kCopyLanes) {
            a.indices[dst + i] = a.tcol[src + i];
            a.data[dst + i] = a.tval[src + i];
        }
    }
}

// ------------------------------------------------------- wide rows

__global__ void __launch_bounds__(kThreads) k_cell_widx(Args a)
{
    const int64_t total = a.M * a.D;
    for (int64_t q = (int64_t)blockIdx.x * kThreads + threadIdx.x; q < total;
         q += (int64_t)gridDim.x * kThreads) {
        const int d = (int)(q % a.D);
        const uint32_t c = a.codes[q];
        int32_t k = -1;
        if ((int64_t)c < a.nlev[d]) {
            const int32_t kk = a.kind[a.offs[d] + c];
            k = kk >= 0 ? kk : -1;
        }
        a.cell_widx[q] = k;
    }
}

// The wide x wide block for W <= 16.  Per group g the block adds
//     C_g(a, b) - (u_a / N_g) u_b
// (the reference's per-cell sum  sum_{i has b} (n_i [i has a] - n_i u_a / N_g)
// regrouped), with u_a = sum of n over g's cells with wide level a and
// C_g(a, b) = sum of n over its cells having both (C_g(a, a) = u_a).  A warp
// takes 32 consecutive groups at a time: their cells are read coalesced (one
// per lane) and summed into the groups' u rows in shared memory (lanes with
// the same group and level combined by __match_any_sync in lane order); then
// the 32 groups' (u_a / N_g) u_b are added as a 16 x 32 by 32 x 16 product on
// the FP64 tensor cores (mma m8n8k4 tiles), lanes a < W add the diagonal's
// u_a, and the pattern is the
// union of the groups' level masks.  Cells with two or more wide levels
// (several small dimensions) add their off-diagonal C, for every pair of
// their wide levels, into its own array by atomic adds (exact for counts;
// in atomic order for weighted n).  Warps and CTAs are summed in a fixed
// order, so the rest of the block is deterministic.
// D += A B for one 8 x 8 x 4 FP64 tile, the whole warp: A row-major (this lane
// holds row lane / 4, column lane % 4), B column-major (row lane % 4, column
// lane / 4), D (row lane / 4, columns 2 (lane % 4) and 2 (lane % 4) + 1)
__device__ __forceinline__ void dmma_m8n8k4(double (&d)[2], double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

constexpr int kWideThreads = 128;
constexpr int kWideWarps = kWideThreads / 32;
constexpr int kWideRounds = 4;          // rounds of 32 cells whose loads are in flight together

__global__ void __launch_bounds__(kWideThreads) k_wide_block_warp(Args a)
{
    __shared__ double s_u[kWideWarps][32][kWideWarp + 1];
    __shared__ double s_w[kWideWarps][32][kWideWarp + 1];
    __shared__ int64_t s_gs[kWideWarps][33];
    __shared__ double s_stage[kWideWarps][32];
    __shared__ double s_acc[kWideWarps][kWideWarp * kWideWarp];
    __shared__ unsigned s_pat[kWideWarps][kWideWarp];
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    const int W = (int)a.W;
    const int E = W * W;
    double (*u)[kWideWarp + 1] = s_u[wl];
    double (*wv)[kWideWarp + 1] = s_w[wl];
    int64_t *gs = s_gs[wl];
    // sum over groups of (u_a / N_g) u_b as 8 x 8 tiles (ta, tb) of the 16 x 16
    // block: this lane holds entries (8 ta + lane / 4, 8 tb + 2 (lane % 4) + i)
    double acc[2][2][2] = {};
    const int r8 = lane >> 2, c4 = lane & 3;
    double dsum = 0.0;          // lane a < W: sum of u_a
    const int wdims = (int)(a.ctr[7] >> 8) & 0xff;     // dimensions with wide levels
    unsigned pat = 0;           // lane a < W: levels sharing a group with a
    const int64_t chunks = (a.G + 31) / 32;
    const int64_t wstep = (int64_t)gridDim.x * kWideWarps;
    for (int64_t ch = (int64_t)blockIdx.x * kWideWarps + wl; ch < chunks; ch += wstep) {
        const int64_t g0 = ch * 32;
        const int ng = (int)min((int64_t)32, a.G - g0);
        gs[lane] = a.starts[g0 + min(lane, ng)];
        if (lane == 0) gs[32] = a.starts[g0 + ng];
        for (int q = lane; q < 32 * (kWideWarp + 1); q += 32) (&u[0][0])[q] = 0.0;
        __syncwarp();
        const int64_t c0 = gs[0], c1 = gs[ng];
        // the chunk's cells, kWideRounds rounds of 32 at a time: every round's
        // loads (n, the codes and their levels' wide indices) issued before the first is used
        for (int64_t b0 = c0; b0 < c1; b0 += 32 * kWideRounds) {
          int gqr[kWideRounds];
          double nir[kWideRounds];
          int32_t kr[kWideRounds][HDFE_MAX_DIMS];
#pragma unroll
          for (int t = 0; t < kWideRounds; t++) {
            const int64_t i = b0 + 32 * t + lane;
            const bool valid = i < c1;
            gqr[t] = 0;
            nir[t] = 0.0;
#pragma unroll
            for (int d = 0; d < HDFE_MAX_DIMS; d++) kr[t][d] = -1;
            if (valid) {
                int lo = 0, hi = ng;        // last group with start <= i
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (gs[mid] <= i) lo = mid; else hi = mid;
                }
                gqr[t] = lo;
                nir[t] = a.n[i];
#pragma unroll
                for (int d = 0; d < HDFE_MAX_DIMS; d++)
                    if (d < a.D && ((wdims >> d) & 1)) {
                        const uint32_t c = a.codes[i * a.D + d];
                        const int32_t k = (int64_t)c < a.nlev[d] ? a.kind[a.offs[d] + c] : -1;
                        kr[t][d] = k >= 0 ? k : -1;
                    }
            }
          }
#pragma unroll
          for (int t = 0; t < kWideRounds; t++) {
            if (b0 + 32 * t >= c1) break;               // warp-uniform
            const int64_t i = b0 + 32 * t + lane;
            const bool valid = i < c1;
            const int gq = gqr[t];
            const double ni = nir[t];
            int ks[HDFE_MAX_DIMS], nk = 0;      // the cell's wide levels so far
#pragma unroll
            for (int d = 0; d < HDFE_MAX_DIMS; d++) {
                if (d >= a.D) break;
                if (!((wdims >> d) & 1)) continue;      // no wide level in this dimension
                const int32_t k = valid ? kr[t][d] : -1;
                const int key = k >= 0 ? gq * 32 + k : -1 - lane;
                const unsigned peers = __match_any_sync(0xffffffffu, key);
                s_stage[wl][lane] = ni;
                __syncwarp();
                if (k >= 0 && lane == __ffs(peers) - 1) {
                    double sum = 0.0;
                    for (unsigned p = peers; p; p &= p - 1) sum += s_stage[wl][__ffs(p) - 1];
                    u[gq][k] += sum;
                }
                if (k >= 0) {
                    // a cell with several wide levels: C(a, k) and C(k, a) for
                    // each wide level a of its earlier dimensions
                    for (int q = 0; q < nk; q++) {
                        atomicAdd(a.wcross + (int64_t)ks[q] * W + k, ni);
                        atomicAdd(a.wcross + (int64_t)k * W + ks[q], ni);
                    }
                    ks[nk++] = k;
                }
                __syncwarp();
            }
          }
        }
        __syncwarp();
        // each group's u / N_g and level mask; rows past the chunk's groups
        // and columns past W are zeros (the tiles below read them)
        unsigned mask = 0;
        {
            const double inv = lane < ng ? 1.0 / a.group_n[g0 + lane] : 0.0;
            for (int k = 0; k < kWideWarp; k++) {
                const double x = (lane < ng && k < W) ? u[lane][k] : 0.0;
                wv[lane][k] = x * inv;
                if (x > 0.0) mask |= 1u << k;
            }
        }
        __syncwarp();
        for (int q = 0; q < ng; q++) {
            const unsigned mq = __shfl_sync(0xffffffffu, mask, q);
            if (lane < W) {
                if ((mq >> lane) & 1u) pat |= mq;
                dsum += u[q][lane];
            }
        }
        // the chunk's products on the FP64 tensor cores: A (a x group) = u / N_g
        // transposed, B (group x b) = u, four groups a step
#pragma unroll
        for (int ks = 0; ks < 8; ks++) {
            if (ks * 4 >= ng) break;                    // warp-uniform
            const int q = ks * 4 + c4;
            const double a0 = wv[q][r8], a1 = wv[q][8 + r8];
            const double b0 = u[q][r8], b1 = u[q][8 + r8];
            dmma_m8n8k4(acc[0][0], a0, b0);
            dmma_m8n8k4(acc[0][1], a0, b1);
            dmma_m8n8k4(acc[1][0], a1, b0);
            dmma_m8n8k4(acc[1][1], a1, b1);
        }
        __syncwarp();
    }
    // the warp's entries, then the CTA's warps summed in order
#pragma unroll
    for (int ta = 0; ta < 2; ta++)
#pragma unroll
        for (int tb = 0; tb < 2; tb++)
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const int ra = 8 * ta + r8, rb = 8 * tb + 2 * c4 + i;
                if (ra < W && rb < W) s_acc[wl][ra * W + rb] = -acc[ta][tb][i];
            }
    if (lane < W) s_pat[wl][lane] = pat;
    __syncwarp();
    if (lane < W) s_acc[wl][lane * W + lane] += dsum;
    __syncthreads();
    for (int en = threadIdx.x; en < E; en += kWideThreads) {
        double sum = 0.0;
        uint8_t p = 0;
        const int ra = en / W, rb = en % W;
        for (int w = 0; w < kWideWarps; w++) {
            sum += s_acc[w][en];
            p |= (uint8_t)((s_pat[w][ra] >> rb) & 1u);
        }
        a.wpart[(int64_t)blockIdx.x * E + en] = sum;
        a.wpres[(int64_t)blockIdx.x * E + en] = p;
    }
}

// per entry: the CTAs' partial sums in CTA order (one warp per entry)
__global__ void __launch_bounds__(kThreads) k_wide_block_reduce(Args a)
{
    const int lane = threadIdx.x & 31;
    const int64_t E = a.W * a.W;
    const int64_t warps = (int64_t)gridDim.x * (kThreads / 32);
    for (int64_t en = ((int64_t)blockIdx.x * kThreads + threadIdx.x) / 32; en < E; en += warps) {
        double sum = 0.0;
        unsigned p = 0;
        for (int64_t b = lane; b < a.wide_ctas; b += 32) {
            sum += a.wpart[b * E + en];
            p |= a.wpres[b * E + en];
        }
        sum = warp_sum(sum);
        p = __any_sync(0xffffffffu, p != 0);
        if (a.small_first < a.L) {          // split form: the dense small block
            if (lane == 0) a.smallb[en] = sum + a.wcross[en];
            continue;
        }
        if (!p || lane != 0) continue;
        const int64_t wa = en / a.W, wb = en % a.W;
        const int64_t lb = a.wide_list[wb];
        a.dval[wa * a.L + lb] = sum + a.wcross[en];
        a.dpres[wa * a.L + lb] = 1;
    }
}

// the wide x wide block for W > 16: atomics into the dense buffer
__global__ void __launch_bounds__(kThreads) k_wide_block_atomic(Args a)
{
    for (int64_t g = (int64_t)blockIdx.x * kThreads + threadIdx.x; g < a.G;
         g += (int64_t)gridDim.x * kThreads) {
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        const double Ng = a.group_n[g];
        for (int da = 0; da < a.D; da++) {
            for (int64_t ia = s; ia < e; ia++) {
                const int32_t wa = a.cell_widx[ia * a.D + da];
                if (wa < 0) continue;
                bool first = true;
                for (int64_t j = s; j < ia; j++)
                    if (a.cell_widx[j * a.D + da] == wa) { first = false; break; }
                if (!first) continue;
                double u = 0.0;
                for (int64_t i = s; i < e; i++)
                    if (a.cell_widx[i * a.D + da] == wa) u += a.n[i];
                const double wv = u / Ng;
                for (int64_t i = s; i < e; i++) {
                    const double ni = a.n[i];
                    double v = 0.0;
                    v -= ni * wv;
                    if (a.cell_widx[i * a.D + da] == wa) v += ni;
                    for (int d = 0; d < a.D; d++) {
                        const int32_t wb = a.cell_widx[i * a.D + d];
                        if (wb < 0) continue;
                        const int64_t lb = a.wide_list[wb];
                        atomicAdd(a.dval + (int64_t)wa * a.L + lb, v);
                        a.dpres[(int64_t)wa * a.L + lb] = 1;
                    }
                }
            }
        }
    }
}

// present columns of each wide row, per segment of kSeg columns
__global__ void __launch_bounds__(kThreads) k_wide_count(Args a)
{
    __shared__ double s_red[kThreads / 32];
    const int64_t jobs = a.W * a.nseg;
    for (int64_t job = blockIdx.x; job < jobs; job += gridDim.x) {
        const int64_t wi = job / a.nseg, sg = job % a.nseg;
        const uint8_t *p = a.dpres + wi * a.L;
        const int64_t c0 = sg * kSeg, c1 = min(c0 + kSeg, a.L);
        int64_t c = 0;
        for (int64_t j = c0 + threadIdx.x; j < c1; j += kThreads) c += p[j];
        const double t = block_sum((double)c, s_red);
        if (threadIdx.x == 0) {
            a.segcnt[job] = (int64_t)t;
            atomicAdd(reinterpret_cast<unsigned long long *>(a.rnnz + a.wide_list[wi]),
                      (unsigned long long)t);
        }
    }
}

// each (wide row, segment): compaction of the dense segment, in column order
__global__ void __launch_bounds__(kThreads) k_wide_fill(Args a)
{
    __shared__ int s_scr[kThreads / 32 + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t jobs = a.W * a.nseg;
    for (int64_t job = blockIdx.x; job < jobs; job += gridDim.x) {
        const int64_t wi = job / a.nseg, sg = job % a.nseg;
        const int64_t r = a.wide_list[wi];
        int64_t at = a.indptr[r];
        for (int64_t s2 = 0; s2 < sg; s2++) at += a.segcnt[wi * a.nseg + s2];
        const uint8_t *p = a.dpres + wi * a.L;
        const double *v = a.dval + wi * a.L;
        const int64_t c0 = sg * kSeg, c1 = min(c0 + kSeg, a.L);
        for (int64_t base = c0; base < c1; base += kThreads) {
            const int64_t j = base + threadIdx.x;
            const int has = (j < c1) ? p[j] : 0;
            const unsigned m = __ballot_sync(0xffffffffu, has);
            if (lane == 0) s_scr[warp] = __popc(m);
            __syncthreads();
            if (threadIdx.x == 0) {
                int run = 0;
                for (int w = 0; w < kThreads / 32; w++) { int t = s_scr[w]; s_scr[w] = run; run += t; }
                s_scr[kThreads / 32] = run;
            }
            __syncthreads();
            if (has) {
                const int64_t q = at + s_scr[warp] + __popc(m & ((1u << lane) - 1));
                a.indices[q] = (int32_t)j;
                a.data[q] = v[j];
            }
            at += s_scr[kThreads / 32];
            __syncthreads();
        }
    }
}

__global__ void k_write_info(Args a, hdfe_sbuild_info *info)
{
    if (threadIdx.x != 0) return;
    info->L = a.L;
    info->n_wide = a.ctr[0];
    info->n_warp_rows = a.ctr[1] + a.ctr[6];
    info->n_block_rows = a.ctr[2];
    info->lgrp_len = a.ctr[3];
    info->nnz = a.ctr[4];
    info->temp_len = a.ctr[5];
    info->status = (int64_t)*a.status;
}

// --------------------------------------------------------------- host

struct Layout {
    int64_t lcount, work, kind, lptr, fillpos, lgrp, lwv, rnnz, toff, wide_list, warp_rows,
        block_rows, tiles, ctr, status, total;
};

inline Layout layout(int64_t L, int64_t M, int D)
{
    Layout o;
    int64_t p = 0;
    auto take = [&](int64_t bytes) { int64_t at = p; p += (bytes + 255) / 256 * 256; return at; };
    o.lcount = take(L * 4);
    o.work = take(L * 8);
    o.kind = take(L * 4);
    o.lptr = take((L + 1) * 8);
    o.fillpos = take(L * 4);
    o.lgrp = take(M * (int64_t)D * 4);
    o.lwv = take(M * (int64_t)D * 8);
    o.rnnz = take((L + 1) * 8);
    o.toff = take((L + 1) * 8);
    o.wide_list = take(L * 4);
    o.warp_rows = take(L * 4);
    o.block_rows = take(L * 4);
    o.tiles = take(((L + 1) / kScanTile + 2) * 8);
    o.ctr = take(8 * 8);
    o.status = take(8);
    o.total = p;
    return o;
}

struct WideLayout {
    int64_t dval, dpres, widx, wpart, wpres, wcross, segcnt, total;
};

inline int64_t wide_ctas_for(int sms) { return (int64_t)sms * 4; }

inline WideLayout wide_layout(int64_t W, int64_t L, int64_t M, int D, int64_t ctas)
{
    WideLayout o;
    int64_t p = 0;
    auto take = [&](int64_t bytes) { int64_t at = p; p += (bytes + 255) / 256 * 256; return at; };
    const int64_t nseg = (L + kSeg - 1) / kSeg;
    o.dval = take(W * L * 8);
    o.dpres = take(W * L);
    o.widx = take(M * (int64_t)D * 4);
    o.wpart = take(ctas * W * W * 8);
    o.wpres = take(ctas * W * W);
    o.wcross = take(W * W * 8);
    o.segcnt = take(W * nseg * 8);
    o.total = p + 256;
    return o;
}

struct Ctx {
    Args a;
    cudaStream_t s;
    int sms;
};

int setup(Ctx &c, const int64_t *starts, int64_t G, const uint32_t *codes, int32_t D,
          const double *n, const double *group_n, int64_t M, const int64_t *n_levels,
          const int32_t *lcount, const int64_t *work, void *ws, int64_t ws_bytes)
{
    // empty arrays may come as null pointers (no identifying group or cell)
    if (D < 1 || D > HDFE_MAX_DIMS || G < 0 || M < 0 || !starts || (M > 0 && (!codes || !n)) ||
        (G > 0 && !group_n) || !n_levels || !ws || ((lcount == nullptr) != (work == nullptr)))
        return hdfe_set_arg_error("hdfe_sbuild: bad argument");
    Args &a = c.a;
    a = Args{};
    a.starts = starts;
    a.G = G;
    a.codes = codes;
    a.n = n;
    a.group_n = group_n;
    a.M = M;
    a.D = D;
    int64_t L = 0;
    for (int d = 0; d < D; d++) {
        if (n_levels[d] < 1) return hdfe_set_arg_error("hdfe_sbuild: n_levels must be >= 1");
        a.offs[d] = L;
        a.nlev[d] = n_levels[d];
        L += n_levels[d];
    }
    if (L >= INT32_MAX) return hdfe_set_arg_error("hdfe_sbuild: more than 2^31 levels");
    a.L = L;
    a.small_first = L;
    Layout lay = layout(L, M, D);
    if (ws_bytes < lay.total) return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_sbuild: workspace too small");
    char *b = (char *)ws;
    a.lcount_ws = (int32_t *)(b + lay.lcount);
    a.work_ws = (unsigned long long *)(b + lay.work);
    a.lcount = lcount ? lcount : a.lcount_ws;
    a.work = work ? reinterpret_cast<const unsigned long long *>(work) : a.work_ws;
    a.kind = (int32_t *)(b + lay.kind);
    a.lptr = (int64_t *)(b + lay.lptr);
    a.fillpos = (int32_t *)(b + lay.fillpos);
    a.lgrp = (int32_t *)(b + lay.lgrp);
    a.lwv = (double *)(b + lay.lwv);
    a.rnnz = (int64_t *)(b + lay.rnnz);
    a.toff = (int64_t *)(b + lay.toff);
    a.wide_list = (int32_t *)(b + lay.wide_list);
    a.warp_rows = (int32_t *)(b + lay.warp_rows);
    a.block_rows = (int32_t *)(b + lay.block_rows);
    a.tiles = (int64_t *)(b + lay.tiles);
    a.ctr = (int64_t *)(b + lay.ctr);
    a.status = (unsigned *)(b + lay.status);
    int dev = 0;
    HDFE_CUDA_TRY(cudaGetDevice(&dev));
    HDFE_CUDA_TRY(cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, dev));
    return HDFE_OK;
}

int set_wide(Ctx &c, int64_t W, void *wide_ws, int64_t wide_bytes_given)
{
    Args &a = c.a;
    a.W = W;
    a.nseg = (a.L + kSeg - 1) / kSeg;
    a.wide_ctas = wide_ctas_for(c.sms);
    if (W == 0) return HDFE_OK;
    WideLayout wl = wide_layout(W, a.L, a.M, a.D, a.wide_ctas);
    if (!wide_ws || wide_bytes_given < wl.total)
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_sbuild: wide workspace too small");
    char *b = (char *)wide_ws;
    a.dval = (double *)(b + wl.dval);
    a.dpres = (uint8_t *)(b + wl.dpres);
    a.cell_widx = (int32_t *)(b + wl.widx);
    a.wpart = (double *)(b + wl.wpart);
    a.wpres = (uint8_t *)(b + wl.wpres);
    a.wcross = (double *)(b + wl.wcross);
    a.segcnt = (int64_t *)(b + wl.segcnt);
    return HDFE_OK;
}

int set_temp(Ctx &c, void *temp, int64_t temp_bytes, int64_t temp_len)
{
    if (temp_len < 0 || (temp_len > 0 && (!temp || temp_bytes < temp_len * 12)))
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_sbuild: temp buffer too small");
    c.a.tval = (double *)temp;
    c.a.tcol = (int32_t *)((char *)temp + temp_len * 8);
    return HDFE_OK;
}

int scan_exclusive(Ctx &c, int64_t *x, int64_t n, int64_t *out, int64_t *total)
{
    const int64_t nt = (n + kScanTile - 1) / kScanTile;
    k_scan_tiles<<<(unsigned)nt, kThreads, 0, c.s>>>(x, n, c.a.tiles);
    k_scan_top<<<1, 1024, 0, c.s>>>(c.a.tiles, nt, total);
    k_scan_apply<<<(unsigned)nt, kThreads, 0, c.s>>>(x, n, c.a.tiles, out, total);
    HDFE_CUDA_TRY(cudaGetLastError());
    return HDFE_OK;
}

// the split form: levels [small_first, L) (the trailing dimensions' levels,
// at most kCross of them) are the small levels
int set_split(Ctx &c, int64_t small_first, int32_t small_count, double *cross, double *small)
{
    Args &a = c.a;
    bool at_dim = false;
    for (int d = 0; d < a.D; d++) at_dim |= a.offs[d] == small_first;
    if (small_count < 1 || small_count > kCross || small_first < 1 ||
        small_first + small_count != a.L || !at_dim)
        return hdfe_set_arg_error("hdfe_sbuild_*_split: the small levels must be the trailing "
                                  "dimensions' levels, 1 to 16 of them, after at least one other");
    a.small_first = small_first;
    a.ns = small_count;
    a.cross = cross;
    a.smallb = small;
    return HDFE_OK;
}

inline unsigned grid_for(int64_t items, int per_cta, int cap)
{
    int64_t b = (items + per_cta - 1) / per_cta;
    if (b > cap) b = cap;
    return (unsigned)(b > 0 ? b : 1);
}

}  // namespace sbuild
}  // namespace hdfe

using namespace hdfe;
using namespace hdfe::sbuild;

extern "C" int64_t hdfe_sbuild_workspace_bytes(int64_t L, int64_t n_cells, int32_t D)
{
    if (L < 1 || n_cells < 0 || D < 1 || D > HDFE_MAX_DIMS) return -1;
    return layout(L, n_cells, D).total;
}

extern "C" int64_t hdfe_sbuild_wide_workspace_bytes(int64_t L, int64_t n_cells, int32_t D,
                                                    int64_t n_wide)
{
    if (L < 1 || n_cells < 0 || D < 1 || D > HDFE_MAX_DIMS || n_wide < 0) return -1;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return -1;
    return wide_layout(n_wide, L, n_cells, D, wide_ctas_for(sms)).total;
}

static int analyze_impl(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                        int32_t D, const double *n, const double *group_n, int64_t n_cells,
                        const int64_t *n_levels, const int32_t *lcount, const int64_t *work,
                        void *workspace, int64_t workspace_bytes, hdfe_sbuild_info *info,
                        void *stream, int64_t small_first, int32_t small_count)
{
    Ctx c;
    c.s = (cudaStream_t)stream;
    int st = setup(c, starts, n_groups, codes, D, n, group_n, n_cells, n_levels, lcount, work,
                   workspace, workspace_bytes);
    if (st != HDFE_OK) return st;
    if (small_count > 0 &&
        (st = set_split(c, small_first, small_count, nullptr, nullptr)) != HDFE_OK)
        return st;
    Args &a = c.a;
    Layout lay = layout(a.L, n_cells, D);
    char *b = (char *)workspace;
    int launched = 0;
    if (!lcount) {
        HDFE_CUDA_TRY(cudaMemsetAsync(b + lay.lcount, 0, a.L * 4, c.s));
        HDFE_CUDA_TRY(cudaMemsetAsync(b + lay.work, 0, a.L * 8, c.s));
    }
    HDFE_CUDA_TRY(cudaMemsetAsync(b + lay.fillpos, 0, a.L * 4, c.s));
    HDFE_CUDA_TRY(cudaMemsetAsync(b + lay.ctr, 0, 64, c.s));
    HDFE_CUDA_TRY(cudaMemsetAsync(b + lay.status, 0, 8, c.s));
    const int cap = c.sms * 8;
    if (!lcount) {
        k_level_stats<<<grid_for(a.G, kThreads, cap), kThreads, 0, c.s>>>(a);
        launched++;
    }
    k_classify<<<grid_for(a.L, kThreads, cap), kThreads, 0, c.s>>>(a);
    k_sort_wide<<<1, 32, 0, c.s>>>(a);
    HDFE_CUDA_TRY(cudaGetLastError());
    if ((st = scan_exclusive(c, a.lptr, a.L, a.lptr, a.ctr + 3)) != HDFE_OK) return st;
    if ((st = scan_exclusive(c, a.toff, a.L, a.toff, a.ctr + 5)) != HDFE_OK) return st;
    {
        const size_t smem = list_smem(a.D);
        HDFE_CUDA_TRY(cudaFuncSetAttribute(k_fill_lists,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per = 0;
        HDFE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_fill_lists,
                                                                  kListWarps * 32, smem));
        const int64_t ctas = ((a.G + 31) / 32 + kListWarps - 1) / kListWarps;
        k_fill_lists<<<grid_for(ctas, 1, c.sms * (per > 0 ? per : 1)), kListWarps * 32, smem,
                       c.s>>>(a);
    }
    k_write_info<<<1, 32, 0, c.s>>>(a, info);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(launched + 11);
    return HDFE_OK;
}

extern "C" int hdfe_sbuild_analyze(const int64_t *starts, int64_t n_groups,
                                   const uint32_t *codes, int32_t D, const double *n,
                                   const double *group_n, int64_t n_cells,
                                   const int64_t *n_levels, const int32_t *lcount,
                                   const int64_t *work, void *workspace,
                                   int64_t workspace_bytes, hdfe_sbuild_info *info, void *stream)
{
    return analyze_impl(starts, n_groups, codes, D, n, group_n, n_cells, n_levels, lcount, work,
                        workspace, workspace_bytes, info, stream, 0, 0);
}

extern "C" int hdfe_sbuild_analyze_split(const int64_t *starts, int64_t n_groups,
                                         const uint32_t *codes, int32_t D, const double *n,
                                         const double *group_n, int64_t n_cells,
                                         const int64_t *n_levels, const int32_t *lcount,
                                         const int64_t *work, int64_t small_first,
                                         int32_t small_count, void *workspace,
                                         int64_t workspace_bytes, hdfe_sbuild_info *info,
                                         void *stream)
{
    if (small_count < 1) return hdfe_set_arg_error("hdfe_sbuild_analyze_split: small_count < 1");
    return analyze_impl(starts, n_groups, codes, D, n, group_n, n_cells, n_levels, lcount, work,
                        workspace, workspace_bytes, info, stream, small_first, small_count);
}

static int count_impl(const int64_t *starts, int64_t n_groups, const uint32_t *codes, int32_t D,
                      const double *n, const double *group_n, int64_t n_cells,
                      const int64_t *n_levels, const int32_t *lcount, const int64_t *work,
                      int64_t n_wide, int64_t temp_len, int64_t *indptr, void *workspace,
                      int64_t workspace_bytes, void *wide_workspace, int64_t wide_workspace_bytes,
                      void *temp, int64_t temp_bytes, hdfe_sbuild_info *info, void *stream,
                      int64_t small_first, int32_t small_count, double *cross, double *small)
{
    Ctx c;
    c.s = (cudaStream_t)stream;
    int st = setup(c, starts, n_groups, codes, D, n, group_n, n_cells, n_levels, lcount, work,
                   workspace, workspace_bytes);
    if (st != HDFE_OK) return st;
    const bool split = small_count > 0;
    if (split) {
        if ((st = set_split(c, small_first, small_count, cross, small)) != HDFE_OK) return st;
        if (!cross || !small || n_wide != small_count)
            return hdfe_set_arg_error("hdfe_sbuild_count_split: cross / small missing, or "
                                      "n_wide is not the number of small levels");
    }
    if ((st = set_wide(c, n_wide, wide_workspace, wide_workspace_bytes)) != HDFE_OK) return st;
    if ((st = set_temp(c, temp, temp_bytes, temp_len)) != HDFE_OK) return st;
    if (!indptr) return hdfe_set_arg_error("hdfe_sbuild_count: indptr is null");
    Args &a = c.a;
    a.indptr = indptr;
    int launched = 0;
    if (split) {
        HDFE_CUDA_TRY(cudaMemsetAsync(cross, 0, small_first * kCross * 8, c.s));
        HDFE_CUDA_TRY(cudaMemsetAsync(small, 0, (int64_t)small_count * small_count * 8, c.s));
    }
    if (n_wide > 0) {
        WideLayout wl = wide_layout(n_wide, a.L, a.M, a.D, a.wide_ctas);
        if (!split)     // the dense wide rows (the split form writes cross instead)
            HDFE_CUDA_TRY(cudaMemsetAsync(wide_workspace, 0, wl.dpres + n_wide * a.L, c.s));
        HDFE_CUDA_TRY(cudaMemsetAsync((char *)wide_workspace + wl.wcross, 0,
                                      n_wide * n_wide * 8, c.s));
        if (n_wide > kWideWarp) {       // the atomic wide block reads each cell's wide index
            k_cell_widx<<<grid_for(a.M * a.D, kThreads, c.sms * 8), kThreads, 0, c.s>>>(a);
            launched++;
        }
    }
    HDFE_CUDA_TRY(cudaMemsetAsync(a.rnnz, 0, (a.L + 1) * 8, c.s));
    // one wave: as many CTAs as stay resident (the rows are grid-strided, so a
    // second partial wave would run its share of rows after the first)
    int per_small = 0, per_warp = 0;
    HDFE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_small, k_small_rows,
                                                              kSmallWarpsPerCta * 32, 0));
    HDFE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_warp, k_warp_rows,
                                                              kWarpsPerCta * 32, 0));
    k_small_rows<<<(unsigned)(c.sms * (per_small > 0 ? per_small : 1)), kSmallWarpsPerCta * 32, 0,
                   c.s>>>(a);
    k_warp_rows<<<(unsigned)(c.sms * (per_warp > 0 ? per_warp : 1)), kWarpsPerCta * 32, 0,
                  c.s>>>(a);
    HDFE_CUDA_TRY(cudaFuncSetAttribute(k_block_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kBlockSmem));
    k_block_rows<<<(unsigned)(c.sms), 32, kBlockSmem, c.s>>>(a);
    launched += 3;
    if (n_wide > 0) {
        if (n_wide <= kWideWarp) {
            k_wide_block_warp<<<(unsigned)a.wide_ctas, kWideThreads, 0, c.s>>>(a);
            k_wide_block_reduce<<<grid_for(n_wide * n_wide * 32, kThreads, 64), kThreads, 0, c.s>>>(a);
            launched += 2;
        } else {
            k_wide_block_atomic<<<(unsigned)(c.sms * 8), kThreads, 0, c.s>>>(a);
            launched++;
        }
        if (!split) {
            k_wide_count<<<grid_for(n_wide * a.nseg, 1, c.sms * 8), kThreads, 0, c.s>>>(a);
            launched++;
        }
    }
    HDFE_CUDA_TRY(cudaGetLastError());
    if ((st = scan_exclusive(c, a.rnnz, a.L, indptr, a.ctr + 4)) != HDFE_OK) return st;
    k_write_info<<<1, 32, 0, c.s>>>(a, info);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(launched + 4);
    return HDFE_OK;
}

extern "C" int hdfe_sbuild_count(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                                 int32_t D, const double *n, const double *group_n,
                                 int64_t n_cells, const int64_t *n_levels, const int32_t *lcount,
                                 const int64_t *work, int64_t n_wide, int64_t temp_len,
                                 int64_t *indptr, void *workspace, int64_t workspace_bytes,
                                 void *wide_workspace, int64_t wide_workspace_bytes, void *temp,
                                 int64_t temp_bytes, hdfe_sbuild_info *info, void *stream)
{
    return count_impl(starts, n_groups, codes, D, n, group_n, n_cells, n_levels, lcount, work,
                      n_wide, temp_len, indptr, workspace, workspace_bytes, wide_workspace,
                      wide_workspace_bytes, temp, temp_bytes, info, stream, 0, 0, nullptr,
                      nullptr);
}

extern "C" int hdfe_sbuild_count_split(const int64_t *starts, int64_t n_groups,
                                       const uint32_t *codes, int32_t D, const double *n,
                                       const double *group_n, int64_t n_cells,
                                       const int64_t *n_levels, const int32_t *lcount,
                                       const int64_t *work, int64_t n_wide, int64_t temp_len,
                                       int64_t small_first, int32_t small_count, int64_t *indptr,
                                       double *cross, double *small, void *workspace,
                                       int64_t workspace_bytes, void *wide_workspace,
                                       int64_t wide_workspace_bytes, void *temp,
                                       int64_t temp_bytes, hdfe_sbuild_info *info, void *stream)
{
    if (small_count < 1) return hdfe_set_arg_error("hdfe_sbuild_count_split: small_count < 1");
    return count_impl(starts, n_groups, codes, D, n, group_n, n_cells, n_levels, lcount, work,
                      n_wide, temp_len, indptr, workspace, workspace_bytes, wide_workspace,
                      wide_workspace_bytes, temp, temp_bytes, info, stream, small_first,
                      small_count, cross, small);
}

static int fill_impl(const int64_t *starts, int64_t n_groups, const uint32_t *codes, int32_t D,
                     const double *n, const double *group_n, int64_t n_cells,
                     const int64_t *n_levels, const int32_t *lcount, const int64_t *work,
                     int64_t n_wide, int64_t temp_len, const int64_t *indptr, int32_t *indices,
                     double *data, void *workspace, int64_t workspace_bytes, void *wide_workspace,
                     int64_t wide_workspace_bytes, void *temp, int64_t temp_bytes,
                     hdfe_sbuild_info *info, void *stream, bool split)
{
    Ctx c;
    c.s = (cudaStream_t)stream;
    int st = setup(c, starts, n_groups, codes, D, n, group_n, n_cells, n_levels, lcount, work,
                   workspace, workspace_bytes);
    if (st != HDFE_OK) return st;
    if ((st = set_wide(c, n_wide, wide_workspace, wide_workspace_bytes)) != HDFE_OK) return st;
    if ((st = set_temp(c, temp, temp_bytes, temp_len)) != HDFE_OK) return st;
    if (!indptr || !indices || !data) return hdfe_set_arg_error("hdfe_sbuild_fill: null output");
    Args &a = c.a;
    a.indptr = const_cast<int64_t *>(indptr);
    a.indices = indices;
    a.data = data;
    k_copy_narrow<<<(unsigned)(c.sms * 8), kThreads, 0, c.s>>>(a);
    int launched = 1;
    if (n_wide > 0 && !split) {
        k_wide_fill<<<grid_for(n_wide * a.nseg, 1, c.sms * 8), kThreads, 0, c.s>>>(a);
        launched++;
    }
    k_write_info<<<1, 32, 0, c.s>>>(a, info);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(launched + 1);
    return HDFE_OK;
}

extern "C" int hdfe_sbuild_fill(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                                int32_t D, const double *n, const double *group_n,
                                int64_t n_cells, const int64_t *n_levels, const int32_t *lcount,
                                const int64_t *work, int64_t n_wide, int64_t temp_len,
                                const int64_t *indptr, int32_t *indices, double *data,
                                void *workspace, int64_t workspace_bytes, void *wide_workspace,
                                int64_t wide_workspace_bytes, void *temp, int64_t temp_bytes,
                                hdfe_sbuild_info *info, void *stream)
{
    return fill_impl(starts, n_groups, codes, D, n, group_n, n_cells, n_levels, lcount, work,
                     n_wide, temp_len, indptr, indices, data, workspace, workspace_bytes,
                     wide_workspace, wide_workspace_bytes, temp, temp_bytes, info, stream, false);
}

extern "C" int hdfe_sbuild_fill_split(const int64_t *starts, int64_t n_groups,
                                      const uint32_t *codes, int32_t D, const double *n,
                                      const double *group_n, int64_t n_cells,
                                      const int64_t *n_levels, const int32_t *lcount,
                                      const int64_t *work, int64_t n_wide, int64_t temp_len,
                                      const int64_t *indptr, int32_t *indices, double *data,
                                      void *workspace, int64_t workspace_bytes,
                                      void *wide_workspace, int64_t wide_workspace_bytes,
                                      void *temp, int64_t temp_bytes, hdfe_sbuild_info *info,
                                      void *stream)
{
    return fill_impl(starts, n_groups, codes, D, n, group_n, n_cells, n_levels, lcount, work,
                     n_wide, temp_len, indptr, indices, data, workspace, workspace_bytes,
                     wide_workspace, wide_workspace_bytes, temp, temp_bytes, info, stream, true);
}
