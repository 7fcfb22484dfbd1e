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
// B200 mapping:
//   analyze     one thread per group: the distinct levels of the group (first
//               occurrences) -> per-level group count and work (cells
//               scanned to build the row), as `_nb_level_groups` /
//               `_nb_row_work`.  Levels are then classed by work: "warp"
//               rows (one warp each, a 512-slot shared hash), "block" rows
//               (one CTA each, an 8192-slot hash) and "wide" rows (levels of
//               small dimensions, e.g. years, in most groups).
//   lists       the groups of each narrow level (level -> group index).
//   count/fill  narrow rows: a warp streams the row's groups (sorted, so the
//               sums have a fixed order) 32 cells at a time; lanes with the
//               same column are combined with __match_any_sync by their
//               lowest lane in lane order, then added to the row's hash
//               slot.  The fill pass sorts the row's (column, value) pairs
//               in shared memory (bitonic) and writes them at indptr[r].
//   wide rows   S is symmetric: a wide row's entries at narrow columns are
//               the narrow rows' entries at the wide column, stored into a
//               dense (wide x L) buffer by the narrow fill; the wide x wide
//               block is summed over all groups, privatised in shared memory
//               per CTA.  Each wide row is then a stream compaction of its
//               dense row, which leaves its columns sorted.
// Values are FP64 sums in a fixed order per row (narrow) or atomic order
// (wide x wide); the pattern and nnz are exact.
#include <cuda_runtime.h>

#include "common.cuh"

namespace hdfe {
namespace sbuild {

constexpr int kThreads = 256;
constexpr int kWarpSlots = 512;                 // hash slots per warp (warp rows)
constexpr int kBlockSlots = 8192;               // hash slots per CTA (block rows)
constexpr int kWarpListCap = 256;               // groups per warp row (sorted in smem)
constexpr int kBlockListCap = 4096;             // groups per block row
constexpr int32_t kEmptyKey = -1;
constexpr int32_t kKindEmpty = -1, kKindWarp = -2, kKindBlock = -3;
constexpr int kWideSmem = 64;                   // wide x wide block in smem up to this W
constexpr int kScanTile = 4096;

// work thresholds: distinct columns <= work * D must stay <= 3/4 of a table
__host__ __device__ inline int64_t warp_work(int D) { return (kWarpSlots * 3 / 4) / D; }
__host__ __device__ inline int64_t block_work(int D)
{
    int64_t by_slots = (kBlockSlots * 3 / 4) / D;
    return by_slots < kBlockListCap ? by_slots : kBlockListCap;
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
    // main workspace
    int32_t *lcount;
    unsigned long long *work;
    int32_t *kind;              // kKind* or the wide index
    int64_t *lptr;              // (L+1)
    int32_t *fillpos;
    int32_t *lgrp;
    int64_t *rnnz;              // (L+1) row nnz, then scanned
    int32_t *wide_list;         // wide index -> level
    int32_t *warp_rows, *block_rows;
    int64_t *tiles;             // scan partials
    int64_t *ctr;               // [0] W, [1] warp rows, [2] block rows, [3] lgrp len, [4] nnz
    unsigned *status;
    // wide workspace (count/fill only)
    double *dval;               // (W, L)
    uint8_t *dpres;             // (W, L)
    int64_t W;
    // output
    int64_t *indptr;
    int32_t *indices;
    double *data;
};

__device__ __forceinline__ int level_dim(const Args &a, int64_t r)
{
    int d = 0;
    while (d + 1 < a.D && a.offs[d + 1] <= r) d++;
    return d;
}

// ------------------------------------------------------------- analyze

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
                atomicAdd(a.lcount + lv, 1);
                atomicAdd(a.work + lv, size);
            }
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_classify(Args a)
{
    const int64_t ww = warp_work(a.D), bw = block_work(a.D);
    for (int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x; r < a.L;
         r += (int64_t)gridDim.x * kThreads) {
        const unsigned long long w = a.work[r];
        int32_t k;
        if (w == 0) k = kKindEmpty;
        else if ((int64_t)w <= ww && a.lcount[r] <= kWarpListCap) k = kKindWarp;
        else if ((int64_t)w <= bw && a.lcount[r] <= kBlockListCap) k = kKindBlock;
        else k = -100;
        if (k == kKindWarp) a.warp_rows[atomicAdd((unsigned long long *)(a.ctr + 1), 1ull)] = (int32_t)r;
        if (k == kKindBlock) a.block_rows[atomicAdd((unsigned long long *)(a.ctr + 2), 1ull)] = (int32_t)r;
        if (k == -100) {
            const int64_t wi = (int64_t)atomicAdd((unsigned long long *)a.ctr, 1ull);
            a.wide_list[wi] = (int32_t)r;
            k = (int32_t)wi;
        }
        a.kind[r] = k;
        // narrow levels keep their group lists
        a.lptr[r] = (k == kKindWarp || k == kKindBlock) ? a.lcount[r] : 0;
    }
}

// The wide list in level order, so a wide row's index does not depend on
// the atomic order above (one CTA; W is small).
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
    // integer sums stay exact in double up to 2^53
    double t = block_sum((double)s, s_red);
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

__global__ void __launch_bounds__(kThreads) k_fill_lists(Args a)
{
    for (int64_t g = (int64_t)blockIdx.x * kThreads + threadIdx.x; g < a.G;
         g += (int64_t)gridDim.x * kThreads) {
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        for (int d = 0; d < a.D; d++) {
            for (int64_t i = s; i < e; i++) {
                const uint32_t c = a.codes[i * a.D + d];
                if ((int64_t)c >= a.nlev[d]) continue;
                bool first = true;
                for (int64_t j = s; j < i; j++)
                    if (a.codes[j * a.D + d] == c) { first = false; break; }
                if (!first) continue;
                const int64_t lv = a.offs[d] + c;
                const int32_t k = a.kind[lv];
                if (k == kKindWarp || k == kKindBlock) {
                    const int32_t at = atomicAdd(a.fillpos + lv, 1);
                    a.lgrp[a.lptr[lv] + at] = (int32_t)g;
                }
            }
        }
    }
}

// ------------------------------------------------------- narrow rows

__device__ __forceinline__ uint32_t slot_of(int32_t col, int bits)
{
    return ((uint32_t)col * 2654435761u) >> (32 - bits);
}

// Sorts n (<= cap, cap a power of two) int32 keys in smem ascending, with
// an optional double payload; the tail up to cap is padded with INT32_MAX.
__device__ void bitonic_sort(int32_t *key, double *val, int n, int cap, int lane, int lanes,
                             bool block)
{
    int size = 1;
    while (size < n) size <<= 1;
    for (int i = n + lane; i < size; i += lanes) key[i] = INT32_MAX;
    if (block) __syncthreads(); else __syncwarp();
    for (int k = 2; k <= size; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < size; i += lanes) {
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
            if (block) __syncthreads(); else __syncwarp();
        }
    }
    (void)cap;
}

// One narrow row, processed by one warp.  `fill` false: count its distinct
// columns (and mark its wide columns); true: accumulate, sort, write.
// Shared buffers: keys/vals (slots), list (list_cap ints), stage (32 doubles).
__device__ void narrow_row(const Args &a, int64_t r, bool fill, int32_t *keys, double *vals,
                           int bits, int32_t *list, double *stage, int *s_cnt)
{
    const int lane = threadIdx.x & 31;
    const int slots = 1 << bits;
    const int dr = level_dim(a, r);
    const uint32_t lr = (uint32_t)(r - a.offs[dr]);
    for (int i = lane; i < slots; i += 32) { keys[i] = kEmptyKey; if (fill) vals[i] = 0.0; }
    // the row's groups, ascending
    const int64_t l0 = a.lptr[r];
    const int nl = (int)(a.lptr[r + 1] - l0);
    for (int i = lane; i < nl; i += 32) list[i] = a.lgrp[l0 + i];
    if (lane == 0) *s_cnt = 0;
    __syncwarp();
    bitonic_sort(list, nullptr, nl, 0, lane, 32, false);
    for (int li = 0; li < nl; li++) {
        const int64_t g = list[li];
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        // u_r over the group's cells
        double ur = 0.0;
        for (int64_t i = s + lane; i < e; i += 32)
            if (a.codes[i * a.D + dr] == lr) ur += a.n[i];
        ur = warp_sum(ur);
        const double wv = ur / a.group_n[g];
        for (int64_t base = s; base < e; base += 32) {
            const int64_t i = base + lane;
            const bool valid = i < e;
            double v = 0.0;
            if (valid) {
                const double ni = a.n[i];
                v -= ni * wv;
                if (a.codes[i * a.D + dr] == lr) v += ni;
            }
            for (int d = 0; d < a.D; d++) {
                const int32_t col = valid ? (int32_t)(a.offs[d] + a.codes[i * a.D + d]) : -1;
                const unsigned peers = __match_any_sync(0xffffffffu, col);
                const int leader = __ffs(peers) - 1;
                stage[lane] = v;
                __syncwarp();
                if (valid && lane == leader) {
                    double sum = 0.0;
                    for (unsigned p = peers; p; p &= p - 1) sum += stage[__ffs(p) - 1];
                    uint32_t h = slot_of(col, bits);
                    for (int probe = 0; probe < slots; probe++) {
                        const int32_t old = atomicCAS(keys + h, kEmptyKey, col);
                        if (old == kEmptyKey || old == col) {
                            if (old == kEmptyKey) atomicAdd(s_cnt, 1);
                            if (fill) vals[h] += sum;
                            break;
                        }
                        h = (h + 1) & (slots - 1);
                    }
                }
                __syncwarp();
            }
        }
    }
    __syncwarp();
    const int cnt = *s_cnt;
    if (!fill) {
        if (lane == 0) a.rnnz[r] = cnt;
        // mark the row's wide columns: the wide rows' entries at column r
        for (int i = lane; i < slots; i += 32) {
            const int32_t c = keys[i];
            if (c == kEmptyKey) continue;
            const int32_t k = a.kind[c];
            if (k >= 0) a.dpres[(int64_t)k * a.L + r] = 1;
        }
        return;
    }
    // compact the table to its first cnt slots, sort by column, write
    __syncwarp();
    if (lane == 0) *s_cnt = 0;
    __syncwarp();
    for (int base = 0; base < slots; base += 32) {
        const int i = base + lane;
        const int32_t c = keys[i];
        const double v = vals[i];
        const bool has = c != kEmptyKey;
        const unsigned m = __ballot_sync(0xffffffffu, has);
        const int before = __popc(m & ((1u << lane) - 1));
        int at0 = 0;
        if (lane == 0) at0 = *s_cnt;
        at0 = __shfl_sync(0xffffffffu, at0, 0);
        __syncwarp();
        // compacted entries never overtake the slots still to be read
        if (has) { keys[at0 + before] = c; vals[at0 + before] = v; }
        __syncwarp();
        if (lane == 0) *s_cnt = at0 + __popc(m);
        __syncwarp();
    }
    bitonic_sort(keys, vals, cnt, slots, lane, 32, false);
    const int64_t p0 = a.indptr[r];
    for (int i = lane; i < cnt; i += 32) {
        a.indices[p0 + i] = keys[i];
        a.data[p0 + i] = vals[i];
        const int32_t k = a.kind[keys[i]];
        if (k >= 0) a.dval[(int64_t)k * a.L + r] = vals[i];
    }
}

constexpr int kWarpsPerCta = 4;      // 4 x 7.4 KB of tables: static smem < 48 KB

__global__ void __launch_bounds__(kWarpsPerCta * 32) k_warp_rows(Args a, bool fill)
{
    __shared__ int32_t s_keys[kWarpsPerCta][kWarpSlots];
    __shared__ double s_vals[kWarpsPerCta][kWarpSlots];
    __shared__ int32_t s_list[kWarpsPerCta][kWarpListCap];
    __shared__ double s_stage[kWarpsPerCta][32];
    __shared__ int s_cnt[kWarpsPerCta];
    const int w = threadIdx.x >> 5;
    const int64_t nrows = a.ctr[1];
    const int bits = 9;     // log2(kWarpSlots)
    for (int64_t k = (int64_t)blockIdx.x * kWarpsPerCta + w; k < nrows;
         k += (int64_t)gridDim.x * kWarpsPerCta)
        narrow_row(a, a.warp_rows[k], fill, s_keys[w], s_vals[w], bits, s_list[w], s_stage[w],
                   &s_cnt[w]);
}

// block rows: one warp per CTA with the large table in dynamic smem
__global__ void __launch_bounds__(32) k_block_rows(Args a, bool fill)
{
    extern __shared__ unsigned char s_raw[];
    double *vals = reinterpret_cast<double *>(s_raw);
    int32_t *keys = reinterpret_cast<int32_t *>(vals + kBlockSlots);
    int32_t *list = keys + kBlockSlots;
    __shared__ double s_stage[32];
    __shared__ int s_cnt;
    const int64_t nrows = a.ctr[2];
    const int bits = 13;    // log2(kBlockSlots)
    for (int64_t k = blockIdx.x; k < nrows; k += gridDim.x)
        narrow_row(a, a.block_rows[k], fill, keys, vals, bits, list, s_stage, &s_cnt);
}

// ------------------------------------------------------- wide rows

// The wide x wide block: over all groups, for each wide level a in the group
// (first occurrence) and each cell i, v_i = n_i [i has a] - n_i u_a / N_g
// added to the wide columns of cell i.  Privatised per CTA when W <= 64.
__global__ void __launch_bounds__(kThreads) k_wide_block(Args a)
{
    __shared__ double s_acc[kWideSmem * kWideSmem];
    __shared__ uint8_t s_pres[kWideSmem * kWideSmem];
    const int64_t W = a.W;
    const bool priv = W <= kWideSmem;
    if (priv) {
        for (int i = threadIdx.x; i < W * W; i += kThreads) { s_acc[i] = 0.0; s_pres[i] = 0; }
        __syncthreads();
    }
    for (int64_t g = (int64_t)blockIdx.x * kThreads + threadIdx.x; g < a.G;
         g += (int64_t)gridDim.x * kThreads) {
        const int64_t s = a.starts[g], e = a.starts[g + 1];
        const double Ng = a.group_n[g];
        for (int da = 0; da < a.D; da++) {
            for (int64_t ia = s; ia < e; ia++) {
                const uint32_t ca = a.codes[ia * a.D + da];
                if ((int64_t)ca >= a.nlev[da]) continue;
                const int32_t wa = a.kind[a.offs[da] + ca];
                if (wa < 0) continue;
                bool first = true;
                for (int64_t j = s; j < ia; j++)
                    if (a.codes[j * a.D + da] == ca) { first = false; break; }
                if (!first) continue;
                double u = 0.0;
                for (int64_t i = s; i < e; i++)
                    if (a.codes[i * a.D + da] == ca) u += a.n[i];
                const double wv = u / Ng;
                for (int64_t i = s; i < e; i++) {
                    const double ni = a.n[i];
                    double v = 0.0;
                    v -= ni * wv;
                    if (a.codes[i * a.D + da] == ca) v += ni;
                    for (int d = 0; d < a.D; d++) {
                        const uint32_t cb = a.codes[i * a.D + d];
                        if ((int64_t)cb >= a.nlev[d]) continue;
                        const int64_t lb = a.offs[d] + cb;
                        const int32_t wb = a.kind[lb];
                        if (wb < 0) continue;
                        if (priv) {
                            atomicAdd(s_acc + wa * W + wb, v);
                            s_pres[wa * W + wb] = 1;
                        } else {
                            atomicAdd(a.dval + (int64_t)wa * a.L + lb, v);
                            a.dpres[(int64_t)wa * a.L + lb] = 1;
                        }
                    }
                }
            }
        }
    }
    if (!priv) return;
    __syncthreads();
    for (int i = threadIdx.x; i < W * W; i += kThreads) {
        if (!s_pres[i]) continue;
        const int64_t wa = i / W, wb = i % W;
        const int64_t lb = a.wide_list[wb];
        atomicAdd(a.dval + wa * a.L + lb, s_acc[i]);
        a.dpres[wa * a.L + lb] = 1;
    }
}

// nnz of each wide row: its present columns (one CTA per wide row)
__global__ void __launch_bounds__(kThreads) k_wide_count(Args a)
{
    __shared__ double s_red[kThreads / 32];
    for (int64_t wi = blockIdx.x; wi < a.W; wi += gridDim.x) {
        const uint8_t *p = a.dpres + wi * a.L;
        int64_t c = 0;
        for (int64_t j = threadIdx.x; j < a.L; j += kThreads) c += p[j];
        double t = block_sum((double)c, s_red);
        if (threadIdx.x == 0) a.rnnz[a.wide_list[wi]] = (int64_t)t;
    }
}

// write each wide row: compaction of its dense row, in column order
__global__ void __launch_bounds__(kThreads) k_wide_fill(Args a)
{
    __shared__ int s_scr[kThreads / 32 + 1];
    for (int64_t wi = blockIdx.x; wi < a.W; wi += gridDim.x) {
        const int64_t r = a.wide_list[wi];
        const uint8_t *p = a.dpres + wi * a.L;
        const double *v = a.dval + wi * a.L;
        int64_t at = a.indptr[r];
        for (int64_t base = 0; base < a.L; base += kThreads) {
            const int64_t j = base + threadIdx.x;
            const int has = (j < a.L) ? p[j] : 0;
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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
    info->n_warp_rows = a.ctr[1];
    info->n_block_rows = a.ctr[2];
    info->lgrp_len = a.ctr[3];
    info->nnz = a.ctr[4];
    info->status = (int64_t)*a.status;
}

// --------------------------------------------------------------- host

struct Layout {
    int64_t lcount, work, kind, lptr, fillpos, lgrp, rnnz, wide_list, warp_rows, block_rows,
        tiles, ctr, status, total;
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
    o.rnnz = take((L + 1) * 8);
    o.wide_list = take(L * 4);
    o.warp_rows = take(L * 4);
    o.block_rows = take(L * 4);
    o.tiles = take(((L + 1) / kScanTile + 2) * 8);
    o.ctr = take(8 * 8);
    o.status = take(8);
    o.total = p;
    return o;
}

inline int64_t wide_bytes(int64_t W, int64_t L) { return W * L * 9 + 256; }

struct Ctx {
    Args a;
    cudaStream_t s;
    int sms;
};

int setup(Ctx &c, const int64_t *starts, int64_t G, const uint32_t *codes, int32_t D,
          const double *n, const double *group_n, int64_t M, const int64_t *n_levels, void *ws,
          int64_t ws_bytes, void *wide_ws, int64_t wide_ws_bytes, int64_t W, void *stream)
{
    if (D < 1 || D > HDFE_MAX_DIMS || G < 0 || M < 0 || !starts || !codes || !n || !group_n ||
        !n_levels || !ws)
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
    Layout lay = layout(L, M, D);
    if (ws_bytes < lay.total) return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_sbuild: workspace too small");
    char *b = (char *)ws;
    a.lcount = (int32_t *)(b + lay.lcount);
    a.work = (unsigned long long *)(b + lay.work);
    a.kind = (int32_t *)(b + lay.kind);
    a.lptr = (int64_t *)(b + lay.lptr);
    a.fillpos = (int32_t *)(b + lay.fillpos);
    a.lgrp = (int32_t *)(b + lay.lgrp);
    a.rnnz = (int64_t *)(b + lay.rnnz);
    a.wide_list = (int32_t *)(b + lay.wide_list);
    a.warp_rows = (int32_t *)(b + lay.warp_rows);
    a.block_rows = (int32_t *)(b + lay.block_rows);
    a.tiles = (int64_t *)(b + lay.tiles);
    a.ctr = (int64_t *)(b + lay.ctr);
    a.status = (unsigned *)(b + lay.status);
    a.W = W;
    if (W >= 0) {
        if (W > 0 && (!wide_ws || wide_ws_bytes < wide_bytes(W, L)))
            return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_sbuild: wide workspace too small");
        a.dval = (double *)wide_ws;
        a.dpres = (uint8_t *)((char *)wide_ws + W * L * 8);
    }
    c.s = (cudaStream_t)stream;
    int dev = 0;
    HDFE_CUDA_TRY(cudaGetDevice(&dev));
    HDFE_CUDA_TRY(cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, dev));
    return HDFE_OK;
}

int scan_exclusive(Ctx &c, int64_t *x, int64_t n, int64_t *out, int64_t *total)
{
    const int64_t nt = (n + kScanTile - 1) / kScanTile;
    if (nt == 0) {
        HDFE_CUDA_TRY(cudaMemsetAsync(out, 0, 8, c.s));
        HDFE_CUDA_TRY(cudaMemsetAsync(total, 0, 8, c.s));
        return HDFE_OK;
    }
    k_scan_tiles<<<(unsigned)nt, kThreads, 0, c.s>>>(x, n, c.a.tiles);
    k_scan_top<<<1, 1024, 0, c.s>>>(c.a.tiles, nt, total);
    k_scan_apply<<<(unsigned)nt, kThreads, 0, c.s>>>(x, n, c.a.tiles, out, total);
    HDFE_CUDA_TRY(cudaGetLastError());
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

extern "C" int64_t hdfe_sbuild_wide_workspace_bytes(int64_t L, int64_t n_wide)
{
    if (L < 1 || n_wide < 0) return -1;
    return wide_bytes(n_wide, L);
}

extern "C" int hdfe_sbuild_analyze(const int64_t *starts, int64_t n_groups,
                                   const uint32_t *codes, int32_t D, const double *n,
                                   const double *group_n, int64_t n_cells,
                                   const int64_t *n_levels, void *workspace,
                                   int64_t workspace_bytes, hdfe_sbuild_info *info, void *stream)
{
    Ctx c;
    int st = setup(c, starts, n_groups, codes, D, n, group_n, n_cells, n_levels, workspace,
                   workspace_bytes, nullptr, 0, -1, stream);
    if (st != HDFE_OK) return st;
    Args &a = c.a;
    Layout lay = layout(a.L, n_cells, D);
    char *b = (char *)workspace;
    HDFE_CUDA_TRY(cudaMemsetAsync(b + lay.lcount, 0, a.L * 4, c.s));
    HDFE_CUDA_TRY(cudaMemsetAsync(b + lay.work, 0, a.L * 8, c.s));
    HDFE_CUDA_TRY(cudaMemsetAsync(b + lay.fillpos, 0, a.L * 4, c.s));
    HDFE_CUDA_TRY(cudaMemsetAsync(b + lay.ctr, 0, 64, c.s));
    HDFE_CUDA_TRY(cudaMemsetAsync(b + lay.status, 0, 8, c.s));
    const int cap = c.sms * 8;
    k_level_stats<<<grid_for(a.G, kThreads, cap), kThreads, 0, c.s>>>(a);
    k_classify<<<grid_for(a.L, kThreads, cap), kThreads, 0, c.s>>>(a);
    k_sort_wide<<<1, 32, 0, c.s>>>(a);
    HDFE_CUDA_TRY(cudaGetLastError());
    // group lists of the narrow levels
    st = scan_exclusive(c, a.lptr, a.L, a.lptr, a.ctr + 3);
    if (st != HDFE_OK) return st;
    k_fill_lists<<<grid_for(a.G, kThreads, cap), kThreads, 0, c.s>>>(a);
    k_write_info<<<1, 32, 0, c.s>>>(a, info);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(8);
    return HDFE_OK;
}

extern "C" int hdfe_sbuild_count(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                                 int32_t D, const double *n, const double *group_n,
                                 int64_t n_cells, const int64_t *n_levels, int64_t n_wide,
                                 int64_t *indptr, void *workspace, int64_t workspace_bytes,
                                 void *wide_workspace, int64_t wide_workspace_bytes,
                                 hdfe_sbuild_info *info, void *stream)
{
    Ctx c;
    int st = setup(c, starts, n_groups, codes, D, n, group_n, n_cells, n_levels, workspace,
                   workspace_bytes, wide_workspace, wide_workspace_bytes, n_wide, stream);
    if (st != HDFE_OK) return st;
    if (!indptr) return hdfe_set_arg_error("hdfe_sbuild_count: indptr is null");
    Args &a = c.a;
    a.indptr = indptr;
    if (n_wide > 0) HDFE_CUDA_TRY(cudaMemsetAsync(wide_workspace, 0, wide_bytes(n_wide, a.L), c.s));
    HDFE_CUDA_TRY(cudaMemsetAsync(a.rnnz, 0, (a.L + 1) * 8, c.s));
    const int cap = c.sms * 8;
    k_warp_rows<<<(unsigned)(c.sms * 4), kWarpsPerCta * 32, 0, c.s>>>(a, false);
    const size_t bsm = (size_t)kBlockSlots * 12 + kBlockListCap * 4;
    HDFE_CUDA_TRY(cudaFuncSetAttribute(k_block_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)bsm));
    k_block_rows<<<(unsigned)(c.sms * 2), 32, bsm, c.s>>>(a, false);
    if (n_wide > 0) {
        k_wide_block<<<(unsigned)cap, kThreads, 0, c.s>>>(a);
        k_wide_count<<<grid_for(n_wide, 1, c.sms * 4), kThreads, 0, c.s>>>(a);
    }
    HDFE_CUDA_TRY(cudaGetLastError());
    st = scan_exclusive(c, a.rnnz, a.L, indptr, a.ctr + 4);
    if (st != HDFE_OK) return st;
    k_write_info<<<1, 32, 0, c.s>>>(a, info);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(n_wide > 0 ? 8 : 6);
    return HDFE_OK;
}

extern "C" int hdfe_sbuild_fill(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                                int32_t D, const double *n, const double *group_n,
                                int64_t n_cells, const int64_t *n_levels, int64_t n_wide,
                                const int64_t *indptr, int32_t *indices, double *data,
                                void *workspace, int64_t workspace_bytes, void *wide_workspace,
                                int64_t wide_workspace_bytes, hdfe_sbuild_info *info,
                                void *stream)
{
    Ctx c;
    int st = setup(c, starts, n_groups, codes, D, n, group_n, n_cells, n_levels, workspace,
                   workspace_bytes, wide_workspace, wide_workspace_bytes, n_wide, stream);
    if (st != HDFE_OK) return st;
    if (!indptr || !indices || !data) return hdfe_set_arg_error("hdfe_sbuild_fill: null output");
    Args &a = c.a;
    a.indptr = const_cast<int64_t *>(indptr);
    a.indices = indices;
    a.data = data;
    k_warp_rows<<<(unsigned)(c.sms * 4), kWarpsPerCta * 32, 0, c.s>>>(a, true);
    const size_t bsm = (size_t)kBlockSlots * 12 + kBlockListCap * 4;
    HDFE_CUDA_TRY(cudaFuncSetAttribute(k_block_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)bsm));
    k_block_rows<<<(unsigned)(c.sms * 2), 32, bsm, c.s>>>(a, true);
    if (n_wide > 0) k_wide_fill<<<grid_for(n_wide, 1, c.sms * 4), kThreads, 0, c.s>>>(a);
    k_write_info<<<1, 32, 0, c.s>>>(a, info);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(n_wide > 0 ? 4 : 3);
    return HDFE_OK;
}
