// Connected components of the bipartite network of two fixed effects, with
// the min_degree core: core/connected.py:378-493 `_find_components` on coded
// rows, with core/kernels_graph.py:188-221 `_nb_peel`, :225-241
// `_nb_union_keys`, :244-266 `_nb_dense_labels` and :277-289 `_nb_pair_rows`
// (and `_DistinctPairs`, core/connected.py:656-687).
//
// Rows come in pass 0's order, sorted by the first dimension and then the
// second, so the distinct (a, b) pairs are runs of rows:
//   pair_heads / pair_write   tile counts of run heads, one scan, the heads'
//                             rows -> pairs a[P], b[P], count[P] in key order
//   peel rounds               per round, the degrees of every level over the
//                             pairs whose two levels are alive, then every
//                             level under its threshold removed at once; the
//                             host repeats until a round removes nothing
//                             (`_nb_peel`'s rounds, same core)
//   unions                    alive pairs joined, larger root under smaller
//   labels                    roots numbered in vertex order (a scan of root
//                             flags), -1 for removed levels; rows per label
//
// The leave-one-out connected set (core/connected.py:503-557 `_leave_one_out`)
// adds a CSR adjacency of the alive pairs and, per round, the articulation
// points of what is alive.  The reference finds them by Tarjan's depth-first
// search (core/kernels_graph.py:23-86), which is sequential; here they come
// from a breadth-first spanning tree and the Tarjan-Vishkin rules, which are
// data-parallel:
//   BFS tree                  level-synchronous, from the smallest alive
//                             vertex; depth and tree parent per vertex
//   subtree sizes, preorder   bottom-up sums per level, then each vertex's
//                             children numbered in turn, top-down
//   low / high                min / max preorder number over every neighbour
//                             of the subtree (bottom-up per level)
//   tree-edge classes         union-find over tree edges (named by their
//                             child): a non-tree edge (x, y) joins x's and
//                             y's; a tree edge (u, v), u not the root, joins
//                             u's when v's subtree reaches outside u's
//                             (low(v) < pre(u) or high(v) >= pre(u)+size(u))
//   cut vertices              u whose children's edges are not all in u's own
//                             edge's class; the root when its children's
//                             edges fall in two classes or more
// A spanning tree by breadth has no edge between vertices of equal depth in a
// bipartite graph and every non-tree edge joins two vertices of which neither
// is an ancestor of the other, which is the case the rules cover.  The set of
// cut vertices is a property of the graph, so it does not depend on the tree
// the race between parents picks.
#include <climits>
#include <cuda_runtime.h>

#include "common.cuh"

namespace hdfe {
namespace pairs {

constexpr int kThreads = 256;
constexpr int kTile = 4096;
constexpr int kMaxSteps = 1 << 22;

inline unsigned grid_for(int64_t n, int64_t cap = 148 * 32)
{
    int64_t b = (n + kThreads - 1) / kThreads;
    if (b > cap) b = cap;
    return (unsigned)(b > 0 ? b : 1);
}

__device__ __forceinline__ bool head(const uint32_t *a, const uint32_t *b, int64_t i)
{
    return i == 0 || a[i] != a[i - 1] || b[i] != b[i - 1];
}

// heads per tile of rows; rows out of (a, b) order are reported
__global__ void __launch_bounds__(kThreads) k_heads(const uint32_t *a, const uint32_t *b,
                                                    int64_t N, int64_t *tiles, unsigned *status)
{
    __shared__ double s_red[kThreads / 32];
    const int64_t t0 = (int64_t)blockIdx.x * kTile, t1 = min(t0 + kTile, N);
    int c = 0;
    for (int64_t i = t0 + threadIdx.x; i < t1; i += kThreads) {
        c += head(a, b, i);
        if (i > 0 && (a[i] < a[i - 1] || (a[i] == a[i - 1] && b[i] < b[i - 1])))
            atomicCAS(status, 0u, (unsigned)HDFE_ERR_ARG);
    }
    const double t = block_sum((double)c, s_red);
    if (threadIdx.x == 0) tiles[blockIdx.x] = (int64_t)t;
}

// exclusive scan of the tile counts, one thread (a few thousand tiles)
__global__ void k_scan(int64_t *tiles, int64_t nt, int64_t *total)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int64_t run = 0;
    for (int64_t t = 0; t < nt; t++) { const int64_t v = tiles[t]; tiles[t] = run; run += v; }
    *total = run;
}

// each pair's first row, in row order
__global__ void __launch_bounds__(kThreads) k_write(const uint32_t *a, const uint32_t *b,
                                                    int64_t N, const int64_t *tiles,
                                                    int64_t *first)
{
    __shared__ int s_w[kThreads / 32 + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t t0 = (int64_t)blockIdx.x * kTile, t1 = min(t0 + kTile, N);
    int64_t run = tiles[blockIdx.x];
    for (int64_t base = t0; base < t1; base += kThreads) {
        const int64_t i = base + threadIdx.x;
        const bool f = i < t1 && head(a, b, i);
        const unsigned m = __ballot_sync(0xffffffffu, f);
        if (lane == 0) s_w[warp] = __popc(m);
        __syncthreads();
        if (threadIdx.x == 0) {
            int r = 0;
            for (int k = 0; k < kThreads / 32; k++) { const int t = s_w[k]; s_w[k] = r; r += t; }
            s_w[kThreads / 32] = r;
        }
        __syncthreads();
        if (f) first[run + s_w[warp] + __popc(m & ((1u << lane) - 1))] = i;
        run += s_w[kThreads / 32];
        __syncthreads();
    }
}

// the pairs: levels and rows behind each (first[P] = N)
__global__ void __launch_bounds__(kThreads) k_pairs(const uint32_t *a, const uint32_t *b,
                                                    const int64_t *first, const int64_t *P,
                                                    int64_t N, int64_t n0, int64_t n1,
                                                    uint32_t *pa, uint32_t *pb, int64_t *count,
                                                    unsigned *status)
{
    const int64_t np = *P;
    for (int64_t p = (int64_t)blockIdx.x * kThreads + threadIdx.x; p < np;
         p += (int64_t)gridDim.x * kThreads) {
        const int64_t i = first[p];
        const int64_t e = p + 1 < np ? first[p + 1] : N;
        uint32_t x = a[i], y = b[i];
        if ((int64_t)x >= n0 || (int64_t)y >= n1) {
            atomicCAS(status, 0u, (unsigned)HDFE_ERR_BAD_CODE);
            x = 0;
            y = 0;
        }
        pa[p] = x;
        pb[p] = y;
        count[p] = e - i;
    }
}

// one peel round, part 1: degrees over the pairs whose levels are both alive
__global__ void __launch_bounds__(kThreads) k_degrees(const uint32_t *pa, const uint32_t *pb,
                                                      const int64_t *P, int64_t n0,
                                                      const uint8_t *alive, int64_t *deg)
{
    const int64_t np = *P;
    for (int64_t p = (int64_t)blockIdx.x * kThreads + threadIdx.x; p < np;
         p += (int64_t)gridDim.x * kThreads) {
        const int64_t x = pa[p], y = n0 + pb[p];
        if (alive[x] && alive[y]) {
            atomicAdd(reinterpret_cast<unsigned long long *>(deg) + x, 1ull);
            atomicAdd(reinterpret_cast<unsigned long long *>(deg) + y, 1ull);
        }
    }
}

// part 2: every alive level under its threshold removed; degrees cleared
__global__ void __launch_bounds__(kThreads) k_mark(int64_t n0, int64_t n, int64_t k0, int64_t k1,
                                                   uint8_t *alive, int64_t *deg,
                                                   unsigned *changed)
{
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * kThreads) {
        const int64_t k = v < n0 ? k0 : k1;
        if (alive[v] && deg[v] < k) {
            alive[v] = 0;
            *changed = 1;
        }
        deg[v] = 0;
    }
}

__device__ __forceinline__ int32_t find_root(int32_t *parent, int32_t x)
{
    int32_t p = parent[x];
    int steps = 0;
    while (p != x && steps < kMaxSteps) {
        const int32_t gp = parent[p];
        if (gp != p) parent[x] = gp;
        x = p;
        p = gp;
        steps++;
    }
    return x;
}

// The root of x without writing: for the flattening passes, where each thread
// writes only its own vertex's entry (a compressing find could overwrite a
// vertex another thread has just set to its root with a non-root ancestor).
__device__ __forceinline__ int32_t root_of(const int32_t *parent, int32_t x)
{
    int steps = 0;
    for (int32_t p = parent[x]; p != x && steps < kMaxSteps; p = parent[x], steps++) x = p;
    return x;
}

__global__ void __launch_bounds__(kThreads) k_init(int32_t *parent, int64_t n)
{
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * kThreads)
        parent[i] = (int32_t)i;
}

// alive pairs joined: the larger root under the smaller (bounded retries)
__global__ void __launch_bounds__(kThreads) k_union(const uint32_t *pa, const uint32_t *pb,
                                                    const int64_t *P, int64_t n0,
                                                    const uint8_t *alive, int32_t *parent,
                                                    unsigned *status)
{
    const int64_t np = *P;
    for (int64_t p = (int64_t)blockIdx.x * kThreads + threadIdx.x; p < np;
         p += (int64_t)gridDim.x * kThreads) {
        int32_t x = (int32_t)pa[p], y = (int32_t)(n0 + pb[p]);
        if (!alive[x] || !alive[y]) continue;
        for (int step = 0;; step++) {
            if (step >= kMaxSteps) { atomicCAS(status, 0u, (unsigned)HDFE_ERR_SPIN_LIMIT); break; }
            x = find_root(parent, x);
            y = find_root(parent, y);
            if (x == y) break;
            const int32_t hi = x > y ? x : y, lo = x > y ? y : x;
            const int32_t old = atomicCAS(parent + hi, hi, lo);
            if (old == hi) break;
            x = hi;
            y = lo;
        }
    }
}

// roots of every vertex, and the alive roots' flags per tile
__global__ void __launch_bounds__(kThreads) k_roots(int32_t *parent, const uint8_t *alive,
                                                    int64_t n, int64_t *tiles)
{
    __shared__ double s_red[kThreads / 32];
    const int64_t t0 = (int64_t)blockIdx.x * kTile, t1 = min(t0 + kTile, n);
    int c = 0;
    for (int64_t v = t0 + threadIdx.x; v < t1; v += kThreads) {
        const int32_t r = root_of(parent, (int32_t)v);
        parent[v] = r;
        c += alive[v] && r == (int32_t)v;
    }
    const double t = block_sum((double)c, s_red);
    if (threadIdx.x == 0) tiles[blockIdx.x] = (int64_t)t;
}

// number the alive roots in vertex order (labels[root] = its number)
__global__ void __launch_bounds__(kThreads) k_number(const int32_t *parent, const uint8_t *alive,
                                                     int64_t n, const int64_t *tiles,
                                                     int32_t *labels)
{
    __shared__ int s_w[kThreads / 32 + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t t0 = (int64_t)blockIdx.x * kTile, t1 = min(t0 + kTile, n);
    int64_t run = tiles[blockIdx.x];
    for (int64_t base = t0; base < t1; base += kThreads) {
        const int64_t v = base + threadIdx.x;
        const bool f = v < t1 && alive[v] && parent[v] == (int32_t)v;
        const unsigned m = __ballot_sync(0xffffffffu, f);
        if (lane == 0) s_w[warp] = __popc(m);
        __syncthreads();
        if (threadIdx.x == 0) {
            int r = 0;
            for (int k = 0; k < kThreads / 32; k++) { const int t = s_w[k]; s_w[k] = r; r += t; }
            s_w[kThreads / 32] = r;
        }
        __syncthreads();
        if (f) labels[v] = (int32_t)(run + s_w[warp] + __popc(m & ((1u << lane) - 1)));
        run += s_w[kThreads / 32];
        __syncthreads();
    }
}

// every vertex's label from its root's (-1 where removed)
__global__ void __launch_bounds__(kThreads) k_label(const int32_t *parent, const uint8_t *alive,
                                                    int64_t n, int32_t *labels)
{
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * kThreads) {
        const int32_t r = parent[v];
        if (!alive[v]) labels[v] = -1;
        else if (r != (int32_t)v) labels[v] = -2 - r;     // resolved by k_resolve
    }
}

__global__ void __launch_bounds__(kThreads) k_resolve(int32_t *labels, int64_t n)
{
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * kThreads) {
        const int32_t l = labels[v];
        if (l <= -2) labels[v] = labels[-2 - l];     // the root's number
    }
}

// rows per component: each pair's count where both levels are labeled
__global__ void __launch_bounds__(kThreads) k_pair_rows(const uint32_t *pa, const uint32_t *pb,
                                                        const int64_t *count, const int64_t *P,
                                                        int64_t n0, const int32_t *labels,
                                                        int64_t *rows)
{
    const int64_t np = *P;
    for (int64_t p = (int64_t)blockIdx.x * kThreads + threadIdx.x; p < np;
         p += (int64_t)gridDim.x * kThreads) {
        const int32_t la = labels[pa[p]], lb = labels[n0 + pb[p]];
        if (la >= 0 && lb >= 0)
            atomicAdd(reinterpret_cast<unsigned long long *>(rows) + la,
                      (unsigned long long)count[p]);
    }
}

// ------------------------------------------------ leave-one-out connected set

// tile sums of v (n int64), for an exclusive scan
__global__ void __launch_bounds__(kThreads) k_tile_sums(const int64_t *v, int64_t n,
                                                        int64_t *tiles)
{
    __shared__ double s_red[kThreads / 32];
    const int64_t t0 = (int64_t)blockIdx.x * kTile, t1 = min(t0 + kTile, n);
    int64_t c = 0;
    for (int64_t i = t0 + threadIdx.x; i < t1; i += kThreads) c += v[i];
    const double t = block_sum((double)c, s_red);
    if (threadIdx.x == 0) tiles[blockIdx.x] = (int64_t)t;
}

// out[i] = tiles[tile of i] + sum of v over the tile before i; out[n] = total
__global__ void __launch_bounds__(kThreads) k_tile_scan(const int64_t *v, int64_t n,
                                                        const int64_t *tiles,
                                                        const int64_t *total, int64_t *out)
{
    constexpr int kPer = kTile / kThreads;
    __shared__ int64_t s_w[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t t0 = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kPer;
    int64_t x[kPer], sum = 0;
#pragma unroll
    for (int k = 0; k < kPer; k++) {
        x[k] = t0 + k < n ? v[t0 + k] : 0;
        sum += x[k];
    }
    int64_t inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    int64_t before = tiles[blockIdx.x];
    for (int k = 0; k < warp; k++) before += s_w[k];
    before += inc - sum;
#pragma unroll
    for (int k = 0; k < kPer; k++) {
        if (t0 + k < n) out[t0 + k] = before;
        before += x[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = *total;
}

// degrees of the alive pairs' levels, both directions
__global__ void __launch_bounds__(kThreads) k_adj_degree(const uint32_t *pa, const uint32_t *pb,
                                                         const int64_t *P, int64_t n0,
                                                         const uint8_t *alive, int64_t *deg)
{
    const int64_t np = *P;
    for (int64_t p = (int64_t)blockIdx.x * kThreads + threadIdx.x; p < np;
         p += (int64_t)gridDim.x * kThreads) {
        const int64_t x = pa[p], y = n0 + pb[p];
        if (alive[x] && alive[y]) {
            atomicAdd(reinterpret_cast<unsigned long long *>(deg) + x, 1ull);
            atomicAdd(reinterpret_cast<unsigned long long *>(deg) + y, 1ull);
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_adj_fill(const uint32_t *pa, const uint32_t *pb,
                                                       const int64_t *P, int64_t n0,
                                                       const uint8_t *alive,
                                                       const int64_t *indptr, int64_t *cursor,
                                                       int32_t *indices)
{
    const int64_t np = *P;
    for (int64_t p = (int64_t)blockIdx.x * kThreads + threadIdx.x; p < np;
         p += (int64_t)gridDim.x * kThreads) {
        const int64_t x = pa[p], y = n0 + pb[p];
        if (alive[x] && alive[y]) {
            const int64_t i = (int64_t)atomicAdd(
                reinterpret_cast<unsigned long long *>(cursor) + x, 1ull);
            const int64_t j = (int64_t)atomicAdd(
                reinterpret_cast<unsigned long long *>(cursor) + y, 1ull);
            indices[indptr[x] + i] = (int32_t)y;
            indices[indptr[y] + j] = (int32_t)x;
        }
    }
}

// the largest component by rows (the first of equals, i.e. the one whose
// smallest vertex comes first): best = its label, -1 when there is none
__global__ void __launch_bounds__(kThreads) k_best(const int64_t *crow, const int64_t *ncomp,
                                                   int64_t *best)
{
    __shared__ int64_t s_r[kThreads], s_i[kThreads];
    const int64_t nc = *ncomp;
    int64_t r = -1, i = -1;
    for (int64_t c = threadIdx.x; c < nc; c += kThreads)
        if (crow[c] > r) { r = crow[c]; i = c; }
    s_r[threadIdx.x] = r;
    s_i[threadIdx.x] = i;
    __syncthreads();
    for (int h = kThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            const int64_t r2 = s_r[threadIdx.x + h], i2 = s_i[threadIdx.x + h];
            if (r2 > s_r[threadIdx.x] || (r2 == s_r[threadIdx.x] && i2 >= 0 &&
                                          (s_i[threadIdx.x] < 0 || i2 < s_i[threadIdx.x]))) {
                s_r[threadIdx.x] = r2;
                s_i[threadIdx.x] = i2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *best = s_i[0];
}

__global__ void __launch_bounds__(kThreads) k_keep(uint8_t *alive, const int32_t *labels,
                                                   int64_t n, const int64_t *best)
{
    const int64_t b = *best;
    if (b < 0) return;
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * kThreads)
        if (alive[v] && labels[v] != (int32_t)b) alive[v] = 0;
}

// rows per first-dimension level over the alive pairs (`_nb_level_rows`)
__global__ void __launch_bounds__(kThreads) k_level_rows(const uint32_t *pa, const uint32_t *pb,
                                                         const int64_t *count, const int64_t *P,
                                                         int64_t n0, const uint8_t *alive,
                                                         int64_t *lrows, int64_t *total)
{
    const int64_t np = *P;
    unsigned long long t = 0;
    for (int64_t p = (int64_t)blockIdx.x * kThreads + threadIdx.x; p < np;
         p += (int64_t)gridDim.x * kThreads) {
        const int64_t x = pa[p];
        if (alive[x] && alive[n0 + pb[p]]) {
            if (lrows) atomicAdd(reinterpret_cast<unsigned long long *>(lrows) + x,
                                 (unsigned long long)count[p]);
            t += (unsigned long long)count[p];
        }
    }
    if (total) {
        t = warp_sum(t);
        if ((threadIdx.x & 31) == 0 && t)
            atomicAdd(reinterpret_cast<unsigned long long *>(total), t);
    }
}

// workers seen once removed; their number added to *removed
__global__ void __launch_bounds__(kThreads) k_single(uint8_t *alive, const int64_t *lrows,
                                                     int64_t n0, int64_t *removed)
{
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n0;
         v += (int64_t)gridDim.x * kThreads)
        if (alive[v] && lrows[v] == 1) {
            alive[v] = 0;
            atomicAdd(reinterpret_cast<unsigned long long *>(removed), 1ull);
        }
}

// smallest alive vertex (the BFS root); depth and tree parent cleared
__global__ void __launch_bounds__(kThreads) k_bfs_init(const uint8_t *alive, int64_t n,
                                                       int32_t *depth, int32_t *tpar,
                                                       int32_t *cut, int *root)
{
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * kThreads) {
        depth[v] = -1;
        tpar[v] = -1;
        cut[v] = 0;
        if (alive[v]) atomicMin(root, (int)v);
    }
}

__global__ void k_reset_root(int *root, int *first_child)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        *root = INT_MAX;
        *first_child = INT_MAX;
    }
}

__global__ void k_bfs_root(const int *root, int64_t n, int32_t *depth, int32_t *pre)
{
    const int r = *root;
    if (threadIdx.x == 0 && blockIdx.x == 0 && r >= 0 && r < n) {
        depth[r] = 0;
        pre[r] = 0;
    }
}

// one BFS level: the vertices at depth `level` claim their unreached neighbours
__global__ void __launch_bounds__(kThreads) k_bfs_level(int level, int64_t n,
                                                        const int64_t *indptr,
                                                        const int32_t *indices,
                                                        const uint8_t *alive, int32_t *depth,
                                                        int32_t *tpar, unsigned *changed)
{
    bool any = false;
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * kThreads) {
        if (depth[v] != level) continue;
        for (int64_t k = indptr[v]; k < indptr[v + 1]; k++) {
            const int32_t u = indices[k];
            if (!alive[u] || depth[u] != -1) continue;
            if (atomicCAS(depth + u, -1, level + 1) == -1) {
                tpar[u] = (int32_t)v;
                any = true;
            }
        }
    }
    if (__any_sync(0xffffffffu, any) && (threadIdx.x & 31) == 0) *changed = 1;
}

__global__ void __launch_bounds__(kThreads) k_size_init(const int32_t *depth, int64_t n,
                                                        int32_t *size)
{
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * kThreads)
        size[v] = depth[v] >= 0 ? 1 : 0;
}

__global__ void __launch_bounds__(kThreads) k_push_size(int level, const int32_t *depth,
                                                        const int32_t *tpar, int64_t n,
                                                        int32_t *size)
{
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * kThreads)
        if (depth[v] == level) atomicAdd(size + tpar[v], size[v]);
}

// each vertex at depth `level` numbers its children in preorder
__global__ void __launch_bounds__(kThreads) k_assign_pre(int level, int64_t n,
                                                         const int64_t *indptr,
                                                         const int32_t *indices,
                                                         const int32_t *depth,
                                                         const int32_t *tpar,
                                                         const int32_t *size, int32_t *pre)
{
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * kThreads) {
        if (depth[v] != level) continue;
        int32_t next = pre[v] + 1;
        for (int64_t k = indptr[v]; k < indptr[v + 1]; k++) {
            const int32_t c = indices[k];
            if (tpar[c] == (int32_t)v && depth[c] == level + 1) {
                pre[c] = next;
                next += size[c];
            }
        }
    }
}

// low / high of each reached vertex over itself and its reached neighbours
__global__ void __launch_bounds__(kThreads) k_local(int64_t n, const int64_t *indptr,
                                                    const int32_t *indices,
                                                    const int32_t *depth, const int32_t *pre,
                                                    int32_t *low, int32_t *high)
{
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * kThreads) {
        if (depth[v] < 0) continue;
        int32_t lo = pre[v], hi = pre[v];
        for (int64_t k = indptr[v]; k < indptr[v + 1]; k++) {
            const int32_t w = indices[k];
            if (depth[w] < 0) continue;
            lo = min(lo, pre[w]);
            hi = max(hi, pre[w]);
        }
        low[v] = lo;
        high[v] = hi;
    }
}

__global__ void __launch_bounds__(kThreads) k_push_low(int level, const int32_t *depth,
                                                       const int32_t *tpar, int64_t n,
                                                       int32_t *low, int32_t *high)
{
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * kThreads)
        if (depth[v] == level) {
            atomicMin(low + tpar[v], low[v]);
            atomicMax(high + tpar[v], high[v]);
        }
}

__device__ __forceinline__ void unite(int32_t *parent, int32_t x, int32_t y, unsigned *status)
{
    for (int step = 0;; step++) {
        if (step >= kMaxSteps) { atomicCAS(status, 0u, (unsigned)HDFE_ERR_SPIN_LIMIT); return; }
        x = find_root(parent, x);
        y = find_root(parent, y);
        if (x == y) return;
        const int32_t hi = x > y ? x : y, lo = x > y ? y : x;
        if (atomicCAS(parent + hi, hi, lo) == hi) return;
        x = hi;
        y = lo;
    }
}

// tree-edge classes, rule 1: a non-tree edge joins its two ends' tree edges
// (each edge taken once, from its smaller end)
__global__ void __launch_bounds__(kThreads) k_tv_cross(int64_t n, const int64_t *indptr,
                                                       const int32_t *indices,
                                                       const int32_t *depth,
                                                       const int32_t *tpar, int32_t *aux,
                                                       unsigned *status)
{
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * kThreads) {
        if (depth[v] < 0) continue;
        for (int64_t k = indptr[v]; k < indptr[v + 1]; k++) {
            const int32_t w = indices[k];
            if (w < (int32_t)v || depth[w] < 0 || tpar[v] == w || tpar[w] == (int32_t)v)
                continue;
            unite(aux, (int32_t)v, w, status);
        }
    }
}

// rule 2: (u, v) joins (parent(u), u) when v's subtree reaches outside u's
__global__ void __launch_bounds__(kThreads) k_tv_tree(int64_t n, const int32_t *depth,
                                                      const int32_t *tpar, const int32_t *pre,
                                                      const int32_t *size, const int32_t *low,
                                                      const int32_t *high, int32_t *aux,
                                                      unsigned *status)
{
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * kThreads) {
        if (depth[v] < 2) continue;                   // u = tpar[v] is not the root
        const int32_t u = tpar[v];
        if (low[v] < pre[u] || high[v] >= pre[u] + size[u]) unite(aux, u, (int32_t)v, status);
    }
}

// cut vertices: u (not the root) when a child's edge is not in u's class; the
// root's first child (smallest vertex) found for the second step
__global__ void __launch_bounds__(kThreads) k_tv_cut(int64_t n, const int32_t *depth,
                                                     const int32_t *tpar, int32_t *aux,
                                                     int32_t *cut, int *first_child)
{
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * kThreads) {
        if (depth[v] < 1) continue;
        const int32_t u = tpar[v];
        if (depth[v] == 1) atomicMin(first_child, (int)v);
        else if (find_root(aux, (int32_t)v) != find_root(aux, u)) cut[u] = 1;
    }
}

// the root: cut when two of its children's edges are in different classes
__global__ void __launch_bounds__(kThreads) k_tv_root(int64_t n, const int32_t *depth,
                                                      const int *root, const int *first_child,
                                                      int32_t *aux, int32_t *cut)
{
    const int c0 = *first_child;
    if (c0 == INT_MAX) return;
    const int32_t r0 = find_root(aux, c0);
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * kThreads)
        if (depth[v] == 1 && find_root(aux, (int32_t)v) != r0) cut[*root] = 1;
}

// workers that are cut vertices removed; their number added to *removed
__global__ void __launch_bounds__(kThreads) k_remove_cut(uint8_t *alive, const int32_t *cut,
                                                         int64_t n0, int64_t *removed)
{
    for (int64_t v = (int64_t)blockIdx.x * kThreads + threadIdx.x; v < n0;
         v += (int64_t)gridDim.x * kThreads)
        if (alive[v] && cut[v]) {
            alive[v] = 0;
            atomicAdd(reinterpret_cast<unsigned long long *>(removed), 1ull);
        }
}

struct Layout {
    int64_t tiles, first, pa, pb, count, deg, parent, scalars, total;
    // leave-one-out only
    int64_t indptr, indices, depth, tpar, size, pre, low, high, aux, cut, lab, crow, lrows;
};

inline Layout layout(int64_t N, int64_t n, bool loo = false)
{
    Layout o = {};
    int64_t p = 0;
    auto take = [&](int64_t bytes) { int64_t at = p; p += (bytes + 255) / 256 * 256; return at; };
    const int64_t nt = ((N > n ? N : n) + kTile - 1) / kTile + 1;
    o.tiles = take(nt * 8);
    o.first = take((N + 1) * 8);
    o.pa = take(N * 4);
    o.pb = take(N * 4);
    o.count = take(N * 8);
    o.deg = take(n * 8);
    o.parent = take(n * 4);
    o.scalars = take(256);
    if (loo) {
        o.indptr = take((n + 1) * 8);
        o.indices = take(2 * N * 4);
        o.depth = take(n * 4);
        o.tpar = take(n * 4);
        o.size = take(n * 4);
        o.pre = take(n * 4);
        o.low = take(n * 4);
        o.high = take(n * 4);
        o.aux = take(n * 4);
        o.cut = take(n * 4);
        o.lab = take(n * 4);
        o.crow = take(n * 8);
        o.lrows = take(n * 8);
    }
    o.total = p;
    return o;
}

}  // namespace pairs
}  // namespace hdfe

using namespace hdfe;

namespace {

// Pointers into the workspace, and the steps both entry points share.
struct Ctx {
    const uint32_t *a, *b;
    int64_t N, n0, n1, n;
    cudaStream_t s;
    pairs::Layout lay;
    int64_t *tiles, *first, *count, *deg;
    uint32_t *pa, *pb;
    int32_t *parent;
    // scalars (8 bytes each): P, ncomp, status, changed, best, root, first child, removed,
    // rows kept, components before, single observations
    int64_t *P, *ncomp, *best, *removed, *kept, *before, *single;
    unsigned *status, *changed;
    int *root, *first_child;
    int launches = 0;

    Ctx(const uint32_t *a_, const uint32_t *b_, int64_t N_, int64_t n0_, int64_t n1_, bool loo,
        void *workspace, cudaStream_t s_)
        : a(a_), b(b_), N(N_), n0(n0_), n1(n1_), n(n0_ + n1_), s(s_),
          lay(pairs::layout(N_, n0_ + n1_, loo))
    {
        char *ws = (char *)workspace;
        tiles = (int64_t *)(ws + lay.tiles);
        first = (int64_t *)(ws + lay.first);
        pa = (uint32_t *)(ws + lay.pa);
        pb = (uint32_t *)(ws + lay.pb);
        count = (int64_t *)(ws + lay.count);
        deg = (int64_t *)(ws + lay.deg);
        parent = (int32_t *)(ws + lay.parent);
        int64_t *sc = (int64_t *)(ws + lay.scalars);
        P = sc;
        ncomp = sc + 1;
        status = (unsigned *)(sc + 2);
        changed = (unsigned *)(sc + 3);
        best = sc + 4;
        root = (int *)(sc + 5);
        first_child = (int *)(sc + 6);
        removed = sc + 7;
        kept = sc + 8;
        before = sc + 9;
        single = sc + 10;
    }

    // the distinct pairs and the (k0, k1)-core; returns the peel rounds
    int pairs_and_core(uint8_t *alive, int64_t k0, int64_t k1, int64_t *rounds)
    {
        using namespace pairs;
        HDFE_CUDA_TRY(cudaMemsetAsync(P, 0, 256, s));
        const int64_t rt = (N + kTile - 1) / kTile;
        k_heads<<<(unsigned)rt, kThreads, 0, s>>>(a, b, N, tiles, status);
        k_scan<<<1, 32, 0, s>>>(tiles, rt, P);
        k_write<<<(unsigned)rt, kThreads, 0, s>>>(a, b, N, tiles, first);
        k_pairs<<<grid_for(N), kThreads, 0, s>>>(a, b, first, P, N, n0, n1, pa, pb, count,
                                                 status);
        launches += 4;
        HDFE_CUDA_TRY(cudaMemsetAsync(alive, 1, n, s));
        HDFE_CUDA_TRY(cudaMemsetAsync(deg, 0, n * 8, s));
        *rounds = 0;
        if (k0 > 1 || k1 > 1) {
            for (;; (*rounds)++) {
                HDFE_CUDA_TRY(cudaMemsetAsync(changed, 0, 4, s));
                k_degrees<<<grid_for(N), kThreads, 0, s>>>(pa, pb, P, n0, alive, deg);
                k_mark<<<grid_for(n), kThreads, 0, s>>>(n0, n, k0, k1, alive, deg, changed);
                launches += 2;
                unsigned h = 0;
                HDFE_CUDA_TRY(cudaMemcpyAsync(&h, changed, 4, cudaMemcpyDeviceToHost, s));
                HDFE_CUDA_TRY(cudaStreamSynchronize(s));
                if (!h || *rounds > n) break;
            }
        }
        return HDFE_OK;
    }

    // components of the alive pairs numbered by their roots into labels, rows
    // per label into rows (n), their number into *ncomp
    void components(const uint8_t *alive, int32_t *labels, int64_t *rows)
    {
        using namespace pairs;
        const int64_t vt = (n + kTile - 1) / kTile;
        k_init<<<grid_for(n), kThreads, 0, s>>>(parent, n);
        k_union<<<grid_for(N), kThreads, 0, s>>>(pa, pb, P, n0, alive, parent, status);
        k_roots<<<(unsigned)vt, kThreads, 0, s>>>(parent, alive, n, tiles);
        k_scan<<<1, 32, 0, s>>>(tiles, vt, ncomp);
        k_number<<<(unsigned)vt, kThreads, 0, s>>>(parent, alive, n, tiles, labels);
        k_label<<<grid_for(n), kThreads, 0, s>>>(parent, alive, n, labels);
        k_resolve<<<grid_for(n), kThreads, 0, s>>>(labels, n);
        cudaMemsetAsync(rows, 0, n * 8, s);
        k_pair_rows<<<grid_for(N), kThreads, 0, s>>>(pa, pb, count, P, n0, labels, rows);
        launches += 8;
    }
};

}  // namespace

extern "C" int64_t hdfe_pair_components_workspace_bytes(int64_t n_rows, int64_t n0, int64_t n1)
{
    if (n_rows < 0 || n0 < 1 || n1 < 1) return -1;
    return pairs::layout(n_rows, n0 + n1).total;
}

extern "C" int hdfe_pair_components(const uint32_t *a, const uint32_t *b, int64_t n_rows,
                                    int64_t n0, int64_t n1, int64_t k0, int64_t k1,
                                    uint8_t *alive, int32_t *labels, int64_t *rows,
                                    int64_t *counts, void *workspace, int64_t workspace_bytes,
                                    void *stream)
{
    if (!a || !b || n_rows < 1 || n0 < 1 || n1 < 1 || n0 + n1 >= INT32_MAX || k0 < 1 || k1 < 1 ||
        !alive || !labels || !rows || !counts || !workspace)
        return hdfe_set_arg_error("hdfe_pair_components: bad argument");
    Ctx c(a, b, n_rows, n0, n1, false, workspace, (cudaStream_t)stream);
    if (workspace_bytes < c.lay.total)
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_pair_components: workspace too small");
    int64_t rounds = 0;
    int st = c.pairs_and_core(alive, k0, k1, &rounds);
    if (st != HDFE_OK) return st;
    c.components(alive, labels, rows);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(c.launches);
    // counts: pairs, components, status, peel rounds
    cudaStream_t s = c.s;
    HDFE_CUDA_TRY(cudaMemcpyAsync(counts, c.P, 16, cudaMemcpyDeviceToDevice, s));
    HDFE_CUDA_TRY(cudaMemsetAsync(counts + 2, 0, 8, s));
    HDFE_CUDA_TRY(cudaMemcpyAsync(counts + 2, c.status, 4, cudaMemcpyDeviceToDevice, s));
    HDFE_CUDA_TRY(cudaMemcpyAsync(counts + 3, &rounds, 8, cudaMemcpyHostToDevice, s));
    HDFE_CUDA_TRY(cudaStreamSynchronize(s));
    return HDFE_OK;
}

extern "C" int64_t hdfe_leave_one_out_workspace_bytes(int64_t n_rows, int64_t n0, int64_t n1)
{
    if (n_rows < 0 || n0 < 1 || n1 < 1) return -1;
    return pairs::layout(n_rows, n0 + n1, true).total;
}

extern "C" int hdfe_leave_one_out(const uint32_t *a, const uint32_t *b, int64_t n_rows,
                                  int64_t n0, int64_t n1, int64_t k0, int64_t k1,
                                  uint8_t *alive, int64_t *counts, void *workspace,
                                  int64_t workspace_bytes, void *stream)
{
    using namespace pairs;
    if (!a || !b || n_rows < 1 || n0 < 1 || n1 < 1 || n0 + n1 >= INT32_MAX || k0 < 1 ||
        k1 < 1 || !alive || !counts || !workspace)
        return hdfe_set_arg_error("hdfe_leave_one_out: bad argument");
    Ctx c(a, b, n_rows, n0, n1, true, workspace, (cudaStream_t)stream);
    if (workspace_bytes < c.lay.total)
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_leave_one_out: workspace too small");
    cudaStream_t s = c.s;
    const int64_t n = c.n, N = n_rows;
    char *ws = (char *)workspace;
    const Layout &L = c.lay;
    int64_t *indptr = (int64_t *)(ws + L.indptr);
    int32_t *indices = (int32_t *)(ws + L.indices);
    int32_t *depth = (int32_t *)(ws + L.depth), *tpar = (int32_t *)(ws + L.tpar);
    int32_t *size = (int32_t *)(ws + L.size), *pre = (int32_t *)(ws + L.pre);
    int32_t *low = (int32_t *)(ws + L.low), *high = (int32_t *)(ws + L.high);
    int32_t *aux = (int32_t *)(ws + L.aux), *cut = (int32_t *)(ws + L.cut);
    int32_t *lab = (int32_t *)(ws + L.lab);
    int64_t *crow = (int64_t *)(ws + L.crow), *lrows = (int64_t *)(ws + L.lrows);
    int64_t peel_rounds = 0;
    int st = c.pairs_and_core(alive, k0, k1, &peel_rounds);
    if (st != HDFE_OK) return st;

    // CSR adjacency of the pairs alive now (later removals only clear `alive`)
    const int64_t vt = (n + kTile - 1) / kTile;
    HDFE_CUDA_TRY(cudaMemsetAsync(c.deg, 0, n * 8, s));
    k_adj_degree<<<grid_for(N), kThreads, 0, s>>>(c.pa, c.pb, c.P, n0, alive, c.deg);
    k_tile_sums<<<(unsigned)vt, kThreads, 0, s>>>(c.deg, n, c.tiles);
    k_scan<<<1, 32, 0, s>>>(c.tiles, vt, c.removed);
    k_tile_scan<<<(unsigned)vt, kThreads, 0, s>>>(c.deg, n, c.tiles, c.removed, indptr);
    HDFE_CUDA_TRY(cudaMemsetAsync(c.deg, 0, n * 8, s));
    k_adj_fill<<<grid_for(N), kThreads, 0, s>>>(c.pa, c.pb, c.P, n0, alive, indptr, c.deg,
                                                indices);
    c.launches += 5;

    auto keep_largest = [&]() {
        c.components(alive, lab, crow);
        k_best<<<1, kThreads, 0, s>>>(crow, c.ncomp, c.best);
        k_keep<<<grid_for(n), kThreads, 0, s>>>(alive, lab, n, c.best);
        c.launches += 2;
    };
    auto read = [&](const void *dev, size_t bytes, void *host) -> int {
        HDFE_CUDA_TRY(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s));
        HDFE_CUDA_TRY(cudaStreamSynchronize(s));
        return HDFE_OK;
    };

    // 1. the largest component
    keep_largest();
    HDFE_CUDA_TRY(cudaMemcpyAsync(c.before, c.ncomp, 8, cudaMemcpyDeviceToDevice, s));
    // 2. workers seen once (their leverage is 1), then the largest piece left
    HDFE_CUDA_TRY(cudaMemsetAsync(lrows, 0, n0 * 8, s));
    k_level_rows<<<grid_for(N), kThreads, 0, s>>>(c.pa, c.pb, c.count, c.P, n0, alive, lrows,
                                                  nullptr);
    k_single<<<grid_for(n0), kThreads, 0, s>>>(alive, lrows, n0, c.single);
    c.launches += 2;
    keep_largest();
    // 3-4. workers that are articulation points, until there are none
    int64_t cut_total = 0, rounds = 0, max_levels = 0;
    for (;;) {
        k_reset_root<<<1, 32, 0, s>>>(c.root, c.first_child);
        k_bfs_init<<<grid_for(n), kThreads, 0, s>>>(alive, n, depth, tpar, cut, c.root);
        k_bfs_root<<<1, 32, 0, s>>>(c.root, n, depth, pre);
        c.launches += 3;
        int levels = 0;
        for (;; levels++) {
            HDFE_CUDA_TRY(cudaMemsetAsync(c.changed, 0, 4, s));
            k_bfs_level<<<grid_for(n), kThreads, 0, s>>>(levels, n, indptr, indices, alive,
                                                         depth, tpar, c.changed);
            c.launches++;
            unsigned h = 0;
            if ((st = read(c.changed, 4, &h)) != HDFE_OK) return st;
            if (!h || levels > n) break;
        }
        // `levels` is now the largest depth
        if (levels > max_levels) max_levels = levels;
        k_size_init<<<grid_for(n), kThreads, 0, s>>>(depth, n, size);
        for (int l = levels; l >= 1; l--)
            k_push_size<<<grid_for(n), kThreads, 0, s>>>(l, depth, tpar, n, size);
        for (int l = 0; l < levels; l++)
            k_assign_pre<<<grid_for(n), kThreads, 0, s>>>(l, n, indptr, indices, depth, tpar,
                                                          size, pre);
        k_local<<<grid_for(n), kThreads, 0, s>>>(n, indptr, indices, depth, pre, low, high);
        for (int l = levels; l >= 1; l--)
            k_push_low<<<grid_for(n), kThreads, 0, s>>>(l, depth, tpar, n, low, high);
        k_init<<<grid_for(n), kThreads, 0, s>>>(aux, n);
        k_tv_cross<<<grid_for(n), kThreads, 0, s>>>(n, indptr, indices, depth, tpar, aux,
                                                    c.status);
        k_tv_tree<<<grid_for(n), kThreads, 0, s>>>(n, depth, tpar, pre, size, low, high, aux,
                                                   c.status);
        k_tv_cut<<<grid_for(n), kThreads, 0, s>>>(n, depth, tpar, aux, cut, c.first_child);
        k_tv_root<<<grid_for(n), kThreads, 0, s>>>(n, depth, c.root, c.first_child, aux, cut);
        HDFE_CUDA_TRY(cudaMemsetAsync(c.removed, 0, 8, s));
        k_remove_cut<<<grid_for(n0), kThreads, 0, s>>>(alive, cut, n0, c.removed);
        c.launches += 9 + 3 * levels;
        int64_t n_cut = 0;
        if ((st = read(c.removed, 8, &n_cut)) != HDFE_OK) return st;
        if (!n_cut || rounds > n) break;
        cut_total += n_cut;
        rounds++;
        keep_largest();
    }
    // rows kept
    HDFE_CUDA_TRY(cudaMemsetAsync(c.kept, 0, 8, s));
    k_level_rows<<<grid_for(N), kThreads, 0, s>>>(c.pa, c.pb, c.count, c.P, n0, alive, nullptr,
                                                  c.kept);
    c.launches++;
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(c.launches);
    // counts: pairs, components before, single observations, workers cut, rounds, rows
    // kept, status, BFS depth (largest over rounds)
    int64_t h[8];
    int64_t dev_sc[11];
    if ((st = read(c.P, sizeof(dev_sc), dev_sc)) != HDFE_OK) return st;
    h[0] = dev_sc[0];
    h[1] = dev_sc[9];
    h[2] = dev_sc[10];
    h[3] = cut_total;
    h[4] = rounds;
    h[5] = dev_sc[8];
    h[6] = (int64_t)(unsigned)(dev_sc[2] & 0xffffffff);
    h[7] = max_levels;
    HDFE_CUDA_TRY(cudaMemcpyAsync(counts, h, sizeof(h), cudaMemcpyHostToDevice, s));
    HDFE_CUDA_TRY(cudaStreamSynchronize(s));
    return HDFE_OK;
}
