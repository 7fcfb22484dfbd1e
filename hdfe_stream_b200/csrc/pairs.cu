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
        const int32_t r = find_root(parent, (int32_t)v);
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

struct Layout {
    int64_t tiles, first, pa, pb, count, deg, parent, scalars, total;
};

inline Layout layout(int64_t N, int64_t n)
{
    Layout o;
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
    o.scalars = take(64);
    o.total = p;
    return o;
}

}  // namespace pairs
}  // namespace hdfe

using namespace hdfe;

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
    const int64_t n = n0 + n1;
    const pairs::Layout lay = pairs::layout(n_rows, n);
    if (workspace_bytes < lay.total)
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_pair_components: workspace too small");
    cudaStream_t s = (cudaStream_t)stream;
    char *ws = (char *)workspace;
    int64_t *tiles = (int64_t *)(ws + lay.tiles);
    int64_t *first = (int64_t *)(ws + lay.first);
    uint32_t *pa = (uint32_t *)(ws + lay.pa);
    uint32_t *pb = (uint32_t *)(ws + lay.pb);
    int64_t *count = (int64_t *)(ws + lay.count);
    int64_t *deg = (int64_t *)(ws + lay.deg);
    int32_t *parent = (int32_t *)(ws + lay.parent);
    int64_t *P = (int64_t *)(ws + lay.scalars);
    int64_t *ncomp = P + 1;
    unsigned *status = (unsigned *)(P + 2);
    unsigned *changed = (unsigned *)(P + 3);
    int launches = 0;
    HDFE_CUDA_TRY(cudaMemsetAsync(ws + lay.scalars, 0, 64, s));
    // the distinct pairs
    const int64_t rt = (n_rows + pairs::kTile - 1) / pairs::kTile;
    pairs::k_heads<<<(unsigned)rt, pairs::kThreads, 0, s>>>(a, b, n_rows, tiles, status);
    pairs::k_scan<<<1, 32, 0, s>>>(tiles, rt, P);
    pairs::k_write<<<(unsigned)rt, pairs::kThreads, 0, s>>>(a, b, n_rows, tiles, first);
    pairs::k_pairs<<<pairs::grid_for(n_rows), pairs::kThreads, 0, s>>>(a, b, first, P, n_rows,
                                                                       n0, n1, pa, pb, count,
                                                                       status);
    launches += 4;
    // the (k0, k1)-core: rounds until one removes nothing
    HDFE_CUDA_TRY(cudaMemsetAsync(alive, 1, n, s));
    HDFE_CUDA_TRY(cudaMemsetAsync(deg, 0, n * 8, s));
    int64_t rounds = 0;
    if (k0 > 1 || k1 > 1) {
        for (;; rounds++) {
            HDFE_CUDA_TRY(cudaMemsetAsync(changed, 0, 4, s));
            pairs::k_degrees<<<pairs::grid_for(n_rows), pairs::kThreads, 0, s>>>(pa, pb, P, n0,
                                                                                 alive, deg);
            pairs::k_mark<<<pairs::grid_for(n), pairs::kThreads, 0, s>>>(n0, n, k0, k1, alive,
                                                                         deg, changed);
            launches += 2;
            unsigned h = 0;
            HDFE_CUDA_TRY(cudaMemcpyAsync(&h, changed, 4, cudaMemcpyDeviceToHost, s));
            HDFE_CUDA_TRY(cudaStreamSynchronize(s));
            if (!h || rounds > n) break;
        }
    }
    // components of the alive pairs, numbered by their roots
    const int64_t vt = (n + pairs::kTile - 1) / pairs::kTile;
    pairs::k_init<<<pairs::grid_for(n), pairs::kThreads, 0, s>>>(parent, n);
    pairs::k_union<<<pairs::grid_for(n_rows), pairs::kThreads, 0, s>>>(pa, pb, P, n0, alive,
                                                                       parent, status);
    pairs::k_roots<<<(unsigned)vt, pairs::kThreads, 0, s>>>(parent, alive, n, tiles);
    pairs::k_scan<<<1, 32, 0, s>>>(tiles, vt, ncomp);
    pairs::k_number<<<(unsigned)vt, pairs::kThreads, 0, s>>>(parent, alive, n, tiles, labels);
    pairs::k_label<<<pairs::grid_for(n), pairs::kThreads, 0, s>>>(parent, alive, n, labels);
    pairs::k_resolve<<<pairs::grid_for(n), pairs::kThreads, 0, s>>>(labels, n);
    HDFE_CUDA_TRY(cudaMemsetAsync(rows, 0, n * 8, s));
    pairs::k_pair_rows<<<pairs::grid_for(n_rows), pairs::kThreads, 0, s>>>(pa, pb, count, P, n0,
                                                                           labels, rows);
    launches += 8;
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(launches);
    // counts: pairs, components, status, peel rounds
    HDFE_CUDA_TRY(cudaMemcpyAsync(counts, P, 16, cudaMemcpyDeviceToDevice, s));
    HDFE_CUDA_TRY(cudaMemsetAsync(counts + 2, 0, 8, s));
    HDFE_CUDA_TRY(cudaMemcpyAsync(counts + 2, status, 4, cudaMemcpyDeviceToDevice, s));
    HDFE_CUDA_TRY(cudaMemcpyAsync(counts + 3, &rounds, 8, cudaMemcpyHostToDevice, s));
    HDFE_CUDA_TRY(cudaStreamSynchronize(s));
    return HDFE_OK;
}
