// Connected components of the levels of one non-streamed dimension (levels
// sharing an identifying group are connected), and the normalisation of the
// solved fixed effects.
//
// Components: core/kernels_base.py:156-174 `_nb_components`.  The device
// union-find links the larger root under the smaller with atomicCAS, so every
// component's root is its smallest level, whatever the order the unions run
// in -- the reference's root, exactly (its serial union-find also links
// toward the smaller index).  Ranking the roots into labels by rows
// (core/passes.py:933-950) is bookkeeping done by the caller.
//
// Normalisation: core/solve.py:383-399 `_normalize`.  The first dimension's
// effects get obs-weighted mean zero within each component, every further
// dimension obs-weighted mean zero overall.  Within-component sums are
// combined per warp (lanes with the same root, __match_any_sync) before one
// atomic per root, so the giant component does not see 500k atomics.
#include <cuda_runtime.h>

#include "common.cuh"

namespace hdfe {
namespace graph {

constexpr int kThreads = 256;
constexpr int kMaxSteps = 1 << 22;     // retries of one union before giving up

__device__ __forceinline__ int32_t find_root(int32_t *parent, int32_t x)
{
    // path halving with relaxed writes: parent pointers only ever decrease
    int32_t p = parent[x];
    int steps = 0;
    while (p != x && steps < kMaxSteps) {
        const int32_t gp = parent[p];
        if (gp != p) parent[x] = gp;    // a benign race: gp is an ancestor of x
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

// link a and b: the larger root under the smaller (bounded retries)
__device__ __forceinline__ void unite(int32_t *parent, int32_t a, int32_t b, unsigned *status)
{
    for (int step = 0;; step++) {
        if (step >= kMaxSteps) { atomicCAS(status, 0u, (unsigned)HDFE_ERR_SPIN_LIMIT); return; }
        a = find_root(parent, a);
        b = find_root(parent, b);
        if (a == b) return;
        const int32_t hi = a > b ? a : b, lo = a > b ? b : a;
        const int32_t old = atomicCAS(parent + hi, hi, lo);
        if (old == hi) return;
        a = hi;         // hi gained a parent meanwhile: retry from there
        b = lo;
    }
}

// The levels (dimension col) of each group joined into one component: a
// warp takes 32 groups, reads their cells coalesced (one per lane, 32 at a
// time) and joins each cell's level with the previous cell's of the same
// group where they differ -- a chain over the group, which connects what the
// reference's star over the group's first level connects (every root is the
// component's smallest level either way).
__global__ void __launch_bounds__(kThreads) k_union(const int64_t *starts, int64_t G,
                                                    const uint32_t *codes, int D, int col,
                                                    int64_t nlev, int32_t *parent,
                                                    unsigned *status)
{
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * kThreads) >> 5;
    for (int64_t g0 = wid * 32; g0 < G; g0 += nw * 32) {
        const int ng = (int)min((int64_t)32, G - g0);
        const int64_t gend = starts[g0 + ng];
        const int64_t st = lane < ng ? starts[g0 + lane] : gend;   // this lane's group start
        for (int64_t base = starts[g0]; base < gend; base += 32) {
            const bool in = lane < ng && st >= base && st < base + 32;
            const unsigned heads = __reduce_or_sync(0xffffffffu, in ? 1u << (int)(st - base) : 0u);
            const int64_t i = base + lane;
            const bool valid = i < gend;
            uint32_t c = valid ? codes[i * D + col] : 0u;
            uint32_t prev = __shfl_up_sync(0xffffffffu, c, 1);
            if (lane == 0 && valid && i > 0) prev = codes[(i - 1) * D + col];
            const bool head = (heads >> lane) & 1u;
            if (valid && (int64_t)c >= nlev) atomicCAS(status, 0u, (unsigned)HDFE_ERR_BAD_CODE);
            if (!valid || head || c == prev || (int64_t)c >= nlev || (int64_t)prev >= nlev)
                continue;
            unite(parent, (int32_t)prev, (int32_t)c, status);
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_flatten(int32_t *parent, int64_t n,
                                                      unsigned long long *n_roots)
{
    unsigned long long roots = 0;
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * kThreads) {
        const int32_t r = root_of(parent, (int32_t)i);
        parent[i] = r;
        roots += (r == (int32_t)i);
    }
    roots = warp_sum(roots);
    if ((threadIdx.x & 31) == 0 && roots) atomicAdd(n_roots, roots);
}

// ------------------------------------------------------------ normalise

// sums per root: cw[root] += w, cs[root, j] += w * Gamma[l, j]
__global__ void __launch_bounds__(kThreads) k_comp_sums(const int32_t *root, const double *w,
                                                        const double *gamma, int64_t nl, int m,
                                                        double *cw, double *cs)
{
    __shared__ double s_stage[kThreads];
    const int lane = threadIdx.x & 31;
    double *stage = s_stage + (threadIdx.x & ~31);
    for (int64_t base = (int64_t)blockIdx.x * kThreads; base < nl;
         base += (int64_t)gridDim.x * kThreads) {
        const int64_t l = base + threadIdx.x;
        const bool valid = l < nl;
        const int32_t r = valid ? root[l] : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, r);
        const bool leader = valid && lane == __ffs(peers) - 1;
        const double wl = valid ? w[l] : 0.0;
        // the peers' values summed in lane order by their leader
        for (int j = -1; j < m; j++) {
            stage[lane] = j < 0 ? wl : (valid ? wl * gamma[l * m + j] : 0.0);
            __syncwarp();
            if (leader) {
                double acc = 0.0;
                for (unsigned p = peers; p; p &= p - 1) acc += stage[__ffs(p) - 1];
                if (j < 0) atomicAdd(cw + r, acc);
                else atomicAdd(cs + (int64_t)r * m + j, acc);
            }
            __syncwarp();
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_comp_apply(const int32_t *root, const double *cw,
                                                         const double *cs, int64_t nl, int m,
                                                         double *gamma)
{
    for (int64_t l = (int64_t)blockIdx.x * kThreads + threadIdx.x; l < nl;
         l += (int64_t)gridDim.x * kThreads) {
        const int32_t r = root[l];
        double c = cw[r];
        if (c == 0.0) c = 1.0;
        for (int j = 0; j < m; j++) gamma[l * m + j] -= cs[(int64_t)r * m + j] / c;
    }
}

// per-CTA partial sums of w and w * Gamma over one dimension's block
__global__ void __launch_bounds__(kThreads) k_dim_sums(const double *w, const double *gamma,
                                                       int64_t nl, int m, double *part)
{
    __shared__ double s_red[kThreads / 32];
    double sw = 0.0;
    for (int64_t l = (int64_t)blockIdx.x * kThreads + threadIdx.x; l < nl;
         l += (int64_t)gridDim.x * kThreads)
        sw += w[l];
    sw = block_sum(sw, s_red);
    if (threadIdx.x == 0) part[blockIdx.x * (1 + m)] = sw;
    for (int j = 0; j < m; j++) {
        double s = 0.0;
        for (int64_t l = (int64_t)blockIdx.x * kThreads + threadIdx.x; l < nl;
             l += (int64_t)gridDim.x * kThreads)
            s += w[l] * gamma[l * m + j];
        s = block_sum(s, s_red);
        if (threadIdx.x == 0) part[blockIdx.x * (1 + m) + 1 + j] = s;
    }
}

__global__ void __launch_bounds__(kThreads) k_dim_apply(const double *part, int nparts,
                                                        double *gamma, int64_t nl, int m)
{
    __shared__ double s_mean[HDFE_MAX_VARS];
    if (threadIdx.x < 32) {
        double sw = 0.0;
        for (int b = 0; b < nparts; b++) sw += part[b * (1 + m)];
        const double den = fmax(sw, 1.0);
        for (int j = (int)threadIdx.x; j < m; j += 32) {
            double s = 0.0;
            for (int b = 0; b < nparts; b++) s += part[b * (1 + m) + 1 + j];
            s_mean[j] = s / den;
        }
    }
    __syncthreads();
    for (int64_t l = (int64_t)blockIdx.x * kThreads + threadIdx.x; l < nl;
         l += (int64_t)gridDim.x * kThreads)
        for (int j = 0; j < m; j++) gamma[l * m + j] -= s_mean[j];
}

inline unsigned grid_for(int64_t n)
{
    int64_t b = (n + kThreads - 1) / kThreads;
    if (b > 4096) b = 4096;
    return (unsigned)(b > 0 ? b : 1);
}

}  // namespace graph
}  // namespace hdfe

using namespace hdfe;

extern "C" int64_t hdfe_components_workspace_bytes(void) { return 256; }

extern "C" int hdfe_components(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                               int32_t D, int32_t col, int64_t n_levels, int32_t *root,
                               int64_t *n_components, void *workspace, int64_t workspace_bytes,
                               void *stream)
{
    if (D < 1 || D > HDFE_MAX_DIMS || col < 0 || col >= D || n_levels < 1 ||
        n_levels >= INT32_MAX || n_groups < 0 || !starts || (n_groups > 0 && !codes) || !root ||
        !n_components || !workspace || workspace_bytes < 256)
        return hdfe_set_arg_error("hdfe_components: bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned *status = (unsigned *)workspace;
    unsigned long long *roots = (unsigned long long *)((char *)workspace + 64);
    HDFE_CUDA_TRY(cudaMemsetAsync(workspace, 0, 128, s));
    graph::k_init<<<graph::grid_for(n_levels), graph::kThreads, 0, s>>>(root, n_levels);
    graph::k_union<<<graph::grid_for(n_groups), graph::kThreads, 0, s>>>(
        starts, n_groups, codes, D, col, n_levels, root, status);
    graph::k_flatten<<<graph::grid_for(n_levels), graph::kThreads, 0, s>>>(root, n_levels, roots);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(3);
    // n_components[0] = roots, n_components[1] = status
    HDFE_CUDA_TRY(cudaMemcpyAsync(n_components, roots, 8, cudaMemcpyDeviceToDevice, s));
    HDFE_CUDA_TRY(cudaMemsetAsync(n_components + 1, 0, 8, s));
    HDFE_CUDA_TRY(cudaMemcpyAsync(n_components + 1, status, 4, cudaMemcpyDeviceToDevice, s));
    return HDFE_OK;
}

extern "C" int64_t hdfe_normalize_workspace_bytes(int64_t n_first, int32_t m)
{
    if (n_first < 0 || m < 1 || m > HDFE_MAX_VARS) return -1;
    return (n_first * (1 + (int64_t)m) + 4096 * (1 + (int64_t)m)) * 8 + 256;
}

extern "C" int hdfe_normalize(double *gamma, int32_t m, int32_t D, const int64_t *n_levels,
                              const double *obs, const int32_t *root, void *workspace,
                              int64_t workspace_bytes, void *stream)
{
    if (!gamma || m < 1 || m > HDFE_MAX_VARS || D < 1 || D > HDFE_MAX_DIMS || !n_levels ||
        !obs || !root || !workspace)
        return hdfe_set_arg_error("hdfe_normalize: bad argument");
    const int64_t n0 = n_levels[0];
    if (workspace_bytes < hdfe_normalize_workspace_bytes(n0, m))
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_normalize: workspace too small");
    cudaStream_t s = (cudaStream_t)stream;
    double *cw = (double *)workspace;
    double *cs = cw + n0;
    double *part = cs + n0 * m;
    HDFE_CUDA_TRY(cudaMemsetAsync(cw, 0, n0 * (1 + (int64_t)m) * 8, s));
    graph::k_comp_sums<<<graph::grid_for(n0), graph::kThreads, 0, s>>>(root, obs, gamma, n0, m,
                                                                       cw, cs);
    graph::k_comp_apply<<<graph::grid_for(n0), graph::kThreads, 0, s>>>(root, cw, cs, n0, m,
                                                                        gamma);
    int64_t off = n0;
    for (int d = 1; d < D; d++) {
        const int64_t nl = n_levels[d];
        const unsigned nb = graph::grid_for(nl) < 1024 ? graph::grid_for(nl) : 1024;
        graph::k_dim_sums<<<nb, graph::kThreads, 0, s>>>(obs + off, gamma + off * m, nl, m, part);
        graph::k_dim_apply<<<graph::grid_for(nl), graph::kThreads, 0, s>>>(part, (int)nb,
                                                                           gamma + off * m, nl, m);
        off += nl;
    }
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(2 + 2 * (D - 1));
    return HDFE_OK;
}
