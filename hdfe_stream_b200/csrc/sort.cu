// Pass 0 on the device: a stable LSD radix sort of 64-bit keys with int32
// payloads, and factorization (the rank of each id among the distinct ids).
//
// Reference: core/passes.py:285-294 codes each fixed effect by the rank of
// its level among the sorted distinct levels, and :359-373 sorts the rows by
// (streamed code, other codes, variables).  The sort here is the one the
// reference's ordering needs: stable, 8 bits per pass over the key's low
// `key_bits` bits (the bits that can be nonzero), so a multi-key order is a
// sequence of sorts, least significant key first.
//   Per pass, tiles of kTile items:
//     hist      each CTA counts its tile's digits (shared-memory histogram)
//               into counts[digit * tiles + tile] (digit-major);
//     scan      exclusive offsets of counts in that order (per-CTA sums, a
//               one-CTA scan of those, then the offsets applied), so digit d
//               of tile t starts after every smaller digit and every earlier
//               tile's d: the order is stable;
//     scatter   each CTA walks its tile in rounds of kThreads items in index
//               order; an item's place among its tile's equal digits is the
//               count of those in earlier rounds, earlier warps of its round
//               (shared-memory counts) and earlier lanes of its warp
//               (__match_any_sync), so equal digits keep their order.
// Factorize: the (id, position) pairs sorted by id; a run head marks each
// distinct id; an exclusive scan of the heads gives the ranks, scattered back
// to the positions; the distinct ids are written in order.
#include <algorithm>
#include <cuda_runtime.h>

#include "common.cuh"

namespace hdfe {
namespace sorting {

constexpr int kThreads = 256;
constexpr int kItems = 16;              // items per thread per tile
constexpr int kTile = kThreads * kItems;
constexpr int kBins = 256;
constexpr int kWarps = kThreads / 32;

__global__ void __launch_bounds__(kThreads) k_hist(const uint64_t *keys, int64_t n, int shift,
                                                   int64_t tiles, uint32_t *counts)
{
    __shared__ uint32_t s_h[kBins];
    s_h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t t0 = (int64_t)blockIdx.x * kTile;
    const int64_t t1 = min(t0 + kTile, n);
    for (int64_t i = t0 + threadIdx.x; i < t1; i += kThreads)
        atomicAdd(s_h + ((keys[i] >> shift) & 0xFF), 1u);
    __syncthreads();
    counts[(int64_t)threadIdx.x * tiles + blockIdx.x] = s_h[threadIdx.x];
}

// exclusive scan of x (n) into out, 3 kernels: per-CTA sums of kTile-item
// chunks, a scan of those (one CTA), then each chunk's scan with its offset
__global__ void __launch_bounds__(kThreads) k_scan_sums(const uint32_t *x, int64_t n,
                                                        int64_t *sums)
{
    __shared__ int64_t s_w[kWarps];
    const int64_t t0 = (int64_t)blockIdx.x * kTile;
    int64_t v = 0;
    for (int64_t i = t0 + threadIdx.x; i < min(t0 + kTile, n); i += kThreads) v += x[i];
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t t = 0;
        for (int w = 0; w < kWarps; w++) t += s_w[w];
        sums[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(1024) k_scan_top(int64_t *sums, int64_t m)
{
    __shared__ int64_t s[1024];
    int64_t carry = 0;
    for (int64_t b0 = 0; b0 < m; b0 += 1024) {
        const int64_t b = b0 + threadIdx.x;
        const int64_t v = b < m ? sums[b] : 0;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            const int64_t y = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
            __syncthreads();
            s[threadIdx.x] += y;
            __syncthreads();
        }
        if (b < m) sums[b] = carry + s[threadIdx.x] - v;
        carry += s[1023];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads) k_scan_apply(const uint32_t *x, int64_t n,
                                                         const int64_t *sums, int64_t *out)
{
    __shared__ int64_t s_w[kWarps + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t t0 = (int64_t)blockIdx.x * kTile;
    int64_t run = sums[blockIdx.x];
    for (int64_t b = t0; b < min(t0 + kTile, n); b += kThreads) {
        const int64_t i = b + threadIdx.x;
        const int64_t v = i < n ? x[i] : 0;
        int64_t inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) s_w[warp] = inc;
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t r = 0;
            for (int w = 0; w < kWarps; w++) { const int64_t t = s_w[w]; s_w[w] = r; r += t; }
            s_w[kWarps] = r;
        }
        __syncthreads();
        if (i < n) out[i] = run + s_w[warp] + inc - v;
        run += s_w[kWarps];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads) k_scatter(const uint64_t *keys, const int32_t *vals,
                                                      int64_t n, int shift, int64_t tiles,
                                                      const int64_t *offsets, uint64_t *keys_out,
                                                      int32_t *vals_out)
{
    __shared__ uint32_t s_base[kBins];              // this tile's items so far, per digit
    __shared__ uint32_t s_warp[kWarps][kBins];      // this round's count per warp and digit
    __shared__ int64_t s_off[kBins];                // the tile's first output slot per digit
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    s_base[threadIdx.x] = 0;
    s_off[threadIdx.x] = offsets[(int64_t)threadIdx.x * tiles + blockIdx.x];
    const int64_t t0 = (int64_t)blockIdx.x * kTile;
    const int64_t t1 = min(t0 + kTile, n);
    for (int64_t b = t0; b < t1; b += kThreads) {
        for (int w = 0; w < kWarps; w++) s_warp[w][threadIdx.x] = 0;
        __syncthreads();
        const int64_t i = b + threadIdx.x;
        const bool valid = i < t1;
        const uint64_t k = valid ? keys[i] : 0;
        const int32_t v = valid ? vals[i] : 0;
        const unsigned d = valid ? (unsigned)((k >> shift) & 0xFF) : kBins;   // kBins: none
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int below = __popc(peers & ((1u << lane) - 1));
        if (valid && below == 0) s_warp[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            unsigned before = 0;
            for (int w = 0; w < warp; w++) before += s_warp[w][d];
            const int64_t at = s_off[d] + s_base[d] + before + below;
            keys_out[at] = k;
            vals_out[at] = v;
        }
        __syncthreads();
        unsigned tot = 0;
        for (int w = 0; w < kWarps; w++) tot += s_warp[w][threadIdx.x];
        s_base[threadIdx.x] += tot;
        __syncthreads();
    }
}

// heads[i] = 1 where the sorted ids change (and at 0)
__global__ void __launch_bounds__(kThreads) k_heads(const uint64_t *ids, int64_t n,
                                                    uint32_t *heads)
{
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * kThreads)
        heads[i] = (i == 0 || ids[i] != ids[i - 1]) ? 1u : 0u;
}

// the rank of sorted item i is (exclusive scan of heads)[i] + heads[i] - 1
__global__ void __launch_bounds__(kThreads) k_ranks(const uint64_t *ids, const int32_t *pos,
                                                    const uint32_t *heads, const int64_t *excl,
                                                    int64_t n, int32_t *codes, uint64_t *levels,
                                                    int64_t *n_levels)
{
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * kThreads) {
        const int64_t r = excl[i] + heads[i] - 1;
        codes[pos[i]] = (int32_t)r;
        if (heads[i] && levels) levels[r] = ids[i];
        if (i == n - 1) *n_levels = r + 1;
    }
}

__global__ void __launch_bounds__(kThreads) k_iota(int32_t *v, int64_t n)
{
    for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * kThreads)
        v[i] = (int32_t)i;
}

struct Work {       // workspace layout
    uint64_t *keys[2];
    int32_t *vals[2];
    uint32_t *counts;
    int64_t *offsets;
    int64_t *sums;
    int64_t tiles, ncounts, nsums;
};

inline int64_t align256(int64_t b) { return (b + 255) / 256 * 256; }

inline Work layout(void *ws, int64_t n)
{
    Work w;
    w.tiles = (n + kTile - 1) / kTile;
    w.ncounts = w.tiles * kBins;
    // chunk sums for either scan: the counts (ncounts entries) or n heads
    w.nsums = std::max((w.ncounts + kTile - 1) / kTile, w.tiles);
    char *p = (char *)ws;
    auto take = [&](int64_t bytes) { char *at = p; p += align256(bytes); return at; };
    w.keys[0] = (uint64_t *)take(n * 8);
    w.keys[1] = (uint64_t *)take(n * 8);
    w.vals[0] = (int32_t *)take(n * 4);
    w.vals[1] = (int32_t *)take(n * 4);
    w.counts = (uint32_t *)take(w.ncounts * 4);
    w.offsets = (int64_t *)take(std::max(w.ncounts, n) * 8);
    w.sums = (int64_t *)take(w.nsums * 8 + 8);
    return w;
}

inline int64_t layout_bytes(int64_t n)
{
    const int64_t tiles = (n + kTile - 1) / kTile, nc = tiles * kBins;
    const int64_t ns = std::max((nc + kTile - 1) / kTile, tiles);
    return 2 * align256(n * 8) + 2 * align256(n * 4) + align256(nc * 4) +
           align256(std::max(nc, n) * 8) + align256(ns * 8 + 8);
}

// exclusive scan of x (m entries) into out
inline void scan(const uint32_t *x, int64_t m, int64_t *sums, int64_t *out, cudaStream_t s)
{
    const int64_t chunks = (m + kTile - 1) / kTile;
    k_scan_sums<<<(unsigned)chunks, kThreads, 0, s>>>(x, m, sums);
    k_scan_top<<<1, 1024, 0, s>>>(sums, chunks);
    k_scan_apply<<<(unsigned)chunks, kThreads, 0, s>>>(x, m, sums, out);
}

// sort (keys, vals) in buffers 0 by the low key_bits bits; the result is in
// buffers *which
void radix_sort(Work &w, int64_t n, int key_bits, int *which, cudaStream_t s)
{
    int cur = 0;
    const unsigned tiles = (unsigned)w.tiles;
    for (int shift = 0; shift < key_bits; shift += 8) {
        k_hist<<<tiles, kThreads, 0, s>>>(w.keys[cur], n, shift, w.tiles, w.counts);
        scan(w.counts, w.ncounts, w.sums, w.offsets, s);
        k_scatter<<<tiles, kThreads, 0, s>>>(w.keys[cur], w.vals[cur], n, shift, w.tiles,
                                             w.offsets, w.keys[1 - cur], w.vals[1 - cur]);
        cur = 1 - cur;
        hdfe_add_launches(5);
    }
    *which = cur;
}

inline unsigned grid_for(int64_t n)
{
    return (unsigned)std::min<int64_t>((n + kThreads - 1) / kThreads, 148 * 32);
}

}  // namespace sorting
}  // namespace hdfe

using namespace hdfe;

extern "C" int64_t hdfe_sort_workspace_bytes(int64_t n)
{
    return n < 0 ? -1 : sorting::layout_bytes(n > 0 ? n : 1);
}

extern "C" int hdfe_sort_pairs(const uint64_t *keys, const int32_t *vals, int64_t n,
                               int32_t key_bits, uint64_t *keys_out, int32_t *vals_out,
                               void *workspace, int64_t workspace_bytes, void *stream)
{
    if (!keys || !keys_out || !vals_out || !workspace || n < 0 || key_bits < 0 || key_bits > 64 ||
        n > INT32_MAX)
        return hdfe_set_arg_error("hdfe_sort_pairs: bad argument");
    if (workspace_bytes < hdfe_sort_workspace_bytes(n))
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_sort_pairs: workspace too small");
    if (n == 0) return HDFE_OK;
    cudaStream_t s = (cudaStream_t)stream;
    sorting::Work w = sorting::layout(workspace, n);
    HDFE_CUDA_TRY(cudaMemcpyAsync(w.keys[0], keys, n * 8, cudaMemcpyDeviceToDevice, s));
    if (vals) {
        HDFE_CUDA_TRY(cudaMemcpyAsync(w.vals[0], vals, n * 4, cudaMemcpyDeviceToDevice, s));
    } else {
        sorting::k_iota<<<sorting::grid_for(n), sorting::kThreads, 0, s>>>(w.vals[0], n);
        hdfe_add_launches(1);
    }
    int which = 0;
    sorting::radix_sort(w, n, key_bits, &which, s);
    HDFE_CUDA_TRY(cudaMemcpyAsync(keys_out, w.keys[which], n * 8, cudaMemcpyDeviceToDevice, s));
    HDFE_CUDA_TRY(cudaMemcpyAsync(vals_out, w.vals[which], n * 4, cudaMemcpyDeviceToDevice, s));
    HDFE_CUDA_TRY(cudaGetLastError());
    return HDFE_OK;
}

extern "C" int hdfe_factorize(const uint64_t *ids, int64_t n, int32_t key_bits, int32_t *codes,
                              uint64_t *levels, int64_t *n_levels, void *workspace,
                              int64_t workspace_bytes, void *stream)
{
    if (!ids || !codes || !n_levels || !workspace || n < 1 || key_bits < 0 || key_bits > 64 ||
        n > INT32_MAX)
        return hdfe_set_arg_error("hdfe_factorize: bad argument");
    if (workspace_bytes < hdfe_sort_workspace_bytes(n))
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_factorize: workspace too small");
    cudaStream_t s = (cudaStream_t)stream;
    sorting::Work w = sorting::layout(workspace, n);
    HDFE_CUDA_TRY(cudaMemcpyAsync(w.keys[0], ids, n * 8, cudaMemcpyDeviceToDevice, s));
    const unsigned grid = sorting::grid_for(n);
    sorting::k_iota<<<grid, sorting::kThreads, 0, s>>>(w.vals[0], n);
    int which = 0;
    sorting::radix_sort(w, n, key_bits, &which, s);
    // the heads in the spare key buffer (n x 8 bytes), their scan in offsets
    uint32_t *heads = reinterpret_cast<uint32_t *>(w.keys[1 - which]);
    sorting::k_heads<<<grid, sorting::kThreads, 0, s>>>(w.keys[which], n, heads);
    sorting::scan(heads, n, w.sums, w.offsets, s);
    sorting::k_ranks<<<grid, sorting::kThreads, 0, s>>>(w.keys[which], w.vals[which], heads,
                                                        w.offsets, n, codes, levels, n_levels);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(6);
    return HDFE_OK;
}
