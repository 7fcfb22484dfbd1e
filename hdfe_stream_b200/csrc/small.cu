// S split into its big block (CSR) and the dense small block (cross, small):
// the form hdfe_pcg_solve_small takes.  The reference keeps all of S in CSR
// (core/solve.py:148-194 `_build_explicit`); this changes the storage of the
// small dimension's rows and columns only, not the matrix.
//
//   count   a warp per row: the row's entries in big columns, and per tile
//           of kTile rows their sum;
//   scan    one CTA: exclusive offsets of the tile sums, and the total;
//   fill    per tile: the rows' offsets by a block scan of their counts, the
//           big entries copied (coalesced), the small-column entries of big
//           rows scattered into cross, the small rows' small-column entries
//           into small (their big-column entries are cross transposed: S is
//           symmetric; columns are sorted, so those are a prefix of the row).
#include <cuda_runtime.h>

#include "common.cuh"

namespace hdfe {
namespace small {

constexpr int kS = HDFE_SMALL_MAX_LEVELS;
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kPer = 8;                         // rows per thread in the tile scan
constexpr int kTile = kThreads * kPer;          // rows per CTA

__global__ void __launch_bounds__(kThreads) k_count(const int64_t *indptr,
                                                    const int32_t *indices, int64_t L,
                                                    int64_t Lb, int64_t *head, int64_t *tile_sum,
                                                    int32_t *status)
{
    __shared__ int64_t s_w[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t t0 = (int64_t)blockIdx.x * kTile;
    int64_t mine = 0;
    for (int64_t r = t0 + warp; r < min(t0 + kTile, L); r += kWarps) {
        const int64_t st = indptr[r], en = indptr[r + 1];
        int64_t n = 0;
        if (r < Lb)
            for (int64_t e = st + lane; e < en; e += 32) {
                const int32_t c = indices[e];
                n += (c >= 0 && c < Lb) ? 1 : 0;
            }
        n = warp_sum(n);
        if (lane == 0) {
            head[r] = n;
            mine += n;
            if (r < Lb && n == 0 && en > st) atomicExch(status, (int32_t)HDFE_ERR_BAD_CODE);
        }
    }
    if (lane == 0) s_w[warp] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t t = 0;
        for (int w = 0; w < kWarps; w++) t += s_w[w];
        tile_sum[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(1024) k_scan(int64_t *tile_sum, int64_t tiles, int64_t *total)
{
    __shared__ int64_t s[1024];
    int64_t carry = 0;
    for (int64_t b0 = 0; b0 < tiles; b0 += 1024) {
        const int64_t b = b0 + threadIdx.x;
        const int64_t v = b < tiles ? tile_sum[b] : 0;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            const int64_t y = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
            __syncthreads();
            s[threadIdx.x] += y;
            __syncthreads();
        }
        if (b < tiles) tile_sum[b] = carry + s[threadIdx.x] - v;
        carry += s[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kThreads) k_fill(const int64_t *indptr, const int32_t *indices,
                                                   const double *data, int64_t L, int64_t Lb,
                                                   int ns, const int64_t *head,
                                                   const int64_t *tile_off, int64_t *indptr_out,
                                                   int32_t *indices_out, double *data_out,
                                                   double *cross, double *small,
                                                   int32_t *status)
{
    __shared__ int64_t s_off[kTile];
    __shared__ int64_t s_w[kWarps + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t t0 = (int64_t)blockIdx.x * kTile;
    // the tile's row offsets: kPer consecutive rows a thread, then a block scan
    int64_t v[kPer], run = 0;
#pragma unroll
    for (int i = 0; i < kPer; i++) {
        const int64_t r = t0 + threadIdx.x * kPer + i;
        v[i] = r < L ? head[r] : 0;
        run += v[i];
    }
    int64_t inc = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t t = 0;
        for (int w = 0; w < kWarps; w++) { const int64_t x = s_w[w]; s_w[w] = t; t += x; }
        s_w[kWarps] = t;
    }
    __syncthreads();
    int64_t at = tile_off[blockIdx.x] + s_w[warp] + inc - run;
#pragma unroll
    for (int i = 0; i < kPer; i++) {
        s_off[threadIdx.x * kPer + i] = at;
        at += v[i];
    }
    __syncthreads();
    for (int64_t r = t0 + warp; r < min(t0 + kTile, L); r += kWarps) {
        const int64_t st = indptr[r], en = indptr[r + 1];
        const int64_t o = s_off[r - t0];
        if (lane == 0) indptr_out[r] = o;
        if (r < Lb) {
            // big entries keep their order: each one's place is the count of
            // big entries before it (a ballot per 32 entries)
            int64_t done = 0;
            for (int64_t b = st; b < en; b += 32) {
                const int64_t e = b + lane;
                const int32_t c = e < en ? indices[e] : 0;
                const bool big = e < en && c >= 0 && c < Lb;
                const unsigned m = __ballot_sync(0xffffffffu, big);
                if (big) {
                    const int64_t pos = o + done + __popc(m & ((1u << lane) - 1));
                    indices_out[pos] = c;
                    data_out[pos] = data[e];
                } else if (e < en) {
                    if (c >= Lb && c < Lb + ns) cross[r * kS + (c - Lb)] = data[e];
                    else atomicExch(status, (int32_t)HDFE_ERR_BAD_CODE);
                }
                done += __popc(m);
            }
        } else {
            // a small row: its small-column entries are the row's tail (sorted
            // columns), found by a binary search rather than a walk over the
            // row's big columns (a year meets every firm)
            int64_t lo = st, hi = en;
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (indices[mid] < Lb) lo = mid + 1; else hi = mid;
            }
            for (int64_t e = lo + lane; e < en; e += 32) {
                const int32_t c = indices[e];
                if (c >= Lb && c < Lb + ns) small[(r - Lb) * ns + (c - Lb)] = data[e];
                else atomicExch(status, (int32_t)HDFE_ERR_BAD_CODE);
            }
        }
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0)
        indptr_out[L] = tile_off[blockIdx.x] + s_w[kWarps];
}

}  // namespace small
}  // namespace hdfe

using namespace hdfe;

extern "C" int64_t hdfe_small_split_workspace_bytes(int64_t L)
{
    if (L < 1) return -1;
    const int64_t tiles = (L + small::kTile - 1) / small::kTile;
    return (L * 8 + 255) / 256 * 256 + (tiles * 8 + 255) / 256 * 256;
}

extern "C" int hdfe_small_split(const int64_t *indptr, const int32_t *indices, const double *data,
                                int64_t L, int64_t small_first, int32_t small_count,
                                int64_t *indptr_out, int32_t *indices_out, double *data_out,
                                double *cross, double *small_block, int64_t *nnz_out,
                                int32_t *status_out, void *workspace, int64_t workspace_bytes,
                                void *stream)
{
    if (!indptr || !indptr_out || !cross || !small_block || !nnz_out || !status_out ||
        !workspace || L < 2 || small_count < 1 || small_count > HDFE_SMALL_MAX_LEVELS ||
        small_first < 1 || small_first + small_count != L || small_first > INT32_MAX)
        return hdfe_set_arg_error("hdfe_small_split: bad argument");
    if (workspace_bytes < hdfe_small_split_workspace_bytes(L))
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_small_split: workspace too small");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t tiles = (L + small::kTile - 1) / small::kTile;
    int64_t *head = (int64_t *)workspace;
    int64_t *tile = (int64_t *)((char *)workspace + (L * 8 + 255) / 256 * 256);
    HDFE_CUDA_TRY(cudaMemsetAsync(cross, 0, small_first * small::kS * 8, s));
    HDFE_CUDA_TRY(cudaMemsetAsync(small_block, 0, (int64_t)small_count * small_count * 8, s));
    HDFE_CUDA_TRY(cudaMemsetAsync(status_out, 0, 4, s));
    small::k_count<<<(unsigned)tiles, small::kThreads, 0, s>>>(indptr, indices, L, small_first,
                                                               head, tile, status_out);
    small::k_scan<<<1, 1024, 0, s>>>(tile, tiles, nnz_out);
    small::k_fill<<<(unsigned)tiles, small::kThreads, 0, s>>>(
        indptr, indices, data, L, small_first, small_count, head, tile, indptr_out, indices_out,
        data_out, cross, small_block, status_out);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(3);
    return HDFE_OK;
}
