// X' W X of a wide design on the 5th-generation tensor cores (split BF16).
//
// Reference: core/inference.py:109-137 `_assemble`, where the reference forms
// the design's cross-products with a BLAS `V.T @ V` in FP64.  For a design of
// c <= 128 columns and N rows, each CTA takes chunks of kRows rows:
//   * its threads load the chunk (FP64, rows scaled by sqrt(w)), split every
//     value into x = hi + lo with hi = bf16(x) and lo = bf16(x - hi), and store
//     hi and lo as the K-major operand tile (M = 128 features x K = kRows
//     rows, core matrices of 8 features x 8 rows, 128 bytes each, no swizzle)
//     of one of two shared-memory stages;
//   * one thread issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32) for
//     D += hi hi' + hi lo' + lo hi' over the chunk's K steps, the same tile
//     serving as A (128 x K) and B (N x K, its first N features); D is a
//     128 x N FP32 accumulator in tensor memory, held across the CTA's chunks;
//     tcgen05.commit signals the stage's mbarrier when the products that read
//     it are done, so the stage is refilled while the other one is multiplied.
// At the end each warp of the first four reads its 32 lanes of D (tcgen05.ld),
// the CTA writes its partial (FP64), and a second kernel sums the CTAs'
// partials in a fixed order.  The dropped lo lo' term and FP32 accumulation
// within a CTA leave a relative error of about 1e-5 per entry; the FP64 sums
// over CTAs keep it from growing with N.
//   Every mbarrier wait is bounded (kSpinLimitNs); a timeout records
// HDFE_ERR_SPIN_LIMIT in the status word, waits (bounded) for the products
// still in flight, frees the tensor memory and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.cuh"

namespace hdfe {
namespace gram {

constexpr int kThreads = 256;
constexpr int kM = 128;             // features per tile (the MMA's M)
constexpr int kRows = 64;           // rows per chunk (K): 4 MMA steps of 16
constexpr int kStages = 2;
constexpr int kSBO = (kRows / 8) * 128;     // bytes between 8-feature groups
constexpr int kTileBytes = (kM / 8) * kSBO; // one operand tile: 16 KB

__device__ __forceinline__ unsigned smem_u32(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

// K-major, no-swizzle shared-memory matrix descriptor (sm_100 layout):
// start address >> 4, leading byte offset (K direction: 128 B between core
// matrices) >> 4, stride byte offset (M/N direction) >> 4, version 1
__device__ __forceinline__ uint64_t smem_desc(unsigned addr)
{
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) |
           ((uint64_t)(kSBO >> 4) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D FP32, A and B BF16, both K-major, N, M
__host__ __device__ constexpr uint32_t instr_desc(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(kM >> 4) << 24);
}

// byte offset of element (feature m, row k) in an operand tile
__device__ __forceinline__ int tile_offset(int m, int k)
{
    return (m >> 3) * kSBO + (k >> 3) * 128 + (m & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity)
{
    const unsigned long long t0 = global_ns();
    for (;;) {
        unsigned done;
        asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;"
                     " selp.u32 %0, 1, 0, p; }"
                     : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
        if (global_ns() - t0 > kSpinLimitNs) return false;
    }
}

struct Args {
    const double *X;        // (N, c) row-major
    const double *w;        // (N) or null
    int64_t N;
    int c, n_pad;           // n_pad: c rounded up to 16 (the MMA's N)
    int tmem_cols;          // power of two >= max(32, n_pad)
    double *partial;        // (gridDim.x, c, c)
    unsigned *status;
};

__global__ void __launch_bounds__(kThreads, 1) k_gram(Args a)
{
    extern __shared__ __align__(1024) unsigned char s_dyn[];
    // stage s: hi tile at s * 2 * kTileBytes, lo tile right after it
    __shared__ __align__(8) uint64_t s_bar[kStages];
    __shared__ uint32_t s_tmem;
    __shared__ int s_ok;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int c = a.c;
    const int64_t nchunks = (a.N + kRows - 1) / kRows;

    // zero both stages (features c .. 127 stay zero), the barriers, TMEM
    for (int i = tid; i < kStages * 2 * kTileBytes / 16; i += kThreads)
        reinterpret_cast<uint4 *>(s_dyn)[i] = make_uint4(0, 0, 0, 0);
    if (tid == 0) {
        for (int s = 0; s < kStages; s++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(s_bar + s))
                         : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_ok = 1;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&s_tmem)), "r"(a.tmem_cols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = instr_desc(a.n_pad);

    unsigned phase = 0;         // bit s: the parity of stage s's next wait
    int64_t uses[kStages] = {0, 0};
    bool first = true;
    int it = 0;
    for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x, it++) {
        const int s = it & 1;
        unsigned char *hi = s_dyn + s * 2 * kTileBytes;
        unsigned char *lo = hi + kTileBytes;
        // the products that last read this stage are done
        if (uses[s] > 0) {
            if (!mbar_wait(smem_u32(s_bar + s), (phase >> s) & 1u)) {
                if (tid == 0) atomicCAS(a.status, 0u, (unsigned)HDFE_ERR_SPIN_LIMIT);
                s_ok = 0;
            }
            phase ^= 1u << s;
        }
        __syncthreads();
        if (!s_ok) break;
        // load, scale, split and store the chunk's rows (row-major elements,
        // 16 loads in flight per thread)
        const int64_t r0 = ch * kRows;
        const int nrow = (int)min((int64_t)kRows, a.N - r0);
        const int total = kRows * c;
        for (int e0 = tid; e0 < total; e0 += 16 * kThreads) {
            double v[16];
#pragma unroll
            for (int u = 0; u < 16; u++) {
                const int e = e0 + u * kThreads;
                const int k = e / c;
                v[u] = (e < total && k < nrow) ? __ldcs(a.X + (r0 + k) * c + (e - k * c)) : 0.0;
                if (a.w && e < total && k < nrow) v[u] *= sqrt(__ldg(a.w + r0 + k));
            }
#pragma unroll
            for (int u = 0; u < 16; u++) {
                const int e = e0 + u * kThreads;
                if (e >= total) break;
                const int k = e / c, m = e - k * c;
                const __nv_bfloat16 h = __float2bfloat16_rn((float)v[u]);
                const __nv_bfloat16 l =
                    __float2bfloat16_rn((float)(v[u] - (double)__bfloat162float(h)));
                const int off = tile_offset(m, k);
                *reinterpret_cast<__nv_bfloat16 *>(hi + off) = h;
                *reinterpret_cast<__nv_bfloat16 *>(lo + off) = l;
            }
        }
        // the generic-proxy stores become visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned hb = smem_u32(hi), lb = smem_u32(lo);
#pragma unroll
            for (int kk = 0; kk < kRows / 16; kk++) {
                const uint64_t dh = smem_desc(hb + kk * 256), dl = smem_desc(lb + kk * 256);
                const unsigned acc0 = (first && kk == 0) ? 0u : 1u;
                // D (+)= hi hi', then += hi lo' and lo hi'
                asm volatile("{ .reg .pred p; setp.ne.u32 p, %4, 0;"
                             " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p; }"
                             :: "r"(tmem), "l"(dh), "l"(dh), "r"(idesc), "r"(acc0) : "memory");
                asm volatile("{ .reg .pred p; setp.ne.u32 p, %4, 0;"
                             " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p; }"
                             :: "r"(tmem), "l"(dh), "l"(dl), "r"(idesc), "r"(1u) : "memory");
                asm volatile("{ .reg .pred p; setp.ne.u32 p, %4, 0;"
                             " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p; }"
                             :: "r"(tmem), "l"(dl), "l"(dh), "r"(idesc), "r"(1u) : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(smem_u32(s_bar + s)) : "memory");
        }
        uses[s]++;
        first = false;
    }
    // every product issued is done: one more wait per stage in use, for its
    // last commit (bounded, also after a timeout above)
    for (int s = 0; s < kStages; s++) {
        if (uses[s] > 0 && !mbar_wait(smem_u32(s_bar + s), (phase >> s) & 1u)) {
            if (tid == 0) atomicCAS(a.status, 0u, (unsigned)HDFE_ERR_SPIN_LIMIT);
        }
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    // D to this CTA's FP64 partial: warp w (of the first four) reads lanes
    // 32 w .. 32 w + 31 (features), 8 columns per load
    if (warp < 4) {
        const int m = warp * 32 + lane;
        double *dst = a.partial + (int64_t)blockIdx.x * c * c;
        for (int n0 = 0; n0 < a.n_pad; n0 += 8) {
            uint32_t r[8];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)n0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                           "=r"(r[6]), "=r"(r[7])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < c) {
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const int n = n0 + u;
                    if (n < c) dst[m * c + n] = first ? 0.0 : (double)__uint_as_float(r[u]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(a.tmem_cols) : "memory");
}

// out[q] = sum over CTAs of partial[b, q], in CTA order
__global__ void k_gram_sum(const double *partial, int64_t blocks, int64_t cc, double *out)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= cc) return;
    double s = 0.0;
    for (int64_t b = 0; b < blocks; b++) s += partial[b * cc + q];
    out[q] = s;
}

inline int grid_for(int64_t N)
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    const int64_t chunks = (N + kRows - 1) / kRows;
    return (int)(chunks < sms ? (chunks > 0 ? chunks : 1) : sms);
}

constexpr int kSmemBytes = kStages * 2 * kTileBytes;

}  // namespace gram
}  // namespace hdfe

using namespace hdfe;

extern "C" int64_t hdfe_gram_workspace_bytes(int64_t n_rows, int32_t c)
{
    if (n_rows < 0 || c < 1 || c > HDFE_GRAM_MAX_COLS) return -1;
    const int blocks = gram::grid_for(n_rows);
    if (blocks < 1) return -1;
    return (int64_t)blocks * c * c * 8 + 256;
}

extern "C" int hdfe_gram_bf16x3(const double *X, int64_t n_rows, int32_t c, const double *w,
                                double *out, void *workspace, int64_t workspace_bytes,
                                void *stream)
{
    if (!X || !out || !workspace || n_rows < 1 || c < 1 || c > HDFE_GRAM_MAX_COLS)
        return hdfe_set_arg_error("hdfe_gram_bf16x3: bad argument");
    const int64_t need = hdfe_gram_workspace_bytes(n_rows, c);
    if (need < 0) return hdfe_set_cuda_error(cudaGetLastError());
    if (workspace_bytes < need)
        return hdfe_set_error(HDFE_ERR_WORKSPACE, "hdfe_gram_bf16x3: workspace too small");
    cudaStream_t s = (cudaStream_t)stream;
    gram::Args a;
    a.X = X;
    a.w = w;
    a.N = n_rows;
    a.c = c;
    a.n_pad = ((c + 15) / 16) * 16;
    int cols = 32;
    while (cols < a.n_pad) cols <<= 1;
    a.tmem_cols = cols;
    const int blocks = gram::grid_for(n_rows);
    a.partial = (double *)((char *)workspace + 256);
    a.status = (unsigned *)workspace;
    HDFE_CUDA_TRY(cudaMemsetAsync(workspace, 0, 16, s));
    HDFE_CUDA_TRY(cudaFuncSetAttribute(gram::k_gram, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       gram::kSmemBytes));
    gram::k_gram<<<blocks, gram::kThreads, gram::kSmemBytes, s>>>(a);
    HDFE_CUDA_TRY(cudaGetLastError());
    const int64_t cc = (int64_t)c * c;
    gram::k_gram_sum<<<(unsigned)((cc + 255) / 256), 256, 0, s>>>(a.partial, blocks, cc, out);
    HDFE_CUDA_TRY(cudaGetLastError());
    hdfe_add_launches(2);
    return HDFE_OK;
}
