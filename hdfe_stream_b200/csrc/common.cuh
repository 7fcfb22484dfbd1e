// Shared device helpers of libhdfe_b200: status codes, a bounded grid-wide
// barrier for the persistent (cooperatively launched) kernels, and warp/block
// reductions whose order is fixed, so sums do not depend on scheduling.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "hdfe_b200.h"

namespace hdfe {

// Upper bound on one wait in a grid barrier.  Every CTA of a cooperative
// launch is resident, so a barrier completes in microseconds; if one does not
// complete within this many nanoseconds the kernel records
// HDFE_ERR_SPIN_LIMIT and every CTA returns instead of waiting on.
constexpr unsigned long long kSpinLimitNs = 1000000000ull;   // 1 s

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(unsigned *p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

// fetch-and-add with release semantics at GPU scope: the writes this thread
// has made or observed (the CTA's, after its __syncthreads) are visible to
// whoever acquires the result
__device__ __forceinline__ unsigned atom_add_release(unsigned *p, unsigned v)
{
    unsigned old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;"
                 : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Grid barrier state: bar[0] arrivals, bar[1] generation, bar[2] error code.
// Zeroed by the host (or a set-up kernel) before the launch that uses it.
struct GridBarrier {
    unsigned *bar;

    // Returns false when the kernel must stop (an error was recorded, by this
    // CTA on a timeout or by another one).  All threads of the CTA return the
    // same value.
    //   Arrival is one release fetch-and-add (it orders the CTA's writes,
    // made visible to thread 0 by the __syncthreads, before it); the last CTA
    // resets the count and publishes the next generation with a release
    // store; the others spin on the generation alone with acquire loads,
    // looking at the error word and the clock every 32 polls (the wait stays
    // bounded by kSpinLimitNs, give or take 32 polls).
    __device__ bool sync() const
    {
        __shared__ int s_ok;
        __syncthreads();
        if (threadIdx.x == 0) {
            int ok = 1;
            const unsigned gen = ld_acquire(bar + 1);
            const unsigned arrived = atom_add_release(bar, 1u);
            if (arrived == gridDim.x - 1) {
                bar[0] = 0;                 // ordered before the release below
                st_release(bar + 1, gen + 1);
            } else {
                const unsigned long long t0 = global_ns();
                for (unsigned polls = 1; ld_acquire(bar + 1) == gen; polls++) {
                    if ((polls & 31u) == 0) {
                        if (ld_acquire(bar + 2) != 0) { ok = 0; break; }
                        if (global_ns() - t0 > kSpinLimitNs) {
                            atomicCAS(bar + 2, 0u, (unsigned)HDFE_ERR_SPIN_LIMIT);
                            ok = 0;
                            break;
                        }
                    }
                }
            }
            if (ok && ld_acquire(bar + 2) != 0) ok = 0;
            s_ok = ok;
        }
        __syncthreads();
        return s_ok != 0;
    }

    __device__ void fail(int code) const { atomicCAS(bar + 2, 0u, (unsigned)code); }
};

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Fixed-order sum over the CTA of one value per thread; result valid in
// thread 0.  `scratch` holds one slot per warp.
template <typename T>
__device__ __forceinline__ T block_sum(T v, T *scratch)
{
    v = warp_sum(v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    T total = T(0);
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        for (int w = 0; w < nw; w++) total += scratch[w];
    }
    __syncthreads();
    return total;
}

}  // namespace hdfe

#define HDFE_CUDA_TRY(expr)                                            \
    do {                                                               \
        cudaError_t _e = (expr);                                       \
        if (_e != cudaSuccess) return hdfe_set_cuda_error(_e);         \
    } while (0)

int hdfe_set_cuda_error(cudaError_t e);
int hdfe_set_error(int code, const char *msg);
int hdfe_set_arg_error(const char *msg);
// counts kernels launched by the library (hdfe_kernel_launches)
void hdfe_add_launches(int n);
