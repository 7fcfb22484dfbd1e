// Error reporting and version of libhdfe_b200.
#include <cstdio>
#include <atomic>
#include <cstring>
#include <cuda_runtime.h>

#include "common.cuh"

namespace {
thread_local char g_msg[512] = "no error";
std::atomic<long long> g_launches{0};
}

void hdfe_add_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

extern "C" int64_t hdfe_kernel_launches(void) { return g_launches.load(); }

int hdfe_set_cuda_error(cudaError_t e)
{
    std::snprintf(g_msg, sizeof g_msg, "CUDA error %d: %s", (int)e, cudaGetErrorString(e));
    return HDFE_ERR_CUDA;
}

int hdfe_set_error(int code, const char *msg)
{
    std::snprintf(g_msg, sizeof g_msg, "%s", msg);
    return code;
}

int hdfe_set_arg_error(const char *msg) { return hdfe_set_error(HDFE_ERR_ARG, msg); }

extern "C" const char *hdfe_error_string(void) { return g_msg; }

extern "C" const char *hdfe_version(void) { return "hdfe_b200 0.1.0 (sm_100a)"; }
