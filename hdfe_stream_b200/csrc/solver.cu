// An opaque solver handle for hosts that bind the C ABI without a CUDA
// allocator of their own (cgo, JNI, N-API): core/gpu.py:186-197
// `explicit_solver` returns a `solve(b, zero, x0)` closure that holds S and the
// preconditioner on the device and answers with host values; the handle is
// that closure.  It keeps the caller's device pointers to S and dinv (which the
// caller keeps alive), and owns the only device memory this library allocates:
// the PCG workspace for up to max_k columns, the info record and the zero
// flags.  A solve is synchronous on its stream, like the reference's (it
// returns the iteration count, the converged flag and the residual on the
// host).  One solve at a time per handle: the workspace is shared.
#include <cstdlib>
#include <cuda_runtime.h>

#include "common.cuh"

struct hdfe_solver {
    const int64_t *indptr;
    const int32_t *indices;
    const double *data;
    int64_t L, nnz;
    const double *dinv;
    double tol;
    int64_t maxiter;
    int32_t max_k;
    int device;
    void *workspace;
    int64_t workspace_bytes;
    hdfe_pcg_info *info;
    uint8_t *zero;
};

extern "C" int hdfe_solver_create(const int64_t *indptr, const int32_t *indices,
                                  const double *data, int64_t L, int64_t nnz, const double *dinv,
                                  double tol, int64_t maxiter, int32_t max_k, hdfe_solver **out)
{
    if (!out || !indptr || L < 1 || nnz < 0 || (nnz > 0 && (!indices || !data)) || !dinv ||
        !(tol > 0.0) || maxiter < 0 || max_k < 1 || max_k > HDFE_PCG_MAX_K)
        return hdfe_set_arg_error("hdfe_solver_create: bad argument");
    *out = nullptr;
    int64_t bytes = 0;
    for (int k = 1; k <= max_k; k++) {
        const int64_t b = hdfe_pcg_workspace_bytes(L, nnz, k);
        if (b < 0) return hdfe_set_error(HDFE_ERR_CUDA, "hdfe_solver_create: workspace size");
        if (b > bytes) bytes = b;
    }
    hdfe_solver *s = (hdfe_solver *)std::calloc(1, sizeof(hdfe_solver));
    if (!s) return hdfe_set_error(HDFE_ERR_CUDA, "hdfe_solver_create: out of host memory");
    s->indptr = indptr;
    s->indices = indices;
    s->data = data;
    s->L = L;
    s->nnz = nnz;
    s->dinv = dinv;
    s->tol = tol;
    s->maxiter = maxiter;
    s->max_k = max_k;
    s->workspace_bytes = bytes;
    cudaError_t e = cudaGetDevice(&s->device);
    if (e == cudaSuccess) e = cudaMalloc(&s->workspace, (size_t)bytes);
    if (e == cudaSuccess) e = cudaMalloc((void **)&s->info, sizeof(hdfe_pcg_info));
    if (e == cudaSuccess) e = cudaMalloc((void **)&s->zero, HDFE_PCG_MAX_K);
    if (e != cudaSuccess) {
        if (s->workspace) cudaFree(s->workspace);
        if (s->info) cudaFree(s->info);
        std::free(s);
        return hdfe_set_cuda_error(e);
    }
    *out = s;
    return HDFE_OK;
}

extern "C" int hdfe_solver_solve(hdfe_solver *s, const double *B, int32_t k,
                                 const uint8_t *zero_host, const double *X0, double *X,
                                 hdfe_pcg_info *info_host, void *stream)
{
    if (!s || !B || !X || !info_host || k < 1 || k > s->max_k)
        return hdfe_set_arg_error("hdfe_solver_solve: bad argument (1 <= k <= max_k)");
    int dev = -1;
    HDFE_CUDA_TRY(cudaGetDevice(&dev));
    if (dev != s->device)
        return hdfe_set_arg_error("hdfe_solver_solve: the handle belongs to another device");
    cudaStream_t st = (cudaStream_t)stream;
    const uint8_t *zp = nullptr;
    if (zero_host) {
        HDFE_CUDA_TRY(cudaMemcpyAsync(s->zero, zero_host, (size_t)k, cudaMemcpyHostToDevice, st));
        zp = s->zero;
    }
    const int rc = hdfe_pcg_solve(s->indptr, s->indices, s->data, s->L, s->nnz, s->dinv, B, k, zp,
                                  X0, s->tol, s->maxiter, X, s->workspace, s->workspace_bytes,
                                  s->info, stream);
    if (rc != HDFE_OK) return rc;
    HDFE_CUDA_TRY(cudaMemcpyAsync(info_host, s->info, sizeof(hdfe_pcg_info),
                                  cudaMemcpyDeviceToHost, st));
    HDFE_CUDA_TRY(cudaStreamSynchronize(st));
    return info_host->status;
}

extern "C" int hdfe_solver_destroy(hdfe_solver *s)
{
    if (!s) return HDFE_OK;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != s->device) cudaSetDevice(s->device);
    cudaFree(s->workspace);
    cudaFree(s->info);
    cudaFree(s->zero);
    if (prev >= 0 && prev != s->device) cudaSetDevice(prev);
    std::free(s);
    return HDFE_OK;
}
