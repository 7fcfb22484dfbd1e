/*
 * hdfe_b200.h -- C ABI of libhdfe_b200.so, the B200 (sm_100a) implementation
 * of hdfe-stream's fixed-effects solve path.
 *
 * Conventions
 *   - Every pointer argument is a DEVICE pointer unless its comment says host.
 *     The caller owns every buffer; the library allocates no device memory
 *     (the scratch each kernel needs is a caller-provided workspace whose size
 *     a *_workspace_bytes function gives).
 *   - `stream` is a cudaStream_t passed as void* (NULL = the legacy default
 *     stream).  Calls are asynchronous on it unless stated otherwise.
 *   - Return value: HDFE_OK (0) or an HDFE_ERR_* code; hdfe_error_string()
 *     describes the last error on the calling thread.
 *   - Layouts are the reference's: row-major (C-order) float64 matrices,
 *     level codes (M, D) uint32, group boundaries `starts` (G+1) int64, CSR
 *     indptr int64 / indices int32 / data float64 with sorted columns.
 *
 * Each entry point cites the reference (hdfe-stream v0.13.4) interface it
 * replaces, by file:line.
 */
#ifndef HDFE_B200_H
#define HDFE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    HDFE_OK = 0,
    HDFE_ERR_ARG = 1,          /* invalid argument (size, null pointer, k out of range) */
    HDFE_ERR_CUDA = 2,         /* a CUDA runtime call failed; see hdfe_error_string() */
    HDFE_ERR_SPIN_LIMIT = 3,   /* a grid-wide wait timed out; the kernel returned early */
    HDFE_ERR_WORKSPACE = 4,    /* the workspace given is smaller than required */
    HDFE_ERR_BAD_CODE = 5,     /* a level code is out of range for its dimension */
    HDFE_ERR_CAPACITY = 6      /* a per-row or per-group capacity of a kernel was exceeded */
};

/* Message for the last error returned on this thread. */
const char *hdfe_error_string(void);

/* Library version string. */
const char *hdfe_version(void);

/* ------------------------------------------------------------ step 2: PCG
 *
 * Jacobi-preconditioned block conjugate gradients on the reduced matrix S,
 * one CG per right-hand-side column in lockstep, in one persistent launch:
 * the SpMM, the vector updates and the column reductions of every iteration
 * run on the device, with the convergence test on the device too (no host
 * round trip per iteration).
 *
 * Replaces core/gpu.py:199-253 `pcg` (and its CPU twin, core/solve.py:66-140
 * `_SolveMixin._pcg`): same `zero` columns (solved by X = 0, no iterations),
 * warm start X0, per-column alpha/beta, `active = rel > tol` with
 * rel = ||R|| / ||B|| (||B|| = 0 taken as 1), iteration count, converged flag
 * and max relative residual.
 */
typedef struct hdfe_pcg_info {
    int64_t iterations;   /* CG iterations run (0 if nothing to do) */
    int32_t converged;    /* 1 when every column met tol */
    int32_t status;       /* HDFE_OK, or HDFE_ERR_SPIN_LIMIT */
    double max_rel;       /* max over columns of ||R|| / ||B|| at exit */
} hdfe_pcg_info;

/* Largest k (right-hand-side columns per solve) hdfe_pcg_solve accepts. */
#define HDFE_PCG_MAX_K 8

/* Device workspace bytes hdfe_pcg_solve needs (for the current device). */
int64_t hdfe_pcg_workspace_bytes(int64_t L, int64_t nnz, int32_t k);

/* Solve S X = B for X (L, k).
 *   indptr (L+1) int64, indices (nnz) int32, data (nnz) float64: S in CSR
 *   (nnz = indptr[L], passed by the caller so the call stays asynchronous)
 *   dinv (L): inverse diagonal (0 where the diagonal is <= 1e-12)
 *   B (L, k); zero (k) uint8 or NULL; X0 (L, k) or NULL; X (L, k) out
 *   info: DEVICE pointer to one hdfe_pcg_info, written at exit.
 * Non-convergence is reported in info, not as an error (the reference warns).
 */
int hdfe_pcg_solve(const int64_t *indptr, const int32_t *indices, const double *data,
                   int64_t L, int64_t nnz, const double *dinv, const double *B, int32_t k,
                   const uint8_t *zero, const double *X0, double tol, int64_t maxiter,
                   double *X, void *workspace, int64_t workspace_bytes,
                   hdfe_pcg_info *info, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* HDFE_B200_H */
