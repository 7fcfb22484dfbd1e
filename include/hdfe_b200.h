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

/* Kernels this library has launched in this process (all entry points). */
int64_t hdfe_kernel_launches(void);

/* Limits of the device path: non-streamed fixed-effect dimensions, and design
 * variables (outcome + covariates) per pass. */
#define HDFE_MAX_DIMS 4
#define HDFE_MAX_VARS 16

/* ------------------------------------------------------------------ pass 1
 *
 * Rows -> cells -> identifying cells, with the level bookkeeping: obs / cnt
 * per level over all cells, the Jacobi diagonal of S and the right-hand side
 * D_o' M_0 V over the identifying cells.  Replaces core/passes.py:397-531
 * `_pass1_cells` with `_cell_chunks` (:533-589), `_nb_run_sums`
 * (core/kernels_base.py:375-422), `_nb_diag` (:87-110) and `_nb_rhs`
 * (:65-83), for the plain case (no varying slopes).
 *
 * Input rows are pass 0's layout: sorted by (gcode, codes...), gcode (N)
 * uint32 the dense code of the streamed dimension, codes (N, D) uint32,
 * V (m, N) float64 one contiguous row per variable (outcome first), w (N)
 * float64 analytic weights or NULL.  n_levels (D) is a HOST array.
 * Outputs are sized for the worst case (every row its own identifying cell):
 * starts (N+1) int64, cell_codes (N, D), cell_n (N), cell_sums (N, m) or NULL,
 * group_n (N): each identifying group's sum of n; obs, cnt, diag (L), rhs
 * (L, m), means and raw_ss (m): the variables' means and sums of squared
 * deviations; lcount (L) int32 and work (L) int64, or both NULL: per level the
 * identifying groups containing it and their cells (what the S build's
 * analysis needs, `_nb_level_groups` / `_nb_row_work`, collected here while
 * the cells are at hand); counts: DEVICE pointer, the actual sizes and a
 * status (HDFE_ERR_BAD_CODE if a code is out of range).
 */
typedef struct hdfe_pass1_counts {
    int64_t n_rows, n_groups, n_cells, n_ident_groups, n_ident_cells, status;
} hdfe_pass1_counts;

int64_t hdfe_pass1_workspace_bytes(int64_t n_rows, int32_t m, int32_t keep_sums);

int hdfe_pass1(const uint32_t *gcode, const uint32_t *codes, int32_t D, const double *V,
               int32_t m, const double *w, int64_t n_rows, const int64_t *n_levels,
               double *means, double *raw_ss, int64_t *starts, uint32_t *cell_codes,
               double *cell_n, double *cell_sums, double *group_n, double *obs, double *cnt,
               double *diag, double *rhs, int32_t *lcount, int64_t *work,
               hdfe_pass1_counts *counts, void *workspace, int64_t workspace_bytes,
               void *stream);

/* ------------------------------------------------------------- explicit S
 *
 * S = D_o' M_0 D_o in CSR with sorted columns, from the identifying cells.
 * Replaces core/solve.py:148-194 `_build_explicit` and its kernels
 * core/kernels_base.py:201-358 (`_nb_level_groups`, `_nb_row_work`,
 * `_nb_row_nnz`, `_nb_row_fill`), plain case.  Three calls on one workspace
 * (hdfe_sbuild_workspace_bytes), because the sizes are data-dependent; the
 * caller reads info (a DEVICE pointer) between them:
 *   analyze  levels' classes and group lists (each entry with its group's
 *            u_r / N_g for the level); info->n_wide (wide rows) and
 *            info->temp_len (entries of the temp buffer)
 *   count    needs the wide workspace (hdfe_sbuild_wide_workspace_bytes with
 *            n_wide) and a temp buffer of temp_len * 12 bytes; writes indptr
 *            (L+1) and info->nnz
 *   fill     writes indices (nnz) int32 and data (nnz) float64
 * lcount / work: pass 1's per-level statistics (hdfe_pass1), or both NULL to
 * compute them here.  The same workspace, wide workspace and temp buffer go
 * to all three calls.
 */
typedef struct hdfe_sbuild_info {
    int64_t L, nnz, n_wide, n_warp_rows, n_block_rows, lgrp_len, temp_len, status;
} hdfe_sbuild_info;

int64_t hdfe_sbuild_workspace_bytes(int64_t L, int64_t n_cells, int32_t D);
int64_t hdfe_sbuild_wide_workspace_bytes(int64_t L, int64_t n_cells, int32_t D, int64_t n_wide);

int hdfe_sbuild_analyze(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                        int32_t D, const double *n, const double *group_n, int64_t n_cells,
                        const int64_t *n_levels, const int32_t *lcount, const int64_t *work,
                        void *workspace, int64_t workspace_bytes, hdfe_sbuild_info *info,
                        void *stream);

int hdfe_sbuild_count(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                      int32_t D, const double *n, const double *group_n, int64_t n_cells,
                      const int64_t *n_levels, const int32_t *lcount, const int64_t *work,
                      int64_t n_wide, int64_t temp_len, int64_t *indptr, void *workspace,
                      int64_t workspace_bytes, void *wide_workspace,
                      int64_t wide_workspace_bytes, void *temp, int64_t temp_bytes,
                      hdfe_sbuild_info *info, void *stream);

int hdfe_sbuild_fill(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                     int32_t D, const double *n, const double *group_n, int64_t n_cells,
                     const int64_t *n_levels, const int32_t *lcount, const int64_t *work,
                     int64_t n_wide, int64_t temp_len, const int64_t *indptr, int32_t *indices,
                     double *data, void *workspace, int64_t workspace_bytes,
                     void *wide_workspace, int64_t wide_workspace_bytes, void *temp,
                     int64_t temp_bytes, hdfe_sbuild_info *info, void *stream);

/* The same build in the split form hdfe_pcg_solve_small takes (see the
 * dense small block below): the levels [small_first, L), the trailing
 * dimensions' levels (1 .. HDFE_SMALL_MAX_LEVELS of them), are the wide rows
 * by force; the CSR (indptr over all L rows, rows >= small_first empty)
 * holds S's big block only, cross (small_first x HDFE_SMALL_MAX_LEVELS) and
 * small (small_count x small_count) the rest, with the very values of the
 * full build (the same additions in the same order).  n_wide must be
 * small_count.  info->status is HDFE_ERR_CAPACITY when a big level is too
 * wide for a narrow row (then build the full CSR and split it with
 * hdfe_small_split).  The workspaces are sized as for the full build. */
int hdfe_sbuild_analyze_split(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                              int32_t D, const double *n, const double *group_n,
                              int64_t n_cells, const int64_t *n_levels, const int32_t *lcount,
                              const int64_t *work, int64_t small_first, int32_t small_count,
                              void *workspace, int64_t workspace_bytes, hdfe_sbuild_info *info,
                              void *stream);

int hdfe_sbuild_count_split(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                            int32_t D, const double *n, const double *group_n, int64_t n_cells,
                            const int64_t *n_levels, const int32_t *lcount, const int64_t *work,
                            int64_t n_wide, int64_t temp_len, int64_t small_first,
                            int32_t small_count, int64_t *indptr, double *cross, double *small,
                            void *workspace, int64_t workspace_bytes, void *wide_workspace,
                            int64_t wide_workspace_bytes, void *temp, int64_t temp_bytes,
                            hdfe_sbuild_info *info, void *stream);

int hdfe_sbuild_fill_split(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                           int32_t D, const double *n, const double *group_n, int64_t n_cells,
                           const int64_t *n_levels, const int32_t *lcount, const int64_t *work,
                           int64_t n_wide, int64_t temp_len, const int64_t *indptr,
                           int32_t *indices, double *data, void *workspace,
                           int64_t workspace_bytes, void *wide_workspace,
                           int64_t wide_workspace_bytes, void *temp, int64_t temp_bytes,
                           hdfe_sbuild_info *info, void *stream);

/* ------------------------------------------------ components, normalisation
 *
 * hdfe_components: union-find over dimension `col` of the identifying cells
 * (levels sharing a group are connected).  Replaces core/kernels_base.py:
 * 156-174 `_nb_components`: root (n_levels) int32 out is each level's
 * component root, its smallest level, as the reference's; n_components is a
 * DEVICE int64[2]: the number of components, then a status.  Ranking the
 * roots by rows (core/passes.py:933-950) is left to the caller.
 *
 * hdfe_normalize: core/solve.py:383-399 `_normalize` on Gamma (L, m) in place:
 * the first dimension's effects get obs-weighted mean zero within each
 * component (root from hdfe_components), further dimensions obs-weighted mean
 * zero.  n_levels (D) is a HOST array.
 */
int64_t hdfe_components_workspace_bytes(void);
int hdfe_components(const int64_t *starts, int64_t n_groups, const uint32_t *codes, int32_t D,
                    int32_t col, int64_t n_levels, int32_t *root, int64_t *n_components,
                    void *workspace, int64_t workspace_bytes, void *stream);

int64_t hdfe_normalize_workspace_bytes(int64_t n_first, int32_t m);
int hdfe_normalize(double *gamma, int32_t m, int32_t D, const int64_t *n_levels,
                   const double *obs, const int32_t *root, void *workspace,
                   int64_t workspace_bytes, void *stream);

/* ------------------------------------------------------- inverse operator
 *
 * Row passes of A S^- A' for the leave-out estimators.  Rows are pass 0's
 * (sorted by the streamed group), `starts` (G+1) their group boundaries
 * (hdfe_row_groups).  The vectors are either explicit, R (N, B) row-major, or
 * (R NULL) Rademacher draws regenerated from (seed, ordinal0 + row,
 * first_draw + j) -- core/kernels_groups.py:53-76 `_nb_rademacher`,
 * bit-identical.  B <= 32 vectors per pass; X (N, c) covariates, c <= 8, or
 * NULL; w (N) weights or NULL for ones; sqrt_weights: the square-root weight
 * metric (vectors scaled by w^(-1/2) going in and w^(1/2) coming out,
 * inverse.py:280-303).  n_levels is a HOST array.
 *
 * hdfe_row_groups: `starts` of rows sorted by gcode; n_groups a DEVICE int64.
 * hdfe_rows_center: kernels_inverse.py:35-71 `_nb_center_rows`: acc (L, B)
 *   = D_o' W M_0 R, acc_x (c, B) = X' W M_0 R, squares (B) = sum w R^2.
 * hdfe_rows_project: kernels_inverse.py:75-107 `_nb_project_rows` given the
 *   solution U (L, B) and covariate block C (c, B): out (N, B) = (A u)_i, and
 *   / or moments (5, N) += the JLA sink's five sums per row over the block
 *   (leaveout.py:181-190).
 * hdfe_jla_combine: leaveout.py:210-282 `_combine_moments` in place: slots
 *   0, 1, 2 of moments become the leverage, its complement and the
 *   non-linearity factor.
 */
int64_t hdfe_row_groups_workspace_bytes(int64_t n_rows);
int hdfe_row_groups(const uint32_t *gcode, int64_t n_rows, int64_t *starts, int64_t *n_groups,
                    void *workspace, int64_t workspace_bytes, void *stream);

int hdfe_rows_center(const int64_t *starts, int64_t n_groups, const uint32_t *codes, int32_t D,
                     const int64_t *n_levels, const double *w, const double *X, int32_t c,
                     const double *R, int32_t B, uint64_t seed, int64_t first_draw,
                     int64_t ordinal0, int32_t sqrt_weights, double *acc, double *acc_x,
                     double *squares, void *workspace, int64_t workspace_bytes, void *stream);

int hdfe_rows_project(const int64_t *starts, int64_t n_groups, const uint32_t *codes, int32_t D,
                      const int64_t *n_levels, const double *w, const double *X, int32_t c,
                      const double *C, const double *U, const double *R, int32_t B,
                      uint64_t seed, int64_t first_draw, int64_t ordinal0, int32_t sqrt_weights,
                      int64_t n_rows, double *out, double *moments, void *stream);

int hdfe_jla_combine(double *moments, int64_t n_rows, int64_t n_draws, void *stream);

/* Coefficient-space right-hand sides (inverse.py:311-374 `apply_inverse`) and
 * the Hutchinson trace's moments (leaveout.py:321-448).  Same row layout and
 * argument conventions as above; `status` is a DEVICE uint32 that a bad code
 * sets to HDFE_ERR_BAD_CODE, or NULL.  acc / acc_x are ADDED into (zero them
 * first); sums over rows are in atomic order (FP64).
 *
 * hdfe_rows_reduce: kernels_inverse.py:112-130 `_nb_reduce_rows` (no
 *   centring) of either explicit rows R (N, B) or, with R NULL, the streamed
 *   block `streamed` (G, B) spread over each group's rows divided by its
 *   weight total (kernels_inverse.py:134-152 `_nb_spread_groups`):
 *   acc[level, j] += w_i R_ij, acc_x[c, j] += X_ic w_i R_ij; with explicit R,
 *   group_sums (G, B) (or NULL) = sum over the group of w_i R_ij
 *   (core/kernels_groups.py:17-27 `_nb_group_sums`).
 * hdfe_rows_project_coef: kernels_inverse.py:157-188 `_nb_project_coef` for
 *   the solution U (L, B), C (c, B) and the spread streamed block: rows
 *   (N, B) = (A u)_i and groups (G, B) = the streamed block (either may be
 *   NULL); with omega (N) given, also the collect sink of the Hutchinson
 *   trace (leaveout.py:423-431) in the same pass: v_i = omega_i (A u)_i
 *   reduced as hdfe_rows_reduce does into acc, acc_x and group_sums.
 * hdfe_trace_moments: kernels_inverse.py:192-231 `_nb_trace_moments`: out
 *   (B, 8) = per vector the eight weighted sums over rows of the psi
 *   dimension's values a (from Z_levels, U_levels (L, B)) and the streamed
 *   values b (Z_groups, U_groups (G, B)); the sums are per CTA in a fixed
 *   order, then over CTAs in a fixed order.
 * hdfe_rademacher: core/kernels_groups.py:53-76 `_nb_rademacher`: out
 *   (n_rows, B) of +-1 from (seed, ordinal0 + row, first_draw + j),
 *   bit-identical.
 */
int hdfe_rows_reduce(const int64_t *starts, int64_t n_groups, const uint32_t *codes, int32_t D,
                     const int64_t *n_levels, const double *w, const double *X, int32_t c,
                     const double *streamed, const double *R, int32_t B, double *acc,
                     double *acc_x, double *group_sums, void *status, void *stream);

int hdfe_rows_project_coef(const int64_t *starts, int64_t n_groups, const uint32_t *codes,
                           int32_t D, const int64_t *n_levels, const double *w, const double *X,
                           int32_t c, const double *C, const double *U, const double *streamed,
                           int32_t B, double *rows, double *groups, const double *omega,
                           double *acc, double *acc_x, double *group_sums, void *status,
                           void *stream);

int64_t hdfe_trace_moments_workspace_bytes(int32_t B);

int hdfe_trace_moments(const int64_t *starts, int64_t n_groups, const uint32_t *codes, int32_t D,
                       const int64_t *n_levels, int32_t psi_column, const double *w,
                       const double *Z_levels, const double *Z_groups, const double *U_levels,
                       const double *U_groups, int32_t B, double *out, void *workspace,
                       int64_t workspace_bytes, void *status, void *stream);

int hdfe_rademacher(double *out, int64_t n_rows, int64_t ordinal0, int32_t B, uint64_t seed,
                    int64_t first_draw, void *stream);

/* core/kernels_base.py:478-507 `_nb_stream_matvec`: out (L, k) =
 * (D_o' M_0 D_o) P for P (L, k), k <= 32, straight from the identifying cells
 * (starts (G'+1), codes (M, D), n (M)) without forming S -- the `stream_cg`
 * solver's product.  out is overwritten; sums in atomic order. */
int hdfe_stream_matvec(const int64_t *starts, int64_t n_groups, const uint32_t *codes, int32_t D,
                       const int64_t *n_levels, const double *n, const double *P, int32_t k,
                       double *out, void *status, void *stream);

/* ------------------------------------------- connected set (pass 0's side)
 *
 * core/connected.py:378-493 `_find_components` for two fixed effects on
 * coded rows, with the min_degree core (core/kernels_graph.py:188-221
 * `_nb_peel`), union-find over the distinct pairs (:225-241
 * `_nb_union_keys`), labels numbered by root (:244-266 `_nb_dense_labels`)
 * and rows per component (:277-289 `_nb_pair_rows`).
 *
 * a, b (n_rows) uint32: the rows' codes of the two dimensions (a < n0,
 *   b < n1), sorted by a and then b (pass 0's order); rows out of order set
 *   status HDFE_ERR_ARG in counts[2].
 * k0, k1: the min_degree thresholds (1, 1: no pruning).
 * Out (DEVICE): alive (n0 + n1) uint8 (1 = in the core), labels (n0 + n1)
 *   int32 (component numbered in the order of its smallest vertex, -1 where
 *   pruned), rows (n0 + n1) int64 (rows per label; the first counts[1]
 *   used), counts[4] int64 = distinct pairs, components, status, peel rounds.
 * The peel rounds read a flag back to the host, and the call synchronises
 * the stream before returning.  Ranking the components by size (the
 * reference's stable sort) is the caller's.
 */
int64_t hdfe_pair_components_workspace_bytes(int64_t n_rows, int64_t n0, int64_t n1);

int hdfe_pair_components(const uint32_t *a, const uint32_t *b, int64_t n_rows, int64_t n0,
                         int64_t n1, int64_t k0, int64_t k1, uint8_t *alive, int32_t *labels,
                         int64_t *rows, int64_t *counts, void *workspace,
                         int64_t workspace_bytes, void *stream);

/* The leave-one-out connected set: core/connected.py:503-557 `_leave_one_out`
 * as `_find_components` (:429-447) runs it, after the (k0, k1)-core -- the
 * largest component by rows, workers (the first dimension) seen in a single
 * row removed, then every worker that is an articulation point of what is
 * left removed and the largest piece kept, until no worker is one.  Same
 * inputs as hdfe_pair_components.  Out (DEVICE): alive (n0 + n1) uint8,
 * counts[8] int64 = distinct pairs, components before, single-observation
 * workers, workers cut, cut rounds, rows kept, status, largest BFS depth.
 * The articulation points come from a breadth-first spanning tree with the
 * Tarjan-Vishkin rules instead of the reference's depth-first search; the
 * set is the same.  Reads sizes back to the host between rounds and
 * synchronises the stream before returning. */
int64_t hdfe_leave_one_out_workspace_bytes(int64_t n_rows, int64_t n0, int64_t n1);

int hdfe_leave_one_out(const uint32_t *a, const uint32_t *b, int64_t n_rows, int64_t n0,
                       int64_t n1, int64_t k0, int64_t k1, uint8_t *alive, int64_t *counts,
                       void *workspace, int64_t workspace_bytes, void *stream);

/* ------------------------------------------------- steps 3-4, KSS components
 *
 * The row passes after step 2 that the leave-out components read, on pass
 * 0's rows (row groups starts (G+1), codes (N, D), V (m, N) one row per
 * variable, y first, w (N) or NULL) and the normalised Gamma (L, m):
 *
 * hdfe_resid_moments: out (m, m) = V' W V of the variables less their
 *   fixed-effect projections Gamma and their weighted group means --
 *   core/kernels_base.py:114-146 `_nb_residualize_rows` with the row
 *   assembly of core/inference.py:109-135 `_assemble`.  Per-CTA partials,
 *   summed in a fixed order: deterministic.
 * hdfe_row_effects: for beta (m-1) and gam_y (L) = Gamma_y - Gamma_x beta
 *   (core/inference.py:454-456), the residual per row resid (N) and the
 *   streamed effect per group alpha (G) (core/kernels_base.py:544-615
 *   `_nb_pass2`; either may be NULL), and sums[7] = (w, w y, w a, w b, w a^2,
 *   w b^2, w a b) over rows, a = the effect of dimension psi_column and b =
 *   the streamed effect: the plug-in moments' sums (leaveout.py:807-833).
 * hdfe_kss_sigma2: out_i = w_i (y_i - ybar) resid_i / complement_i * factor_i,
 *   the KSS per-row variance of leaveout.py:949-1016 `_leave_one_out_sigma2`
 *   (stayers "own", weighted centring); w may be NULL.
 * status: a device uint32 that an out-of-range code sets to
 *   HDFE_ERR_BAD_CODE, or NULL.  m <= 8.
 */
int64_t hdfe_assemble_workspace_bytes(int32_t m);

int hdfe_resid_moments(const int64_t *starts, int64_t n_groups, const uint32_t *codes, int32_t D,
                       const int64_t *n_levels, const double *w, const double *V, int32_t m,
                       int64_t n_rows, const double *Gamma, double *out, void *workspace,
                       int64_t workspace_bytes, void *status, void *stream);

int hdfe_row_effects(const int64_t *starts, int64_t n_groups, const uint32_t *codes, int32_t D,
                     const int64_t *n_levels, int32_t psi_column, const double *w,
                     const double *V, int32_t m, int64_t n_rows, const double *beta,
                     const double *gam_y, double *resid, double *alpha, double *sums,
                     void *workspace, int64_t workspace_bytes, void *status, void *stream);

/* hdfe_variance_sums: the row pass's sums for the variances of beta,
 * core/kernels_base.py:544-615 `_nb_pass2` with core/inference.py:566-578
 * (OLS, analytic weights): for h the covariates V[1:] less their Gamma
 * projections and weighted group means and e the y equation's residuals,
 * out[3 T + 1] (T = k (k + 1) / 2, k = m - 1; upper triangles row by row) =
 * sum w h h', sum (w e)^2 h h', sum over the streamed groups of s s' with s
 * the group's sum of w e h, then sum w e^2.  Deterministic.  2 <= m <= 8. */
int64_t hdfe_variance_sums_workspace_bytes(int32_t m);

int hdfe_variance_sums(const int64_t *starts, int64_t n_groups, const uint32_t *codes, int32_t D,
                       const int64_t *n_levels, const double *w, const double *V, int32_t m,
                       int64_t n_rows, const double *Gamma, const double *beta, double *out,
                       void *workspace, int64_t workspace_bytes, void *status, void *stream);

/* hdfe_row_scores: the same row pass's per-row scores w e h, out (N, m - 1)
 * row-major (core/inference.py:594-603 `he`), which pass 2 sums per cluster
 * for a CRV1 term other than the streamed dimension (core/inference.py:
 * 509-510, 597-606, 656-658); h_out (N, m - 1) or NULL: the residualised
 * covariates h themselves (the per-cluster sums w h h' of the CRV3
 * jackknife, core/kernels_base.py:658-670).  2 <= m <= 8. */
int hdfe_row_scores(const int64_t *starts, int64_t n_groups, const uint32_t *codes, int32_t D,
                    const int64_t *n_levels, const double *w, const double *V, int32_t m,
                    int64_t n_rows, const double *Gamma, const double *beta, double *out,
                    double *h_out, void *status, void *stream);

int hdfe_kss_sigma2(const double *y, const double *w, const double *resid,
                    const double *complement, const double *factor, double ybar,
                    int64_t n_rows, double *out, void *stream);

/* ------------------------------------------------- KSS standard errors
 *
 * The row passes of leaveout_se.py's standard errors, in the layouts above:
 * hdfe_rows_readout: kernels_se.py:19-43 `_nb_readout`, out (N, B) =
 *   (A u)_i = U_groups[g(i)] + sum_d U_levels[level_d(i)] + x_i' U_cov,
 *   times sqrt(w_i) when w is given (NULL: not scaled).
 * hdfe_cov_cross: kernels_se.py:46-77 `_nb_cov_cross`: acc (L, B) is ADDED
 *   per psi level the sum of w_i U_groups[g(i)] (atomic order), out_groups
 *   (G, B) = per group the sum of w_i U_levels[psi(i)]; B <= 32.
 * hdfe_bii_moments: kernels_se.py:80-98 `_nb_bii_moments`: out (3, N) +=
 *   per row the sums over j < size of (root r1_j)^2, (root r2_j)^2 and
 *   root^2 r1_j r2_j, rows (N, 2 size) = [r1 | r2], root = sqrt(w) (1 if w
 *   is NULL).
 * hdfe_c_sums: leaveout_se.py:579-596 (C v per component, from v, b (3, N)
 *   and the root-scaled readouts base (N, (n_in + 3) size) of S^- X'[v | b.*v]
 *   and through_q (N, 3 size) of S^- Q S^- X'v) with the sums the first
 *   term, theta and the trace term take (:718-726, :918-925): sums[6] =
 *   per component sum_i s_k,i sum_j cv_kij^2, then sum_i y_i cv_ki0 (y NULL:
 *   0).  per_component: v is the draws z (N, size) and component k's input is
 *   z sqrt(max(s_k, 0)); else v (N, size) is shared.  Deterministic.
 * hdfe_c_sums_ext: hdfe_c_sums with low-rank terms added to C v and one
 *   more sum.  n_vec (<= 4) row vectors u (n_vec, 3, N) and coef
 *   (3, 1 + n_vec, size): cv_kij += coef[k][0][j] + sum_r u_rki
 *   coef[k][1 + r][j] -- the reference-centred kernel of the match level,
 *   K = C + (1 u' + u 1') / (2R) with u = M b (leaveout_se.py:616-636,
 *   :536-543, :591-595), and the deflated kernel C2 = C - lambda_1 x1 x1' +
 *   ... of the q = 1 interval (:580-582, :786-876).  g (3, N) non-NULL: sums
 *   has 9 entries, sums[6 + k] = sum_i g_ki cv_ki0.  coef NULL: exactly
 *   hdfe_c_sums.
 * hdfe_smooth_cells / hdfe_smooth_eval: leaveout_se.py:982-1054: each row's
 *   cell in the grid of the quantile knots (knots0 of the leverage, knots1 of
 *   B_ii or NULL for one axis; fp the rank of each knot, n_bins + 1 values
 *   each), totals / counts (n_bins^dims) ADDED per cell; and the bilinear
 *   evaluation of the cell means between cell centres.
 */
int hdfe_rows_readout(const int64_t *starts, int64_t n_groups, const uint32_t *codes, int32_t D,
                      const int64_t *n_levels, const double *X, int32_t c,
                      const double *U_levels, const double *U_cov, const double *U_groups,
                      int32_t B, const double *w, double *out, void *status, void *stream);

int hdfe_cov_cross(const int64_t *starts, int64_t n_groups, const uint32_t *codes, int32_t D,
                   const int64_t *n_levels, int32_t psi_column, const double *w,
                   const double *U_levels, const double *U_groups, int32_t B, double *acc,
                   double *out_groups, void *status, void *stream);

int hdfe_bii_moments(const double *rows, int32_t size, const double *w, int64_t n_rows,
                     double *out, void *stream);

int64_t hdfe_c_sums_workspace_bytes(void);

int hdfe_c_sums(const double *v, int32_t size, int32_t per_component, const double *b,
                const double *s, const double *base, const double *through_q, const double *y,
                int64_t n_rows, double *sums, void *workspace, int64_t workspace_bytes,
                void *stream);

int hdfe_c_sums_ext(const double *v, int32_t size, int32_t per_component, const double *b,
                    const double *s, const double *base, const double *through_q,
                    const double *y, int32_t n_vec, const double *u, const double *coef,
                    const double *g, int64_t n_rows, double *sums, void *workspace,
                    int64_t workspace_bytes, void *stream);

int hdfe_smooth_cells(const double *knots0, const double *knots1, const double *fp,
                      int32_t n_bins, const double *leverage, const double *b_ii,
                      const double *sigma2, int64_t n_rows, double *totals, double *counts,
                      void *stream);

int hdfe_smooth_eval(const double *knots0, const double *knots1, const double *fp,
                     int32_t n_bins, const double *means, const double *leverage,
                     const double *b_ii, int64_t n_rows, double *out, void *stream);

/* ------------------------------------------- many systems in one launch
 *
 * The Jacobi block PCG of core/solve.py:66-140 for many independent systems
 * at once: their reduced matrices on the diagonal of one CSR matrix (L rows,
 * each system's a contiguous range), B (L, k) and X (L, k) row-major, the
 * zero flags (n_systems, k) uint8 or NULL.  The caller splits the rows over
 * the grid's warps (hdfe_batch_pcg_grid gives blocks x warps_per_block):
 * warp_rows (W + 1) int64 each warp's first row (a warp's rows inside one
 * system), warp_system (W) int32, system_warps (n_systems + 1) int32 each
 * system's first warp.  Long rows are cut into n_chunks chunks of nonzeros
 * (chunk_row (n_chunks) int32, chunk_lo / chunk_hi (n_chunks) int64, in row
 * order; row_chunk (L) int32 a long row's first chunk, -1 for the others)
 * taken by warps of their system: warp_chunks (W + 1) int32 each warp's
 * first chunk, warp_chunks[W] = n_chunks.  Per system: its own alpha / beta / active flags and
 * relative residuals; iterations (n_systems) int64, max_rel (n_systems),
 * converged (n_systems) int32 out; status (int32, DEVICE) HDFE_OK or
 * HDFE_ERR_SPIN_LIMIT / HDFE_ERR_BAD_CODE.  lanes_per_row 4, 8, 16 or 32:
 * the SpMV's lanes per matrix row.  One cooperative launch; no host reads.
 * No reference counterpart: the reference fits one system at a time.
 */
int hdfe_batch_pcg_grid(int32_t k, int32_t lanes_per_row, int32_t *blocks,
                        int32_t *warps_per_block);

int64_t hdfe_batch_pcg_workspace_bytes(int64_t L, int32_t k, int64_t warps, int64_t n_chunks);

int hdfe_batch_pcg_solve(const int64_t *indptr, const int32_t *indices, const double *data,
                         int64_t L, const double *dinv, const double *B, int32_t k,
                         const uint8_t *zero, int64_t n_systems, const int64_t *warp_rows,
                         const int32_t *warp_system, const int32_t *system_warps,
                         const int32_t *warp_chunks, const int32_t *chunk_row,
                         const int64_t *chunk_lo, const int64_t *chunk_hi,
                         const int32_t *row_chunk, int64_t n_chunks, int32_t blocks,
                         int32_t lanes_per_row, double tol, int64_t maxiter, double *X,
                         int64_t *iterations, double *max_rel, int32_t *converged,
                         int32_t *status, void *workspace, int64_t workspace_bytes,
                         void *stream);

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

/* Largest k (right-hand-side columns per solve) hdfe_pcg_solve accepts.
 * Blocks of up to 4 columns keep each row's k values in one thread's
 * registers; wider blocks (the JLA's probe blocks) run one column per lane,
 * padded to 8, 16 or 32 columns, so every column of the block shares one
 * pass over S per iteration. */
#define HDFE_PCG_MAX_K 32

/* Largest k hdfe_pcg_solve_mixed accepts: blocks of up to 4 columns keep a
 * row's k values in one thread's registers, wider ones run one column per
 * lane (padded to 8, 16 or 32), as hdfe_pcg_solve does. */
#define HDFE_PCG_MIXED_MAX_K 32

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

/* ------------------------------------------- the dense small block
 *
 * A dimension with few levels (the years) meets nearly every level of the
 * others, so its rows and columns of S are nearly dense (on the 5M-worker
 * panel: 7.28M of the 7.50M firm-year entries exist, 64% of S's nonzeros).
 * When those levels are S's last `small_count` <= HDFE_SMALL_MAX_LEVELS
 * levels [small_first, L), the solve can take S split in three:
 *   the CSR of S[big, big] (rows >= small_first empty), columns < small_first;
 *   cross (small_first x HDFE_SMALL_MAX_LEVELS, row-major, zero-padded):
 *     cross[r * 16 + j] = S[r, small_first + j];
 *   small (small_count x small_count): S[small_first + i, small_first + j].
 * hdfe_small_split makes this form from S's CSR (columns sorted in each row):
 * indptr_out (L+1), indices_out / data_out (at most nnz entries), cross and
 * small as above, the big block's nonzero count to *nnz_out (a DEVICE
 * pointer), and status to *status_out (DEVICE): HDFE_OK, or
 * HDFE_ERR_BAD_CODE when a big row holds small-level entries but none of
 * the big block (the split would lose it from the row walk).
 * hdfe_pcg_solve_small is hdfe_pcg_solve (k <= HDFE_PCG_SMALL_MAX_K, the
 * same workspace size) on the split form: the big rows' products with the
 * small levels are coalesced rows of cross, the small rows' products the
 * column sums of cross reduced with p'Ap, no index round trips.  The
 * reference stores all of S in CSR (core/solve.py:148-194); the algorithm
 * (core/solve.py:66-140) is unchanged, only the order of the additions in
 * S P differs. */
#define HDFE_SMALL_MAX_LEVELS 16
#define HDFE_PCG_SMALL_MAX_K 4

int64_t hdfe_small_split_workspace_bytes(int64_t L);

int hdfe_small_split(const int64_t *indptr, const int32_t *indices, const double *data,
                     int64_t L, int64_t small_first, int32_t small_count, int64_t *indptr_out,
                     int32_t *indices_out, double *data_out, double *cross, double *small,
                     int64_t *nnz_out, int32_t *status_out, void *workspace,
                     int64_t workspace_bytes, void *stream);

int hdfe_pcg_solve_small(const int64_t *indptr, const int32_t *indices, const double *data,
                         int64_t L, int64_t nnz, int64_t small_first, int32_t small_count,
                         const double *cross, const double *small, const double *dinv,
                         const double *B, int32_t k, const uint8_t *zero, const double *X0,
                         double tol, int64_t maxiter, double *X, void *workspace,
                         int64_t workspace_bytes, hdfe_pcg_info *info, void *stream);

/* Mixed precision: the same solve with the inner CG in FP32 and iterative
 * refinement in FP64 -- the outer residual B - S X (S's FP64 values in
 * `data`), the update X += D and every dot product and norm are FP64; the
 * inner PCG on S D = R runs on S's values as FP32 (`data32`, nnz floats) and
 * FP32 vectors until ||R_inner|| <= inner_tol ||R||.  It stops, like
 * hdfe_pcg_solve, when every column's ||B - S X|| / ||B|| <= tol (checked in
 * FP64); info->iterations counts inner iterations, bounded by maxiter.  An
 * addition of this library (the reference's solve is FP64 only). */
int64_t hdfe_pcg_mixed_workspace_bytes(int64_t L, int64_t nnz, int32_t k);

int hdfe_pcg_solve_mixed(const int64_t *indptr, const int32_t *indices, const double *data,
                         const float *data32, int64_t L, int64_t nnz, const double *dinv,
                         const double *B, int32_t k, const uint8_t *zero, const double *X0,
                         double tol, double inner_tol, int64_t maxiter, double *X,
                         void *workspace, int64_t workspace_bytes, hdfe_pcg_info *info,
                         void *stream);

/* The same solve for callers that cannot allocate device memory -- a host
 * binding with no CUDA allocator of its own, or code that must not call
 * cudaMalloc because it synchronises the device.  No counterpart in the
 * reference: it is an addition of this library.  The scratch that
 * hdfe_pcg_solve takes as `workspace` lives instead in a device array inside
 * the library, HDFE_PCG_NOALLOC_BYTES (16 MiB) on every GPU that loads it,
 * held until the process exits.  Sizes whose scratch exceeds it
 * (hdfe_pcg_workspace_bytes(L, nnz, k) > HDFE_PCG_NOALLOC_BYTES; about
 * L * k <= 600,000 values) are rejected with HDFE_ERR_WORKSPACE.  The first
 * call on a device looks up the array's device address (cudaGetSymbolAddress)
 * with that device current, so make it before any stream capture.  That
 * address is cached for the library's lifetime: do not reset the device
 * (cudaDeviceReset) or re-create its primary context between calls.  Every
 * call shares the one array: calls that overlap on the GPU (other streams,
 * other host threads) race and corrupt each other; serialise them.  Nothing
 * in the array needs clearing between calls: each solve rewrites what it
 * reads.  No memory is allocated by this call. */
#define HDFE_PCG_NOALLOC_BYTES (16ll << 20)

int hdfe_pcg_solve_noalloc(const int64_t *indptr, const int32_t *indices, const double *data,
                           int64_t L, int64_t nnz, const double *dinv, const double *B,
                           int32_t k, const uint8_t *zero, const double *X0, double tol,
                           int64_t maxiter, double *X, hdfe_pcg_info *info, void *stream);

/* ------------------------------------------- pass 0: sort and factorize
 *
 * core/passes.py:285-294 codes each fixed effect by the rank of its level
 * among the sorted distinct levels; :359-373 orders the rows by (streamed
 * code, other codes, variables).  hdfe_sort_pairs: a stable LSD radix sort of
 * n keys (uint64, ordered by their value; key_bits = how many low bits can be
 * nonzero, 8 bits a pass) with int32 payloads (NULL: the positions 0 .. n-1),
 * into keys_out / vals_out; several keys sort as successive calls, least
 * significant key first.  hdfe_factorize: codes[i] = the rank of ids[i] among
 * the distinct ids (unsigned order), the distinct ids in order to levels (n
 * entries, or NULL), their number to *n_levels (a DEVICE pointer).  n < 2^31.
 * Both take a workspace of hdfe_sort_workspace_bytes(n) bytes (256-byte
 * aligned).  They replace Polars' factorize and sort. */
int64_t hdfe_sort_workspace_bytes(int64_t n);

int hdfe_sort_pairs(const uint64_t *keys, const int32_t *vals, int64_t n, int32_t key_bits,
                    uint64_t *keys_out, int32_t *vals_out, void *workspace,
                    int64_t workspace_bytes, void *stream);

int hdfe_factorize(const uint64_t *ids, int64_t n, int32_t key_bits, int32_t *codes,
                   uint64_t *levels, int64_t *n_levels, void *workspace, int64_t workspace_bytes,
                   void *stream);

/* ------------------------------------------- X' W X of a wide design
 *
 * core/inference.py:109-137 `_assemble` forms the design's cross-products
 * V' W V with a BLAS product in FP64.  For wide designs this computes X' W X on
 * the tensor cores: X (n_rows, c) row-major FP64, w (n_rows) or NULL, out
 * (c, c) FP64.  Every value is split as x = hi + lo, hi = bf16(x), lo =
 * bf16(x - hi) (rows scaled by sqrt(w)), and hi hi' + hi lo' + lo hi' is
 * accumulated in FP32 by tcgen05.mma per CTA over chunks of 64 rows, the CTAs'
 * partials summed in FP64: about 1e-5 relative accuracy per entry.  c <=
 * HDFE_GRAM_MAX_COLS.  The first 16 bytes of the workspace hold a status word
 * (HDFE_OK, or HDFE_ERR_SPIN_LIMIT if a wait on the tensor core timed out),
 * readable once the stream has run the call.  An addition of this library. */
#define HDFE_GRAM_MAX_COLS 128

int64_t hdfe_gram_workspace_bytes(int64_t n_rows, int32_t c);

int hdfe_gram_bf16x3(const double *X, int64_t n_rows, int32_t c, const double *w, double *out,
                     void *workspace, int64_t workspace_bytes, void *stream);

/* ------------------------------------------- the solver handle
 *
 * core/gpu.py:186-197 `explicit_solver(S, dinv, tol, maxiter)` returns a
 * `solve(b, zero, x0) -> (X, iterations, converged, max_rel)` closure that
 * keeps S and the preconditioner on the device; these three calls are that
 * closure for hosts binding the C ABI (cgo, JNI, N-API).  The handle keeps the
 * caller's device pointers to S (CSR, as for hdfe_pcg_solve) and dinv, which
 * must stay alive until hdfe_solver_destroy, and owns the one piece of device
 * memory this library allocates: the PCG workspace for up to max_k columns
 * (<= HDFE_PCG_MAX_K), the info record and the zero flags, allocated on the
 * current device by hdfe_solver_create.  hdfe_solver_solve: B (L, k), X0 (L,
 * k) or NULL and X (L, k) out are DEVICE pointers; zero (k) uint8 is a HOST
 * array or NULL; info is HOST memory, filled before the call returns (the
 * call synchronises its stream, as the reference's solve returns host
 * values).  It returns info->status (HDFE_OK unless the kernel stopped early;
 * non-convergence is info->converged = 0, not an error).  One solve at a time
 * per handle, on the device the handle was created on. */
typedef struct hdfe_solver hdfe_solver;

int hdfe_solver_create(const int64_t *indptr, const int32_t *indices, const double *data,
                       int64_t L, int64_t nnz, const double *dinv, double tol, int64_t maxiter,
                       int32_t max_k, hdfe_solver **out);

int hdfe_solver_solve(hdfe_solver *solver, const double *B, int32_t k, const uint8_t *zero,
                      const double *X0, double *X, hdfe_pcg_info *info, void *stream);

int hdfe_solver_destroy(hdfe_solver *solver);

#ifdef __cplusplus
}
#endif

#endif /* HDFE_B200_H */
