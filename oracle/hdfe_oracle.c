/*
 * hdfe_oracle.c -- CPU restatement of hdfe-stream's fixed-effects solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the CUDA library is
 * checked against, and the CPU baseline that bench.py times beside it.  Nothing
 * in the product (hdfe_stream_b200/) links, loads or calls it.
 *
 * Every function restates one numba kernel of the reference (hdfe-stream
 * v0.13.4) and cites it by file:line.  The loops keep the reference's order of
 * floating-point operations (same per-row / per-group / per-block sums, no
 * fused multiply-add: build with -ffp-contract=off), so on the same inputs the
 * results are bit-identical to the numba kernels'; tests/test_oracle.py pins
 * that against golden vectors produced by the reference itself.  Where the
 * reference runs `prange` over independent rows, groups or fixed blocks, the
 * restatement runs the same split under OpenMP: the results do not depend on
 * the thread count, exactly as in the reference.
 *
 * Layouts follow the reference's arrays:
 *   starts (G+1) int64         group boundaries (rows or cells sorted by fe[0])
 *   codes  (M, D) uint32       level codes of the non-streamed dimensions
 *   offs   (D) int64           start of each dimension's block in the stacked
 *                              level vector
 *   row-major (C-order) float64 matrices everywhere else.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <omp.h>

typedef int64_t i64;
typedef uint64_t u64;
typedef uint32_t u32;

int orc_num_threads(void) { return omp_get_max_threads(); }
void orc_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

/* ------------------------------------------------------------------ pass 1 */

/* _nb_run_sums, core/kernels_base.py:375-422 (without the within-cell
 * scatter, which only assembly="cells" reads).  cs (C+1) run starts, ZT (m, n)
 * centred variables one row per variable, w (n) or NULL, ST (m, C) out. */
void orc_run_sums(const i64 *cs, i64 C, const double *ZT, i64 m, i64 n,
                  const double *w, double *ST)
{
#pragma omp parallel for schedule(static)
    for (i64 c = 0; c < C; c++) {
        i64 s = cs[c], e = cs[c + 1];
        for (i64 j = 0; j < m; j++) {
            double acc = 0.0;
            const double *z = ZT + j * n;
            if (w) { for (i64 i = s; i < e; i++) acc += w[i] * z[i]; }
            else   { for (i64 i = s; i < e; i++) acc += z[i]; }
            ST[j * C + c] = acc;
        }
    }
}

/* _nb_rhs, core/kernels_base.py:65-83: b += D_o' M_0 V (serial). */
void orc_rhs(const i64 *starts, i64 G, const u32 *codes, i64 D, const double *n,
             const double *sums, i64 m, const i64 *offs, double *b)
{
    double *vbar = (double *)malloc(sizeof(double) * (m > 0 ? m : 1));
    for (i64 gi = 0; gi < G; gi++) {
        i64 s = starts[gi], e = starts[gi + 1];
        double Ng = 0.0;
        for (i64 j = 0; j < m; j++) vbar[j] = 0.0;
        for (i64 i = s; i < e; i++) {
            Ng += n[i];
            for (i64 j = 0; j < m; j++) vbar[j] += sums[i * m + j];
        }
        for (i64 j = 0; j < m; j++) vbar[j] /= Ng;
        for (i64 i = s; i < e; i++)
            for (i64 d = 0; d < D; d++) {
                i64 a = offs[d] + codes[i * D + d];
                for (i64 j = 0; j < m; j++)
                    b[a * m + j] += sums[i * m + j] - n[i] * vbar[j];
            }
    }
    free(vbar);
}

/* _nb_diag, core/kernels_base.py:87-110: exact diagonal of S (serial). */
void orc_diag(const i64 *starts, i64 G, const u32 *codes, i64 D, const double *n,
              const i64 *offs, double *diag)
{
    i64 cap = 0;
    for (i64 gi = 0; gi < G; gi++) {
        i64 sz = starts[gi + 1] - starts[gi];
        if (sz > cap) cap = sz;
    }
    cap *= D;
    i64 *lev = (i64 *)malloc(sizeof(i64) * (cap > 0 ? cap : 1));
    double *u = (double *)malloc(sizeof(double) * (cap > 0 ? cap : 1));
    for (i64 gi = 0; gi < G; gi++) {
        i64 s = starts[gi], e = starts[gi + 1];
        double Ng = 0.0;
        i64 q = 0;
        for (i64 i = s; i < e; i++) {
            Ng += n[i];
            for (i64 d = 0; d < D; d++) {
                i64 a = offs[d] + codes[i * D + d];
                diag[a] += n[i];
                i64 r = 0;
                while (r < q && lev[r] != a) r++;
                if (r == q) { lev[q] = a; u[q] = 0.0; q++; }
                u[r] += n[i];
            }
        }
        for (i64 r = 0; r < q; r++) diag[lev[r]] -= u[r] * u[r] / Ng;
    }
    free(lev);
    free(u);
}

/* ------------------------------------------------------------- union-find */

static i64 uf_find(i64 *parent, i64 x)
{   /* _uf_find, core/kernels_base.py:148-153 (path halving) */
    while (parent[x] != x) {
        parent[x] = parent[parent[x]];
        x = parent[x];
    }
    return x;
}

/* _nb_components, core/kernels_base.py:156-174: union-find over dimension
 * `col`; levels sharing an fe[0] group are connected.  parent (n_levels) out:
 * the root (smallest level) of each level's component. */
void orc_components(const i64 *starts, i64 G, const u32 *codes, i64 D, i64 col,
                    i64 n_levels, i64 *parent)
{
    for (i64 x = 0; x < n_levels; x++) parent[x] = x;
    for (i64 gi = 0; gi < G; gi++) {
        i64 s = starts[gi], e = starts[gi + 1];
        if (e <= s) continue;
        i64 r0 = uf_find(parent, codes[s * D + col]);
        for (i64 i = s + 1; i < e; i++) {
            i64 r = uf_find(parent, codes[i * D + col]);
            if (r != r0) {
                if (r < r0) { parent[r0] = r; r0 = r; }
                else parent[r] = r0;
            }
        }
    }
    for (i64 x = 0; x < n_levels; x++) parent[x] = uf_find(parent, x);
}

/* _nb_union_pairs, core/kernels_base.py:178-189 */
void orc_union_pairs(i64 *parent, const u32 *a, const u32 *b, i64 n, i64 off)
{
    for (i64 i = 0; i < n; i++) {
        i64 ra = uf_find(parent, a[i]);
        i64 rb = uf_find(parent, off + b[i]);
        if (ra != rb) {
            if (ra < rb) parent[rb] = ra; else parent[ra] = rb;
        }
    }
}

/* ------------------------------------------------------------ explicit S */

/* _nb_level_groups, core/kernels_base.py:201-229.  ptr (L+1) out; grp must
 * hold ptr[L] entries, so this is called twice: once with grp NULL to size it. */
void orc_level_groups(const i64 *starts, i64 G, const u32 *codes, i64 D,
                      const i64 *offs, i64 L, i64 *ptr, int32_t *grp)
{
    i64 *mark = (i64 *)malloc(sizeof(i64) * (L > 0 ? L : 1));
    for (i64 a = 0; a < L; a++) mark[a] = -1;
    if (!grp) {
        memset(ptr, 0, sizeof(i64) * (L + 1));
        for (i64 g = 0; g < G; g++)
            for (i64 i = starts[g]; i < starts[g + 1]; i++)
                for (i64 d = 0; d < D; d++) {
                    i64 a = offs[d] + codes[i * D + d];
                    if (mark[a] != g) { mark[a] = g; ptr[a + 1]++; }
                }
        for (i64 a = 0; a < L; a++) ptr[a + 1] += ptr[a];
    } else {
        i64 *fill = (i64 *)malloc(sizeof(i64) * (L > 0 ? L : 1));
        memcpy(fill, ptr, sizeof(i64) * L);
        for (i64 g = 0; g < G; g++)
            for (i64 i = starts[g]; i < starts[g + 1]; i++)
                for (i64 d = 0; d < D; d++) {
                    i64 a = offs[d] + codes[i * D + d];
                    if (mark[a] != g) { mark[a] = g; grp[fill[a]++] = (int32_t)g; }
                }
        free(fill);
    }
    free(mark);
}

/* _nb_row_work, core/kernels_base.py:232-240 */
void orc_row_work(const i64 *starts, const i64 *lptr, const int32_t *lgrp, i64 L, i64 *out)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (i64 r = 0; r < L; r++) {
        i64 w = 0;
        for (i64 k = lptr[r]; k < lptr[r + 1]; k++) {
            i64 g = lgrp[k];
            w += starts[g + 1] - starts[g];
        }
        out[r] = w;
    }
}

/* _nb_row_nnz, core/kernels_base.py:243-276: distinct columns of each row.
 * The reference splits rows into blocks of similar work; each row's count is
 * independent of the split, so rows are scheduled dynamically here. */
void orc_row_nnz(const i64 *starts, const u32 *codes, i64 D, const i64 *offs,
                 const i64 *lptr, const int32_t *lgrp, const i64 *work, i64 wide,
                 i64 L, i64 *out)
{
#pragma omp parallel
    {
        int32_t *mark = (int32_t *)malloc(sizeof(int32_t) * (L > 0 ? L : 1));
        uint8_t *flag = NULL;
        for (i64 c = 0; c < L; c++) mark[c] = -1;
#pragma omp for schedule(dynamic, 64)
        for (i64 r = 0; r < L; r++) {
            i64 cnt = 0;
            if (work[r] > wide) {
                if (!flag) flag = (uint8_t *)malloc(L > 0 ? L : 1);
                memset(flag, 0, L);
                for (i64 j = lptr[r]; j < lptr[r + 1]; j++) {
                    i64 g = lgrp[j];
                    for (i64 i = starts[g]; i < starts[g + 1]; i++)
                        for (i64 d = 0; d < D; d++) flag[offs[d] + codes[i * D + d]] = 1;
                }
                for (i64 c = 0; c < L; c++) cnt += flag[c];
            } else {
                for (i64 j = lptr[r]; j < lptr[r + 1]; j++) {
                    i64 g = lgrp[j];
                    for (i64 i = starts[g]; i < starts[g + 1]; i++)
                        for (i64 d = 0; d < D; d++) {
                            i64 c = offs[d] + codes[i * D + d];
                            if (mark[c] != (int32_t)r) { mark[c] = (int32_t)r; cnt++; }
                        }
                }
            }
            out[r] = cnt;
        }
        free(mark);
        free(flag);
    }
}

static int cmp_pair(const void *x, const void *y)
{
    const i64 *a = (const i64 *)x, *b = (const i64 *)y;
    return (a[0] > b[0]) - (a[0] < b[0]);
}

/* _nb_row_fill, core/kernels_base.py:280-358, for the plain case (no varying
 * slopes: st = n, correction u_r / N_g).  indptr (L+1), indices (nnz) and
 * data (nnz) out; indices are int32 (nnz, L < 2^31). */
void orc_row_fill(const i64 *starts, const u32 *codes, i64 D, const double *n,
                  const double *Ng, const i64 *offs, i64 Dn, const i64 *lptr,
                  const int32_t *lgrp, const i64 *work, i64 wide, i64 L,
                  const i64 *indptr, int32_t *indices, double *data)
{
    (void)Dn;
#pragma omp parallel
    {
        int32_t *mark = (int32_t *)malloc(sizeof(int32_t) * (L > 0 ? L : 1));
        int32_t *pos = (int32_t *)malloc(sizeof(int32_t) * (L > 0 ? L : 1));
        double *acc = NULL;
        uint8_t *flag = NULL;
        i64 *tmp = NULL;
        i64 tmpcap = 0;
        for (i64 c = 0; c < L; c++) mark[c] = -1;
#pragma omp for schedule(dynamic, 64)
        for (i64 r = 0; r < L; r++) {
            i64 dr = 0;
            while (dr + 1 < D && offs[dr + 1] <= r) dr++;
            i64 lr = r - offs[dr];
            i64 p0 = indptr[r];
            int dense = work[r] > wide;
            if (dense && !acc) {
                acc = (double *)calloc(L > 0 ? L : 1, sizeof(double));
                flag = (uint8_t *)calloc(L > 0 ? L : 1, 1);
            }
            i64 q = 0;
            for (i64 j = lptr[r]; j < lptr[r + 1]; j++) {
                i64 g = lgrp[j];
                i64 s = starts[g], e = starts[g + 1];
                double ur = 0.0;
                for (i64 i = s; i < e; i++)
                    if (codes[i * D + dr] == (u32)lr) ur += n[i];
                double wv = ur / Ng[g];
                for (i64 i = s; i < e; i++) {
                    double v = 0.0;
                    v -= n[i] * wv;
                    if (codes[i * D + dr] == (u32)lr) v += n[i];
                    for (i64 d = 0; d < D; d++) {
                        i64 col = offs[d] + codes[i * D + d];
                        if (dense) { acc[col] += v; flag[col] = 1; }
                        else if (mark[col] != (int32_t)r) {
                            mark[col] = (int32_t)r;
                            pos[col] = (int32_t)q;
                            indices[p0 + q] = (int32_t)col;
                            data[p0 + q] = v;
                            q++;
                        } else data[p0 + pos[col]] += v;
                    }
                }
            }
            if (dense) {
                for (i64 c = 0; c < L; c++)
                    if (flag[c]) {
                        indices[p0 + q] = (int32_t)c;
                        data[p0 + q] = acc[c];
                        q++;
                        acc[c] = 0.0;
                        flag[c] = 0;
                    }
            } else if (q > 1) {
                if (q > tmpcap) {
                    free(tmp);
                    tmpcap = 2 * q;
                    tmp = (i64 *)malloc(sizeof(i64) * 2 * tmpcap);
                }
                /* column indices are distinct within a row, so any sort gives
                 * the reference's argsort order */
                for (i64 k = 0; k < q; k++) {
                    tmp[2 * k] = indices[p0 + k];
                    memcpy(&tmp[2 * k + 1], &data[p0 + k], sizeof(double));
                }
                qsort(tmp, q, 2 * sizeof(i64), cmp_pair);
                for (i64 k = 0; k < q; k++) {
                    indices[p0 + k] = (int32_t)tmp[2 * k];
                    memcpy(&data[p0 + k], &tmp[2 * k + 1], sizeof(double));
                }
            }
        }
        free(mark); free(pos); free(acc); free(flag); free(tmp);
    }
}

/* -------------------------------------------------------------------- PCG */

/* _nb_csr_matmat, core/kernels_base.py:362-371: out = S @ X, X (L, k) */
void orc_csr_matmat(const i64 *indptr, const int32_t *indices, const double *data,
                    i64 L, const double *X, i64 k, double *out)
{
#pragma omp parallel for schedule(dynamic, 512)
    for (i64 i = 0; i < L; i++) {
        for (i64 j = 0; j < k; j++) out[i * k + j] = 0.0;
        for (i64 p = indptr[i]; p < indptr[i + 1]; p++) {
            i64 c = indices[p];
            double v = data[p];
            for (i64 j = 0; j < k; j++) out[i * k + j] += v * X[c * k + j];
        }
    }
}

/* _nb_cg_dot, core/kernels_base.py:432-441 (parts (nblk, k)) */
void orc_cg_dot(const double *A, const double *B, i64 L, i64 k, i64 nblk, double *parts)
{
#pragma omp parallel for schedule(static)
    for (i64 b = 0; b < nblk; b++) {
        for (i64 j = 0; j < k; j++) parts[b * k + j] = 0.0;
        for (i64 i = b * L / nblk; i < (b + 1) * L / nblk; i++)
            for (i64 j = 0; j < k; j++) parts[b * k + j] += A[i * k + j] * B[i * k + j];
    }
}

/* _nb_cg_step, core/kernels_base.py:445-462 (parts (nblk, 2, k)); dinv NULL
 * for no Jacobi. */
void orc_cg_step(double *X, double *R, const double *P, const double *AP,
                 const double *alpha, const double *dinv, i64 L, i64 k, i64 nblk,
                 double *parts)
{
#pragma omp parallel for schedule(static)
    for (i64 b = 0; b < nblk; b++) {
        double *p0 = parts + b * 2 * k, *p1 = p0 + k;
        for (i64 j = 0; j < k; j++) { p0[j] = 0.0; p1[j] = 0.0; }
        for (i64 i = b * L / nblk; i < (b + 1) * L / nblk; i++)
            for (i64 j = 0; j < k; j++) {
                X[i * k + j] += alpha[j] * P[i * k + j];
                double r = R[i * k + j] - alpha[j] * AP[i * k + j];
                R[i * k + j] = r;
                p0[j] += r * r;
                if (dinv) p1[j] += r * r * dinv[i];
            }
    }
}

/* _nb_cg_direction, core/kernels_base.py:466-474 */
void orc_cg_direction(double *P, const double *Z, const double *dinv, const double *beta,
                      i64 L, i64 k)
{
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < L; i++)
        for (i64 j = 0; j < k; j++) {
            double z = dinv ? Z[i * k + j] * dinv[i] : Z[i * k + j];
            P[i * k + j] = z + beta[j] * P[i * k + j];
        }
}

/* ------------------------------------------------------- random draws */

/* _nb_rademacher, core/kernels_groups.py:53-76: splitmix64 on
 * (seed, row ordinal, draw), sign bit -> +/-1. out (n_rows, draws). */
void orc_rademacher(i64 ordinal, i64 n_rows, i64 draws, u64 seed, i64 first_draw,
                    double *out)
{
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < n_rows; i++) {
        u64 row = (u64)(ordinal + i);
        for (i64 j = 0; j < draws; j++) {
            u64 d = (u64)(first_draw + j);
            u64 x = seed ^ (row * 0x9E3779B97F4A7C15ULL) ^ (d * 0xBF58476D1CE4E5B9ULL);
            x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
            x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
            x = x ^ (x >> 31);
            out[i * draws + j] = (x >> 63) == 0 ? 1.0 : -1.0;
        }
    }
}

/* ------------------------------------------------------ inverse operator */

/* _nb_center_rows, kernels_inverse.py:35-71.  acc (nt, L, m), acc_x (nt, k, m):
 * thread block t takes groups [G*t/nt, G*(t+1)/nt). */
void orc_center_rows(const i64 *starts, i64 G, const i64 *codes, i64 D, const i64 *offs,
                     const double *w, const double *X, i64 k, const double *R, i64 m,
                     i64 nt, i64 L, double *acc, double *acc_x)
{
#pragma omp parallel for schedule(static)
    for (i64 t = 0; t < nt; t++) {
        double *a = acc + t * L * m, *ax = acc_x + t * k * m;
        for (i64 gi = G * t / nt; gi < G * (t + 1) / nt; gi++) {
            i64 s = starts[gi], e = starts[gi + 1];
            double sw = 0.0;
            for (i64 i = s; i < e; i++) sw += w[i];
            if (sw <= 0.0) continue;
            for (i64 j = 0; j < m; j++) {
                double total = 0.0;
                for (i64 i = s; i < e; i++) total += w[i] * R[i * m + j];
                double mean = total / sw;
                for (i64 i = s; i < e; i++) {
                    double v = w[i] * (R[i * m + j] - mean);
                    for (i64 d = 0; d < D; d++) a[(offs[d] + codes[i * D + d]) * m + j] += v;
                    for (i64 c = 0; c < k; c++) ax[c * m + j] += X[i * k + c] * v;
                }
            }
        }
    }
}

/* _nb_project_rows, kernels_inverse.py:75-107 */
void orc_project_rows(const i64 *starts, i64 G, const i64 *codes, i64 D, const i64 *offs,
                      const double *w, const double *X, i64 k, const double *C,
                      const double *R, i64 m, const double *U, double *out)
{
#pragma omp parallel for schedule(dynamic, 1024)
    for (i64 gi = 0; gi < G; gi++) {
        i64 s = starts[gi], e = starts[gi + 1];
        double sw = 0.0;
        for (i64 i = s; i < e; i++) sw += w[i];
        for (i64 j = 0; j < m; j++) {
            double total = 0.0;
            for (i64 i = s; i < e; i++) {
                double h = 0.0;
                for (i64 d = 0; d < D; d++) h += U[(offs[d] + codes[i * D + d]) * m + j];
                for (i64 c = 0; c < k; c++) h += X[i * k + c] * C[c * m + j];
                out[i * m + j] = h;
                total += w[i] * (R[i * m + j] - h);
            }
            double mean = sw > 0.0 ? total / sw : 0.0;
            for (i64 i = s; i < e; i++) out[i * m + j] += mean;
        }
    }
}

/* _nb_reduce_rows, kernels_inverse.py:112-130 */
void orc_reduce_rows(const i64 *starts, i64 G, const i64 *codes, i64 D, const i64 *offs,
                     const double *w, const double *X, i64 k, const double *R, i64 m,
                     i64 nt, i64 L, double *acc, double *acc_x)
{
#pragma omp parallel for schedule(static)
    for (i64 t = 0; t < nt; t++) {
        double *a = acc + t * L * m, *ax = acc_x + t * k * m;
        for (i64 gi = G * t / nt; gi < G * (t + 1) / nt; gi++)
            for (i64 i = starts[gi]; i < starts[gi + 1]; i++)
                for (i64 j = 0; j < m; j++) {
                    double v = w[i] * R[i * m + j];
                    for (i64 d = 0; d < D; d++) a[(offs[d] + codes[i * D + d]) * m + j] += v;
                    for (i64 c = 0; c < k; c++) ax[c * m + j] += X[i * k + c] * v;
                }
    }
}

/* _nb_spread_groups, kernels_inverse.py:134-152 */
void orc_spread_groups(const i64 *starts, i64 G, const double *w, const double *gv, i64 m,
                       double *out)
{
#pragma omp parallel for schedule(dynamic, 1024)
    for (i64 gi = 0; gi < G; gi++) {
        i64 s = starts[gi], e = starts[gi + 1];
        double sw = 0.0;
        for (i64 i = s; i < e; i++) sw += w[i];
        double inv = sw > 0.0 ? 1.0 / sw : 0.0;
        for (i64 j = 0; j < m; j++) {
            double value = gv[gi * m + j] * inv;
            for (i64 i = s; i < e; i++) out[i * m + j] = value;
        }
    }
}

/* _nb_project_coef, kernels_inverse.py:157-188 */
void orc_project_coef(const i64 *starts, i64 G, const i64 *codes, i64 D, const i64 *offs,
                      const double *w, const double *X, i64 k, const double *C,
                      const double *RHO, i64 m, const double *U, double *out_rows,
                      double *out_groups)
{
#pragma omp parallel for schedule(dynamic, 1024)
    for (i64 gi = 0; gi < G; gi++) {
        i64 s = starts[gi], e = starts[gi + 1];
        double sw = 0.0;
        for (i64 i = s; i < e; i++) sw += w[i];
        for (i64 j = 0; j < m; j++) {
            double total = 0.0;
            for (i64 i = s; i < e; i++) {
                double h = 0.0;
                for (i64 d = 0; d < D; d++) h += U[(offs[d] + codes[i * D + d]) * m + j];
                for (i64 c = 0; c < k; c++) h += X[i * k + c] * C[c * m + j];
                out_rows[i * m + j] = h;
                total += w[i] * (RHO[i * m + j] - h);
            }
            double mean = sw > 0.0 ? total / sw : 0.0;
            out_groups[gi * m + j] = mean;
            for (i64 i = s; i < e; i++) out_rows[i * m + j] += mean;
        }
    }
}

/* _nb_group_sums, core/kernels_groups.py:17-27 */
void orc_group_sums(const i64 *starts, i64 G, const double *w, const double *R, i64 m,
                    double *out)
{
#pragma omp parallel for schedule(dynamic, 1024)
    for (i64 gi = 0; gi < G; gi++) {
        i64 s = starts[gi], e = starts[gi + 1];
        for (i64 j = 0; j < m; j++) {
            double total = 0.0;
            for (i64 i = s; i < e; i++) total += w[i] * R[i * m + j];
            out[gi * m + j] = total;
        }
    }
}

/* _nb_trace_moments, kernels_inverse.py:192-231.  acc (nt, m, 8) */
void orc_trace_moments(const i64 *starts, i64 G, const i64 *codes, i64 D, i64 psi_column,
                       i64 psi_offset, const double *w, const double *Zl, const double *Zg,
                       const double *Ul, const double *Ug, i64 m, i64 nt, double *acc)
{
#pragma omp parallel for schedule(static)
    for (i64 t = 0; t < nt; t++) {
        for (i64 gi = G * t / nt; gi < G * (t + 1) / nt; gi++) {
            i64 s = starts[gi], e = starts[gi + 1];
            for (i64 j = 0; j < m; j++) {
                double b1 = Zg[gi * m + j], b2 = Ug[gi * m + j];
                double *a = acc + (t * m + j) * 8;
                for (i64 i = s; i < e; i++) {
                    i64 level = psi_offset + codes[i * D + psi_column];
                    double a1 = Zl[level * m + j], a2 = Ul[level * m + j];
                    double wt = w[i];
                    a[0] += wt;
                    a[1] += wt * a1 * a2;
                    a[2] += wt * b1 * b2;
                    a[3] += wt * (a1 * b2 + b1 * a2);
                    a[4] += wt * a1;
                    a[5] += wt * a2;
                    a[6] += wt * b1;
                    a[7] += wt * b2;
                }
            }
        }
    }
}

/* --------------------------------------------------- bipartite network */

/* _nb_peel, core/kernels_graph.py:188-221: (k0, k1)-core of the distinct
 * pairs keys = a * n1 + b.  Returns the rounds that removed something. */
i64 orc_peel(const u64 *keys, i64 E, u64 n1, i64 k0, i64 k1, uint8_t *alive0, i64 n0,
             uint8_t *alive1, i64 nl1)
{
    i64 *deg0 = (i64 *)malloc(sizeof(i64) * (n0 > 0 ? n0 : 1));
    i64 *deg1 = (i64 *)malloc(sizeof(i64) * (nl1 > 0 ? nl1 : 1));
    i64 rounds = 0;
    for (;;) {
        memset(deg0, 0, sizeof(i64) * n0);
        memset(deg1, 0, sizeof(i64) * nl1);
        for (i64 e = 0; e < E; e++) {
            i64 a = (i64)(keys[e] / n1), b = (i64)(keys[e] % n1);
            if (alive0[a] && alive1[b]) { deg0[a]++; deg1[b]++; }
        }
        int changed = 0;
        for (i64 v = 0; v < n0; v++)
            if (alive0[v] && deg0[v] < k0) { alive0[v] = 0; changed = 1; }
        for (i64 v = 0; v < nl1; v++)
            if (alive1[v] && deg1[v] < k1) { alive1[v] = 0; changed = 1; }
        if (!changed) break;
        rounds++;
    }
    free(deg0);
    free(deg1);
    return rounds;
}

/* _nb_union_keys, core/kernels_graph.py:225-240 */
void orc_union_keys(i64 *parent, const u64 *keys, i64 E, u64 n1, const uint8_t *alive0,
                    i64 n0, const uint8_t *alive1)
{
    for (i64 e = 0; e < E; e++) {
        i64 a = (i64)(keys[e] / n1), b = (i64)(keys[e] % n1);
        if (!(alive0[a] && alive1[b])) continue;
        i64 ra = uf_find(parent, a), rb = uf_find(parent, n0 + b);
        if (ra != rb) { if (ra < rb) parent[rb] = ra; else parent[ra] = rb; }
    }
}

/* _nb_dense_labels, core/kernels_graph.py:244-262 */
i64 orc_dense_labels(i64 *parent, i64 n, const uint8_t *alive)
{
    for (i64 x = 0; x < n; x++) parent[x] = uf_find(parent, x);
    i64 nc = 0;
    for (i64 x = 0; x < n; x++) {
        if (!alive[x]) parent[x] = -1;
        else if (parent[x] == x) parent[x] = nc++;
        else parent[x] = parent[parent[x]];
    }
    return nc;
}

/* _nb_pair_rows, core/kernels_graph.py:274-284 */
void orc_pair_rows(const u64 *keys, const u32 *counts, i64 E, u64 n1, const i64 *labels,
                   i64 nlab, i64 *out)
{
    i64 off = nlab - (i64)n1;
    for (i64 e = 0; e < E; e++) {
        i64 a = (i64)(keys[e] / n1), b = (i64)(keys[e] % n1);
        if (labels[a] >= 0 && labels[off + b] >= 0) out[labels[a]] += counts[e];
    }
}

/* _nb_pairs_degree + _nb_pairs_fill, core/kernels_graph.py:314-343: CSR
 * adjacency of the alive distinct pairs, both directions.  indices NULL on the
 * first call (sizes indptr). */
void orc_pairs_csr(const u64 *keys, i64 E, u64 n1, i64 n0, const uint8_t *alive, i64 nv,
                   i64 *indptr, i64 *indices)
{
    if (!indices) {
        memset(indptr, 0, sizeof(i64) * (nv + 1));
        for (i64 e = 0; e < E; e++) {
            i64 a = (i64)(keys[e] / n1), b = n0 + (i64)(keys[e] % n1);
            if (alive[a] && alive[b]) { indptr[a + 1]++; indptr[b + 1]++; }
        }
        for (i64 v = 0; v < nv; v++) indptr[v + 1] += indptr[v];
        return;
    }
    i64 *pos = (i64 *)malloc(sizeof(i64) * (nv > 0 ? nv : 1));
    memcpy(pos, indptr, sizeof(i64) * nv);
    for (i64 e = 0; e < E; e++) {
        i64 a = (i64)(keys[e] / n1), b = n0 + (i64)(keys[e] % n1);
        if (alive[a] && alive[b]) { indices[pos[a]++] = b; indices[pos[b]++] = a; }
    }
    free(pos);
}

/* _nb_articulation_points, core/kernels_graph.py:23-86 (iterative Tarjan) */
void orc_articulation_points(const i64 *indptr, const i64 *indices, i64 n, uint8_t *is_cut,
                             const uint8_t *alive)
{
    i64 *disc = (i64 *)malloc(sizeof(i64) * (n > 0 ? n : 1));
    i64 *low = (i64 *)calloc(n > 0 ? n : 1, sizeof(i64));
    i64 *parent = (i64 *)malloc(sizeof(i64) * (n > 0 ? n : 1));
    i64 *stack_v = (i64 *)malloc(sizeof(i64) * (n > 0 ? n : 1));
    i64 *stack_ptr = (i64 *)malloc(sizeof(i64) * (n > 0 ? n : 1));
    for (i64 v = 0; v < n; v++) { disc[v] = -1; parent[v] = -1; }
    i64 timer = 0;
    for (i64 start = 0; start < n; start++) {
        if (disc[start] != -1 || !alive[start]) continue;
        disc[start] = low[start] = timer++;
        stack_v[0] = start;
        stack_ptr[0] = indptr[start];
        i64 top = 0, root_children = 0;
        while (top >= 0) {
            i64 u = stack_v[top];
            if (stack_ptr[top] < indptr[u + 1]) {
                i64 v = indices[stack_ptr[top]];
                stack_ptr[top]++;
                if (v == parent[u] || !alive[v]) continue;
                if (disc[v] == -1) {
                    parent[v] = u;
                    disc[v] = low[v] = timer++;
                    top++;
                    stack_v[top] = v;
                    stack_ptr[top] = indptr[v];
                    if (u == start) root_children++;
                } else if (disc[v] < low[u]) low[u] = disc[v];
            } else {
                top--;
                if (top >= 0) {
                    i64 p = stack_v[top];
                    if (low[u] < low[p]) low[p] = low[u];
                    if (p != start && low[u] >= disc[p]) is_cut[p] = 1;
                }
            }
        }
        if (root_children > 1) is_cut[start] = 1;
    }
    free(disc); free(low); free(parent); free(stack_v); free(stack_ptr);
}

/* _nb_bfs_components, core/kernels_graph.py:90-116 */
i64 orc_bfs_components(const i64 *indptr, const i64 *indices, i64 n, const uint8_t *alive,
                       i64 *label)
{
    i64 *queue = (i64 *)malloc(sizeof(i64) * (n > 0 ? n : 1));
    for (i64 v = 0; v < n; v++) label[v] = -1;
    i64 component = 0;
    for (i64 start = 0; start < n; start++) {
        if (!alive[start] || label[start] != -1) continue;
        label[start] = component;
        queue[0] = start;
        i64 head = 0, tail = 1;
        while (head < tail) {
            i64 u = queue[head++];
            for (i64 k = indptr[u]; k < indptr[u + 1]; k++) {
                i64 v = indices[k];
                if (alive[v] && label[v] == -1) { label[v] = component; queue[tail++] = v; }
            }
        }
        component++;
    }
    free(queue);
    return component;
}

/* _nb_level_rows, core/kernels_graph.py:346-352 */
void orc_level_rows(const u64 *keys, const u32 *counts, i64 E, u64 n1, const uint8_t *alive,
                    i64 n0, i64 *out)
{
    for (i64 e = 0; e < E; e++) {
        i64 a = (i64)(keys[e] / n1);
        if (alive[a] && alive[n0 + (i64)(keys[e] % n1)]) out[a] += counts[e];
    }
}
