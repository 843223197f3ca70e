/*
 * oracle.c -- CPU restatement of HiFlow3's lmp hot path (TEST INFRASTRUCTURE).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library.  Each function cites the reference routine it restates, with
 * paths relative to the HiFlow3 2.0 source tree (src/linear_algebra/lmp unless
 * another directory is named).  Compiled with plain -O2 (no -ffast-math, no
 * FMA contraction) so that floating-point operation order is the one written.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ================================================================== */
/* Structured Q1 systems                                               */
/* ================================================================== */

int orc_q1_sizes(int dim, int N, int *n_out, int64_t *nnz_out)
{
    if (dim < 2 || dim > 3 || N < 1) return -1;
    int64_t n = 1, nnz = 1;
    for (int d = 0; d < dim; ++d) { n *= (N + 1); nnz *= (3 * (int64_t)N + 1); }
    if (n > 0x7fffffff || nnz > 0x7fffffff) return -2;
    *n_out = (int)n;
    *nnz_out = nnz;
    return 0;
}

int orc_q1_structure(int dim, int N, int *coo_row, int *coo_col)
{
    const int P = N + 1;
    const int PZ = (dim == 3) ? P : 1;
    int64_t e = 0;
    for (int k = 0; k < PZ; ++k)
        for (int j = 0; j < P; ++j)
            for (int i = 0; i < P; ++i) {
                const int r = i + P * (j + P * k);
                for (int dk = (dim == 3 ? -1 : 0); dk <= (dim == 3 ? 1 : 0); ++dk) {
                    const int kk = k + dk;
                    if (kk < 0 || kk >= PZ) continue;
                    for (int dj = -1; dj <= 1; ++dj) {
                        const int jj = j + dj;
                        if (jj < 0 || jj >= P) continue;
                        for (int di = -1; di <= 1; ++di) {
                            const int ii = i + di;
                            if (ii < 0 || ii >= P) continue;
                            coo_row[e] = r;
                            coo_col[e] = ii + P * (jj + P * kk);
                            ++e;
                        }
                    }
                }
            }
    return (int)e;
}

/* Q1 shape data at the 2^dim Gauss points of the unit cell, local vertex
 * a = ax + 2 ay + 4 az, quadrature points ordered x fastest. */
static void q1_shape(int dim, double h, double *phi /*[8][8]*/, double *grad /*[8][8][3]*/, double *wq)
{
    const double g = 1.0 / sqrt(3.0);
    const double qp[2] = { (1.0 - g) / 2.0, (1.0 + g) / 2.0 };
    const int nq = 1 << dim, nv = 1 << dim;
    for (int q = 0; q < nq; ++q) {
        double xi[3] = { qp[q & 1], qp[(q >> 1) & 1], qp[(q >> 2) & 1] };
        double w = 1.0;
        for (int d = 0; d < dim; ++d) w *= 0.5;
        wq[q] = w;
        for (int a = 0; a < nv; ++a) {
            double f[3];
            for (int d = 0; d < dim; ++d) f[d] = ((a >> d) & 1) ? xi[d] : 1.0 - xi[d];
            double p = 1.0;
            for (int d = 0; d < dim; ++d) p *= f[d];
            phi[q * 8 + a] = p;
            for (int d = 0; d < dim; ++d) {
                double gd = ((a >> d) & 1) ? 1.0 : -1.0;
                for (int e = 0; e < dim; ++e)
                    if (e != d) gd *= f[e];
                grad[(q * 8 + a) * 3 + d] = gd / h;
            }
        }
    }
}

/* dot(grad_j, grad_i) per quadrature point (the part of the integrand that
 * does not depend on the coefficient). */
static void q1_graddots(int dim, const double *grad, double *D /*[8][8][8]*/)
{
    const int nq = 1 << dim, nv = 1 << dim;
    for (int q = 0; q < nq; ++q)
        for (int i = 0; i < nv; ++i)
            for (int j = 0; j < nv; ++j) {
                double s = 0.0;
                for (int d = 0; d < dim; ++d)
                    s += grad[(q * 8 + j) * 3 + d] * grad[(q * 8 + i) * 3 + d];
                D[(q * 8 + i) * 8 + j] = s;
            }
}

static void q1_element_from(int dim, double h, int kind, double coef, const double *beta,
                            const double *phi, const double *grad, const double *wq,
                            const double *D, double *Ke)
{
    const int nq = 1 << dim, nv = 1 << dim;
    double dJ = 1.0;
    for (int d = 0; d < dim; ++d) dJ *= h;
    for (int i = 0; i < nv * nv; ++i) Ke[i] = 0.0;
    for (int q = 0; q < nq; ++q) {
        /* a1(u,v) = int coef grad(u).grad(v)   (convdiff.cc:97-105, poisson_tutorial.h:163-170) */
        for (int i = 0; i < nv; ++i)
            for (int j = 0; j < nv; ++j)
                Ke[i * nv + j] += wq[q] * (coef * D[(q * 8 + i) * 8 + j]) * dJ;
        if (kind == 1) {
            /* a2(u,v) = int (beta.grad(u)) v   (convdiff.cc:107-115) */
            for (int i = 0; i < nv; ++i)
                for (int j = 0; j < nv; ++j) {
                    double bg = 0.0;
                    for (int d = 0; d < dim; ++d) bg += beta[d] * grad[(q * 8 + j) * 3 + d];
                    Ke[i * nv + j] += wq[q] * (bg * phi[q * 8 + i]) * dJ;
                }
        }
    }
}

void orc_q1_element(int dim, double h, int kind, double coef, const double *beta, double *Ke)
{
    double phi[64], grad[192], wq[8], D[512];
    q1_shape(dim, h, phi, grad, wq);
    q1_graddots(dim, grad, D);
    q1_element_from(dim, h, kind, coef, beta, phi, grad, wq, D, Ke);
}

int orc_q1_dirichlet(int dim, int N, int *idx)
{
    const int P = N + 1, PZ = (dim == 3) ? P : 1;
    int c = 0;
    for (int k = 0; k < PZ; ++k)
        for (int j = 0; j < P; ++j)
            for (int i = 0; i < P; ++i) {
                int bnd = (i == 0 || i == N || j == 0 || j == N);
                if (dim == 3) bnd = bnd || k == 0 || k == N;
                if (bnd) idx[c++] = i + P * (j + P * k);
            }
    return c;
}

int orc_q1_assemble(int dim, int N, int kind, const double *kcell, double nu,
                    const double *beta, int *row, int *col, double *val)
{
    int n;
    int64_t nnz;
    if (orc_q1_sizes(dim, N, &n, &nnz)) return -1;
    int *cr = (int *)malloc(sizeof(int) * nnz), *cc = (int *)malloc(sizeof(int) * nnz);
    if (!cr || !cc) { free(cr); free(cc); return -2; }
    orc_q1_structure(dim, N, cr, cc);
    /* init_structure (lmatrix_csr_cpu.cc:1101-1121) then Zeros */
    orc_coo_to_csr(n, (int)nnz, cr, cc, NULL, row, col, NULL);
    free(cr);
    free(cc);
    memset(val, 0, sizeof(double) * nnz);

    const double h = 1.0 / N;
    const int nv = 1 << dim, P = N + 1, CZ = (dim == 3) ? N : 1;
    double phi[64], grad[192], wq[8], D[512], Ke[64];
    q1_shape(dim, h, phi, grad, wq);
    q1_graddots(dim, grad, D);
    const double c0 = (kind == 0) ? 1.0 : nu;
    if (!kcell) q1_element_from(dim, h, kind, c0, beta, phi, grad, wq, D, Ke);
    int dofs[8];
    for (int cz = 0; cz < CZ; ++cz)
        for (int cy = 0; cy < N; ++cy)
            for (int cx = 0; cx < N; ++cx) {
                const int64_t cell = cx + (int64_t)N * (cy + (int64_t)N * cz);
                for (int a = 0; a < nv; ++a)
                    dofs[a] = (cx + (a & 1)) + P * ((cy + ((a >> 1) & 1)) + P * (cz + ((a >> 2) & 1)));
                if (kcell) q1_element_from(dim, h, kind, kcell[cell], beta, phi, grad, wq, D, Ke);
                orc_add_values(row, col, val, dofs, nv, dofs, nv, Ke);
            }
    int *bnd = (int *)malloc(sizeof(int) * n);
    if (!bnd) return -2;
    int nb = orc_q1_dirichlet(dim, N, bnd);
    orc_zero_rows(row, col, val, bnd, nb, 1.0);
    free(bnd);
    return 0;
}

uint64_t orc_splitmix64(uint64_t *state)
{
    uint64_t z = (*state += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

double orc_uniform_pm1(uint64_t *state)
{
    const uint64_t z = orc_splitmix64(state);
    return 2.0 * ((double)(z >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
}

void orc_q1_rhs(uint64_t seed, int dim, int N, double *b)
{
    const int P = N + 1, PZ = (dim == 3) ? P : 1;
    uint64_t s = seed;
    for (int k = 0; k < PZ; ++k)
        for (int j = 0; j < P; ++j)
            for (int i = 0; i < P; ++i) {
                const int64_t r = i + (int64_t)P * (j + (int64_t)P * k);
                const double u = orc_uniform_pm1(&s); /* one draw per DoF, in DoF order */
                int bnd = (i == 0 || i == N || j == 0 || j == N);
                if (dim == 3) bnd = bnd || k == 0 || k == N;
                b[r] = bnd ? 0.0 : u;
            }
}

/* ================================================================== */
/* CSR construction                                                    */
/* ================================================================== */

void orc_coo_to_csr(int n_rows, int nnz, const int *coo_row, const int *coo_col,
                    const double *coo_val, int *row, int *col, double *val)
{
    /* lmatrix_csr_cpu.cc:961-1004: count entries per row, exclusive scan, scatter */
    memset(row, 0, sizeof(int) * (n_rows + 1));
    for (int i = 0; i < nnz; ++i) ++row[coo_row[i]];
    row[n_rows] = nnz;
    int *next = (int *)malloc(sizeof(int) * (n_rows > 0 ? n_rows : 1));
    int acc = 0;
    for (int i = 0; i < n_rows; ++i) {
        const int c = row[i];
        row[i] = acc;
        next[i] = acc;
        acc += c;
    }
    for (int i = 0; i < nnz; ++i) {
        const int t = next[coo_row[i]]++;
        col[t] = coo_col[i];
        if (coo_val) val[t] = coo_val[i];
    }
    free(next);
    /* lmatrix_csr_cpu.cc:1016-1043: selection sort of each row's columns,
     * swapping the value with its column */
    for (int k = 0; k < n_rows; ++k) {
        const int e = row[k + 1];
        for (int i = row[k]; i != e; ++i) {
            int mi = i, mv = col[i];
            for (int j = i + 1; j < e; ++j)
                if (col[j] < mv) { mi = j; mv = col[j]; }
            const int ti = col[i];
            col[i] = col[mi];
            col[mi] = ti;
            if (coo_val) {
                const double tv = val[i];
                val[i] = val[mi];
                val[mi] = tv;
            }
        }
    }
}

void orc_add_values(const int *row, const int *col, double *val,
                    const int *rows, int num_rows, const int *cols, int num_cols,
                    const double *values)
{
    for (int i = 0; i != num_rows; ++i) {
        int k = 0;
        const int off = i * num_cols;
        for (int j = row[rows[i]], je = row[rows[i] + 1]; k < num_cols && j != je; ++j) {
            if (cols[k] == col[j]) {
                val[j] += values[off + k];
                ++k;
            } else if (cols[k] < col[j]) {
                while (k < num_cols && cols[k] < col[j]) ++k;
                if (k >= num_cols) break;
                if (cols[k] == col[j]) {
                    val[j] += values[off + k];
                    ++k;
                }
            }
        }
    }
}

void orc_zero_rows(const int *row, const int *col, double *val,
                   const int *index_set, int size, double alpha)
{
    for (int i = 0; i != size; ++i) {
        const int r = index_set[i];
        for (int j = row[r]; j != row[r + 1]; ++j) val[j] = (col[j] == r) ? alpha : 0.0;
    }
}

/* ================================================================== */
/* SpMV / BLAS1                                                        */
/* ================================================================== */

void orc_spmv_d(int n, const int *row, const int *col, const double *val,
                const double *x, double *y)
{
    for (int i = 0; i < n; ++i) {
        double res = 0.0;
        for (int j = row[i]; j != row[i + 1]; ++j) res += val[j] * x[col[j]];
        y[i] = res;
    }
}

void orc_spmv_f(int n, const int *row, const int *col, const float *val,
                const float *x, float *y)
{
    for (int i = 0; i < n; ++i) {
        float res = 0.0f;
        for (int j = row[i]; j != row[i + 1]; ++j) res += val[j] * x[col[j]];
        y[i] = res;
    }
}

void orc_spmv_add_d(int n, const int *row, const int *col, const double *val,
                    const double *x, double *y)
{
    for (int i = 0; i < n; ++i) {
        double res = 0.0;
        for (int j = row[i]; j != row[i + 1]; ++j) res += val[j] * x[col[j]];
        y[i] += res;
    }
}

#define ORC_DOT5(T, ACC)                                                              \
    ACC t = 0;                                                                          \
    const int M = n % 5;                                                                \
    if (M == 0) {                                                                       \
        for (int i = 0; i < n; i += 5)                                                  \
            t += (ACC)x[i] * y[i] + (ACC)x[i + 1] * y[i + 1] + (ACC)x[i + 2] * y[i + 2] + \
                 (ACC)x[i + 3] * y[i + 3] + (ACC)x[i + 4] * y[i + 4];                   \
    } else {                                                                            \
        for (int i = 0; i != M; ++i) t += (ACC)x[i] * y[i];                             \
        if (n > 5)                                                                      \
            for (int i = M; i < n; i += 5)                                              \
                t += (ACC)x[i] * y[i] + (ACC)x[i + 1] * y[i + 1] + (ACC)x[i + 2] * y[i + 2] + \
                     (ACC)x[i + 3] * y[i + 3] + (ACC)x[i + 4] * y[i + 4];               \
    }                                                                                   \
    return t;

double orc_dot_d(int n, const double *x, const double *y) { ORC_DOT5(double, double) }
float orc_dot_f(int n, const float *x, const float *y) { ORC_DOT5(float, float) }
double orc_dot_f_acc_d(int n, const float *x, const float *y) { ORC_DOT5(float, double) }

/* ================================================================== */
/* Graph analysis                                                      */
/* ================================================================== */

int orc_multicoloring(int n, const int *row, const int *col,
                      int *ncolors, int *color_sizes, int *perm)
{
    /* lmatrix_csr_cpu.cc:2175-2222.  The reference repeats the neighbour scan
     * (row length) times; a scan that changes nothing leaves every later scan
     * unchanged too, so stopping there gives the identical colours. */
    int *nc = (int *)calloc(n > 0 ? n : 1, sizeof(int));
    if (!nc) return -2;
    int hicol = 0;
    for (int j = 0; j < n; ++j) {
        nc[j]++;
        const int m = row[j], m1 = row[j + 1];
        for (int k = m; k < m1; ++k) {
            int changed = 0;
            for (int i = m; i < m1; ++i) {
                const int dep = col[i];
                if (dep != j) {
                    if (nc[dep] == nc[j]) { ++nc[j]; changed = 1; }
                    if (nc[j] > hicol) hicol = nc[j];
                }
            }
            if (!changed) break;
        }
    }
    if (hicol == 0) { free(nc); return -1; }   /* the reference indexes colour -1 here */
    *ncolors = hicol;
    /* lmatrix_csr_cpu.cc:2240-2289: colour multiplicities and colour-major order */
    for (int k = 0; k < hicol; ++k) color_sizes[k] = 0;
    for (int i = 0; i < n; ++i) ++color_sizes[nc[i] - 1];
    int *start = (int *)malloc(sizeof(int) * hicol);
    int acc = 0;
    for (int k = 0; k < hicol; ++k) { start[k] = acc; acc += color_sizes[k]; }
    for (int j = 0; j < n; ++j) perm[start[nc[j] - 1]++] = j;
    free(start);
    free(nc);
    return 0;
}

static int has_entry(const int *row, const int *col, int r, int c)
{
    int lo = row[r], hi = row[r + 1] - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        if (col[mid] == c) return 1;
        if (col[mid] < c) lo = mid + 1; else hi = mid - 1;
    }
    /* columns may be unsorted in general CSR: fall back to a scan */
    for (int j = row[r]; j < row[r + 1]; ++j)
        if (col[j] == c) return 1;
    return 0;
}

int orc_levelscheduling(int n, const int *row, const int *col,
                        int *nlevels, int *level_sizes, int *perm)
{
    /* lmatrix_csr_cpu.cc:2295-2392.  A node is placed on the first sweep L with
     * depth == L once all its lower-triangular neighbours are placed; placing a
     * node raises the depth of its upper-triangular neighbours.  When the
     * pattern is structurally symmetric, this is level(k) = 1 + max level of
     * the lower neighbours, nodes within a level in index order, which is what
     * the fast path computes.  Otherwise the sweep is replayed literally. */
    int symmetric = 1;
    for (int i = 0; i < n && symmetric; ++i)
        for (int j = row[i]; j < row[i + 1]; ++j)
            if (col[j] != i && !has_entry(row, col, col[j], i)) { symmetric = 0; break; }
    if (symmetric) {
        int *lev = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
        int maxl = -1;
        for (int k = 0; k < n; ++k) {
            int l = 0;
            for (int j = row[k]; j < row[k + 1]; ++j)
                if (col[j] < k && lev[col[j]] + 1 > l) l = lev[col[j]] + 1;
            lev[k] = l;
            if (l > maxl) maxl = l;
        }
        const int nl = maxl + 1;
        for (int l = 0; l < nl; ++l) level_sizes[l] = 0;
        for (int k = 0; k < n; ++k) ++level_sizes[lev[k]];
        int *start = (int *)malloc(sizeof(int) * (nl > 0 ? nl : 1));
        int acc = 0;
        for (int l = 0; l < nl; ++l) { start[l] = acc; acc += level_sizes[l]; }
        for (int k = 0; k < n; ++k) perm[start[lev[k]]++] = k;
        free(start);
        free(lev);
        *nlevels = nl;
        return 0;
    }
    int *depth = (int *)calloc(n > 0 ? n : 1, sizeof(int));
    char *seen = (char *)calloc(n > 0 ? n : 1, 1);
    int done = 0, nlev = 0, ok = 0;
    for (int L = 0; L < n; ++L) {
        if (done == n) { ok = 1; break; }
        const int before = done;
        for (int k = 0; k < n; ++k) {
            if (seen[k] || depth[k] != L) continue;
            int stop = 0;
            for (int j = row[k]; j < row[k + 1]; ++j)
                if (col[j] < k && !seen[col[j]]) { stop = 1; break; }
            if (stop) continue;
            perm[done++] = k;
            seen[k] = 1;
            for (int j = row[k]; j < row[k + 1]; ++j)
                if (col[j] > k && depth[col[j]] <= depth[k]) depth[col[j]] = depth[k] + 1;
        }
        level_sizes[nlev++] = done - before;
    }
    if (!ok && done == n) ok = 1;
    free(depth);
    free(seen);
    if (!ok) { *nlevels = 0; return -1; }
    *nlevels = nlev;
    return 0;
}

void orc_reorder_csr(int n, const int *row, const int *col, const double *val,
                     const int *perm, int *row_out, int *col_out, double *val_out)
{
    /* CSR -> COO in CSR order, indices mapped old -> new
     * (lmatrix_coo_cpu.cc:1033-1050), then COO -> CSR (TransformFromCOO). */
    const int nnz = row[n];
    int *ind = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    int *cr = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    int *cc = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    for (int i = 0; i < n; ++i) ind[perm[i]] = i;
    for (int i = 0; i < n; ++i)
        for (int j = row[i]; j < row[i + 1]; ++j) { cr[j] = ind[i]; cc[j] = ind[col[j]]; }
    orc_coo_to_csr(n, nnz, cr, cc, val, row_out, col_out, val_out);
    free(ind);
    free(cr);
    free(cc);
}

void orc_reorder_vec(int n, const double *in, const int *perm, double *out)
{
    for (int i = 0; i < n; ++i) out[i] = in[perm[i]];
}

/* ================================================================== */
/* ILU(0)                                                              */
/* ================================================================== */

void orc_ilu0(int n, const int *row, const int *col, double *val)
{
    /* lmatrix_csr_cpu.cc:1880-1930.  (The reference also evaluates a progress
     * modulus that divides by zero for n <= 20; that has no numerical role.) */
    int diag_k = 0;
    for (int i = 1; i < n; ++i) {
        for (int nz_ik = row[i]; col[nz_ik] < i; ++nz_ik) {
            const int k = col[nz_ik];
            for (int p = row[k]; p < row[k + 1]; ++p)
                if (col[p] == k) diag_k = p;
            val[nz_ik] = val[nz_ik] / (1.0 * val[diag_k]);
            for (int nz_ij = nz_ik + 1; nz_ij < row[i + 1]; ++nz_ij) {
                double t = 0.0;
                for (int p = row[k]; p < row[k + 1]; ++p)
                    if (col[p] == col[nz_ij]) t = val[p];
                val[nz_ij] = val[nz_ij] - val[nz_ik] * t;
            }
        }
    }
}

void orc_ilu_solve(int n, const int *row, const int *col, const double *val,
                   const double *r, double *z)
{
    /* lmatrix_csr_cpu.cc:2127-2169 */
    int last_j = 0;
    for (int i = 0; i < n; ++i) {
        z[i] = r[i];
        for (int j = row[i]; j < row[i + 1]; ++j) {
            if (i > col[j]) z[i] -= z[col[j]] * val[j];
            if (i == col[j]) { last_j = j; break; }
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        for (int j = row[i]; j < row[i + 1]; ++j) {
            if (i == col[j]) last_j = j;
            if (i < col[j]) z[i] -= z[col[j]] * val[j];
        }
        z[i] /= val[last_j];
    }
}

/* ================================================================== */
/* Block sweep preconditioners                                         */
/* ================================================================== */

/* dropoffs (lpreconditioner_mc.cc:647-693) followed by compress_me
 * (lmatrix_csr_cpu.cc:2436-2495): zero the off-diagonals that couple two
 * rows of the same block; if any were zeroed, remove every zero entry. */
static void dropoffs(int n, int nblocks, const int *block_off, int **prow, int **pcol, double **pval)
{
    int *row = *prow, *col = *pcol;
    double *val = *pval;
    int *blk = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    for (int b = 0; b < nblocks; ++b)
        for (int i = block_off[b]; i < block_off[b + 1]; ++i) blk[i] = b;
    int ndel = 0;
    for (int i = 0; i < n; ++i)
        for (int j = row[i]; j < row[i + 1]; ++j)
            if (col[j] != i && blk[col[j]] == blk[i]) { val[j] = 0.0; ++ndel; }
    free(blk);
    if (ndel == 0) return;
    int keep = 0;
    for (int j = 0; j < row[n]; ++j) keep += (val[j] != 0.0);
    if (keep >= row[n]) return;
    int *r2 = (int *)malloc(sizeof(int) * (n + 1));
    int *c2 = (int *)malloc(sizeof(int) * (keep > 0 ? keep : 1));
    double *v2 = (double *)malloc(sizeof(double) * (keep > 0 ? keep : 1));
    int t = 0;
    for (int i = 0; i < n; ++i) {
        r2[i] = t;
        for (int j = row[i]; j < row[i + 1]; ++j)
            if (val[j] != 0.0) { c2[t] = col[j]; v2[t] = val[j]; ++t; }
    }
    r2[n] = t;
    free(row); free(col); free(val);
    *prow = r2; *pcol = c2; *pval = v2;
}

static void block_finish(orc_block_precond *P, int kind, double omega)
{
    /* extract_mat: ScaleOffdiag(omega) (lpreconditioner_mc.cc:485-488,
     * lmatrix_csr_cpu.cc:215-224); convert_Dmat2vec (:587-617) */
    const int n = P->n;
    for (int i = 0; i < n; ++i)
        for (int j = P->row[i]; j < P->row[i + 1]; ++j)
            if (P->col[j] != i) P->val[j] *= omega;
    P->Dv = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
    P->iDv = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
    for (int i = 0; i < n; ++i)
        for (int j = P->row[i]; j < P->row[i + 1]; ++j)
            if (P->col[j] == i) { P->Dv[i] = P->val[j]; P->iDv[i] = 1 / P->val[j]; }
    /* scale_D: lpreconditioner_mc_sgs.cc:46-59 (SGS) / lpreconditioner_mc_ilup.cc:197-205 (ILU) */
    for (int i = 0; i < n; ++i) {
        P->iDv[i] *= -1.0;
        if (kind == 0) {
            P->Dv[i] *= -1.0;
            P->Dv[i] *= 1.0 / (omega * (2.0 - omega));
        }
    }
    P->kind = kind;
    P->omega = omega;
}

static int *sizes_to_offsets(int nb, const int *sizes)
{
    int *off = (int *)malloc(sizeof(int) * (nb + 1));
    off[0] = 0;
    for (int b = 0; b < nb; ++b) off[b + 1] = off[b] + sizes[b];
    return off;
}

int orc_mcsgs_build(int n, const int *row, const int *col, const double *val, double omega,
                    orc_block_precond *P, int *Ap_row, int *Ap_col, double *Ap_val)
{
    memset(P, 0, sizeof(*P));
    const int nnz = row[n];
    int *sizes = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    P->perm = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    int nc;
    if (orc_multicoloring(n, row, col, &nc, sizes, P->perm)) { free(sizes); return -1; }
    P->n = n;
    P->nblocks = nc;
    P->block_off = sizes_to_offsets(nc, sizes);
    free(sizes);
    /* permute (lpreconditioner_mc.cc:353-387): operator and LU = P A P^T */
    orc_reorder_csr(n, row, col, val, P->perm, Ap_row, Ap_col, Ap_val);
    P->row = (int *)malloc(sizeof(int) * (n + 1));
    P->col = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    P->val = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
    memcpy(P->row, Ap_row, sizeof(int) * (n + 1));
    memcpy(P->col, Ap_col, sizeof(int) * nnz);
    memcpy(P->val, Ap_val, sizeof(double) * nnz);
    /* factorize: no-op (lpreconditioner_mc_gs.cc:71-74); dropoffs */
    dropoffs(n, nc, P->block_off, &P->row, &P->col, &P->val);
    block_finish(P, 0, omega);
    return 0;
}

int orc_ilu0_build(int n, const int *row, const int *col, const double *val, int mode,
                   orc_block_precond *P, int *Ap_row, int *Ap_col, double *Ap_val)
{
    memset(P, 0, sizeof(*P));
    const int nnz = row[n];
    int *sizes = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    P->perm = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    P->n = n;
    P->row = (int *)malloc(sizeof(int) * (n + 1));
    P->col = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    P->val = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
    int nb;
    if (mode == 0) {
        /* ILU(0) in natural order, then level scheduling of the factors and
         * permute_all (lpreconditioner_mc.cc:176-192, 310-351) */
        memcpy(P->row, row, sizeof(int) * (n + 1));
        memcpy(P->col, col, sizeof(int) * nnz);
        memcpy(P->val, val, sizeof(double) * nnz);
        orc_ilu0(n, P->row, P->col, P->val);
        if (orc_levelscheduling(n, P->row, P->col, &nb, sizes, P->perm)) { free(sizes); return -1; }
        int *r2 = (int *)malloc(sizeof(int) * (n + 1));
        int *c2 = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
        double *v2 = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
        orc_reorder_csr(n, P->row, P->col, P->val, P->perm, r2, c2, v2);
        free(P->row); free(P->col); free(P->val);
        P->row = r2; P->col = c2; P->val = v2;
        orc_reorder_csr(n, row, col, val, P->perm, Ap_row, Ap_col, Ap_val);
    } else {
        /* multicolouring, permute, ILU(0) of the permuted operator */
        if (orc_multicoloring(n, row, col, &nb, sizes, P->perm)) { free(sizes); return -1; }
        orc_reorder_csr(n, row, col, val, P->perm, Ap_row, Ap_col, Ap_val);
        memcpy(P->row, Ap_row, sizeof(int) * (n + 1));
        memcpy(P->col, Ap_col, sizeof(int) * nnz);
        memcpy(P->val, Ap_val, sizeof(double) * nnz);
        orc_ilu0(n, P->row, P->col, P->val);
    }
    P->nblocks = nb;
    P->block_off = sizes_to_offsets(nb, sizes);
    free(sizes);
    dropoffs(n, nb, P->block_off, &P->row, &P->col, &P->val);
    block_finish(P, 1, 1.0);
    return 0;
}

/* Pattern of A^p: rows of the symbolic product by A, p - 1 times, columns
 * ascending (MatrixSupSPower / MatrixMultSupStructure, lmatrix_csr_cpu.cc:
 * 1520-1664, whose COO round trip sorts every row).  p = 1 copies A's
 * pattern.  Outputs allocated here (free with orc_free); returns nnz. */
int orc_power_pattern(int n, const int *row, const int *col, int p, int **row_out, int **col_out)
{
    int nnz = row[n];
    int *r = (int *)malloc(sizeof(int) * (n + 1));
    int *c = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    memcpy(r, row, sizeof(int) * (n + 1));
    memcpy(c, col, sizeof(int) * nnz);
    int *seen = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    int *buf = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    for (int it = 1; it < p; ++it) {
        for (int j = 0; j < n; ++j) seen[j] = -1;
        int cap = nnz * 2 + n, m = 0;
        int *r2 = (int *)malloc(sizeof(int) * (n + 1));
        int *c2 = (int *)malloc(sizeof(int) * cap);
        r2[0] = 0;
        for (int i = 0; i < n; ++i) {
            int len = 0;
            for (int a = r[i]; a < r[i + 1]; ++a) {
                const int k = c[a];
                for (int b = row[k]; b < row[k + 1]; ++b)
                    if (seen[col[b]] != i) { seen[col[b]] = i; buf[len++] = col[b]; }
            }
            /* insertion sort of the row's columns */
            for (int x = 1; x < len; ++x) {
                const int v = buf[x];
                int y = x - 1;
                while (y >= 0 && buf[y] > v) { buf[y + 1] = buf[y]; --y; }
                buf[y + 1] = v;
            }
            if (m + len > cap) { cap = 2 * (m + len); c2 = (int *)realloc(c2, sizeof(int) * cap); }
            memcpy(c2 + m, buf, sizeof(int) * len);
            m += len;
            r2[i + 1] = m;
        }
        free(r); free(c);
        r = r2; c = c2; nnz = m;
    }
    free(seen); free(buf);
    *row_out = r;
    *col_out = c;
    return nnz;
}

void orc_free(void *p) { free(p); }

/* ILU(p) (lmatrix_csr_cpu.cc:1933-2104): A's values on the pattern of
 * A^(p+1), level 0 for nonzero entries and 9999 for the rest; IKJ
 * elimination over the lower entries of level <= p with
 * lev_ij = min(lev_ij, 1 + lev_kj + lev_ik); entries above level p are zeroed
 * after each row; the result keeps the entries of level <= p.  Outputs
 * allocated here; returns nnz. */
int orc_ilup(int n, const int *row, const int *col, const double *val, int p, int **row_out, int **col_out,
             double **val_out)
{
    int *fr, *fc;
    const int fn = orc_power_pattern(n, row, col, p + 1, &fr, &fc);
    double *fv = (double *)malloc(sizeof(double) * (fn > 0 ? fn : 1));
    double *lev = (double *)malloc(sizeof(double) * (fn > 0 ? fn : 1));
    for (int i = 0; i < n; ++i)
        for (int j = fr[i]; j < fr[i + 1]; ++j) {
            double v = 0.0;   /* MatrixAdd onto the zeroed pattern */
            for (int k = row[i]; k < row[i + 1]; ++k)
                if (fc[j] == col[k]) v += val[k];
            fv[j] = v;
            lev[j] = v * v > 0.0 ? 0.0 : 9999.0;
        }
    const double pp = (double)p;
    int kk = 0;
    for (int i = 1; i < n; ++i) {
        for (int ik = fr[i]; fc[ik] < i; ++ik) {
            if (!(lev[ik] <= pp)) continue;
            const int k = fc[ik];
            for (int h = fr[k]; h < fr[k + 1]; ++h)
                if (fc[h] == k) { kk = h; break; }
            fv[ik] = fv[ik] / (1.0 * fv[kk]);
            for (int ij = ik + 1; ij < fr[i + 1]; ++ij) {
                double vkj = 0.0, lkj = 9999.0;
                for (int h = fr[k]; h < fr[k + 1]; ++h)
                    if (fc[h] == fc[ij]) { vkj = fv[h]; lkj = lev[h]; break; }
                const double lt = 1 + lkj + lev[ik];
                fv[ij] = fv[ij] - vkj * fv[ik];
                if (lev[ij] > lt) lev[ij] = lt;
            }
        }
        for (int h = fr[i]; h < fr[i + 1]; ++h)
            if (lev[h] > pp) { fv[h] = 0.0; lev[h] = 9999.0; }
    }
    int m = 0;
    for (int j = 0; j < fn; ++j) m += lev[j] <= pp;
    int *r = (int *)malloc(sizeof(int) * (n + 1));
    int *c = (int *)malloc(sizeof(int) * (m > 0 ? m : 1));
    double *v = (double *)malloc(sizeof(double) * (m > 0 ? m : 1));
    int t = 0;
    r[0] = 0;
    for (int i = 0; i < n; ++i) {
        for (int h = fr[i]; h < fr[i + 1]; ++h)
            if (lev[h] <= pp) { c[t] = fc[h]; v[t] = fv[h]; ++t; }
        r[i + 1] = t;
    }
    free(fr); free(fc); free(fv); free(lev);
    *row_out = r; *col_out = c; *val_out = v;
    return m;
}

int orc_ilup_build(int n, const int *row, const int *col, const double *val, int mode, int ilu_p, int mat_power,
                   orc_block_precond *P, int *Ap_row, int *Ap_col, double *Ap_val)
{
    /* lpreconditioner_mc.cc:157-195 with lpreconditioner_mc_ilup.cc:107-194:
     * mode 0 ILU(p) in natural order, levels of the factors, permute_all;
     * mode 1 colouring of the pattern of A^mat_power, permute, ILU(p) of the
     * permuted operator. */
    if (ilu_p == 0 && mat_power == 1) return orc_ilu0_build(n, row, col, val, mode, P, Ap_row, Ap_col, Ap_val);
    memset(P, 0, sizeof(*P));
    int *sizes = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    P->perm = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    P->n = n;
    int nb, *fr, *fc;
    double *fv;
    if (mode == 0) {
        const int fn = orc_ilup(n, row, col, val, ilu_p, &fr, &fc, &fv);
        if (orc_levelscheduling(n, fr, fc, &nb, sizes, P->perm)) { free(sizes); return -1; }
        P->row = (int *)malloc(sizeof(int) * (n + 1));
        P->col = (int *)malloc(sizeof(int) * (fn > 0 ? fn : 1));
        P->val = (double *)malloc(sizeof(double) * (fn > 0 ? fn : 1));
        orc_reorder_csr(n, fr, fc, fv, P->perm, P->row, P->col, P->val);
        free(fr); free(fc); free(fv);
        orc_reorder_csr(n, row, col, val, P->perm, Ap_row, Ap_col, Ap_val);
    } else {
        int *ar = (int *)row, *ac = (int *)col;
        if (mat_power > 1) orc_power_pattern(n, row, col, mat_power, &ar, &ac);
        const int bad = orc_multicoloring(n, ar, ac, &nb, sizes, P->perm);
        if (mat_power > 1) { free(ar); free(ac); }
        if (bad) { free(sizes); return -1; }
        orc_reorder_csr(n, row, col, val, P->perm, Ap_row, Ap_col, Ap_val);
        if (ilu_p > 0) {
            orc_ilup(n, Ap_row, Ap_col, Ap_val, ilu_p, &P->row, &P->col, &P->val);
        } else {
            const int nnz = row[n];
            P->row = (int *)malloc(sizeof(int) * (n + 1));
            P->col = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
            P->val = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
            memcpy(P->row, Ap_row, sizeof(int) * (n + 1));
            memcpy(P->col, Ap_col, sizeof(int) * nnz);
            memcpy(P->val, Ap_val, sizeof(double) * nnz);
            orc_ilu0(n, P->row, P->col, P->val);
        }
    }
    P->nblocks = nb;
    P->block_off = sizes_to_offsets(nb, sizes);
    free(sizes);
    dropoffs(n, nb, P->block_off, &P->row, &P->col, &P->val);
    block_finish(P, 1, 1.0);
    return 0;
}

void orc_block_apply(const orc_block_precond *P, const double *r, double *z)
{
    /* ApplylPreconditioner (lpreconditioner_mc.cc:716-728): the per-block
     * VectorMultAdd sums one block's row entries, then adds that partial sum
     * to the output chunk, blocks in ascending (forward) or descending
     * (backward) order; blocks with no entries at all are skipped. */
    const int n = P->n, nb = P->nblocks;
    const int *off = P->block_off;
    int *blk = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    for (int b = 0; b < nb; ++b)
        for (int i = off[b]; i < off[b + 1]; ++i) blk[i] = b;
    /* non-empty flags of the (row block, column block) submatrices */
    char *ne = (char *)calloc((size_t)nb * nb, 1);
    for (int i = 0; i < n; ++i)
        for (int j = P->row[i]; j < P->row[i + 1]; ++j) ne[(size_t)blk[i] * nb + blk[P->col[j]]] = 1;
    /* splitvectors; forwardstep */
    for (int b = 0; b < nb; ++b) {
        for (int i = off[b]; i < off[b + 1]; ++i) {
            double y = r[i] * -1.0;
            int j = P->row[i];
            for (int cb = 0; cb < b; ++cb) {
                double res = 0.0;
                while (j < P->row[i + 1] && P->col[j] < off[cb + 1]) {
                    if (P->col[j] >= off[cb]) res += P->val[j] * z[P->col[j]];
                    ++j;
                }
                if (ne[(size_t)b * nb + cb]) y += res;
            }
            if (P->kind == 0) z[i] = y * P->iDv[i];
            else z[i] = y * -1.0;
        }
    }
    /* diagonalstep */
    for (int i = 0; i < n; ++i) z[i] = (P->kind == 0) ? z[i] * P->Dv[i] : z[i] * -1.0;
    /* backwardstep */
    for (int b = nb - 1; b >= 0; --b) {
        for (int i = off[b]; i < off[b + 1]; ++i) {
            double y = z[i];
            for (int cb = nb - 1; cb > b; --cb) {
                double res = 0.0;
                for (int j = P->row[i]; j < P->row[i + 1]; ++j) {
                    const int c = P->col[j];
                    if (c >= off[cb] && c < off[cb + 1]) res += P->val[j] * z[c];
                }
                if (ne[(size_t)b * nb + cb]) y += res;
            }
            z[i] = y * P->iDv[i];
        }
    }
    free(ne);
    free(blk);
}

void orc_block_free(orc_block_precond *P)
{
    free(P->block_off); free(P->perm); free(P->row); free(P->col); free(P->val);
    free(P->Dv); free(P->iDv);
    memset(P, 0, sizeof(*P));
}

/* ================================================================== */
/* Solvers                                                             */
/* ================================================================== */

int orc_check(const orc_control *c, int step, double value, double *first_value)
{
    /* iterate_control.cc:84-110 (first_step = 0) */
    if (step == 0) *first_value = value;
    if (value < c->abstol) return ORC_SUCCESS_ABS;
    if (value < c->reltol * *first_value) return ORC_SUCCESS_REL;
    if (value > c->divtol * *first_value) return ORC_FAIL_DIV;
    if (step >= c->maxits) return ORC_FAIL_MAXITS;
    return ORC_ITERATE;
}

void orc_invdiag(int n, const int *row, const int *col, const double *val, double *invdiag)
{
    for (int i = 0; i < n; ++i)
        for (int j = row[i]; j < row[i + 1]; ++j)
            if (col[j] == i) invdiag[i] = 1 / val[j];
}

void orc_jacobi_apply(void *jacobi_ctx, const double *r, double *z)
{
    /* CopyFrom + ElementWiseMult (lpreconditioner.cc:151-165) */
    const orc_jacobi *J = (const orc_jacobi *)jacobi_ctx;
    for (int i = 0; i < J->n; ++i) z[i] = r[i] * J->invdiag[i];
}

void orc_block_apply_cb(void *P, const double *r, double *z)
{
    orc_block_apply((const orc_block_precond *)P, r, z);
}

static void axpy_d(int n, double a, const double *x, double *y)
{
    for (int i = 0; i < n; ++i) y[i] += a * x[i];
}

static void scaleadd_d(int n, double a, const double *x, double *y)
{
    for (int i = 0; i < n; ++i) y[i] = a * y[i] + x[i];
}

int orc_pcg(int n, const int *row, const int *col, const double *val,
            orc_precond_fn precond, void *ctx, const double *b, double *x,
            const orc_control *ctl, orc_result *out, double *res_hist)
{
    double *r = (double *)malloc(sizeof(double) * n), *p = (double *)malloc(sizeof(double) * n);
    double *z = (double *)malloc(sizeof(double) * n), *Ap = (double *)malloc(sizeof(double) * n);
    double first = 0.0, beta, rr, res;
    int iter = 0, conv;
    /* cg.cc:200-206 (SolvePrecond) / cg.cc:104-109 (SolveNoPrecond) */
    orc_spmv_d(n, row, col, val, x, r);
    scaleadd_d(n, -1.0, b, r);
    rr = orc_dot_d(n, r, r);
    res = sqrt(rr);
    conv = orc_check(ctl, iter, res, &first);
    if (res_hist) res_hist[0] = res;
    if (precond) {
        memset(z, 0, sizeof(double) * n);
        precond(ctx, r, z);
        memcpy(p, z, sizeof(double) * n);
        beta = orc_dot_d(n, r, z);
    } else {
        memcpy(p, r, sizeof(double) * n);
        beta = rr;
    }
    while (conv == ORC_ITERATE) {
        ++iter;
        orc_spmv_d(n, row, col, val, p, Ap);
        const double alpha = beta / orc_dot_d(n, Ap, p);
        axpy_d(n, alpha, p, x);
        axpy_d(n, -alpha, Ap, r);
        rr = orc_dot_d(n, r, r);
        res = sqrt(rr);
        if (res_hist) res_hist[iter] = res;
        conv = orc_check(ctl, iter, res, &first);
        if (conv != ORC_ITERATE) break;
        if (precond) {
            memset(z, 0, sizeof(double) * n);
            precond(ctx, r, z);
            const double gamma = orc_dot_d(n, r, z);
            beta = gamma / beta;
            scaleadd_d(n, beta, z, p);
            beta = gamma;
        } else {
            beta = rr / beta;
            scaleadd_d(n, beta, r, p);
            beta = rr;
        }
    }
    out->iters = iter;
    out->status = conv;
    out->res0 = first;
    out->res = res;
    free(r); free(p); free(z); free(Ap);
    return (conv == ORC_FAIL_DIV || conv == ORC_FAIL_MAXITS) ? 1 : 0;
}

static void rot_apply(double cs, double sn, double *dx, double *dy)
{
    /* gmres.h:77-83 */
    const double t = cs * (*dx) + sn * (*dy);
    *dy = -sn * (*dx) + cs * (*dy);
    *dx = t;
}

static void rot_generate(double dx, double dy, double *cs, double *sn)
{
    /* gmres.h:91-97 */
    const double beta = sqrt(dx * dx + dy * dy);
    *cs = dx / beta;
    *sn = dy / beta;
}

int orc_gmres(int n, const int *row, const int *col, const double *val,
              orc_precond_fn precond, void *ctx, int m, const double *b, double *x,
              const orc_control *ctl, orc_result *out)
{
    const int mb = (m < ctl->maxits) ? m : ctl->maxits;   /* gmres.cc:301 */
    double *V = (double *)malloc(sizeof(double) * (size_t)n * (mb + 1));
    double *w = (double *)malloc(sizeof(double) * n), *z = (double *)malloc(sizeof(double) * n);
    double *H = (double *)calloc((size_t)mb * (mb + 1), sizeof(double));   /* H(j,i) = H[j*(mb+1)+i] */
    double *g = (double *)calloc(mb + 1, sizeof(double));
    double *cs = (double *)calloc(mb + 1, sizeof(double)), *sn = (double *)calloc(mb + 1, sizeof(double));
    double *y = (double *)calloc(mb + 1, sizeof(double));
    double first = 0.0, res;
    int iter = 0, conv;
#define HH(j, i) H[(size_t)(j) * (mb + 1) + (i)]
#define VV(k) (V + (size_t)(k) * n)
#define PREC(src, dst) do { if (precond) { memset(dst, 0, sizeof(double) * n); precond(ctx, src, dst); } \
                            else memcpy(dst, src, sizeof(double) * n); } while (0)
    orc_spmv_d(n, row, col, val, x, VV(0));
    scaleadd_d(n, -1.0, b, VV(0));
    res = sqrt(orc_dot_d(n, VV(0), VV(0)));
    conv = orc_check(ctl, iter, res, &first);
    while (conv == ORC_ITERATE) {
        for (int i = 0; i <= mb; ++i) g[i] = 0.0;
        for (size_t i = 0; i < (size_t)mb * (mb + 1); ++i) H[i] = 0.0;
        { const double s = 1.0 / res; for (int i = 0; i < n; ++i) VV(0)[i] *= s; }
        g[0] = res;
        int j_end = mb - 1;
        for (int j = 0; j != mb; ++j) {
            ++iter;
            PREC(VV(j), z);
            orc_spmv_d(n, row, col, val, z, w);
            for (int i = 0; i <= j; ++i) {
                HH(j, i) = orc_dot_d(n, w, VV(i));
                axpy_d(n, -1.0 * HH(j, i), VV(i), w);
            }
            HH(j, j + 1) = sqrt(orc_dot_d(n, w, w));
            { const double s = 1.0 / HH(j, j + 1); for (int i = 0; i < n; ++i) w[i] *= s; }
            memcpy(VV(j + 1), w, sizeof(double) * n);
            for (int k = 0; k != j; ++k) rot_apply(cs[k], sn[k], &HH(j, k), &HH(j, k + 1));
            rot_generate(HH(j, j), HH(j, j + 1), &cs[j], &sn[j]);
            rot_apply(cs[j], sn[j], &HH(j, j), &HH(j, j + 1));
            rot_apply(cs[j], sn[j], &g[j], &g[j + 1]);
            res = fabs(g[j + 1]);
            conv = orc_check(ctl, iter, res, &first);
            if (conv != ORC_ITERATE) { j_end = j; break; }
        }
        /* UpdateSolution (gmres.cc:487-510), preconditioner, x += w */
        for (int i = 0; i <= mb; ++i) y[i] = g[i];
        for (int i = j_end + 1; i--;) {
            y[i] /= HH(i, i);
            const double t = y[i];
            for (int k = 0; k < i; ++k) y[k] -= HH(i, k) * t;
        }
        memset(z, 0, sizeof(double) * n);
        for (int k = 0; k <= j_end; ++k) axpy_d(n, y[k], VV(k), z);
        PREC(z, w);
        axpy_d(n, 1.0, w, x);
        if (conv == ORC_ITERATE) {
            orc_spmv_d(n, row, col, val, x, VV(0));
            scaleadd_d(n, -1.0, b, VV(0));
        }
    }
#undef HH
#undef VV
#undef PREC
    out->iters = iter;
    out->status = conv;
    out->res0 = first;
    out->res = res;
    free(V); free(w); free(z); free(H); free(g); free(cs); free(sn); free(y);
    return (conv == ORC_FAIL_DIV || conv == ORC_FAIL_MAXITS) ? 1 : 0;
}

int orc_pcg_f32(int n, const int *row, const int *col, const float *val,
                const float *invdiag, const float *b, float *x,
                const orc_control *ctl, orc_result *out)
{
    float *r = (float *)malloc(sizeof(float) * n), *p = (float *)malloc(sizeof(float) * n);
    float *z = (float *)malloc(sizeof(float) * n), *Ap = (float *)malloc(sizeof(float) * n);
    double first = 0.0, beta, rr, res;
    int iter = 0, conv;
    orc_spmv_f(n, row, col, val, x, r);
    for (int i = 0; i < n; ++i) r[i] = b[i] - r[i];
    rr = orc_dot_f_acc_d(n, r, r);
    res = sqrt(rr);
    conv = orc_check(ctl, iter, res, &first);
    for (int i = 0; i < n; ++i) z[i] = r[i] * invdiag[i];
    memcpy(p, z, sizeof(float) * n);
    beta = orc_dot_f_acc_d(n, r, z);
    while (conv == ORC_ITERATE) {
        ++iter;
        orc_spmv_f(n, row, col, val, p, Ap);
        const double alpha = beta / orc_dot_f_acc_d(n, Ap, p);
        const float af = (float)alpha;
        for (int i = 0; i < n; ++i) { x[i] += af * p[i]; r[i] -= af * Ap[i]; }
        rr = orc_dot_f_acc_d(n, r, r);
        res = sqrt(rr);
        conv = orc_check(ctl, iter, res, &first);
        if (conv != ORC_ITERATE) break;
        for (int i = 0; i < n; ++i) z[i] = r[i] * invdiag[i];
        const double gamma = orc_dot_f_acc_d(n, r, z);
        const float bf = (float)(gamma / beta);
        for (int i = 0; i < n; ++i) p[i] = bf * p[i] + z[i];
        beta = gamma;
    }
    out->iters = iter;
    out->status = conv;
    out->res0 = first;
    out->res = res;
    free(r); free(p); free(z); free(Ap);
    return (conv == ORC_FAIL_DIV || conv == ORC_FAIL_MAXITS) ? 1 : 0;
}

int orc_mpir(int n, const int *row, const int *col, const double *val,
             const double *b, double *x, const orc_control *outer,
             const orc_control *inner, int max_outer, int res0_mode,
             orc_result *out, int *inner_iters_total)
{
    const int nnz = row[n];
    float *vl = (float *)malloc(sizeof(float) * (nnz > 0 ? nnz : 1));
    float *dl = (float *)malloc(sizeof(float) * n);
    float *rl = (float *)malloc(sizeof(float) * n), *cl = (float *)malloc(sizeof(float) * n);
    double *r = (double *)malloc(sizeof(double) * n), *invd = (double *)malloc(sizeof(double) * n);
    /* CastFrom of the operator (CPUsimple_csr_lmatrix.cc:115-164) and of D^-1 */
    for (int j = 0; j < nnz; ++j) vl[j] = (float)val[j];
    orc_invdiag(n, row, col, val, invd);
    for (int i = 0; i < n; ++i) dl[i] = (float)invd[i];
    /* mpir.cc:125-128 */
    orc_spmv_d(n, row, col, val, x, r);
    scaleadd_d(n, -1.0, b, r);
    double res = sqrt(orc_dot_d(n, r, r));
    double res0 = res;
    const double first = res;
    int n_outer = 0, total = 0;
    while (res > outer->abstol && res > res0 * outer->reltol && res < outer->divtol &&
           n_outer < max_outer) {
        ++n_outer;
        for (int i = 0; i < n; ++i) { rl[i] = (float)r[i]; cl[i] = 0.0f; }   /* mpir.cc:169-170 */
        orc_result ir;
        orc_pcg_f32(n, row, col, vl, dl, rl, cl, inner, &ir);                  /* mpir.cc:193 */
        total += ir.iters;
        for (int i = 0; i < n; ++i) x[i] += (double)cl[i];                     /* mpir.cc:223,253 */
        orc_spmv_d(n, row, col, val, x, r);                                    /* mpir.cc:271-273 */
        scaleadd_d(n, -1.0, b, r);
        res = sqrt(orc_dot_d(n, r, r));
        if (res0_mode == 1) res0 = res;                                        /* mpir.cc:274 */
    }
    out->iters = n_outer;
    out->res0 = first;
    out->res = res;
    out->status = (res < outer->abstol || res < res0 * outer->reltol) ? ORC_SUCCESS_REL : ORC_FAIL_MAXITS;
    if (inner_iters_total) *inner_iters_total = total;
    free(vl); free(dl); free(rl); free(cl); free(r); free(invd);
    return out->status == ORC_SUCCESS_REL ? 0 : 1;
}

/* ------------------------------------------------------------------ */
/* Matrix value and structure operations                               */
/* ------------------------------------------------------------------ */

/* CPU_CSR_lMatrix::Scale / ScaleOffdiag / Zeros (lmp/lmatrix_csr_cpu.cc:100-103, 205-224). */
void orc_csr_scale(int n, const int *row, const int *col, double *val, double alpha, int mode)
{
    for (int i = 0; i < n; ++i)
        for (int j = row[i]; j < row[i + 1]; ++j) {
            if (mode == 2) val[j] = 0.0;
            else if (mode == 0 || col[j] != i) val[j] *= alpha;
        }
}

/* CPU_CSR_lMatrix::extract_diagelements / extract_invdiagelements (:2395-2431):
 * every stored diagonal entry of the row assigns, so the last one stays. */
void orc_csr_diag(const int *row, const int *col, const double *val, int start, int end, int inverse,
                  double *out)
{
    for (int i = start; i < end; ++i)
        for (int j = row[i]; j < row[i + 1]; ++j)
            if (col[j] == i) out[i - start] = inverse ? 1 / val[j] : val[j];
}

/* CPU_CSR_lMatrix::extract_submatrix (:1768-1843) and Compress (:142-202). */
int orc_csr_extract(int n, const int *row, const int *col, const double *val, int mode, int sr, int sc, int er,
                    int ec, int **row_out, int **col_out, double **val_out)
{
    const int r0 = mode == 0 ? sr : 0, r1 = mode == 0 ? er : n, rows = r1 - r0;
    int *ro = (int *)calloc((size_t)rows + 1, sizeof(int));
    int cnt = 0;
    for (int i = r0; i < r1; ++i) {
        for (int j = row[i]; j < row[i + 1]; ++j)
            if (mode == 0 ? (col[j] >= sc && col[j] < ec) : (val[j] != 0.0)) ++cnt;
        ro[i - r0 + 1] = cnt;
    }
    int *co = (int *)malloc(sizeof(int) * (size_t)(cnt > 0 ? cnt : 1));
    double *vo = (double *)malloc(sizeof(double) * (size_t)(cnt > 0 ? cnt : 1));
    for (int i = r0; i < r1; ++i) {
        int k = ro[i - r0];
        if (mode == 1) {
            /* Compress keeps the nonzero entries in their order */
            for (int j = row[i]; j < row[i + 1]; ++j)
                if (val[j] != 0.0) { co[k] = col[j]; vo[k] = val[j]; ++k; }
            continue;
        }
        /* init_structure: the row's block columns, sorted (TransformFromCOO,
         * :951-1044); then Zeros and add_value in source order (:1127-1181),
         * each value added to the first stored entry of its column */
        const int b = k;
        for (int j = row[i]; j < row[i + 1]; ++j)
            if (col[j] >= sc && col[j] < ec) co[k++] = col[j] - sc;
        for (int a = b; a < k; ++a)           /* ascending columns */
            for (int c = a + 1; c < k; ++c)
                if (co[c] < co[a]) { int t = co[a]; co[a] = co[c]; co[c] = t; }
        for (int a = b; a < k; ++a) vo[a] = 0.0;
        for (int j = row[i]; j < row[i + 1]; ++j)
            if (col[j] >= sc && col[j] < ec)
                for (int a = b; a < k; ++a)
                    if (co[a] == col[j] - sc) { vo[a] += val[j]; break; }
    }
    *row_out = ro;
    *col_out = co;
    *val_out = vo;
    return cnt;
}

/* ------------------------------------------------------------------ */
/* lVector BLAS1 members beyond the Krylov hot path                    */
/* ------------------------------------------------------------------ */

/* CPUsimple_lVector::ArgMin (lmp/CPUsimple_lvector.cc:51-70). */
int orc_iamin(int n, const double *x)
{
    int k = 0;
    double v = fabs(x[0]);
    for (int i = 1; i < n; ++i)
        if (fabs(x[i]) < v) { k = i; v = fabs(x[i]); }
    return k;
}

/* CPUsimple_lVector::ArgMax (:73-92). */
int orc_iamax(int n, const double *x)
{
    int k = 0;
    double v = fabs(x[0]);
    for (int i = 1; i < n; ++i)
        if (fabs(x[i]) > v) { k = i; v = fabs(x[i]); }
    return k;
}

/* CPUsimple_lVector::Norm1 (:95-151): the n % 5 leading terms one by one,
 * then groups of five summed left to right and added. */
double orc_asum(int n, const double *x)
{
    const int m = n % 5;
    double t = 0.0;
    if (m == 0) {
        for (int i = 0; i < n; i += 5)
            t += fabs(x[i]) + fabs(x[i + 1]) + fabs(x[i + 2]) + fabs(x[i + 3]) + fabs(x[i + 4]);
    } else {
        for (int i = 0; i < m; ++i) t += fabs(x[i]);
        if (n > 5)
            for (int i = m; i < n; i += 5)
                t += fabs(x[i]) + fabs(x[i + 1]) + fabs(x[i + 2]) + fabs(x[i + 3]) + fabs(x[i + 4]);
    }
    return t;
}

/* CPUsimple_lVector::Rot (:448-466). */
void orc_rot(int n, double *x, double *y, double c, double s)
{
    for (int i = 0; i < n; ++i) {
        const double t = c * x[i] + s * y[i];
        y[i] = c * y[i] - s * x[i];
        x[i] = t;
    }
}

/* CPUsimple_lVector::Rotm (:540-600): flag -2 leaves both vectors. */
void orc_rotm(int n, double *x, double *y, const double *param)
{
    const double flag = param[0];
    for (int i = 0; i < n; ++i) {
        const double t1 = y[i], t2 = x[i];
        if (flag == -1) {
            y[i] = t1 * param[1] + t2 * param[3];
            x[i] = t1 * param[2] + t2 * param[4];
        } else if (flag == 0) {
            y[i] = t1 + t2 * param[3];
            x[i] = t1 * param[2] + t2;
        } else if (flag == 1) {
            y[i] = t1 * param[1] + t2;
            x[i] = t2 * param[4] - t1;
        }
    }
}

/* CPUsimple_lVector::Rotg (:492-535). */
void orc_rotg(double *a, double *b, double *c, double *s)
{
    const double ta = fabs(*a), tb = fabs(*b);
    const double roe = ta > tb ? *a : *b;
    const double scal = ta + tb;
    if (scal == 0) {
        *c = 1;
        *s = *a = *b = 0;
        return;
    }
    const double t0 = ta / scal, t1 = tb / scal;
    double r = scal * sqrt(t0 * t0 + t1 * t1);
    if (roe < 0) r = -r;
    *c = *a / r;
    *s = *b / r;
    double z;
    if (ta > tb) z = *s;
    else if (*c != 0) z = 1 / *c;
    else z = 1;
    *a = r;
    *b = z;
}
