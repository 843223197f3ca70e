/*
 * oracle.h -- CPU restatement of HiFlow3's local linear-algebra (lmp) hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the B200 platform:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it.  The product library (libb200la.so) never links or calls it.
 *
 * Every function restates one reference routine and cites it (paths are
 * relative to the HiFlow3 2.0 source tree).  The restatement is pinned against
 * the reference itself: oracle/Makefile compiles the reference's own CPU lmp
 * sources into oracle/_ref/, and tests/golden/gen_golden.py records their
 * outputs as fixtures that tests/test_oracle_pin.py compares with this code.
 *
 * Conventions (as in the reference, src/linear_algebra/lmp/lmatrix_formats.h:40-45):
 * CSR with int32 row[n+1], col[nnz], val[nnz]; DoFs of the structured Q1 grids
 * are numbered lexicographically, x fastest.
 */
#ifndef HIFLOW_B200_ORACLE_H
#define HIFLOW_B200_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Structured Q1 systems (the workloads' source of truth)              */
/* ------------------------------------------------------------------ */

/* Number of DoFs and stored nonzeros of a dim-D Q1 grid with N cells per axis. */
int orc_q1_sizes(int dim, int N, int *n_out, int64_t *nnz_out);

/* Sparsity pattern as COO pairs, rows ascending and columns ascending per row. */
int orc_q1_structure(int dim, int N, int *coo_row, int *coo_col);

/* Element matrix (2^dim x 2^dim, row-major, local vertices x fastest) of
 *   kind 0: int coef * grad(phi_j).grad(phi_i)                  (Poisson)
 *   kind 1: int coef * grad(phi_j).grad(phi_i) + (beta.grad phi_j) phi_i  (conv-diff)
 * on an axis-aligned cube of edge h, 2-point Gauss per axis.  Restates
 * examples/poisson/poisson_tutorial.h:152-176 and
 * examples/convection_diffusion/convdiff.cc:75-117. */
void orc_q1_element(int dim, double h, int kind, double coef, const double *beta, double *Ke);

/* Boundary DoFs (ascending).  Returns their count. */
int orc_q1_dirichlet(int dim, int N, int *idx);

/* Full assembly: init_structure (COO->CSR) + add_values per cell in
 * lexicographic cell order + ZeroRows(boundary, 1.0).
 * kcell: per-cell coefficient (N^dim, x fastest) or NULL for coef == 1 (kind 0)
 * or nu (kind 1).  row/col/val must hold n+1 / nnz / nnz entries. */
int orc_q1_assemble(int dim, int N, int kind, const double *kcell, double nu,
                    const double *beta, int *row, int *col, double *val);

/* RHS: i.i.d. uniform[-1,1) on interior DoFs from splitmix64 (53-bit
 * mantissa), 0 on boundary DoFs. */
void orc_q1_rhs(uint64_t seed, int dim, int N, double *b);

/* splitmix64 step and the derived uniform[-1,1) double (used by the RHS). */
uint64_t orc_splitmix64(uint64_t *state);
double orc_uniform_pm1(uint64_t *state);

/* ------------------------------------------------------------------ */
/* CSR construction / assembly (lmatrix_csr_cpu.cc)                    */
/* ------------------------------------------------------------------ */

/* TransformFromCOO: counting sort by row, then per-row selection sort of the
 * columns that swaps values with them.  val_in may be NULL (init_structure);
 * then val_out is left untouched.  Restates lmatrix_csr_cpu.cc:951-1044. */
void orc_coo_to_csr(int n_rows, int nnz, const int *coo_row, const int *coo_col,
                    const double *coo_val, int *row, int *col, double *val);

/* add_values: merge of sorted element columns into a CSR row.
 * Restates lmatrix_csr_cpu.cc:1148-1181. */
void orc_add_values(const int *row, const int *col, double *val,
                    const int *rows, int num_rows, const int *cols, int num_cols,
                    const double *values);

/* ZeroRows: rows in index_set become alpha on the diagonal, 0 elsewhere,
 * structure kept.  Restates lmatrix_csr_cpu.cc:1047-1068. */
void orc_zero_rows(const int *row, const int *col, double *val,
                   const int *index_set, int size, double alpha);

/* ------------------------------------------------------------------ */
/* SpMV and BLAS1 (CPUsimple_csr_lmatrix.cc, CPUsimple_lvector.cc)     */
/* ------------------------------------------------------------------ */

/* y = A x, sequential row sums.  Restates CPUsimple_csr_lmatrix.cc:75-112. */
void orc_spmv_d(int n, const int *row, const int *col, const double *val,
                const double *x, double *y);
void orc_spmv_f(int n, const int *row, const int *col, const float *val,
                const float *x, float *y);
/* y += A x (per-row partial sum added once).  Restates lmatrix_csr_cpu.cc:1352-1375. */
void orc_spmv_add_d(int n, const int *row, const int *col, const double *val,
                    const double *x, double *y);

/* Dot with the reference's unroll-by-5 order.  Restates CPUsimple_lvector.cc:160-209. */
double orc_dot_d(int n, const double *x, const double *y);
float orc_dot_f(int n, const float *x, const float *y);
/* Dot of float vectors accumulated in double (the B200 mixed-precision rule). */
double orc_dot_f_acc_d(int n, const float *x, const float *y);

/* ------------------------------------------------------------------ */
/* Graph analysis and permutation                                      */
/* ------------------------------------------------------------------ */

/* CPU_CSR_lMatrix::Multicoloring (lmatrix_csr_cpu.cc:2175-2290).
 * color_sizes must hold n entries (only ncolors are written); perm[new] = old. */
int orc_multicoloring(int n, const int *row, const int *col,
                      int *ncolors, int *color_sizes, int *perm);

/* CPU_CSR_lMatrix::Levelscheduling (lmatrix_csr_cpu.cc:2295-2392).
 * level_sizes must hold n entries; perm[new] = old.  Returns 0, or -1 when the
 * reference algorithm would not finish (then *nlevels = 0 as in the reference). */
int orc_levelscheduling(int n, const int *row, const int *col,
                        int *nlevels, int *level_sizes, int *perm);

/* Symmetric permutation B = P A P^T with perm[new] = old, rows sorted by column
 * (CPU_CSR_lMatrix::Reorder via COO, lmatrix_csr_cpu.cc:1847-1861 and
 * lmatrix_coo_cpu.cc:1019-1060). */
void orc_reorder_csr(int n, const int *row, const int *col, const double *val,
                     const int *perm, int *row_out, int *col_out, double *val_out);
/* out[i] = in[perm[i]] (CPU_lVector::Reorder, lvector_cpu.cc:75-94). */
void orc_reorder_vec(int n, const double *in, const int *perm, double *out);

/* ------------------------------------------------------------------ */
/* ILU(0)                                                               */
/* ------------------------------------------------------------------ */

/* In-place ILU(0): strictly-lower part holds L (unit diagonal implied), the
 * rest holds U.  Restates lmatrix_csr_cpu.cc:1880-1930. */
void orc_ilu0(int n, const int *row, const int *col, double *val);
/* Natural-order forward (unit L) / backward (U) solve.
 * Restates lmatrix_csr_cpu.cc:2108-2170. */
void orc_ilu_solve(int n, const int *row, const int *col, const double *val,
                   const double *r, double *z);

/* ------------------------------------------------------------------ */
/* Block (colour / level) preconditioners, lpreconditioner_mc*.cc      */
/* ------------------------------------------------------------------ */

/* A block-sweep preconditioner in the permuted numbering: blocks are the
 * colours (MC) or levels (LS); LU is the permuted matrix with intra-block
 * off-diagonals dropped and zeros compressed (lpreconditioner_mc.cc:647-693). */
typedef struct orc_block_precond {
    int n, nblocks;
    int *block_off;        /* nblocks+1 */
    int *perm;             /* perm[new] = old */
    int *row, *col;        /* LU (dropped + compressed) */
    double *val;
    double *Dv, *iDv;      /* scaled as scale_D() of the variant */
    int kind;              /* 0 = SGS (lpreconditioner_mc_sgs.cc), 1 = ILU (lpreconditioner_mc_ilup.cc) */
    double omega;
} orc_block_precond;

/* MC-SGS build (lpreconditioner_mc.cc:157-195 Build with flag_mc, factorize no-op,
 * dropoffs, extract_mat, convert_Dmat2vec, lpreconditioner_mc_sgs.cc:46-59 scale_D)
 * on the natural-order operator.  Also returns the permuted operator (Ap_*), which
 * must hold nnz entries. */
int orc_mcsgs_build(int n, const int *row, const int *col, const double *val, double omega,
                    orc_block_precond *P, int *Ap_row, int *Ap_col, double *Ap_val);

/* ILU(0) build.  mode 0: level scheduling (mc = false, ls = true): ilu0 in natural
 * order, then Levelscheduling of the factors and permute_all.  mode 1: multicolour
 * (mc = true, ls = false): Multicoloring, permute, ilu0 on the permuted matrix.
 * Restates lpreconditioner_mc.cc:157-195 and lpreconditioner_mc_ilup.cc:172-262. */
int orc_ilu0_build(int n, const int *row, const int *col, const double *val, int mode,
                   orc_block_precond *P, int *Ap_row, int *Ap_col, double *Ap_val);

/* Pattern of A^p (MatrixSupSPower, lmatrix_csr_cpu.cc:1520-1664) and ILU(p)
 * (ilup, lmatrix_csr_cpu.cc:1933-2104); outputs allocated, free with orc_free;
 * both return nnz. */
int orc_power_pattern(int n, const int *row, const int *col, int p, int **row_out, int **col_out);
int orc_ilup(int n, const int *row, const int *col, const double *val, int p, int **row_out, int **col_out,
             double **val_out);
void orc_free(void *p);
/* ILU(p) block build (lpreconditioner_mc_ilup.cc:84-194): mode as orc_ilu0_build;
 * the colouring (mode 1) runs on the pattern of A^mat_power. */
int orc_ilup_build(int n, const int *row, const int *col, const double *val, int mode, int ilu_p, int mat_power,
                   orc_block_precond *P, int *Ap_row, int *Ap_col, double *Ap_val);

/* z = M^{-1} r in the permuted numbering (ApplylPreconditioner,
 * lpreconditioner_mc.cc:716-728 with the variant's forward/diagonal/backward). */
void orc_block_apply(const orc_block_precond *P, const double *r, double *z);
void orc_block_free(orc_block_precond *P);

/* ------------------------------------------------------------------ */
/* lVector BLAS1 members beyond the Krylov hot path                    */
/* (lmp/CPUsimple_lvector.cc)                                          */
/* ------------------------------------------------------------------ */

/* ArgMin / ArgMax (:51-92): first index of the smallest / largest |x_i|. */
int orc_iamin(int n, const double *x);
int orc_iamax(int n, const double *x);
/* Norm1 (:95-151): sum |x_i| in the reference's unroll-by-5 order. */
double orc_asum(int n, const double *x);
/* Rot (:448-466): x_i, y_i <- c x_i + s y_i, c y_i - s x_i. */
void orc_rot(int n, double *x, double *y, double c, double s);
/* Rotm (:540-600): the modified Givens rotation param[0..4] (flag, h11, h21,
 * h12, h22) applied to the pairs (y_i, x_i). */
void orc_rotm(int n, double *x, double *y, const double *param);
/* Rotg (:492-535). */
void orc_rotg(double *a, double *b, double *c, double *s);

/* ------------------------------------------------------------------ */
/* Matrix value and structure operations (lmp/lmatrix_csr_cpu.cc)       */
/* ------------------------------------------------------------------ */

/* Scale (:205-212), ScaleOffdiag (:215-224), Zeros (:100-103) of an
 * n-row CSR, values in place: mode 0, 1, 2. */
void orc_csr_scale(int n, const int *row, const int *col, double *val, double alpha, int mode);
/* extract_diagelements / extract_invdiagelements (:2395-2431) of rows
 * [start, end): the last stored diagonal entry of each row (or 1 / it).  A
 * row without one leaves its output untouched, as in the reference. */
void orc_csr_diag(const int *row, const int *col, const double *val, int start, int end, int inverse,
                  double *out);
/* extract_submatrix (:1768-1843): the block [sr, er) x [sc, ec) through
 * init_structure (TransformFromCOO, columns sorted per row) and add_value
 * (each entry added to the first stored entry of its column); mode 0.
 * Compress (:142-202): the entries whose value is not zero, in place order;
 * mode 1.  Outputs allocated (free with orc_free); returns nnz. */
int orc_csr_extract(int n, const int *row, const int *col, const double *val, int mode, int sr, int sc, int er,
                    int ec, int **row_out, int **col_out, double **val_out);

/* ------------------------------------------------------------------ */
/* Krylov solvers (src/linear_solver/*.cc) and IterateControl          */
/* ------------------------------------------------------------------ */

typedef struct orc_control {
    int maxits;
    double abstol, reltol, divtol;
} orc_control;

enum { ORC_ITERATE = 0, ORC_SUCCESS_ABS = 1, ORC_SUCCESS_REL = 2,
       ORC_FAIL_DIV = 3, ORC_FAIL_MAXITS = 4 };

/* IterateControl::Check (src/common/iterate_control.cc:84-110). */
int orc_check(const orc_control *c, int step, double value, double *first_value);

/* Preconditioner callback: z = M^{-1} r. */
typedef void (*orc_precond_fn)(void *ctx, const double *r, double *z);

/* Diagonal (Jacobi) preconditioner context: z = r .* invdiag
 * (lpreconditioner.cc:127-165, extract_invdiagelements lmatrix_csr_cpu.cc:2414-2431). */
typedef struct orc_jacobi { int n; const double *invdiag; } orc_jacobi;
void orc_invdiag(int n, const int *row, const int *col, const double *val, double *invdiag);
void orc_jacobi_apply(void *jacobi_ctx, const double *r, double *z);
/* Adapter for orc_block_apply. */
void orc_block_apply_cb(void *P, const double *r, double *z);

typedef struct orc_result {
    int iters;
    int status;
    double res0, res;
} orc_result;

/* CG<LAD>::SolvePrecond (src/linear_solver/cg.cc:164-248); precond NULL gives
 * SolveNoPrecond (cg.cc:84-160). */
int orc_pcg(int n, const int *row, const int *col, const double *val,
            orc_precond_fn precond, void *ctx, const double *b, double *x,
            const orc_control *ctl, orc_result *res, double *res_hist);

/* GMRES<LAD>::SolveRight with restart m (src/linear_solver/gmres.cc:285-510). */
int orc_gmres(int n, const int *row, const int *col, const double *val,
              orc_precond_fn precond, void *ctx, int m, const double *b, double *x,
              const orc_control *ctl, orc_result *res);

/* Single-precision Jacobi-PCG with float matrix/vectors and double dots
 * (the inner solve of the mixed-precision form). */
int orc_pcg_f32(int n, const int *row, const int *col, const float *val,
                const float *invdiag, const float *b, float *x,
                const orc_control *ctl, orc_result *res);

/* MPIR<LAD_high,LAD_low>::Solve with low-precision Jacobi-CG error correction
 * (src/linear_solver/mpir.cc:69-326).  res0_mode 0: the relative stop uses the
 * initial residual ||b - A x0|| (the stated benchmark criterion); 1: the
 * reference's reset res0_ = res_ after every correction (mpir.cc:274). */
int orc_mpir(int n, const int *row, const int *col, const double *val,
             const double *b, double *x, const orc_control *outer,
             const orc_control *inner, int max_outer, int res0_mode,
             orc_result *res, int *inner_iters_total);

#ifdef __cplusplus
}
#endif
#endif
