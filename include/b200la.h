/*
 * b200la.h -- C ABI of the B200 lmp platform for HiFlow3.
 *
 * The B200 platform is one more lmp ("local multi-platform") backend of
 * HiFlow3's linear algebra.  Its C++ subclasses of lVector<T> / lMatrix<T>
 * and the LinearSolver<LAD> implementations call only the functions below.
 * Plain C types only: every pointer argument is either a host pointer or a
 * device pointer as stated, sizes are ints (the reference's index type,
 * src/linear_algebra/lmp/lmatrix_formats.h:40-45), scalars are doubles.
 *
 * Every function returns a b200la_status (0 = success).  On failure the
 * context keeps a message, b200la_last_error().  Values are computed in the
 * matrix/vector dtype (B200LA_F64 or B200LA_F32); reductions accumulate
 * globally in double.
 *
 * Citations name the reference interface each entry point stands in for
 * (paths relative to the HiFlow3 2.0 source tree).
 */
#ifndef B200LA_H
#define B200LA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B200LA_F64 0
#define B200LA_F32 1

typedef enum {
    B200LA_OK = 0,
    B200LA_ERR_ARG = 1,        /* invalid argument (null, size, dtype) */
    B200LA_ERR_CUDA = 2,       /* a CUDA call failed */
    B200LA_ERR_ALLOC = 3,      /* device or host allocation failed */
    B200LA_ERR_DEVICE = 4,     /* no usable sm_100 device */
    B200LA_ERR_CSR = 5,        /* malformed CSR (non-monotone rows, column out of range) */
    B200LA_ERR_BUDGET = 6,     /* request refused by the serving memory budget */
    B200LA_ERR_TIMEOUT = 7,    /* a bounded device wait gave up */
    B200LA_ERR_SETUP = 8,      /* preconditioner analysis failed (e.g. no colours / levels) */
    B200LA_ERR_NOTFOUND = 9,   /* unknown serving request id */
    B200LA_PENDING = 10,       /* serving request still queued or running */
    B200LA_ERR_IO = 11,        /* a file could not be opened, read or written */
    B200LA_ERR_FORMAT = 12,    /* unsupported or malformed file contents */
    B200LA_ERR_COMM = 13       /* the communicator failed (NCCL error, NCCL absent, a rank that never arrived) */
} b200la_status;

/* IterateControl (src/common/iterate_control.h) */
typedef struct {
    int maxits;
    double abstol, reltol, divtol;
} b200la_control;

/* IterateControl::State of the stop test (src/common/iterate_control.cc:84-110) */
#define B200LA_ITERATE 0
#define B200LA_SUCCESS_ABS 1
#define B200LA_SUCCESS_REL 2
#define B200LA_FAIL_DIV 3
#define B200LA_FAIL_MAXITS 4

typedef struct {
    int iters;          /* Krylov iterations (inner iterations for MPIR) */
    int status;         /* B200LA_SUCCESS_* / B200LA_FAIL_* */
    double res0, res;   /* initial and final residual norm */
    int outer;          /* MPIR outer corrections (0 otherwise) */
    int launches;       /* kernels launched by the solve */
    double solve_ms;    /* device time of the solve */
} b200la_result;

typedef struct b200la_ctx b200la_ctx;
typedef struct b200la_csr b200la_csr;
typedef struct b200la_precond b200la_precond;

/* ---------------------------------------------------------------- context */

/* init_platform_gpu (src/linear_algebra/lmp/cuda/platform_management_gpu.cu:78-171):
 * select `device`, create the platform's stream and reduction scratch. */
int b200la_create(int device, b200la_ctx **out);
int b200la_destroy(b200la_ctx *ctx);
/* Run the context's work on a caller-owned cudaStream_t (NULL: the context's own).
 * Calls without a host result return once their kernels are enqueued on this
 * stream: a device buffer passed to one may be freed or reused by the caller
 * only in this stream's order (after b200la_sync, an event recorded on it,
 * or a stream-ordered free on the same stream). */
int b200la_set_stream(b200la_ctx *ctx, void *cuda_stream);
void *b200la_get_stream(b200la_ctx *ctx);
/* lVector::Sync (src/linear_algebra/lmp/lvector.h:245) */
int b200la_sync(b200la_ctx *ctx);
const char *b200la_last_error(const b200la_ctx *ctx);
const char *b200la_status_string(int status);
int b200la_num_sms(const b200la_ctx *ctx);

/* ----------------------------------------------------------------- memory */

/* memallocdev / memfreedev / memcpy2dev / memcpy2host / memcpydev
 * (src/linear_algebra/lmp/lmp_mem.h:28-88, cuda/mem_cuda.cu:42-107).
 * Copies are ordered on the context's stream; host buffers of the async
 * forms must stay valid until b200la_sync. */
int b200la_malloc(b200la_ctx *ctx, size_t bytes, void **dptr);
int b200la_free(b200la_ctx *ctx, void *dptr);
int b200la_memcpy_h2d(b200la_ctx *ctx, void *dst, const void *src, size_t bytes);
int b200la_memcpy_d2h(b200la_ctx *ctx, void *dst, const void *src, size_t bytes);
int b200la_memcpy_d2d(b200la_ctx *ctx, void *dst, const void *src, size_t bytes);
int b200la_memset_zero(b200la_ctx *ctx, void *dptr, size_t bytes);
/* Page-locked host buffers for asynchronous transfers (memallochost, lmp_mem.h:28-40). */
int b200la_host_alloc(b200la_ctx *ctx, size_t bytes, void **hptr);
int b200la_host_free(b200la_ctx *ctx, void *hptr);
/* Device-time measurement on the context's stream, the CUDA-event counterpart
 * of the ScopedTimer harness (src/tools/ScopedTimer.h:31-163): timer_start
 * records an event, timer_stop records a second one, waits for it and returns
 * the milliseconds between them. */
int b200la_timer_start(b200la_ctx *ctx);
int b200la_timer_stop(b200la_ctx *ctx, double *ms);

/* ----------------------------------------------------------------- matrix */

/* CSR_lMatrix<T>::Init + CopyFrom of a host CPU_CSR_lMatrix
 * (src/linear_algebra/lmp/lmatrix_csr_cpu.cc:106-139; cuda/lmatrix_csr_gpu.cc:85-95).
 * row/col/val are HOST arrays (val of type dtype).  The CSR is validated,
 * uploaded and given its tile schedule (lanes per row from the mean row length). */
int b200la_csr_create(b200la_ctx *ctx, int n_rows, int n_cols, int nnz, const int *row, const int *col,
                      const void *val, int dtype, b200la_csr **out);
/* Same with rows grouped into segments [seg_off[s], seg_off[s+1]) that the
 * schedule never mixes (colours / levels), n_seg segments. */
int b200la_csr_create_segmented(b200la_ctx *ctx, int n_rows, int n_cols, int nnz, const int *row,
                                const int *col, const void *val, int dtype, int n_seg, const int *seg_off,
                                b200la_csr **out);
int b200la_csr_destroy(b200la_csr *A);
/* lMatrix::CastFrom (src/linear_algebra/lmp/lmatrix.h:297-301): device-side copy in dtype. */
int b200la_csr_cast(b200la_ctx *ctx, const b200la_csr *A, int dtype, b200la_csr **out);
int b200la_csr_info(const b200la_csr *A, int *n_rows, int *n_cols, int *nnz, int *dtype, int *lanes_per_row,
                    int *n_tiles, int *n_long_rows);
/* Storage form the SpMV uses: *npat = number of distinct row patterns in the
 * matrix's row-pattern dictionary (0: none), *uses_dict = 1 when SpMV reads
 * the dictionary instead of the explicit column indices, 2 when it reads the
 * stencil layout (row patterns within 3 or 9 bands of three consecutive
 * column offsets: values only, no indices), 3 the half stencil layout
 * (symmetric stencil operators: diagonal and upper half), 4 the lattice
 * layout (an operator or sweep part of a multicolour preconditioner on a
 * parity-coloured structured Q1 grid: values by neighbour slot, no
 * indices). */
int b200la_csr_format(const b200la_csr *A, int *npat, int *uses_dict);
/* lMatrix::CopyTo a host CSR (host arrays, val of the matrix dtype). */
int b200la_csr_download(b200la_ctx *ctx, const b200la_csr *A, int *row, int *col, void *val);
/* New values, same structure (host array of the matrix dtype). */
int b200la_csr_set_values(b200la_ctx *ctx, b200la_csr *A, const void *val);
/* CSR_lMatrix value operations in place on the device; the SpMV layouts
 * follow the new values.  mode B200LA_SCALE_ALL: Scale (every value times
 * alpha, src/linear_algebra/lmp/lmatrix_csr_cpu.cc:205-212);
 * B200LA_SCALE_OFFDIAG: ScaleOffdiag (values with col != row, :215-224);
 * B200LA_SCALE_ZERO: Zeros (every value 0, alpha unused, :100-103). */
enum { B200LA_SCALE_ALL = 0, B200LA_SCALE_OFFDIAG = 1, B200LA_SCALE_ZERO = 2 };
int b200la_csr_scale(b200la_ctx *ctx, b200la_csr *A, double alpha, int mode);
/* extract_diagelements / extract_invdiagelements (lmatrix_csr_cpu.cc:2395-2431)
 * of rows [start, end) into out_dev[0 .. end - start) (device, matrix dtype):
 * the row's last stored diagonal entry, or 1 over it.  A row without one
 * leaves its output untouched (the reference writes an uninitialised value). */
int b200la_csr_diag(b200la_ctx *ctx, const b200la_csr *A, int start, int end, int inverse, void *out_dev);
/* extract_submatrix (lmatrix_csr_cpu.cc:1768-1843): a new matrix holding the
 * block [start_row, end_row) x [start_col, end_col), built as the reference
 * builds it (columns ascending per row; an entry whose column repeats is added
 * into the first one, the repeat left as a stored zero).  Destroy with
 * b200la_csr_destroy.  B200LA_ERR_ARG for an empty or out-of-range block. */
int b200la_csr_extract_submatrix(b200la_ctx *ctx, const b200la_csr *A, int start_row, int start_col, int end_row,
                                 int end_col, b200la_csr **out);
/* Compress (lmatrix_csr_cpu.cc:142-202): a new matrix without the entries
 * whose value is zero, the others in their order.  The reference compresses
 * in place; the caller replaces its handle (and destroys the old one). */
int b200la_csr_compress(b200la_ctx *ctx, const b200la_csr *A, b200la_csr **out);
/* extract_invdiagelements (src/linear_algebra/lmp/lmatrix_csr_cpu.cc:2414-2431): out[i] = 1/a_ii, device. */
int b200la_csr_invdiag(b200la_ctx *ctx, const b200la_csr *A, void *out_dev);

/* ------------------------------------------------------------------- SpMV */

/* lMatrix::VectorMult y = A x (src/linear_algebra/lmp/lmatrix.h:331; GPU
 * cuda/GPUscalar_csr_lmatrix.cu:89-111).  x, y device vectors of A's dtype. */
int b200la_spmv(b200la_ctx *ctx, const b200la_csr *A, const void *x, void *y);
/* lMatrix::VectorMultAdd y += A x (src/linear_algebra/lmp/lmatrix.h:336). */
int b200la_spmv_add(b200la_ctx *ctx, const b200la_csr *A, const void *x, void *y);
/* Fused y = A x and *dot_dev = x . y (device double), as CG's
 * VectorMult + Dot (src/linear_solver/cg.cc:211-212). */
int b200la_spmv_dot(b200la_ctx *ctx, const b200la_csr *A, const void *x, void *y, double *dot_dev);
/* Fused r = b - A x and *nrm_dev = ||r||^2 (cg.cc:200-202: VectorMult, ScaleAdd, Dot). */
int b200la_residual(b200la_ctx *ctx, const b200la_csr *A, const void *b, const void *x, void *r,
                    double *nrm2sq_dev);

/* ------------------------------------------------------- GMG level steps */
/* Geometric-multigrid grid transfers on operators split into a diagonal block
 * (columns of this rank's vectors) and an optional off-diagonal block (columns
 * of the ghost vector; pass NULL on one rank).  Replace the GPU kernels of
 * lmp/cuda/cuda_gmg.h (kernel_gmg_compute_residual / _restriction /
 * _updated_solution, lmp/cuda/cuda_gmg_kernel.h), with and without the
 * off-diagonal block.  Device pointers; the blocks share the dtype and the
 * row count; outputs must not alias inputs (rhs may not be sol). */
/* res = rhs - A_diag sol - A_offdiag sol_ghost */
int b200la_gmg_residual(b200la_ctx *ctx, const b200la_csr *A_diag, const b200la_csr *A_offdiag, const void *sol,
                        const void *rhs, const void *sol_ghost, void *res);
/* res = R_diag tmp + R_offdiag res_ghost (restriction to the coarse level) */
int b200la_gmg_restriction(b200la_ctx *ctx, const b200la_csr *R_diag, const b200la_csr *R_offdiag,
                           const void *tmp, const void *res_ghost, void *res);
/* sol += P_diag res + P_offdiag res_ghost (prolongation of a coarse correction) */
int b200la_gmg_prolongation_add(b200la_ctx *ctx, const b200la_csr *P_diag, const b200la_csr *P_offdiag,
                                const void *res, const void *res_ghost, void *sol);

/* ------------------------------------------------------------------- BLAS1 */

/* lVector::Dot / Norm2 (src/linear_algebra/lmp/lvector.h:266,274; GPU
 * cuda/GPUblas_lvector.cu:204-220).  Result to a HOST double (synchronises). */
int b200la_dot(b200la_ctx *ctx, int dtype, int n, const void *x, const void *y, double *result);
int b200la_nrm2(b200la_ctx *ctx, int dtype, int n, const void *x, double *result);
/* lVector::ArgMin / ArgMax (src/linear_algebra/lmp/CPUsimple_lvector.cc:51-92):
 * the first index of the smallest / largest |x_i| (a NaN is never chosen,
 * except at index 0, as in the reference's scan); NormMax (:154-158): that
 * largest |x_i|; Norm1 (:95-151): sum |x_i| (FP64 tree order).  n >= 1 for
 * the first three.  Results to HOST memory (synchronises). */
int b200la_iamin(b200la_ctx *ctx, int dtype, int n, const void *x, int *result);
int b200la_iamax(b200la_ctx *ctx, int dtype, int n, const void *x, int *result);
int b200la_normmax(b200la_ctx *ctx, int dtype, int n, const void *x, double *result);
int b200la_asum(b200la_ctx *ctx, int dtype, int n, const void *x, double *result);
/* lVector::Rot (:448-466): x_i, y_i <- c x_i + s y_i, c y_i - s x_i, with x
 * the vector the method is called on.  Rotm (:540-600): the modified Givens
 * rotation param[0..4] = (flag, h11, h21, h12, h22) (HOST array) applied to
 * the pairs (y_i, x_i); flag -2 (or any value but -1, 0, 1) changes nothing.
 * Each product and sum rounded on its own, as in the reference. */
int b200la_rot(b200la_ctx *ctx, int dtype, int n, void *x, void *y, double c, double s);
int b200la_rotm(b200la_ctx *ctx, int dtype, int n, void *x, void *y, const double *param);
/* lVector::Rotg (:492-535) on HOST scalars of the dtype. */
int b200la_rotg(int dtype, void *a, void *b, void *c, void *s);
/* lVector::add_values / add_value (src/linear_algebra/lmp/lvector_cpu.cc:114-135):
 * x[indices[k]] += values[k]; lVector::SetValues (lvector_cpu.cc:137-150):
 * x[indices[k]] = values[k].  HOST indices and values (of the dtype), x on the
 * device; a repeated index is applied in the caller's order (added in turn,
 * or the last value kept), as the reference's loops do.  An index outside
 * [0, n) returns B200LA_ERR_ARG before anything is written. */
int b200la_vec_add_values(b200la_ctx *ctx, int dtype, int n, void *x, int length, const int *indices,
                          const void *values);
int b200la_vec_set_values(b200la_ctx *ctx, int dtype, int n, void *x, int length, const int *indices,
                          const void *values);
/* Same, result to a DEVICE double, no synchronisation. */
int b200la_dot_dev(b200la_ctx *ctx, int dtype, int n, const void *x, const void *y, double *result_dev);
/* Dot product x . y written to *result_dev (a DEVICE double) without a
 * context and without allocating any device memory.  No counterpart in the
 * reference: it serves callers that cannot allocate -- an application that
 * owns all device memory through its own pool, or a stream-ordered pipeline
 * in which cudaMalloc (which may synchronise the device) is not allowed after
 * set-up.  Its scratch is a fixed array inside the library (about 135 KB per
 * GPU, held until exit), so n is limited to B200LA_NOALLOC_MAX_N; larger n
 * returns B200LA_ERR_ARG before anything is launched.  stream is a
 * cudaStream_t (NULL: the default stream).  The first call on a device sets up
 * the array's device address and should come before any stream capture; calls
 * whose kernels overlap on the GPU share the array and race.  The address is
 * kept for the life of the process: after cudaDeviceReset on a device, do not
 * call this again on that device.  An error already pending in the CUDA
 * runtime when the call starts is left to the caller (the call returns
 * B200LA_ERR_CUDA and launches nothing); this call's own CUDA failures are
 * cleared and reported by the return code. */
#define B200LA_NOALLOC_MAX_N 67108864
int b200la_dot_noalloc(int dtype, int n, const void *x, const void *y, double *result_dev, void *stream);
/* lVector::Axpy: y += alpha x (lvector.h:283) */
int b200la_axpy(b200la_ctx *ctx, int dtype, int n, double alpha, const void *x, void *y);
/* lVector::ScaleAdd: y = alpha y + x (lvector.h:289) */
int b200la_scaleadd(b200la_ctx *ctx, int dtype, int n, double alpha, const void *x, void *y);
/* lVector::Scale: y *= alpha (lvector.h:278) */
int b200la_scale(b200la_ctx *ctx, int dtype, int n, double alpha, void *y);
/* lVector::ElementWiseMult: y = y .* x (lvector.h:248) */
int b200la_ewmul(b200la_ctx *ctx, int dtype, int n, const void *x, void *y);
/* lVector::CastFrom / CastTo double <-> float (lvector.h:231-235) */
int b200la_cast(b200la_ctx *ctx, int src_dtype, const void *src, int dst_dtype, void *dst, int n);
/* GetIndexedValues / SetIndexedValues (lvector.h:152-160): out[i] = x[idx[i]] / x[idx[i]] = v[i];
 * idx is a device array of n_idx entries, each in [0, size of x). */
int b200la_gather(b200la_ctx *ctx, int dtype, int n_idx, const int *idx_dev, const void *x, void *out);
int b200la_scatter(b200la_ctx *ctx, int dtype, int n_idx, const int *idx_dev, const void *vals, void *x);
/* lVector::Reorder (src/linear_algebra/lmp/lvector_cpu.cc:75-94): out[i] = in[perm[i]], device perm. */
int b200la_permute(b200la_ctx *ctx, int dtype, int n, const int *perm_dev, const void *in, void *out);

/* ------------------------------------------------------- host-side setup */
/* One-time host algorithms, results identical to the reference's. */

/* TransformFromCOO / init_structure (lmatrix_csr_cpu.cc:951-1044, 1101-1121); coo_val may be NULL. */
int b200la_coo_to_csr(int n_rows, int nnz, const int *coo_row, const int *coo_col, const double *coo_val,
                      int *row, int *col, double *val);
/* add_values (lmatrix_csr_cpu.cc:1148-1181) */
int b200la_add_values(const int *row, const int *col, double *val, const int *rows, int num_rows,
                      const int *cols, int num_cols, const double *values);
/* ZeroRows (lmatrix_csr_cpu.cc:1047-1068; via CoupledMatrix::diagonalize_rows, coupled_matrix.cc:550-576) */
int b200la_zero_rows(const int *row, const int *col, double *val, const int *index_set, int size, double alpha);
/* Multicoloring (lmatrix_csr_cpu.cc:2175-2290); sizes holds n entries; perm[new] = old. */
int b200la_multicoloring(int n, const int *row, const int *col, int *ncolors, int *sizes, int *perm);
/* Levelscheduling (lmatrix_csr_cpu.cc:2295-2392); sizes holds n entries; perm[new] = old. */
int b200la_levelscheduling(int n, const int *row, const int *col, int *nlevels, int *sizes, int *perm);
/* Reorder (lmatrix_csr_cpu.cc:1847-1861): B = P A P^T, perm[new] = old. */
int b200la_reorder_csr(int n, const int *row, const int *col, const double *val, const int *perm, int *row_out,
                       int *col_out, double *val_out);
/* ilu0 (lmatrix_csr_cpu.cc:1880-1930), in place on val. */
int b200la_ilu0(int n, const int *row, const int *col, double *val);
/* Two-call convention for a CSR result: *nnz always; the arrays too when
 * row_out is given (row_out n+1, col_out / val_out *nnz entries).
 * MatrixSupSPower (lmatrix_csr_cpu.cc:1641-1664 over MatrixMultSupStructure
 * :1520-1636): the pattern of A^p, p >= 1, columns ascending. */
int b200la_matrix_power_pattern(int n, const int *row, const int *col, int p, int *nnz, int *row_out, int *col_out);
/* ilup (lmatrix_csr_cpu.cc:1933-2104): ILU(p) by levels of fill on the pattern
 * of A^(p+1), keeping the entries of level <= p (unit-lower L strictly below,
 * U with the diagonal, in one CSR).  p = 0 uses the pattern of A itself. */
int b200la_ilup(int n, const int *row, const int *col, const double *val, int p, int *nnz, int *row_out,
                int *col_out, double *val_out);
/* Structured Q1 workloads (lexicographic DoFs; weak forms of
 * examples/poisson/poisson_tutorial.h:152-176 and examples/convection_diffusion/convdiff.cc:75-117):
 * kind 0 Poisson (kcell per cell or NULL), kind 1 convection-diffusion (nu, beta). */
int b200la_q1_sizes(int dim, int N, int *n, int64_t *nnz);
int b200la_q1_assemble(int dim, int N, int kind, const double *kcell, double nu, const double *beta, int *row,
                       int *col, double *val);
int b200la_q1_rhs(uint64_t seed, int dim, int N, double *b);
/* The same CSR (bit-identical values) and right-hand side built on the device
 * on the context's stream: row (n+1), col, val (nnz) and b (n) device arrays,
 * kcell a device array of N^dim cell coefficients or NULL, beta 3 host doubles
 * or NULL.  No counterpart in the reference, which assembles on the host
 * (src/assembly/standard_assembly.cc, coupled_matrix.cc:579-607). */
int b200la_q1_assemble_device(b200la_ctx *ctx, int dim, int N, int kind, const double *kcell, double nu,
                              const double *beta, int *row, int *col, double *val);
int b200la_q1_rhs_device(b200la_ctx *ctx, uint64_t seed, int dim, int N, double *b);

/* --------------------------------------------------------- preconditioners */

#define B200LA_PRECOND_JACOBI 1
#define B200LA_PRECOND_MCSGS 2
#define B200LA_PRECOND_ILU0_LS 3
#define B200LA_PRECOND_ILU0_MC 4

/* lPreconditioner_Jacobi::Build (src/linear_algebra/lmp/lpreconditioner.cc:127-148). */
int b200la_precond_jacobi(b200la_ctx *ctx, const b200la_csr *A, b200la_precond **out);
/* lPreconditioner_MultiColoring_SymmetricGaussSeidel Build (lpreconditioner_mc.cc:157-195,
 * lpreconditioner_mc_sgs.cc:46-59) from the natural-order HOST CSR: colouring, the
 * permuted operator (returned in *A_perm, dtype), dropped L/U sweep matrices and D. */
int b200la_precond_mcsgs(b200la_ctx *ctx, int n, const int *row, const int *col, const double *val,
                         double omega, int dtype, b200la_precond **out, b200la_csr **A_perm);
/* lPreconditioner_MultiColoring_ILUp with ILU(0) (lpreconditioner_mc_ilup.cc:84-262):
 * mode B200LA_PRECOND_ILU0_LS factorises in natural order then level-schedules
 * (mc = false, ls = true); B200LA_PRECOND_ILU0_MC colours first (mc = true). */
int b200la_precond_ilu0(b200la_ctx *ctx, int n, const int *row, const int *col, const double *val, int mode,
                        int dtype, b200la_precond **out, b200la_csr **A_perm);
/* The same with ILU(p) factors (lpreconditioner_mc_ilup.cc:84-194): ilu_p levels
 * of fill; with B200LA_PRECOND_ILU0_MC the colouring runs on the pattern of
 * A^mat_power (build_aux_matrix), with B200LA_PRECOND_ILU0_LS mat_power is 1
 * and the levels come from the factor's pattern.  ilu_p = 0, mat_power = 1 is
 * b200la_precond_ilu0. */
int b200la_precond_ilup(b200la_ctx *ctx, int n, const int *row, const int *col, const double *val, int mode,
                        int ilu_p, int mat_power, int dtype, b200la_precond **out, b200la_csr **A_perm);
/* Permutation (perm[new] = old, host array of n) and block structure
 * (colours or levels; sizes holds n entries). */
int b200la_precond_info(const b200la_precond *P, int *kind, int *n, int *nblocks, int *block_sizes, int *perm);
/* ApplylPreconditioner: z = M^-1 r (device vectors of the preconditioner's dtype). */
int b200la_precond_apply(b200la_ctx *ctx, const b200la_precond *P, const void *r, void *z);
int b200la_precond_destroy(b200la_precond *P);

/* ---------------------------------------------------------------- solvers */

/* CG<LAD>::Solve (src/linear_solver/cg.cc:68-248): P NULL = SolveNoPrecond.
 * b, x device vectors of A's dtype; x holds the start vector and the result.
 * Scalars stay on the device; the host polls the stop state in batches. */
int b200la_cg(b200la_ctx *ctx, const b200la_csr *A, const b200la_precond *P, const void *b, void *x,
              const b200la_control *ctl, b200la_result *res);
/* As b200la_cg, with the residual norm after every iteration written to the
 * host array hist (max hist_len entries). */
int b200la_cg_hist(b200la_ctx *ctx, const b200la_csr *A, const b200la_precond *P, const void *b, void *x,
                   const b200la_control *ctl, b200la_result *res, double *hist, int hist_len);
/* GMRES<LAD>::SolveRight with restart m (src/linear_solver/gmres.cc:285-510). */
int b200la_gmres(b200la_ctx *ctx, const b200la_csr *A, const b200la_precond *P, int m, const void *b, void *x,
                 const b200la_control *ctl, b200la_result *res);
/* MPIR<LAD_high,LAD_low>::Solve (src/linear_solver/mpir.cc:69-326) with an FP32 Jacobi-CG
 * error correction.  A64 is the FP64 operator; A32 (may be NULL: cast here) its FP32 copy.
 * outer->reltol is relative to ||b - A x0||. */
int b200la_mpir(b200la_ctx *ctx, const b200la_csr *A64, const b200la_csr *A32, const double *b, double *x,
                const b200la_control *outer, const b200la_control *inner, int max_outer, b200la_result *res);
/* MPIR<LAD_high, LAD_low>::Solve with a GMRES(m) error correction in FP32
 * (mpir.cc:69-326 with a GMRES<LAD_low> inner solver): A64 and A32 the same
 * operator (in the numbering of P32, e.g. the level-scheduled permutation of
 * an FP32 ILU(0)), P32 an FP32 preconditioner or NULL.  Nonsymmetric systems
 * in the mixed form: FP32 factors and Arnoldi, FP64 outer residual. */
int b200la_mpir_gmres(b200la_ctx *ctx, const b200la_csr *A64, const b200la_csr *A32, const b200la_precond *P32,
                      int m, const double *b, double *x, const b200la_control *outer, const b200la_control *inner,
                      int max_outer, b200la_result *res);

/* Asynchronous block-Jacobi iteration (src/linear_solver/gpu-based/async_iter_gpu.cc:538-943,
 * kernels lmp/cuda/cuda_async_iter_kernels.h): batches of n_block launches,
 * each updating every row n_inner times,
 *   x_i <- D_ii^-1 (b_i - sum_{j != i} A_ij x_j - sum_g O_ig x_ghost_g)
 * (w != 1: x_i <- w * that + (1 - w) x_i), rows reading their neighbours'
 * current values with no barrier, then ||b - A x - O x_ghost|| and
 * IterateControl::Check (iterations counted in sweeps).  A square with a
 * nonzero diagonal; A_offdiag and x_ghost optional (NULL on one rank; the
 * ghost values stay fixed during the call).  The iterates are not reproducible
 * bit for bit (asynchronous by design); the stop decision is. */
int b200la_async_jacobi(b200la_ctx *ctx, const b200la_csr *A, const b200la_csr *A_offdiag, const void *b, void *x,
                        const void *x_ghost, int n_inner, int n_block, double w, const b200la_control *ctl,
                        b200la_result *res);

/* ------------------------------------------------------ row-block coupling */
/* The rows of one rank (n_rows, global column numbers) split into the
 * diagonal block (columns in [col_begin, col_end), shifted to local numbers)
 * and the off-diagonal block (columns numbered by their rank among the distinct
 * ghost columns, ascending), with the ghosts' global numbers: replaces
 * CoupledMatrix::InitStructure (coupled_matrix.cc:253-340) with the ghost
 * numbering of LaCouplings::InitializeCouplings (la_couplings.cc:62-130).
 * Entry order within a row is kept.  Two-call: sizes first (row_d NULL),
 * then row_d/row_o (n_rows + 1), col/val of each block, ghost_global. */
int b200la_rowblock_split(int n_rows, int n_global, const int *row, const int *col, const double *val, int col_begin,
                          int col_end, int *nnz_diag, int *nnz_offdiag, int *n_ghost, int *row_d, int *col_d,
                          double *val_d, int *row_o, int *col_o, double *val_o, int *ghost_global);

/* y += A_offdiag g with every ghost value read from its owner:
 * g[k] = owners[ghost_owner[k]][ghost_index[k]] (device arrays; owners holds
 * device pointers of the matrix dtype, on this GPU or on peer GPUs made
 * accessible with b200la_enable_peer_access).  Replaces the ghost exchange of
 * CoupledVector::UpdateGhost (coupled_vector.cc:975-1128) followed by the
 * off-diagonal product of CoupledMatrix::VectorMult (coupled_matrix.cc:433-467)
 * when the owners' vectors are addressable: no pack, transfer or ghost
 * buffer.  The caller orders the streams (owners' vectors final before, not
 * rewritten until this product has finished). */
int b200la_spmv_add_remote(b200la_ctx *ctx, const b200la_csr *A_offdiag, const void *const *owners_dev,
                           const int *ghost_owner_dev, const int *ghost_index_dev, void *y);
/* Let kernels running on `device` load from `peer_device`'s memory
 * (cudaDeviceEnablePeerAccess; B200LA_ERR_DEVICE when the pair has no peer
 * path).  Same device: nothing to do. */
int b200la_enable_peer_access(int device, int peer_device);

/* Communicator of the ranks of a coupled system, one rank per GPU: replaces
 * the MPI communicator behind CoupledVector / CoupledMatrix (the Isend /
 * Irecv of CoupledVector::SendBorder / ReceiveGhost, coupled_vector.cc:975-1128,
 * and the MPI_Allreduce of CoupledVector::Dot, coupled_vector.cc:331-344).
 * NCCL communicators: rank 0 makes an id with b200la_comm_unique_id (the
 * process's libnccl.so.2, loaded at run time), the caller hands the
 * B200LA_COMM_ID_BYTES bytes to every rank (as HiFlow3 would with
 * MPI_Bcast), and each rank creates its communicator on its context's device
 * (ncclCommInitRank).  Local communicators: b200la_comm_create_local makes
 * nranks communicators for ranks that are host threads of one process (each
 * with its own context, on one GPU or on several); their transfers are
 * device copies ordered by events and the threads meet at a host barrier
 * (60 s limit, then B200LA_ERR_COMM), so no kernel waits for another rank. */
#define B200LA_COMM_ID_BYTES 128
typedef struct b200la_comm b200la_comm;
int b200la_comm_unique_id(void *id);
int b200la_comm_create_nccl(b200la_ctx *ctx, const void *id, int rank, int nranks, b200la_comm **out);
int b200la_comm_create_local(int nranks, b200la_comm **out);
int b200la_comm_info(const b200la_comm *comm, int *rank, int *nranks);
int b200la_comm_destroy(b200la_comm *comm);

/* The coupled operator of one rank: LaCouplings (la_couplings.cc:62-230) plus
 * CoupledMatrix (coupled_matrix.cc:433-467).  diag: the owned rows and
 * columns; offdiag: the owned rows against the ghost columns (NULL when
 * there are none), both as b200la_rowblock_split returns them and kept by
 * the caller while the coupled operator lives.  ghost_offsets (nranks + 1):
 * the ghosts owned by rank q are ghost columns [ghost_offsets[q],
 * ghost_offsets[q+1]); border_offsets (nranks + 1) and border_indices: rank
 * q reads, in that order, the owned rows border_indices[border_offsets[q] ..
 * border_offsets[q+1]) as its ghosts owned here. */
typedef struct b200la_coupled b200la_coupled;
int b200la_coupled_create(b200la_ctx *ctx, b200la_comm *comm, const b200la_csr *diag, const b200la_csr *offdiag,
                          const int *ghost_offsets, const int *border_offsets, const int *border_indices,
                          b200la_coupled **out);
int b200la_coupled_destroy(b200la_coupled *M);
/* CoupledVector::UpdateGhost: the ghost values of x (owned values, device)
 * into ghost (device, n_ghost values; NULL: only the operator's own ghost
 * buffer).  Synchronous. */
int b200la_coupled_update_ghost(b200la_ctx *ctx, b200la_coupled *M, const void *x, void *ghost);
/* CoupledMatrix::VectorMult: y = A x over this rank's rows; the border is
 * packed on the context's stream, exchanged on a second stream while the
 * diagonal block is multiplied, and the off-diagonal block is added after
 * it.  Stream-ordered; every rank calls it. */
int b200la_coupled_spmv(b200la_ctx *ctx, b200la_coupled *M, const void *x, void *y);
/* CoupledVector::Dot: the sum over all ranks of x . y (owned values). */
int b200la_coupled_dot(b200la_ctx *ctx, b200la_coupled *M, const void *x, const void *y, double *out);
/* CG<LAD>::Solve over the coupled operator (cg.cc:164-248), block-Jacobi
 * across ranks: no preconditioner, the Jacobi preconditioner of this rank's
 * diagonal block (b200la_precond_jacobi on diag, as
 * PreconditionerBlockJacobiStand binds op.diagonal()), or a multicolour /
 * ILU preconditioner built on the block's host CSR (b200la_precond_mcsgs,
 * _ilu0, _ilup: r is gathered into its permuted numbering, the sweeps run,
 * z is scattered back -- PreconditionerMultiColoring on op.diagonal()).  The
 * recurrence scalars stay on the device and are reduced across ranks by the
 * communicator; every rank gets the same iteration count and status. */
int b200la_coupled_cg(b200la_ctx *ctx, b200la_coupled *M, const b200la_precond *P, const void *b, void *x,
                      const b200la_control *ctl, b200la_result *res);

/* ---------------------------------------------------------------- file I/O */
/* Host arrays.  MatrixMarket matrices: replaces CPU_CSR_lMatrix::ReadFile / WriteFile
 * (lmp/lmatrix_csr_cpu.cc:1733-1765) over CPU_COO_lMatrix::ReadFile /
 * WriteFile (lmp/lmatrix_coo_cpu.cc:133-299) and lmp/mmio.cc.  Sparse real or
 * integer coordinate files; "symmetric" files are expanded (each off-diagonal
 * entry followed by its mirror), "skew-symmetric" ones read as general, as the
 * reference does.  The CSR is the reference's (TransformFromCOO order).
 * read_info parses the whole file and reports the CSR's sizes; read_csr fills
 * row[n_rows + 1], col[nnz], val[nnz].  The writer emits the reference's text
 * byte for byte, including its "column row value" entry order (a written file
 * read back holds the transpose).  Errors: B200LA_ERR_IO (open/read/write),
 * B200LA_ERR_FORMAT (banner, type, size line or an entry line), B200LA_ERR_CSR
 * (entry index outside the declared size). */
int b200la_mm_read_info(const char *path, int *n_rows, int *n_cols, int *nnz);
int b200la_mm_read_csr(const char *path, int n_rows, int nnz, int *row, int *col, double *val);
int b200la_mm_write_csr(const char *path, int n_rows, int n_cols, int nnz, const int *row, const int *col,
                        const double *val);
/* Plain-text vectors, one value per line: replaces CPU_lVector::ReadFile /
 * WriteFile (lmp/lvector_cpu.cc:582-663), including the reference's count (a
 * last value not followed by a line break is dropped) and its "%e"-style
 * output (std::scientific, 6 digits). */
int b200la_vec_read_info(const char *path, int *n);
int b200la_vec_read(const char *path, int n, double *x);
int b200la_vec_write(const char *path, int n, const double *x);

/* ---------------------------------------------------------------- serving */

/* A continuous-batching solve server; the reference has no counterpart (its
 * solvers run one system at a time, src/linear_solver/cg.cc:68-248).
 * Requests are admitted against a device-memory budget as they arrive, kept
 * resident in HBM (operator, Jacobi diagonal, Krylov state), and every
 * admitted SPD request joins the batch that one CUDA-graph replay advances by
 * iters_per_round iterations; finished requests leave between replays and
 * their memory admits the next.  A system's arithmetic does not depend on the
 * batch it runs in: its result is bit-identical alone and in any mix.
 * Nonsymmetric requests run on a second stream, one at a time (GMRES).
 * Requests start from x0 = 0.  Host arrays named by a request must stay valid
 * until the request has finished. */
typedef struct b200la_server b200la_server;

typedef struct {
    int device;
    double budget_bytes;     /* device bytes resident requests may hold (0: 60e9) */
    int max_slots;           /* resident requests at most (0: 4096) */
    double active_bytes;     /* bytes one batch iteration may stream (0: 4 GiB) */
    int max_active;          /* requests iterated together at most (0: 1024) */
    int iters_per_round;     /* batch iterations per graph replay (0: 16) */
    int autotune;            /* 1: time the kernel shapes on a calibration batch at start */
    int warps;               /* kernel shape when not tuned (0: defaults) */
    int ctas_per_sm;
    int chunks_per_warp;
} b200la_serve_config;

#define B200LA_SERVE_CG 0       /* SPD: Jacobi-PCG (FP64) or FP32 Jacobi-CG inside FP64 defect correction */
#define B200LA_SERVE_GMRES 1    /* nonsymmetric: GMRES(m), FP64, Jacobi or ILU(0) level-scheduled */
#define B200LA_SERVE_F64 0
#define B200LA_SERVE_MIXED 1

typedef struct {
    int method;              /* B200LA_SERVE_CG / B200LA_SERVE_GMRES */
    int precision;           /* B200LA_SERVE_F64 / B200LA_SERVE_MIXED (CG only) */
    /* operator: a host CSR (FP64) ... */
    int n, nnz;
    const int *row, *col;
    const double *val;
    /* ... or, when row is NULL, the structured Q1 system of b200la_q1_assemble
     * assembled on the device (kcell: host array of N^dim coefficients or NULL) */
    int q1_dim, q1_N, q1_kind;
    const double *q1_kcell;
    double q1_nu;
    double q1_beta[3];
    /* right-hand side: host array, or when NULL the Q1 stream of rhs_seed */
    const double *b;
    uint64_t rhs_seed;
    double *x;               /* host result, n doubles */
    b200la_control ctl;      /* CG / GMRES stop test; mixed: the outer defect-correction test */
    b200la_control inner;    /* mixed: the FP32 CG's stop test */
    int max_outer;           /* mixed: corrections at most */
    int gmres_m;             /* GMRES restart length */
    int gmres_precond;       /* B200LA_PRECOND_JACOBI or B200LA_PRECOND_ILU0_LS */
} b200la_request;

typedef struct {
    int status;              /* B200LA_SUCCESS_* / B200LA_FAIL_*, or -B200LA_ERR_* when it failed to run */
    int iters;               /* Krylov iterations (inner iterations in total for mixed) */
    int outer;               /* mixed: corrections */
    double res0, res;        /* first and last residual norm of the stop test */
    double t_submit, t_admit, t_ready, t_done;   /* seconds since the server started */
    double bytes;            /* device bytes the request held */
} b200la_serve_result;

typedef struct {
    long long submitted, completed, failed;
    long long rounds, batch_iters;
    double busy_ms;          /* device time of the graph replays */
    double resident_bytes, peak_resident_bytes;
    int peak_active;
    int warps, ctas_per_sm, chunks_per_warp, iters_per_round;   /* kernel shape in use */
    double active_bytes;
} b200la_serve_info;

int b200la_serve_start(const b200la_serve_config *cfg, b200la_server **out);
/* Queue a request; returns its id.  B200LA_ERR_BUDGET when it could never fit
 * the budget, B200LA_ERR_CSR / B200LA_ERR_ARG for malformed input. */
int b200la_serve_submit(b200la_server *s, const b200la_request *req, long long *id);
/* B200LA_OK with the result once finished, B200LA_PENDING before,
 * B200LA_ERR_NOTFOUND for an unknown id. */
int b200la_serve_poll(b200la_server *s, long long id, b200la_serve_result *res);
/* As poll, waiting up to timeout_s seconds (B200LA_PENDING if still running). */
int b200la_serve_wait(b200la_server *s, long long id, double timeout_s, b200la_serve_result *res);
int b200la_serve_stats(b200la_server *s, b200la_serve_info *out);
/* Finish every queued request, then release the server. */
int b200la_serve_stop(b200la_server *s);

#ifdef __cplusplus
}
#endif
#endif /* B200LA_H */
