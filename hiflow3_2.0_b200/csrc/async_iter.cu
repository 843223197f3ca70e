// async_iter.cu -- asynchronous (chaotic) block-Jacobi iteration on the B200.
//
// The reference's GPU asynchronous iteration (src/linear_solver/gpu-based/
// async_iter_gpu.cc:538-943 with the kernels of lmp/cuda/cuda_async_iter_kernels.h)
// updates every row of its local block n_inner times in a row,
//     x_i <- D_ii^-1 (b_i - sum_{j != i} A_ij x_j - sum_g O_ig x_ghost_g)
// (damped: x_i <- w of that + (1 - w) x_i), each thread reading whatever
// values its neighbours hold at that moment: no barrier between sweeps,
// between rows or between blocks.  The order of the reads is therefore not
// fixed and the iterates are not reproducible bit for bit; what the method
// guarantees (and the tests check) is convergence to the solution of A x = b
// for matrices where Jacobi converges, with the residual test of
// IterateControl::Check between batches of sweeps.
//
// B200 layout: a warp per row for the row sum (lanes stride over the row's
// entries, a shuffle tree folds them), so long rows do not serialise a
// thread; the sweep loop of the row stays inside the warp, as in the
// reference.  Neighbour values are read with ld.global.cg, from L2, where
// other warps' updates land (a plain load could keep serving a stale L1 line).
// The off-diagonal (ghost) part of the row is summed once per launch.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "b200la.h"
#include "b200la_internal.h"
#include "common.cuh"
#include "kernels.cuh"

namespace b200 {
namespace {

constexpr int kAsyncBlock = 256;

template <typename T>
__global__ void __launch_bounds__(kAsyncBlock) async_jacobi_kernel(int n, const int *__restrict__ row,
                                                                   const int *__restrict__ col,
                                                                   const T *__restrict__ val, const int *__restrict__ orow,
                                                                   const int *__restrict__ ocol,
                                                                   const T *__restrict__ oval, const T *__restrict__ xg,
                                                                   const T *__restrict__ invd, const T *__restrict__ b,
                                                                   T *x, int n_inner, T w, int damped)
{
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * kAsyncBlock + threadIdx.x) >> 5, nw = (gridDim.x * kAsyncBlock) >> 5;
    for (int i = gw; i < n; i += nw) {
        const int r0 = row[i], r1 = row[i + 1];
        // c = b - A_offdiag x_ghost (precomputed once, kernel_async_inner_iter)
        T c = T(0);
        if (orow)
            for (int j = orow[i] + lane; j < orow[i + 1]; j += 32) c += oval[j] * xg[ocol[j]];
        c = warp_sum(c);
        c = b[i] - c;
        const T di = invd[i];
        for (int it = 0; it < n_inner; ++it) {
            T s = T(0);
            for (int j = r0 + lane; j < r1; j += 32) {
                const int cj = col[j];
                if (cj != i) s += val[j] * __ldcg(x + cj);
            }
            s = warp_sum(s);
            if (lane == 0) {
                const T xn = di * (c - s);
                __stcg(x + i, damped ? w * xn + (T(1) - w) * __ldcg(x + i) : xn);
            }
            __syncwarp();
        }
    }
}

int status_check(double v, int step, double res0, const b200la_control &c)
{
    // IterateControl::Check (src/common/iterate_control.cc:84-110)
    if (v < c.abstol) return B200LA_SUCCESS_ABS;
    if (v < c.reltol * res0) return B200LA_SUCCESS_REL;
    if (v > c.divtol * res0) return B200LA_FAIL_DIV;
    if (step >= c.maxits) return B200LA_FAIL_MAXITS;
    return B200LA_ITERATE;
}

}  // namespace
}  // namespace b200

using namespace b200;

// ||b - A x - O x_ghost||^2 into *dev (the residual itself into r).
static int async_residual(b200la_ctx *ctx, const b200la_csr *A, const b200la_csr *O, const void *b, const void *x,
                          const void *xg, void *r, double *dev)
{
    SpmvOp op;
    op.epi = EPI_RESID;
    op.fin = O ? FIN_NONE : FIN_STORE;
    op.x = x;
    op.y = r;
    op.b = b;
    op.dot_out = dev;
    int rc = spmv_run(ctx, A, A->all, op);
    if (rc || !O) return rc;
    op.fin = FIN_STORE;
    op.x = xg;
    op.b = r;
    return spmv_run(ctx, O, O->all, op);
}

extern "C" int b200la_async_jacobi(b200la_ctx *ctx, const b200la_csr *A, const b200la_csr *A_offdiag,
                                   const void *b, void *x, const void *x_ghost, int n_inner, int n_block,
                                   double w, const b200la_control *ctl, b200la_result *res)
{
    NvtxScope nvtx_range("b200la_async_jacobi");
    if (!ctx || !A || !b || !x || !ctl || A->n != A->m || n_inner < 1 || n_block < 1 || !(w > 0.0) ||
        (A_offdiag && (!x_ghost || A_offdiag->n != A->n || A_offdiag->dtype != A->dtype)))
        return ctx_fail(ctx, B200LA_ERR_ARG, "async_jacobi: invalid argument", cudaSuccess);
    const int n = A->n, es = A->dtype == B200LA_F64 ? 8 : 4;
    void *work = nullptr;
    const size_t vb = ((size_t)es * n + 255) & ~size_t(255);
    int rc = ctx_work(ctx, 2 * vb + 256, &work);
    if (rc) return rc;
    void *invd = work, *r = static_cast<char *>(work) + vb;
    double *dnorm = reinterpret_cast<double *>(static_cast<char *>(work) + 2 * vb);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, ctx->stream);
    cudaError_t ce = launch_invdiag(A->dtype, n, A->row, A->col, A->val, invd, ctx->stream);
    if (ce != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "async_jacobi: invdiag", ce);
    long long launches = 1;
    auto norm = [&](double *out) -> int {
        int r2 = async_residual(ctx, A, A_offdiag, b, x, x_ghost, r, dnorm);
        if (r2) return r2;
        launches += A_offdiag ? 2 : 1;
        double h = 0.0;
        cudaError_t e = cudaMemcpyAsync(&h, dnorm, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "async_jacobi: residual", e);
        *out = std::sqrt(h);
        return B200LA_OK;
    };
    double res0 = 0.0, rn = 0.0;
    if ((rc = norm(&res0))) return rc;
    rn = res0;
    int iter = 0, status = status_check(res0, 0, res0, *ctl);
    // a warp for every row, as the reference has a thread for every row: all
    // rows of a launch are in flight together as far as the GPU holds them
    const int grid = std::max(1, (n + kAsyncBlock / 32 - 1) / (kAsyncBlock / 32));
    const int damped = w != 1.0;
    while (status == B200LA_ITERATE) {
        // one batch: n_block launches of n_inner asynchronous sweeps (Run / RunDamped)
        for (int k = 0; k < n_block; ++k) {
            if (A->dtype == B200LA_F64)
                async_jacobi_kernel<double><<<grid, kAsyncBlock, 0, ctx->stream>>>(
                    n, A->row, A->col, (const double *)A->val, A_offdiag ? A_offdiag->row : nullptr,
                    A_offdiag ? A_offdiag->col : nullptr, A_offdiag ? (const double *)A_offdiag->val : nullptr,
                    (const double *)x_ghost, (const double *)invd, (const double *)b, (double *)x, n_inner, w,
                    damped);
            else
                async_jacobi_kernel<float><<<grid, kAsyncBlock, 0, ctx->stream>>>(
                    n, A->row, A->col, (const float *)A->val, A_offdiag ? A_offdiag->row : nullptr,
                    A_offdiag ? A_offdiag->col : nullptr, A_offdiag ? (const float *)A_offdiag->val : nullptr,
                    (const float *)x_ghost, (const float *)invd, (const float *)b, (float *)x, n_inner, (float)w,
                    damped);
            ce = cudaGetLastError();
            if (ce != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "async_jacobi: sweep", ce);
            ++launches;
            iter += n_inner;
        }
        if ((rc = norm(&rn))) return rc;
        status = status_check(rn, iter, res0, *ctl);
    }
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->launches += launches;
    if (res) {
        res->iters = iter;
        res->status = status;
        res->res0 = res0;
        res->res = rn;
        res->outer = 0;
        res->launches = (int)launches;
        res->solve_ms = ms;
    }
    return B200LA_OK;
}
