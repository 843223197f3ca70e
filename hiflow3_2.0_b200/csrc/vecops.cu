// vecops.cu -- the lVector BLAS1 members beyond the Krylov hot path, on the
// device: ArgMin / ArgMax, Norm1, NormMax, Rot, Rotm (and Rotg on host
// scalars), as CPUsimple_lVector defines them
// (src/linear_algebra/lmp/CPUsimple_lvector.cc:51-158, 448-600).
//
// ArgMin / ArgMax return the reference's index exactly: the order (|x_i|,
// then i) is total, so the two-level reduction (per CTA, then one CTA over
// the CTA results) finds the first smallest / largest |x_i| whatever the
// grid.  A NaN is never chosen, except at index 0, where the reference's
// scan keeps it (every comparison with it is false).  Rot and Rotm round each
// product and sum separately (no fused multiply-add), as the reference's
// loops do, so they equal it bit for bit.  Norm1 sums |x_i| in FP64 in a
// fixed tree order (the reference sums in unroll-by-5 order): agreement
// within rounding.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <numeric>
#include <vector>

#include "b200la.h"
#include "b200la_internal.h"
#include "common.cuh"

#include <cstring>

namespace b200 {
namespace {

int vgrid(const b200la_ctx *ctx, int n)
{
    const int g = (n + kBlock * 4 - 1) / (kBlock * 4);
    const int cap = ctx->num_sms * 4 < kMaxGrid ? ctx->num_sms * 4 : kMaxGrid;
    return g < 1 ? 1 : (g > cap ? cap : g);
}

template <bool MAX>
__device__ __forceinline__ bool better(double v, int i, double bv, int bi)
{
    return MAX ? (v > bv || (v == bv && i < bi)) : (v < bv || (v == bv && i < bi));
}

// (best |x_i|, its index) of one CTA's grid-strided share; index n = none.
template <bool MAX>
__device__ __forceinline__ void block_best(double &bv, int &bi, int n)
{
    __shared__ double sv[kBlock];
    __shared__ int si[kBlock];
    sv[threadIdx.x] = bv;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int s = kBlock / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            const double ov = sv[threadIdx.x + s];
            const int oi = si[threadIdx.x + s];
            if (oi != n && (si[threadIdx.x] == n || better<MAX>(ov, oi, sv[threadIdx.x], si[threadIdx.x]))) {
                sv[threadIdx.x] = ov;
                si[threadIdx.x] = oi;
            }
        }
        __syncthreads();
    }
    bv = sv[0];
    bi = si[0];
}

template <typename T, bool MAX>
__global__ void __launch_bounds__(kBlock) arg_partial(int n, const T *__restrict__ x, double *part)
{
    double bv = 0.0;
    int bi = n;
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        const double v = fabs((double)x[i]);
        if (v != v) continue;
        if (bi == n || better<MAX>(v, i, bv, bi)) {
            bv = v;
            bi = i;
        }
    }
    block_best<MAX>(bv, bi, n);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = bv;
        part[kMaxGrid + blockIdx.x] = (double)bi;
    }
}

// One CTA: the best of the CTA results; out[0] = index, out[1] = |x_index|.
template <typename T, bool MAX>
__global__ void __launch_bounds__(kBlock) arg_final(int nb, int n, const T *__restrict__ x, const double *part,
                                                    double *out)
{
    double bv = 0.0;
    int bi = n;
    for (int b = threadIdx.x; b < nb; b += kBlock) {
        const int i = (int)part[kMaxGrid + b];
        if (i != n && (bi == n || better<MAX>(part[b], i, bv, bi))) {
            bv = part[b];
            bi = i;
        }
    }
    block_best<MAX>(bv, bi, n);
    if (threadIdx.x == 0) {
        const double x0 = fabs((double)x[0]);
        if (bi == n || x0 != x0) bi = 0;
        out[0] = (double)bi;
        out[1] = fabs((double)x[bi]);
    }
}

template <typename T>
__global__ void __launch_bounds__(kBlock) asum_partial(int n, const T *__restrict__ x, double *part)
{
    __shared__ double sm[kBlock / 32];
    double v[1] = {0.0};
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) v[0] += fabs((double)x[i]);
    block_sum<1>(v, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

__global__ void __launch_bounds__(kBlock) asum_final(int nb, const double *part, double *out)
{
    __shared__ double sm[kBlock / 32];
    double v[1] = {0.0};
    for (int b = threadIdx.x; b < nb; b += kBlock) v[0] += part[b];
    block_sum<1>(v, sm);
    if (threadIdx.x == 0) out[0] = v[0];
}

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }

// Rot: x_i, y_i <- c x_i + s y_i, c y_i - s x_i.
template <typename T>
__global__ void __launch_bounds__(kBlock) rot_kernel(int n, T *x, T *y, T c, T s)
{
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        const T xi = x[i], yi = y[i];
        x[i] = add(mul(c, xi), mul(s, yi));
        y[i] = sub(mul(c, yi), mul(s, xi));
    }
}

// Rotm on the pairs (t1, t2) = (y_i, x_i), flag -1, 0 or 1.
template <typename T>
__global__ void __launch_bounds__(kBlock) rotm_kernel(int n, T *x, T *y, int flag, T h11, T h21, T h12, T h22)
{
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        const T t1 = y[i], t2 = x[i];
        if (flag == -1) {
            y[i] = add(mul(t1, h11), mul(t2, h12));
            x[i] = add(mul(t1, h21), mul(t2, h22));
        } else if (flag == 0) {
            y[i] = add(t1, mul(t2, h12));
            x[i] = add(mul(t1, h21), t2);
        } else {
            y[i] = add(mul(t1, h11), t2);
            x[i] = sub(mul(t2, h22), t1);
        }
    }
}

// Indexed writes with repeated targets in the caller's order: the entries
// come sorted by target (a stable sort, so each target's run keeps the
// caller's order) and one thread walks each run.  add: x_i <- ((x_i + v_1) +
// v_2) ..., as the reference's loop adds; set: the run's last value stays.
template <typename T>
__global__ void __launch_bounds__(kBlock) indexed_runs_kernel(int nruns, const int *__restrict__ run_off,
                                                              const int *__restrict__ idx, const T *__restrict__ v,
                                                              T *x, int add_mode)
{
    for (int r = blockIdx.x * kBlock + threadIdx.x; r < nruns; r += gridDim.x * kBlock) {
        const int b = run_off[r], e = run_off[r + 1], i = idx[b];
        if (add_mode) {
            T a = x[i];
            for (int k = b; k < e; ++k) a = add(a, v[k]);
            x[i] = a;
        } else {
            x[i] = v[e - 1];
        }
    }
}

template <typename T>
void rotg_host(T *a, T *b, T *c, T *s)
{
    const T ta = std::fabs(*a), tb = std::fabs(*b);
    const T roe = ta > tb ? *a : *b;
    const T scal = ta + tb;
    if (scal == 0) {
        *c = 1;
        *s = *a = *b = 0;
        return;
    }
    const T t0 = ta / scal, t1 = tb / scal;
    T r = scal * std::sqrt(t0 * t0 + t1 * t1);
    if (roe < 0) r = -r;
    *c = *a / r;
    *s = *b / r;
    T z;
    if (ta > tb) z = *s;
    else if (*c != 0) z = 1 / *c;
    else z = 1;
    *a = r;
    *b = z;
}

}  // namespace
}  // namespace b200

using namespace b200;

#define VCK(call)                                                                     \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, #call, e_);      \
    } while (0)

static bool vdt(int dtype) { return dtype == B200LA_F64 || dtype == B200LA_F32; }

// index and |x_index| of ArgMin (MAX false) / ArgMax (MAX true) into dscal[0..1]
template <bool MAX>
static int arg_run(b200la_ctx *ctx, int dtype, int n, const void *x)
{
    const int g = vgrid(ctx, n);
    if (dtype == B200LA_F64) {
        arg_partial<double, MAX><<<g, kBlock, 0, ctx->stream>>>(n, (const double *)x, ctx->partials);
        arg_final<double, MAX><<<1, kBlock, 0, ctx->stream>>>(g, n, (const double *)x, ctx->partials, ctx->dscal);
    } else {
        arg_partial<float, MAX><<<g, kBlock, 0, ctx->stream>>>(n, (const float *)x, ctx->partials);
        arg_final<float, MAX><<<1, kBlock, 0, ctx->stream>>>(g, n, (const float *)x, ctx->partials, ctx->dscal);
    }
    VCK(cudaGetLastError());
    VCK(cudaMemcpyAsync(ctx->hscal, ctx->dscal, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    VCK(cudaStreamSynchronize(ctx->stream));
    ctx->launches += 2;
    return B200LA_OK;
}

extern "C" int b200la_iamin(b200la_ctx *ctx, int dtype, int n, const void *x, int *result)
{
    if (!ctx || !vdt(dtype) || n < 1 || !x || !result) return B200LA_ERR_ARG;
    const int rc = arg_run<false>(ctx, dtype, n, x);
    if (!rc) *result = (int)ctx->hscal[0];
    return rc;
}

extern "C" int b200la_iamax(b200la_ctx *ctx, int dtype, int n, const void *x, int *result)
{
    if (!ctx || !vdt(dtype) || n < 1 || !x || !result) return B200LA_ERR_ARG;
    const int rc = arg_run<true>(ctx, dtype, n, x);
    if (!rc) *result = (int)ctx->hscal[0];
    return rc;
}

extern "C" int b200la_normmax(b200la_ctx *ctx, int dtype, int n, const void *x, double *result)
{
    if (!ctx || !vdt(dtype) || n < 1 || !x || !result) return B200LA_ERR_ARG;
    const int rc = arg_run<true>(ctx, dtype, n, x);
    if (!rc) *result = ctx->hscal[1];
    return rc;
}

extern "C" int b200la_asum(b200la_ctx *ctx, int dtype, int n, const void *x, double *result)
{
    if (!ctx || !vdt(dtype) || n < 0 || (n && !x) || !result) return B200LA_ERR_ARG;
    const int g = vgrid(ctx, n);
    if (dtype == B200LA_F64) asum_partial<double><<<g, kBlock, 0, ctx->stream>>>(n, (const double *)x, ctx->partials);
    else asum_partial<float><<<g, kBlock, 0, ctx->stream>>>(n, (const float *)x, ctx->partials);
    asum_final<<<1, kBlock, 0, ctx->stream>>>(g, ctx->partials, ctx->dscal);
    VCK(cudaGetLastError());
    VCK(cudaMemcpyAsync(ctx->hscal, ctx->dscal, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    VCK(cudaStreamSynchronize(ctx->stream));
    ctx->launches += 2;
    *result = ctx->hscal[0];
    return B200LA_OK;
}

extern "C" int b200la_rot(b200la_ctx *ctx, int dtype, int n, void *x, void *y, double c, double s)
{
    if (!ctx || !vdt(dtype) || n < 0 || (n && (!x || !y)) || x == y) return B200LA_ERR_ARG;
    if (!n) return B200LA_OK;
    const int g = vgrid(ctx, n);
    if (dtype == B200LA_F64) rot_kernel<double><<<g, kBlock, 0, ctx->stream>>>(n, (double *)x, (double *)y, c, s);
    else rot_kernel<float><<<g, kBlock, 0, ctx->stream>>>(n, (float *)x, (float *)y, (float)c, (float)s);
    VCK(cudaGetLastError());
    ctx->launches += 1;
    return B200LA_OK;
}

extern "C" int b200la_rotm(b200la_ctx *ctx, int dtype, int n, void *x, void *y, const double *param)
{
    if (!ctx || !vdt(dtype) || n < 0 || (n && (!x || !y)) || x == y || !param) return B200LA_ERR_ARG;
    const double f = param[0];
    if (!n || !(f == -1.0 || f == 0.0 || f == 1.0)) return B200LA_OK;   // flag -2 (or any other): no change
    const int g = vgrid(ctx, n), flag = (int)f;
    if (dtype == B200LA_F64)
        rotm_kernel<double><<<g, kBlock, 0, ctx->stream>>>(n, (double *)x, (double *)y, flag, param[1], param[2],
                                                           param[3], param[4]);
    else
        rotm_kernel<float><<<g, kBlock, 0, ctx->stream>>>(n, (float *)x, (float *)y, flag, (float)param[1],
                                                          (float)param[2], (float)param[3], (float)param[4]);
    VCK(cudaGetLastError());
    ctx->launches += 1;
    return B200LA_OK;
}

extern "C" int b200la_rotg(int dtype, void *a, void *b, void *c, void *s)
{
    if (!vdt(dtype) || !a || !b || !c || !s) return B200LA_ERR_ARG;
    if (dtype == B200LA_F64) rotg_host((double *)a, (double *)b, (double *)c, (double *)s);
    else rotg_host((float *)a, (float *)b, (float *)c, (float *)s);
    return B200LA_OK;
}

// x[indices[k]] (+)= values[k], k = 0 .. length - 1, host indices and values
// (of the dtype), in the caller's order for repeated indices.
static int indexed_write(b200la_ctx *ctx, int dtype, int n, void *x, int length, const int *indices,
                         const void *values, int add_mode)
{
    if (!ctx || !vdt(dtype) || n < 0 || length < 0 || (length && (!x || !indices || !values)))
        return B200LA_ERR_ARG;
    for (int k = 0; k < length; ++k)
        if (indices[k] < 0 || indices[k] >= n) return B200LA_ERR_ARG;
    if (!length) return B200LA_OK;
    const size_t es = dtype == B200LA_F64 ? 8 : 4;
    std::vector<int> ord(length);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return indices[a] < indices[b]; });
    std::vector<int> sidx(length), off;
    std::vector<char> sval(es * length);
    off.reserve(length + 1);
    for (int k = 0; k < length; ++k) {
        sidx[k] = indices[ord[k]];
        std::memcpy(sval.data() + es * k, static_cast<const char *>(values) + es * ord[k], es);
        if (k == 0 || sidx[k] != sidx[k - 1]) off.push_back(k);
    }
    const int nruns = (int)off.size();
    off.push_back(length);
    const size_t b_idx = ((size_t)4 * length + 255) & ~size_t(255), b_off = ((size_t)4 * (nruns + 1) + 255) & ~size_t(255);
    void *work = nullptr;
    const int rc = ctx_work(ctx, b_idx + b_off + es * length, &work);
    if (rc) return rc;
    int *d_idx = static_cast<int *>(work);
    int *d_off = reinterpret_cast<int *>(static_cast<char *>(work) + b_idx);
    void *d_val = static_cast<char *>(work) + b_idx + b_off;
    VCK(cudaMemcpyAsync(d_idx, sidx.data(), 4 * (size_t)length, cudaMemcpyHostToDevice, ctx->stream));
    VCK(cudaMemcpyAsync(d_off, off.data(), 4 * (size_t)(nruns + 1), cudaMemcpyHostToDevice, ctx->stream));
    VCK(cudaMemcpyAsync(d_val, sval.data(), es * length, cudaMemcpyHostToDevice, ctx->stream));
    const int g = std::max(1, std::min((nruns + kBlock - 1) / kBlock, ctx->num_sms * 8));
    if (dtype == B200LA_F64)
        indexed_runs_kernel<double><<<g, kBlock, 0, ctx->stream>>>(nruns, d_off, d_idx, (const double *)d_val,
                                                                   (double *)x, add_mode);
    else
        indexed_runs_kernel<float><<<g, kBlock, 0, ctx->stream>>>(nruns, d_off, d_idx, (const float *)d_val,
                                                                  (float *)x, add_mode);
    VCK(cudaGetLastError());
    // the host arrays above go out of scope: the copies from them must be done
    VCK(cudaStreamSynchronize(ctx->stream));
    ctx->launches += 1;
    return B200LA_OK;
}

extern "C" int b200la_vec_add_values(b200la_ctx *ctx, int dtype, int n, void *x, int length, const int *indices,
                                     const void *values)
{
    return indexed_write(ctx, dtype, n, x, length, indices, values, 1);
}

extern "C" int b200la_vec_set_values(b200la_ctx *ctx, int dtype, int n, void *x, int length, const int *indices,
                                     const void *values)
{
    return indexed_write(ctx, dtype, n, x, length, indices, values, 0);
}
