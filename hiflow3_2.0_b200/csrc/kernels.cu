// kernels.cu -- BLAS1 and Krylov-step kernels of the B200 lmp platform
// (the CSR SpMV kernels are in spmv.cu).
#include "common.cuh"
#include "kernels.cuh"

#include <cstdlib>

#include <cmath>

namespace b200 {


namespace {

// ------------------------------------------------------------------ BLAS1

// 16-byte vectors: 2 doubles or 4 floats per load / store.
template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
    using type = double2;
    static constexpr int W = 2;
};
template <>
struct Vec16<float> {
    using type = float4;
    static constexpr int W = 4;
};


// Grid of the streaming BLAS1 / Krylov-update kernels: at most four CTAs per
// SM, so each thread strides over several 16-byte vectors and the last CTA's
// reduction sums fewer partials (3-D 128^3 mixed solve: 35.1 ms against 35.6 ms
// with eight per SM; two per SM slowed the FP64 updates).
inline int stream_grid(const Scratch *s, int n, int per_thread = 4)
{
    int g = (n + kBlock * per_thread - 1) / (kBlock * per_thread);
    const int cap = (s ? s->num_sms : 148) * 4;
    if (g > cap) g = cap;
    if (g > kMaxGrid) g = kMaxGrid;
    return g < 1 ? 1 : g;
}

template <typename T>
__global__ void __launch_bounds__(kBlock) dot_kernel(int n, const T *__restrict__ x, const T *__restrict__ y,
                                                     double *out, bool sqrt_out, const int *gate, Scratch sc)
{
    if (gate_closed(gate)) return;
    using V = typename Vec16<T>::type;
    constexpr int W = Vec16<T>::W;
    const int tid = blockIdx.x * kBlock + threadIdx.x, stride = gridDim.x * kBlock;
    double a = 0.0;
    const bool vec = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0;
    const int nv = vec ? n / W : 0;
    for (int iv = tid; iv < nv; iv += stride) {
        const V xv = __ldg(reinterpret_cast<const V *>(x) + iv), yv = __ldg(reinterpret_cast<const V *>(y) + iv);
        const T *xe = reinterpret_cast<const T *>(&xv), *ye = reinterpret_cast<const T *>(&yv);
        T s = T(0);
#pragma unroll
        for (int k = 0; k < W; ++k) s += xe[k] * ye[k];
        a += (double)s;
    }
    for (int i = nv * W + tid; i < n; i += stride) a += (double)(x[i] * y[i]);
    double v[1] = {a}, o[1];
    if (grid_reduce<1>(v, sc.partials, sc.ticket, o)) *out = sqrt_out ? sqrt(o[0]) : o[0];
}

template <typename T>
__global__ void axpy_kernel(int n, T a, const T *__restrict__ x, T *__restrict__ y)
{
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) y[i] += a * x[i];
}

template <typename T>
__global__ void scaleadd_kernel(int n, T a, const T *__restrict__ x, T *__restrict__ y)
{
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) y[i] = a * y[i] + x[i];
}

template <typename T>
__global__ void scale_kernel(int n, T a, T *__restrict__ y)
{
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) y[i] *= a;
}

template <typename T>
__global__ void fill_kernel(int n, T a, T *__restrict__ y)
{
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) y[i] = a;
}

template <typename T>
__global__ void ewmul_kernel(int n, const T *__restrict__ x, T *__restrict__ y)
{
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) y[i] *= x[i];
}

template <typename S, typename D>
__global__ void cast_kernel(int n, const S *__restrict__ s, D *__restrict__ d)
{
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) d[i] = (D)s[i];
}

template <typename T>
__global__ void gather_kernel(int n, const int *__restrict__ idx, const T *__restrict__ x, T *__restrict__ out)
{
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) out[i] = x[idx[i]];
}

template <typename T>
__global__ void scatter_kernel(int n, const int *__restrict__ idx, const T *__restrict__ v, T *__restrict__ x)
{
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) x[idx[i]] = v[i];
}

// ------------------------------------------------------------------ Krylov

// x += alpha p; r -= alpha Ap; rr += r^2 and (Jacobi) rz += r (invd r) for
// element i, partial sums of one 16-byte vector kept in T, then folded to double.
template <typename T>
__device__ __forceinline__ void cg_update_elem(T alpha, T &x, T &r, T p, T ap, T d, bool jac, T &rr, T &rz)
{
    x += alpha * p;
    r -= alpha * ap;
    rr += r * r;
    if (jac) rz += r * (r * d);
}

// COND: the last CTA also sets the conditional handle cond (a kernel with the
// device-side graph call is a separate instance: profilers replay only the
// plain one, which the host-polled batches use)
template <typename T, bool COND>
__global__ void __launch_bounds__(kBlock) cg_update_kernel(int n, int precond, T *__restrict__ x, T *__restrict__ r,
                                                           const T *__restrict__ p, const T *__restrict__ Ap,
                                                           const T *__restrict__ invd, DevState *st, Scratch sc,
                                                           unsigned long long cond)
{
    if (gate_closed(&st->status)) return;
    using V = typename Vec16<T>::type;
    constexpr int W = Vec16<T>::W;
    const T alpha = (T)cta_scalar(&st->alpha);
    const bool jac = precond == 1;
    double rr = 0.0, rz = 0.0;
    const uintptr_t al = reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(r) |
                         reinterpret_cast<uintptr_t>(p) | reinterpret_cast<uintptr_t>(Ap) |
                         (jac ? reinterpret_cast<uintptr_t>(invd) : 0);
    const int nv = (al & 15) ? 0 : n / W;
    const int tid = blockIdx.x * kBlock + threadIdx.x, stride = gridDim.x * kBlock;
    for (int iv = tid; iv < nv; iv += stride) {
        V xv = reinterpret_cast<const V *>(x)[iv], rv = reinterpret_cast<const V *>(r)[iv];
        const V pv = reinterpret_cast<const V *>(p)[iv], av = __ldcs(reinterpret_cast<const V *>(Ap) + iv);
        V dv = pv;
        if (jac) dv = __ldg(reinterpret_cast<const V *>(invd) + iv);
        T *xe = reinterpret_cast<T *>(&xv), *re = reinterpret_cast<T *>(&rv);
        const T *pe = reinterpret_cast<const T *>(&pv), *ae = reinterpret_cast<const T *>(&av),
                *de = reinterpret_cast<const T *>(&dv);
        T prr = T(0), prz = T(0);
#pragma unroll
        for (int k = 0; k < W; ++k) cg_update_elem(alpha, xe[k], re[k], pe[k], ae[k], de[k], jac, prr, prz);
        reinterpret_cast<V *>(x)[iv] = xv;
        reinterpret_cast<V *>(r)[iv] = rv;
        rr += (double)prr;
        rz += (double)prz;
    }
    for (int i = nv * W + tid; i < n; i += stride) {
        T xi = x[i], ri = r[i], prr = T(0), prz = T(0);
        cg_update_elem(alpha, xi, ri, p[i], Ap[i], jac ? invd[i] : T(0), jac, prr, prz);
        x[i] = xi;
        r[i] = ri;
        rr += (double)prr;
        rz += (double)prz;
    }
    double v[2] = {rr, rz}, o[2];
    if (grid_reduce<2>(v, sc.partials, sc.ticket, o)) {
        const int it = st->iter + 1;
        st->iter = it;
        st->rr = o[0];
        const double res = sqrt(o[0]);
        st->res = res;
        if (st->hist && it < st->hist_len) st->hist[it] = res;
        const int status = check_state(st, it, res);
        st->status = status;
        if (status == kIterate && precond != 2) {
            const double g = (precond == 1) ? o[1] : o[0];
            st->beta = g / st->rho;
            st->rho = g;
        }
        if constexpr (COND) cudaGraphSetConditional((cudaGraphConditionalHandle)cond, status == kIterate ? 1u : 0u);
    }
}

template <typename T>
__global__ void cg_pupdate_kernel(int n, int precond, T *__restrict__ p, const T *__restrict__ r,
                                  const T *__restrict__ invd, const T *__restrict__ z, DevState *st)
{
    if (gate_closed(&st->status)) return;
    using V = typename Vec16<T>::type;
    constexpr int W = Vec16<T>::W;
    const T beta = (T)cta_scalar(&st->beta);
    const uintptr_t al = reinterpret_cast<uintptr_t>(p) | reinterpret_cast<uintptr_t>(precond == 2 ? z : r) |
                         (precond == 1 ? reinterpret_cast<uintptr_t>(invd) : 0);
    const int nv = (al & 15) ? 0 : n / W;
    const int tid = blockIdx.x * kBlock + threadIdx.x, stride = gridDim.x * kBlock;
    for (int iv = tid; iv < nv; iv += stride) {
        V pv = reinterpret_cast<const V *>(p)[iv];
        const V rv = reinterpret_cast<const V *>(precond == 2 ? z : r)[iv];
        V dv = rv;
        if (precond == 1) dv = __ldg(reinterpret_cast<const V *>(invd) + iv);
        T *pe = reinterpret_cast<T *>(&pv);
        const T *re = reinterpret_cast<const T *>(&rv), *de = reinterpret_cast<const T *>(&dv);
#pragma unroll
        for (int k = 0; k < W; ++k) pe[k] = precond == 1 ? cg_direction(beta, pe[k], re[k], de[k]) : beta * pe[k] + re[k];
        reinterpret_cast<V *>(p)[iv] = pv;
    }
    for (int i = nv * W + tid; i < n; i += stride) {
        if (precond == 1) {
            p[i] = cg_direction(beta, p[i], r[i], invd[i]);
            continue;
        }
        const T zi = precond == 0 ? r[i] : z[i];
        p[i] = beta * p[i] + zi;
    }
}

template <typename T>
__global__ void __launch_bounds__(kBlock) cg_start_kernel(int n, int precond, const T *__restrict__ r,
                                                          const T *__restrict__ invd, const T *__restrict__ z,
                                                          T *__restrict__ p, DevState *st, Scratch sc)
{
    double a = 0.0;
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        const T ri = r[i];
        const T zi = (precond == 1) ? ri * invd[i] : (precond == 0 ? ri : z[i]);
        p[i] = zi;
        a += (double)(ri * zi);
    }
    double v[1] = {a}, o[1];
    if (grid_reduce<1>(v, sc.partials, sc.ticket, o)) st->rho = o[0];
}

template <typename T>
__global__ void __launch_bounds__(kBlock) cg_rz_kernel(int n, const T *__restrict__ r, const T *__restrict__ z,
                                                       DevState *st, Scratch sc)
{
    if (gate_closed(&st->status)) return;
    double a = 0.0;
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) a += (double)(r[i] * z[i]);
    double v[1] = {a}, o[1];
    if (grid_reduce<1>(v, sc.partials, sc.ticket, o)) {
        st->rz = o[0];
        st->beta = o[0] / st->rho;
        st->rho = o[0];
    }
}

__global__ void cast_residual_kernel(int n, const double *__restrict__ r, float *__restrict__ rl,
                                     float *__restrict__ xl)
{
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        rl[i] = (float)r[i];
        xl[i] = 0.0f;
    }
}

__global__ void add_correction_kernel(int n, const float *__restrict__ cl, double *__restrict__ x)
{
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) x[i] += (double)cl[i];
}

template <typename T>
__global__ void axpy_dev_kernel(int n, const double *coef, double sign, const T *__restrict__ x, T *__restrict__ y,
                                const int *gate)
{
    if (gate_closed(gate)) return;
    const T a = (T)(sign * cta_scalar(coef));
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) y[i] += a * x[i];
}

template <typename T>
__global__ void scale_dev_kernel(int n, const double *coef, bool reciprocal, const T *__restrict__ x,
                                 T *__restrict__ y, const int *gate)
{
    if (gate_closed(gate)) return;
    const double cv = cta_scalar(coef);
    const T a = (T)(reciprocal ? 1.0 / cv : cv);
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) y[i] = a * x[i];
}

}  // namespace

#define B200_DISPATCH(dtype, ...)                 \
    do {                                          \
        if ((dtype) == 0) {                       \
            using T = double;                     \
            __VA_ARGS__;                          \
        } else {                                  \
            using T = float;                      \
            __VA_ARGS__;                          \
        }                                         \
    } while (0)

cudaError_t launch_dot(const Scratch &s, int dtype, int n, const void *x, const void *y, double *out, bool sqrt_out,
                       cudaStream_t st)
{
    const int g = stream_grid(&s, n);
    B200_DISPATCH(dtype, dot_kernel<T><<<g, kBlock, 0, st>>>(n, (const T *)x, (const T *)y, out, sqrt_out,
                                                             nullptr, s));
    return cudaGetLastError();
}

cudaError_t launch_dot_to(const Scratch &s, int dtype, int n, const void *x, const void *y, double *out,
                          const int *gate, cudaStream_t st)
{
    const int g = stream_grid(&s, n);
    B200_DISPATCH(dtype, dot_kernel<T><<<g, kBlock, 0, st>>>(n, (const T *)x, (const T *)y, out, false, gate, s));
    return cudaGetLastError();
}

cudaError_t launch_dot_norm_to(const Scratch &s, int dtype, int n, const void *x, double *out, const int *gate,
                               cudaStream_t st)
{
    const int g = stream_grid(&s, n);
    B200_DISPATCH(dtype, dot_kernel<T><<<g, kBlock, 0, st>>>(n, (const T *)x, (const T *)x, out, true, gate, s));
    return cudaGetLastError();
}

cudaError_t launch_axpy(int dtype, int n, double a, const void *x, void *y, cudaStream_t st)
{
    B200_DISPATCH(dtype, axpy_kernel<T><<<stream_grid(nullptr, n), kBlock, 0, st>>>(n, (T)a, (const T *)x, (T *)y));
    return cudaGetLastError();
}

cudaError_t launch_scaleadd(int dtype, int n, double a, const void *x, void *y, cudaStream_t st)
{
    B200_DISPATCH(dtype,
                  scaleadd_kernel<T><<<stream_grid(nullptr, n), kBlock, 0, st>>>(n, (T)a, (const T *)x, (T *)y));
    return cudaGetLastError();
}

cudaError_t launch_scale(int dtype, int n, double a, void *y, cudaStream_t st)
{
    B200_DISPATCH(dtype, scale_kernel<T><<<stream_grid(nullptr, n), kBlock, 0, st>>>(n, (T)a, (T *)y));
    return cudaGetLastError();
}

cudaError_t launch_fill(int dtype, int n, double v, void *y, cudaStream_t st)
{
    B200_DISPATCH(dtype, fill_kernel<T><<<stream_grid(nullptr, n), kBlock, 0, st>>>(n, (T)v, (T *)y));
    return cudaGetLastError();
}

cudaError_t launch_ewmul(int dtype, int n, const void *x, void *y, cudaStream_t st)
{
    B200_DISPATCH(dtype, ewmul_kernel<T><<<stream_grid(nullptr, n), kBlock, 0, st>>>(n, (const T *)x, (T *)y));
    return cudaGetLastError();
}

cudaError_t launch_cast(int src_dtype, const void *src, int dst_dtype, void *dst, int n, cudaStream_t st)
{
    const int g = stream_grid(nullptr, n);
    if (src_dtype == 0 && dst_dtype == 1) cast_kernel<double, float><<<g, kBlock, 0, st>>>(n, (const double *)src, (float *)dst);
    else if (src_dtype == 1 && dst_dtype == 0) cast_kernel<float, double><<<g, kBlock, 0, st>>>(n, (const float *)src, (double *)dst);
    else if (src_dtype == 0) cast_kernel<double, double><<<g, kBlock, 0, st>>>(n, (const double *)src, (double *)dst);
    else cast_kernel<float, float><<<g, kBlock, 0, st>>>(n, (const float *)src, (float *)dst);
    return cudaGetLastError();
}

cudaError_t launch_gather(int dtype, int n, const int *idx, const void *x, void *out, cudaStream_t st)
{
    B200_DISPATCH(dtype, gather_kernel<T><<<stream_grid(nullptr, n), kBlock, 0, st>>>(n, idx, (const T *)x, (T *)out));
    return cudaGetLastError();
}

cudaError_t launch_scatter(int dtype, int n, const int *idx, const void *vals, void *x, cudaStream_t st)
{
    B200_DISPATCH(dtype,
                  scatter_kernel<T><<<stream_grid(nullptr, n), kBlock, 0, st>>>(n, idx, (const T *)vals, (T *)x));
    return cudaGetLastError();
}

cudaError_t launch_cg_update(const Scratch &s, int dtype, int n, int precond, void *x, void *r, const void *p,
                             const void *Ap, const void *invd, DevState *st, cudaStream_t stm,
                             unsigned long long cond)
{
    const int g = stream_grid(&s, n);
    if (cond)
        B200_DISPATCH(dtype, cg_update_kernel<T, true><<<g, kBlock, 0, stm>>>(n, precond, (T *)x, (T *)r, (const T *)p,
                                                                          (const T *)Ap, (const T *)invd, st, s, cond));
    else
        B200_DISPATCH(dtype, cg_update_kernel<T, false><<<g, kBlock, 0, stm>>>(
                                 n, precond, (T *)x, (T *)r, (const T *)p, (const T *)Ap, (const T *)invd, st, s, 0ull));
    return cudaGetLastError();
}

cudaError_t launch_cg_pupdate(int dtype, int n, int precond, void *p, const void *r, const void *invd, const void *z,
                              DevState *st, cudaStream_t stm)
{
    B200_DISPATCH(dtype, cg_pupdate_kernel<T><<<stream_grid(nullptr, n), kBlock, 0, stm>>>(
                             n, precond, (T *)p, (const T *)r, (const T *)invd, (const T *)z, st));
    return cudaGetLastError();
}

cudaError_t launch_cg_start(const Scratch &s, int dtype, int n, int precond, const void *r, const void *invd,
                            const void *z, void *p, DevState *st, cudaStream_t stm)
{
    const int g = stream_grid(&s, n);
    B200_DISPATCH(dtype, cg_start_kernel<T><<<g, kBlock, 0, stm>>>(n, precond, (const T *)r, (const T *)invd,
                                                                   (const T *)z, (T *)p, st, s));
    return cudaGetLastError();
}

cudaError_t launch_cg_rz(const Scratch &s, int dtype, int n, const void *r, const void *z, DevState *st,
                         cudaStream_t stm)
{
    const int g = stream_grid(&s, n);
    B200_DISPATCH(dtype, cg_rz_kernel<T><<<g, kBlock, 0, stm>>>(n, (const T *)r, (const T *)z, st, s));
    return cudaGetLastError();
}

cudaError_t launch_cast_residual(int n, const double *r, float *rl, float *xl, cudaStream_t st)
{
    cast_residual_kernel<<<stream_grid(nullptr, n), kBlock, 0, st>>>(n, r, rl, xl);
    return cudaGetLastError();
}

cudaError_t launch_add_correction(int n, const float *cl, double *x, cudaStream_t st)
{
    add_correction_kernel<<<stream_grid(nullptr, n), kBlock, 0, st>>>(n, cl, x);
    return cudaGetLastError();
}

cudaError_t launch_axpy_dev(int dtype, int n, const double *coef, double sign, const void *x, void *y,
                            const int *gate, cudaStream_t st)
{
    B200_DISPATCH(dtype, axpy_dev_kernel<T><<<stream_grid(nullptr, n), kBlock, 0, st>>>(n, coef, sign, (const T *)x,
                                                                                       (T *)y, gate));
    return cudaGetLastError();
}

cudaError_t launch_scale_dev(int dtype, int n, const double *coef, bool reciprocal, const void *x, void *y,
                             const int *gate, cudaStream_t st)
{
    B200_DISPATCH(dtype, scale_dev_kernel<T><<<stream_grid(nullptr, n), kBlock, 0, st>>>(
                             n, coef, reciprocal, (const T *)x, (T *)y, gate));
    return cudaGetLastError();
}

}  // namespace b200
