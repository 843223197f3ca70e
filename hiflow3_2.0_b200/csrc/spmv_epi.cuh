// spmv_epi.cuh -- row epilogues and reduction finalisers shared by the SpMV
// kernel families (CSR, dictionary, stencil, lattice).
#pragma once

#include "common.cuh"
#include "kernels.cuh"

namespace b200 {
namespace {

__device__ __forceinline__ void finalize(const SpmvOp &op, double v)
{
    DevState *st = op.st;
    switch (op.fin) {
    case FIN_STORE: *op.dot_out = v; break;
    case FIN_CG_ALPHA:
        st->pap = v;
        st->alpha = st->rho / v;
        break;
    case FIN_RES_INIT: {
        st->rr = v;
        const double res = sqrt(v);
        st->res = res;
        st->iter = 0;
        if (st->hist && st->hist_len > 0) st->hist[0] = res;
        st->status = check_state(st, 0, res);
        break;
    }
    default: break;
    }
}

template <typename T, int EPI>
__device__ __forceinline__ void epilogue(int r, T s, const SpmvOp &op, double &acc)
{
    T *y = static_cast<T *>(op.y);
    if constexpr (EPI == EPI_SET) {
        y[r] = s;
    } else if constexpr (EPI == EPI_ADD) {
        y[r] += s;
    } else if constexpr (EPI == EPI_DOT_X) {
        y[r] = s;
        acc += (double)(__ldg(static_cast<const T *>(op.x) + r) * s);
    } else if constexpr (EPI == EPI_RESID) {
        const T v = static_cast<const T *>(op.b)[r] - s;
        y[r] = v;
        acc += (double)(v * v);
    } else if constexpr (EPI == EPI_SGS_F) {
        y[r] = (-static_cast<const T *>(op.b)[r] + s) * static_cast<const T *>(op.d1)[r];
    } else if constexpr (EPI == EPI_SGS_B) {
        y[r] = (y[r] * static_cast<const T *>(op.d2)[r] + s) * static_cast<const T *>(op.d1)[r];
    } else if constexpr (EPI == EPI_ILU_F) {
        y[r] = -(-static_cast<const T *>(op.b)[r] + s);
    } else if constexpr (EPI == EPI_ILU_B) {
        y[r] = (-y[r] + s) * static_cast<const T *>(op.d1)[r];
    } else if constexpr (EPI == EPI_SGS_FB) {
        const T d1 = static_cast<const T *>(op.d1)[r];
        const T f = (-static_cast<const T *>(op.b)[r] + s) * d1;
        y[r] = (f * static_cast<const T *>(op.d2)[r] + T(0)) * d1;
    } else if constexpr (EPI == EPI_ILU_FB) {
        const T f = -(-static_cast<const T *>(op.b)[r] + s);
        y[r] = (-f + T(0)) * static_cast<const T *>(op.d1)[r];
    }
}

template <int EPI>
constexpr bool reduces()
{
    return EPI == EPI_DOT_X || EPI == EPI_RESID;
}

}  // namespace
}  // namespace b200
