// matops.cu -- CSR value and structure operations of lMatrix on the device.
//
//   Scale / ScaleOffdiag / Zeros      (lmp/lmatrix_csr_cpu.cc:100-103, 205-224)
//   extract_diagelements / extract_invdiagelements (:2395-2431)
//   extract_submatrix                 (:1768-1843)
//   Compress                          (:142-202)
//
// The reference runs these on the host (its GPU matrices round-trip the CPU
// for extract_submatrix, lmp/lmatrix.cc:315-330).  Here the value operations
// run in place on the device CSR; the structure operations filter the CSR on
// the device (a count pass, the row pointer, a fill pass) and the host only
// builds the new matrix's SpMV schedule from the result.  Every output equals
// the reference's bit for bit: the same products, the same first-match
// accumulation of duplicate columns, the same column order.
#include <cuda_runtime.h>

#include <algorithm>

#include "b200la.h"
#include "b200la_internal.h"
#include "common.cuh"

namespace b200 {
namespace {

constexpr int kMatBlock = 256;

int grid_for(long long threads)
{
    return (int)std::max<long long>(1, std::min<long long>((threads + kMatBlock - 1) / kMatBlock, 148LL * 32));
}

// Scale (mode 0), ScaleOffdiag (1: entries off the diagonal), Zeros (2).
// A warp per row, lanes over its entries.
template <typename T>
__global__ void __launch_bounds__(kMatBlock) csr_scale_kernel(int n, const int *__restrict__ row,
                                                           const int *__restrict__ col, T *val, T alpha, int mode)
{
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * kMatBlock) >> 5;
    for (int i = (blockIdx.x * kMatBlock + threadIdx.x) >> 5; i < n; i += nw)
        for (int j = row[i] + lane; j < row[i + 1]; j += 32) {
            if (mode == 2) val[j] = T(0);
            else if (mode == 0 || col[j] != i) val[j] *= alpha;
        }
}

// Rows [start, end): every stored diagonal entry assigns, so the last one
// stays; a row without one leaves its output untouched.
template <typename T>
__global__ void __launch_bounds__(kMatBlock) csr_diag_kernel(int start, int end, const int *__restrict__ row,
                                                          const int *__restrict__ col, const T *__restrict__ val,
                                                          int inverse, T *out)
{
    for (int i = start + blockIdx.x * kMatBlock + threadIdx.x; i < end; i += gridDim.x * kMatBlock) {
        bool found = false;
        T d = T(0);
        for (int j = row[i]; j < row[i + 1]; ++j)
            if (col[j] == i) {
                d = val[j];
                found = true;
            }
        if (found) out[i - start] = inverse ? T(1) / d : d;
    }
}

__device__ __forceinline__ bool keep_entry(int mode, int c, int sc, int ec, double v)
{
    return mode == 0 ? (c >= sc && c < ec) : (v != 0.0);
}

// Entries of rows [r0, r1) that the filter keeps (mode 0: columns in
// [sc, ec); mode 1: nonzero values), one count per row.  Warp per row.
template <typename T>
__global__ void __launch_bounds__(kMatBlock) csr_filter_count(int r0, int r1, const int *__restrict__ row,
                                                           const int *__restrict__ col, const T *__restrict__ val,
                                                           int mode, int sc, int ec, int *cnt)
{
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * kMatBlock) >> 5;
    for (int i = r0 + ((blockIdx.x * kMatBlock + threadIdx.x) >> 5); i < r1; i += nw) {
        int c = 0;
        for (int j = row[i] + lane; j < row[i + 1]; j += 32) c += keep_entry(mode, col[j], sc, ec, (double)val[j]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) cnt[i - r0] = c;
    }
}

// The filtered rows into [off[i - r0], off[i - r0 + 1]), a thread per row.
// Compress keeps the entries in order.  A block row is built as the
// reference's init_structure + add_value build it: the kept columns (shifted
// by sc) sorted ascending, values zero, then every kept source entry, in
// source order, added to the first stored entry of its column.
template <typename T>
__global__ void __launch_bounds__(kMatBlock) csr_filter_fill(int r0, int r1, const int *__restrict__ row,
                                                          const int *__restrict__ col, const T *__restrict__ val,
                                                          int mode, int sc, int ec, const int *__restrict__ off,
                                                          int *co, T *vo)
{
    for (int i = r0 + blockIdx.x * kMatBlock + threadIdx.x; i < r1; i += gridDim.x * kMatBlock) {
        const int b = off[i - r0];
        int k = b;
        if (mode == 1) {
            for (int j = row[i]; j < row[i + 1]; ++j)
                if (val[j] != T(0)) {
                    co[k] = col[j];
                    vo[k] = val[j];
                    ++k;
                }
            continue;
        }
        for (int j = row[i]; j < row[i + 1]; ++j)
            if (col[j] >= sc && col[j] < ec) co[k++] = col[j] - sc;
        for (int a = b + 1; a < k; ++a) {   // insertion sort, ascending columns
            const int c = co[a];
            int q = a - 1;
            while (q >= b && co[q] > c) {
                co[q + 1] = co[q];
                --q;
            }
            co[q + 1] = c;
        }
        for (int a = b; a < k; ++a) vo[a] = T(0);
        for (int j = row[i]; j < row[i + 1]; ++j) {
            const int c = col[j];
            if (c < sc || c >= ec) continue;
            for (int a = b; a < k; ++a)
                if (co[a] == c - sc) {
                    vo[a] += val[j];
                    break;
                }
        }
    }
}

}  // namespace

cudaError_t launch_csr_scale(int dtype, int n, const int *row, const int *col, void *val, double alpha, int mode,
                             cudaStream_t st)
{
    const int g = grid_for(32LL * n);
    if (dtype == B200LA_F64)
        csr_scale_kernel<double><<<g, kMatBlock, 0, st>>>(n, row, col, static_cast<double *>(val), alpha, mode);
    else
        csr_scale_kernel<float><<<g, kMatBlock, 0, st>>>(n, row, col, static_cast<float *>(val), (float)alpha, mode);
    return cudaGetLastError();
}

cudaError_t launch_csr_diag(int dtype, int start, int end, const int *row, const int *col, const void *val,
                            int inverse, void *out, cudaStream_t st)
{
    const int g = grid_for(end - start);
    if (dtype == B200LA_F64)
        csr_diag_kernel<double><<<g, kMatBlock, 0, st>>>(start, end, row, col, static_cast<const double *>(val),
                                                      inverse, static_cast<double *>(out));
    else
        csr_diag_kernel<float><<<g, kMatBlock, 0, st>>>(start, end, row, col, static_cast<const float *>(val), inverse,
                                                     static_cast<float *>(out));
    return cudaGetLastError();
}

cudaError_t launch_csr_filter_count(int dtype, int r0, int r1, const int *row, const int *col, const void *val,
                                    int mode, int sc, int ec, int *cnt, cudaStream_t st)
{
    const int g = grid_for(32LL * (r1 - r0));
    if (dtype == B200LA_F64)
        csr_filter_count<double><<<g, kMatBlock, 0, st>>>(r0, r1, row, col, static_cast<const double *>(val), mode, sc,
                                                       ec, cnt);
    else
        csr_filter_count<float><<<g, kMatBlock, 0, st>>>(r0, r1, row, col, static_cast<const float *>(val), mode, sc,
                                                      ec, cnt);
    return cudaGetLastError();
}

cudaError_t launch_csr_filter_fill(int dtype, int r0, int r1, const int *row, const int *col, const void *val,
                                   int mode, int sc, int ec, const int *off, int *co, void *vo, cudaStream_t st)
{
    const int g = grid_for(r1 - r0);
    if (dtype == B200LA_F64)
        csr_filter_fill<double><<<g, kMatBlock, 0, st>>>(r0, r1, row, col, static_cast<const double *>(val), mode, sc,
                                                      ec, off, co, static_cast<double *>(vo));
    else
        csr_filter_fill<float><<<g, kMatBlock, 0, st>>>(r0, r1, row, col, static_cast<const float *>(val), mode, sc,
                                                     ec, off, co, static_cast<float *>(vo));
    return cudaGetLastError();
}

}  // namespace b200
