// ref_gpu_spmv.cu -- HiFlow3's own GPU SpMV kernel, built for sm_100a, timed as a baseline.
//
// kernel_spmv_csr_scalar (src/linear_algebra/lmp/cuda/cuda_spmv_kernel_csr_scalar.h:21-34)
// is included from the HiFlow3 tree at build time (baseline/Makefile) and
// launched as GPUscalar_CSR_lMatrix::VectorMult launches it
// (cuda/GPUscalar_csr_lmatrix.cu:89-111): one thread per row, 256 threads per
// block, ceil(n / 256) blocks (GPU_CSR_lMatrix::set_thread_blocks,
// cuda/lmatrix_csr_gpu.cc:85-95).  The reference also synchronises the device
// before every launch (cudaThreadSynchronize); the timing here is the
// kernel's alone: back-to-back launches between two CUDA events.
//
// Nothing of the B200 platform is used; this library only measures the
// reference's kernel on the same matrix for comparison.
#include <cuda_runtime.h>

#include "cuda_spmv_kernel_csr_scalar.h"

namespace {
template <typename T>
int run(int n, int nnz, const int *row, const int *col, const T *val, const T *x, T *y, int reps, double *ms)
{
    int *d_row = nullptr, *d_col = nullptr;
    T *d_val = nullptr, *d_x = nullptr, *d_y = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaSuccess;
    float t = 0.f;
    const int block = 256, grid = (n + block - 1) / block;
    if ((e = cudaMalloc(&d_row, sizeof(int) * (n + 1))) || (e = cudaMalloc(&d_col, sizeof(int) * (size_t)nnz)) ||
        (e = cudaMalloc(&d_val, sizeof(T) * (size_t)nnz)) || (e = cudaMalloc(&d_x, sizeof(T) * (size_t)n)) ||
        (e = cudaMalloc(&d_y, sizeof(T) * (size_t)n)) ||
        (e = cudaMemcpy(d_row, row, sizeof(int) * (n + 1), cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(d_col, col, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(d_val, val, sizeof(T) * (size_t)nnz, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(d_x, x, sizeof(T) * (size_t)n, cudaMemcpyHostToDevice)) || (e = cudaEventCreate(&e0)) ||
        (e = cudaEventCreate(&e1)))
        goto done;
    kernel_spmv_csr_scalar<T><<<grid, block>>>(d_val, d_col, d_row, d_x, d_y, n);   // warm-up
    if ((e = cudaGetLastError()) || (e = cudaDeviceSynchronize()) || (e = cudaEventRecord(e0))) goto done;
    for (int k = 0; k < reps; ++k) kernel_spmv_csr_scalar<T><<<grid, block>>>(d_val, d_col, d_row, d_x, d_y, n);
    if ((e = cudaGetLastError()) || (e = cudaEventRecord(e1)) || (e = cudaEventSynchronize(e1)) ||
        (e = cudaEventElapsedTime(&t, e0, e1)))
        goto done;
    *ms = reps > 0 ? t / reps : 0.0;
    e = cudaMemcpy(y, d_y, sizeof(T) * (size_t)n, cudaMemcpyDeviceToHost);
done:
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d_row);
    cudaFree(d_col);
    cudaFree(d_val);
    cudaFree(d_x);
    cudaFree(d_y);
    return e == cudaSuccess ? 0 : (int)e;
}
}  // namespace

// dtype 0: double, 1: float.  y = A x on the device, copied back; *ms the
// mean kernel time of `reps` back-to-back launches.  0 on success, else the
// CUDA error code.
extern "C" int refgpu_spmv(int dtype, int n, int nnz, const int *row, const int *col, const void *val,
                           const void *x, void *y, int reps, double *ms)
{
    if (n <= 0 || nnz < 0 || !row || !col || !val || !x || !y || !ms) return -1;
    if (dtype == 0)
        return run<double>(n, nnz, row, col, static_cast<const double *>(val), static_cast<const double *>(x),
                           static_cast<double *>(y), reps, ms);
    return run<float>(n, nnz, row, col, static_cast<const float *>(val), static_cast<const float *>(x),
                      static_cast<float *>(y), reps, ms);
}
