// ref_gpu_gmg.cu -- HiFlow3's own GPU multigrid level kernels, built for
// sm_100a, as the checker of the platform's b200la_gmg_* steps.
//
// The reference's cuda_gmg.cu (src/linear_algebra/lmp/cuda/cuda_gmg.cu with
// the kernels of cuda_gmg_kernel.h: residual, restriction, updated solution,
// each with and without the off-diagonal ghost block) is compiled from the
// HiFlow3 tree by baseline/Makefile together with this file, which moves host
// CSR blocks and vectors to the device, calls the reference's own launch
// functions (one thread per row, 256 per block) and copies the result back.
// Test infrastructure only; nothing of the B200 platform links it.
#include <cuda_runtime.h>

#include <vector>

#include "cuda_gmg.h"

namespace {

struct Dev {
    std::vector<void *> ptrs;
    cudaError_t e = cudaSuccess;
    template <typename T>
    T *up(const T *h, size_t n)
    {
        void *d = nullptr;
        if (e == cudaSuccess && n) e = cudaMalloc(&d, sizeof(T) * n);
        if (e == cudaSuccess && n && h) e = cudaMemcpy(d, h, sizeof(T) * n, cudaMemcpyHostToDevice);
        if (d) ptrs.push_back(d);
        return static_cast<T *>(d);
    }
    ~Dev()
    {
        for (void *p : ptrs) cudaFree(p);
    }
};

struct Csr {
    const int *row, *col;
    const double *val;
    int n;
};

int grid_of(int n) { return (n + 255) / 256; }

}  // namespace

// mode 0: res = rhs - A_d sol - A_o ghost; 1: res = R_d tmp + R_o ghost;
// 2: sol += P_d res + P_o ghost.  The off-diagonal block is used when o_row
// is non-null.  in0 / in1 are (sol, rhs), (tmp, -) or (res, -); io is the
// output (mode 2: sol, updated in place).
extern "C" int refgpu_gmg(int mode, int n, const int *d_row, const int *d_col, const double *d_val, int m_cols,
                          const int *o_row, const int *o_col, const double *o_val, int n_ghost, const double *ghost,
                          const double *in0, const double *in1, double *io)
{
    Dev D;
    const int nnz = d_row[n], onnz = o_row ? o_row[n] : 0;
    int *r = D.up(d_row, n + 1), *c = D.up(d_col, nnz);
    double *v = D.up(d_val, nnz);
    int *orw = o_row ? D.up(o_row, n + 1) : nullptr, *oc = o_row ? D.up(o_col, onnz) : nullptr;
    double *ov = o_row ? D.up(o_val, onnz) : nullptr;
    double *g = o_row ? D.up(ghost, n_ghost) : nullptr;
    double *a = D.up(in0, mode == 1 ? m_cols : (mode == 2 ? m_cols : n));
    double *b = mode == 0 ? D.up(in1, n) : nullptr;
    double *out = D.up(mode == 2 ? io : static_cast<const double *>(nullptr), n);
    if (D.e != cudaSuccess) return (int)D.e;
    const int gr = grid_of(n);
    if (mode == 0) {
        if (o_row) cuda_gmg_compute_residual<double>(v, c, r, n, ov, oc, orw, a, b, out, g, gr, 256, 0);
        else cuda_gmg_compute_residual_no_offdiag<double>(v, c, r, n, a, b, out, gr, 256, 0);
    } else if (mode == 1) {
        if (o_row) cuda_gmg_compute_restriction<double>(v, c, r, n, ov, oc, orw, out, g, a, gr, 256, 0);
        else cuda_gmg_compute_restriction_no_offdiag<double>(v, c, r, n, out, a, gr, 256, 0);
    } else {
        if (o_row) cuda_gmg_compute_updated_solution<double>(v, c, r, n, ov, oc, orw, out, a, g, gr, 256, 0);
        else cuda_gmg_compute_updated_solution_no_offdiag<double>(v, c, r, n, out, a, gr, 256, 0);
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(io, out, sizeof(double) * n, cudaMemcpyDeviceToHost);
    return (int)e;
}
