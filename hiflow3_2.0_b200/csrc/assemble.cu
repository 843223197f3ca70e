// assemble.cu -- Q1 assembly and right-hand sides on the device.
//
// The host assembler (host_setup.cc q1_assemble) restates the reference's
// assembly of a structured Q1 system: element matrices from 2-point Gauss
// quadrature (examples/poisson/poisson_tutorial.h:152-176, kind 0;
// examples/convection_diffusion/convdiff.cc:75-117, kind 1) added element by
// element into the CSR (lmp/lmatrix_csr_cpu.cc:1148-1181 add_values), then
// Dirichlet rows replaced by identity rows (lmp/lmatrix_csr_cpu.cc:1047-1068
// ZeroRows).  This file produces the same CSR on the device, bit for bit:
//   * row pointers in closed form: a node's stencil has w(i) = 2 neighbours
//     per axis on the boundary (i = 0 or N) and 3 inside, so with
//     S = 3N + 1 = sum_i w(i) and W(i) = sum_{i' < i} w(i') = 3i - [i > 0],
//     row[(ix,iy,iz)] = W(iz) S^2 + w(iz) (W(iy) S + w(iy) W(ix));
//   * columns in the host's (dk, dj, di) loop order, which is ascending;
//   * each value as the host forms it: 0.0 plus the element contributions in
//     element order (cz, cy, cx ascending), each contribution the element
//     matrix entry folded over the quadrature points with the host's operand
//     order.  __dmul_rn / __dadd_rn keep the device from contracting a
//     multiply and an add into one rounding, which the host (-ffp-contract=off)
//     never does;
//   * Dirichlet rows: alpha = 1 on the diagonal, 0.0 elsewhere.
// The quadrature tables are the host's own (q1_tables), passed by value.
#include <cuda_runtime.h>

#include <cstring>

#include "b200la.h"
#include "b200la_internal.h"

namespace b200 {
namespace {

struct Q1Dev {
    int dim, nv, nq, kind, N;
    double c0;                // coefficient without a cell field (1 or nu)
    double beta[3];
    double w[8];
    double dJ;
    double gg[8][8][8];       // [q][a][b]
    double phi[8][8];         // [q][a]
    double grad[8][8][3];     // [q][a][d]
};

__device__ __forceinline__ int q1_w(int i, int N) { return (i == 0 || i == N) ? 2 : 3; }
__device__ __forceinline__ long long q1_W(int i) { return 3LL * i - (i > 0 ? 1 : 0); }

// Element matrix entry Ke[a][b] of q1_element (host_setup.cc) for coefficient coef.
__device__ __forceinline__ double q1_ke(const Q1Dev &t, double coef, int a, int b)
{
    double ke = 0.0;
    for (int q = 0; q < t.nq; ++q) {
        ke = __dadd_rn(ke, __dmul_rn(__dmul_rn(t.w[q], __dmul_rn(coef, t.gg[q][a][b])), t.dJ));
        if (t.kind == 1) {
            double bg = 0.0;
            for (int d = 0; d < t.dim; ++d) bg = __dadd_rn(bg, __dmul_rn(t.beta[d], t.grad[q][b][d]));
            ke = __dadd_rn(ke, __dmul_rn(__dmul_rn(t.w[q], __dmul_rn(bg, t.phi[q][a])), t.dJ));
        }
    }
    return ke;
}

__global__ void __launch_bounds__(kBlock) q1_assemble_kernel(const Q1Dev tp, const double *__restrict__ kcell,
                                                             int *__restrict__ row, int *__restrict__ col,
                                                             double *__restrict__ val)
{
    __shared__ Q1Dev t;
    {
        const int words = (int)(sizeof(Q1Dev) / sizeof(int));
        const int *src = reinterpret_cast<const int *>(&tp);
        int *dst = reinterpret_cast<int *>(&t);
        for (int k = threadIdx.x; k < words; k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();
    const int N = t.N, P = N + 1, PZ = t.dim == 3 ? P : 1, CZ = t.dim == 3 ? N : 1;
    const long long S = 3LL * N + 1;
    const long long n = (long long)P * P * PZ;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(i % P), iy = (int)((i / P) % P), iz = (int)(i / ((long long)P * P));
        const int wz = t.dim == 3 ? q1_w(iz, N) : 1;
        const long long r0 = (t.dim == 3 ? q1_W(iz) * S * S : 0) + wz * (q1_W(iy) * S + q1_w(iy, N) * q1_W(ix));
        row[i] = (int)r0;
        if (i == n - 1) row[n] = (int)(t.dim == 3 ? S * S * S : S * S);
        const bool bnd = ix == 0 || ix == N || iy == 0 || iy == N || (t.dim == 3 && (iz == 0 || iz == N));
        long long e = r0;
        for (int dk = (t.dim == 3 ? -1 : 0); dk <= (t.dim == 3 ? 1 : 0); ++dk)
            for (int dj = -1; dj <= 1; ++dj)
                for (int di = -1; di <= 1; ++di) {
                    const int jx = ix + di, jy = iy + dj, jz = iz + dk;
                    if (jx < 0 || jx >= P || jy < 0 || jy >= P || jz < 0 || jz >= PZ) continue;
                    const long long j = jx + (long long)P * (jy + (long long)P * jz);
                    double v = 0.0;
                    if (bnd) {
                        v = (j == i) ? 1.0 : 0.0;
                    } else {
                        // cells holding both nodes, in element order
                        const int z0 = max(max(iz, jz) - 1, 0), z1 = min(min(iz, jz), CZ - 1);
                        const int y0 = max(max(iy, jy) - 1, 0), y1 = min(min(iy, jy), N - 1);
                        const int x0 = max(max(ix, jx) - 1, 0), x1 = min(min(ix, jx), N - 1);
                        for (int cz = z0; cz <= z1; ++cz)
                            for (int cy = y0; cy <= y1; ++cy)
                                for (int cx = x0; cx <= x1; ++cx) {
                                    const int a = (ix - cx) + 2 * (iy - cy) + 4 * (iz - cz);
                                    const int b = (jx - cx) + 2 * (jy - cy) + 4 * (jz - cz);
                                    const double coef =
                                        kcell ? kcell[cx + (long long)N * (cy + (long long)N * cz)] : t.c0;
                                    v = __dadd_rn(v, q1_ke(t, coef, a, b));
                                }
                    }
                    col[e] = (int)j;
                    val[e] = v;
                    ++e;
                }
    }
}

// splitmix64 draw k = i + 1 mapped to [-1, 1) with 53 bits; 0 on Dirichlet DoFs
// (the stream of host_setup.cc q1_rhs).
__global__ void q1_rhs_kernel(unsigned long long seed, int dim, int N, double *__restrict__ b)
{
    const int P = N + 1, PZ = dim == 3 ? P : 1;
    const long long n = (long long)P * P * PZ;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(i % P), iy = (int)((i / P) % P), iz = (int)(i / ((long long)P * P));
        unsigned long long z = seed + (unsigned long long)(i + 1) * 0x9E3779B97F4A7C15ULL;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        const double u = __dadd_rn(__dmul_rn(2.0, __dmul_rn((double)(z >> 11), 1.0 / 9007199254740992.0)), -1.0);
        const bool on = ix == 0 || ix == N || iy == 0 || iy == N || (dim == 3 && (iz == 0 || iz == N));
        b[i] = on ? 0.0 : u;
    }
}

int grid_for(long long n) { return (int)std::min<long long>((n + kBlock - 1) / kBlock, 148LL * 16); }

}  // namespace

cudaError_t launch_q1_assemble(int dim, int N, int kind, const double *kcell, double nu, const double *beta, int *row,
                               int *col, double *val, cudaStream_t st)
{
    host::Q1Tables h;
    host::q1_tables(dim, 1.0 / N, h);
    Q1Dev t;
    std::memset(&t, 0, sizeof t);
    t.dim = dim;
    t.nv = h.nv;
    t.nq = h.nq;
    t.kind = kind;
    t.N = N;
    t.c0 = kind == 0 ? 1.0 : nu;
    for (int d = 0; d < 3; ++d) t.beta[d] = beta ? beta[d] : 0.0;
    std::memcpy(t.w, h.w, sizeof t.w);
    t.dJ = h.dJ;
    std::memcpy(t.gg, h.gg, sizeof t.gg);
    std::memcpy(t.phi, h.phi, sizeof t.phi);
    std::memcpy(t.grad, h.grad, sizeof t.grad);
    const long long P = N + 1, n = dim == 3 ? P * P * P : P * P;
    q1_assemble_kernel<<<grid_for(n), kBlock, 0, st>>>(t, kcell, row, col, val);
    return cudaGetLastError();
}

cudaError_t launch_q1_rhs(unsigned long long seed, int dim, int N, double *b, cudaStream_t st)
{
    const long long P = N + 1, n = dim == 3 ? P * P * P : P * P;
    q1_rhs_kernel<<<grid_for(n), kBlock, 0, st>>>(seed, dim, N, b);
    return cudaGetLastError();
}

}  // namespace b200

extern "C" int b200la_q1_assemble_device(b200la_ctx *ctx, int dim, int N, int kind, const double *kcell, double nu,
                                         const double *beta, int *row, int *col, double *val)
{
    int n;
    int64_t nnz;
    if (!ctx || !row || !col || !val || (kind != 0 && kind != 1) || b200::host::q1_sizes(dim, N, &n, &nnz))
        return ctx_fail(ctx, B200LA_ERR_ARG, "q1_assemble_device: invalid argument", cudaSuccess);
    const cudaError_t e =
        b200::launch_q1_assemble(dim, N, kind, kcell, nu, beta, row, col, val, ctx->stream);
    if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "q1_assemble_device", e);
    ctx->launches += 1;
    return B200LA_OK;
}

extern "C" int b200la_q1_rhs_device(b200la_ctx *ctx, uint64_t seed, int dim, int N, double *b)
{
    int n;
    int64_t nnz;
    if (!ctx || !b || b200::host::q1_sizes(dim, N, &n, &nnz))
        return ctx_fail(ctx, B200LA_ERR_ARG, "q1_rhs_device: invalid argument", cudaSuccess);
    const cudaError_t e = b200::launch_q1_rhs(seed, dim, N, b, ctx->stream);
    if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "q1_rhs_device", e);
    ctx->launches += 1;
    return B200LA_OK;
}
