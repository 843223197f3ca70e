// remote.cu -- the off-diagonal product of a row-block matrix with the ghost
// values read straight from the ranks that own them.
//
// The reference moves ghost values with MPI (CoupledVector::UpdateGhost,
// src/linear_algebra/coupled_vector.cc:975-1128: pack the border, Isend /
// Irecv, unpack into the ghost buffer) before the off-diagonal product
// (coupled_matrix.cc:433-467).  When the owners' vectors are addressable from
// this GPU -- ranks that share a GPU, or GPUs of one process with peer access
// over NVLink -- the product itself can fetch each ghost value from its
// owner: y_i += sum_j O_ij x_owner(j)[index(j)].  No pack, no transfer, no
// ghost buffer; over NVLink every value crosses once, as a plain load (no
// multicast, no bulk copy from peer memory).  The caller orders the streams:
// the owners' vectors are final before this kernel runs and are not written
// again until it has finished.
#include <cuda_runtime.h>

#include <algorithm>

#include "b200la.h"
#include "b200la_internal.h"
#include "common.cuh"

namespace b200 {
namespace {

constexpr int kRemBlock = 256;

// A warp per row of the off-diagonal block; lanes over its entries, a fixed
// shuffle tree over the lanes.  Ghost k lives at owners[owner[k]][index[k]].
template <typename T>
__global__ void __launch_bounds__(kRemBlock) spmv_add_remote_kernel(int n, const int *__restrict__ row,
                                                                    const int *__restrict__ col,
                                                                    const T *__restrict__ val,
                                                                    const T *const *__restrict__ owners,
                                                                    const int *__restrict__ owner,
                                                                    const int *__restrict__ index, T *y)
{
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * kRemBlock) >> 5;
    for (int i = (blockIdx.x * kRemBlock + threadIdx.x) >> 5; i < n; i += nw) {
        T s = T(0);
        for (int j = row[i] + lane; j < row[i + 1]; j += 32) {
            const int k = col[j];
            const T *src = owners[__ldg(owner + k)];
            s += val[j] * __ldcg(src + __ldg(index + k));   // through L2: the owner's latest values
        }
        s = warp_sum(s);
        if (lane == 0) y[i] += s;
    }
}

}  // namespace
}  // namespace b200

using namespace b200;

extern "C" int b200la_spmv_add_remote(b200la_ctx *ctx, const b200la_csr *A_offdiag, const void *const *owners_dev,
                                      const int *ghost_owner_dev, const int *ghost_index_dev, void *y)
{
    if (!ctx || !A_offdiag || !y || (A_offdiag->nnz && (!owners_dev || !ghost_owner_dev || !ghost_index_dev)))
        return ctx_fail(ctx, B200LA_ERR_ARG, "spmv_add_remote: invalid argument", cudaSuccess);
    const int n = A_offdiag->n;
    if (!n || !A_offdiag->nnz) return B200LA_OK;
    const int g = std::max(1, std::min((n + kRemBlock / 32 - 1) / (kRemBlock / 32), ctx->num_sms * 8));
    if (A_offdiag->dtype == B200LA_F64)
        spmv_add_remote_kernel<double><<<g, kRemBlock, 0, ctx->stream>>>(
            n, A_offdiag->row, A_offdiag->col, (const double *)A_offdiag->val, (const double *const *)owners_dev,
            ghost_owner_dev, ghost_index_dev, (double *)y);
    else
        spmv_add_remote_kernel<float><<<g, kRemBlock, 0, ctx->stream>>>(
            n, A_offdiag->row, A_offdiag->col, (const float *)A_offdiag->val, (const float *const *)owners_dev,
            ghost_owner_dev, ghost_index_dev, (float *)y);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "spmv_add_remote", e);
    ctx->launches += 1;
    return B200LA_OK;
}

extern "C" int b200la_enable_peer_access(int device, int peer_device)
{
    int can = 0;
    if (device == peer_device) return B200LA_OK;
    if (cudaDeviceCanAccessPeer(&can, device, peer_device) != cudaSuccess || !can) {
        (void)cudaGetLastError();   // leave no error behind for the next launch check
        return B200LA_ERR_DEVICE;
    }
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) return B200LA_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return B200LA_ERR_CUDA;
    cudaError_t e = cudaDeviceEnablePeerAccess(peer_device, 0);
    if (e == cudaErrorPeerAccessAlreadyEnabled) {
        (void)cudaGetLastError();
        e = cudaSuccess;
    }
    cudaSetDevice(cur);
    return e == cudaSuccess ? B200LA_OK : B200LA_ERR_CUDA;
}
