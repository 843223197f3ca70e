// noalloc.cu -- a dot product for callers that cannot allocate device memory.
//
// Who needs it: a host application that owns all device memory and hands out
// pre-sized buffers from its own pool (a larger GPU code embedding HiFlow3's
// solvers), or a stream-ordered pipeline in which cudaMalloc -- which may
// synchronise the whole device -- is not allowed once set-up is over.
// b200la_dot needs a context, and creating one allocates device memory; this
// entry point needs no context and allocates nothing.
//
// Scratch: g_noalloc_scratch below, a file-scope __device__ array holding the
// per-block partial sums (kNoAllocBlocks doubles, one per 4096 elements, so n
// is limited to B200LA_NOALLOC_MAX_N) and the ticket counters of the last-block
// reduction, about 135 KB on every GPU that loads the library, held until the
// process exits.  Every call clears the tickets first (cudaMemsetAsync, no
// allocation); the partials are always written before they are read.  All
// calls share the one array: calls whose kernels overlap on the GPU (two
// streams, two host threads) race on it and must be ordered by the caller.
//
// Set-up: in host code the array's name is only a host-side stand-in, not a
// device address.  The first call on each device (with that device current)
// resolves the address with cudaGetSymbolAddress, checks it and caches it;
// later calls on that device reuse it.  Make that first call before any stream
// capture begins.  The cached address belongs to the device's primary context:
// after cudaDeviceReset on a device, this entry point must not be called on it
// again in the same process.
//
// Errors: an error already pending in the CUDA runtime when the call starts
// (an earlier asynchronous failure of the caller's own work) is left in place
// for the caller and the call returns B200LA_ERR_CUDA without launching; a
// failure of this call's own set-up or launch is cleared from the runtime and
// reported as B200LA_ERR_CUDA.
#include "b200la.h"
#include "common.cuh"

#include <cuda_runtime.h>

#include <mutex>

namespace {

constexpr int kPerBlock = 4096;                                  // elements per block
constexpr int kNoAllocBlocks = B200LA_NOALLOC_MAX_N / kPerBlock;  // partials
constexpr int kGroups = 32, kStride = 32;                        // ticket layout (words)
constexpr int kTicketWordsNA = (kGroups + 1) * kStride;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocBlocks + kTicketWordsNA / 2];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double *g_addr[kMaxDevices] = {};

template <typename T>
__global__ void __launch_bounds__(b200::kBlock) dot_noalloc_kernel(int n, const T *__restrict__ x,
                                                                    const T *__restrict__ y, double *out,
                                                                    double *scratch)
{
    using b200::kBlock;
    double *partials = scratch;
    unsigned *ticket = reinterpret_cast<unsigned *>(scratch + kNoAllocBlocks);
    __shared__ double sm[kBlock / 32];
    __shared__ bool last;
    // fixed order: thread t of block b sums elements b*4096 + t + 256 k
    double a = 0.0;
    const int base = blockIdx.x * kPerBlock + threadIdx.x;
#pragma unroll 4
    for (int k = 0; k < kPerBlock / kBlock; ++k) {
        const int i = base + k * kBlock;
        if (i < n) a += (double)(x[i] * y[i]);
    }
    double v[1] = {a};
    b200::block_sum<1>(v, sm);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = v[0];
        __threadfence();
        const unsigned ng = gridDim.x < kGroups ? gridDim.x : kGroups;
        const unsigned g = blockIdx.x % ng;
        const unsigned gsize = (gridDim.x - g + ng - 1) / ng;
        unsigned *gc = ticket + kStride * (1 + g);
        bool l = false;
        if (atomicAdd(gc, 1u) == gsize - 1) {
            __threadfence();
            l = atomicAdd(ticket, 1u) == ng - 1;
        }
        last = l;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double w[1] = {0.0};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kBlock) w[0] += __ldcg(partials + b);
    b200::block_sum<1>(w, sm);
    if (threadIdx.x == 0) *out = w[0];
}

}  // namespace

extern "C" int b200la_dot_noalloc(int dtype, int n, const void *x, const void *y, double *result_dev, void *stream)
{
    if ((dtype != B200LA_F64 && dtype != B200LA_F32) || n < 0 || !result_dev || (n > 0 && (!x || !y)))
        return B200LA_ERR_ARG;
    if (n > B200LA_NOALLOC_MAX_N) return B200LA_ERR_ARG;   // the scratch holds partials for at most this many
    // an earlier, unrelated error stays with the caller: report it, clear nothing
    if (cudaPeekAtLastError() != cudaSuccess) return B200LA_ERR_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return B200LA_ERR_DEVICE;
    }
    double *scratch;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        if (!g_addr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
                cudaGetLastError();   // this call's own failure, reported by the return code
                return B200LA_ERR_CUDA;
            }
            g_addr[dev] = static_cast<double *>(p);
        }
        scratch = g_addr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (n == 0) return cudaMemsetAsync(result_dev, 0, sizeof(double), s) == cudaSuccess ? B200LA_OK : B200LA_ERR_CUDA;
    // the ticket counters must start at zero
    if (cudaMemsetAsync(scratch + kNoAllocBlocks, 0, sizeof(unsigned) * kTicketWordsNA, s) != cudaSuccess)
        return B200LA_ERR_CUDA;
    const int grid = (n + kPerBlock - 1) / kPerBlock;
    if (dtype == B200LA_F64)
        dot_noalloc_kernel<double><<<grid, b200::kBlock, 0, s>>>(n, static_cast<const double *>(x),
                                                                 static_cast<const double *>(y), result_dev, scratch);
    else
        dot_noalloc_kernel<float><<<grid, b200::kBlock, 0, s>>>(n, static_cast<const float *>(x),
                                                                static_cast<const float *>(y), result_dev, scratch);
    return cudaGetLastError() == cudaSuccess ? B200LA_OK : B200LA_ERR_CUDA;
}
