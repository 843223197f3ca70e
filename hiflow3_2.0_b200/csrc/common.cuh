// common.cuh -- device helpers shared by the B200 lmp platform kernels.
//
// * PTX wrappers for mbarrier + cp.async.bulk (the bulk-copy engine streams
//   CSR tiles into shared memory without occupying registers or threads),
// * warp/block reductions,
// * a deterministic grid reduction: every CTA writes one partial per quantity,
//   the last CTA to finish (atomic ticket) sums the partials in CTA order and
//   runs a caller-supplied finaliser on thread 0.  The result depends only on
//   the grid size, never on CTA timing.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#ifndef B200LA_BLOCK
#define B200LA_BLOCK 256
#endif

namespace b200 {

constexpr int kBlock = B200LA_BLOCK;
constexpr int kMaxGrid = 148 * 8;           // partial slots per reduction quantity
constexpr long long kSpinLimit = 1LL << 28; // bounded waits: ~seconds, never forever

// Error flags written by kernels (ctx->dev_err); the host reads them after sync.
enum DevErr : int { kDevOk = 0, kDevWaitTimeout = 1, kDevBadIndex = 2 };

__device__ __forceinline__ unsigned smem_u32(const void *p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on an mbarrier phase.  Returns false (and records the error)
// if the phase does not complete within kSpinLimit polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, int *err)
{
    for (long long i = 0; i < kSpinLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicExch(err, kDevWaitTimeout);
    return false;
}

__device__ __forceinline__ uint64_t l2_evict_first_policy()
{
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// L2 eviction policies for individual loads.  A sparse operator streams its
// values and indices once per product while the gathered vector is re-read
// by every row: the stream is marked evict-first (and skips L1) and the
// vector evict-last, so that vector traffic of the kernels between two
// products cannot push the vector out of L2.  kind: 0 normal, 1 first, 2 last.
__device__ __forceinline__ uint64_t l2_policy(int kind)
{
    uint64_t p;
    if (kind == 1) asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    else if (kind == 2) asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    else asm("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// 16-byte streaming loads (L1 not allocated, the given L2 policy)
__device__ __forceinline__ void ld_stream_vec(const double *a, uint64_t pol, double (&v)[2])
{
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
        : "=d"(v[0]), "=d"(v[1]) : "l"(a), "l"(pol));
}
__device__ __forceinline__ void ld_stream_vec(const float *a, uint64_t pol, float (&v)[4])
{
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
        : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]) : "l"(a), "l"(pol));
}
__device__ __forceinline__ void ld_stream_vec(const int *a, uint64_t pol, int (&v)[2])
{
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.s32 {%0, %1}, [%2], %3;"
        : "=r"(v[0]), "=r"(v[1]) : "l"(a), "l"(pol));
}
__device__ __forceinline__ void ld_stream_vec(const int *a, uint64_t pol, int (&v)[4])
{
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0, %1, %2, %3}, [%4], %5;"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]) : "l"(a), "l"(pol));
}

__device__ __forceinline__ double ld_stream(const double *a, uint64_t pol)
{
    double v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_stream(const float *a, uint64_t pol)
{
    float v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ int ld_stream(const int *a, uint64_t pol)
{
    int v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
    return v;
}
// Coherent (not .nc) loads with an L2 policy: for data that a kernel still
// running when this one started -- a programmatic-launch predecessor -- writes
// before the grid dependency wait; the read-only path may not see such writes.
__device__ __forceinline__ double ld_coherent(const double *a, uint64_t pol)
{
    double v;
    asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol) : "memory");
    return v;
}
__device__ __forceinline__ float ld_coherent(const float *a, uint64_t pol)
{
    float v;
    asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol) : "memory");
    return v;
}

__device__ __forceinline__ double ld_keep(const double *a, uint64_t pol)
{
    double v;
    asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_keep(const float *a, uint64_t pol)
{
    float v;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
    return v;
}

// Global -> shared bulk copy completing on an mbarrier.  dst, src 16-byte
// aligned; bytes a multiple of 16.  The L2 policy marks the streamed matrix
// as evict-first so the gathered vector stays resident in L2.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar,
                                         uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1], %2, [%3], %4;" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

// Programmatic dependent launch: let the next launch on the stream start its
// CTAs now, and wait for the previous launch's completion (and memory) --
// both no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dependents_launch() { asm volatile("griddepcontrol.launch_dependents;"); }

// True when the stop-state word *gate is set (a solver's IterateControl
// state has left "iterate").  One thread per CTA reads it (through L2) and
// broadcasts it: a load by every thread of the grid on one address would
// serialise in L2.  Must be called by all threads of the CTA.
__device__ __forceinline__ bool gate_closed(const int *gate)
{
    if (!gate) return false;
    __shared__ int s_gate;
    if (threadIdx.x == 0) s_gate = __ldcg(gate);
    __syncthreads();
    return s_gate != 0;
}

// One double read once per CTA and broadcast (scalars of the recurrences).
__device__ __forceinline__ double cta_scalar(const double *p)
{
    __shared__ double s_val;
    __syncthreads();
    if (threadIdx.x == 0) s_val = __ldcg(p);
    __syncthreads();
    return s_val;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum of NQ values over the block; result valid on thread 0.  sm must hold
// NQ * (kBlock / 32) doubles.
template <int NQ>
__device__ __forceinline__ void block_sum(double (&v)[NQ], double *sm)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int nw = kBlock / 32;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        const double w = warp_sum(v[q]);
        if (lane == 0) sm[q * nw + warp] = w;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double s = 0.0;
            for (int w = 0; w < nw; ++w) s += sm[q * nw + w];
            v[q] = s;
        }
    }
    __syncthreads();
}

// Ticket words: kTicketGroups group counters and one final counter, each on
// its own 128-byte line (a single counter hit by ~1000 CTAs serialises for
// tens of microseconds).
constexpr int kTicketGroups = 32;
constexpr int kTicketStride = 32;   // unsigned words between counters
constexpr int kTicketWords = (kTicketGroups + 1) * kTicketStride;

// Grid-wide deterministic reduction tail.  Each CTA passes its per-thread
// values; partials is [NQ][kMaxGrid].  CTAs report to one of kTicketGroups
// group counters; the last CTA of a group reports to the final counter; the
// CTA that completes the final counter sums all partials.  Counters are reset
// by the CTAs that complete them.  Returns true on thread 0 of the last CTA,
// with out[] holding the totals in a fixed order.
template <int NQ>
__device__ __forceinline__ bool grid_reduce(double (&v)[NQ], double *partials, unsigned *ticket,
                                            double (&out)[NQ])
{
    __shared__ double sm[NQ * (kBlock / 32)];
    __shared__ bool last;
    block_sum<NQ>(v, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) partials[q * kMaxGrid + blockIdx.x] = v[q];
        __threadfence();
        const unsigned ngroups = gridDim.x < kTicketGroups ? gridDim.x : kTicketGroups;
        const unsigned g = blockIdx.x % ngroups;
        const unsigned gsize = (gridDim.x - g + ngroups - 1) / ngroups;
        unsigned *gc = ticket + kTicketStride * (1 + g);
        bool l = false;
        if (atomicAdd(gc, 1u) == gsize - 1) {
            *gc = 0u;
            __threadfence();
            if (atomicAdd(ticket, 1u) == ngroups - 1) {
                *ticket = 0u;
                l = true;
            }
        }
        last = l;
    }
    __syncthreads();
    if (!last) return false;
    // last CTA: every thread sums a fixed strided subset of the partials
    // (loads issued together, through L2), then a fixed block tree -- the
    // summation order depends only on the grid size
    __threadfence();
    double w[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) w[q] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kBlock) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) w[q] += __ldcg(partials + q * kMaxGrid + b);
    }
    block_sum<NQ>(w, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) out[q] = w[q];
    }
    return threadIdx.x == 0;
}

}  // namespace b200
