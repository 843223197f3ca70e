// serve_kernels.cu -- batched Krylov kernels of the solve server (sm_100a).
//
// One batch iteration is two launches over the system table:
//   k1  SpMV  Ap = A p_new with p_new = beta p + z formed on the fly at every
//       gathered column (and stored for the own rows into the other of two p
//       buffers), with the partials of p_new.Ap; on completion of a system
//       alpha = rho / p.Ap and the p buffer flips (CG, inner CG).  The outer
//       step of a mixed system runs here too: r = b - A (x + x_low) in FP64
//       with x + x_low formed at every gathered column, r_low = (float) r,
//       and the outer test on completion.
//   k2  update x += alpha p, r -= alpha Ap, z = D^-1 r with the partials of
//       r.r and r.z; on completion IterateControl::Check
//       (src/common/iterate_control.cc:84-110) and beta, rho.  The CG start
//       (r = b) runs here, and after an outer step x += x_low, x_low = 0.
// Folding the p-update of CG<LAD> (cg.cc:240-246) into the next product
// removes a launch and a pass per iteration; the update is written with
// explicit roundings so that every gathering thread forms the same p_new as
// the thread that stores it.
//
// Work split: the active systems' 32-row chunks form one sequence, each
// chunk weighted by the bytes per row the kernel streams for its system; each
// warp takes one contiguous range of equal weight, with no CTA barrier.  A warp loads a
// system's descriptor and state into its own shared-memory slot when its
// range enters the system.  Reductions: one partial per chunk; a warp reports
// its run of each system's chunks to the run's groups of 32 chunks, the warp
// completing a group sums its partials (fixed shuffle tree) and reports the
// group to the system, and the warp completing the last group sums the group
// partials in a fixed order and runs the finaliser.  Counters are reset by
// their completers.  Operator values and indices are streamed past L1,
// gathered vectors go through L1.
#include <cuda_runtime.h>

#include <cstdlib>

#include "common.cuh"
#include "serve.cuh"

#ifndef B200LA_SRV_MINCTA
#define B200LA_SRV_MINCTA 4
#endif

namespace b200 {
namespace srv {
namespace {

// Resident 256-thread CTAs per SM the batched kernels are compiled for
// (register budget 65536 / (256 x this)).
constexpr int kMinCta256 = B200LA_SRV_MINCTA;

// IterateControl::Check with the first step 0 (res0 passed in).
__device__ __forceinline__ int check_cg(double v, int step, double res0, double abstol, double reltol,
                                        double divtol, int maxits)
{
    if (v < abstol) return 1;
    if (v < reltol * res0) return 2;
    if (v > divtol * res0) return 3;
    if (step >= maxits) return 4;
    return 0;
}

struct WarpCtx {
    SysDesc d;
    SysState s;
};

// Descriptor and state of slot `slot` into the warp's context (all lanes).
__device__ __forceinline__ void warp_load(const SysDesc *sys, const SysState *state, int slot, WarpCtx &c)
{
    const int lane = threadIdx.x & 31;
    constexpr int dw = (int)(sizeof(SysDesc) / sizeof(int));
    constexpr int sw = (int)(sizeof(SysState) / sizeof(int));
    const int *src = reinterpret_cast<const int *>(sys + slot);
    const int *sst = reinterpret_cast<const int *>(state + slot);
    __syncwarp();
    for (int k = lane; k < dw; k += 32) reinterpret_cast<int *>(&c.d)[k] = __ldcg(src + k);
    for (int k = lane; k < sw; k += 32) reinterpret_cast<int *>(&c.s)[k] = __ldcg(sst + k);
    __syncwarp();
}

// p_new(j) = beta p_old(j) + z(j), rounded the same wherever it is formed.
__device__ __forceinline__ double pnew_at(double beta, const double *__restrict__ po, const double *__restrict__ z,
                                          int j)
{
    return __fma_rn(beta, __ldg(po + j), __ldg(z + j));
}
__device__ __forceinline__ float pnew_at(float beta, const float *__restrict__ po, const float *__restrict__ z, int j)
{
    return __fmaf_rn(beta, __ldg(po + j), __ldg(z + j));
}
// z = D^-1 r as stored (one rounding)
__device__ __forceinline__ double zmul(double r, double d) { return __dmul_rn(r, d); }
__device__ __forceinline__ float zmul(float r, float d) { return __fmul_rn(r, d); }

// One band of a stencil row: centre w gathered by every lane, neighbours by
// shuffle, lanes 0 / 31 gather their halo column; products in column order.
// Columns outside [0, n) belong to zero entries and are clamped into range.
template <typename T, typename G>
__device__ __forceinline__ void band(T &s, T a0, T a1, T a2, int i, int he, int d, int n, int lane, G gather)
{
    const int last = n - 1;
    const T w = gather(min(max(i + d, 0), last));
    const T h = (lane == 0 || lane == 31) ? gather(min(max(he + d, 0), last)) : T(0);
    T left = __shfl_up_sync(0xffffffffu, w, 1);
    T right = __shfl_down_sync(0xffffffffu, w, 1);
    if (lane == 0) left = h;
    if (lane == 31) right = h;
    s += a0 * left;
    s += a1 * w;
    s += a2 * right;
}

__device__ __forceinline__ int band_offset(int dim, int P, int b)
{
    return dim == 3 ? ((b / 3 - 1) * P + (b % 3 - 1)) * P : (b - 1) * P;
}

// Stencil row, FP64: groups of three bands, value loads and gathers of a
// group issued together.
template <int NB, typename G>
__device__ __forceinline__ double stencil_row(const double *__restrict__ val, int c, int lane, int n, int P,
                                              uint64_t pol, G gather)
{
    constexpr int DIM = NB == 9 ? 3 : 2;
    const int r0 = c * kChunk, i = r0 + lane, he = lane == 0 ? r0 - 1 : r0 + 32;
    const double *v = val + (size_t)c * kChunk * 3 * NB + lane;
    double s = 0.0;
#pragma unroll
    for (int b0 = 0; b0 < NB; b0 += 3) {
        double a[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) a[k] = ld_stream(v + 32 * (3 * b0 + k), pol);
#pragma unroll
        for (int bb = 0; bb < 3; ++bb)
            band(s, a[3 * bb], a[3 * bb + 1], a[3 * bb + 2], i, he, band_offset(DIM, P, b0 + bb), n, lane, gather);
    }
    return s;
}

// Stencil row, FP32: the row's first 4 (L / 4) positions in groups of four
// per lane (one 16-byte load each), the last L % 4 positions one by one
// (position-major, 128 bytes per warp load), then the bands.  A chunk holds
// exactly 32 L values: no padding.
template <int NB, typename G>
__device__ __forceinline__ float stencil_row(const float *__restrict__ val, int c, int lane, int n, int P,
                                             uint64_t pol, G gather)
{
    constexpr int DIM = NB == 9 ? 3 : 2, L = 3 * NB, G4 = L / 4, TL = L % 4;
    const int r0 = c * kChunk, i = r0 + lane, he = lane == 0 ? r0 - 1 : r0 + 32;
    const float *cv = val + (size_t)c * kChunk * L;
    const float4 *v = reinterpret_cast<const float4 *>(cv) + lane;
    float a[L];
#pragma unroll
    for (int g = 0; g < G4; ++g) {
        float4 q;
        asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
            : "=f"(q.x), "=f"(q.y), "=f"(q.z), "=f"(q.w)
            : "l"(v + 32 * g), "l"(pol));
        a[4 * g] = q.x;
        a[4 * g + 1] = q.y;
        a[4 * g + 2] = q.z;
        a[4 * g + 3] = q.w;
    }
#pragma unroll
    for (int t = 0; t < TL; ++t) a[4 * G4 + t] = ld_stream(cv + 128 * G4 + 32 * t + lane, pol);
    float s = 0.0f;
#pragma unroll
    for (int b = 0; b < NB; ++b)
        band(s, a[3 * b], a[3 * b + 1], a[3 * b + 2], i, he, band_offset(DIM, P, b), n, lane, gather);
    return s;
}

// Half stencil rows (layout: serve.cuh).  The lower half of row i is read
// from the rows that own it: (i, i + d + m - 1) of lower band b (centre d)
// is row (i + d + m - 1)'s entry at position 2 - m of upper band U - 1 - b
// (mirror bands), and (i, i - 1) is row (i - 1)'s +1 entry.  Those rows'
// values are streamed by other warps in the same launch, at most a plane of
// rows away, so the second read is served by L2.  The band values are
// assembled in the full layout's (band, column) order and added as
// stencil_row adds them, so a row sums to the same bits.
template <int NB>
__device__ __forceinline__ void half_identity(const unsigned *__restrict__ smask, int c, int lane, double (&av)[NB][3])
{
    constexpr int U = (NB - 1) / 2;
    if ((__ldg(smask + c) >> lane) & 1u) {
#pragma unroll
        for (int b = 0; b < NB; ++b)
#pragma unroll
            for (int m = 0; m < 3; ++m)
                if (b != U || m != 1) av[b][m] = 0.0;
    }
}

template <int NB>
__device__ __forceinline__ void half_identity(const unsigned *__restrict__ smask, int c, int lane, float (&av)[NB][3])
{
    constexpr int U = (NB - 1) / 2;
    if ((__ldg(smask + c) >> lane) & 1u) {
#pragma unroll
        for (int b = 0; b < NB; ++b)
#pragma unroll
            for (int m = 0; m < 3; ++m)
                if (b != U || m != 1) av[b][m] = 0.0f;
    }
}

template <int NB, typename G>
__device__ __forceinline__ double stencil_row_half(const double *__restrict__ val, const unsigned *__restrict__ smask,
                                                   int c, int lane, int n, int P, uint64_t pol, G gather)
{
    constexpr int DIM = NB == 9 ? 3 : 2, U = (NB - 1) / 2, H = 2 + 3 * U;
    const int r0 = c * kChunk, i = r0 + lane, he = lane == 0 ? r0 - 1 : r0 + 32;
    const double *own = val + (size_t)c * kChunk * H + lane;
    auto at = [&](int q, int p) {
        return q >= 0 ? ld_keep(val + ((size_t)(q >> 5) * H + p) * kChunk + (q & 31), pol) : 0.0;
    };
    const bool ident = (__ldg(smask + c) >> lane) & 1u;
    double s = 0.0;
    // groups of three bands: the values of a group (own upper slots, or the
    // owners' slots for the lower bands) are loaded together, then its
    // gathers and products -- the registers of one group, not of the row
#pragma unroll
    for (int b0 = 0; b0 < NB; b0 += 3) {
        double a[3][3];
#pragma unroll
        for (int bb = 0; bb < 3; ++bb) {
            const int b = b0 + bb;
            if (b > U) {
#pragma unroll
                for (int m = 0; m < 3; ++m) a[bb][m] = ld_stream(own + 32 * (2 + 3 * (b - U - 1) + m), pol);
            } else if (b == U) {
                a[bb][0] = at(i - 1, 1);
                a[bb][1] = ld_stream(own, pol);
                a[bb][2] = ld_stream(own + 32, pol);
            } else {
                const int q = i + band_offset(DIM, P, b), p = 2 + 3 * (U - 1 - b);
                a[bb][0] = at(q - 1, p + 2);
                a[bb][1] = at(q, p + 1);
                a[bb][2] = at(q + 1, p);
            }
            if (ident) {
                // identity row: its upper slots serve the neighbours; off-diagonals are zero
#pragma unroll
                for (int m = 0; m < 3; ++m)
                    if (b != U || m != 1) a[bb][m] = 0.0;
            }
        }
#pragma unroll
        for (int bb = 0; bb < 3; ++bb)
            band(s, a[bb][0], a[bb][1], a[bb][2], i, he, band_offset(DIM, P, b0 + bb), n, lane, gather);
    }
    return s;
}

__device__ __forceinline__ float4 ld_f4(const float *p, uint64_t pol)
{
    float4 q;
    asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
        : "=f"(q.x), "=f"(q.y), "=f"(q.z), "=f"(q.w)
        : "l"(p), "l"(pol));
    return q;
}

template <int NB, typename G>
__device__ __forceinline__ float stencil_row_half(const float *__restrict__ val, const unsigned *__restrict__ smask,
                                                  int c, int lane, int n, int P, uint64_t pol, G gather)
{
    constexpr int DIM = NB == 9 ? 3 : 2, U = (NB - 1) / 2, H = 4 * U + (U < 2 ? 1 : 0);
    const int r0 = c * kChunk, i = r0 + lane, he = lane == 0 ? r0 - 1 : r0 + 32, rows = (n + 31) & ~31;
    const bool edge = lane == 0 || lane == 31;
    const float *cv = val + (size_t)c * kChunk * H;
    auto grp = [&](int q, int u) { return val + (size_t)(q >> 5) * kChunk * H + 128 * u + 4 * (q & 31); };
    auto plus1 = [&](int q) {   // row q's +1 entry
        return U >= 2 ? ld_f4(grp(q, 1), pol).w : ld_keep(val + (size_t)(q >> 5) * kChunk * H + 128 * U + (q & 31), pol);
    };
    float av[NB][3];
    float4 u[U];
#pragma unroll
    for (int g = 0; g < U; ++g) {
        asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
            : "=f"(u[g].x), "=f"(u[g].y), "=f"(u[g].z), "=f"(u[g].w)
            : "l"(cv + 128 * g + 4 * lane), "l"(pol));
    }
    const float pl = U >= 2 ? u[U >= 2 ? 1 : 0].w : ld_stream(cv + 128 * U + lane, pol);
#pragma unroll
    for (int ub = 0; ub < U; ++ub) {
        av[U + 1 + ub][0] = u[ub].x;
        av[U + 1 + ub][1] = u[ub].y;
        av[U + 1 + ub][2] = u[ub].z;
    }
    av[U][1] = u[0].w;
    av[U][2] = pl;
    float lm = __shfl_up_sync(0xffffffffu, pl, 1);
    if (lane == 0) lm = r0 > 0 ? plus1(r0 - 1) : 0.0f;
    av[U][0] = lm;
#pragma unroll
    for (int b = 0; b < U; ++b) {
        const int d = band_offset(DIM, P, b), ub = U - 1 - b, q = i + d;
        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 g = q >= 0 ? ld_f4(grp(q, ub), pol) : z4;
        const int hq = lane == 0 ? r0 + d - 1 : r0 + 32 + d;
        const float4 h = (edge && hq >= 0 && hq < rows) ? ld_f4(grp(hq, ub), pol) : z4;
        float left = __shfl_up_sync(0xffffffffu, g.z, 1);
        float right = __shfl_down_sync(0xffffffffu, g.x, 1);
        if (lane == 0) left = h.z;
        if (lane == 31) right = h.x;
        av[b][0] = left;
        av[b][1] = g.y;
        av[b][2] = right;
    }
    half_identity<NB>(smask, c, lane, av);
    float s = 0.0f;
#pragma unroll
    for (int b = 0; b < NB; ++b) band(s, av[b][0], av[b][1], av[b][2], i, he, band_offset(DIM, P, b), n, lane, gather);
    return s;
}

// Stencil row of a system, full or half layout.
template <typename T, int NB, typename G>
__device__ __forceinline__ T stencil_any(const SysDesc &d, const T *__restrict__ val, int c, int lane, uint64_t pol,
                                         G gather)
{
    if (d.half) return stencil_row_half<NB>(val, d.smask, c, lane, d.n, d.sP, pol, gather);
    return stencil_row<NB>(val, c, lane, d.n, d.sP, pol, gather);
}

// SELL and CSRW rows (uploaded CSR requests), out of line.
template <typename T, typename G>
__device__ __noinline__ T row_indexed(const SysDesc &d, const T *__restrict__ val, int c, int lane, uint64_t pol,
                                      G gather)
{
    const int n = d.n;
    const int *off = d.off, *col = d.col;
    if (d.fmt == FMT_SELL) {
        const int b = __ldg(off + c), L = (__ldg(off + c + 1) - b) >> 5;
        const int *cp = col + b + lane;
        const T *vp = val + b + lane;
        T s = T(0);
#pragma unroll 3
        for (int k = 0; k < L; ++k) s += ld_stream(vp + 32 * k, pol) * gather(ld_stream(cp + 32 * k, pol));
        return s;
    }
    T mine = T(0);
    const int r0 = c * kChunk;
    for (int rr = 0; rr < kChunk; ++rr) {
        const int i = r0 + rr;
        if (i >= n) break;
        const int b = __ldg(off + i), e = __ldg(off + i + 1);
        T s = T(0);
        for (int j = b + lane; j < e; j += 32) s += ld_stream(val + j, pol) * gather(ld_stream(col + j, pol));
        s = warp_sum(s);
        if (lane == rr) mine = s;
    }
    return mine;
}

// Row 32 c + lane of A v, v given by gather(j).
template <typename T, typename G>
__device__ __forceinline__ T row_spmv(const SysDesc &d, const T *__restrict__ val, int c, int lane, uint64_t pol,
                                      G gather)
{
    if (d.fmt == FMT_STENCIL) {
        if (d.sdim == 3) return stencil_any<T, 9>(d, val, c, lane, pol, gather);
        return stencil_any<T, 3>(d, val, c, lane, pol, gather);
    }
    return row_indexed<T>(d, val, c, lane, pol, gather);
}

// ------------------------------------------------------------------ system table

constexpr int kTabSmem = 2048;   // weighted starts of up to this many systems kept in shared memory

// Weighted start of every active system into shared memory (one barrier).
template <int K>
__device__ __forceinline__ void load_wb(const SysRun *tab, int nsys, int *s_wb)
{
    for (int k = threadIdx.x; k < min(nsys, kTabSmem); k += blockDim.x)
        s_wb[k] = __ldcg(K == 1 ? &tab[k].wb1 : &tab[k].wb2);
    __syncthreads();
}

// The last system whose weighted start is <= pos (binary search; shared
// memory when the table fits).
template <int K>
__device__ __forceinline__ int find_system(const SysRun *tab, int nsys, const int *s_wb, int pos)
{
    int lo = 0, hi = nsys - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int wb = nsys <= kTabSmem ? s_wb[mid] : __ldcg(K == 1 ? &tab[mid].wb1 : &tab[mid].wb2);
        if (wb <= pos) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The chunks of a system that one warp processes: first, first + step, ...
// below c1, out of the run [c0, c1).
struct Run {
    int c0, c1, first, step;
};

// The warp's share of kernel K's weighted chunk sequence: one contiguous
// range [P0, P1) of weight W / warps.  Chunk c of a system belongs to the
// warp whose range holds the chunk's start wb + c w, so every chunk has one
// owner.  body(slot, run) runs once per system the range touches.
template <int K, int NW, typename F>
__device__ __forceinline__ void for_warp_runs(const int *__restrict__ tb, const SysRun *tab, int nsys,
                                              const int *s_wb, F body)
{
    const long long W = __ldcg(tb + 3 + K);
    const int gw = blockIdx.x * NW + (threadIdx.x >> 5), nw = gridDim.x * NW;
    const int P0 = (int)((long long)gw * W / nw), P1 = (int)((long long)(gw + 1) * W / nw);
    if (P0 >= P1 || nsys <= 0) return;
    for (int si = find_system<K>(tab, nsys, s_wb, P0); si < nsys; ++si) {
        const int wb = nsys <= kTabSmem ? s_wb[si] : __ldcg(K == 1 ? &tab[si].wb1 : &tab[si].wb2);
        if (wb >= P1) break;
        const int wt = __ldcg(K == 1 ? &tab[si].w1 : &tab[si].w2), nch = __ldcg(&tab[si].nch);
        const int c0 = P0 > wb ? (P0 - wb + wt - 1) / wt : 0;
        const int c1 = min(nch, (P1 - wb + wt - 1) / wt);
        if (c0 < c1) body(__ldcg(&tab[si].slot), Run{c0, c1, c0, 1});
    }
}

// ------------------------------------------------------------------ reporting

// After the warp has written the partials of chunks [c0, c1) of its system
// (lane 0 writes them): report them to their groups; a completed group is
// summed; the completion of the last group runs fin(o) on the warp (o valid
// on every lane).  NQ quantities.
template <int NQ, typename F>
__device__ __forceinline__ void report(const WarpCtx &c, const Run &R, F fin)
{
    const int lane = threadIdx.x & 31;
    const SysDesc &d = c.d;
    if (lane == 0) __threadfence();
    for (int g = R.first / kGroup; g * kGroup < R.c1; ++g) {
        // the warp's chunks in group g: first + k step within [a, b)
        const int a = max(R.first, g * kGroup), b = min(R.c1, (g + 1) * kGroup);
        const int f = a + (R.first - a % R.step + R.step) % R.step;   // first chunk >= a of the residue
        const int cnt = f < b ? (b - f + R.step - 1) / R.step : 0;
        if (cnt == 0) continue;
        const int gsize = min(d.nchunks, (g + 1) * kGroup) - g * kGroup;
        int done = 0;
        if (lane == 0) {
            const unsigned old = atomicAdd(d.gcnt + g, (unsigned)cnt);
            done = old + (unsigned)cnt == (unsigned)gsize;
        }
        done = __shfl_sync(0xffffffffu, done, 0);
        if (!done) continue;
        // group g complete: sum its chunk partials (fixed xor tree)
        __threadfence();
        double v[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const int ch = g * kGroup + lane;
            v[q] = warp_sum(ch < d.nchunks ? __ldcg(d.part + (size_t)q * d.pstride + ch) : 0.0);
        }
        int last = 0;
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < NQ; ++q) d.gpart[(size_t)q * d.gstride + g] = v[q];
            d.gcnt[g] = 0u;
            __threadfence();
            const unsigned old = atomicAdd(d.ticket, 1u);
            last = old + 1u == (unsigned)d.ngroups;
            if (last) d.ticket[0] = 0u;
        }
        last = __shfl_sync(0xffffffffu, last, 0);
        if (!last) continue;
        // all groups complete: lane l sums groups l, l + 32, ... in order
        __threadfence();
        double o[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double w = 0.0;
            for (int k = lane; k < d.ngroups; k += 32) w += __ldcg(d.gpart + (size_t)q * d.gstride + k);
            o[q] = warp_sum(w);
        }
        fin(o);
    }
}

// ------------------------------------------------------------------ k1

template <typename T>
__device__ __forceinline__ void k1_range(const WarpCtx &c, SysState *st, const Run R, uint64_t pol)
{
    const int lane = threadIdx.x & 31;
    const SysDesc &d = c.d;
    const int n = d.n;
    const T beta = (T)c.s.beta;
    const bool b0 = c.s.pbuf == 0;
    const T *po = static_cast<const T *>(b0 ? d.p0 : d.p1);
    T *pn = static_cast<T *>(b0 ? d.p1 : d.p0);
    const T *z = static_cast<const T *>(d.z);
    T *ap = static_cast<T *>(d.ap);
    const T *val = sizeof(T) == 8 ? reinterpret_cast<const T *>(d.val64) : reinterpret_cast<const T *>(d.val32);
    auto gather = [=](int j) { return pnew_at(beta, po, z, j); };
    auto finish_row = [&](int ch, T s) {
        const int i = ch * kChunk + lane;
        double dp = 0.0;
        if (i < n) {
            const T pi = pnew_at(beta, po, z, i);
            pn[i] = pi;
            ap[i] = s;
            dp = (double)(pi * s);
        }
        return dp;
    };
    int ch = R.first;
    if (d.fmt == FMT_STENCIL && d.sdim == 2) {
        // 2-D stencil rows stream few bytes per chunk: two chunks per step
        // keep twice the loads in flight (FP64 too: 328.5 -> 330.8 solves/s
        // on the full request stream)
        for (; ch + R.step < R.c1; ch += 2 * R.step) {
            const int chb = ch + R.step;
            const T sa = stencil_any<T, 3>(d, val, ch, lane, pol, gather);
            const T sb = stencil_any<T, 3>(d, val, chb, lane, pol, gather);
            double da = finish_row(ch, sa), db = finish_row(chb, sb);
            da = warp_sum(da);
            db = warp_sum(db);
            if (lane == 0) {
                d.part[ch] = da;
                d.part[chb] = db;
            }
        }
    }
    for (; ch < R.c1; ch += R.step) {
        const double dp = warp_sum(finish_row(ch, row_spmv<T>(d, val, ch, lane, pol, gather)));
        if (lane == 0) d.part[ch] = dp;
    }
    const double rho = c.s.rho;
    const int pbuf = c.s.pbuf;
    report<1>(c, R, [&](const double *o) {
        if (lane == 0) {
            st->alpha = rho / o[0];
            st->pbuf = pbuf ^ 1;
            st->corr = 0;
        }
    });
}

// x + (double) x_low as the outer correction forms it, everywhere the same
// (a zero correction leaves x untouched)
__device__ __forceinline__ double xcorr(double x, float xl) { return xl == 0.0f ? x : __dadd_rn(x, (double)xl); }

__device__ void k2_finish(const SysState &cs, SysState *st, int *done, int ph, const double *o);

// Outer step of a mixed system (mpir.cc:125-128, 271-273, 308-326): the FP64
// residual of the corrected iterate, its FP32 copy and D^-1 r_low, the norms
// for the outer and first inner tests.  x itself is corrected by the update
// kernel, after every gather of this launch.  Out of line: runs once per
// outer step.
__device__ __noinline__ void k1_outer(const WarpCtx &c, SysState *st, const Run R, uint64_t pol)
{
    const int lane = threadIdx.x & 31;
    const SysDesc &d = c.d;
    const int n = d.n, ps = d.pstride;
    const double *b = d.b, *x = d.x;
    const float *xl = static_cast<const float *>(d.xl);
    float *rl = static_cast<float *>(d.r), *zl = static_cast<float *>(d.z);
    const float *dv = static_cast<const float *>(d.invd);
    auto gather = [=](int j) { return xcorr(__ldg(x + j), __ldg(xl + j)); };
    for (int ch = R.first; ch < R.c1; ch += R.step) {
        const int i = ch * kChunk + lane;
        const double s = row_spmv<double>(d, d.val64, ch, lane, pol, gather);
        double q0 = 0.0, q1 = 0.0, q2 = 0.0;
        if (i < n) {
            const double r = b[i] - s;
            const float f = (float)r;
            const float zf = zmul(f, dv[i]);
            rl[i] = f;
            zl[i] = zf;
            q0 = r * r;
            q1 = (double)(f * zf);
            q2 = (double)(f * f);
        }
        q0 = warp_sum(q0);
        q1 = warp_sum(q1);
        q2 = warp_sum(q2);
        if (lane == 0) {
            d.part[ch] = q0;
            d.part[ps + ch] = q1;
            d.part[2 * ps + ch] = q2;
        }
    }
    const SysState cs = c.s;
    const int ph = cs.phase;
    report<3>(c, R, [&](const double *o) {
        if (lane == 0) {
            k2_finish(cs, st, d.done, ph, o);
            st->corr = ph == PH_CORRECT ? 1 : 2;
        }
    });
}

// After an outer step: x += (double) x_low (corr 1), x_low = 0.
__device__ __forceinline__ void k2_corr(const WarpCtx &c, const Run R)
{
    const int lane = threadIdx.x & 31;
    const int n = c.d.n, corr = c.s.corr;
    double *x = c.d.x;
    float *xl = static_cast<float *>(c.d.xl);
    for (int ch = R.first; ch < R.c1; ch += R.step) {
        const int i = ch * kChunk + lane;
        if (i < n) {
            if (corr == 1) x[i] = xcorr(x[i], xl[i]);
            xl[i] = 0.0f;
        }
    }
}

// MINC: 256-thread CTAs per SM the registers are budgeted for (4: 64
// registers with some spilled; 3: 80 registers; B200LA_SERVE_K1_MINCTA)
template <int NW, int MINC = kMinCta256>
__global__ void __launch_bounds__(NW * 32, MINC * 8 / NW) k1_kernel(const SysDesc *__restrict__ sys,
                                                                       SysState *state, const int *__restrict__ tb)
{
    __shared__ WarpCtx ctx[NW];
    __shared__ int s_wb[kTabSmem];
    WarpCtx &c = ctx[threadIdx.x >> 5];
    const int nsys = __ldcg(tb);
    const SysRun *tab = reinterpret_cast<const SysRun *>(tb + kTabHdrWords);
    load_wb<1>(tab, nsys, s_wb);
    // the systems' values stream evict-first in L2 (full request stream:
    // 330.7 -> 337.0 solves/s against evict-normal)
    const uint64_t pol = l2_policy(1);
    for_warp_runs<1, NW>(tb, tab, nsys, s_wb, [&](int slot, const Run R) {
        warp_load(sys, state, slot, c);
        const int ph = c.s.phase;
        if (ph == PH_CG) k1_range<double>(c, state + slot, R, pol);
        else if (ph == PH_INNER) k1_range<float>(c, state + slot, R, pol);
        else if (ph == PH_OUTER || ph == PH_CORRECT) k1_outer(c, state + slot, R, pol);
    });
}

// ------------------------------------------------------------------ k2

// Lane 0 of the completing warp.  cs: the state as read before this launch
// changed it (nothing else writes it during the launch).
__device__ void k2_finish(const SysState &cs, SysState *st, int *done, int ph, const double *o)
{
    if (ph == PH_CG) {
        // cg.cc:222-247 with IterateControl::Check on ||r||
        const int it = cs.iter + 1;
        st->iter = it;
        const double res = sqrt(o[0]);
        st->res = res;
        const int s = check_cg(res, it, cs.res0, cs.abstol, cs.reltol, cs.divtol, cs.maxits);
        st->status = s;
        if (s == 0) {
            st->beta = o[1] / cs.rho;
            st->rho = o[1];
        } else {
            st->phase = PH_DONE;
            *done = s;
        }
    } else if (ph == PH_CG_START) {
        // cg.cc:164-200: r = b - A x0 (x0 = 0), z = M^-1 r, rho = r.z, Check(0)
        const double res = sqrt(o[0]);
        st->res = res;
        st->res0 = res;
        st->rho = o[1];
        st->beta = 0.0;
        const int s = check_cg(res, 0, res, cs.abstol, cs.reltol, cs.divtol, cs.maxits);
        st->status = s;
        if (s == 0) {
            st->phase = PH_CG;
        } else {
            st->phase = PH_DONE;
            *done = s;
        }
    } else if (ph == PH_INNER) {
        const int it = cs.inner_iter + 1;
        st->inner_iter = it;
        st->iter = cs.iter + 1;
        const double res = sqrt(o[0]);
        const int s = check_cg(res, it, cs.res_in0, cs.in_abstol, cs.in_reltol, cs.in_divtol, cs.in_maxits);
        if (s == 0) {
            st->beta = o[1] / cs.rho;
            st->rho = o[1];
        } else {
            st->phase = PH_CORRECT;
        }
    } else {
        // outer step of mpir.cc:125-128, 271-273, 308-326 (relative test
        // against the first outer residual)
        const double rn = sqrt(o[0]);
        const double res0 = ph == PH_OUTER ? rn : cs.res0;
        st->res0 = res0;
        st->res = rn;
        const bool cont = rn > cs.abstol && rn > cs.reltol * res0 && rn < cs.divtol && cs.outer < cs.max_outer;
        if (!cont) {
            const int s = rn < cs.abstol ? 1 : rn < cs.reltol * res0 ? 2 : rn >= cs.divtol ? 3 : 4;
            st->status = s;
            st->phase = PH_DONE;
            *done = s;
        } else {
            st->outer = cs.outer + 1;
            st->rho = o[1];
            const double ri = sqrt(o[2]);
            st->res_in0 = ri;
            st->inner_iter = 0;
            st->beta = 0.0;
            const int s = check_cg(ri, 0, ri, cs.in_abstol, cs.in_reltol, cs.in_divtol, cs.in_maxits);
            st->phase = s == 0 ? PH_INNER : PH_CORRECT;
        }
    }
}

template <typename T>
__device__ __forceinline__ void k2_update(const WarpCtx &c, SysState *st, const Run R)
{
    const int lane = threadIdx.x & 31;
    const SysDesc &d = c.d;
    const int n = d.n, ps = d.pstride;
    const T alpha = (T)c.s.alpha;
    T *x = sizeof(T) == 8 ? reinterpret_cast<T *>(d.x) : static_cast<T *>(d.xl);
    T *r = static_cast<T *>(d.r), *z = static_cast<T *>(d.z);
    const T *p = static_cast<const T *>(c.s.pbuf == 0 ? d.p0 : d.p1);
    const T *ap = static_cast<const T *>(d.ap), *dv = static_cast<const T *>(d.invd);
    // two chunks per step: the loads of both are in flight together
    for (int ch = R.first; ch < R.c1; ch += 2 * R.step) {
        const int chb = ch + R.step;
        const int ia = ch * kChunk + lane, ib = chb * kChunk + lane;
        const bool va = ia < n, vb = chb < R.c1 && ib < n;
        T xa = T(0), pa = T(0), ra = T(0), aa = T(0), da = T(0);
        T xb = T(0), pb = T(0), rb = T(0), ab = T(0), db = T(0);
        if (va) {
            xa = x[ia];
            pa = p[ia];
            ra = r[ia];
            aa = __ldcs(ap + ia);
            da = dv[ia];
        }
        if (vb) {
            xb = x[ib];
            pb = p[ib];
            rb = r[ib];
            ab = __ldcs(ap + ib);
            db = dv[ib];
        }
        double rra = 0.0, rza = 0.0, rrb = 0.0, rzb = 0.0;
        if (va) {
            const T ri = ra - alpha * aa, zi = zmul(ri, da);
            x[ia] = xa + alpha * pa;
            r[ia] = ri;
            z[ia] = zi;
            rra = (double)(ri * ri);
            rza = (double)(ri * zi);
        }
        if (vb) {
            const T ri = rb - alpha * ab, zi = zmul(ri, db);
            x[ib] = xb + alpha * pb;
            r[ib] = ri;
            z[ib] = zi;
            rrb = (double)(ri * ri);
            rzb = (double)(ri * zi);
        }
        rra = warp_sum(rra);
        rza = warp_sum(rza);
        rrb = warp_sum(rrb);
        rzb = warp_sum(rzb);
        if (lane == 0) {
            d.part[ch] = rra;
            d.part[ps + ch] = rza;
            if (chb < R.c1) {
                d.part[chb] = rrb;
                d.part[ps + chb] = rzb;
            }
        }
    }
    const SysState cs = c.s;
    const int ph = cs.phase;
    report<2>(c, R, [&](const double *o) {
        if (lane == 0) k2_finish(cs, st, d.done, ph, o);
    });
}

__device__ __forceinline__ void k2_start(const WarpCtx &c, SysState *st, const Run R)
{
    const int lane = threadIdx.x & 31;
    const SysDesc &d = c.d;
    const int n = d.n, ps = d.pstride;
    double *r = static_cast<double *>(d.r), *z = static_cast<double *>(d.z);
    const double *b = d.b, *dv = static_cast<const double *>(d.invd);
    for (int ch = R.first; ch < R.c1; ch += R.step) {
        const int i = ch * kChunk + lane;
        double rr = 0.0, rz = 0.0;
        if (i < n) {
            const double ri = b[i];
            const double zi = zmul(ri, dv[i]);
            r[i] = ri;
            z[i] = zi;
            rr = ri * ri;
            rz = ri * zi;
        }
        rr = warp_sum(rr);
        rz = warp_sum(rz);
        if (lane == 0) {
            d.part[ch] = rr;
            d.part[ps + ch] = rz;
        }
    }
    const SysState cs = c.s;
    report<2>(c, R, [&](const double *o) {
        if (lane == 0) k2_finish(cs, st, d.done, PH_CG_START, o);
    });
}

template <int NW>
__global__ void __launch_bounds__(NW * 32, kMinCta256 * 8 / NW) k2_kernel(const SysDesc *__restrict__ sys,
                                                                       SysState *state, const int *__restrict__ tb)
{
    __shared__ WarpCtx ctx[NW];
    __shared__ int s_wb[kTabSmem];
    WarpCtx &c = ctx[threadIdx.x >> 5];
    const int nsys = __ldcg(tb);
    const SysRun *tab = reinterpret_cast<const SysRun *>(tb + kTabHdrWords);
    load_wb<2>(tab, nsys, s_wb);
    for_warp_runs<2, NW>(tb, tab, nsys, s_wb, [&](int slot, const Run R) {
        warp_load(sys, state, slot, c);
        const int ph = c.s.phase;
        SysState *st = state + slot;
        if (c.s.corr) k2_corr(c, R);   // the outer step ran in k1 (the phase is already the next one)
        else if (ph == PH_CG) k2_update<double>(c, st, R);
        else if (ph == PH_INNER) k2_update<float>(c, st, R);
        else if (ph == PH_CG_START) k2_start(c, st, R);
    });
}

// ------------------------------------------------------------ slot build

__global__ void build_slot_kernel(SysDesc d, const int *__restrict__ row, const int *__restrict__ col,
                                  const double *__restrict__ val)
{
    const int n = d.n, rows = d.nchunks * kChunk;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        int rb = 0, re = 0;
        if (i < n) {
            rb = row[i];
            re = row[i + 1];
        }
        if (d.fmt == FMT_STENCIL) {
            // values zero-filled before; each stored entry to its position
            // (the half layout is filled by half_build_slot_kernel)
            if (i < n && !d.half) {
                const int c = i / kChunk, lane = i % kChunk, L = d.sL, G4 = L / 4;
                const size_t base = (size_t)c * kChunk * L + lane;
                const size_t base32 = (size_t)c * kChunk * L;   // FP32: groups of four, then the tail
                double *ov = const_cast<double *>(d.val64);
                float *of = const_cast<float *>(d.val32);
                for (int j = rb; j < re; ++j) {
                    const int dl = col[j] - i;
                    for (int k = 0; k < L; ++k)
                        if (stencil_delta(d.sdim, d.sP, k) == dl) {
                            ov[base + (size_t)kChunk * k] = val[j];
                            if (d.mixed)
                                of[base32 + (k < 4 * G4 ? (size_t)(k / 4) * 128 + 4 * lane + k % 4
                                                        : (size_t)G4 * 128 + (size_t)(k - 4 * G4) * 32 + lane)] =
                                    (float)val[j];
                        }
                }
            }
        } else if (d.fmt == FMT_SELL) {
            const int c = i / kChunk, lane = i % kChunk;
            const int b = d.off[c], L = (d.off[c + 1] - b) / kChunk;
            int *oc = const_cast<int *>(d.col);
            double *ov = const_cast<double *>(d.val64);
            float *of = const_cast<float *>(d.val32);
            for (int k = 0; k < L; ++k) {
                const int j = rb + k;
                const size_t pos = (size_t)b + (size_t)kChunk * k + lane;
                int cj;
                double v;
                if (j < re) {
                    cj = col[j];
                    v = val[j];
                } else {
                    cj = i < n ? i : 0;
                    v = 0.0;
                }
                oc[pos] = cj;
                ov[pos] = v;
                if (d.mixed) of[pos] = (float)v;
            }
        } else if (d.mixed && i < n) {
            float *of = const_cast<float *>(d.val32);
            for (int j = rb; j < re; ++j) of[j] = (float)val[j];
        }
        if (i < n) {
            // extract_invdiagelements (lmp/lmatrix_csr_cpu.cc:2414-2431); the
            // FP32 Jacobi of the mixed form rounds the FP64 1 / a_ii once
            double dg = 0.0;
            for (int j = rb; j < re; ++j)
                if (col[j] == i) dg = val[j];
            const double inv = 1.0 / dg;
            if (d.mixed) const_cast<float *>(static_cast<const float *>(d.invd))[i] = (float)inv;
            else const_cast<double *>(static_cast<const double *>(d.invd))[i] = inv;
        }
    }
}

// Half stencil, pass 1: smask[c] bit l = row 32 c + l has no off-diagonal
// value other than +0.0 (rows past n count as such).
__global__ void half_mask_slot_kernel(SysDesc d, const int *__restrict__ row, const int *__restrict__ col,
                                      const double *__restrict__ val)
{
    unsigned *mask = const_cast<unsigned *>(d.smask);
    const int rows = d.nchunks * kChunk;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        bool ident = true;
        if (i < d.n)
            for (int j = row[i]; j < row[i + 1]; ++j)
                if (col[j] != i && __double_as_longlong(val[j]) != 0) ident = false;
        const unsigned bits = __ballot_sync(0xffffffffu, ident);
        if ((threadIdx.x & 31) == 0) mask[i >> 5] = bits;
    }
}

// Half stencil, pass 2: the diagonal and upper half of every row, FP64 and
// (mixed) FP32.  An identity row stores in its upper slots the transposed
// entries (i + off, i) that its neighbours read as their lower half.  Pairs
// of rows that are not identity rows must hold the same value bit for bit
// in both directions; otherwise smask[nchunks] is set.
__global__ void half_build_slot_kernel(SysDesc d, const int *__restrict__ row, const int *__restrict__ col,
                                       const double *__restrict__ val)
{
    const int n = d.n, dim = d.sdim, P = d.sP, U = half_u(dim), H64 = half_len64(dim), H32 = half_len32(dim);
    const unsigned *mask = d.smask;
    unsigned *asym = const_cast<unsigned *>(d.smask) + d.nchunks;
    double *ov = const_cast<double *>(d.val64);
    float *of = const_cast<float *>(d.val32);
    auto find = [&](int r, int cc) -> double {
        for (int j = row[r]; j < row[r + 1]; ++j)
            if (col[j] == cc) return val[j];
        return 0.0;
    };
    auto flagged = [&](int q) { return (mask[q >> 5] >> (q & 31)) & 1u; };
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const bool fr = flagged(i);
        auto upper = [&](int off) -> double {
            const int q = i + off;
            const bool inr = q < n;
            if (fr) return inr ? find(q, i) : 0.0;
            const double v = inr ? find(i, q) : 0.0;
            if (inr && !flagged(q) && __double_as_longlong(v) != __double_as_longlong(find(q, i))) atomicOr(asym, 1u);
            return v;
        };
        const int c = i / kChunk, lane = i % kChunk;
        const double dg = find(i, i), p1 = upper(1);
        double *o64 = ov + (size_t)c * kChunk * H64 + lane;
        o64[0] = dg;
        o64[kChunk] = p1;
        float *o32 = d.mixed ? of + (size_t)c * kChunk * H32 : nullptr;
        for (int u = 0; u < U; ++u)
            for (int m = 0; m < 3; ++m) {
                const double v = upper(band_offset(dim, P, U + 1 + u) + m - 1);
                o64[kChunk * (2 + 3 * u + m)] = v;
                if (o32) o32[128 * u + 4 * lane + m] = (float)v;
            }
        if (o32) {
            o32[4 * lane + 3] = (float)dg;
            if (U >= 2) o32[128 + 4 * lane + 3] = (float)p1;
            else o32[128 * U + lane] = (float)p1;
        }
    }
}

}  // namespace

cudaError_t launch_round(int nw, int grid, const SysDesc *sys, SysState *state, const int *tab, cudaStream_t st)
{
    static const int minc = [] {
        const char *e = std::getenv("B200LA_SERVE_K1_MINCTA");
        return e ? std::atoi(e) : kMinCta256;
    }();
    if (nw == 4) {
        if (minc == 3) k1_kernel<4, 3><<<grid, 128, 0, st>>>(sys, state, tab);
        else k1_kernel<4><<<grid, 128, 0, st>>>(sys, state, tab);
        k2_kernel<4><<<grid, 128, 0, st>>>(sys, state, tab);
    } else {
        if (minc == 3) k1_kernel<8, 3><<<grid, 256, 0, st>>>(sys, state, tab);
        else k1_kernel<8><<<grid, 256, 0, st>>>(sys, state, tab);
        k2_kernel<8><<<grid, 256, 0, st>>>(sys, state, tab);
    }
    return cudaGetLastError();
}

cudaError_t launch_build_slot(const SysDesc &d, const int *row, const int *col, const double *val, cudaStream_t st)
{
    const long long rows = (long long)d.nchunks * kChunk;
    const int g = (int)std::min<long long>((rows + 255) / 256, 148LL * 16);
    if (d.fmt == FMT_STENCIL && d.half) {
        half_mask_slot_kernel<<<g, 256, 0, st>>>(d, row, col, val);
        half_build_slot_kernel<<<g, 256, 0, st>>>(d, row, col, val);
    }
    build_slot_kernel<<<g, 256, 0, st>>>(d, row, col, val);
    return cudaGetLastError();
}

}  // namespace srv
}  // namespace b200
