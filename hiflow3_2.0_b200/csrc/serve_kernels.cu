// serve_kernels.cu -- batched Krylov kernels of the solve server (sm_100a).
//
// One batch iteration is two launches over the system table:
//   k1  SpMV  Ap = A p_new with p_new = beta p + z formed on the fly at every
//       gathered column (and stored for the own rows into the other of two p
//       buffers), with the partials of p_new.Ap; on completion of a system
//       alpha = rho / p.Ap and the p buffer flips (CG, inner CG).  Mixed
//       systems between two inner solves apply x += (double) x_low here.
//   k2  update x += alpha p, r -= alpha Ap, z = D^-1 r with the partials of
//       r.r and r.z; on completion IterateControl::Check
//       (src/common/iterate_control.cc:84-110) and beta, rho.  Start phases
//       (CG: r = b; mixed: r = b - A x in FP64, r_low = (float) r) run here.
// Folding the p-update of CG<LAD> (cg.cc:240-246) into the next product
// removes a launch and a pass per iteration; the update is written with
// explicit roundings so that every gathering thread forms the same p_new as
// the thread that stores it.
//
// Work split: the active systems' 32-row chunks form one sequence; each warp
// takes one contiguous range of it, with no CTA barrier.  A warp loads a
// system's descriptor and state into its own shared-memory slot when its
// range enters the system.  Reductions: one partial per chunk; a warp reports
// its run of each system's chunks to the run's groups of 32 chunks, the warp
// completing a group sums its partials (fixed shuffle tree) and reports the
// group to the system, and the warp completing the last group sums the group
// partials in a fixed order and runs the finaliser.  Counters are reset by
// their completers.  Operator values and indices are streamed past L1,
// gathered vectors go through L1.
#include <cuda_runtime.h>

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

// Stencil row, FP32: the row's positions in groups of four per lane (one
// 16-byte load each), then the bands.
template <int NB, typename G>
__device__ __forceinline__ float stencil_row(const float *__restrict__ val, int c, int lane, int n, int P,
                                             uint64_t pol, G gather)
{
    constexpr int DIM = NB == 9 ? 3 : 2, L = 3 * NB, GR = (L + 3) / 4;
    const int r0 = c * kChunk, i = r0 + lane, he = lane == 0 ? r0 - 1 : r0 + 32;
    const float4 *v = reinterpret_cast<const float4 *>(val + (size_t)c * kChunk * 4 * GR) + lane;
    float a[4 * GR];
#pragma unroll
    for (int g = 0; g < GR; ++g) {
        float4 q;
        asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
            : "=f"(q.x), "=f"(q.y), "=f"(q.z), "=f"(q.w)
            : "l"(v + 32 * g), "l"(pol));
        a[4 * g] = q.x;
        a[4 * g + 1] = q.y;
        a[4 * g + 2] = q.z;
        a[4 * g + 3] = q.w;
    }
    float s = 0.0f;
#pragma unroll
    for (int b = 0; b < NB; ++b)
        band(s, a[3 * b], a[3 * b + 1], a[3 * b + 2], i, he, band_offset(DIM, P, b), n, lane, gather);
    return s;
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
        if (d.sdim == 3) return stencil_row<9>(val, c, lane, d.n, d.sP, pol, gather);
        return stencil_row<3>(val, c, lane, d.n, d.sP, pol, gather);
    }
    return row_indexed<T>(d, val, c, lane, pol, gather);
}

// ------------------------------------------------------------------ system table

constexpr int kTabSmem = 2048;   // first chunks of up to this many systems kept in shared memory

// First chunk of every active system into shared memory (one barrier).
__device__ __forceinline__ void load_cbeg(const SysRun *tab, int nsys, int *s_cbeg)
{
    for (int k = threadIdx.x; k < min(nsys, kTabSmem); k += blockDim.x) s_cbeg[k] = __ldcg(&tab[k].cbeg);
    __syncthreads();
}

// The system whose chunks contain g (binary search; shared memory when the
// table fits).
__device__ __forceinline__ int find_system(const SysRun *tab, int nsys, const int *s_cbeg, int g)
{
    int lo = 0, hi = nsys - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int cb = nsys <= kTabSmem ? s_cbeg[mid] : __ldcg(&tab[mid].cbeg);
        if (cb <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ------------------------------------------------------------------ reporting

// After the warp has written the partials of chunks [c0, c1) of its system
// (lane 0 writes them): report them to their groups; a completed group is
// summed; the completion of the last group runs fin(o) on the warp (o valid
// on every lane).  NQ quantities.
template <int NQ, typename F>
__device__ __forceinline__ void report(const WarpCtx &c, int c0, int c1, F fin)
{
    const int lane = threadIdx.x & 31;
    const SysDesc &d = c.d;
    if (lane == 0) __threadfence();
    for (int g = c0 / kGroup; g * kGroup < c1; ++g) {
        const int a = max(c0, g * kGroup), b = min(c1, (g + 1) * kGroup);
        const int gsize = min(d.nchunks, (g + 1) * kGroup) - g * kGroup;
        int done = 0;
        if (lane == 0) {
            const unsigned old = atomicAdd(d.gcnt + g, (unsigned)(b - a));
            done = old + (unsigned)(b - a) == (unsigned)gsize;
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
__device__ __forceinline__ void k1_range(const WarpCtx &c, SysState *st, int c0, int c1, uint64_t pol)
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
    for (int ch = c0; ch < c1; ++ch) {
        const int i = ch * kChunk + lane;
        const T s = row_spmv<T>(d, val, ch, lane, pol, gather);
        double dp = 0.0;
        if (i < n) {
            const T pi = pnew_at(beta, po, z, i);
            pn[i] = pi;
            ap[i] = s;
            dp = (double)(pi * s);
        }
        dp = warp_sum(dp);
        if (lane == 0) d.part[ch] = dp;
    }
    const double rho = c.s.rho;
    const int pbuf = c.s.pbuf;
    report<1>(c, c0, c1, [&](const double *o) {
        if (lane == 0) {
            st->alpha = rho / o[0];
            st->pbuf = pbuf ^ 1;
        }
    });
}

__device__ __forceinline__ void k1_correct(const WarpCtx &c, int c0, int c1)
{
    const int lane = threadIdx.x & 31;
    const int n = c.d.n;
    double *x = c.d.x;
    const float *xl = static_cast<const float *>(c.d.xl);
    for (int ch = c0; ch < c1; ++ch) {
        const int i = ch * kChunk + lane;
        if (i < n) x[i] += (double)xl[i];
    }
}

template <int NW>
__global__ void __launch_bounds__(NW * 32, kMinCta256 * 8 / NW) k1_kernel(const SysDesc *__restrict__ sys,
                                                                       SysState *state, const int *__restrict__ tb)
{
    __shared__ WarpCtx ctx[NW];
    __shared__ int s_cbeg[kTabSmem];
    WarpCtx &c = ctx[threadIdx.x >> 5];
    const int nsys = __ldcg(tb), T = __ldcg(tb + 1), C = __ldcg(tb + 2);
    const SysRun *tab = reinterpret_cast<const SysRun *>(tb + kTabHdrWords);
    load_cbeg(tab, nsys, s_cbeg);
    const uint64_t pol = l2_policy(0);
    const int gw = blockIdx.x * NW + (threadIdx.x >> 5), nw = gridDim.x * NW;
    (void)C;
    // one contiguous range of the chunk sequence per warp: runs within a
    // system are long, so a warp reports about once per system it touches
    const int g0 = (int)((long long)gw * T / nw), g1 = (int)((long long)(gw + 1) * T / nw);
    int si = 0, loaded = -1;
    if (g0 < g1) {
        si = find_system(tab, nsys, s_cbeg, g0);
        for (int g = g0; g < g1;) {
            const int slot = __ldcg(&tab[si].slot), cb = __ldcg(&tab[si].cbeg), nch = __ldcg(&tab[si].nch);
            const int e = min(g1, cb + nch);
            if (slot != loaded) {
                warp_load(sys, state, slot, c);
                loaded = slot;
            }
            const int ph = c.s.phase, c0 = g - cb, c1 = e - cb;
            if (ph == PH_CG) k1_range<double>(c, state + slot, c0, c1, pol);
            else if (ph == PH_INNER) k1_range<float>(c, state + slot, c0, c1, pol);
            else if (ph == PH_CORRECT) k1_correct(c, c0, c1);
            g = e;
            if (g < g1) ++si;
        }
    }
}

// ------------------------------------------------------------------ k2

// Lane 0 of the completing warp.  cs: the state as read before this launch
// changed it (nothing else writes it during the launch).
__device__ __forceinline__ void k2_finish(const SysState &cs, SysState *st, int *done, int ph, const double *o)
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
__device__ __forceinline__ void k2_update(const WarpCtx &c, SysState *st, int c0, int c1)
{
    const int lane = threadIdx.x & 31;
    const SysDesc &d = c.d;
    const int n = d.n, ps = d.pstride;
    const T alpha = (T)c.s.alpha;
    T *x = sizeof(T) == 8 ? reinterpret_cast<T *>(d.x) : static_cast<T *>(d.xl);
    T *r = static_cast<T *>(d.r), *z = static_cast<T *>(d.z);
    const T *p = static_cast<const T *>(c.s.pbuf == 0 ? d.p0 : d.p1);
    const T *ap = static_cast<const T *>(d.ap), *dv = static_cast<const T *>(d.invd);
    for (int ch = c0; ch < c1; ++ch) {
        const int i = ch * kChunk + lane;
        double rr = 0.0, rz = 0.0;
        if (i < n) {
            const T xi = x[i] + alpha * p[i];
            const T ri = r[i] - alpha * __ldcs(ap + i);
            const T zi = zmul(ri, dv[i]);
            x[i] = xi;
            r[i] = ri;
            z[i] = zi;
            rr = (double)(ri * ri);
            rz = (double)(ri * zi);
        }
        rr = warp_sum(rr);
        rz = warp_sum(rz);
        if (lane == 0) {
            d.part[ch] = rr;
            d.part[ps + ch] = rz;
        }
    }
    const SysState cs = c.s;
    const int ph = cs.phase;
    report<2>(c, c0, c1, [&](const double *o) {
        if (lane == 0) k2_finish(cs, st, d.done, ph, o);
    });
}

__device__ __forceinline__ void k2_start(const WarpCtx &c, SysState *st, int c0, int c1)
{
    const int lane = threadIdx.x & 31;
    const SysDesc &d = c.d;
    const int n = d.n, ps = d.pstride;
    double *r = static_cast<double *>(d.r), *z = static_cast<double *>(d.z);
    const double *b = d.b, *dv = static_cast<const double *>(d.invd);
    for (int ch = c0; ch < c1; ++ch) {
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
    report<2>(c, c0, c1, [&](const double *o) {
        if (lane == 0) k2_finish(cs, st, d.done, PH_CG_START, o);
    });
}

// Runs once per outer step of a mixed system: kept out of line so that its
// registers do not constrain the per-iteration update.
__device__ __noinline__ void k2_outer(const WarpCtx &c, SysState *st, int c0, int c1, uint64_t pol)
{
    const int lane = threadIdx.x & 31;
    const SysDesc &d = c.d;
    const int n = d.n, ps = d.pstride;
    const double *b = d.b, *x = d.x;
    float *rl = static_cast<float *>(d.r), *zl = static_cast<float *>(d.z), *xl = static_cast<float *>(d.xl);
    const float *dv = static_cast<const float *>(d.invd);
    auto gather = [=](int j) { return __ldg(x + j); };
    for (int ch = c0; ch < c1; ++ch) {
        const int i = ch * kChunk + lane;
        const double s = row_spmv<double>(d, d.val64, ch, lane, pol, gather);
        double q0 = 0.0, q1 = 0.0, q2 = 0.0;
        if (i < n) {
            const double r = b[i] - s;
            const float f = (float)r;
            const float zf = zmul(f, dv[i]);
            rl[i] = f;
            zl[i] = zf;
            xl[i] = 0.0f;
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
    report<3>(c, c0, c1, [&](const double *o) {
        if (lane == 0) k2_finish(cs, st, d.done, ph, o);
    });
}

template <int NW>
__global__ void __launch_bounds__(NW * 32, kMinCta256 * 8 / NW) k2_kernel(const SysDesc *__restrict__ sys,
                                                                       SysState *state, const int *__restrict__ tb)
{
    __shared__ WarpCtx ctx[NW];
    __shared__ int s_cbeg[kTabSmem];
    WarpCtx &c = ctx[threadIdx.x >> 5];
    const int nsys = __ldcg(tb), T = __ldcg(tb + 1), C = __ldcg(tb + 2);
    const SysRun *tab = reinterpret_cast<const SysRun *>(tb + kTabHdrWords);
    load_cbeg(tab, nsys, s_cbeg);
    const uint64_t pol = l2_policy(0);
    const int gw = blockIdx.x * NW + (threadIdx.x >> 5), nw = gridDim.x * NW;
    (void)C;
    // one contiguous range of the chunk sequence per warp: runs within a
    // system are long, so a warp reports about once per system it touches
    const int g0 = (int)((long long)gw * T / nw), g1 = (int)((long long)(gw + 1) * T / nw);
    int si = 0, loaded = -1;
    if (g0 < g1) {
        si = find_system(tab, nsys, s_cbeg, g0);
        for (int g = g0; g < g1;) {
            const int slot = __ldcg(&tab[si].slot), cb = __ldcg(&tab[si].cbeg), nch = __ldcg(&tab[si].nch);
            const int e = min(g1, cb + nch);
            if (slot != loaded) {
                warp_load(sys, state, slot, c);
                loaded = slot;
            }
            const int ph = c.s.phase, c0 = g - cb, c1 = e - cb;
            SysState *st = state + slot;
            if (ph == PH_CG) k2_update<double>(c, st, c0, c1);
            else if (ph == PH_INNER) k2_update<float>(c, st, c0, c1);
            else if (ph == PH_CG_START) k2_start(c, st, c0, c1);
            else if (ph == PH_OUTER || ph == PH_CORRECT) k2_outer(c, st, c0, c1, pol);
            g = e;
            if (g < g1) ++si;
        }
    }
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
            if (i < n) {
                const int c = i / kChunk, lane = i % kChunk, L = d.sL, GR = (L + 3) / 4;
                const size_t base = (size_t)c * kChunk * L + lane;
                const size_t base32 = (size_t)c * kChunk * 4 * GR + 4 * lane;
                double *ov = const_cast<double *>(d.val64);
                float *of = const_cast<float *>(d.val32);
                for (int j = rb; j < re; ++j) {
                    const int dl = col[j] - i;
                    for (int k = 0; k < L; ++k)
                        if (stencil_delta(d.sdim, d.sP, k) == dl) {
                            ov[base + (size_t)kChunk * k] = val[j];
                            if (d.mixed) of[base32 + (size_t)(k / 4) * 128 + k % 4] = (float)val[j];
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

}  // namespace

cudaError_t launch_round(int nw, int grid, const SysDesc *sys, SysState *state, const int *tab, cudaStream_t st)
{
    if (nw == 4) {
        k1_kernel<4><<<grid, 128, 0, st>>>(sys, state, tab);
        k2_kernel<4><<<grid, 128, 0, st>>>(sys, state, tab);
    } else {
        k1_kernel<8><<<grid, 256, 0, st>>>(sys, state, tab);
        k2_kernel<8><<<grid, 256, 0, st>>>(sys, state, tab);
    }
    return cudaGetLastError();
}

cudaError_t launch_build_slot(const SysDesc &d, const int *row, const int *col, const double *val, cudaStream_t st)
{
    const long long rows = (long long)d.nchunks * kChunk;
    const int g = (int)std::min<long long>((rows + 255) / 256, 148LL * 16);
    build_slot_kernel<<<g, 256, 0, st>>>(d, row, col, val);
    return cudaGetLastError();
}

}  // namespace srv
}  // namespace b200
