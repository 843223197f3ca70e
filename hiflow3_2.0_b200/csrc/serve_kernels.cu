// serve_kernels.cu -- batched Krylov kernels of the solve server (sm_100a).
//
// One batch iteration is two launches over the tile table:
//   k1  SpMV  Ap = A p_new with p_new = beta p + D^-1 r formed on the fly at
//       every gathered column (and stored for the own rows into the other of
//       two p buffers), with the chunk partials of p_new.Ap; the CTA
//       completing a system's tiles sets alpha = rho / p.Ap and flips the p
//       buffer (CG, inner CG).  Mixed systems between two inner solves apply
//       the correction x += (double) x_low here.
//   k2  update x += alpha p, r -= alpha Ap with the partials of r.r and
//       r.(D^-1 r); the completing CTA runs IterateControl::Check
//       (src/common/iterate_control.cc:84-110) and sets beta, rho.  Start
//       phases (CG: r = b; mixed: r = b - A x in FP64, r_low = (float) r)
//       run here too.
// Folding the p-update of CG<LAD> (cg.cc:240-246) into the next product
// removes a launch and a pass per iteration; the update is written with
// explicit roundings so that every gathering thread forms the same p_new as
// the thread that stores it.
// Each CTA takes a contiguous range of tiles and keeps the current system's
// descriptor and state in shared memory while consecutive tiles share it.
// Systems whose phase has no work in a launch skip their tiles.  Operator
// values and indices are streamed past L1; gathered vectors go through L1.
#include <cuda_runtime.h>

#include "common.cuh"
#include "serve.cuh"

#ifndef B200LA_SRV_MINCTA
#define B200LA_SRV_MINCTA 2
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

struct TileCtx {
    SysDesc d;
    SysState s;
    Tile t;
    int next_sys;    // system of the CTA's next tile (-1: none)
};

// Tile walk of one CTA over its contiguous range [t0, t1).  Warp 0 keeps the
// next tile's entry in flight while the current tile is processed; the
// system's descriptor and state are fetched only when the system changes
// (consecutive tiles of one system share them).  All threads call next().
struct TileWalk {
    int t, t1, cached;
    int nx;          // warp 0, lanes 0..3: word `lane` of tile t + 1
    __device__ __forceinline__ void prefetch(const Tile *tiles)
    {
        if (threadIdx.x < 4) nx = (t + 1 < t1) ? __ldcg(reinterpret_cast<const int *>(tiles + t + 1) + threadIdx.x) : -1;
    }
    // Make tile t current in c (first call: loads it; later calls: commits
    // the prefetched entry), then prefetch t + 1.
    __device__ __forceinline__ void enter(const SysDesc *sys, const SysState *state, const Tile *tiles, TileCtx &c,
                                          bool first)
    {
        __syncthreads();
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            int w = -1;
            if (first) {
                if (lane < 4) w = __ldcg(reinterpret_cast<const int *>(tiles + t) + lane);
            } else {
                w = nx;
            }
            const int s = __shfl_sync(0xffffffffu, w, 0);
            if (lane < 4) reinterpret_cast<int *>(&c.t)[lane] = w;
            if (s != cached) {
                constexpr int dw = (int)(sizeof(SysDesc) / sizeof(int));
                constexpr int sw = (int)(sizeof(SysState) / sizeof(int));
                const int *src = reinterpret_cast<const int *>(sys + s);
                const int *sst = reinterpret_cast<const int *>(state + s);
                for (int k = lane; k < dw; k += 32) reinterpret_cast<int *>(&c.d)[k] = __ldcg(src + k);
                for (int k = lane; k < sw; k += 32) reinterpret_cast<int *>(&c.s)[k] = __ldcg(sst + k);
            }
            prefetch(tiles);
        }
        __syncthreads();
        cached = c.t.sys;
    }
    // After the tile's work: publish the next tile's system (the prefetched
    // entry has arrived by now) for the end-of-run test.
    __device__ __forceinline__ void publish_next(TileCtx &c)
    {
        if (threadIdx.x < 32) {
            const int ns = __shfl_sync(0xffffffffu, nx, 0);
            if (threadIdx.x == 0) c.next_sys = (t + 1 < t1) ? ns : -1;
        }
        __syncthreads();
    }
};

// Ticket of a system's tiles in one launch: a CTA reports a run of `run`
// consecutive tiles of one system at once.  The writers of the run's chunk
// partials (lane 0 of every warp) fence them first.
__device__ __forceinline__ bool run_done(unsigned *ticket, int run, int ntiles, bool &s_last)
{
    if ((threadIdx.x & 31) == 0) __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const bool l = atomicAdd(ticket, (unsigned)run) + (unsigned)run == (unsigned)ntiles;
        if (l) atomicExch(ticket, 0u);
        s_last = l;
    }
    __syncthreads();
    const bool l = s_last;
    if (l) __threadfence();
    return l;
}

// Sum of the chunk partials part[q][0..nch) (rows of pstride) in a fixed
// order: virtual lane v of 256 sums the chunk pairs (2v, 2v+1), (2v+512,
// 2v+513), ... in index order; the 8 virtual warps fold by a fixed shuffle
// tree and their sums add in order.  The order is the same for 128 or 256
// threads; the result is on thread 0.
template <int NQ, int NW>
__device__ __forceinline__ void fin_sum(const double *part, int nch, int pstride, double (&o)[NQ], double *sm)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int rep = 0; rep < kFinLanes / (NW * 32); ++rep) {
        const int v = threadIdx.x + rep * NW * 32;
        double w[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) w[q] = 0.0;
#pragma unroll 4
        for (int c = 2 * v; c < nch; c += 2 * kFinLanes) {
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const double2 a = __ldcg(reinterpret_cast<const double2 *>(part + (size_t)q * pstride + c));
                w[q] += a.x;
                if (c + 1 < nch) w[q] += a.y;
            }
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const double s = warp_sum(w[q]);
            if (lane == 0) sm[q * 8 + (v >> 5)] = s;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double s = 0.0;
            for (int k = 0; k < 8; ++k) s += sm[q * 8 + k];
            o[q] = s;
        }
    }
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

// SELL row sum, entries added in column order in batches of 9: every load of
// a batch is issued before its first product.
template <typename T, typename G>
__device__ __forceinline__ T sell_row(const int *__restrict__ cp, const T *__restrict__ vp, int L, uint64_t pol,
                                      G gather)
{
    constexpr int B = 9;
    T s = T(0);
    for (int k0 = 0; k0 < L; k0 += B) {
        int cj[B];
        T a[B];
#pragma unroll
        for (int k = 0; k < B; ++k) {
            if (k0 + k < L) {
                cj[k] = ld_stream(cp + 32 * (k0 + k), pol);
                a[k] = ld_stream(vp + 32 * (k0 + k), pol);
            }
        }
#pragma unroll
        for (int k = 0; k < B; ++k)
            if (k0 + k < L) s += a[k] * gather(cj[k]);
    }
    return s;
}

// Stencil row sum (FMT_STENCIL).  The positions form bands of three
// consecutive columns (di = -1, 0, 1 around i + d); lane l gathers only the
// band centre i + d, takes its left / right neighbours from lanes l - 1 /
// l + 1, and lanes 0 / 31 gather the one column beyond the chunk.  Products
// are added in column order, each gathered value formed by gather(j) exactly
// as a direct gather would.  Columns outside [0, n) belong to zero entries
// and are clamped into range.
template <typename T, int DIM, int U, typename G>
__device__ __forceinline__ void stencil_rows(const T *__restrict__ val, int L, const int (&cc)[U], int lane, int n,
                                             int P, uint64_t pol, G gather, T (&s)[U])
{
    constexpr int NB = DIM == 3 ? 9 : 3;
    const bool edge = lane == 0 || lane == 31;
#pragma unroll
    for (int u = 0; u < U; ++u) s[u] = T(0);
#pragma unroll
    for (int b0 = 0; b0 < NB; b0 += 3) {
        T a[U][9], w[U][3], h[U][3];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int r0 = cc[u] * kChunk, i = r0 + lane;
            const int he = lane == 0 ? r0 - 1 : r0 + 32;     // halo column before the band offset
            const T *vp = val + (size_t)cc[u] * kChunk * L + lane;
#pragma unroll
            for (int bb = 0; bb < 3; ++bb) {
                const int band = b0 + bb;
                const int d = DIM == 3 ? ((band / 3 - 1) * P + (band % 3 - 1)) * P : (band - 1) * P;
#pragma unroll
                for (int m = 0; m < 3; ++m) a[u][3 * bb + m] = ld_stream(vp + 32 * (3 * band + m), pol);
                w[u][bb] = gather(min(max(i + d, 0), n - 1));
                h[u][bb] = edge ? gather(min(max(he + d, 0), n - 1)) : T(0);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
#pragma unroll
            for (int bb = 0; bb < 3; ++bb) {
                T left = __shfl_up_sync(0xffffffffu, w[u][bb], 1);
                T right = __shfl_down_sync(0xffffffffu, w[u][bb], 1);
                if (lane == 0) left = h[u][bb];
                if (lane == 31) right = h[u][bb];
                s[u] += a[u][3 * bb] * left;
                s[u] += a[u][3 * bb + 1] * w[u][bb];
                s[u] += a[u][3 * bb + 2] * right;
            }
        }
        // keep one group of three bands in flight at a time (register budget)
        if (b0 + 3 < NB) asm volatile("" ::: "memory");
    }
}

template <typename T, typename G>
__device__ __noinline__ T row_spmv_indexed(const SysDesc &d, const T *__restrict__ val, int c, int lane,
                                           uint64_t pol, G gather);

// Row 32 c + lane of A v, v given by gather(j).  SELL / STENCIL: one thread
// per row, entries in column order.  CSRW: one warp per row, lanes strided
// over the row, a fixed xor tree.
template <typename T, typename G>
__device__ __forceinline__ T row_spmv(const SysDesc &d, const T *__restrict__ val, int c, int lane, uint64_t pol,
                                      G gather)
{
    const int fmt = d.fmt, n = d.n;
    if (fmt == FMT_STENCIL) {
        const int cc[1] = {c};
        T s[1];
        if (d.sdim == 3) stencil_rows<T, 3, 1>(val, d.sL, cc, lane, n, d.sP, pol, gather, s);
        else stencil_rows<T, 2, 1>(val, d.sL, cc, lane, n, d.sP, pol, gather, s);
        return s[0];
    }
    return row_spmv_indexed<T>(d, val, c, lane, pol, gather);
}

// SELL and CSRW rows (uploaded CSR requests), out of line so that their
// registers do not constrain the stencil path.
template <typename T, typename G>
__device__ __noinline__ T row_spmv_indexed(const SysDesc &d, const T *__restrict__ val, int c, int lane,
                                           uint64_t pol, G gather)
{
    const int fmt = d.fmt, n = d.n;
    const int *off = d.off, *col = d.col;
    if (fmt == FMT_SELL) {
        const int b = __ldg(off + c), L = (__ldg(off + c + 1) - b) >> 5;
        return sell_row<T>(col + b + lane, val + b + lane, L, pol, gather);
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

// ------------------------------------------------------------------ k1

template <typename T, int NW>
__device__ __forceinline__ void k1_chunks(const TileCtx &c, const T *val, uint64_t pol)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = c.d.n;
    const T beta = (T)c.s.beta;
    const bool b0 = c.s.pbuf == 0;
    const T *po = static_cast<const T *>(b0 ? c.d.p0 : c.d.p1);
    T *pn = static_cast<T *>(b0 ? c.d.p1 : c.d.p0);
    const T *z = static_cast<const T *>(c.d.z);
    T *ap = static_cast<T *>(c.d.ap);
    double *part = c.d.part;
    auto gather = [=](int j) { return pnew_at(beta, po, z, j); };
    int ch = c.t.c0 + warp;
    if (c.d.fmt == FMT_STENCIL && c.d.sdim == 2) {
        // 2-D stencil: two chunks per warp with their loads in flight together
        for (; ch + NW < c.t.c1; ch += 2 * NW) {
            const int cc[2] = {ch, ch + NW};
            T s2[2];
            stencil_rows<T, 2, 2>(val, c.d.sL, cc, lane, n, c.d.sP, pol, gather, s2);
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int i = cc[u] * kChunk + lane;
                double dp = 0.0;
                if (i < n) {
                    const T pi = pnew_at(beta, po, z, i);
                    pn[i] = pi;
                    ap[i] = s2[u];
                    dp = (double)(pi * s2[u]);
                }
                dp = warp_sum(dp);
                if (lane == 0) part[cc[u]] = dp;
            }
        }
    }
    for (; ch < c.t.c1; ch += NW) {
        const int i = ch * kChunk + lane;
        const T s = row_spmv<T>(c.d, val, ch, lane, pol, gather);
        double dp = 0.0;
        if (i < n) {
            const T pi = pnew_at(beta, po, z, i);
            pn[i] = pi;
            ap[i] = s;
            dp = (double)(pi * s);
        }
        dp = warp_sum(dp);
        if (lane == 0) part[ch] = dp;
    }
}

template <int NW>
__device__ __forceinline__ void k1_correct(const TileCtx &c)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = c.d.n;
    double *x = c.d.x;
    const float *xl = static_cast<const float *>(c.d.xl);
    for (int ch = c.t.c0 + warp; ch < c.t.c1; ch += NW) {
        const int i = ch * kChunk + lane;
        if (i < n) x[i] += (double)xl[i];
    }
}

template <int NW>
__global__ void __launch_bounds__(NW * 32, kMinCta256 * 8 / NW) k1_kernel(const SysDesc *__restrict__ sys, SysState *state,
                                                     const int *__restrict__ tb)
{
    __shared__ TileCtx c;
    __shared__ double sm[8 * 3];
    __shared__ bool last;
    const int ntiles = __ldcg(tb);
    const Tile *tiles = reinterpret_cast<const Tile *>(tb + kTileHdrWords);
    const uint64_t pol = l2_policy(0);
    const int t0 = (int)((long long)blockIdx.x * ntiles / gridDim.x);
    const int t1 = (int)((long long)(blockIdx.x + 1) * ntiles / gridDim.x);
    TileWalk w{t0, t1, -1, -1};
    int run = 0;
    for (; w.t < t1; ++w.t) {
        w.enter(sys, state, tiles, c, w.t == t0);
        const int ph = c.s.phase;
        if (ph == PH_CORRECT) {
            k1_correct<NW>(c);
            continue;
        }
        if (ph != PH_CG && ph != PH_INNER) continue;
        if (ph == PH_CG) k1_chunks<double, NW>(c, c.d.val64, pol);
        else k1_chunks<float, NW>(c, c.d.val32, pol);
        ++run;
        w.publish_next(c);
        if (c.next_sys == c.t.sys) continue;
        const int r = run;
        run = 0;
        if (run_done(c.d.ticket, r, c.t.ntiles, last)) {
            double o[1];
            fin_sum<1, NW>(c.d.part, c.d.nchunks, c.d.pstride, o, sm);
            if (threadIdx.x == 0) {
                SysState *st = state + c.t.sys;
                st->alpha = c.s.rho / o[0];
                st->pbuf = c.s.pbuf ^ 1;
            }
        }
    }
}

// ------------------------------------------------------------------ k2

template <typename T, int NW>
__device__ __forceinline__ void k2_update(const TileCtx &c, T *x)
{
    constexpr int U = 4;   // chunks per warp with loads in flight together
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = c.d.n, ps = c.d.pstride, c1 = c.t.c1;
    const T alpha = (T)c.s.alpha;
    T *r = static_cast<T *>(c.d.r), *z = static_cast<T *>(c.d.z);
    const T *p = static_cast<const T *>(c.s.pbuf == 0 ? c.d.p0 : c.d.p1);
    const T *ap = static_cast<const T *>(c.d.ap), *dv = static_cast<const T *>(c.d.invd);
    double *part = c.d.part;
    for (int ch0 = c.t.c0 + warp; ch0 < c1; ch0 += U * NW) {
        T xv[U], rv[U], pv[U], av[U], dd[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int ch = ch0 + u * NW, i = ch * kChunk + lane;
            if (ch < c1 && i < n) {
                xv[u] = x[i];
                rv[u] = r[i];
                pv[u] = p[i];
                av[u] = __ldcs(ap + i);
                dd[u] = dv[i];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int ch = ch0 + u * NW, i = ch * kChunk + lane;
            if (ch >= c1) break;
            double rr = 0.0, rz = 0.0;
            if (i < n) {
                const T xi = xv[u] + alpha * pv[u];
                const T ri = rv[u] - alpha * av[u];
                const T zi = zmul(ri, dd[u]);
                x[i] = xi;
                r[i] = ri;
                z[i] = zi;
                rr = (double)(ri * ri);
                rz = (double)(ri * zi);
            }
            rr = warp_sum(rr);
            rz = warp_sum(rz);
            if (lane == 0) {
                part[ch] = rr;
                part[ps + ch] = rz;
            }
        }
    }
}

template <int NW>
__device__ __forceinline__ void k2_start(const TileCtx &c)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = c.d.n, ps = c.d.pstride;
    double *r = static_cast<double *>(c.d.r), *z = static_cast<double *>(c.d.z);
    const double *b = c.d.b, *dv = static_cast<const double *>(c.d.invd);
    double *part = c.d.part;
    for (int ch = c.t.c0 + warp; ch < c.t.c1; ch += NW) {
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
            part[ch] = rr;
            part[ps + ch] = rz;
        }
    }
}

// Runs once per outer step of a mixed system: kept out of line so that its
// registers do not constrain the per-iteration update.
template <int NW>
__device__ __noinline__ void k2_outer(const TileCtx &c, uint64_t pol)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = c.d.n, ps = c.d.pstride;
    const double *b = c.d.b, *x = c.d.x, *val = c.d.val64;
    float *rl = static_cast<float *>(c.d.r), *zl = static_cast<float *>(c.d.z), *xl = static_cast<float *>(c.d.xl);
    const float *dv = static_cast<const float *>(c.d.invd);
    double *part = c.d.part;
    auto gather = [=](int j) { return __ldg(x + j); };
    for (int ch = c.t.c0 + warp; ch < c.t.c1; ch += NW) {
        const int i = ch * kChunk + lane;
        const double s = row_spmv<double>(c.d, val, ch, lane, pol, gather);
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
            part[ch] = q0;
            part[ps + ch] = q1;
            part[2 * ps + ch] = q2;
        }
    }
}

// Thread 0 of the CTA completing a system's update tiles.  cs: the state as
// read at the tile start (nothing else writes it during this launch).
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

// The completing CTA of a system's update tiles (out of line: once per
// system and launch).
template <int NW>
__device__ __noinline__ void k2_final(const TileCtx &c, SysState *state, int ph, int nq, double *sm)
{
    double o[3] = {0.0, 0.0, 0.0};
    if (nq == 2) {
        double o2[2];
        fin_sum<2, NW>(c.d.part, c.d.nchunks, c.d.pstride, o2, sm);
        o[0] = o2[0];
        o[1] = o2[1];
    } else {
        fin_sum<3, NW>(c.d.part, c.d.nchunks, c.d.pstride, o, sm);
    }
    if (threadIdx.x == 0) k2_finish(c.s, state + c.t.sys, c.d.done, ph, o);
}

template <int NW>
__global__ void __launch_bounds__(NW * 32, kMinCta256 * 8 / NW) k2_kernel(const SysDesc *__restrict__ sys, SysState *state,
                                                     const int *__restrict__ tb)
{
    __shared__ TileCtx c;
    __shared__ double sm[8 * 3];
    __shared__ bool last;
    const int ntiles = __ldcg(tb);
    const Tile *tiles = reinterpret_cast<const Tile *>(tb + kTileHdrWords);
    const uint64_t pol = l2_policy(0);
    const int t0 = (int)((long long)blockIdx.x * ntiles / gridDim.x);
    const int t1 = (int)((long long)(blockIdx.x + 1) * ntiles / gridDim.x);
    TileWalk w{t0, t1, -1, -1};
    int run = 0;
    for (; w.t < t1; ++w.t) {
        w.enter(sys, state, tiles, c, w.t == t0);
        const int ph = c.s.phase;
        int nq;
        if (ph == PH_CG) {
            k2_update<double, NW>(c, c.d.x);
            nq = 2;
        } else if (ph == PH_INNER) {
            k2_update<float, NW>(c, static_cast<float *>(c.d.xl));
            nq = 2;
        } else if (ph == PH_CG_START) {
            k2_start<NW>(c);
            nq = 2;
        } else if (ph == PH_OUTER || ph == PH_CORRECT) {
            k2_outer<NW>(c, pol);
            nq = 3;
        } else {
            continue;
        }
        ++run;
        w.publish_next(c);
        if (c.next_sys == c.t.sys) continue;
        const int r = run;
        run = 0;
        if (run_done(c.d.ticket + 32, r, c.t.ntiles, last)) k2_final<NW>(c, state, ph, nq, sm);
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
                const int c = i / kChunk, lane = i % kChunk;
                const size_t base = (size_t)c * kChunk * d.sL + lane;
                double *ov = const_cast<double *>(d.val64);
                float *of = const_cast<float *>(d.val32);
                for (int j = rb; j < re; ++j) {
                    const int dl = col[j] - i;
                    for (int k = 0; k < d.sL; ++k)
                        if (stencil_delta(d.sdim, d.sP, k) == dl) {
                            ov[base + (size_t)kChunk * k] = val[j];
                            if (d.mixed) of[base + (size_t)kChunk * k] = (float)val[j];
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

cudaError_t launch_round(int nw, int grid, const SysDesc *sys, SysState *state, const int *tiles, cudaStream_t st)
{
    if (nw == 4) {
        k1_kernel<4><<<grid, 128, 0, st>>>(sys, state, tiles);
        k2_kernel<4><<<grid, 128, 0, st>>>(sys, state, tiles);
    } else {
        k1_kernel<8><<<grid, 256, 0, st>>>(sys, state, tiles);
        k2_kernel<8><<<grid, 256, 0, st>>>(sys, state, tiles);
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
