// spmv.cu -- CSR SpMV kernels of the B200 lmp platform (sm_100a).
//
// The reference's hot loop (lmp/CPUsimple_csr_lmatrix.cc:75-112; on the GPU
// the thread-per-row kernel lmp/cuda/cuda_spmv_kernel_csr_scalar.h:21-49,
// which re-writes y[i] once per nonzero) becomes one of two kernel families:
//
// * tile kernels: a persistent grid walks a precomputed list of row tiles.
//   Thread 0 of each CTA keeps ST tiles of values, column indices and row
//   pointers in flight with cp.async.bulk (evict-first in L2); the CTA reduces
//   the current tile from shared memory with 2^lg lanes per row and gathers x
//   through the read-only path, where it stays L2-resident.
// * the direct kernel: no staging; 2^lg lanes per row read values and column
//   indices with streaming (evict-first) loads at full occupancy, so the
//   unified L1 is left to the x gathers of neighbouring rows.
//
// The lanes per row come from the mean row length (vector vs warp per row).
// Epilogues fuse what the Krylov recurrences do next: dot with x, residual
// and its norm, and the multicolour Gauss-Seidel / ILU sweep updates.
#include "common.cuh"
#include "kernels.cuh"
#include "spmv_epi.cuh"

#include <cmath>
#include <cstdlib>

namespace b200 {

namespace {

template <int CAP>
struct TileSmem {
    template <typename T>
    __host__ __device__ static constexpr int val_bytes() { return (((CAP + 8) * (int)sizeof(T)) + 127) & ~127; }
    __host__ __device__ static constexpr int col_bytes() { return (((CAP + 8) * 4) + 127) & ~127; }
    __host__ __device__ static constexpr int row_bytes() { return (((kBlock + 16) * 4) + 127) & ~127; }
    template <typename T>
    __host__ __device__ static constexpr int stage_bytes() { return val_bytes<T>() + col_bytes() + row_bytes(); }
};


// Rows too long for a tile: one warp per row straight from global memory.
template <typename T, int EPI>
__device__ __forceinline__ void long_rows(const CsrView &A, const Seg &seg, const SpmvOp &op, double &acc)
{
    const int *__restrict__ row = A.row;
    const int *__restrict__ col = A.col;
    const T *__restrict__ val = static_cast<const T *>(A.val);
    const T *__restrict__ x = static_cast<const T *>(op.x);
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    const int nw = gridDim.x * (kBlock / 32);
    for (int li = seg.l0 + gw; li < seg.l1; li += nw) {
        const int r = A.long_rows[li];
        const int j1 = __ldg(row + r + 1);
        T s = T(0);
        for (int j = __ldg(row + r) + lane; j < j1; j += 32) s += __ldcs(val + j) * __ldg(x + __ldcs(col + j));
        s = warp_sum(s);
        if (lane == 0) epilogue<T, EPI>(r, s, op, acc);
    }
}

template <typename T, int EPI, int CAP, int ST, int MINB>
__global__ void __launch_bounds__(kBlock, MINB) spmv_tile_kernel(CsrView A, Seg seg, SpmvOp op, Scratch sc)
{
    if (gate_closed(op.gate)) return;
    extern __shared__ __align__(128) unsigned char smem[];
    using L = TileSmem<CAP>;
    constexpr int kVB = L::template val_bytes<T>();
    constexpr int kCB = L::col_bytes();
    constexpr int kSB = L::template stage_bytes<T>();
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + ST * kSB);

    const int *__restrict__ row = A.row;
    const int *__restrict__ col = A.col;
    const T *__restrict__ val = static_cast<const T *>(A.val);
    const T *__restrict__ x = static_cast<const T *>(op.x);
    const int G = 1 << A.lg;
    const int grp = threadIdx.x >> A.lg;
    const int lane_g = threadIdx.x & (G - 1);
    const int ntiles = seg.t1 - seg.t0;
    const int my_n = ((int)blockIdx.x < ntiles) ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
    }
    __syncthreads();

    uint64_t pol = 0;
    // tile k of this CTA into stage stg: values, column indices and the row
    // pointers row[r0 .. r1], each widened to 16-byte units
    auto issue = [&](int k, int stg) {
        const Tile t = A.tiles[seg.t0 + blockIdx.x + k * gridDim.x];
        const unsigned n4 = (unsigned)(t.a1 - t.a0);
        const int b0 = t.r0 & ~3;
        const unsigned nr = (unsigned)(((t.r1 + 1 + 3) & ~3) - b0);
        unsigned char *base = smem + stg * kSB;
        mbar_arrive_expect_tx(&bars[stg], n4 * (unsigned)(sizeof(T) + 4) + nr * 4u);
        if (n4) {
            bulk_g2s(base, val + t.a0, n4 * (unsigned)sizeof(T), &bars[stg], pol);
            bulk_g2s(base + kVB, col + t.a0, n4 * 4u, &bars[stg], pol);
        }
        bulk_g2s(base + kVB + kCB, row + b0, nr * 4u, &bars[stg], pol);
    };
    if (threadIdx.x == 0) {
        pol = l2_evict_first_policy();
        for (int k = 0; k < ST && k < my_n; ++k) issue(k, k);
    }

    double acc = 0.0;
    for (int k = 0; k < my_n; ++k) {
        const int stg = k % ST;
        const unsigned par = (unsigned)(k / ST) & 1u;
        const Tile t = A.tiles[seg.t0 + blockIdx.x + k * gridDim.x];
        const bool ok = mbar_wait_bounded(&bars[stg], par, sc.err);
        if (__syncthreads_or(!ok)) break;
        const unsigned char *base = smem + stg * kSB;
        const T *sv = reinterpret_cast<const T *>(base);
        const int *scol = reinterpret_cast<const int *>(base + kVB);
        const int *srow = reinterpret_cast<const int *>(base + kVB + kCB) - (t.r0 & ~3);
        const int r = t.r0 + grp;
        const bool active = r < t.r1;
        T s = T(0);
        if (active) {
            const int j1 = srow[r + 1] - t.a0;
#pragma unroll 4
            for (int j = srow[r] - t.a0 + lane_g; j < j1; j += G) s += sv[j] * __ldg(x + scol[j]);
        }
        for (int o = G >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (active && lane_g == 0) epilogue<T, EPI>(r, s, op, acc);
        __syncthreads();
        if (threadIdx.x == 0 && k + ST < my_n) issue(k + ST, stg);
    }
    long_rows<T, EPI>(A, seg, op, acc);
    if constexpr (reduces<EPI>()) {
        double v[1] = {acc}, out[1];
        if (grid_reduce<1>(v, sc.partials, sc.ticket, out)) finalize(op, out[0]);
    }
}



template <typename T, int EPI>
__global__ void __launch_bounds__(kBlock) spmv_direct_kernel(CsrView A, Seg seg, SpmvOp op, Scratch sc)
{
    if (gate_closed(op.gate)) return;
    const int *__restrict__ row = A.row;
    const int *__restrict__ col = A.col;
    const T *__restrict__ val = static_cast<const T *>(A.val);
    const T *__restrict__ x = static_cast<const T *>(op.x);
    const int G = 1 << A.lg;
    const int rpb = kBlock >> A.lg;
    const int grp = threadIdx.x >> A.lg;
    const int lane_g = threadIdx.x & (G - 1);
    const uint64_t pol_s = l2_policy(A.l2hint & 1 ? 1 : 0), pol_x = l2_policy(A.l2hint & 2 ? 2 : 0);
    double acc = 0.0;
    const int bstep = gridDim.x * rpb;
    // the row pointers of the group's next row are loaded one row ahead, so
    // their round trip overlaps this row's value, index and x loads
    int nj0 = 0, nj1 = 0;
    if (seg.r0 + blockIdx.x * rpb + grp < seg.r1) {
        nj0 = __ldg(row + seg.r0 + blockIdx.x * rpb + grp);
        nj1 = __ldg(row + seg.r0 + blockIdx.x * rpb + grp + 1);
    }
    for (int base = seg.r0 + blockIdx.x * rpb; base < seg.r1; base += bstep) {
        const int r = base + grp;
        const bool active = r < seg.r1;
        const int j0 = nj0, j1 = nj1;
        if (r + bstep < seg.r1) {
            nj0 = __ldg(row + r + bstep);
            nj1 = __ldg(row + r + bstep + 1);
        }
        T s = T(0);
        if (active) {
            // 16-byte loads: E values and E column indices per lane per step,
            // the group's windows of E * G elements aligned to their size,
            // elements outside the row masked (the arrays are
            // padded by 8 entries past nnz, so a window never leaves the
            // allocation).  No unrolling: measured on B200 (128^3 Q1, FP64)
            // 145 us against 158 us unrolled by 2 and 166 us for 8-byte loads.
            constexpr int E = 16 / (int)sizeof(T);
            const int W = E * G;
#pragma unroll 1
            for (int j = (j0 & ~(W - 1)) + E * lane_g; j < j1; j += W) {
                T v[E];
                int c[E];
                ld_stream_vec(val + j, pol_s, v);
                ld_stream_vec(col + j, pol_s, c);
#pragma unroll
                for (int e = 0; e < E; ++e)
                    if (j + e >= j0 && j + e < j1) s += v[e] * ld_keep(x + c[e], pol_x);
            }
        }
        for (int o = G >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (active && lane_g == 0) epilogue<T, EPI>(r, s, op, acc);
    }
    if constexpr (reduces<EPI>()) {
        double v[1] = {acc}, out[1];
        if (grid_reduce<1>(v, sc.partials, sc.ticket, out)) finalize(op, out[0]);
    }
}

// Pattern-dictionary SpMV: the CTA loads the pattern table into shared
// memory once; each row then reads its values (streaming), its 2-byte pattern
// id and the row pointer, and forms column indices from the table -- 4 bytes
// per nonzero less traffic than CSR's explicit indices.
template <typename T, int EPI>
__global__ void __launch_bounds__(kBlock) spmv_pattern_kernel(CsrView A, Seg seg, SpmvOp op, Scratch sc)
{
    if (gate_closed(op.gate)) return;
    extern __shared__ int s_pat[];   // pattern offsets, then the offsets' table
    int *s_off = s_pat;
    int *s_delta = s_pat + A.npat + 1;
    for (int i = threadIdx.x; i <= A.npat; i += kBlock) s_off[i] = A.pat_off[i];
    for (int i = threadIdx.x; i < A.ndelta; i += kBlock) s_delta[i] = A.pat_delta[i];
    __syncthreads();
    const int *__restrict__ row = A.row;
    const T *__restrict__ val = static_cast<const T *>(A.val);
    const T *__restrict__ x = static_cast<const T *>(op.x);
    const int G = 1 << A.lg;
    const int rpb = kBlock >> A.lg;
    const int grp = threadIdx.x >> A.lg;
    const int lane_g = threadIdx.x & (G - 1);
    const uint64_t pol_s = l2_policy(A.l2hint & 1 ? 1 : 0), pol_x = l2_policy(A.l2hint & 2 ? 2 : 0);
    double acc = 0.0;
    for (int base = seg.r0 + blockIdx.x * rpb; base < seg.r1; base += gridDim.x * rpb) {
        const int r = base + grp;
        const bool active = r < seg.r1;
        T s = T(0);
        if (active) {
            const int j0 = __ldg(row + r), len = __ldg(row + r + 1) - j0;
            const int *d = s_delta + s_off[__ldg(A.pid + r)];
#pragma unroll 4
            for (int k = lane_g; k < len; k += G) s += ld_stream(val + j0 + k, pol_s) * ld_keep(x + r + d[k], pol_x);
        }
        for (int o = G >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (active && lane_g == 0) epilogue<T, EPI>(r, s, op, acc);
    }
    if constexpr (reduces<EPI>()) {
        double v[1] = {acc}, out[1];
        if (grid_reduce<1>(v, sc.partials, sc.ticket, out)) finalize(op, out[0]);
    }
}

// Pattern-dictionary SpMV on the sliced layout (SELL-32): warp w takes chunk
// c of 32 consecutive rows, lane l row 32c + l; the chunk's values are stored
// k-major (value k of all 32 rows together), so each load instruction reads
// one 128-byte line of values, and in a chunk whose rows share a pattern the
// gathers x[r + d_k] of one k are 32 consecutive entries as well.  Rows
// shorter than the chunk's longest row are padded with zeros.
template <typename T, int EPI>
__global__ void __launch_bounds__(kBlock) spmv_sell_kernel(CsrView A, Seg seg, SpmvOp op, Scratch sc)
{
    if (gate_closed(op.gate)) return;
    extern __shared__ int s_pat[];
    int *s_off = s_pat;
    int *s_delta = s_pat + A.npat + 1;
    for (int i = threadIdx.x; i <= A.npat; i += kBlock) s_off[i] = A.pat_off[i];
    for (int i = threadIdx.x; i < A.ndelta; i += kBlock) s_delta[i] = A.pat_delta[i];
    __syncthreads();
    const T *__restrict__ sv = static_cast<const T *>(A.sell_val);
    const T *__restrict__ x = static_cast<const T *>(op.x);
    const uint64_t pol_s = l2_policy(A.l2hint & 1 ? 1 : 0), pol_x = l2_policy(A.l2hint & 2 ? 2 : 0);
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    const int nw = gridDim.x * (kBlock / 32);
    const int c0 = seg.r0 >> 5, c1 = (seg.r1 - 1) >> 5;
    double acc = 0.0;
    for (int c = c0 + gw; c <= c1; c += nw) {
        const int r = (c << 5) + lane;
        const bool active = r >= seg.r0 && r < seg.r1;
        const int base = __ldg(A.sell_off + c), L = (__ldg(A.sell_off + c + 1) - base) >> 5;
        const int p = active ? (int)__ldg(A.pid + r) : 0;
        const int len = active ? s_off[p + 1] - s_off[p] : 0;
        const int *d = s_delta + s_off[p];
        const T *v = sv + base + lane;
        T s = T(0);
#pragma unroll 9
        for (int k = 0; k < L; ++k) {
            const T a = ld_stream(v + (k << 5), pol_s);
            if (k < len) s += a * ld_keep(x + r + d[k], pol_x);
        }
        if (active) epilogue<T, EPI>(r, s, op, acc);
    }
    if constexpr (reduces<EPI>()) {
        double vv[1] = {acc}, out[1];
        if (grid_reduce<1>(vv, sc.partials, sc.ticket, out)) finalize(op, out[0]);
    }
}

// The sliced dictionary SpMV with the values brought in by the bulk-copy
// engine: a tile is 8 consecutive 32-row chunks -- one contiguous, 128-byte
// aligned range of the sliced values -- and a persistent grid keeps kSellStages
// tiles per CTA in flight (one cp.async.bulk each, evict-first in L2).  Warp w
// of the CTA reduces chunk w of the tile from shared memory, one row per lane.
constexpr int kSellStages = 3;
constexpr size_t kSellTmaMaxSmem = 200 * 1024;

template <typename T, int EPI>
__global__ void __launch_bounds__(kBlock, 2)
    spmv_sell_tma_kernel(CsrView A, Seg seg, SpmvOp op, Scratch sc, int stage_elems)
{
    if (gate_closed(op.gate)) return;
    extern __shared__ __align__(128) unsigned char smem[];
    int *s_off = reinterpret_cast<int *>(smem);
    int *s_delta = s_off + A.npat + 1;
    const int head = ((A.npat + 1 + A.ndelta) * 4 + 127) & ~127;
    T *stages = reinterpret_cast<T *>(smem + head);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + head + kSellStages * stage_elems * (int)sizeof(T));
    for (int i = threadIdx.x; i <= A.npat; i += kBlock) s_off[i] = A.pat_off[i];
    for (int i = threadIdx.x; i < A.ndelta; i += kBlock) s_delta[i] = A.pat_delta[i];
    if (threadIdx.x == 0) {
        for (int s = 0; s < kSellStages; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    const T *__restrict__ sv = static_cast<const T *>(A.sell_val);
    const T *__restrict__ x = static_cast<const T *>(op.x);
    const uint64_t pol_x = l2_policy(A.l2hint & 2 ? 2 : 0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c0 = seg.r0 >> 5, c1 = (seg.r1 - 1) >> 5;
    const int ntile = (c1 - c0 + 1 + kBlock / 32 - 1) / (kBlock / 32);
    const int my_n = ((int)blockIdx.x < ntile) ? (ntile - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    uint64_t pol = 0;
    auto issue = [&](int k, int stg) {
        const int t = blockIdx.x + k * gridDim.x;
        const int cb = c0 + t * (kBlock / 32);
        const int ce = min(cb + kBlock / 32, c1 + 1);
        const int e0 = __ldg(A.sell_off + cb), e1 = __ldg(A.sell_off + ce);
        const unsigned bytes = (unsigned)(e1 - e0) * (unsigned)sizeof(T);
        mbar_arrive_expect_tx(&bars[stg], bytes);
        if (bytes) bulk_g2s(stages + stg * stage_elems, sv + e0, bytes, &bars[stg], pol);
    };
    if (threadIdx.x == 0) {
        pol = l2_evict_first_policy();
        for (int k = 0; k < kSellStages && k < my_n; ++k) issue(k, k);
    }
    double acc = 0.0;
    for (int k = 0; k < my_n; ++k) {
        const int stg = k % kSellStages;
        const bool ok = mbar_wait_bounded(&bars[stg], (unsigned)(k / kSellStages) & 1u, sc.err);
        if (__syncthreads_or(!ok)) break;
        const int t = blockIdx.x + k * gridDim.x;
        const int cb = c0 + t * (kBlock / 32);
        const int c = cb + warp;
        if (c <= c1) {
            const int ebase = __ldg(A.sell_off + cb);
            const int e0 = __ldg(A.sell_off + c), L = (__ldg(A.sell_off + c + 1) - e0) >> 5;
            const T *v = stages + stg * stage_elems + (e0 - ebase) + lane;
            const int r = (c << 5) + lane;
            const bool active = r >= seg.r0 && r < seg.r1;
            const int p = active ? (int)__ldg(A.pid + r) : 0;
            const int len = active ? s_off[p + 1] - s_off[p] : 0;
            const int *d = s_delta + s_off[p];
            T s = T(0);
#pragma unroll 9
            for (int q = 0; q < L; ++q) {
                const T a = v[q << 5];
                if (q < len) s += a * ld_keep(x + r + d[q], pol_x);
            }
            if (active) epilogue<T, EPI>(r, s, op, acc);
        }
        __syncthreads();
        if (threadIdx.x == 0 && k + kSellStages < my_n) issue(k + kSellStages, stg);
    }
    if constexpr (reduces<EPI>()) {
        double vv[1] = {acc}, out[1];
        if (grid_reduce<1>(vv, sc.partials, sc.ticket, out)) finalize(op, out[0]);
    }
}

// Pattern-dictionary SpMV with x staged in shared memory.  Rows are taken in
// tiles of R = kBlock / 2^lg consecutive rows; the x values a tile needs lie
// on the dictionary's gather lines shifted by the tile's first row, so the
// CTA loads those lines with coalesced loads (R + span values each, zero
// outside [0, n)) and every row gathers from shared memory through a
// precomputed per-entry offset.  The unified L1 then carries only the
// streamed values.
template <typename T, int EPI>
__global__ void __launch_bounds__(kBlock) spmv_pattern_staged_kernel(CsrView A, Seg seg, SpmvOp op, Scratch sc,
                                                                     int n_x)
{
    if (gate_closed(op.gate)) return;
    extern __shared__ __align__(16) unsigned char s_raw[];
    const int R = kBlock >> A.lg;
    int *s_off = reinterpret_cast<int *>(s_raw);              // npat + 1
    int *s_soff = s_off + A.npat + 1;                          // ndelta: staged offset of each entry
    int *s_lbase = s_soff + A.ndelta;                          // nlines + 1
    int *s_lstart = s_lbase + A.nlines + 1;                    // nlines
    const int head = (A.npat + 1 + A.ndelta + 2 * A.nlines + 1 + 3) & ~3;   // ints, 16-byte multiple
    T *s_x = reinterpret_cast<T *>(reinterpret_cast<int *>(s_raw) + head);
    for (int i = threadIdx.x; i <= A.npat; i += kBlock) s_off[i] = A.pat_off[i];
    for (int i = threadIdx.x; i < A.nlines; i += kBlock) s_lstart[i] = A.line_start[i];
    if (threadIdx.x == 0) {
        int b = 0;
        for (int l = 0; l < A.nlines; ++l) {
            s_lbase[l] = b;
            b += R + A.line_span[l];
        }
        s_lbase[A.nlines] = b;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < A.ndelta; i += kBlock) s_soff[i] = s_lbase[A.entry_line[i]] + A.entry_lo[i];
    const int *__restrict__ row = A.row;
    const T *__restrict__ val = static_cast<const T *>(A.val);
    const T *__restrict__ x = static_cast<const T *>(op.x);
    const int G = 1 << A.lg;
    const int grp = threadIdx.x >> A.lg;
    const int lane_g = threadIdx.x & (G - 1);
    const int staged = s_lbase[A.nlines];
    double acc = 0.0;
    for (int r0 = seg.r0 + blockIdx.x * R; r0 < seg.r1; r0 += gridDim.x * R) {
        __syncthreads();
        // stage the tile's gather lines (coalesced, line by line)
        for (int l = 0; l < A.nlines; ++l) {
            const int len = s_lbase[l + 1] - s_lbase[l];
            const int g0 = r0 + s_lstart[l];
            T *dst = s_x + s_lbase[l];
            for (int i = threadIdx.x; i < len; i += kBlock) {
                const int gi = g0 + i;
                dst[i] = (gi >= 0 && gi < n_x) ? __ldg(x + gi) : T(0);
            }
        }
        __syncthreads();
        const int r = r0 + grp;
        const bool active = r < seg.r1;
        T s = T(0);
        if (active) {
            const int j0 = __ldg(row + r), len = __ldg(row + r + 1) - j0;
            const int *so = s_soff + s_off[__ldg(A.pid + r)];
#pragma unroll 4
            for (int k = lane_g; k < len; k += G) s += __ldcs(val + j0 + k) * s_x[so[k] + grp];
        }
        for (int o = G >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (active && lane_g == 0) epilogue<T, EPI>(r, s, op, acc);
    }
    (void)staged;
    if constexpr (reduces<EPI>()) {
        double v[1] = {acc}, out[1];
        if (grid_reduce<1>(v, sc.partials, sc.ticket, out)) finalize(op, out[0]);
    }
}

template <typename T, int EPI, int CAP, int ST, int MINB>
cudaError_t set_tile_attr()
{
    return cudaFuncSetAttribute(spmv_tile_kernel<T, EPI, CAP, ST, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                ST * TileSmem<CAP>::template stage_bytes<T>() + ST * 8);
}

template <typename T, int EPI>
cudaError_t set_sell_attr()
{
    return cudaFuncSetAttribute(spmv_sell_tma_kernel<T, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kSellTmaMaxSmem);
}

template <typename T>
cudaError_t configure_sell()
{
    cudaError_t e;
    if ((e = set_sell_attr<T, EPI_SET>())) return e;
    if ((e = set_sell_attr<T, EPI_ADD>())) return e;
    if ((e = set_sell_attr<T, EPI_DOT_X>())) return e;
    if ((e = set_sell_attr<T, EPI_RESID>())) return e;
    if ((e = set_sell_attr<T, EPI_SGS_F>())) return e;
    if ((e = set_sell_attr<T, EPI_SGS_B>())) return e;
    if ((e = set_sell_attr<T, EPI_ILU_F>())) return e;
    return set_sell_attr<T, EPI_ILU_B>();
}

template <typename T, int CAP, int ST, int MINB>
cudaError_t configure_tile()
{
    cudaError_t e;
    if ((e = set_tile_attr<T, EPI_SET, CAP, ST, MINB>())) return e;
    if ((e = set_tile_attr<T, EPI_ADD, CAP, ST, MINB>())) return e;
    if ((e = set_tile_attr<T, EPI_DOT_X, CAP, ST, MINB>())) return e;
    if ((e = set_tile_attr<T, EPI_RESID, CAP, ST, MINB>())) return e;
    if ((e = set_tile_attr<T, EPI_SGS_F, CAP, ST, MINB>())) return e;
    if ((e = set_tile_attr<T, EPI_SGS_B, CAP, ST, MINB>())) return e;
    if ((e = set_tile_attr<T, EPI_ILU_F, CAP, ST, MINB>())) return e;
    return set_tile_attr<T, EPI_ILU_B, CAP, ST, MINB>();
}

template <typename T, int EPI, int CAP, int ST, int MINB>
void launch_tile(int grid, const CsrView &A, const Seg &seg, const SpmvOp &op, const Scratch &s, cudaStream_t st)
{
    spmv_tile_kernel<T, EPI, CAP, ST, MINB>
        <<<grid, kBlock, ST * TileSmem<CAP>::template stage_bytes<T>() + ST * 8, st>>>(A, seg, op, s);
}

template <typename T, int W>
struct StencilVec;
template <>
struct StencilVec<double, 1> {
    using type = double;
    static __device__ __forceinline__ void load(const double *p, uint64_t pol, double *o) { o[0] = ld_stream(p, pol); }
};
template <>
struct StencilVec<float, 4> {
    using type = float4;
    static __device__ __forceinline__ void load(const float4 *p, uint64_t pol, float *o)
    {
        float4 v;
        asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
            : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
            : "l"(p), "l"(pol));
        o[0] = v.x;
        o[1] = v.y;
        o[2] = v.z;
        o[3] = v.w;
    }
};

// Stencil SpMV (structured operators): the row patterns' offsets lie in NB
// bands of three consecutive columns.  One warp per 32-row chunk, one row per
// lane; for each band a lane gathers only the band centre x[i + c_b] (32
// consecutive entries), its left / right neighbours come from lanes -1 / +1
// by shuffle and lanes 0 / 31 load the one column beyond the chunk.  The
// values arrive k-major (three 128- or 256-byte lines per band) with no
// index of any kind; products are added in column order.  Columns outside
// [0, n) belong to zero entries and are clamped into range.
template <typename T, int EPI, int NB>
__global__ void __launch_bounds__(kBlock) spmv_stencil_kernel(CsrView A, SpmvOp op, Scratch sc)
{
    if (gate_closed(op.gate)) return;
    // positions per lane and load: FP32 values come in groups of four (one
    // 16-byte load per lane), FP64 one by one
    constexpr int W = stencil_group<T>();
    constexpr int L = 3 * NB, G = (L + W - 1) / W;
    using V = typename StencilVec<T, W>::type;
    const V *__restrict__ sv = static_cast<const V *>(A.st_val);
    const T *__restrict__ x = static_cast<const T *>(op.x);
    // values: the stream (evict-first in L2 by the matrix's hint, so that x and the
    // solver's vectors stay resident); gathers: normal
    const uint64_t pol = l2_policy(0), pol_v = l2_policy(A.l2hint & 4 ? 1 : 0);
    auto gx = [&](int j) -> T { return ld_keep(x + j, pol); };
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    const int nw = gridDim.x * (kBlock / 32);
    const int n = A.n_rows, last = n - 1, nch = (n + 31) >> 5;
    const bool edge = lane == 0 || lane == 31;
    int cen[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) cen[b] = A.st_center[b];
    double acc = 0.0;
    for (int c = gw; c < nch; c += nw) {
        const int r0 = c << 5, r = r0 + lane;
        const int he = lane == 0 ? r0 - 1 : r0 + 32;
        const V *v = sv + (size_t)c * (32 * G) + lane;
        T s = T(0);
        if constexpr (W > 1) {
            // FP32: the whole row's values first (G vector loads), then the bands
            T a[G * W];
#pragma unroll
            for (int g = 0; g < G; ++g) StencilVec<T, W>::load(v + 32 * g, pol_v, a + W * g);
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const int d = cen[b];
                const T w = gx(min(max(r + d, 0), last));
                const T h = edge ? gx(min(max(he + d, 0), last)) : T(0);
                T left = __shfl_up_sync(0xffffffffu, w, 1);
                T right = __shfl_down_sync(0xffffffffu, w, 1);
                if (lane == 0) left = h;
                if (lane == 31) right = h;
                s += a[3 * b] * left;
                s += a[3 * b + 1] * w;
                s += a[3 * b + 2] * right;
            }
        } else {
            // FP64: groups of three bands, their value loads and gathers issued together
#pragma unroll
            for (int b0 = 0; b0 < NB; b0 += 3) {
                T a[9], w[3], h[3];
#pragma unroll
                for (int bb = 0; bb < 3; ++bb)
#pragma unroll
                    for (int m = 0; m < 3; ++m) StencilVec<T, W>::load(v + 32 * (3 * (b0 + bb) + m), pol_v, a + 3 * bb + m);
#pragma unroll
                for (int bb = 0; bb < 3; ++bb) {
                    const int d = cen[b0 + bb];
                    w[bb] = gx(min(max(r + d, 0), last));
                    h[bb] = edge ? gx(min(max(he + d, 0), last)) : T(0);
                }
#pragma unroll
                for (int bb = 0; bb < 3; ++bb) {
                    T left = __shfl_up_sync(0xffffffffu, w[bb], 1);
                    T right = __shfl_down_sync(0xffffffffu, w[bb], 1);
                    if (lane == 0) left = h[bb];
                    if (lane == 31) right = h[bb];
                    s += a[3 * bb] * left;
                    s += a[3 * bb + 1] * w[bb];
                    s += a[3 * bb + 2] * right;
                }
            }
        }
        if (r < n) epilogue<T, EPI>(r, s, op, acc);
    }
    if constexpr (reduces<EPI>()) {
        double vv[1] = {acc}, out[1];
        if (grid_reduce<1>(vv, sc.partials, sc.ticket, out)) finalize(op, out[0]);
    }
}


// Half stencil SpMV (symmetric stencil operators).  A symmetric operator's
// value at (i, i + d), d < 0, equals the one at (i + d, i), which row i + d
// stores among its upper positions; so only the diagonal and the upper half
// are stored (14 of 27 positions in 3-D, 5 of 9 in 2-D) and a row's lower
// half is read from the rows that own it.  Those reads fall on values that
// other warps stream in the same pass (at most one plane of rows back), so
// they are served by L2 and the operator crosses HBM about once at half the
// bytes.  Rows whose off-diagonal values are all zero (the identity rows of
// Dirichlet nodes, flagged in sh_mask) hold in their upper slots the
// transposed entries that their neighbours need, and use only their own
// diagonal.  The band values are assembled into the same (band, column)
// order as the full stencil kernel above and the products are added in the
// same order, so y equals that kernel's result bit for bit.
template <typename T, int NB>
struct HalfRow;

template <int NB>
struct HalfRow<float, NB> {
    static constexpr int U = (NB - 1) / 2, GH = half_groups(NB);
    static __device__ __forceinline__ float4 ld(const float4 *p, uint64_t pol)
    {
        float4 v;
        asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
            : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
            : "l"(p), "l"(pol));
        return v;
    }
    // av[b][m]: value of row 32 c + lane at column offset center[b] + m - 1
    static __device__ __forceinline__ void values(const void *sh, const int (&cen)[NB], int c, int lane, int rows,
                                                  uint64_t pol, float (&av)[NB][3])
    {
        const float4 *__restrict__ hv = static_cast<const float4 *>(sh);
        const int r0 = c << 5, r = r0 + lane;
        float4 u[GH];
#pragma unroll
        for (int g = 0; g < GH; ++g) StencilVec<float, 4>::load(hv + ((size_t)c * GH + g) * 32 + lane, pol, &u[g].x);
#pragma unroll
        for (int ub = 0; ub < U; ++ub) {
            av[U + 1 + ub][0] = u[ub].x;
            av[U + 1 + ub][1] = u[ub].y;
            av[U + 1 + ub][2] = u[ub].z;
        }
        av[U][1] = u[0].w;
        av[U][2] = u[1].w;
        // (r, r - 1) is row r - 1's +1 entry: lane - 1's, or the previous chunk's last row
        float lm = __shfl_up_sync(0xffffffffu, u[1].w, 1);
        if (lane == 0) lm = r0 > 0 ? ld(hv + ((size_t)(c - 1) * GH + 1) * 32 + 31, pol).w : 0.f;
        av[U][0] = lm;
        // lower band b mirrors upper band U - 1 - b: (r, r + d + m - 1) is
        // row (r + d + m - 1)'s entry at slot 2 - m of that band
#pragma unroll
        for (int b = 0; b < U; ++b) {
            const int d = cen[b], ub = U - 1 - b, q = r + d;
            const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 g = q >= 0 ? ld(hv + ((size_t)(q >> 5) * GH + ub) * 32 + (q & 31), pol) : z;
            const int hq = lane == 0 ? r0 + d - 1 : r0 + 32 + d;
            const float4 h = ((lane == 0 || lane == 31) && hq >= 0 && hq < rows)
                                 ? ld(hv + ((size_t)(hq >> 5) * GH + ub) * 32 + (hq & 31), pol)
                                 : z;
            float left = __shfl_up_sync(0xffffffffu, g.z, 1);
            float right = __shfl_down_sync(0xffffffffu, g.x, 1);
            if (lane == 0) left = h.z;
            if (lane == 31) right = h.x;
            av[b][0] = left;
            av[b][1] = g.y;
            av[b][2] = right;
        }
    }
};

template <int NB>
struct HalfRow<double, NB> {
    static constexpr int U = (NB - 1) / 2, H = half_positions(NB);
    static __device__ __forceinline__ double at(const double *hv, int q, int p, uint64_t pol)
    {
        return q >= 0 ? ld_keep(hv + ((size_t)(q >> 5) * H + p) * 32 + (q & 31), pol) : 0.0;
    }
    static __device__ __forceinline__ void values(const void *sh, const int (&cen)[NB], int c, int lane, int rows,
                                                  uint64_t pol, double (&av)[NB][3])
    {
        const double *__restrict__ hv = static_cast<const double *>(sh);
        const int r = (c << 5) + lane;
        const double *own = hv + (size_t)c * H * 32 + lane;
        av[U][1] = ld_stream(own, pol);
        av[U][2] = ld_stream(own + 32, pol);
#pragma unroll
        for (int ub = 0; ub < U; ++ub)
#pragma unroll
            for (int m = 0; m < 3; ++m) av[U + 1 + ub][m] = ld_stream(own + 32 * (2 + 3 * ub + m), pol);
        av[U][0] = at(hv, r - 1, 1, pol);
#pragma unroll
        for (int b = 0; b < U; ++b) {
            const int q = r + cen[b], p = 2 + 3 * (U - 1 - b);
            av[b][0] = at(hv, q - 1, p + 2, pol);
            av[b][1] = at(hv, q, p + 1, pol);
            av[b][2] = at(hv, q + 1, p, pol);
        }
    }
    // the three values of band b alone (the same loads as values())
    static __device__ __forceinline__ void band(const double *__restrict__ hv, int d, int c, int lane, int b,
                                                uint64_t pol, uint64_t pol_own, double (&a)[3])
    {
        const int r = (c << 5) + lane;
        const double *own = hv + (size_t)c * H * 32 + lane;
        if (b > U) {
#pragma unroll
            for (int m = 0; m < 3; ++m) a[m] = ld_stream(own + 32 * (2 + 3 * (b - U - 1) + m), pol_own);
        } else if (b == U) {
            a[0] = at(hv, r - 1, 1, pol);
            a[1] = ld_stream(own, pol_own);
            a[2] = ld_stream(own + 32, pol_own);
        } else {
            const int q = r + d, p = 2 + 3 * (U - 1 - b);
            a[0] = at(hv, q - 1, p + 2, pol);
            a[1] = at(hv, q, p + 1, pol);
            a[2] = at(hv, q + 1, p, pol);
        }
    }
};

// MINB: CTAs per SM the registers are budgeted for.  FP64: 4 (64 registers,
// no spills; unbounded, the compiler hoists every group's loads and takes
// 152 registers, one CTA per SM), or 5 with about 100 spilled bytes in the
// reducing epilogues (B200LA_HALF_MINB=5).
template <typename T, int EPI, int NB, int MINB = (sizeof(T) == 8 ? 4 : 1)>
__global__ void __launch_bounds__(kBlock, MINB) spmv_half_kernel(CsrView A, SpmvOp op, Scratch sc)
{
    if (gate_closed(op.gate)) return;
    constexpr int U = (NB - 1) / 2;
    const T *__restrict__ x = static_cast<const T *>(op.x);
    const unsigned *__restrict__ mask = A.sh_mask;
    const uint64_t pol = l2_policy(0), pol_own = l2_policy(A.l2hint & 8 ? 1 : 0);
    auto gx = [&](int j) -> T { return ld_keep(x + j, pol); };
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    const int nw = gridDim.x * (kBlock / 32);
    const int n = A.n_rows, last = n - 1, nch = (n + 31) >> 5, rows = nch << 5;
    const bool edge = lane == 0 || lane == 31;
    int cen[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) cen[b] = A.st_center[b];
    double acc = 0.0;
    for (int c = gw; c < nch; c += nw) {
        const int r0 = c << 5, r = r0 + lane;
        const int he = lane == 0 ? r0 - 1 : r0 + 32;
        if constexpr (sizeof(T) == 8) {
            // FP64: groups of three bands, their value loads and gathers
            // issued together (register pressure of one group, not of the row)
            if (A.l2hint & 16) {   // the chunk's own value lines into L2 before the first group's loads
                constexpr int kLines = HalfRow<double, NB>::H * 32 * 8 / 128;
                if (lane < kLines) {
                    const char *q = reinterpret_cast<const char *>(static_cast<const double *>(A.sh_val) +
                                                                   (size_t)c * HalfRow<double, NB>::H * 32) + 128 * lane;
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(q));
                }
            }
            const bool ident = (__ldg(mask + c) >> lane) & 1u;
            T s = T(0);
#pragma unroll
            for (int b0 = 0; b0 < NB; b0 += 3) {
                T a[3][3], w[3], h[3];
#pragma unroll
                for (int bb = 0; bb < 3; ++bb) {
                    const int b = b0 + bb, d = cen[b];
                    HalfRow<double, NB>::band(static_cast<const double *>(A.sh_val), d, c, lane, b, pol, pol_own, a[bb]);
                    if (ident) {
                        // identity row: its upper slots serve the neighbours; off-diagonals are zero
#pragma unroll
                        for (int m = 0; m < 3; ++m)
                            if (b != U || m != 1) a[bb][m] = T(0);
                    }
                }
#pragma unroll
                for (int bb = 0; bb < 3; ++bb) {
                    const int d = cen[b0 + bb];
                    w[bb] = gx(min(max(r + d, 0), last));
                    h[bb] = edge ? gx(min(max(he + d, 0), last)) : T(0);
                }
#pragma unroll
                for (int bb = 0; bb < 3; ++bb) {
                    T left = __shfl_up_sync(0xffffffffu, w[bb], 1);
                    T right = __shfl_down_sync(0xffffffffu, w[bb], 1);
                    if (lane == 0) left = h[bb];
                    if (lane == 31) right = h[bb];
                    s += a[bb][0] * left;
                    s += a[bb][1] * w[bb];
                    s += a[bb][2] * right;
                }
            }
            if (r < n) epilogue<T, EPI>(r, s, op, acc);
            continue;
        }
        T av[NB][3];
        HalfRow<T, NB>::values(A.sh_val, cen, c, lane, rows, pol, av);
        if ((__ldg(mask + c) >> lane) & 1u) {
            // identity row: its upper slots serve the neighbours; off-diagonals are zero
#pragma unroll
            for (int b = 0; b < NB; ++b)
#pragma unroll
                for (int m = 0; m < 3; ++m)
                    if (b != U || m != 1) av[b][m] = T(0);
        }
        T s = T(0);
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int d = cen[b];
            const T w = gx(min(max(r + d, 0), last));
            const T h = edge ? gx(min(max(he + d, 0), last)) : T(0);
            T left = __shfl_up_sync(0xffffffffu, w, 1);
            T right = __shfl_down_sync(0xffffffffu, w, 1);
            if (lane == 0) left = h;
            if (lane == 31) right = h;
            s += av[b][0] * left;
            s += av[b][1] * w;
            s += av[b][2] * right;
        }
        if (r < n) epilogue<T, EPI>(r, s, op, acc);
    }
    if constexpr (reduces<EPI>()) {
        double vv[1] = {acc}, out[1];
        if (grid_reduce<1>(vv, sc.partials, sc.ticket, out)) finalize(op, out[0]);
    }
}

// Launch of a stencil-family kernel in one wave of resident CTAs (grid-stride
// warps): a second, partial wave left SMs idle at the end (FP32 128^3:
// 48.4 -> 45.3 us).  The occupancy query runs once per kernel instance.
template <typename K>
void launch_one_wave(K kern, int &resident, const Scratch &s, int n_rows, const CsrView &A, const SpmvOp &op,
                     cudaStream_t st)
{
    const int chunks = (n_rows + 31) >> 5;
    int grid = (chunks + kBlock / 32 - 1) / (kBlock / 32);
    if (!resident && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kern, kBlock, 0) != cudaSuccess)
        resident = 4;
    // B200LA_STENCIL_CTAS: fewer CTAs per SM than fit (the share of warps
    // with one chunk more than the others sets the tail of the pass)
    static const int cap_env = [] {
        const char *e = std::getenv("B200LA_STENCIL_CTAS");
        return e ? std::atoi(e) : 0;
    }();
    const int cap = s.num_sms * (cap_env > 0 ? std::min(cap_env, resident) : resident);
    if (grid > cap) grid = cap;
    if (grid < 1) grid = 1;
    kern<<<grid, kBlock, 0, st>>>(A, op, s);
}

template <typename T, int EPI>
void launch_epi(const Scratch &s, const CsrView &A, const Seg &seg, const SpmvOp &op, cudaStream_t st)
{
    if constexpr (EPI == EPI_SET || EPI == EPI_ADD || EPI == EPI_DOT_X || EPI == EPI_RESID) {
        if (A.sh_use && A.sh_val && A.st_use && seg.r0 == 0 && seg.r1 == A.n_rows && (A.st_nb == 3 || A.st_nb == 9)) {
            static int res_nb[3] = {0, 0, 0};
            static const int minb = [] {
                const char *e = std::getenv("B200LA_HALF_MINB");
                return e ? std::atoi(e) : 0;
            }();
            if (A.st_nb == 9 && minb == 5 && sizeof(T) == 8)
                launch_one_wave(spmv_half_kernel<T, EPI, 9, 5>, res_nb[2], s, A.n_rows, A, op, st);
            else if (A.st_nb == 9)
                launch_one_wave(spmv_half_kernel<T, EPI, 9>, res_nb[1], s, A.n_rows, A, op, st);
            else
                launch_one_wave(spmv_half_kernel<T, EPI, 3>, res_nb[0], s, A.n_rows, A, op, st);
            return;
        }
        if (A.st_use && A.st_val && seg.r0 == 0 && seg.r1 == A.n_rows && (A.st_nb == 3 || A.st_nb == 9)) {
            const int chunks = (A.n_rows + 31) >> 5;
            int grid = (chunks + kBlock / 32 - 1) / (kBlock / 32);
            // grid-stride warps in one wave of resident CTAs: a second,
            // partial wave left SMs idle at the end (FP32 128^3: 48.4 -> 45.3 us)
            (void)grid;
            static int res_nb[2] = {0, 0};
            if (A.st_nb == 9)
                launch_one_wave(spmv_stencil_kernel<T, EPI, 9>, res_nb[1], s, A.n_rows, A, op, st);
            else
                launch_one_wave(spmv_stencil_kernel<T, EPI, 3>, res_nb[0], s, A.n_rows, A, op, st);
            return;
        }
    }
    const int ntiles = seg.t1 - seg.t0, nlong = seg.l1 - seg.l0;
    const int stage_elems = (kBlock / 32) * 32 * A.sell_lmax;
    const size_t sell_sm = (((A.npat + 1 + A.ndelta) * 4 + 127) & ~127) +
                           (size_t)kSellStages * stage_elems * sizeof(T) + kSellStages * 8;
    if (A.use_pat && A.sell_val && A.sell_tma && sell_sm <= kSellTmaMaxSmem) {
        const size_t sm = sell_sm;
        const int chunks = ((seg.r1 - 1) >> 5) - (seg.r0 >> 5) + 1;
        int grid = (chunks + kBlock / 32 - 1) / (kBlock / 32);
        const int cap = s.num_sms * 2;
        if (grid > cap) grid = cap;
        if (grid < 1) grid = 1;
        spmv_sell_tma_kernel<T, EPI><<<grid, kBlock, sm, st>>>(A, seg, op, s, stage_elems);
        return;
    }
    if (A.use_pat && A.sell_val) {
        const int chunks = ((seg.r1 - 1) >> 5) - (seg.r0 >> 5) + 1;
        int grid = (chunks + kBlock / 32 - 1) / (kBlock / 32);
        const int cap = s.num_sms * 8;
        if (grid > cap) grid = cap;
        if (grid < 1) grid = 1;
        const size_t sm = sizeof(int) * (A.npat + 1 + A.ndelta);
        spmv_sell_kernel<T, EPI><<<grid, kBlock, sm, st>>>(A, seg, op, s);
        return;
    }
    if (A.use_pat) {
        const int rpb = kBlock >> A.lg;
        int grid = (seg.r1 - seg.r0 + rpb - 1) / rpb;
        const int cap = s.num_sms * 8;
        if (grid > cap) grid = cap;
        if (grid < 1) grid = 1;
        const int staged = A.nlines * rpb + A.span_sum;
        // measured on B200 (128^3 Q1): staging x per 64-row tile costs more
        // (two barriers and nine short line copies per tile) than the L1 hits
        // of the direct gathers save, so it is opt-in
        if (A.stage_x && A.nlines > 0 && staged <= kMaxStagedX) {
            const int head = (A.npat + 1 + A.ndelta + 2 * A.nlines + 1 + 3) & ~3;
            const size_t sm = sizeof(int) * (head + 2) + sizeof(T) * staged;
            spmv_pattern_staged_kernel<T, EPI><<<grid, kBlock, sm, st>>>(A, seg, op, s, A.n_cols);
            return;
        }
        const size_t sm = sizeof(int) * (A.npat + 1 + A.ndelta);
        spmv_pattern_kernel<T, EPI><<<grid, kBlock, sm, st>>>(A, seg, op, s);
        return;
    }
    if (A.cfg == kSpmvDirect) {
        const int rpb = kBlock >> A.lg;
        int grid = (seg.r1 - seg.r0 + rpb - 1) / rpb;
        const int cap = s.num_sms * 8;
        if (grid > cap) grid = cap;
        if (grid < 1) grid = 1;
        spmv_direct_kernel<T, EPI><<<grid, kBlock, 0, st>>>(A, seg, op, s);
        return;
    }
    const int minb = A.cfg == kSpmvTileSmall ? 4 : 2;
    int grid = ntiles;
    const int lg_need = (nlong + kBlock / 32 - 1) / (kBlock / 32);
    if (lg_need > grid) grid = lg_need;
    const int cap = s.num_sms * minb;
    if (grid > cap) grid = cap;
    if (grid < 1) grid = 1;
    if (A.cfg == kSpmvTileSmall) launch_tile<T, EPI, 1024, 3, 4>(grid, A, seg, op, s, st);
    else launch_tile<T, EPI, 2048, 4, 2>(grid, A, seg, op, s, st);
}

template <typename T>
cudaError_t launch_t(const Scratch &s, const CsrView &A, const Seg &seg, const SpmvOp &op, cudaStream_t st)
{
    switch (op.epi) {
    case EPI_SET: launch_epi<T, EPI_SET>(s, A, seg, op, st); break;
    case EPI_ADD: launch_epi<T, EPI_ADD>(s, A, seg, op, st); break;
    case EPI_DOT_X: launch_epi<T, EPI_DOT_X>(s, A, seg, op, st); break;
    case EPI_RESID: launch_epi<T, EPI_RESID>(s, A, seg, op, st); break;
    case EPI_SGS_F: launch_epi<T, EPI_SGS_F>(s, A, seg, op, st); break;
    case EPI_SGS_B: launch_epi<T, EPI_SGS_B>(s, A, seg, op, st); break;
    case EPI_ILU_F: launch_epi<T, EPI_ILU_F>(s, A, seg, op, st); break;
    case EPI_ILU_B: launch_epi<T, EPI_ILU_B>(s, A, seg, op, st); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace

int spmv_tile_cap(int cfg) { return cfg == kSpmvTileSmall ? 1024 : 2048; }

namespace {
template <typename T>
__global__ void csr_to_sell_kernel(int n, const int *__restrict__ row, const T *__restrict__ val,
                                   const int *__restrict__ sell_off, T *__restrict__ sv)
{
    for (int r = blockIdx.x * kBlock + threadIdx.x; r < n; r += gridDim.x * kBlock) {
        const int base = sell_off[r >> 5] + (r & 31);
        const int j0 = row[r], len = row[r + 1] - j0;
        for (int k = 0; k < len; ++k) sv[base + (k << 5)] = val[j0 + k];
    }
}
}  // namespace

cudaError_t launch_csr_to_sell(int dtype, int n, const int *row, const void *val, const int *sell_off, void *sv,
                               cudaStream_t st)
{
    const int g = (n + kBlock - 1) / kBlock < 148 * 8 ? (n + kBlock - 1) / kBlock : 148 * 8;
    if (g < 1) return cudaSuccess;
    if (dtype == 0)
        csr_to_sell_kernel<double><<<g, kBlock, 0, st>>>(n, row, (const double *)val, sell_off, (double *)sv);
    else
        csr_to_sell_kernel<float><<<g, kBlock, 0, st>>>(n, row, (const float *)val, sell_off, (float *)sv);
    return cudaGetLastError();
}

namespace {
struct StencilUnion {
    int u[3 * kMaxBands];
};

template <typename T>
__global__ void csr_to_stencil_kernel(int n, const int *__restrict__ row, const int *__restrict__ col,
                                      const T *__restrict__ val, StencilUnion un, int L, T *__restrict__ out)
{
    constexpr int W = stencil_group<T>();
    const int G = (L + W - 1) / W;
    for (int r = blockIdx.x * kBlock + threadIdx.x; r < n; r += gridDim.x * kBlock) {
        const size_t base = (size_t)(r >> 5) * 32 * G * W + (size_t)(r & 31) * W;
        for (int j = row[r]; j < row[r + 1]; ++j) {
            const int dl = col[j] - r;
            for (int k = 0; k < L; ++k)
                if (un.u[k] == dl) out[base + (size_t)(k / W) * 32 * W + k % W] = val[j];
        }
    }
}
}  // namespace

cudaError_t launch_csr_to_stencil(int dtype, int n, const int *row, const int *col, const void *val, const int *uni,
                                  int nb, void *out, cudaStream_t st)
{
    StencilUnion un;
    const int L = 3 * nb;
    for (int k = 0; k < 3 * kMaxBands; ++k) un.u[k] = k < L ? uni[k] : 0;
    const int g = (n + kBlock - 1) / kBlock < 148 * 8 ? (n + kBlock - 1) / kBlock : 148 * 8;
    if (g < 1) return cudaSuccess;
    if (dtype == 0)
        csr_to_stencil_kernel<double><<<g, kBlock, 0, st>>>(n, row, col, (const double *)val, un, L, (double *)out);
    else
        csr_to_stencil_kernel<float><<<g, kBlock, 0, st>>>(n, row, col, (const float *)val, un, L, (float *)out);
    return cudaGetLastError();
}

namespace {
struct HalfCenters {
    int c[kMaxBands];
};

// position k of row r in the full stencil layout
template <typename T>
__device__ __forceinline__ size_t full_at(int r, int k, int L)
{
    constexpr int W = stencil_group<T>();
    const int G = (L + W - 1) / W;
    return (size_t)(r >> 5) * 32 * G * W + (size_t)(k / W) * 32 * W + (size_t)(r & 31) * W + k % W;
}

template <typename T>
__device__ __forceinline__ bool is_zero_bits(T v)
{
    if constexpr (sizeof(T) == 8) return __double_as_longlong(v) == 0;
    else return __float_as_uint(v) == 0u;
}

// Pass 1: sh_mask[c] bit l = row 32 c + l has no off-diagonal value other
// than +0.0 (rows past n count as such).
template <typename T>
__global__ void half_mask_kernel(int n, int nb, const T *__restrict__ st, unsigned *__restrict__ mask)
{
    const int L = 3 * nb, diag = 3 * ((nb - 1) / 2) + 1;
    const int rows = ((n + 31) >> 5) << 5;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        bool ident = true;
        if (r < n)
            for (int k = 0; k < L; ++k)
                if (k != diag && !is_zero_bits(st[full_at<T>(r, k, L)])) ident = false;
        const unsigned bits = __ballot_sync(0xffffffffu, ident);
        if ((threadIdx.x & 31) == 0) mask[r >> 5] = bits;
    }
}

// Pass 2: the diagonal and upper half of every row, checked for symmetry.
template <typename T>
__global__ void half_build_kernel(int n, int nb, HalfCenters hc, const T *__restrict__ st,
                                  const unsigned *__restrict__ mask, T *__restrict__ sh, int *asym)
{
    const int L = 3 * nb, U = (nb - 1) / 2, diag = 3 * U + 1;
    const int rows = ((n + 31) >> 5) << 5;
    auto flagged = [&](int q) { return (mask[q >> 5] >> (q & 31)) & 1u; };
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        const bool fr = flagged(r);
        // upper slot j: j = 0 the +1 entry (k = diag + 1), j = 1 + 3 u + m band U + 1 + u
        auto upper = [&](int j) -> T {
            const int k = j == 0 ? diag + 1 : 3 * (U + 1) + (j - 1);
            const int q = r + hc.c[k / 3] + k % 3 - 1, kk = L - 1 - k;
            const bool inr = r < n && q >= 0 && q < n;
            if (r >= n) return T(0);
            if (fr) return inr ? st[full_at<T>(q, kk, L)] : T(0);
            const T v = st[full_at<T>(r, k, L)];
            if (inr && !flagged(q)) {
                const T w = st[full_at<T>(q, kk, L)];
                const bool same = sizeof(T) == 8 ? __double_as_longlong((double)v) == __double_as_longlong((double)w)
                                                 : __float_as_uint((float)v) == __float_as_uint((float)w);
                if (!same) atomicOr(asym, 1);
            }
            return v;
        };
        const T dv = r < n ? st[full_at<T>(r, diag, L)] : T(0);
        const size_t c = r >> 5, lane = r & 31;
        if constexpr (sizeof(T) == 8) {
            const int H = 2 + 3 * U;
            T *o = sh + c * H * 32 + lane;
            o[0] = dv;
            for (int j = 0; j < 1 + 3 * U; ++j) o[32 * (1 + j)] = upper(j);
        } else {
            const int GH = U < 2 ? 2 : U;
            T *o = sh + c * GH * 128 + lane * 4;
            for (int g = 0; g < GH; ++g) {
                T *q4 = o + 128 * g;
                for (int m = 0; m < 3; ++m) q4[m] = g < U ? upper(1 + 3 * g + m) : T(0);
                q4[3] = g == 0 ? dv : g == 1 ? upper(0) : T(0);
            }
        }
    }
}
}  // namespace

cudaError_t launch_stencil_to_half(int dtype, int n, int nb, const int *center, const void *st_val, void *sh_val,
                                   unsigned *sh_mask, int *asym, cudaStream_t st)
{
    HalfCenters hc;
    for (int b = 0; b < kMaxBands; ++b) hc.c[b] = b < nb ? center[b] : 0;
    const int rows = ((n + 31) / 32) * 32;
    const int g = (rows + kBlock - 1) / kBlock < 148 * 8 ? (rows + kBlock - 1) / kBlock : 148 * 8;
    if (g < 1) return cudaSuccess;
    if (dtype == 0) {
        half_mask_kernel<double><<<g, kBlock, 0, st>>>(n, nb, (const double *)st_val, sh_mask);
        half_build_kernel<double><<<g, kBlock, 0, st>>>(n, nb, hc, (const double *)st_val, sh_mask, (double *)sh_val,
                                                        asym);
    } else {
        half_mask_kernel<float><<<g, kBlock, 0, st>>>(n, nb, (const float *)st_val, sh_mask);
        half_build_kernel<float><<<g, kBlock, 0, st>>>(n, nb, hc, (const float *)st_val, sh_mask, (float *)sh_val,
                                                       asym);
    }
    return cudaGetLastError();
}

cudaError_t spmv_configure()
{
    cudaError_t e;
    if ((e = configure_tile<double, 2048, 4, 2>())) return e;
    if ((e = configure_tile<float, 2048, 4, 2>())) return e;
    if ((e = configure_tile<double, 1024, 3, 4>())) return e;
    if ((e = configure_tile<float, 1024, 3, 4>())) return e;
    if ((e = configure_sell<double>())) return e;
    return configure_sell<float>();
}

cudaError_t launch_spmv(const Scratch &s, const CsrView &A, const Seg &seg, const SpmvOp &op, cudaStream_t st)
{
    if (seg.r1 <= seg.r0) return cudaSuccess;
    return A.dtype == 0 ? launch_t<double>(s, A, seg, op, st) : launch_t<float>(s, A, seg, op, st);
}

}  // namespace b200
