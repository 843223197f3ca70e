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

#include <cmath>

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

__device__ __forceinline__ void finalize(const SpmvOp &op, double v)
{
    DevState *st = op.st;
    switch (op.fin) {
    case FIN_STORE: *op.dot_out = v; break;
    case FIN_CG_ALPHA:
        st->pap = v;
        st->alpha = st->rho / v;
        break;
    case FIN_RES_INIT: {
        st->rr = v;
        const double res = sqrt(v);
        st->res = res;
        st->iter = 0;
        if (st->hist && st->hist_len > 0) st->hist[0] = res;
        st->status = check_state(st, 0, res);
        break;
    }
    default: break;
    }
}

template <typename T, int EPI>
__device__ __forceinline__ void epilogue(int r, T s, const SpmvOp &op, double &acc)
{
    T *y = static_cast<T *>(op.y);
    if constexpr (EPI == EPI_SET) {
        y[r] = s;
    } else if constexpr (EPI == EPI_ADD) {
        y[r] += s;
    } else if constexpr (EPI == EPI_DOT_X) {
        y[r] = s;
        acc += (double)(__ldg(static_cast<const T *>(op.x) + r) * s);
    } else if constexpr (EPI == EPI_RESID) {
        const T v = static_cast<const T *>(op.b)[r] - s;
        y[r] = v;
        acc += (double)(v * v);
    } else if constexpr (EPI == EPI_SGS_F) {
        y[r] = (-static_cast<const T *>(op.b)[r] + s) * static_cast<const T *>(op.d1)[r];
    } else if constexpr (EPI == EPI_SGS_B) {
        y[r] = (y[r] * static_cast<const T *>(op.d2)[r] + s) * static_cast<const T *>(op.d1)[r];
    } else if constexpr (EPI == EPI_ILU_F) {
        y[r] = -(-static_cast<const T *>(op.b)[r] + s);
    } else if constexpr (EPI == EPI_ILU_B) {
        y[r] = (-y[r] + s) * static_cast<const T *>(op.d1)[r];
    }
}

template <int EPI>
constexpr bool reduces()
{
    return EPI == EPI_DOT_X || EPI == EPI_RESID;
}

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
    if (op.gate && *reinterpret_cast<const volatile int *>(op.gate) != 0) return;
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
    if (op.gate && *reinterpret_cast<const volatile int *>(op.gate) != 0) return;
    const int *__restrict__ row = A.row;
    const int *__restrict__ col = A.col;
    const T *__restrict__ val = static_cast<const T *>(A.val);
    const T *__restrict__ x = static_cast<const T *>(op.x);
    const int G = 1 << A.lg;
    const int rpb = kBlock >> A.lg;
    const int grp = threadIdx.x >> A.lg;
    const int lane_g = threadIdx.x & (G - 1);
    double acc = 0.0;
    for (int base = seg.r0 + blockIdx.x * rpb; base < seg.r1; base += gridDim.x * rpb) {
        const int r = base + grp;
        const bool active = r < seg.r1;
        T s = T(0);
        if (active) {
            const int j1 = __ldg(row + r + 1);
#pragma unroll 4
            for (int j = __ldg(row + r) + lane_g; j < j1; j += G) s += __ldcs(val + j) * __ldg(x + __ldcs(col + j));
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
    if (op.gate && *reinterpret_cast<const volatile int *>(op.gate) != 0) return;
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
    double acc = 0.0;
    for (int base = seg.r0 + blockIdx.x * rpb; base < seg.r1; base += gridDim.x * rpb) {
        const int r = base + grp;
        const bool active = r < seg.r1;
        T s = T(0);
        if (active) {
            const int j0 = __ldg(row + r), len = __ldg(row + r + 1) - j0;
            const int *d = s_delta + s_off[__ldg(A.pid + r)];
#pragma unroll 4
            for (int k = lane_g; k < len; k += G) s += __ldcs(val + j0 + k) * __ldg(x + r + d[k]);
        }
        for (int o = G >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (active && lane_g == 0) epilogue<T, EPI>(r, s, op, acc);
    }
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

template <typename T, int EPI>
void launch_epi(const Scratch &s, const CsrView &A, const Seg &seg, const SpmvOp &op, cudaStream_t st)
{
    const int ntiles = seg.t1 - seg.t0, nlong = seg.l1 - seg.l0;
    if (A.use_pat) {
        const int rpb = kBlock >> A.lg;
        int grid = (seg.r1 - seg.r0 + rpb - 1) / rpb;
        const int cap = s.num_sms * 8;
        if (grid > cap) grid = cap;
        if (grid < 1) grid = 1;
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

cudaError_t spmv_configure()
{
    cudaError_t e;
    if ((e = configure_tile<double, 2048, 4, 2>())) return e;
    if ((e = configure_tile<float, 2048, 4, 2>())) return e;
    if ((e = configure_tile<double, 1024, 3, 4>())) return e;
    return configure_tile<float, 1024, 3, 4>();
}

cudaError_t launch_spmv(const Scratch &s, const CsrView &A, const Seg &seg, const SpmvOp &op, cudaStream_t st)
{
    if (seg.r1 <= seg.r0) return cudaSuccess;
    return A.dtype == 0 ? launch_t<double>(s, A, seg, op, st) : launch_t<float>(s, A, seg, op, st);
}

}  // namespace b200
