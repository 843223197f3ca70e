// serve.cuh -- device layout of the continuous-batching solve server.
//
// Every resident request (a "slot") owns one SysDesc in a device table and
// one SysState.  Its operator is stored in 32-row chunks: the SELL layout
// (chunk c holds its rows' entries k-major, sell[off[c] + 32 k + lane], rows
// zero-padded to the chunk's longest row) or, for rows too long for that, the
// CSR with one warp per row.  Two batched kernels advance every active
// system by one iteration of its Krylov recurrence; a system table lists the
// active systems and where their chunks start in the batch's chunk sequence.
//
// Determinism: a system's arithmetic never depends on the batch it is in.
// Row sums run in a fixed order (one thread per row in column order, or a
// fixed shuffle tree per row).  Reductions go through one partial per 32-row
// chunk; the warp that completes a group of 32 chunks sums them by a fixed
// shuffle tree, and the warp that completes the last group sums the group
// partials in a fixed order.  Warp ranges, block size, grid size and the
// other systems of the batch change only the schedule.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace b200 {
namespace srv {

// Per-system phase of the state machine run by the two kernels.
//   FP64 Jacobi-PCG (CG<LAD>::SolvePrecond, src/linear_solver/cg.cc:164-248):
//     CG_START (update kernel: r = b, rho = r.z, res0) -> CG ... -> DONE
//   Mixed (MPIR<LAD_high, LAD_low>::Solve, src/linear_solver/mpir.cc:69-326,
//   with an FP32 Jacobi-CG error correction):
//     OUTER (update kernel: r = b - A x in FP64, r_low = (float) r, x_low = 0)
//       -> INNER (FP32 CG on A x_low = r_low) -> CORRECT (SpMV kernel:
//       x += (double) x_low; update kernel: the next outer residual) -> ... -> DONE
enum Phase : int { PH_CG_START = 0, PH_CG = 1, PH_OUTER = 2, PH_INNER = 3, PH_CORRECT = 4, PH_DONE = 5 };
// FMT_STENCIL: a structured Q1 operator stored by stencil position: entry k
// of row i is the coupling to column i + delta_k (the 9 / 27 offsets
// (dk P + dj) P + di in column order, P = N + 1 nodes per line), zero where
// the row has no such neighbour; FP64 values at val64[32 L c + 32 k + lane],
// FP32 values in groups of four positions per lane at
// val32[128 G c + 128 (k / 4) + 4 lane + k % 4], G = ceil(L / 4).  No column
// indices or offsets are stored or loaded.
// Half stencil (FMT_STENCIL with half = 1: Q1 Poisson requests, symmetric
// outside their identity rows): only the diagonal and the upper half are
// stored, and a row's lower half is read from the rows that own it (see
// half_len64 / half_len32); smask[c] bit l flags row 32 c + l as an identity
// row (no nonzero off-diagonal value), which uses its diagonal alone and
// keeps in its upper slots the transposed entries its neighbours need.
enum Fmt : int { FMT_SELL = 0, FMT_CSRW = 1, FMT_STENCIL = 2 };

constexpr int kChunk = 32;          // rows per chunk
constexpr int kFinLanes = 256;      // virtual lanes of the per-system final sums
constexpr int kTicketWords = 32;    // the system ticket of a slot, alone on its 128-byte line
constexpr int kGroup = 32;          // chunks per reduction group
constexpr int kMaxRowSell = 64;     // longest row kept in the SELL layout

struct SysState {
    double rho, alpha, beta, res, res0, res_in0;
    double abstol, reltol, divtol, in_abstol, in_reltol, in_divtol;
    int iter;        // FP64: CG iterations; mixed: inner iterations in total
    int inner_iter;  // mixed: iterations of the running inner solve
    int outer;       // mixed: corrections applied
    int status;      // B200LA_ITERATE / SUCCESS_* / FAIL_*
    int phase, maxits, in_maxits, max_outer;
    int pbuf;        // which of the two search-direction buffers holds p
    int corr;        // mixed: the update kernel applies x += x_low (1) or only clears x_low (2)
    int pad[2];
};

struct SysDesc {
    int n, nchunks, mixed, fmt;
    int pstride;           // chunk partials per quantity (nchunks rounded up to even)
    int sdim, sP, sL;      // FMT_STENCIL: dimension, nodes per line, stencil width
    int ngroups, gstride;  // reduction groups of kGroup chunks; group partials per quantity
    int half, hpad;        // FMT_STENCIL: half stencil layout (1) or full (0)
    const unsigned *smask; // half stencil: identity-row mask per chunk [nchunks + 1; the last word: set-up check]
    const int *off;        // SELL: chunk offsets [nchunks + 1]; CSRW: row pointer [n + 1]
    const int *col;
    const double *val64;
    const float *val32;    // mixed only
    const double *b;
    double *x;
    void *r, *z, *p0, *p1, *ap, *xl;  // FP64 system: double r, z = D^-1 r, p, Ap; mixed: float ... and x_low
    const void *invd;      // 1 / a_ii: double, or float for mixed
    double *part;          // [3][pstride] chunk partials
    double *gpart;         // [3][gstride] group partials
    unsigned *gcnt;        // [ngroups] chunks reported per group (0 between launches)
    unsigned *ticket;      // groups completed (0 between launches)
    int *done;             // final status word polled by the host (0 while running)
};

// Half stencil layout: U = 4 (3-D) or 1 (2-D) bands above the centre band.
// FP64: per 32-row chunk, half_len64 positions position-major
// (val64[32 H c + 32 p + lane]): p = 0 the diagonal, p = 1 the +1 entry,
// p = 2 + 3 u + m position m of upper band U + 1 + u.  FP32: per chunk,
// half_len32 floats per row: U groups of four (val32[32 H c + 128 u + 4 lane
// + m]: band U + 1 + u in slots 0-2; slot 3 the diagonal in group 0, the +1
// entry in group 1, zero above), and when U = 1 the +1 entry alone after the
// groups (val32[32 H c + 128 U + lane]).
__host__ __device__ __forceinline__ int half_u(int dim) { return dim == 3 ? 4 : 1; }
__host__ __device__ __forceinline__ int half_len64(int dim) { return 2 + 3 * half_u(dim); }
__host__ __device__ __forceinline__ int half_len32(int dim) { return 4 * half_u(dim) + (half_u(dim) < 2 ? 1 : 0); }

// Column offset of stencil position k (column order).
__host__ __device__ __forceinline__ int stencil_delta(int dim, int P, int k)
{
    return dim == 3 ? ((k / 9 - 1) * P + (k / 3 % 3 - 1)) * P + (k % 3 - 1) : (k / 3 - 1) * P + (k % 3 - 1);
}

// Active system: slot, first chunk in the batch's chunk sequence, chunk
// count, and per kernel (SpMV k1, update k2) the cost weight of one chunk
// (bytes per row it streams) and the system's first position in the
// weighted sequence (ascending).  Warps split the weighted sequence evenly,
// so a 3-D FP64 chunk counts for about five 2-D FP32 ones.
struct SysRun {
    int slot, cbeg, nch, w1, w2, wb1, wb2, pad;
};

// System table in device memory: words [0] systems, [1] chunks in total,
// [2] unused, [3] unused, [4] total weight of k1, [5] total weight of k2;
// entries from word 8.
constexpr int kTabHdrWords = 8;

// One batch iteration (SpMV kernel, update kernel) over the system table.
// SysDesc and SysState tables are indexed by slot.
cudaError_t launch_round(int nw, int grid, const SysDesc *sys, SysState *state, const int *tab, cudaStream_t st);
// CSR (device, FP64) -> the slot's chunk layout, 1 / a_ii, and FP32 values when mixed.
cudaError_t launch_build_slot(const SysDesc &d, const int *row, const int *col, const double *val,
                              cudaStream_t st);

}  // namespace srv

cudaError_t launch_q1_assemble(int dim, int N, int kind, const double *kcell, double nu, const double *beta, int *row,
                               int *col, double *val, cudaStream_t st);
cudaError_t launch_q1_rhs(unsigned long long seed, int dim, int N, double *b, cudaStream_t st);

}  // namespace b200
