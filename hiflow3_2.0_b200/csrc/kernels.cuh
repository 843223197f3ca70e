// kernels.cuh -- launch interface of the B200 lmp platform kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace b200 {

// Matrix tiles: a run of whole rows [r0, r1) whose nonzeros [row[r0], row[r1])
// fit one shared-memory stage.  a0/a1 are that nonzero range widened to
// multiples of 4 elements, the unit the bulk-copy engine moves (16 bytes of
// column indices, 32 / 16 bytes of double / float values).
struct Tile {
    int r0, r1, a0, a1;
};

// Row segment [r0, r1) of a matrix schedule: tiles [t0, t1) and overlong rows
// [l0, l1) (rows with more nonzeros than one stage holds, done warp-per-row).
struct Seg {
    int t0, t1, l0, l1, r0, r1;
};

constexpr int kCtasPerSm = 2;    // persistent CTAs per SM of the widest tile variant (grid caps)

// IterateControl state kept in device memory by the fused solvers.
struct DevState {
    double rho, alpha, beta, res, res0, pap, rz, rr;
    double abstol, reltol, divtol, pad0;
    int iter, status, maxits, hist_len;
    double *hist;     // optional residual history (hist_len entries)
};

enum Status : int { kIterate = 0, kSuccessAbs = 1, kSuccessRel = 2, kFailDiv = 3, kFailMaxits = 4 };

#ifdef __CUDACC__
// IterateControl::Check (src/common/iterate_control.cc:84-110), first step 0.
__device__ __forceinline__ int check_state(DevState *st, int step, double value)
{
    if (step == 0) st->res0 = value;
    if (value < st->abstol) return kSuccessAbs;
    if (value < st->reltol * st->res0) return kSuccessRel;
    if (value > st->divtol * st->res0) return kFailDiv;
    if (step >= st->maxits) return kFailMaxits;
    return kIterate;
}
// The Jacobi-CG direction p_new = beta p + z with z = r d (cg.cc:241 and
// lpreconditioner.cc:127-165): one rounding of r d, then one fused
// multiply-add.
__device__ __forceinline__ double cg_direction(double beta, double p, double r, double d)
{
    return fma(beta, p, __dmul_rn(r, d));
}
__device__ __forceinline__ float cg_direction(float beta, float p, float r, float d)
{
    return fmaf(beta, p, __fmul_rn(r, d));
}
#endif

// SpMV kernel variants (chosen per matrix when it is created):
//   kSpmvTileWide  -- bulk-copy tiles of <= 2048 nonzeros, 4 stages, 2 CTAs/SM
//   kSpmvTileSmall -- bulk-copy tiles of <= 1024 nonzeros, 3 stages, 4 CTAs/SM
//   kSpmvDirect    -- no staging: 2^lg lanes per row read values / indices
//                     with streaming loads, high occupancy, x through L1
enum SpmvCfg : int { kSpmvTileWide = 0, kSpmvTileSmall = 1, kSpmvDirect = 2 };
int spmv_tile_cap(int cfg);

// SpMV epilogues (per row i, s = sum_j a_ij x_j):
enum Epi : int {
    EPI_SET = 0,     // y_i = s
    EPI_ADD = 1,     // y_i += s
    EPI_DOT_X = 2,   // y_i = s; reduce x_i * y_i
    EPI_RESID = 3,   // y_i = b_i - s; reduce y_i^2
    EPI_SGS_F = 4,   // y_i = (-b_i + s) * d1_i            (MC-SGS forward, d1 = -1/d)
    EPI_SGS_B = 5,   // y_i = (y_i * d2_i + s) * d1_i      (MC-SGS diagonal + backward, d2 = -d)
    EPI_ILU_F = 6,   // y_i = -(-b_i + s)                  (ILU forward, unit L)
    EPI_ILU_B = 7,   // y_i = (-y_i + s) * d1_i            (ILU backward, d1 = -1/u_ii)
    // the last colour's forward step followed by its backward step, which has
    // no couplings (nothing lies right of the last colour): the two epilogues
    // in turn, with the backward sum 0 -- the same roundings as two launches
    EPI_SGS_FB = 8,  // y_i = (-b_i + s) * d1_i;  y_i = (y_i * d2_i + 0) * d1_i
    EPI_ILU_FB = 9,  // y_i = -(-b_i + s);        y_i = (-y_i + 0) * d1_i
};

// What the last CTA does with a reduced value v (EPI_DOT_X / EPI_RESID).
enum Fin : int {
    FIN_NONE = 0,
    FIN_STORE = 1,       // *dot_out = v
    FIN_CG_ALPHA = 2,    // st->pap = v; st->alpha = st->rho / v
    FIN_RES_INIT = 3,    // st->rr = v; st->res = sqrt(v); st->status = Check(0, res)
};

constexpr int kMaxBands = 9;
// Positions per lane and load in the stencil layout: FP32 values are grouped
// by four (position k of row 32 c + lane at
// 32 G W c + 32 W (k / W) + W lane + k % W, G = ceil(3 nb / W)), FP64 by one.
template <typename T>
__host__ __device__ constexpr int stencil_group()
{
    return sizeof(T) == 4 ? 4 : 1;
}
inline size_t stencil_len(int n, int nb, int dtype)
{
    const int W = dtype == 1 ? 4 : 1, G = (3 * nb + W - 1) / W;
    return (size_t)((n + 31) / 32) * 32 * G * W;
}
// Half stencil layout of a symmetric stencil operator (see spmv.cu): U =
// (nb - 1) / 2 bands above the centre band.  FP64 stores 2 + 3 U positions
// per row (diagonal, +1, the upper bands); FP32 stores max(U, 2) groups of
// four (group u: band U + 1 + u in slots 0-2; slot 3 holds the diagonal in
// group 0 and the +1 entry in group 1).
__host__ __device__ constexpr int half_positions(int nb) { return 2 + 3 * ((nb - 1) / 2); }
__host__ __device__ constexpr int half_groups(int nb) { return (nb - 1) / 2 < 2 ? 2 : (nb - 1) / 2; }
inline size_t half_len(int n, int nb, int dtype)
{
    const size_t rows = (size_t)((n + 31) / 32) * 32;
    return dtype == 1 ? rows * 4 * half_groups(nb) : rows * half_positions(nb);
}

struct CsrView {
    const int *row;
    const int *col;
    const void *val;
    const Tile *tiles;
    const int *long_rows;
    int lg;          // log2 of lanes per row
    int dtype;       // 0 double, 1 float
    int cfg;         // SpmvCfg
    // row-pattern dictionary (used when use_pat): column j of row i is
    // i + pat_delta[pat_off[pid[i]] + (j - row[i])]
    const uint16_t *pid;
    const int *pat_off;
    const int *pat_delta;
    int npat, ndelta, use_pat;
    // gather lines of the dictionary (x staged in shared memory per row tile
    // when nlines > 0): see host::pattern_lines
    const int *line_start, *line_span, *entry_line, *entry_lo;
    int nlines, span_sum;
    int stage_x;     // stage x through shared memory (B200LA_STAGE_X=1)
    int l2hint;      // L2 priorities (B200LA_L2HINT): bit 0 CSR streams evict-first, bit 1 CSR gathers
                     // evict-last, bit 2 stencil / lattice values evict-first, bit 3 half layout's own rows
                     // evict-first, bit 4 half layout's chunk lines prefetched into L2
    // sliced layout of the dictionary operator (null when absent): chunk c of
    // 32 rows holds its values k-major at sell_val[sell_off[c] + 32 k + lane]
    const int *sell_off;
    const void *sell_val;
    int sell_lmax;   // longest chunk (values per row) of the sliced layout
    int sell_tma;    // bulk-copy tiles for the sliced layout
    int n_cols;      // length of x
    int n_rows;
    // stencil layout (null when absent): the row patterns' offsets all lie in
    // st_nb bands {c - 1, c, c + 1} (centres st_center[], ascending); the
    // value of row i = 32 c + lane at offset st_center[b] + m - 1 is position
    // k = 3 b + m of the row (see stencil_group for the address), zero where
    // the row has no such column
    const void *st_val;
    int st_nb, st_use;
    int st_center[kMaxBands];
    // half stencil layout (null when absent: the operator is not symmetric
    // outside its identity rows): sh_val by half_positions / half_groups,
    // sh_mask[c] bit l set when row 32 c + l has no nonzero off-diagonal value
    const void *sh_val;
    const unsigned *sh_mask;
    int sh_use;
};

// Lattice layout of an operator in the multicolour numbering of a structured
// Q1 node grid (mx x my x mz nodes, lexicographic, x fastest), coloured by
// node parity -- colour c = px + 2 py + 4 pz holds the nodes whose coordinate
// parities are (px, py, pz), in lexicographic order.  This is the colouring
// and permutation the greedy multicolouring gives on such a grid.  Row t of
// colour c is node (2 xs + px, 2 ys + py, 2 zs + pz) with t = (zs ny + ys) nx
// + xs, and its neighbour at (dx, dy, dz) sits in colour c ^ (|dx| + 2|dy| +
// 4|dz|) at a row computed the same way, so no index is stored: a colour
// keeps, per 32-row chunk, the values of its nslot neighbour positions
// k-major (slot k of all 32 rows together), zero where a row lacks the
// neighbour.  Slots are ordered by (neighbour colour, dz, dy, dx), which is
// the row's ascending column order in the coloured numbering.
constexpr int kLatMaxColours = 8;
constexpr int kLatMaxSlots = 27;
struct LatticeColour {
    int row0, rows;          // rows [row0, row0 + rows) of the coloured numbering
    int nx, ny;              // sublattice extents in x and y
    int px, py, pz;          // coordinate parities of the colour
    int nslot;               // stored positions per row
    int chunk0;              // first chunk of the colour (chunks of all colours numbered together)
    int pad;
    long long val0;          // offset of the colour's values (elements)
    // slot k: (dx + 1) | (dy + 1) << 2 | (dz + 1) << 4 | neighbour colour << 8
    unsigned slot[kLatMaxSlots];
};
struct LatticeDesc {
    int ncol, mx, my, mz;    // colours (4 in 2-D, 8 in 3-D) and node extents (mz = 1 in 2-D)
    int chunks;              // chunks of all colours
    int part;                // 0 strictly lower, 1 strictly upper, 2 whole operator
    int l2hint;              // the matrix's L2 hint (bit 2: the value stream evict-first)
    int pad;
    LatticeColour col[kLatMaxColours];
};

constexpr int kMaxPatterns = 1024;
constexpr int kMaxPatternDeltas = 6144;
constexpr int kMaxGatherLines = 64;
constexpr int kMaxStagedX = 6144;     // staged x values per row tile

struct SpmvOp {
    int epi = EPI_SET;
    int fin = FIN_NONE;
    const void *x = nullptr;
    void *y = nullptr;
    const void *b = nullptr;
    const void *d1 = nullptr;
    const void *d2 = nullptr;
    double *dot_out = nullptr;
    DevState *st = nullptr;
    const int *gate = nullptr;    // skip the launch body when *gate != 0
    // launch as a programmatic dependent of the previous kernel on the stream
    // (lattice colour sweeps only: the value loads overlap the previous
    // colour's tail; every read of what that colour wrote comes after the
    // grid dependency wait, through coherent loads)
    int pdl = 0;
};

struct Scratch {
    double *partials;    // [8][kMaxGrid]
    unsigned *ticket;
    int *err;
    int num_sms;
};

cudaError_t spmv_configure();
// Scatter CSR values (row order) into the sliced layout (zero-filled before).
cudaError_t launch_csr_to_sell(int dtype, int n, const int *row, const void *val, const int *sell_off, void *sv,
                               cudaStream_t st);
// Scatter CSR values into the stencil layout (zero-filled before); uni holds
// the 3 nb offsets of the bands in ascending order.
cudaError_t launch_csr_to_stencil(int dtype, int n, const int *row, const int *col, const void *val, const int *uni,
                                  int nb, void *out, cudaStream_t st);
// Half stencil layout from the full one (same dtype): the identity-row mask,
// the diagonal and upper half (a row without nonzero off-diagonal values
// keeps, in its upper slots, the transposed entries its neighbours need),
// and *asym != 0 afterwards when some pair of non-identity rows i, j has
// a_ij != a_ji bitwise.
cudaError_t launch_stencil_to_half(int dtype, int n, int nb, const int *center, const void *st_val, void *sh_val,
                                   unsigned *sh_mask, int *asym, cudaStream_t st);
cudaError_t launch_spmv(const Scratch &s, const CsrView &A, const Seg &seg, const SpmvOp &op, cudaStream_t st);
// Lattice-layout SpMV / colour sweep over colours [c0, c1): y by the epilogue
// of op (EPI_SET, EPI_ADD, EPI_DOT_X, EPI_RESID, EPI_SGS_F/B, EPI_ILU_F/B).
cudaError_t launch_lattice(const Scratch &s, int dtype, const LatticeDesc &d, const void *val, int c0, int c1,
                           const SpmvOp &op, cudaStream_t st);

// ---- BLAS1 (dtype 0 double, 1 float; scalars in double) ----
cudaError_t launch_dot(const Scratch &s, int dtype, int n, const void *x, const void *y, double *out,
                       bool sqrt_out, cudaStream_t st);
cudaError_t launch_axpy(int dtype, int n, double a, const void *x, void *y, cudaStream_t st);
cudaError_t launch_scaleadd(int dtype, int n, double a, const void *x, void *y, cudaStream_t st);
cudaError_t launch_scale(int dtype, int n, double a, void *y, cudaStream_t st);
cudaError_t launch_ewmul(int dtype, int n, const void *x, void *y, cudaStream_t st);
cudaError_t launch_cast(int src_dtype, const void *src, int dst_dtype, void *dst, int n, cudaStream_t st);
cudaError_t launch_gather(int dtype, int n, const int *idx, const void *x, void *out, cudaStream_t st);
cudaError_t launch_scatter(int dtype, int n, const int *idx, const void *vals, void *x, cudaStream_t st);
cudaError_t launch_fill(int dtype, int n, double v, void *y, cudaStream_t st);

// ---- fused Krylov steps (vectors of type dtype, scalars in DevState) ----
// CG update: x += alpha p; r -= alpha Ap; with invd (Jacobi) reduce rr and
// r.(invd r), without reduce rr only (rz = rr when precond == 0, nothing when
// precond == 2: the caller reduces r.z after its own apply).  The last CTA
// advances iter, stores res, runs Check and, when iterating, sets
// beta = rz / rho and rho = rz (precond 0/1).
// cond: a graph conditional handle (0: none) that the last CTA sets to
// "keep iterating" after its Check -- the loop condition of a device-side
// while node around the iterations.
cudaError_t launch_cg_update(const Scratch &s, int dtype, int n, int precond, void *x, void *r, const void *p,
                             const void *Ap, const void *invd, DevState *st, cudaStream_t stm,
                             unsigned long long cond = 0);
// p = beta p + z with z = invd .* r (precond 1), z = r (precond 0), or z given.
cudaError_t launch_cg_pupdate(int dtype, int n, int precond, void *p, const void *r, const void *invd,
                              const void *z, DevState *st, cudaStream_t stm);
// CG start after r = b - A x: z = M r for Jacobi/none, p = z, rho = r.z,
// res = ||r||, status = Check(0, res).  precond 2: caller supplies z.
cudaError_t launch_cg_start(const Scratch &s, int dtype, int n, int precond, const void *r, const void *invd,
                            const void *z, void *p, DevState *st, cudaStream_t stm);
// rz = r.z; beta = rz / rho; rho = rz (gated on status).
cudaError_t launch_cg_rz(const Scratch &s, int dtype, int n, const void *r, const void *z, DevState *st,
                         cudaStream_t stm);
// Mixed precision helpers: rl = (float) r, xl = 0; x += (double) cl.
cudaError_t launch_cast_residual(int n, const double *r, float *rl, float *xl, cudaStream_t st);
cudaError_t launch_add_correction(int n, const float *cl, double *x, cudaStream_t st);

// GMRES pieces (double or float basis; scalars double):
// h[i] = w.v ; then w -= h v  (one modified Gram-Schmidt step), device scalars.
cudaError_t launch_dot_to(const Scratch &s, int dtype, int n, const void *x, const void *y, double *out,
                          const int *gate, cudaStream_t st);
cudaError_t launch_dot_norm_to(const Scratch &s, int dtype, int n, const void *x, double *out, const int *gate,
                               cudaStream_t st);
cudaError_t launch_axpy_dev(int dtype, int n, const double *coef, double sign, const void *x, void *y,
                            const int *gate, cudaStream_t st);
cudaError_t launch_scale_dev(int dtype, int n, const double *coef, bool reciprocal, const void *x, void *y,
                             const int *gate, cudaStream_t st);

}  // namespace b200
