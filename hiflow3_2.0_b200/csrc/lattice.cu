// lattice.cu -- index-free layout of multicoloured structured Q1 operators.
//
// The multicolour preconditioners (lmp/lpreconditioner_mc.cc:157-777, with
// the symmetric Gauss-Seidel sweeps of lpreconditioner_mc_sgs.cc:46-90 and
// lpreconditioner_mc_gs.cc:52-135) permute the operator into colour blocks and
// sweep block by block.  On a Q1 grid in lexicographic node order the greedy
// colouring (lmatrix_csr_cpu.cc:2175-2290) gives the node-parity classes, each
// in lexicographic order; then every row's columns follow from its position
// in its colour, and the sweeps and the coloured operator's SpMV need only the
// values.  At 128^3 (FP64) the strictly lower and upper parts drop from
// 12 (nnz - n) bytes with indices to 8 x 26 bytes per row, and the coloured
// operator from 12 nnz + 4 n to 8 x 27 bytes per row.
//
// Set-up (host): lattice::grid() reads the node grid off row 0's columns,
// lattice::perm_ok() checks that the colouring is the parity colouring, and
// lattice::values() places every CSR entry of a part (strictly lower, strictly
// upper, or all) into its neighbour slot, failing on any entry that is not a
// lattice neighbour of its row or that breaks the slot order -- the caller
// then keeps the CSR path.  Products are added in slot order, which is the
// row's CSR (ascending column) order; absent neighbours add nothing.
//
// Kernels: one instance per colour and part, so the slot table is a
// compile-time constant (neighbour offsets, neighbour colours, which grid
// bounds to test); the colour sweeps after the first launch of an apply run
// as programmatic dependents of the previous one (value loads first, then
// griddepcontrol.wait before anything an earlier colour wrote).
#include "b200la.h"
#include "b200la_internal.h"
#include "spmv_epi.cuh"

#include <algorithm>
#include <cstdlib>
#include <type_traits>
#include <vector>

namespace b200 {

namespace {

constexpr int kLatGroup = 9;   // slots whose loads are issued together

// Neighbour slots of colour c for a part (0 strictly lower: neighbour colour
// < c; 1 strictly upper: > c; 2 every position with the diagonal), ordered by
// (neighbour colour, dz, dy, dx) -- the row's ascending column order.  The
// same table drives the host's placement of the values and, as a compile-time
// constant, the kernels.
struct SlotTab {
    int n;
    signed char dx[kLatMaxSlots], dy[kLatMaxSlots], dz[kLatMaxSlots], cp[kLatMaxSlots];
};

__host__ __device__ constexpr SlotTab slot_table(int dim, int c, int part)
{
    SlotTab t{};
    for (int dz = dim == 3 ? -1 : 0; dz <= (dim == 3 ? 1 : 0); ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int m = (dx != 0 ? 1 : 0) + (dy != 0 ? 2 : 0) + (dz != 0 ? 4 : 0);
                const int cp = c ^ m;
                if ((part == 0 && cp < c) || (part == 1 && cp > c) || part == 2) {
                    t.dx[t.n] = (signed char)dx;
                    t.dy[t.n] = (signed char)dy;
                    t.dz[t.n] = (signed char)dz;
                    t.cp[t.n] = (signed char)cp;
                    ++t.n;
                }
            }
    // insertion sort by (cp, dz, dy, dx)
    for (int i = 1; i < t.n; ++i)
        for (int j = i; j > 0; --j) {
            const int a = ((t.cp[j - 1] * 4 + t.dz[j - 1] + 1) * 4 + t.dy[j - 1] + 1) * 4 + t.dx[j - 1] + 1;
            const int b = ((t.cp[j] * 4 + t.dz[j] + 1) * 4 + t.dy[j] + 1) * 4 + t.dx[j] + 1;
            if (a <= b) break;
            signed char v = 0;
            v = t.dx[j - 1]; t.dx[j - 1] = t.dx[j]; t.dx[j] = v;
            v = t.dy[j - 1]; t.dy[j - 1] = t.dy[j]; t.dy[j] = v;
            v = t.dz[j - 1]; t.dz[j - 1] = t.dz[j]; t.dz[j] = v;
            v = t.cp[j - 1]; t.cp[j - 1] = t.cp[j]; t.cp[j] = v;
        }
    return t;
}

template <int DIM, int C, int PART>
struct Slots {
    static constexpr SlotTab tab = slot_table(DIM, C, PART);
};

// the sublattice step of an offset: floor((parity + d) / 2)
__host__ __device__ constexpr int sub_step(int parity, int d) { return parity + d < 0 ? -1 : (parity + d) / 2; }

// f(integral_constant<K>) for K in [K, N): host code (the launch dispatch)
// and device code (the unrolled slot loops) both use it
template <int K, int N, class F>
__host__ __device__ __forceinline__ void static_for(F &&f)
{
    if constexpr (K < N) {
        f(std::integral_constant<int, K>());
        static_for<K + 1, N>(f);
    }
}

// One 32-row chunk of colour C (chunk g of the launch's numbering): each lane
// forms its row's lattice position, one row base per neighbour colour, and
// then, slot by slot, a column that is that base plus compile-time multiples
// of the neighbour colour's extents.  Neighbours outside the grid (their
// values are zero) are not loaded.
template <typename T, int EPI, int DIM, int PART, int C>
__device__ __forceinline__ void lattice_chunk(const LatticeDesc &d, const T *__restrict__ val,
                                              const T *__restrict__ x, int g, int lane, const SpmvOp &op,
                                              uint64_t pol, uint64_t pol_v, double &acc)
{
    constexpr SlotTab S = Slots<DIM, C, PART>::tab;
    constexpr int px = C & 1, py = (C >> 1) & 1, pz = (C >> 2) & 1;
    const LatticeColour &L = d.col[C];
    const int t = ((g - L.chunk0) << 5) + lane;
    const bool active = t < L.rows;
    // padding lanes of a colour's last chunk take its last row's node
    const int tt = active ? t : L.rows - 1;
    const int q = tt / L.nx, xs = tt - q * L.nx;
    int ys = q, zs = 0;
    if constexpr (DIM == 3) {
        zs = q / L.ny;
        ys = q - zs * L.ny;
    }
    const int X = 2 * xs + px, Y = 2 * ys + py, Z = 2 * zs + pz;
    const bool xlo = X > 0, xhi = X < d.mx - 1, ylo = Y > 0, yhi = Y < d.my - 1, zlo = Z > 0, zhi = Z < d.mz - 1;
    int base[kLatMaxColours];
    static_for<0, kLatMaxColours>([&](auto cc) {
        constexpr int cp = decltype(cc)::value;
        bool used = false;
        for (int k = 0; k < S.n; ++k) used |= S.cp[k] == cp;
        if (used) {
            const LatticeColour &P = d.col[cp];
            base[cp] = P.row0 + (zs * P.ny + ys) * P.nx + xs;
        }
    });
    const T *v = val + L.val0 + (size_t)(g - L.chunk0) * (S.n * 32) + lane;
    T s = T(0);
    // PREALL: every value load of the row issued first (before the grid
    // dependency wait of a sweep), one round trip for all of them.  Measured
    // per kernel: faster for the sweeps and the reducing products, slower for
    // the plain product y = Ax (89.8 -> 92.5 us at 128^3), which keeps groups
    constexpr bool PREALL = S.n > 0 && !(PART == 2 && EPI == EPI_SET);
    T aall[PREALL ? S.n : 1];
    if constexpr (PREALL) {
        static_for<0, S.n>([&](auto kk) {
            constexpr int k = decltype(kk)::value;
            aall[k] = ld_stream(v + 32 * k, pol_v);
        });
        grid_dependency_wait();
    }
    static_for<0, (S.n + kLatGroup - 1) / kLatGroup>([&](auto gg) {
        constexpr int k0 = decltype(gg)::value * kLatGroup;
        constexpr int cnt = S.n - k0 < kLatGroup ? S.n - k0 : kLatGroup;
        T a[kLatGroup], w[kLatGroup];
        static_for<0, cnt>([&](auto jj) {
            constexpr int j = decltype(jj)::value;
            if constexpr (PREALL) a[j] = aall[k0 + j];
            else a[j] = ld_stream(v + 32 * (k0 + j), pol_v);
        });
        // x (what earlier colours wrote) only after the previous launch completed
        if constexpr (!PREALL && decltype(gg)::value == 0) grid_dependency_wait();
        static_for<0, cnt>([&](auto jj) {
            constexpr int j = decltype(jj)::value, k = k0 + j;
            constexpr int dx = S.dx[k], dy = S.dy[k], dz = S.dz[k], cp = S.cp[k];
            constexpr int ex = sub_step(px, dx), ey = sub_step(py, dy), ez = sub_step(pz, dz);
            const LatticeColour &P = d.col[cp];
            int col = base[cp] + ex;
            if constexpr (ey != 0) col += ey * P.nx;
            if constexpr (ez != 0) col += ez * (P.ny * P.nx);
            bool ok = true;
            if constexpr (dx < 0) ok = ok && xlo;
            if constexpr (dx > 0) ok = ok && xhi;
            if constexpr (dy < 0) ok = ok && ylo;
            if constexpr (dy > 0) ok = ok && yhi;
            if constexpr (dz < 0) ok = ok && zlo;
            if constexpr (dz > 0) ok = ok && zhi;
            w[j] = ok ? ld_coherent(x + col, pol) : T(0);
        });
        static_for<0, cnt>([&](auto jj) {
            constexpr int j = decltype(jj)::value;
            s += a[j] * w[j];
        });
    });
    if constexpr (S.n == 0) grid_dependency_wait();   // the epilogue reads and writes vectors
    if (active) epilogue<T, EPI>(L.row0 + t, s, op, acc);
}

// CF >= 0: every chunk belongs to colour CF (one sweep step); CF < 0: chunks
// of colours [c0, c1), each dispatched to its colour's compiled body.
template <typename T, int EPI, int DIM, int PART, int CF>
__global__ void __launch_bounds__(kBlock) lattice_kernel(const __grid_constant__ LatticeDesc d,
                                                         const T *__restrict__ val, int c0, int c1, SpmvOp op,
                                                         Scratch sc)
{
    if (gate_closed(op.gate)) return;
    grid_dependents_launch();
    const T *__restrict__ x = static_cast<const T *>(op.x);
    // gathers evict-last, the value stream evict-first (the matrix's hint):
    // the gathered vector and the solver's vectors stay in L2 (C2 32.9 -> 32.45 ms)
    const uint64_t pol = l2_policy(2), pol_v = l2_policy(d.l2hint & 4 ? 1 : 0);
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    const int nw = gridDim.x * (kBlock / 32);
    const int g0 = d.col[c0].chunk0;
    const int g1 = d.col[c1 - 1].chunk0 + ((d.col[c1 - 1].rows + 31) >> 5);
    double acc = 0.0;
    for (int g = g0 + gw; g < g1; g += nw) {
        if constexpr (CF >= 0) {
            lattice_chunk<T, EPI, DIM, PART, CF>(d, val, x, g, lane, op, pol, pol_v, acc);
        } else {
            int c = c0;
            while (c + 1 < c1 && g >= d.col[c + 1].chunk0) ++c;
            static_for<0, (DIM == 3 ? 8 : 4)>([&](auto cc) {
                constexpr int C = decltype(cc)::value;
                if (c == C) lattice_chunk<T, EPI, DIM, PART, C>(d, val, x, g, lane, op, pol, pol_v, acc);
            });
        }
    }
    if constexpr (reduces<EPI>()) {
        double vv[1] = {acc}, out[1];
        if (grid_reduce<1>(vv, sc.partials, sc.ticket, out)) finalize(op, out[0]);
    }
}

template <typename T, int EPI, int DIM, int PART, int CF>
cudaError_t launch_k(const Scratch &s, const LatticeDesc &d, const void *val, int c0, int c1, const SpmvOp &op,
                     cudaStream_t st)
{
    static int resident = 0;
    auto kern = lattice_kernel<T, EPI, DIM, PART, CF>;
    if (!resident && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kern, kBlock, 0) != cudaSuccess)
        resident = 4;
    const int chunks = d.col[c1 - 1].chunk0 + ((d.col[c1 - 1].rows + 31) >> 5) - d.col[c0].chunk0;
    int grid = (chunks + kBlock / 32 - 1) / (kBlock / 32);
    grid = std::min(grid, std::min(s.num_sms * std::max(resident, 1), kMaxGrid));
    grid = std::max(grid, 1);
    if (!op.pdl) {
        kern<<<grid, kBlock, 0, st>>>(d, static_cast<const T *>(val), c0, c1, op, s);
        return cudaGetLastError();
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kBlock);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, d, static_cast<const T *>(val), c0, c1, op, s);
}

// One sweep step: colour c0 of a strictly lower / upper part.
template <typename T, int EPI, int DIM, int PART>
cudaError_t launch_sweep(const Scratch &s, const LatticeDesc &d, const void *val, int c0, const SpmvOp &op,
                         cudaStream_t st)
{
    cudaError_t e = cudaErrorNotSupported;
    static_for<0, (DIM == 3 ? 8 : 4)>([&](auto cc) {
        constexpr int C = decltype(cc)::value;
        if (c0 == C) e = launch_k<T, EPI, DIM, PART, C>(s, d, val, c0, c0 + 1, op, st);
    });
    return e;
}

template <typename T, int DIM>
cudaError_t launch_dim(const Scratch &s, const LatticeDesc &d, const void *val, int c0, int c1, const SpmvOp &op,
                       cudaStream_t st)
{
    const int part = d.part;
    if (part == 2) {
        switch (op.epi) {
        case EPI_SET: return launch_k<T, EPI_SET, DIM, 2, -1>(s, d, val, c0, c1, op, st);
        case EPI_ADD: return launch_k<T, EPI_ADD, DIM, 2, -1>(s, d, val, c0, c1, op, st);
        case EPI_DOT_X: return launch_k<T, EPI_DOT_X, DIM, 2, -1>(s, d, val, c0, c1, op, st);
        case EPI_RESID: return launch_k<T, EPI_RESID, DIM, 2, -1>(s, d, val, c0, c1, op, st);
        default: return cudaErrorNotSupported;
        }
    }
    if (c1 != c0 + 1) return cudaErrorNotSupported;
    if (part == 0 && op.epi == EPI_SGS_F) return launch_sweep<T, EPI_SGS_F, DIM, 0>(s, d, val, c0, op, st);
    if (part == 0 && op.epi == EPI_ILU_F) return launch_sweep<T, EPI_ILU_F, DIM, 0>(s, d, val, c0, op, st);
    if (part == 0 && c0 == d.ncol - 1 && op.epi == EPI_SGS_FB)
        return launch_k<T, EPI_SGS_FB, DIM, 0, (DIM == 3 ? 7 : 3)>(s, d, val, c0, c1, op, st);
    if (part == 0 && c0 == d.ncol - 1 && op.epi == EPI_ILU_FB)
        return launch_k<T, EPI_ILU_FB, DIM, 0, (DIM == 3 ? 7 : 3)>(s, d, val, c0, c1, op, st);
    if (part == 1 && op.epi == EPI_SGS_B) return launch_sweep<T, EPI_SGS_B, DIM, 1>(s, d, val, c0, op, st);
    if (part == 1 && op.epi == EPI_ILU_B) return launch_sweep<T, EPI_ILU_B, DIM, 1>(s, d, val, c0, op, st);
    return cudaErrorNotSupported;
}

}  // namespace

// cudaErrorNotSupported: no lattice kernel for this part, epilogue and
// colour range (the caller then runs the CSR path).
cudaError_t launch_lattice(const Scratch &s, int dtype, const LatticeDesc &d, const void *val, int c0, int c1,
                           const SpmvOp &op, cudaStream_t st)
{
    if (c0 < 0 || c1 > d.ncol || c0 >= c1) return cudaErrorInvalidValue;
    if (d.ncol == 8)
        return dtype == 0 ? launch_dim<double, 3>(s, d, val, c0, c1, op, st)
                          : launch_dim<float, 3>(s, d, val, c0, c1, op, st);
    return dtype == 0 ? launch_dim<double, 2>(s, d, val, c0, c1, op, st)
                      : launch_dim<float, 2>(s, d, val, c0, c1, op, st);
}

// The host's slot table (the kernels use the same one at compile time).
SlotTab lattice_slots(int dim, int c, int part) { return slot_table(dim, c, part); }

}  // namespace b200

// ------------------------------------------------------------------ set-up (host)

namespace lattice {

using b200::LatticeColour;
using b200::LatticeDesc;

// The node grid of a Q1 operator in lexicographic node order, read off row
// 0's sorted columns: {0, 1, mx, mx + 1} in 2-D, and {0, 1, mx, mx + 1,
// mx my, mx my + 1, mx my + mx, mx my + mx + 1} in 3-D.
bool grid(int n, const int *row, const int *col, int *mx, int *my, int *mz)
{
    if (n < 4 || !row || !col) return false;
    const int len = row[1] - row[0];
    const int *c = col + row[0];
    if (len != 4 && len != 8) return false;
    const int x = c[2];
    if (x < 2 || c[0] != 0 || c[1] != 1 || c[3] != x + 1) return false;
    if (len == 4) {
        if (n % x) return false;
        *mx = x;
        *my = n / x;
        *mz = 1;
        return *my >= 2;
    }
    const int xy = c[4];
    if (xy < 2 * x || xy % x || n % xy || c[5] != xy + 1 || c[6] != xy + x || c[7] != xy + x + 1) return false;
    *mx = x;
    *my = xy / x;
    *mz = n / xy;
    return *my >= 2 && *mz >= 2;
}

// The colouring is the parity colouring: ncol = 4 (2-D) or 8 (3-D) blocks,
// block c the nodes of parities (c & 1, c >> 1 & 1, c >> 2 & 1) in
// lexicographic order (perm[new] = old).
bool perm_ok(int mx, int my, int mz, const std::vector<int> &perm, const std::vector<int> &off)
{
    const int ncol = mz > 1 ? 8 : 4;
    if ((int)off.size() != ncol + 1) return false;
    size_t k = 0;
    for (int c = 0; c < ncol; ++c) {
        if ((size_t)off[c] != k) return false;
        const int px = c & 1, py = (c >> 1) & 1, pz = (c >> 2) & 1;
        for (int z = pz; z < mz; z += 2)
            for (int y = py; y < my; y += 2)
                for (int x = px; x < mx; x += 2) {
                    if (k >= perm.size() || perm[k] != (z * my + y) * mx + x) return false;
                    ++k;
                }
    }
    return k == perm.size() && (size_t)off[ncol] == k;
}

// Slots of colour c for a part, packed for the descriptor (the table the kernels use).
static std::vector<unsigned> slots(int c, int dim3, int part)
{
    const b200::SlotTab t = b200::lattice_slots(dim3 ? 3 : 2, c, part);
    std::vector<unsigned> out;
    for (int k = 0; k < t.n; ++k)
        out.push_back((unsigned)(t.dx[k] + 1) | (unsigned)(t.dy[k] + 1) << 2 | (unsigned)(t.dz[k] + 1) << 4 |
                      (unsigned)t.cp[k] << 8);
    return out;
}

// Descriptor and values of one part of M (rows and columns in the coloured
// numbering).  False when an entry of M is not a lattice neighbour of its row
// in the part, or when the row's entries are not in slot order.
bool values(int mx, int my, int mz, const b200::host::Csr &M, int part, LatticeDesc &d, std::vector<double> &out)
{
    const int dim3 = mz > 1, ncol = dim3 ? 8 : 4;
    if (M.n != mx * my * mz || M.m != M.n) return false;
    d = LatticeDesc{};
    d.ncol = ncol;
    d.mx = mx;
    d.my = my;
    d.mz = mz;
    int row0 = 0, chunk0 = 0;
    long long val0 = 0;
    for (int c = 0; c < ncol; ++c) {
        LatticeColour &L = d.col[c];
        L.px = c & 1;
        L.py = (c >> 1) & 1;
        L.pz = (c >> 2) & 1;
        L.nx = (mx - L.px + 1) / 2;
        L.ny = (my - L.py + 1) / 2;
        const int nz = dim3 ? (mz - L.pz + 1) / 2 : 1;
        L.rows = L.nx * L.ny * nz;
        L.row0 = row0;
        L.chunk0 = chunk0;
        L.val0 = val0;
        const std::vector<unsigned> sl = slots(c, dim3, part);
        L.nslot = (int)sl.size();
        std::copy(sl.begin(), sl.end(), L.slot);
        row0 += L.rows;
        const int nch = (L.rows + 31) / 32;
        chunk0 += nch;
        val0 += (long long)nch * L.nslot * 32;
    }
    d.chunks = chunk0;
    d.part = part;
    if (row0 != M.n) return false;
    out.assign((size_t)val0, 0.0);
    for (int c = 0; c < ncol; ++c) {
        const LatticeColour &L = d.col[c];
        for (int t = 0; t < L.rows; ++t) {
            const int q = t / L.nx, xs = t - q * L.nx, zs = q / L.ny, ys = q - zs * L.ny;
            const int X = 2 * xs + L.px, Y = 2 * ys + L.py, Z = 2 * zs + L.pz;
            const int r = L.row0 + t;
            int e = M.row[r];
            const int end = M.row[r + 1];
            double *dst = out.data() + L.val0 + (size_t)(t >> 5) * L.nslot * 32 + (t & 31);
            for (int k = 0; k < L.nslot && e < end; ++k) {
                const unsigned sl = L.slot[k];
                const int xn = X + (int)(sl & 3u) - 1, yn = Y + (int)((sl >> 2) & 3u) - 1,
                          zn = Z + (int)((sl >> 4) & 3u) - 1;
                if (xn < 0 || xn >= mx || yn < 0 || yn >= my || zn < 0 || zn >= mz) continue;
                const LatticeColour &P = d.col[sl >> 8];
                const int colk = P.row0 + ((zn >> 1) * P.ny + (yn >> 1)) * P.nx + (xn >> 1);
                if (M.col[e] == colk) {
                    dst[32 * k] = M.val[e];
                    ++e;
                }
            }
            if (e != end) return false;
        }
    }
    return true;
}

}  // namespace lattice

// Whether lattice layouts are built (B200LA_LATTICE=0: never).
static bool lattice_policy()
{
    const char *e = std::getenv("B200LA_LATTICE");
    return !e || std::atoi(e) != 0;
}

void lattice_free(b200la_csr *A)
{
    if (A->lt_val) cudaFree(A->lt_val);
    delete A->lt;
    A->lt_val = nullptr;
    A->lt = nullptr;
}

// Attach the lattice layout of part `part` of Mh (the host copy of A, in the
// coloured numbering of a mx x my x mz grid) to A.  Returns B200LA_OK also
// when the operator does not fit the layout (A keeps its CSR path only).
int lattice_attach(b200la_ctx *ctx, b200la_csr *A, const b200::host::Csr &Mh, int mx, int my, int mz, int part)
{
    if (!lattice_policy()) return B200LA_OK;
    b200::LatticeDesc d;
    std::vector<double> v;
    if (!lattice::values(mx, my, mz, Mh, part, d, v)) return B200LA_OK;
    const size_t es = A->dtype == B200LA_F64 ? 8 : 4;
    void *dv = nullptr;
    cudaError_t e = cudaMalloc(&dv, es * std::max<size_t>(v.size(), 1));
    if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_ALLOC, "lattice layout", e);
    if (A->dtype == B200LA_F64) {
        e = cudaMemcpy(dv, v.data(), 8 * v.size(), cudaMemcpyHostToDevice);
    } else {
        std::vector<float> f(v.begin(), v.end());
        e = cudaMemcpy(dv, f.data(), 4 * f.size(), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        cudaFree(dv);
        return ctx_fail(ctx, B200LA_ERR_CUDA, "lattice layout upload", e);
    }
    lattice_free(A);
    A->lt_val = dv;
    A->lt = new b200::LatticeDesc(d);
    A->lt->l2hint = A->l2hint;
    A->bytes += es * v.size();
    return B200LA_OK;
}

// The lattice launch for a row segment of A that is a run of whole colours;
// false when A has no lattice layout or the segment is not such a run.
bool lattice_segment(const b200la_csr *A, const b200::Seg &seg, int *c0, int *c1)
{
    if (!A->lt || !A->lt_val) return false;
    const b200::LatticeDesc &d = *A->lt;
    int a = -1, b = -1;
    for (int c = 0; c < d.ncol; ++c) {
        if (d.col[c].row0 == seg.r0 && a < 0) a = c;
        if (d.col[c].row0 + d.col[c].rows == seg.r1) b = c + 1;
    }
    if (a < 0 || b <= a) return false;
    *c0 = a;
    *c1 = b;
    return true;
}

// After the values of A changed (set_values, scale): rebuild its lattice
// layout from the CSR, or drop it if the values no longer fit.
int lattice_refresh(b200la_ctx *ctx, b200la_csr *A)
{
    if (!A->lt) return B200LA_OK;
    const b200::LatticeDesc d = *A->lt;
    b200::host::Csr M;
    M.n = A->n;
    M.m = A->m;
    M.row.resize(A->n + 1);
    M.col.resize(A->nnz);
    M.val.resize(A->nnz);
    cudaError_t e;
    if ((e = cudaMemcpy(M.row.data(), A->row, sizeof(int) * (A->n + 1), cudaMemcpyDeviceToHost)) ||
        (A->nnz && (e = cudaMemcpy(M.col.data(), A->col, sizeof(int) * A->nnz, cudaMemcpyDeviceToHost))))
        return ctx_fail(ctx, B200LA_ERR_CUDA, "lattice refresh", e);
    if (A->dtype == B200LA_F64) {
        if (A->nnz && (e = cudaMemcpy(M.val.data(), A->val, 8 * A->nnz, cudaMemcpyDeviceToHost)))
            return ctx_fail(ctx, B200LA_ERR_CUDA, "lattice refresh", e);
    } else {
        std::vector<float> f(A->nnz);
        if (A->nnz && (e = cudaMemcpy(f.data(), A->val, 4 * A->nnz, cudaMemcpyDeviceToHost)))
            return ctx_fail(ctx, B200LA_ERR_CUDA, "lattice refresh", e);
        std::copy(f.begin(), f.end(), M.val.begin());
    }
    lattice_free(A);
    return lattice_attach(ctx, A, M, d.mx, d.my, d.mz, d.part);
}
