// b200la_internal.h -- objects behind the opaque handles of include/b200la.h.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <string>
#include <vector>

// An NVTX range named after a C-ABI entry point, open for the call's scope:
// profilers group the call's kernels under it (ncu --nvtx, nsys).  Costs a
// function-pointer check when no tool is attached.
struct NvtxScope {
    explicit NvtxScope(const char *name) { nvtxRangePushA(name); }
    ~NvtxScope() { nvtxRangePop(); }
    NvtxScope(const NvtxScope &) = delete;
    NvtxScope &operator=(const NvtxScope &) = delete;
};

#include "common.cuh"
#include "host_setup.h"
#include "kernels.cuh"

struct GraphEntry {
    std::vector<const void *> key;
    cudaGraphExec_t exec = nullptr;
    int launches = 0;
};

struct b200la_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    double *partials = nullptr;     // grid-reduction partials [8][kMaxGrid]
    unsigned *ticket = nullptr;     // last-CTA tickets
    int *dev_err = nullptr;         // device error flag (bounded waits)
    b200::DevState *st = nullptr;   // device solver state
    b200::DevState *st_host = nullptr;   // pinned mirror
    double *dscal = nullptr;        // device scalars (256)
    double *hscal = nullptr;        // pinned host scalars (256)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;     // solver-internal timing
    cudaEvent_t tev0 = nullptr, tev1 = nullptr;   // b200la_timer_start / stop
    void *work = nullptr;           // solver workspace
    size_t work_bytes = 0;
    void *work_outer = nullptr;     // outer-loop workspace of the GMRES defect correction
    size_t work_outer_bytes = 0;
    long long launches = 0;         // kernels launched through this context
    std::vector<GraphEntry> graphs; // captured solver iteration batches
    std::string msg;
};

struct b200la_csr {
    int n = 0, m = 0, nnz = 0, dtype = 0, lg = 0, cfg = 0;
    int *row = nullptr, *col = nullptr;
    void *val = nullptr;
    b200::Tile *tiles = nullptr;
    int *long_rows = nullptr;
    int ntiles = 0, nlong = 0;
    b200::Seg all{};                  // whole-matrix schedule
    std::vector<b200::Seg> segs;      // segs[0] = all, then one per row segment
    std::vector<int> seg_off;         // row offsets of the segments (if any)
    std::vector<int> h_row;           // host copy of the row pointer
    size_t bytes = 0;
    // row-pattern dictionary (null when the matrix has too many patterns)
    uint16_t *pid = nullptr;
    int *pat_off = nullptr, *pat_delta = nullptr;
    int npat = 0, ndelta = 0;
    bool use_pat = false;             // SpMV runs on the dictionary
    // gather lines of the dictionary (null when there are too many)
    int *line_start = nullptr, *line_span = nullptr, *entry_line = nullptr, *entry_lo = nullptr;
    int nlines = 0, span_sum = 0;
    int stage_x = 0;                  // x staged per row tile (B200LA_STAGE_X=1 at creation)
    int l2hint = 0;                   // L2 priorities on SpMV loads (bits as in CsrView::l2hint; set at creation)
    // sliced (SELL-32) copy of the values for the dictionary SpMV
    int *sell_off = nullptr;
    void *sell_val = nullptr;
    size_t sell_len = 0;
    int sell_lmax = 0;                // longest chunk row length
    int sell_tma = 0;                 // bulk-copy tiles (B200LA_SELL_TMA at creation)
    // stencil layout (square operators whose row patterns all lie in one set
    // of 3 or 9 bands of three consecutive column offsets): see kernels.cuh
    std::vector<int> st_union;        // the union of the row patterns' offsets (host)
    void *st_val = nullptr;
    int st_nb = 0;                    // bands (0: no stencil layout)
    int st_use = 0;                   // SpMV of the whole operator runs on it
    // half stencil layout (stencil operators symmetric outside their identity
    // rows): diagonal and upper half, identity-row mask; see kernels.cuh
    void *sh_val = nullptr;
    unsigned *sh_mask = nullptr;
    int sh_use = 0;                   // SpMV runs on it instead of the full layout
    // lattice layout (multicoloured structured Q1 operators): see kernels.cuh
    void *lt_val = nullptr;
    b200::LatticeDesc *lt = nullptr;
    // FP32 Jacobi scaling (float)(1 / a_ii) of an FP64 operator, kept for the
    // defect correction's inner solves; dropped when the values change
    float *invd32 = nullptr;
};

struct b200la_precond {
    int kind = 0, n = 0, dtype = 0;
    void *invd = nullptr;             // Jacobi: 1/a_ii
    // block sweeps (colours / levels) in the permuted numbering
    int nblocks = 0;
    std::vector<int> block_off;
    std::vector<int> perm;            // perm[new] = old
    b200la_csr *L = nullptr;          // entries left of the row's block (no diagonal)
    b200la_csr *U = nullptr;          // entries right of the row's block (no diagonal)
    void *Dv = nullptr, *iDv = nullptr;
    int *perm_dev = nullptr;
    // level-scheduled sync-free sweeps
    int use_syncfree = 0;
    unsigned *flags = nullptr;        // per-row completion epochs
    unsigned *sync = nullptr;         // [epoch, fwd counter, bwd counter, done]
    void *syncfree_plan = nullptr;    // chunk lists of the two sweeps
};

// shared helpers (capi.cu)
int ctx_fail(const b200la_ctx *ctx, int code, const char *what, cudaError_t e);
b200::Scratch ctx_scratch(const b200la_ctx *ctx);
b200::CsrView csr_view(const b200la_csr *A);
int ctx_work(b200la_ctx *ctx, size_t bytes, void **out);
int ctx_work_outer(b200la_ctx *ctx, size_t bytes, void **out);
int ctx_check_device_error(b200la_ctx *ctx);
int spmv_run(b200la_ctx *ctx, const b200la_csr *A, const b200::Seg &seg, b200::SpmvOp op);
int csr_upload(b200la_ctx *ctx, int n_rows, int n_cols, int nnz, const int *row, const int *col, const void *val,
               int dtype, int n_seg, const int *seg_off, b200la_csr **out);
// precond.cu
int precond_apply_async(b200la_ctx *ctx, const b200la_precond *P, const void *r, void *z, const int *gate);
int syncfree_setup(b200la_ctx *ctx, b200la_precond *P);
int syncfree_apply(b200la_ctx *ctx, const b200la_precond *P, const void *r, void *z, const int *gate);
void syncfree_free(b200la_precond *P);
// solvers.cu
void graph_cache_clear(b200la_ctx *ctx);
// lattice.cu
namespace lattice {
bool grid(int n, const int *row, const int *col, int *mx, int *my, int *mz);
bool perm_ok(int mx, int my, int mz, const std::vector<int> &perm, const std::vector<int> &off);
bool values(int mx, int my, int mz, const b200::host::Csr &M, int part, b200::LatticeDesc &d,
            std::vector<double> &out);
}  // namespace lattice
int lattice_attach(b200la_ctx *ctx, b200la_csr *A, const b200::host::Csr &Mh, int mx, int my, int mz, int part);
bool lattice_segment(const b200la_csr *A, const b200::Seg &seg, int *c0, int *c1);
void lattice_free(b200la_csr *A);
int lattice_refresh(b200la_ctx *ctx, b200la_csr *A);

namespace b200 {
cudaError_t sweeps_configure();
cudaError_t launch_invdiag(int dtype, int n, const int *row, const int *col, const void *val, void *out,
                           cudaStream_t st);
cudaError_t launch_jacobi(int dtype, int n, const void *invd, const void *r, void *z, const int *gate,
                          cudaStream_t st);
// matops.cu
cudaError_t launch_csr_scale(int dtype, int n, const int *row, const int *col, void *val, double alpha, int mode,
                             cudaStream_t st);
cudaError_t launch_csr_diag(int dtype, int start, int end, const int *row, const int *col, const void *val,
                            int inverse, void *out, cudaStream_t st);
cudaError_t launch_csr_filter_count(int dtype, int r0, int r1, const int *row, const int *col, const void *val,
                                    int mode, int sc, int ec, int *cnt, cudaStream_t st);
cudaError_t launch_csr_filter_fill(int dtype, int r0, int r1, const int *row, const int *col, const void *val,
                                   int mode, int sc, int ec, const int *off, int *co, void *vo, cudaStream_t st);
}  // namespace b200
