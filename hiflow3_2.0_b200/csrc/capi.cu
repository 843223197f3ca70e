// capi.cu -- the C ABI of the B200 lmp platform (declared in include/b200la.h).
//
// Host orchestration only: argument checks, device memory, tile schedules,
// preconditioner setup and the device-resident solver loops.  Every
// arithmetic operation on vectors and matrices runs in a kernel of
// kernels.cu / sweeps.cu; there is no host fallback.
#include "b200la.h"
#include "b200la_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace b200;

// ------------------------------------------------------------------ helpers

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, #call, e_);         \
    } while (0)

int ctx_fail(const b200la_ctx *ctx, int code, const char *what, cudaError_t e)
{
    if (ctx) {
        char buf[512];
        std::snprintf(buf, sizeof buf, "%s: %s", what, e == cudaSuccess ? "" : cudaGetErrorString(e));
        const_cast<b200la_ctx *>(ctx)->msg = buf;
    }
    return code;
}

static int ctx_msg(const b200la_ctx *ctx, int code, const std::string &m)
{
    if (ctx) const_cast<b200la_ctx *>(ctx)->msg = m;
    return code;
}

static size_t dsize(int dtype) { return dtype == B200LA_F64 ? 8 : 4; }

Scratch ctx_scratch(const b200la_ctx *ctx)
{
    Scratch s;
    s.partials = ctx->partials;
    s.ticket = ctx->ticket;
    s.err = ctx->dev_err;
    s.num_sms = ctx->num_sms;
    return s;
}

// Whether SpMV on a matrix of this dtype runs on its row-pattern dictionary
// (when the matrix has one).  B200LA_PATTERN = 0: never, 1: FP32 only
// (default; FP64 operators keep explicit 32-bit column indices), 2: always.
static bool pattern_policy(int dtype)
{
    const char *e = std::getenv("B200LA_PATTERN");
    const int mode = e ? std::atoi(e) : 1;
    return mode == 2 || (mode == 1 && dtype == B200LA_F32);
}

// Whether SpMV of the whole operator runs on the stencil layout (when the
// matrix has one).  B200LA_STENCIL = 0: never, 1: FP32 only, 2: always (default).
static bool stencil_policy(int dtype)
{
    const char *e = std::getenv("B200LA_STENCIL");
    const int mode = e ? std::atoi(e) : 2;
    return mode == 2 || (mode == 1 && dtype == B200LA_F32);
}

// The cached FP32 Jacobi scaling no longer matches changed values.
static void drop_invd32(b200la_csr *A)
{
    if (A->invd32) cudaFree(A->invd32);
    A->invd32 = nullptr;
}

CsrView csr_view(const b200la_csr *A)
{
    CsrView v;
    v.row = A->row;
    v.col = A->col;
    v.val = A->val;
    v.tiles = A->tiles;
    v.long_rows = A->long_rows;
    v.lg = A->lg;
    v.dtype = A->dtype;
    v.cfg = A->cfg;
    v.pid = A->pid;
    v.pat_off = A->pat_off;
    v.pat_delta = A->pat_delta;
    v.npat = A->npat;
    v.ndelta = A->ndelta;
    v.use_pat = A->pid != nullptr && A->use_pat;
    v.line_start = A->line_start;
    v.line_span = A->line_span;
    v.entry_line = A->entry_line;
    v.entry_lo = A->entry_lo;
    v.nlines = A->nlines;
    v.span_sum = A->span_sum;
    v.stage_x = A->stage_x;
    v.l2hint = A->l2hint;
    v.sell_off = A->sell_off;
    v.sell_val = A->sell_val;
    v.sell_lmax = A->sell_lmax;
    v.sell_tma = A->sell_tma;
    v.n_cols = A->m;
    v.n_rows = A->n;
    v.st_val = A->st_val;
    v.st_nb = A->st_nb;
    v.st_use = A->st_use && (A->st_val != nullptr || (A->sh_use && A->sh_val != nullptr));
    for (int b = 0; b < kMaxBands; ++b) v.st_center[b] = b < A->st_nb ? A->st_union[3 * b + 1] : 0;
    v.sh_val = A->sh_val;
    v.sh_mask = A->sh_mask;
    v.sh_use = A->sh_use && A->sh_val != nullptr;
    return v;
}

int ctx_work(b200la_ctx *ctx, size_t bytes, void **out)
{
    if (bytes > ctx->work_bytes) {
        if (ctx->work) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(ctx->work);
            ctx->work = nullptr;
            ctx->work_bytes = 0;
        }
        cudaError_t e = cudaMalloc(&ctx->work, bytes);
        if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_ALLOC, "workspace", e);
        ctx->work_bytes = bytes;
    }
    *out = ctx->work;
    return B200LA_OK;
}

// A second workspace for loops that call a solver which itself uses ctx_work.
int ctx_work_outer(b200la_ctx *ctx, size_t bytes, void **out)
{
    if (bytes > ctx->work_outer_bytes) {
        if (ctx->work_outer) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(ctx->work_outer);
            ctx->work_outer = nullptr;
            ctx->work_outer_bytes = 0;
        }
        cudaError_t e = cudaMalloc(&ctx->work_outer, bytes);
        if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_ALLOC, "outer workspace", e);
        ctx->work_outer_bytes = bytes;
    }
    *out = ctx->work_outer;
    return B200LA_OK;
}

int ctx_check_device_error(b200la_ctx *ctx)
{
    int h = 0;
    CK(cudaMemcpyAsync(&h, ctx->dev_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (h != kDevOk) {
        cudaMemsetAsync(ctx->dev_err, 0, sizeof(int), ctx->stream);
        return ctx_msg(ctx, B200LA_ERR_TIMEOUT, "a bounded device wait gave up (error flag " + std::to_string(h) + ")");
    }
    return B200LA_OK;
}

// ------------------------------------------------------------------ context

extern "C" int b200la_create(int device, b200la_ctx **out)
{
    if (!out) return B200LA_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return B200LA_ERR_DEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return B200LA_ERR_DEVICE;
    if (prop.major != 10) return B200LA_ERR_DEVICE;   // sm_100 family only
    if (cudaSetDevice(device) != cudaSuccess) return B200LA_ERR_DEVICE;
    b200la_ctx *ctx = new b200la_ctx();
    ctx->device = device;
    ctx->num_sms = prop.multiProcessorCount;
    if (ctx->num_sms * kCtasPerSm > kMaxGrid || ctx->num_sms * 8 > kMaxGrid) ctx->num_sms = kMaxGrid / 8;
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking)) ||
        (e = cudaMalloc(&ctx->partials, sizeof(double) * 8 * kMaxGrid)) ||
        (e = cudaMalloc(&ctx->ticket, sizeof(unsigned) * kTicketWords)) || (e = cudaMalloc(&ctx->dev_err, sizeof(int))) ||
        (e = cudaMalloc(&ctx->st, sizeof(DevState))) || (e = cudaMalloc(&ctx->dscal, sizeof(double) * 256)) ||
        (e = cudaMallocHost(&ctx->st_host, sizeof(DevState))) ||
        (e = cudaMallocHost(&ctx->hscal, sizeof(double) * 256)) || (e = cudaEventCreate(&ctx->ev0)) ||
        (e = cudaEventCreate(&ctx->ev1)) || (e = cudaMemset(ctx->ticket, 0, sizeof(unsigned) * kTicketWords)) ||
        (e = cudaMemset(ctx->dev_err, 0, sizeof(int))) || (e = spmv_configure()) || (e = sweeps_configure())) {
        ctx->stream = ctx->own_stream;
        b200la_destroy(ctx);
        return e == cudaErrorMemoryAllocation ? B200LA_ERR_ALLOC : B200LA_ERR_CUDA;
    }
    ctx->stream = ctx->own_stream;
    *out = ctx;
    return B200LA_OK;
}

extern "C" int b200la_destroy(b200la_ctx *ctx)
{
    if (!ctx) return B200LA_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    graph_cache_clear(ctx);
    if (ctx->work) cudaFree(ctx->work);
    if (ctx->work_outer) cudaFree(ctx->work_outer);
    if (ctx->partials) cudaFree(ctx->partials);
    if (ctx->ticket) cudaFree(ctx->ticket);
    if (ctx->dev_err) cudaFree(ctx->dev_err);
    if (ctx->st) cudaFree(ctx->st);
    if (ctx->dscal) cudaFree(ctx->dscal);
    if (ctx->st_host) cudaFreeHost(ctx->st_host);
    if (ctx->hscal) cudaFreeHost(ctx->hscal);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->tev0) cudaEventDestroy(ctx->tev0);
    if (ctx->tev1) cudaEventDestroy(ctx->tev1);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return B200LA_OK;
}

extern "C" int b200la_set_stream(b200la_ctx *ctx, void *s)
{
    if (!ctx) return B200LA_ERR_ARG;
    cudaStreamSynchronize(ctx->stream);
    graph_cache_clear(ctx);
    ctx->stream = s ? static_cast<cudaStream_t>(s) : ctx->own_stream;
    return B200LA_OK;
}

extern "C" void *b200la_get_stream(b200la_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

extern "C" int b200la_sync(b200la_ctx *ctx)
{
    if (!ctx) return B200LA_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    return ctx_check_device_error(ctx);
}

extern "C" const char *b200la_last_error(const b200la_ctx *ctx) { return ctx ? ctx->msg.c_str() : "no context"; }

extern "C" const char *b200la_status_string(int s)
{
    switch (s) {
    case B200LA_OK: return "ok";
    case B200LA_ERR_ARG: return "invalid argument";
    case B200LA_ERR_CUDA: return "CUDA error";
    case B200LA_ERR_ALLOC: return "allocation failed";
    case B200LA_ERR_DEVICE: return "no usable sm_100 device";
    case B200LA_ERR_CSR: return "malformed CSR";
    case B200LA_ERR_BUDGET: return "refused by memory budget";
    case B200LA_ERR_TIMEOUT: return "bounded device wait gave up";
    case B200LA_ERR_SETUP: return "preconditioner setup failed";
    case B200LA_ERR_NOTFOUND: return "unknown request";
    case B200LA_PENDING: return "request pending";
    case B200LA_ERR_IO: return "file I/O failed";
    case B200LA_ERR_FORMAT: return "unsupported or malformed file";
    case B200LA_ERR_COMM: return "communicator failed";
    default: return "unknown status";
    }
}

extern "C" int b200la_num_sms(const b200la_ctx *ctx) { return ctx ? ctx->num_sms : 0; }

// ------------------------------------------------------------------ memory

extern "C" int b200la_malloc(b200la_ctx *ctx, size_t bytes, void **dptr)
{
    if (!ctx || !dptr) return B200LA_ERR_ARG;
    cudaError_t e = cudaMalloc(dptr, bytes ? bytes : 16);
    if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_ALLOC, "cudaMalloc", e);
    return B200LA_OK;
}

extern "C" int b200la_free(b200la_ctx *ctx, void *dptr)
{
    if (!ctx) return B200LA_ERR_ARG;
    if (!dptr) return B200LA_OK;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaFree(dptr));
    return B200LA_OK;
}

extern "C" int b200la_memcpy_h2d(b200la_ctx *ctx, void *dst, const void *src, size_t bytes)
{
    if (!ctx || (bytes && (!dst || !src))) return B200LA_ERR_ARG;
    if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return B200LA_OK;
}

extern "C" int b200la_memcpy_d2h(b200la_ctx *ctx, void *dst, const void *src, size_t bytes)
{
    if (!ctx || (bytes && (!dst || !src))) return B200LA_ERR_ARG;
    if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return B200LA_OK;
}

extern "C" int b200la_memcpy_d2d(b200la_ctx *ctx, void *dst, const void *src, size_t bytes)
{
    if (!ctx || (bytes && (!dst || !src))) return B200LA_ERR_ARG;
    if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    return B200LA_OK;
}

extern "C" int b200la_memset_zero(b200la_ctx *ctx, void *dptr, size_t bytes)
{
    if (!ctx || (bytes && !dptr)) return B200LA_ERR_ARG;
    if (bytes) CK(cudaMemsetAsync(dptr, 0, bytes, ctx->stream));
    return B200LA_OK;
}

extern "C" int b200la_host_alloc(b200la_ctx *ctx, size_t bytes, void **hptr)
{
    if (!ctx || !hptr) return B200LA_ERR_ARG;
    cudaError_t e = cudaMallocHost(hptr, bytes ? bytes : 16);
    if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_ALLOC, "cudaMallocHost", e);
    return B200LA_OK;
}

extern "C" int b200la_host_free(b200la_ctx *ctx, void *hptr)
{
    if (!ctx) return B200LA_ERR_ARG;
    if (!hptr) return B200LA_OK;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaFreeHost(hptr));
    return B200LA_OK;
}

extern "C" int b200la_timer_start(b200la_ctx *ctx)
{
    if (!ctx) return B200LA_ERR_ARG;
    if (!ctx->tev0) {
        CK(cudaEventCreate(&ctx->tev0));
        CK(cudaEventCreate(&ctx->tev1));
    }
    CK(cudaEventRecord(ctx->tev0, ctx->stream));
    return B200LA_OK;
}

extern "C" int b200la_timer_stop(b200la_ctx *ctx, double *ms)
{
    if (!ctx || !ms || !ctx->tev0) return B200LA_ERR_ARG;
    CK(cudaEventRecord(ctx->tev1, ctx->stream));
    CK(cudaEventSynchronize(ctx->tev1));
    float f = 0.f;
    CK(cudaEventElapsedTime(&f, ctx->tev0, ctx->tev1));
    *ms = f;
    return B200LA_OK;
}

// ------------------------------------------------------------------ matrix

static int lanes_log2(int n, long long nnz)
{
    if (const char *e = std::getenv("B200LA_LANES")) {
        const int l = std::atoi(e);
        for (int lg = 0; lg <= 5; ++lg)
            if ((1 << lg) == l) return lg;
    }
    const double mean = n > 0 ? (double)nnz / n : 0.0;
    int lg = 0;
    while (lg < 5 && (double)(8 << lg) < mean) ++lg;
    return lg;
}

// SpMV variant for new matrices: B200LA_SPMV = wide | small | direct.
static int spmv_cfg_choice()
{
    if (const char *e = std::getenv("B200LA_SPMV")) {
        if (!std::strcmp(e, "small")) return kSpmvTileSmall;
        if (!std::strcmp(e, "direct")) return kSpmvDirect;
        if (!std::strcmp(e, "wide")) return kSpmvTileWide;
    }
    // measured on B200 (128^3 Q1, 27 nonzeros per row): the direct variant
    // reaches 72% of HBM peak in FP64, the staged tiles 67%
    return kSpmvDirect;
}

// Tile schedule of rows [s0, s1): runs of whole rows of at most kBlock >> lg
// rows and `cap` nonzeros; longer rows go to the warp-per-row list.
static void build_segment(const int *row, int s0, int s1, int lg, int cap, std::vector<Tile> &tiles,
                          std::vector<int> &longs, std::vector<Seg> &segs)
{
    const int kTileCap = cap;
    Seg sg;
    sg.r0 = s0;
    sg.r1 = s1;
    sg.t0 = (int)tiles.size();
    sg.l0 = (int)longs.size();
    const int rows_max = kBlock >> lg;
    int r = s0;
    while (r < s1) {
        if (row[r + 1] - row[r] > kTileCap) {
            longs.push_back(r++);
            continue;
        }
        const int r0 = r;
        while (r < s1 && r - r0 < rows_max && row[r + 1] - row[r] <= kTileCap && row[r + 1] - row[r0] <= kTileCap)
            ++r;
        Tile t;
        t.r0 = r0;
        t.r1 = r;
        t.a0 = row[r0] & ~3;
        t.a1 = (row[r] + 3) & ~3;
        tiles.push_back(t);
    }
    sg.t1 = (int)tiles.size();
    sg.l1 = (int)longs.size();
    segs.push_back(sg);
}

// (Re)build the sliced copy of A's values from A->val (device); needs the
// dictionary.  Chunk c holds 32 * (longest row of the chunk) values.
static int build_sell(b200la_ctx *ctx, b200la_csr *A)
{
    if (!A->pid || !A->use_pat || A->n == 0) return B200LA_OK;
    // its whole-operator products run on the stencil layout: no sliced copy
    if (A->st_use && A->st_nb && A->seg_off.empty()) return B200LA_OK;
    const size_t es = dsize(A->dtype);
    cudaError_t e;
    if (!A->sell_off) {
        const int nch = (A->n + 31) / 32;
        std::vector<int> off(nch + 1, 0);
        A->sell_lmax = 0;
        for (int c = 0; c < nch; ++c) {
            int L = 0;
            for (int r = 32 * c; r < std::min(A->n, 32 * c + 32); ++r) L = std::max(L, A->h_row[r + 1] - A->h_row[r]);
            off[c + 1] = off[c] + 32 * L;
            A->sell_lmax = std::max(A->sell_lmax, L);
        }
        if (const char *e = std::getenv("B200LA_SELL_TMA")) A->sell_tma = std::atoi(e);
        A->sell_len = (size_t)off[nch];
        if ((e = cudaMalloc(&A->sell_off, sizeof(int) * (nch + 1))) ||
            (e = cudaMalloc(&A->sell_val, es * std::max<size_t>(A->sell_len, 32))) ||
            (e = cudaMemcpy(A->sell_off, off.data(), sizeof(int) * (nch + 1), cudaMemcpyHostToDevice)))
            return ctx_fail(ctx, B200LA_ERR_ALLOC, "sliced layout", e);
        A->bytes += sizeof(int) * (nch + 1) + es * A->sell_len;
    }
    if ((e = cudaMemsetAsync(A->sell_val, 0, es * std::max<size_t>(A->sell_len, 32), ctx->stream)) ||
        (e = launch_csr_to_sell(A->dtype, A->n, A->row, A->val, A->sell_off, A->sell_val, ctx->stream)) ||
        (e = cudaStreamSynchronize(ctx->stream)))
        return ctx_fail(ctx, B200LA_ERR_CUDA, "sliced layout", e);
    return B200LA_OK;
}

// The stencil layout of a square operator whose row patterns' offsets (their
// union `uni`, ascending) form 3 or 9 bands of three consecutive offsets, with
// at most 30 % zero padding.  Values are (re)scattered from the CSR.
static void stencil_plan(b200la_csr *A, const std::vector<int> &uni)
{
    A->st_nb = 0;
    A->st_union.clear();
    const int L = (int)uni.size();
    if (A->n != A->m || A->n == 0 || (L != 9 && L != 27)) return;
    for (int b = 0; b < L / 3; ++b)
        if (uni[3 * b + 1] != uni[3 * b] + 1 || uni[3 * b + 2] != uni[3 * b] + 2) return;
    const double padded = (double)((A->n + 31) / 32) * 32 * L;
    if (padded > 1.30 * (double)A->nnz) return;
    A->st_union = uni;
    A->st_nb = L / 3;
}

// Whether the half stencil layout is built for a symmetric stencil operator
// of this precision.  B200LA_HALF_STENCIL = 0: never; 1 (default): FP64
// only; 2: both precisions.  The half layout halves the HBM bytes of the
// values but not the on-chip ones (each value is read twice from L2): the
// FP64 product, bound by HBM, gains (128^3: 80.5 -> 73.4 us), the FP32 one,
// already bound by on-chip latency, loses (45.5 -> 55.5 us).
static bool half_policy(int dtype)
{
    const char *e = std::getenv("B200LA_HALF_STENCIL");
    const int mode = e ? std::atoi(e) : 1;
    return mode == 2 || (mode == 1 && dtype == B200LA_F64);
}

static void free_half(b200la_csr *A)
{
    if (A->sh_val) cudaFree(A->sh_val);
    if (A->sh_mask) cudaFree(A->sh_mask);
    A->sh_val = nullptr;
    A->sh_mask = nullptr;
    A->sh_use = 0;
}

// The half stencil layout from the full one: built when the band centres are
// symmetric about a centre band at offset 0 and the values are symmetric
// bit for bit between rows that are not identity rows; dropped otherwise.
static int build_half(b200la_ctx *ctx, b200la_csr *A)
{
    const int nb = A->st_nb;
    bool ok = half_policy(A->dtype) && A->st_val && (nb == 3 || nb == 9);
    for (int b = 0; ok && b < nb; ++b)
        if (A->st_union[3 * b + 1] != -A->st_union[3 * (nb - 1 - b) + 1]) ok = false;
    if (!ok) {
        free_half(A);
        return B200LA_OK;
    }
    const size_t es = dsize(A->dtype), len = half_len(A->n, nb, A->dtype), nch = (A->n + 31) / 32;
    cudaError_t e;
    if (!A->sh_val) {
        // one word past the mask receives the symmetry check's result
        if ((e = cudaMalloc(&A->sh_val, es * len)) || (e = cudaMalloc(&A->sh_mask, sizeof(unsigned) * (nch + 1)))) {
            free_half(A);
            return ctx_fail(ctx, B200LA_ERR_ALLOC, "half stencil layout", e);
        }
    }
    int centers[kMaxBands];
    for (int b = 0; b < nb; ++b) centers[b] = A->st_union[3 * b + 1];
    int *asym = reinterpret_cast<int *>(A->sh_mask + nch);
    int h_asym = 0;
    if ((e = cudaMemsetAsync(asym, 0, sizeof(int), ctx->stream)) ||
        (e = launch_stencil_to_half(A->dtype, A->n, nb, centers, A->st_val, A->sh_val, A->sh_mask, asym,
                                    ctx->stream)) ||
        (e = cudaMemcpyAsync(&h_asym, asym, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream)) ||
        (e = cudaStreamSynchronize(ctx->stream))) {
        free_half(A);
        return ctx_fail(ctx, B200LA_ERR_CUDA, "half stencil layout", e);
    }
    if (h_asym) {
        free_half(A);
        return B200LA_OK;
    }
    A->sh_use = 1;
    // the half layout now carries the operator's products: the full layout's
    // values are dropped (rebuilt from the CSR when the values change)
    if (A->st_use && A->st_val) {
        cudaFree(A->st_val);
        A->st_val = nullptr;
        A->bytes -= es * stencil_len(A->n, nb, A->dtype);
    }
    return B200LA_OK;
}

static int build_stencil(b200la_ctx *ctx, b200la_csr *A)
{
    if (!A->st_nb) {
        free_half(A);
        return B200LA_OK;
    }
    const size_t es = dsize(A->dtype), len = stencil_len(A->n, A->st_nb, A->dtype);
    cudaError_t e;
    if (!A->st_val) {
        if ((e = cudaMalloc(&A->st_val, es * len))) return ctx_fail(ctx, B200LA_ERR_ALLOC, "stencil layout", e);
        A->bytes += es * len;
    }
    if ((e = cudaMemsetAsync(A->st_val, 0, es * len, ctx->stream)) ||
        (e = launch_csr_to_stencil(A->dtype, A->n, A->row, A->col, A->val, A->st_union.data(), A->st_nb, A->st_val,
                                   ctx->stream)) ||
        (e = cudaStreamSynchronize(ctx->stream)))
        return ctx_fail(ctx, B200LA_ERR_CUDA, "stencil layout", e);
    return build_half(ctx, A);
}

static int upload_lines(b200la_ctx *ctx, b200la_csr *A, const std::vector<int> &ls, const std::vector<int> &lsp,
                        const std::vector<int> &el, const std::vector<int> &elo)
{
    cudaError_t e;
    const size_t L = ls.size(), E = std::max<size_t>(el.size(), 1);
    if ((e = cudaMalloc(&A->line_start, sizeof(int) * L)) || (e = cudaMalloc(&A->line_span, sizeof(int) * L)) ||
        (e = cudaMalloc(&A->entry_line, sizeof(int) * E)) || (e = cudaMalloc(&A->entry_lo, sizeof(int) * E)) ||
        (e = cudaMemcpy(A->line_start, ls.data(), sizeof(int) * L, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(A->line_span, lsp.data(), sizeof(int) * L, cudaMemcpyHostToDevice)) ||
        (!el.empty() && (e = cudaMemcpy(A->entry_line, el.data(), sizeof(int) * el.size(), cudaMemcpyHostToDevice))) ||
        (!el.empty() && (e = cudaMemcpy(A->entry_lo, elo.data(), sizeof(int) * el.size(), cudaMemcpyHostToDevice))))
        return ctx_fail(ctx, B200LA_ERR_ALLOC, "csr_create: gather lines", e);
    A->nlines = (int)L;
    A->span_sum = 0;
    for (int s : lsp) A->span_sum += s;
    return B200LA_OK;
}

static int copy_lines(b200la_ctx *ctx, const b200la_csr *A, b200la_csr *B)
{
    B->line_start = B->line_span = B->entry_line = B->entry_lo = nullptr;
    if (!A->line_start) return B200LA_OK;
    cudaError_t e;
    const size_t L = A->nlines, E = std::max(A->ndelta, 1);
    if ((e = cudaMalloc(&B->line_start, sizeof(int) * L)) || (e = cudaMalloc(&B->line_span, sizeof(int) * L)) ||
        (e = cudaMalloc(&B->entry_line, sizeof(int) * E)) || (e = cudaMalloc(&B->entry_lo, sizeof(int) * E)) ||
        (e = cudaMemcpy(B->line_start, A->line_start, sizeof(int) * L, cudaMemcpyDeviceToDevice)) ||
        (e = cudaMemcpy(B->line_span, A->line_span, sizeof(int) * L, cudaMemcpyDeviceToDevice)) ||
        (e = cudaMemcpy(B->entry_line, A->entry_line, sizeof(int) * E, cudaMemcpyDeviceToDevice)) ||
        (e = cudaMemcpy(B->entry_lo, A->entry_lo, sizeof(int) * E, cudaMemcpyDeviceToDevice)))
        return ctx_fail(ctx, B200LA_ERR_ALLOC, "csr_cast: gather lines", e);
    return B200LA_OK;
}

int csr_upload(b200la_ctx *ctx, int n_rows, int n_cols, int nnz, const int *row, const int *col,
               const void *val, int dtype, int n_seg, const int *seg_off, b200la_csr **out)
{
    if (!ctx || !out || !row || (nnz && (!col || !val)) || n_rows < 0 || n_cols < 0 || nnz < 0 ||
        (dtype != B200LA_F64 && dtype != B200LA_F32))
        return ctx_msg(ctx, B200LA_ERR_ARG, "csr_create: invalid argument");
    long long bad = -1;
    const int v = host::validate_csr(n_rows, n_cols, nnz, row, col, &bad);
    if (v) return ctx_msg(ctx, B200LA_ERR_CSR, "csr_create: malformed CSR (code " + std::to_string(v) + " at " +
                                                   std::to_string(bad) + ")");
    if (n_seg > 0) {
        if (!seg_off || seg_off[0] != 0 || seg_off[n_seg] != n_rows)
            return ctx_msg(ctx, B200LA_ERR_ARG, "csr_create: bad segment offsets");
        for (int s = 0; s < n_seg; ++s)
            if (seg_off[s + 1] < seg_off[s]) return ctx_msg(ctx, B200LA_ERR_ARG, "csr_create: bad segment offsets");
    }
    b200la_csr *A = new b200la_csr();
    A->n = n_rows;
    A->m = n_cols;
    A->nnz = nnz;
    A->dtype = dtype;
    A->lg = lanes_log2(n_rows, nnz);
    A->cfg = spmv_cfg_choice();
    // L2 priorities of the SpMV loads (B200LA_L2HINT overrides): bit 0 CSR-family
    // value / index streams evict-first, bit 1 their x gathers evict-last, bit 2
    // the stencil and lattice value streams evict-first, bit 3 the half
    // layout's own rows evict-first, bit 4 the half layout's chunk lines
    // prefetched into L2 before its band groups load them.  Default bits 2
    // and 4: a structured layout's stream then leaves x and the solver's
    // vectors resident in L2 (128^3: FP32 stencil SpMV 45.2 -> 41.2 us, mixed
    // solve 34.8 -> 29.7 ms, MC-SGS apply 138 -> 124 us), and the half
    // layout's three band groups wait on L2, not DRAM, after the first (FP64
    // SpMV 59.6 -> 58.9 us).  The CSR kernels lose with bits 0 and 1 (FP64
    // CSR CG 71 -> 103 and 88 ms); the half layout gains nothing from bit 3.
    A->l2hint = 4 | 16;
    if (const char *h = std::getenv("B200LA_L2HINT")) A->l2hint = std::atoi(h);
    const int cap = spmv_tile_cap(A->cfg);
    A->h_row.assign(row, row + n_rows + 1);
    std::vector<Tile> tiles;
    std::vector<int> longs;
    build_segment(row, 0, n_rows, A->lg, cap, tiles, longs, A->segs);   // segs[0] = whole matrix
    A->all = A->segs[0];
    if (n_seg > 0) {
        // per-segment schedules follow the whole-matrix schedule
        for (int s = 0; s < n_seg; ++s) build_segment(row, seg_off[s], seg_off[s + 1], A->lg, cap, tiles, longs, A->segs);
        A->seg_off.assign(seg_off, seg_off + n_seg + 1);
    }
    A->ntiles = (int)tiles.size();
    A->nlong = (int)longs.size();
    const size_t pad = 8;
    const size_t es = dsize(dtype);
    cudaError_t e;
    size_t bytes = sizeof(int) * (n_rows + 1) + (sizeof(int) + es) * (nnz + pad) + sizeof(Tile) * tiles.size() +
                   sizeof(int) * (longs.size() + 1);
    // row pointers, columns and values are padded by 8 entries: the bulk
    // copies move whole 16-byte units past the last row / nonzero
    if ((e = cudaMalloc(&A->row, sizeof(int) * (n_rows + 1 + pad))) ||
        (e = cudaMalloc(&A->col, sizeof(int) * (nnz + pad))) ||
        (e = cudaMalloc(&A->val, es * (nnz + pad))) ||
        (e = cudaMalloc(&A->tiles, sizeof(Tile) * std::max<size_t>(tiles.size(), 1))) ||
        (e = cudaMalloc(&A->long_rows, sizeof(int) * std::max<size_t>(longs.size(), 1)))) {
        b200la_csr_destroy(A);
        return ctx_fail(ctx, B200LA_ERR_ALLOC, "csr_create: device allocation", e);
    }
    A->bytes = bytes;
    cudaStream_t s = ctx->stream;
    if ((e = cudaMemsetAsync(A->row + n_rows + 1, 0, sizeof(int) * pad, s)) ||
        (e = cudaMemcpyAsync(A->row, row, sizeof(int) * (n_rows + 1), cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemsetAsync(A->col + nnz, 0, sizeof(int) * pad, s)) ||
        (e = cudaMemsetAsync(static_cast<char *>(A->val) + es * nnz, 0, es * pad, s)) ||
        (nnz && (e = cudaMemcpyAsync(A->col, col, sizeof(int) * nnz, cudaMemcpyHostToDevice, s))) ||
        (nnz && (e = cudaMemcpyAsync(A->val, val, es * nnz, cudaMemcpyHostToDevice, s))) ||
        (!tiles.empty() && (e = cudaMemcpyAsync(A->tiles, tiles.data(), sizeof(Tile) * tiles.size(),
                                                cudaMemcpyHostToDevice, s))) ||
        (!longs.empty() &&
         (e = cudaMemcpyAsync(A->long_rows, longs.data(), sizeof(int) * longs.size(), cudaMemcpyHostToDevice, s))) ||
        (e = cudaStreamSynchronize(s))) {
        b200la_csr_destroy(A);
        return ctx_fail(ctx, B200LA_ERR_CUDA, "csr_create: upload", e);
    }
    // row-pattern dictionary (kept beside the explicit indices) when the
    // matrix has few distinct row patterns, as stencil operators do
    std::vector<uint16_t> pid;
    std::vector<int> poff, pdel;
    if (n_rows > 0 && host::row_patterns(n_rows, row, col, kMaxPatterns, kMaxPatternDeltas, pid, poff, pdel)) {
        A->npat = (int)poff.size() - 1;
        A->ndelta = (int)pdel.size();
        if ((e = cudaMalloc(&A->pid, sizeof(uint16_t) * n_rows)) ||
            (e = cudaMalloc(&A->pat_off, sizeof(int) * poff.size())) ||
            (e = cudaMalloc(&A->pat_delta, sizeof(int) * std::max<size_t>(pdel.size(), 1))) ||
            (e = cudaMemcpy(A->pid, pid.data(), sizeof(uint16_t) * n_rows, cudaMemcpyHostToDevice)) ||
            (e = cudaMemcpy(A->pat_off, poff.data(), sizeof(int) * poff.size(), cudaMemcpyHostToDevice)) ||
            (!pdel.empty() &&
             (e = cudaMemcpy(A->pat_delta, pdel.data(), sizeof(int) * pdel.size(), cudaMemcpyHostToDevice)))) {
            b200la_csr_destroy(A);
            return ctx_fail(ctx, B200LA_ERR_ALLOC, "csr_create: pattern dictionary", e);
        }
        A->bytes += sizeof(uint16_t) * n_rows + sizeof(int) * (poff.size() + pdel.size());
        A->use_pat = pattern_policy(dtype);
        if (const char *sx = std::getenv("B200LA_STAGE_X")) A->stage_x = std::atoi(sx);
        std::vector<int> ls, lsp, el, elo;
        host::pattern_lines(pdel, ls, lsp, el, elo);
        if (!ls.empty() && (int)ls.size() <= kMaxGatherLines) {
            int rc = upload_lines(ctx, A, ls, lsp, el, elo);
            if (rc) {
                b200la_csr_destroy(A);
                return rc;
            }
        }
        if (n_seg == 0) {
            std::vector<int> uni(pdel);
            std::sort(uni.begin(), uni.end());
            uni.erase(std::unique(uni.begin(), uni.end()), uni.end());
            stencil_plan(A, uni);
            A->st_use = stencil_policy(dtype);
        }
        int rc = build_sell(ctx, A);
        if (!rc && n_seg == 0) rc = build_stencil(ctx, A);
        if (rc) {
            b200la_csr_destroy(A);
            return rc;
        }
    }
    *out = A;
    return B200LA_OK;
}

extern "C" int b200la_csr_create(b200la_ctx *ctx, int n_rows, int n_cols, int nnz, const int *row, const int *col,
                                 const void *val, int dtype, b200la_csr **out)
{
    return csr_upload(ctx, n_rows, n_cols, nnz, row, col, val, dtype, 0, nullptr, out);
}

extern "C" int b200la_csr_create_segmented(b200la_ctx *ctx, int n_rows, int n_cols, int nnz, const int *row,
                                           const int *col, const void *val, int dtype, int n_seg, const int *seg_off,
                                           b200la_csr **out)
{
    if (n_seg < 1) return ctx_msg(ctx, B200LA_ERR_ARG, "csr_create_segmented: n_seg < 1");
    return csr_upload(ctx, n_rows, n_cols, nnz, row, col, val, dtype, n_seg, seg_off, out);
}

extern "C" int b200la_csr_destroy(b200la_csr *A)
{
    if (!A) return B200LA_OK;
    cudaDeviceSynchronize();
    if (A->row) cudaFree(A->row);
    if (A->col) cudaFree(A->col);
    if (A->val) cudaFree(A->val);
    if (A->tiles) cudaFree(A->tiles);
    if (A->long_rows) cudaFree(A->long_rows);
    if (A->pid) cudaFree(A->pid);
    if (A->pat_off) cudaFree(A->pat_off);
    if (A->pat_delta) cudaFree(A->pat_delta);
    if (A->line_start) cudaFree(A->line_start);
    if (A->line_span) cudaFree(A->line_span);
    if (A->entry_line) cudaFree(A->entry_line);
    if (A->entry_lo) cudaFree(A->entry_lo);
    if (A->sell_off) cudaFree(A->sell_off);
    if (A->sell_val) cudaFree(A->sell_val);
    if (A->st_val) cudaFree(A->st_val);
    free_half(A);
    lattice_free(A);
    if (A->invd32) cudaFree(A->invd32);
    delete A;
    return B200LA_OK;
}

extern "C" int b200la_csr_cast(b200la_ctx *ctx, const b200la_csr *A, int dtype, b200la_csr **out)
{
    if (!ctx || !A || !out || (dtype != B200LA_F64 && dtype != B200LA_F32)) return B200LA_ERR_ARG;
    b200la_csr *B = new b200la_csr(*A);
    B->dtype = dtype;
    B->row = nullptr;
    B->col = nullptr;
    B->val = nullptr;
    B->tiles = nullptr;
    B->long_rows = nullptr;
    B->pid = nullptr;
    B->pat_off = nullptr;
    B->pat_delta = nullptr;
    B->line_start = B->line_span = B->entry_line = B->entry_lo = nullptr;
    B->sell_off = nullptr;
    B->sell_val = nullptr;
    B->sell_len = 0;
    B->st_val = nullptr;
    B->st_use = stencil_policy(dtype);
    B->sh_val = nullptr;
    B->sh_mask = nullptr;
    B->sh_use = 0;
    B->lt_val = nullptr;   // the lattice layout stays with A (built by the preconditioners)
    B->lt = nullptr;
    B->invd32 = nullptr;
    const size_t pad = 8, es = dsize(dtype);
    cudaError_t e;
    if (A->pid) {
        if ((e = cudaMalloc(&B->pid, sizeof(uint16_t) * A->n)) ||
            (e = cudaMalloc(&B->pat_off, sizeof(int) * (A->npat + 1))) ||
            (e = cudaMalloc(&B->pat_delta, sizeof(int) * std::max(A->ndelta, 1))) ||
            (e = cudaMemcpy(B->pid, A->pid, sizeof(uint16_t) * A->n, cudaMemcpyDeviceToDevice)) ||
            (e = cudaMemcpy(B->pat_off, A->pat_off, sizeof(int) * (A->npat + 1), cudaMemcpyDeviceToDevice)) ||
            (e = cudaMemcpy(B->pat_delta, A->pat_delta, sizeof(int) * std::max(A->ndelta, 1),
                            cudaMemcpyDeviceToDevice))) {
            b200la_csr_destroy(B);
            return ctx_fail(ctx, B200LA_ERR_ALLOC, "csr_cast: pattern dictionary", e);
        }
        B->use_pat = pattern_policy(dtype);
        const int rc = copy_lines(ctx, A, B);
        if (rc) {
            b200la_csr_destroy(B);
            return rc;
        }
    }
    if ((e = cudaMalloc(&B->row, sizeof(int) * (A->n + 1 + pad))) ||
        (e = cudaMalloc(&B->col, sizeof(int) * (A->nnz + pad))) ||
        (e = cudaMalloc(&B->val, es * (A->nnz + pad))) ||
        (e = cudaMalloc(&B->tiles, sizeof(Tile) * std::max(A->ntiles, 1))) ||
        (e = cudaMalloc(&B->long_rows, sizeof(int) * std::max(A->nlong, 1)))) {
        b200la_csr_destroy(B);
        return ctx_fail(ctx, B200LA_ERR_ALLOC, "csr_cast: allocation", e);
    }
    B->bytes = sizeof(int) * (A->n + 1) + (sizeof(int) + es) * (A->nnz + pad) + sizeof(Tile) * A->ntiles +
               sizeof(int) * (A->nlong + 1);
    cudaStream_t s = ctx->stream;
    if ((e = cudaMemcpyAsync(B->row, A->row, sizeof(int) * (A->n + 1 + pad), cudaMemcpyDeviceToDevice, s)) ||
        (e = cudaMemcpyAsync(B->col, A->col, sizeof(int) * (A->nnz + pad), cudaMemcpyDeviceToDevice, s)) ||
        (e = launch_cast(A->dtype, A->val, dtype, B->val, (int)(A->nnz + pad), s)) ||
        (e = cudaMemcpyAsync(B->tiles, A->tiles, sizeof(Tile) * std::max(A->ntiles, 1), cudaMemcpyDeviceToDevice, s)) ||
        (e = cudaMemcpyAsync(B->long_rows, A->long_rows, sizeof(int) * std::max(A->nlong, 1), cudaMemcpyDeviceToDevice,
                             s)) ||
        (e = cudaStreamSynchronize(s))) {
        b200la_csr_destroy(B);
        return ctx_fail(ctx, B200LA_ERR_CUDA, "csr_cast", e);
    }
    int rc = build_sell(ctx, B);
    if (!rc) rc = build_stencil(ctx, B);
    if (rc) {
        b200la_csr_destroy(B);
        return rc;
    }
    *out = B;
    return B200LA_OK;
}

extern "C" int b200la_csr_info(const b200la_csr *A, int *n_rows, int *n_cols, int *nnz, int *dtype, int *lanes,
                               int *n_tiles, int *n_long)
{
    if (!A) return B200LA_ERR_ARG;
    if (n_rows) *n_rows = A->n;
    if (n_cols) *n_cols = A->m;
    if (nnz) *nnz = A->nnz;
    if (dtype) *dtype = A->dtype;
    if (lanes) *lanes = 1 << A->lg;
    if (n_tiles) *n_tiles = A->all.t1 - A->all.t0;
    if (n_long) *n_long = A->all.l1 - A->all.l0;
    return B200LA_OK;
}

extern "C" int b200la_csr_format(const b200la_csr *A, int *npat, int *uses_dict)
{
    if (!A) return B200LA_ERR_ARG;
    if (npat) *npat = A->pid ? A->npat : 0;
    if (uses_dict)
        *uses_dict = (A->lt && A->lt_val)                     ? 4
                     : (A->st_use && A->sh_use && A->sh_val) ? 3
                     : (A->st_use && A->st_val)              ? 2
                                                                 : (A->pid && A->use_pat) ? 1 : 0;
    return B200LA_OK;
}

extern "C" int b200la_csr_download(b200la_ctx *ctx, const b200la_csr *A, int *row, int *col, void *val)
{
    if (!ctx || !A) return B200LA_ERR_ARG;
    cudaStream_t s = ctx->stream;
    if (row) CK(cudaMemcpyAsync(row, A->row, sizeof(int) * (A->n + 1), cudaMemcpyDeviceToHost, s));
    if (col && A->nnz) CK(cudaMemcpyAsync(col, A->col, sizeof(int) * A->nnz, cudaMemcpyDeviceToHost, s));
    if (val && A->nnz) CK(cudaMemcpyAsync(val, A->val, dsize(A->dtype) * A->nnz, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return B200LA_OK;
}

extern "C" int b200la_csr_set_values(b200la_ctx *ctx, b200la_csr *A, const void *val)
{
    if (!ctx || !A || (A->nnz && !val)) return B200LA_ERR_ARG;
    if (A->nnz) CK(cudaMemcpyAsync(A->val, val, dsize(A->dtype) * A->nnz, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    drop_invd32(A);
    int rc = build_sell(ctx, A);
    if (!rc) rc = build_stencil(ctx, A);
    return rc ? rc : lattice_refresh(ctx, A);
}

extern "C" int b200la_csr_scale(b200la_ctx *ctx, b200la_csr *A, double alpha, int mode)
{
    if (!ctx || !A || mode < B200LA_SCALE_ALL || mode > B200LA_SCALE_ZERO)
        return ctx_msg(ctx, B200LA_ERR_ARG, "csr_scale: invalid argument");
    if (A->nnz) CK(launch_csr_scale(A->dtype, A->n, A->row, A->col, A->val, alpha, mode, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    drop_invd32(A);
    // the SpMV layouts derived from the values follow them
    int rc = build_sell(ctx, A);
    if (!rc) rc = build_stencil(ctx, A);
    return rc ? rc : lattice_refresh(ctx, A);
}

extern "C" int b200la_csr_diag(b200la_ctx *ctx, const b200la_csr *A, int start, int end, int inverse, void *out)
{
    if (!ctx || !A || start < 0 || end < start || end > A->n || end > A->m || (end > start && !out))
        return ctx_msg(ctx, B200LA_ERR_ARG, "csr_diag: invalid argument");
    if (end > start) CK(launch_csr_diag(A->dtype, start, end, A->row, A->col, A->val, inverse, out, ctx->stream));
    return B200LA_OK;
}

// Rows [r0, r1) filtered on the device (mode 0: columns [sc, ec) shifted to
// 0; mode 1: nonzero values), then a new matrix of n_cols columns from them.
static int csr_filter(b200la_ctx *ctx, const b200la_csr *A, int mode, int r0, int r1, int sc, int ec, int n_cols,
                      b200la_csr **out)
{
    const int rows = r1 - r0;
    const size_t es = dsize(A->dtype);
    int *d_cnt = nullptr, *d_off = nullptr, *d_col = nullptr;
    void *d_val = nullptr;
    std::vector<int> h_row(rows + 1, 0), h_col;
    std::vector<char> h_val;
    cudaError_t e = cudaMalloc(&d_cnt, sizeof(int) * std::max(rows, 1));
    if (e == cudaSuccess && rows) e = launch_csr_filter_count(A->dtype, r0, r1, A->row, A->col, A->val, mode, sc, ec,
                                                              d_cnt, ctx->stream);
    if (e == cudaSuccess && rows)
        e = cudaMemcpyAsync(h_row.data() + 1, d_cnt, sizeof(int) * rows, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    for (int i = 0; e == cudaSuccess && i < rows; ++i) h_row[i + 1] += h_row[i];
    const int k = h_row[rows];
    if (e == cudaSuccess && k) {
        h_col.resize(k);
        h_val.resize(es * k);
        e = cudaMalloc(&d_off, sizeof(int) * (rows + 1));
        if (e == cudaSuccess) e = cudaMalloc(&d_col, sizeof(int) * k);
        if (e == cudaSuccess) e = cudaMalloc(&d_val, es * k);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_off, h_row.data(), sizeof(int) * (rows + 1), cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess)
            e = launch_csr_filter_fill(A->dtype, r0, r1, A->row, A->col, A->val, mode, sc, ec, d_off, d_col, d_val,
                                       ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(h_col.data(), d_col, sizeof(int) * k, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_val.data(), d_val, es * k, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    }
    cudaFree(d_cnt);
    cudaFree(d_off);
    cudaFree(d_col);
    cudaFree(d_val);
    if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "csr_extract", e);
    return csr_upload(ctx, rows, n_cols, k, h_row.data(), k ? h_col.data() : nullptr,
                      k ? static_cast<const void *>(h_val.data()) : nullptr, A->dtype, 0, nullptr, out);
}

extern "C" int b200la_csr_extract_submatrix(b200la_ctx *ctx, const b200la_csr *A, int start_row, int start_col,
                                            int end_row, int end_col, b200la_csr **out)
{
    if (!ctx || !A || !out || start_row < 0 || start_col < 0 || end_row <= start_row || end_col <= start_col ||
        end_row > A->n || end_col > A->m)
        return ctx_msg(ctx, B200LA_ERR_ARG, "csr_extract_submatrix: invalid argument");
    return csr_filter(ctx, A, 0, start_row, end_row, start_col, end_col, end_col - start_col, out);
}

extern "C" int b200la_csr_compress(b200la_ctx *ctx, const b200la_csr *A, b200la_csr **out)
{
    if (!ctx || !A || !out) return ctx_msg(ctx, B200LA_ERR_ARG, "csr_compress: invalid argument");
    return csr_filter(ctx, A, 1, 0, A->n, 0, 0, A->m, out);
}

extern "C" int b200la_csr_invdiag(b200la_ctx *ctx, const b200la_csr *A, void *out)
{
    if (!ctx || !A || !out || A->n != A->m) return B200LA_ERR_ARG;
    CK(launch_invdiag(A->dtype, A->n, A->row, A->col, A->val, out, ctx->stream));
    return B200LA_OK;
}

// ------------------------------------------------------------------- SpMV

int spmv_run(b200la_ctx *ctx, const b200la_csr *A, const Seg &seg, SpmvOp op)
{
    int c0, c1;
    if (lattice_segment(A, seg, &c0, &c1)) {
        const cudaError_t e = launch_lattice(ctx_scratch(ctx), A->dtype, *A->lt, A->lt_val, c0, c1, op, ctx->stream);
        if (e != cudaErrorNotSupported) {   // not supported: this epilogue and range run on the CSR below
            CK(e);
            ctx->launches += 1;
            return B200LA_OK;
        }
        cudaGetLastError();
    }
    CK(launch_spmv(ctx_scratch(ctx), csr_view(A), seg, op, ctx->stream));
    ctx->launches += 1;
    return B200LA_OK;
}

extern "C" int b200la_spmv(b200la_ctx *ctx, const b200la_csr *A, const void *x, void *y)
{
    if (!ctx || !A || !x || !y || x == y) return ctx_msg(ctx, B200LA_ERR_ARG, "spmv: invalid argument");
    SpmvOp op;
    op.epi = EPI_SET;
    op.x = x;
    op.y = y;
    return spmv_run(ctx, A, A->all, op);
}

extern "C" int b200la_spmv_add(b200la_ctx *ctx, const b200la_csr *A, const void *x, void *y)
{
    if (!ctx || !A || !x || !y || x == y) return ctx_msg(ctx, B200LA_ERR_ARG, "spmv_add: invalid argument");
    SpmvOp op;
    op.epi = EPI_ADD;
    op.x = x;
    op.y = y;
    return spmv_run(ctx, A, A->all, op);
}

extern "C" int b200la_spmv_dot(b200la_ctx *ctx, const b200la_csr *A, const void *x, void *y, double *dot_dev)
{
    if (!ctx || !A || !x || !y || !dot_dev || x == y || A->n != A->m)
        return ctx_msg(ctx, B200LA_ERR_ARG, "spmv_dot: invalid argument");
    SpmvOp op;
    op.epi = EPI_DOT_X;
    op.fin = FIN_STORE;
    op.x = x;
    op.y = y;
    op.dot_out = dot_dev;
    return spmv_run(ctx, A, A->all, op);
}

extern "C" int b200la_residual(b200la_ctx *ctx, const b200la_csr *A, const void *b, const void *x, void *r,
                               double *nrm2sq_dev)
{
    if (!ctx || !A || !b || !x || !r || !nrm2sq_dev || x == r || A->n != A->m)
        return ctx_msg(ctx, B200LA_ERR_ARG, "residual: invalid argument");
    SpmvOp op;
    op.epi = EPI_RESID;
    op.fin = FIN_STORE;
    op.x = x;
    op.y = r;
    op.b = b;
    op.dot_out = nrm2sq_dev;
    return spmv_run(ctx, A, A->all, op);
}

// ------------------------------------------------------------------ GMG level steps

// The grid-transfer steps of a geometric multigrid level on the B200
// (lmp/cuda/cuda_gmg.h, kernels lmp/cuda/cuda_gmg_kernel.h): each operator
// is split into its diagonal block (columns of this rank's vector) and an
// optional off-diagonal block (columns of the ghost vector; null on one rank).
static int gmg_args(b200la_ctx *ctx, const b200la_csr *D, const b200la_csr *O, const void *in, const void *ghost,
                    const void *out, const char *what)
{
    if (!ctx || !D || !in || !out || in == out || (O && (!ghost || ghost == out)))
        return ctx_msg(ctx, B200LA_ERR_ARG, std::string(what) + ": invalid argument");
    if (O && (O->n != D->n || O->dtype != D->dtype))
        return ctx_msg(ctx, B200LA_ERR_ARG, std::string(what) + ": blocks differ in rows or precision");
    return B200LA_OK;
}

// res = rhs - A_diag sol - A_offdiag sol_ghost   (kernel_gmg_compute_residual)
extern "C" int b200la_gmg_residual(b200la_ctx *ctx, const b200la_csr *A_diag, const b200la_csr *A_offdiag,
                                   const void *sol, const void *rhs, const void *sol_ghost, void *res)
{
    int rc = gmg_args(ctx, A_diag, A_offdiag, sol, sol_ghost, res, "gmg_residual");
    if (rc) return rc;
    if (!rhs || rhs == sol) return ctx_msg(ctx, B200LA_ERR_ARG, "gmg_residual: invalid argument");
    SpmvOp op;
    op.epi = EPI_RESID;
    op.fin = FIN_NONE;
    op.x = sol;
    op.y = res;
    op.b = rhs;
    rc = spmv_run(ctx, A_diag, A_diag->all, op);
    if (rc || !A_offdiag) return rc;
    op.x = sol_ghost;
    op.b = res;   // res -= A_offdiag sol_ghost, row by row in place
    return spmv_run(ctx, A_offdiag, A_offdiag->all, op);
}

// res = R_diag tmp + R_offdiag res_ghost   (kernel_gmg_compute_restriction)
extern "C" int b200la_gmg_restriction(b200la_ctx *ctx, const b200la_csr *R_diag, const b200la_csr *R_offdiag,
                                      const void *tmp, const void *res_ghost, void *res)
{
    int rc = gmg_args(ctx, R_diag, R_offdiag, tmp, res_ghost, res, "gmg_restriction");
    if (rc) return rc;
    SpmvOp op;
    op.epi = EPI_SET;
    op.x = tmp;
    op.y = res;
    rc = spmv_run(ctx, R_diag, R_diag->all, op);
    if (rc || !R_offdiag) return rc;
    op.epi = EPI_ADD;
    op.x = res_ghost;
    return spmv_run(ctx, R_offdiag, R_offdiag->all, op);
}

// sol += P_diag res + P_offdiag res_ghost   (kernel_gmg_compute_updated_solution)
extern "C" int b200la_gmg_prolongation_add(b200la_ctx *ctx, const b200la_csr *P_diag, const b200la_csr *P_offdiag,
                                           const void *res, const void *res_ghost, void *sol)
{
    int rc = gmg_args(ctx, P_diag, P_offdiag, res, res_ghost, sol, "gmg_prolongation_add");
    if (rc) return rc;
    SpmvOp op;
    op.epi = EPI_ADD;
    op.x = res;
    op.y = sol;
    rc = spmv_run(ctx, P_diag, P_diag->all, op);
    if (rc || !P_offdiag) return rc;
    op.x = res_ghost;
    return spmv_run(ctx, P_offdiag, P_offdiag->all, op);
}

// ------------------------------------------------------------------ BLAS1

static bool dt_ok(int dtype) { return dtype == B200LA_F64 || dtype == B200LA_F32; }

extern "C" int b200la_dot_dev(b200la_ctx *ctx, int dtype, int n, const void *x, const void *y, double *out)
{
    if (!ctx || !dt_ok(dtype) || n < 0 || (n && (!x || !y)) || !out) return B200LA_ERR_ARG;
    CK(launch_dot(ctx_scratch(ctx), dtype, n, x, y, out, false, ctx->stream));
    return B200LA_OK;
}

extern "C" int b200la_dot(b200la_ctx *ctx, int dtype, int n, const void *x, const void *y, double *result)
{
    if (!ctx || !result) return B200LA_ERR_ARG;
    int rc = b200la_dot_dev(ctx, dtype, n, x, y, ctx->dscal);
    if (rc) return rc;
    CK(cudaMemcpyAsync(ctx->hscal, ctx->dscal, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *result = ctx->hscal[0];
    return B200LA_OK;
}

extern "C" int b200la_nrm2(b200la_ctx *ctx, int dtype, int n, const void *x, double *result)
{
    if (!ctx || !result || !dt_ok(dtype) || n < 0 || (n && !x)) return B200LA_ERR_ARG;
    CK(launch_dot(ctx_scratch(ctx), dtype, n, x, x, ctx->dscal, true, ctx->stream));
    CK(cudaMemcpyAsync(ctx->hscal, ctx->dscal, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *result = ctx->hscal[0];
    return B200LA_OK;
}

#define VEC_ARGS_OK (ctx && dt_ok(dtype) && n >= 0)

extern "C" int b200la_axpy(b200la_ctx *ctx, int dtype, int n, double alpha, const void *x, void *y)
{
    if (!VEC_ARGS_OK || (n && (!x || !y))) return B200LA_ERR_ARG;
    if (n) CK(launch_axpy(dtype, n, alpha, x, y, ctx->stream));
    return B200LA_OK;
}

extern "C" int b200la_scaleadd(b200la_ctx *ctx, int dtype, int n, double alpha, const void *x, void *y)
{
    if (!VEC_ARGS_OK || (n && (!x || !y))) return B200LA_ERR_ARG;
    if (n) CK(launch_scaleadd(dtype, n, alpha, x, y, ctx->stream));
    return B200LA_OK;
}

extern "C" int b200la_scale(b200la_ctx *ctx, int dtype, int n, double alpha, void *y)
{
    if (!VEC_ARGS_OK || (n && !y)) return B200LA_ERR_ARG;
    if (n) CK(launch_scale(dtype, n, alpha, y, ctx->stream));
    return B200LA_OK;
}

extern "C" int b200la_ewmul(b200la_ctx *ctx, int dtype, int n, const void *x, void *y)
{
    if (!VEC_ARGS_OK || (n && (!x || !y))) return B200LA_ERR_ARG;
    if (n) CK(launch_ewmul(dtype, n, x, y, ctx->stream));
    return B200LA_OK;
}

extern "C" int b200la_cast(b200la_ctx *ctx, int src_dtype, const void *src, int dst_dtype, void *dst, int n)
{
    if (!ctx || !dt_ok(src_dtype) || !dt_ok(dst_dtype) || n < 0 || (n && (!src || !dst))) return B200LA_ERR_ARG;
    if (n) CK(launch_cast(src_dtype, src, dst_dtype, dst, n, ctx->stream));
    return B200LA_OK;
}

extern "C" int b200la_gather(b200la_ctx *ctx, int dtype, int n_idx, const int *idx, const void *x, void *out)
{
    if (!ctx || !dt_ok(dtype) || n_idx < 0 || (n_idx && (!idx || !x || !out))) return B200LA_ERR_ARG;
    if (n_idx) CK(launch_gather(dtype, n_idx, idx, x, out, ctx->stream));
    return B200LA_OK;
}

extern "C" int b200la_scatter(b200la_ctx *ctx, int dtype, int n_idx, const int *idx, const void *vals, void *x)
{
    if (!ctx || !dt_ok(dtype) || n_idx < 0 || (n_idx && (!idx || !x || !vals))) return B200LA_ERR_ARG;
    if (n_idx) CK(launch_scatter(dtype, n_idx, idx, vals, x, ctx->stream));
    return B200LA_OK;
}

extern "C" int b200la_permute(b200la_ctx *ctx, int dtype, int n, const int *perm, const void *in, void *out)
{
    if (!ctx || !dt_ok(dtype) || n < 0 || (n && (!perm || !in || !out)) || in == out) return B200LA_ERR_ARG;
    if (n) CK(launch_gather(dtype, n, perm, in, out, ctx->stream));
    return B200LA_OK;
}

// ------------------------------------------------------- host-side setup

extern "C" int b200la_coo_to_csr(int n_rows, int nnz, const int *coo_row, const int *coo_col, const double *coo_val,
                                 int *row, int *col, double *val)
{
    if (n_rows < 0 || nnz < 0 || !row || (nnz && (!coo_row || !coo_col || !col)) || (coo_val && !val))
        return B200LA_ERR_ARG;
    for (int e = 0; e < nnz; ++e)
        if (coo_row[e] < 0 || coo_row[e] >= n_rows) return B200LA_ERR_CSR;
    host::coo_to_csr(n_rows, nnz, coo_row, coo_col, coo_val, row, col, val);
    return B200LA_OK;
}

extern "C" int b200la_add_values(const int *row, const int *col, double *val, const int *rows, int num_rows,
                                 const int *cols, int num_cols, const double *values)
{
    if (!row || !col || !val || num_rows < 0 || num_cols < 0 || (num_rows && (!rows || !values)) ||
        (num_cols && !cols))
        return B200LA_ERR_ARG;
    host::add_values(row, col, val, rows, num_rows, cols, num_cols, values);
    return B200LA_OK;
}

extern "C" int b200la_zero_rows(const int *row, const int *col, double *val, const int *idx, int size, double alpha)
{
    if (!row || !col || !val || size < 0 || (size && !idx)) return B200LA_ERR_ARG;
    host::zero_rows(row, col, val, idx, size, alpha);
    return B200LA_OK;
}

extern "C" int b200la_multicoloring(int n, const int *row, const int *col, int *ncolors, int *sizes, int *perm)
{
    if (n < 0 || !row || !col || !ncolors || !sizes || !perm) return B200LA_ERR_ARG;
    std::vector<int> s, p;
    if (host::multicoloring(n, row, col, ncolors, s, p)) return B200LA_ERR_SETUP;
    std::copy(s.begin(), s.end(), sizes);
    std::copy(p.begin(), p.end(), perm);
    return B200LA_OK;
}

extern "C" int b200la_levelscheduling(int n, const int *row, const int *col, int *nlevels, int *sizes, int *perm)
{
    if (n < 0 || !row || !col || !nlevels || !sizes || !perm) return B200LA_ERR_ARG;
    std::vector<int> s, p;
    if (host::levelscheduling(n, row, col, nlevels, s, p)) return B200LA_ERR_SETUP;
    std::copy(s.begin(), s.end(), sizes);
    std::copy(p.begin(), p.end(), perm);
    return B200LA_OK;
}

extern "C" int b200la_reorder_csr(int n, const int *row, const int *col, const double *val, const int *perm,
                                  int *row_out, int *col_out, double *val_out)
{
    if (n < 0 || !row || !col || !val || !perm || !row_out || !col_out || !val_out) return B200LA_ERR_ARG;
    host::Csr A, B;
    A.n = A.m = n;
    A.row.assign(row, row + n + 1);
    A.col.assign(col, col + row[n]);
    A.val.assign(val, val + row[n]);
    std::vector<int> p(perm, perm + n);
    host::reorder(A, p, B);
    std::copy(B.row.begin(), B.row.end(), row_out);
    std::copy(B.col.begin(), B.col.end(), col_out);
    std::copy(B.val.begin(), B.val.end(), val_out);
    return B200LA_OK;
}

extern "C" int b200la_ilu0(int n, const int *row, const int *col, double *val)
{
    if (n < 0 || !row || !col || !val) return B200LA_ERR_ARG;
    for (int i = 0; i < n; ++i) {
        bool diag = false;
        for (int j = row[i]; j < row[i + 1]; ++j) diag |= (col[j] == i);
        if (!diag) return B200LA_ERR_CSR;   // the factorisation walks each row up to its diagonal
    }
    host::ilu0(n, row, col, val);
    return B200LA_OK;
}

static int host_csr_in(int n, const int *row, const int *col, const double *val, host::Csr &A)
{
    if (n < 0 || !row || !col) return B200LA_ERR_ARG;
    long long bad = -1;
    if (host::validate_csr(n, n, row[n], row, col, &bad)) return B200LA_ERR_CSR;
    A.n = A.m = n;
    A.row.assign(row, row + n + 1);
    A.col.assign(col, col + row[n]);
    if (val) A.val.assign(val, val + row[n]);
    else A.val.assign(row[n], 1.0);
    return B200LA_OK;
}

// Copy out a host CSR in the two-call convention: always *nnz; the arrays
// when row_out is given (then col_out and val_out, if given, hold *nnz).
static int host_csr_out(const host::Csr &B, int *nnz, int *row_out, int *col_out, double *val_out)
{
    *nnz = B.nnz();
    if (!row_out) return B200LA_OK;
    std::copy(B.row.begin(), B.row.end(), row_out);
    if (col_out) std::copy(B.col.begin(), B.col.end(), col_out);
    if (val_out) std::copy(B.val.begin(), B.val.end(), val_out);
    return B200LA_OK;
}

extern "C" int b200la_matrix_power_pattern(int n, const int *row, const int *col, int p, int *nnz, int *row_out,
                                           int *col_out)
{
    if (p < 1 || !nnz) return B200LA_ERR_ARG;
    host::Csr A, P;
    int rc = host_csr_in(n, row, col, nullptr, A);
    if (rc) return rc;
    host::matrix_sup_power(A, p, P);
    return host_csr_out(P, nnz, row_out, col_out, nullptr);
}

extern "C" int b200la_ilup(int n, const int *row, const int *col, const double *val, int p, int *nnz, int *row_out,
                           int *col_out, double *val_out)
{
    if (p < 0 || !val || !nnz) return B200LA_ERR_ARG;
    host::Csr A, LU;
    int rc = host_csr_in(n, row, col, val, A);
    if (rc) return rc;
    for (int i = 0; i < n; ++i) {
        bool diag = false;
        for (int j = row[i]; j < row[i + 1]; ++j) diag |= (col[j] == i);
        if (!diag) return B200LA_ERR_CSR;   // the factorisation walks each row up to its diagonal
    }
    host::ilup(A, p, LU);
    return host_csr_out(LU, nnz, row_out, col_out, val_out);
}

extern "C" int b200la_rowblock_split(int n_rows, int n_global, const int *row, const int *col, const double *val,
                                     int col_begin, int col_end, int *nnz_diag, int *nnz_offdiag, int *n_ghost,
                                     int *row_d, int *col_d, double *val_d, int *row_o, int *col_o, double *val_o,
                                     int *ghost_global)
{
    // CoupledMatrix::InitStructure (coupled_matrix.cc:253-340) with the ghost
    // numbering of LaCouplings::InitializeCouplings (la_couplings.cc:62-130):
    // owned columns shifted to local numbering, the others numbered by their
    // rank among the distinct ghost columns in ascending order (per owner in
    // ascending order, owners being contiguous ranges)
    if (n_rows < 0 || !row || !nnz_diag || !nnz_offdiag || !n_ghost || col_begin < 0 || col_end < col_begin ||
        col_end > n_global)
        return B200LA_ERR_ARG;
    long long bad = -1;
    if (host::validate_csr(n_rows, n_global, row[n_rows], row, col, &bad)) return B200LA_ERR_CSR;
    std::vector<int> ghosts;
    int nd = 0, no = 0;
    for (int j = 0; j < row[n_rows]; ++j) {
        if (col[j] >= col_begin && col[j] < col_end) ++nd;
        else {
            ++no;
            ghosts.push_back(col[j]);
        }
    }
    std::sort(ghosts.begin(), ghosts.end());
    ghosts.erase(std::unique(ghosts.begin(), ghosts.end()), ghosts.end());
    *nnz_diag = nd;
    *nnz_offdiag = no;
    *n_ghost = (int)ghosts.size();
    if (!row_d) return B200LA_OK;
    if (!row_o || (nd && (!col_d || !val_d || !val)) || (no && (!col_o || !val_o)) || (!ghosts.empty() && !ghost_global))
        return B200LA_ERR_ARG;
    int td = 0, to = 0;
    row_d[0] = row_o[0] = 0;
    for (int i = 0; i < n_rows; ++i) {
        for (int j = row[i]; j < row[i + 1]; ++j) {
            const int c = col[j];
            if (c >= col_begin && c < col_end) {
                col_d[td] = c - col_begin;
                val_d[td++] = val[j];
            } else {
                col_o[to] = (int)(std::lower_bound(ghosts.begin(), ghosts.end(), c) - ghosts.begin());
                val_o[to++] = val[j];
            }
        }
        row_d[i + 1] = td;
        row_o[i + 1] = to;
    }
    std::copy(ghosts.begin(), ghosts.end(), ghost_global);
    return B200LA_OK;
}

extern "C" int b200la_q1_sizes(int dim, int N, int *n, int64_t *nnz)
{
    if (!n || !nnz) return B200LA_ERR_ARG;
    return host::q1_sizes(dim, N, n, nnz) ? B200LA_ERR_ARG : B200LA_OK;
}

extern "C" int b200la_q1_assemble(int dim, int N, int kind, const double *kcell, double nu, const double *beta,
                                  int *row, int *col, double *val)
{
    if (!row || !col || !val || (kind == 1 && !beta) || (kind != 0 && kind != 1)) return B200LA_ERR_ARG;
    return host::q1_assemble(dim, N, kind, kcell, nu, beta, row, col, val) ? B200LA_ERR_ARG : B200LA_OK;
}

extern "C" int b200la_q1_rhs(uint64_t seed, int dim, int N, double *b)
{
    int n;
    int64_t nnz;
    if (!b || host::q1_sizes(dim, N, &n, &nnz)) return B200LA_ERR_ARG;
    host::q1_rhs(seed, dim, N, b);
    return B200LA_OK;
}
