// solvers.cu -- device-resident Krylov loops of the B200 lmp platform.
//
// The reference's solvers (src/linear_solver/cg.cc, gmres.cc, mpir.cc) return
// every dot product to the host and synchronise the device before each of
// the ~11 launches of an iteration.  Here the recurrence scalars and the
// IterateControl test live in device memory (DevState): the last CTA of each
// reducing kernel updates them, every later kernel of the iteration checks the
// stop state first and does nothing once the test has fired, and iterations
// are replayed from a captured CUDA graph in batches, so the host reads the
// state only once per batch.  The iteration count and the stop decision are
// exactly those of IterateControl::Check (src/common/iterate_control.cc:84-110).
#include "b200la.h"
#include "b200la_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace b200;

#define SK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, #call, e_);        \
    } while (0)

void graph_cache_clear(b200la_ctx *ctx)
{
    for (auto &g : ctx->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    ctx->graphs.clear();
}

static int batch_size()
{
    if (const char *e = std::getenv("B200LA_BATCH")) return std::max(1, std::atoi(e));
    return 16;
}

// Capture `body` (which enqueues kernels on ctx->stream) into a graph keyed by
// `key`, or reuse the cached one.  Returns the executable graph.
template <class Body>
static int get_graph(b200la_ctx *ctx, const std::vector<const void *> &key, Body body, cudaGraphExec_t *exec,
                     int *nodes)
{
    for (auto &g : ctx->graphs)
        if (g.key == key) {
            *exec = g.exec;
            *nodes = g.launches;
            return B200LA_OK;
        }
    if (ctx->graphs.size() >= 32) graph_cache_clear(ctx);
    cudaGraph_t graph;
    SK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const long long before = ctx->launches;
    const int rc = body();
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (rc) {
        if (e == cudaSuccess) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "graph capture", e);
    GraphEntry g;
    g.key = key;
    g.launches = (int)(ctx->launches - before);
    ctx->launches = before;
    e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "graph instantiate", e);
    ctx->graphs.push_back(g);
    *exec = g.exec;
    *nodes = g.launches;
    return B200LA_OK;
}

// The same for a graph whose single node is a device-side while loop: its
// body is `body(h)` captured once (K iterations), and the loop runs again as
// long as the conditional handle h -- set by the update kernel after each
// Check -- says "iterate".  One launch runs the solve to its stop; the host
// waits once instead of once per batch, and no batch of gated iterations
// runs after the stop.
template <class Body>
static int get_while_graph(b200la_ctx *ctx, const std::vector<const void *> &key, Body body, cudaGraphExec_t *exec,
                           int *nodes)
{
    for (auto &g : ctx->graphs)
        if (g.key == key) {
            *exec = g.exec;
            *nodes = g.launches;
            return B200LA_OK;
        }
    if (ctx->graphs.size() >= 32) graph_cache_clear(ctx);
    cudaGraph_t graph = nullptr;
    SK(cudaGraphCreate(&graph, 0));
    struct GraphGuard {
        cudaGraph_t g;
        ~GraphGuard()
        {
            if (g) cudaGraphDestroy(g);
        }
    } guard{graph};
    cudaGraphConditionalHandle h;
    SK(cudaGraphConditionalHandleCreate(&h, graph, 1u, cudaGraphCondAssignDefault));
    cudaGraphNodeParams prm = {cudaGraphNodeTypeConditional};
    prm.conditional.handle = h;
    prm.conditional.type = cudaGraphCondTypeWhile;
    prm.conditional.size = 1;
    cudaGraphNode_t node;
    SK(cudaGraphAddNode(&node, graph, nullptr, 0, &prm));
    cudaGraph_t loop = prm.conditional.phGraph_out[0];
    SK(cudaStreamBeginCaptureToGraph(ctx->stream, loop, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const long long before = ctx->launches;
    const int rc = body((unsigned long long)h);
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &loop);
    if (rc) return rc;
    if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "loop body capture", e);
    GraphEntry g;
    g.key = key;
    g.launches = (int)(ctx->launches - before);
    ctx->launches = before;
    e = cudaGraphInstantiate(&g.exec, graph, 0);
    if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "loop graph instantiate", e);
    ctx->graphs.push_back(g);
    *exec = g.exec;
    *nodes = g.launches;
    return B200LA_OK;
}

// Device-side loop control of the CG iterations (B200LA_GRAPH_LOOP=0: host
// reads the stop state after every batch instead).
static bool loop_policy()
{
    const char *e = std::getenv("B200LA_GRAPH_LOOP");
    return !e || std::atoi(e) != 0;
}

static void state_init(DevState &s, const b200la_control *ctl, double *hist, int hist_len)
{
    std::memset(&s, 0, sizeof s);
    s.maxits = ctl->maxits;
    s.abstol = ctl->abstol;
    s.reltol = ctl->reltol;
    s.divtol = ctl->divtol;
    s.status = kIterate;
    s.hist = hist;
    s.hist_len = hist_len;
}

// ------------------------------------------------------------------ CG

struct CgWork {
    void *r, *p, *Ap, *z;
};

static int cg_core(b200la_ctx *ctx, const b200la_csr *A, const b200la_precond *P, const void *b, void *x,
                   const b200la_control *ctl, b200la_result *res, double *hist_dev, int hist_len, CgWork w,
                   bool time_it)
{
    const int n = A->n, dt = A->dtype;
    const int pc = !P ? 0 : (P->kind == B200LA_PRECOND_JACOBI ? 1 : 2);
    const void *invd = (pc == 1) ? P->invd : nullptr;
    const int *gate = &ctx->st->status;
    const Scratch sc = ctx_scratch(ctx);
    const long long l0 = ctx->launches;

    DevState *hs = ctx->st_host;
    state_init(*hs, ctl, hist_dev, hist_len);
    SK(cudaMemcpyAsync(ctx->st, hs, sizeof(DevState), cudaMemcpyHostToDevice, ctx->stream));
    if (time_it) SK(cudaEventRecord(ctx->ev0, ctx->stream));

    // r = b - A x; res0 = ||r||; status = Check(0, res0)   (cg.cc:200-204)
    SpmvOp op;
    op.epi = EPI_RESID;
    op.fin = FIN_RES_INIT;
    op.x = x;
    op.y = w.r;
    op.b = b;
    op.st = ctx->st;
    int rc = spmv_run(ctx, A, A->all, op);
    if (rc) return rc;
    // z = M^-1 r; p = z; rho = r.z   (cg.cc:205-214)
    if (pc == 2) {
        rc = precond_apply_async(ctx, P, w.r, w.z, nullptr);
        if (rc) return rc;
    }
    SK(launch_cg_start(sc, dt, n, pc, w.r, invd, w.z, w.p, ctx->st, ctx->stream));
    ctx->launches += 1;
    unsigned long long cond = 0;   // loop condition of the device-side while node (when captured in one)

    auto iteration = [&]() -> int {
        // Ap = A p; alpha = rho / (Ap.p)                       (cg.cc:219-220)
        SpmvOp o;
        o.epi = EPI_DOT_X;
        o.fin = FIN_CG_ALPHA;
        o.x = w.p;
        o.y = w.Ap;
        o.st = ctx->st;
        o.gate = gate;
        int r2 = spmv_run(ctx, A, A->all, o);
        if (r2) return r2;
        // x += alpha p; r -= alpha Ap; res = ||r||; Check       (cg.cc:221-230)
        SK(launch_cg_update(sc, dt, n, pc, x, w.r, w.p, w.Ap, invd, ctx->st, ctx->stream, cond));
        ctx->launches += 1;
        if (pc == 2) {
            // z = M^-1 r; gamma = r.z; beta = gamma / rho     (cg.cc:236-240)
            r2 = precond_apply_async(ctx, P, w.r, w.z, gate);
            if (r2) return r2;
            SK(launch_cg_rz(sc, dt, n, w.r, w.z, ctx->st, ctx->stream));
            ctx->launches += 1;
        }
        // p = beta p + z                                        (cg.cc:241)
        SK(launch_cg_pupdate(dt, n, pc, w.p, w.r, invd, w.z, ctx->st, ctx->stream));
        ctx->launches += 1;
        return B200LA_OK;
    };

    const int K = batch_size();
    cudaGraphExec_t exec = nullptr;
    int nodes = 0;
    const bool no_graph = std::getenv("B200LA_NOGRAPH") != nullptr;
    if (no_graph) {
        // batches launched kernel by kernel on the stream (same work, no graph)
        SK(cudaMemcpyAsync(hs, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
        SK(cudaStreamSynchronize(ctx->stream));
        const long long max_b = (long long)ctl->maxits / K + 2;
        for (long long bt = 0; hs->status == kIterate && bt < max_b; ++bt) {
            for (int k = 0; k < K; ++k) {
                rc = iteration();
                if (rc) return rc;
            }
            SK(cudaMemcpyAsync(hs, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
            SK(cudaStreamSynchronize(ctx->stream));
        }
    }
    const bool loop = !no_graph && loop_policy();
    const std::vector<const void *> key = {A, P, b, x, w.r, w.p, w.Ap, w.z, (const void *)(intptr_t)K,
                                           (const void *)(intptr_t)pc, ctx->stream, (const void *)(intptr_t)loop};
    auto batch = [&]() -> int {
        for (int k = 0; k < K; ++k) {
            int r2 = iteration();
            if (r2) return r2;
        }
        return B200LA_OK;
    };
    if (loop)
        rc = get_while_graph(
            ctx, key,
            [&](unsigned long long h) -> int {
                cond = h;
                const int r2 = batch();
                cond = 0;
                return r2;
            },
            &exec, &nodes);
    else if (!no_graph)
        rc = get_graph(ctx, key, batch, &exec, &nodes);
    if (rc) return rc;
    SK(cudaMemcpyAsync(hs, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
    SK(cudaStreamSynchronize(ctx->stream));
    long long graph_launches = 0;
    if (loop && hs->status == kIterate) {
        // one launch; the loop ends on the device at the stop of IterateControl
        const int it0 = hs->iter;
        SK(cudaGraphLaunch(exec, ctx->stream));
        SK(cudaMemcpyAsync(hs, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
        SK(cudaStreamSynchronize(ctx->stream));
        graph_launches += (long long)nodes * std::max(1, (hs->iter - it0 + K - 1) / K);
    }
    const long long max_batches = (long long)ctl->maxits / K + 2;
    for (long long bt = 0; !no_graph && !loop && hs->status == kIterate && bt < max_batches; ++bt) {
        SK(cudaGraphLaunch(exec, ctx->stream));
        graph_launches += nodes;
        SK(cudaMemcpyAsync(hs, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
        SK(cudaStreamSynchronize(ctx->stream));
    }
    float ms = 0.f;
    if (time_it) {
        SK(cudaEventRecord(ctx->ev1, ctx->stream));
        SK(cudaEventSynchronize(ctx->ev1));
        SK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    }
    rc = ctx_check_device_error(ctx);
    if (rc) return rc;
    if (res) {
        res->iters = hs->iter;
        res->status = hs->status;
        res->res0 = hs->res0;
        res->res = hs->res;
        res->outer = 0;
        res->launches = (int)(ctx->launches - l0 + graph_launches);
        res->solve_ms = ms;
    }
    ctx->launches += graph_launches;
    return B200LA_OK;
}

static int cg_entry(b200la_ctx *ctx, const b200la_csr *A, const b200la_precond *P, const void *b, void *x,
                    const b200la_control *ctl, b200la_result *res, double *hist, int hist_len)
{
    if (!ctx || !A || !b || !x || !ctl || A->n != A->m || ctl->maxits < 0)
        return ctx_fail(ctx, B200LA_ERR_ARG, "cg: invalid argument", cudaSuccess);
    if (P && (P->dtype != A->dtype || P->n != A->n))
        return ctx_fail(ctx, B200LA_ERR_ARG, "cg: preconditioner does not match the operator", cudaSuccess);
    const size_t es = A->dtype == B200LA_F64 ? 8 : 4;
    const size_t vb = ((es * std::max(A->n, 1) + 255) / 256) * 256;
    const int hl = hist ? hist_len : 0;
    void *wk;
    int rc = ctx_work(ctx, 4 * vb + sizeof(double) * (hl + 1), &wk);
    if (rc) return rc;
    char *base = static_cast<char *>(wk);
    CgWork w{base, base + vb, base + 2 * vb, base + 3 * vb};
    double *hd = hl ? reinterpret_cast<double *>(base + 4 * vb) : nullptr;
    rc = cg_core(ctx, A, P, b, x, ctl, res, hd, hl, w, true);
    if (rc) return rc;
    if (hl) {
        const int cnt = std::min(hl, (res ? res->iters : 0) + 1);
        SK(cudaMemcpy(hist, hd, sizeof(double) * cnt, cudaMemcpyDeviceToHost));
    }
    return B200LA_OK;
}

extern "C" int b200la_cg(b200la_ctx *ctx, const b200la_csr *A, const b200la_precond *P, const void *b, void *x,
                         const b200la_control *ctl, b200la_result *res)
{
    NvtxScope nvtx_range("b200la_cg");
    return cg_entry(ctx, A, P, b, x, ctl, res, nullptr, 0);
}

extern "C" int b200la_cg_hist(b200la_ctx *ctx, const b200la_csr *A, const b200la_precond *P, const void *b,
                              void *x, const b200la_control *ctl, b200la_result *res, double *hist, int hist_len)
{
    NvtxScope nvtx_range("b200la_cg_hist");
    return cg_entry(ctx, A, P, b, x, ctl, res, hist, hist_len);
}

// ------------------------------------------------------------------ MPIR

extern "C" int b200la_mpir(b200la_ctx *ctx, const b200la_csr *A64, const b200la_csr *A32in, const double *b,
                           double *x, const b200la_control *outer, const b200la_control *inner, int max_outer,
                           b200la_result *res)
{
    NvtxScope nvtx_range("b200la_mpir");
    if (!ctx || !A64 || !b || !x || !outer || !inner || A64->dtype != B200LA_F64 || A64->n != A64->m ||
        max_outer < 0 || (A32in && (A32in->dtype != B200LA_F32 || A32in->n != A64->n || A32in->nnz != A64->nnz)))
        return ctx_fail(ctx, B200LA_ERR_ARG, "mpir: invalid argument", cudaSuccess);
    const int n = A64->n;
    b200la_csr *A32 = const_cast<b200la_csr *>(A32in);
    bool own32 = false;
    if (!A32) {
        int rc = b200la_csr_cast(ctx, A64, B200LA_F32, &A32);
        if (rc) return rc;
        own32 = true;
    }
    struct Guard {
        b200la_csr *m;
        bool own;
        ~Guard()
        {
            if (own) b200la_csr_destroy(m);
        }
    } guard{A32, own32};
    const size_t v8 = ((8 * (size_t)std::max(n, 1) + 255) / 256) * 256, v4 = ((4 * (size_t)std::max(n, 1) + 255) / 256) * 256;
    void *wk;
    // r (f64), invd64 scratch (f64), rl, cl, and the inner CG's r, p, Ap (f32)
    int rc = ctx_work(ctx, 2 * v8 + 6 * v4, &wk);
    if (rc) return rc;
    char *base = static_cast<char *>(wk);
    double *r = reinterpret_cast<double *>(base);
    double *invd64 = reinterpret_cast<double *>(base + v8);
    float *invd32 = nullptr;   // the operator's cached FP32 Jacobi scaling (below)
    float *rl = reinterpret_cast<float *>(base + 2 * v8 + v4);
    float *cl = reinterpret_cast<float *>(base + 2 * v8 + 2 * v4);
    CgWork w{base + 2 * v8 + 3 * v4, base + 2 * v8 + 4 * v4, base + 2 * v8 + 5 * v4, nullptr};
    const long long l0 = ctx->launches;

    // FP32 Jacobi from the FP64 diagonal (1/a_ii rounded once), made at the
    // operator's first defect correction and kept with it until its values change
    if (!A64->invd32) {
        b200la_csr *Am = const_cast<b200la_csr *>(A64);
        SK(cudaMalloc(&Am->invd32, sizeof(float) * std::max(n, 1)));
        SK(launch_invdiag(B200LA_F64, n, A64->row, A64->col, A64->val, invd64, ctx->stream));
        SK(launch_cast(B200LA_F64, invd64, B200LA_F32, Am->invd32, n, ctx->stream));
        ctx->launches += 2;
    }
    invd32 = A64->invd32;
    SK(cudaEventRecord(ctx->ev0, ctx->stream));
    b200la_precond J;
    J.kind = B200LA_PRECOND_JACOBI;
    J.n = n;
    J.dtype = B200LA_F32;
    J.invd = invd32;

    auto residual = [&](double *out) -> int {
        // r = b - A x in FP64 and ||r||   (mpir.cc:125-128, 271-273)
        SpmvOp op;
        op.epi = EPI_RESID;
        op.fin = FIN_STORE;
        op.x = x;
        op.y = r;
        op.b = b;
        op.dot_out = ctx->dscal;
        int r2 = spmv_run(ctx, A64, A64->all, op);
        if (r2) return r2;
        SK(cudaMemcpyAsync(ctx->hscal, ctx->dscal, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        SK(cudaStreamSynchronize(ctx->stream));
        *out = std::sqrt(ctx->hscal[0]);
        return B200LA_OK;
    };
    double rnorm;
    rc = residual(&rnorm);
    if (rc) return rc;
    const double res0 = rnorm;
    int n_outer = 0, inner_total = 0;
    long long inner_launches = 0;
    // ContinueIteration (mpir.cc:308-326) with the relative test against the
    // initial residual
    while (rnorm > outer->abstol && rnorm > outer->reltol * res0 && rnorm < outer->divtol && n_outer < max_outer) {
        ++n_outer;
        // resl = (float) resh; corl = 0   (mpir.cc:169-170)
        SK(launch_cast_residual(n, r, rl, cl, ctx->stream));
        ctx->launches += 1;
        // low-precision error correction: Jacobi-CG on A32 (mpir.cc:193)
        b200la_result ir;
        std::memset(&ir, 0, sizeof ir);
        rc = cg_core(ctx, A32, &J, rl, cl, inner, &ir, nullptr, 0, w, false);
        if (rc) return rc;
        inner_total += ir.iters;
        inner_launches += ir.launches;
        // x += (double) corl   (mpir.cc:223, 253)
        SK(launch_add_correction(n, cl, x, ctx->stream));
        ctx->launches += 1;
        rc = residual(&rnorm);
        if (rc) return rc;
    }
    SK(cudaEventRecord(ctx->ev1, ctx->stream));
    SK(cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    SK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    if (res) {
        res->iters = inner_total;
        res->outer = n_outer;
        res->res0 = res0;
        res->res = rnorm;
        res->status = rnorm < outer->abstol ? B200LA_SUCCESS_ABS
                      : rnorm < outer->reltol * res0 ? B200LA_SUCCESS_REL
                      : rnorm >= outer->divtol     ? B200LA_FAIL_DIV
                                                   : B200LA_FAIL_MAXITS;
        res->launches = (int)(ctx->launches - l0);
        res->solve_ms = ms;
    }
    (void)inner_launches;
    return ctx_check_device_error(ctx);
}

// ------------------------------------------------------------------ MPIR with a GMRES correction

extern "C" int b200la_mpir_gmres(b200la_ctx *ctx, const b200la_csr *A64, const b200la_csr *A32,
                                 const b200la_precond *P32, int m, const double *b, double *x,
                                 const b200la_control *outer, const b200la_control *inner, int max_outer,
                                 b200la_result *res)
{
    NvtxScope nvtx_range("b200la_mpir_gmres");
    if (!ctx || !A64 || !A32 || !b || !x || !outer || !inner || m < 1 || max_outer < 0 ||
        A64->dtype != B200LA_F64 || A32->dtype != B200LA_F32 || A64->n != A64->m || A32->n != A64->n ||
        (P32 && (P32->dtype != B200LA_F32 || P32->n != A64->n)))
        return ctx_fail(ctx, B200LA_ERR_ARG, "mpir_gmres: invalid argument", cudaSuccess);
    const int n = A64->n;
    const size_t v8 = ((8 * (size_t)std::max(n, 1) + 255) / 256) * 256, v4 = ((4 * (size_t)std::max(n, 1) + 255) / 256) * 256;
    void *wk;
    int rc = ctx_work_outer(ctx, v8 + 2 * v4, &wk);
    if (rc) return rc;
    char *base = static_cast<char *>(wk);
    double *r = reinterpret_cast<double *>(base);
    float *rl = reinterpret_cast<float *>(base + v8);
    float *cl = reinterpret_cast<float *>(base + v8 + v4);
    const long long l0 = ctx->launches;
    // own events: the inner GMRES times itself with the context's
    struct Ev {
        cudaEvent_t a = nullptr, b = nullptr;
        ~Ev()
        {
            if (a) cudaEventDestroy(a);
            if (b) cudaEventDestroy(b);
        }
    } ev;
    SK(cudaEventCreate(&ev.a));
    SK(cudaEventCreate(&ev.b));
    SK(cudaEventRecord(ev.a, ctx->stream));
    auto residual = [&](double *out) -> int {
        // r = b - A x in FP64 and ||r||   (mpir.cc:125-128, 271-273)
        SpmvOp op;
        op.epi = EPI_RESID;
        op.fin = FIN_STORE;
        op.x = x;
        op.y = r;
        op.b = b;
        op.dot_out = ctx->dscal;
        int r2 = spmv_run(ctx, A64, A64->all, op);
        if (r2) return r2;
        SK(cudaMemcpyAsync(ctx->hscal, ctx->dscal, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        SK(cudaStreamSynchronize(ctx->stream));
        *out = std::sqrt(ctx->hscal[0]);
        return B200LA_OK;
    };
    double rnorm;
    rc = residual(&rnorm);
    if (rc) return rc;
    const double res0 = rnorm;
    int n_outer = 0, inner_total = 0, inner_launches = 0;
    while (rnorm > outer->abstol && rnorm > outer->reltol * res0 && rnorm < outer->divtol && n_outer < max_outer) {
        ++n_outer;
        // resl = (float) resh; corl = 0   (mpir.cc:169-170)
        SK(launch_cast_residual(n, r, rl, cl, ctx->stream));
        ctx->launches += 1;
        // low-precision error correction: GMRES(m) on A32 with P32 (mpir.cc:193)
        b200la_result ir;
        std::memset(&ir, 0, sizeof ir);
        rc = b200la_gmres(ctx, A32, P32, m, rl, cl, inner, &ir);
        if (rc) return rc;
        inner_total += ir.iters;
        inner_launches += ir.launches;
        // x += (double) corl   (mpir.cc:223, 253)
        SK(launch_add_correction(n, cl, x, ctx->stream));
        ctx->launches += 1;
        rc = residual(&rnorm);
        if (rc) return rc;
    }
    SK(cudaEventRecord(ev.b, ctx->stream));
    SK(cudaEventSynchronize(ev.b));
    float ms = 0.f;
    SK(cudaEventElapsedTime(&ms, ev.a, ev.b));
    if (res) {
        res->iters = inner_total;
        res->outer = n_outer;
        res->res0 = res0;
        res->res = rnorm;
        res->status = rnorm < outer->abstol ? B200LA_SUCCESS_ABS
                      : rnorm < outer->reltol * res0 ? B200LA_SUCCESS_REL
                      : rnorm >= outer->divtol     ? B200LA_FAIL_DIV
                                                   : B200LA_FAIL_MAXITS;
        res->launches = (int)(ctx->launches - l0);
        res->solve_ms = ms;
    }
    (void)inner_launches;
    return ctx_check_device_error(ctx);
}

// ------------------------------------------------------------------ GMRES

namespace {

struct GmresDev {
    double *H;      // H(j, i) = H[j * (m + 1) + i]
    double *g, *cs, *sn, *y;
    int *jend;
};

__device__ __forceinline__ int check_dev(DevState *st, int step, double value)
{
    if (step == 0) st->res0 = value;
    if (value < st->abstol) return kSuccessAbs;
    if (value < st->reltol * st->res0) return kSuccessRel;
    if (value > st->divtol * st->res0) return kFailDiv;
    if (step >= st->maxits) return kFailMaxits;
    return kIterate;
}

// Givens part of one Arnoldi step (gmres.cc:380-402 with gmres.h:77-97).
__global__ void gmres_givens_kernel(int j, int m, GmresDev d, DevState *st)
{
    if (st->status != kIterate) return;
    const int ld = m + 1;
    double *Hj = d.H + (size_t)j * ld;
    for (int k = 0; k < j; ++k) {
        const double t = d.cs[k] * Hj[k] + d.sn[k] * Hj[k + 1];
        Hj[k + 1] = -d.sn[k] * Hj[k] + d.cs[k] * Hj[k + 1];
        Hj[k] = t;
    }
    const double beta = sqrt(Hj[j] * Hj[j] + Hj[j + 1] * Hj[j + 1]);
    d.cs[j] = Hj[j] / beta;
    d.sn[j] = Hj[j + 1] / beta;
    {
        const double t = d.cs[j] * Hj[j] + d.sn[j] * Hj[j + 1];
        Hj[j + 1] = -d.sn[j] * Hj[j] + d.cs[j] * Hj[j + 1];
        Hj[j] = t;
    }
    {
        const double t = d.cs[j] * d.g[j] + d.sn[j] * d.g[j + 1];
        d.g[j + 1] = -d.sn[j] * d.g[j] + d.cs[j] * d.g[j + 1];
        d.g[j] = t;
    }
    const double res = fabs(d.g[j + 1]);
    const int it = st->iter + 1;
    st->iter = it;
    st->res = res;
    const int s = check_dev(st, it, res);
    st->status = s;
    if (s != kIterate) *d.jend = j;
}

// Back substitution of UpdateSolution (gmres.cc:487-504) into y[0..k].
__global__ void gmres_backsub_kernel(int k, int m, GmresDev d)
{
    const int ld = m + 1;
    for (int i = 0; i <= m; ++i) d.y[i] = d.g[i];
    for (int i = k + 1; i--;) {
        d.y[i] /= d.H[(size_t)i * ld + i];
        const double t = d.y[i];
        for (int q = 0; q < i; ++q) d.y[q] -= d.H[(size_t)i * ld + q] * t;
    }
}

// Cycle start: H = 0, g = 0, g[0] = res (gmres.cc:344-350).  As in the
// reference, a restart normalises the new residual by the last Givens
// estimate |g[j+1]| held in res, not by a recomputed norm.
__global__ void gmres_cycle_kernel(int m, GmresDev d, const DevState *st)
{
    const int ld = m + 1;
    for (int i = threadIdx.x; i < m * ld; i += blockDim.x) d.H[i] = 0.0;
    for (int i = threadIdx.x; i <= m; i += blockDim.x) d.g[i] = 0.0;
    __syncthreads();
    if (threadIdx.x == 0) d.g[0] = st->res;
}

// z = sum_{i<=k} y_i V_i (the vectors V_i at stride ld elements).
template <typename T>
__global__ void lincomb_kernel(int n, int k, const T *__restrict__ V, size_t ld, const double *__restrict__ y,
                               T *__restrict__ z)
{
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        T s = T(0);
        for (int q = 0; q <= k; ++q) s += (T)y[q] * V[(size_t)q * ld + i];
        z[i] = s;
    }
}

}  // namespace

extern "C" int b200la_gmres(b200la_ctx *ctx, const b200la_csr *A, const b200la_precond *P, int m, const void *b,
                            void *x, const b200la_control *ctl, b200la_result *res)
{
    NvtxScope nvtx_range("b200la_gmres");
    if (!ctx || !A || !b || !x || !ctl || A->n != A->m || m < 1)
        return ctx_fail(ctx, B200LA_ERR_ARG, "gmres: invalid argument", cudaSuccess);
    if (P && (P->dtype != A->dtype || P->n != A->n))
        return ctx_fail(ctx, B200LA_ERR_ARG, "gmres: preconditioner does not match the operator", cudaSuccess);
    const int n = A->n, dt = A->dtype;
    const int mb = std::max(1, std::min(m, ctl->maxits));   // gmres.cc:301
    const size_t es = dt == B200LA_F64 ? 8 : 4;
    const size_t ldv = ((es * std::max(n, 1) + 255) / 256) * 256;   // bytes per basis vector
    const size_t small = sizeof(double) * ((size_t)mb * (mb + 1) + 4 * (mb + 1) + 8);
    void *wk;
    int rc = ctx_work(ctx, ldv * (mb + 1 + 2) + small, &wk);
    if (rc) return rc;
    char *base = static_cast<char *>(wk);
    auto V = [&](int k) { return (void *)(base + ldv * k); };
    void *w = base + ldv * (mb + 1), *z = base + ldv * (mb + 2);
    double *sm = reinterpret_cast<double *>(base + ldv * (mb + 3));
    GmresDev d;
    d.H = sm;
    d.g = sm + (size_t)mb * (mb + 1);
    d.cs = d.g + (mb + 1);
    d.sn = d.cs + (mb + 1);
    d.y = d.sn + (mb + 1);
    d.jend = reinterpret_cast<int *>(d.y + (mb + 1));
    const int *gate = &ctx->st->status;
    const Scratch sc = ctx_scratch(ctx);
    const long long l0 = ctx->launches;
    const size_t ld_el = ldv / es;

    DevState *hs = ctx->st_host;
    state_init(*hs, ctl, nullptr, 0);
    SK(cudaMemcpyAsync(ctx->st, hs, sizeof(DevState), cudaMemcpyHostToDevice, ctx->stream));
    SK(cudaEventRecord(ctx->ev0, ctx->stream));
    // V0 = b - A x; res = ||V0||; Check(0)   (gmres.cc:323-335)
    SpmvOp op;
    op.epi = EPI_RESID;
    op.fin = FIN_RES_INIT;
    op.x = x;
    op.y = V(0);
    op.b = b;
    op.st = ctx->st;
    rc = spmv_run(ctx, A, A->all, op);
    if (rc) return rc;
    long long graph_launches = 0;
    for (;;) {
        SK(cudaMemcpyAsync(hs, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
        SK(cudaStreamSynchronize(ctx->stream));
        if (hs->status != kIterate) break;
        // one restart cycle: captured once, replayed per cycle
        auto cycle = [&]() -> int {
            gmres_cycle_kernel<<<1, 256, 0, ctx->stream>>>(mb, d, ctx->st);
            SK(cudaGetLastError());
            SK(launch_scale_dev(dt, n, d.g, true, V(0), V(0), nullptr, ctx->stream));
            ctx->launches += 2;
            for (int j = 0; j < mb; ++j) {
                const void *zin = V(j);
                if (P) {
                    int r2 = precond_apply_async(ctx, P, V(j), z, gate);
                    if (r2) return r2;
                    zin = z;
                }
                SpmvOp o;
                o.epi = EPI_SET;
                o.x = zin;
                o.y = w;
                o.gate = gate;
                int r2 = spmv_run(ctx, A, A->all, o);
                if (r2) return r2;
                // modified Gram-Schmidt (gmres.cc:373-377)
                for (int i = 0; i <= j; ++i) {
                    SK(launch_dot_to(sc, dt, n, w, V(i), d.H + (size_t)j * (mb + 1) + i, gate, ctx->stream));
                    SK(launch_axpy_dev(dt, n, d.H + (size_t)j * (mb + 1) + i, -1.0, V(i), w, gate, ctx->stream));
                    ctx->launches += 2;
                }
                // H(j, j+1) = ||w||; V_{j+1} = w / H(j, j+1)   (gmres.cc:379-383)
                SK(launch_dot_norm_to(sc, dt, n, w, d.H + (size_t)j * (mb + 1) + j + 1, gate, ctx->stream));
                SK(launch_scale_dev(dt, n, d.H + (size_t)j * (mb + 1) + j + 1, true, w, V(j + 1), gate, ctx->stream));
                gmres_givens_kernel<<<1, 1, 0, ctx->stream>>>(j, mb, d, ctx->st);
                SK(cudaGetLastError());
                ctx->launches += 3;
            }
            return B200LA_OK;
        };
        cudaGraphExec_t exec;
        int nodes = 0;
        rc = get_graph(ctx, {A, P, b, x, wk, (const void *)(intptr_t)mb, (const void *)(intptr_t)(-7), ctx->stream},
                       cycle, &exec, &nodes);
        if (rc) return rc;
        SK(cudaGraphLaunch(exec, ctx->stream));
        graph_launches += nodes;
        SK(cudaMemcpyAsync(hs, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
        int jend = mb - 1;
        SK(cudaMemcpyAsync(&ctx->hscal[8], d.jend, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        SK(cudaStreamSynchronize(ctx->stream));
        if (hs->status != kIterate) std::memcpy(&jend, &ctx->hscal[8], sizeof(int));
        // UpdateSolution + preconditioner + x += w   (gmres.cc:404-445)
        gmres_backsub_kernel<<<1, 1, 0, ctx->stream>>>(jend, mb, d);
        SK(cudaGetLastError());
        const int g = std::max(1, std::min((n + kBlock * 4 - 1) / (kBlock * 4), ctx->num_sms * 8));
        if (dt == B200LA_F64)
            lincomb_kernel<double><<<g, kBlock, 0, ctx->stream>>>(n, jend, (const double *)V(0), ld_el, d.y, (double *)z);
        else
            lincomb_kernel<float><<<g, kBlock, 0, ctx->stream>>>(n, jend, (const float *)V(0), ld_el, d.y, (float *)z);
        SK(cudaGetLastError());
        ctx->launches += 2;
        const void *corr = z;
        if (P) {
            rc = precond_apply_async(ctx, P, z, w, nullptr);
            if (rc) return rc;
            corr = w;
        }
        SK(launch_axpy(dt, n, 1.0, corr, x, ctx->stream));
        ctx->launches += 1;
        if (hs->status != kIterate) break;
        // restart residual (gmres.cc:433-436)
        SpmvOp o;
        o.epi = EPI_RESID;
        o.fin = FIN_NONE;
        o.x = x;
        o.y = V(0);
        o.b = b;
        rc = spmv_run(ctx, A, A->all, o);
        if (rc) return rc;
    }
    SK(cudaEventRecord(ctx->ev1, ctx->stream));
    SK(cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    SK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    rc = ctx_check_device_error(ctx);
    if (rc) return rc;
    if (res) {
        res->iters = hs->iter;
        res->status = hs->status;
        res->res0 = hs->res0;
        res->res = hs->res;
        res->outer = 0;
        res->launches = (int)(ctx->launches - l0 + graph_launches);
        res->solve_ms = ms;
    }
    ctx->launches += graph_launches;
    return B200LA_OK;
}
