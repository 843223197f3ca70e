// coupled.cu -- row-block operators over several ranks, one rank per GPU.
//
// The reference distributes a system by rows over MPI ranks: LaCouplings
// (src/linear_algebra/la_couplings.cc:62-230) lists, per rank, the ghost
// columns it reads (grouped by owner) and the border values every peer reads
// from it; CoupledVector::UpdateGhost packs the border and moves it with
// MPI_Isend / MPI_Irecv into the ghost buffer (coupled_vector.cc:975-1128);
// CoupledMatrix::VectorMult multiplies the diagonal block while the ghosts
// travel and then adds the off-diagonal block (coupled_matrix.cc:433-467);
// dots and norms end in MPI_Allreduce (coupled_vector.cc:331-436).
//
// Here the communicator is NCCL (loaded at run time, so the library has no
// link-time NCCL dependency and shares the process's NCCL when one is already
// loaded), or a local communicator for ranks that are threads of one process
// (device copies ordered by events, the host threads meeting at a barrier;
// no kernel ever waits for another rank).  Border packing is a gather kernel,
// the exchange runs on a second stream and overlaps the diagonal-block
// product, and the coupled CG (cg.cc:164-248 with block-Jacobi: Jacobi, or a
// multicolour / ILU preconditioner of each rank's diagonal block, as
// PreconditionerMultiColoring binds op.diagonal()) keeps its scalars on the device: the local partial
// sums are reduced across ranks by the communicator on the stream, and small
// kernels apply IterateControl::Check to the global values.  The host reads
// the stop state once per batch of iterations; every rank takes the same
// decisions from the same global values, so all ranks post the same
// collectives.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "b200la.h"
#include "b200la_internal.h"

using namespace b200;

#define CCK(call)                                                                        \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, #call, e_);        \
    } while (0)

static int cfail(b200la_ctx *ctx, int code, const std::string &m)
{
    if (ctx) ctx->msg = m;
    return code;
}

// ------------------------------------------------------------------ NCCL, loaded at run time

namespace {

struct NcclApi {
    ncclResult_t (*GetUniqueId)(ncclUniqueId *);
    ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int);
    ncclResult_t (*CommDestroy)(ncclComm_t);
    ncclResult_t (*GroupStart)();
    ncclResult_t (*GroupEnd)();
    ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
    ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
    ncclResult_t (*AllReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t, cudaStream_t);
    const char *(*GetErrorString)(ncclResult_t);
    bool ok = false;
};

// The process's NCCL (the one already loaded, e.g. by PyTorch, else the
// system's libnccl.so.2); null when none can be loaded.
const NcclApi *nccl()
{
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
        if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) return;
        auto sym = [&](const char *name) { return dlsym(h, name); };
        api.GetUniqueId = reinterpret_cast<decltype(api.GetUniqueId)>(sym("ncclGetUniqueId"));
        api.CommInitRank = reinterpret_cast<decltype(api.CommInitRank)>(sym("ncclCommInitRank"));
        api.CommDestroy = reinterpret_cast<decltype(api.CommDestroy)>(sym("ncclCommDestroy"));
        api.GroupStart = reinterpret_cast<decltype(api.GroupStart)>(sym("ncclGroupStart"));
        api.GroupEnd = reinterpret_cast<decltype(api.GroupEnd)>(sym("ncclGroupEnd"));
        api.Send = reinterpret_cast<decltype(api.Send)>(sym("ncclSend"));
        api.Recv = reinterpret_cast<decltype(api.Recv)>(sym("ncclRecv"));
        api.AllReduce = reinterpret_cast<decltype(api.AllReduce)>(sym("ncclAllReduce"));
        api.GetErrorString = reinterpret_cast<decltype(api.GetErrorString)>(sym("ncclGetErrorString"));
        api.ok = api.GetUniqueId && api.CommInitRank && api.CommDestroy && api.GroupStart && api.GroupEnd &&
                 api.Send && api.Recv && api.AllReduce && api.GetErrorString;
    });
    return api.ok ? &api : nullptr;
}

// ------------------------------------------------------------------ local ranks

// Host meeting point of the ranks of one process, with a time limit: a rank
// that never arrives turns into an error on the others, not a hang.
struct Fabric {
    int size;
    std::mutex mu;
    std::condition_variable cv;
    int arrived = 0;
    long long generation = 0;
    bool broken = false;
    // mailboxes, one slot per rank
    std::vector<const void *> border;       // rank's border buffer
    std::vector<const int *> border_off;    // rank's border offsets (host), nranks + 1
    std::vector<cudaEvent_t> ready;     // rank's last pack / contribution copy
    std::vector<cudaEvent_t> done;      // rank's last ghost copy / contribution sum
    std::vector<const double *> contrib;    // rank's all-reduce contribution (device)
    explicit Fabric(int n)
        : size(n), border(n), border_off(n), ready(n), done(n), contrib(n) {}

    bool barrier()
    {
        std::unique_lock<std::mutex> lk(mu);
        if (broken) return false;
        const long long gen = generation;
        if (++arrived == size) {
            arrived = 0;
            ++generation;
            cv.notify_all();
            return true;
        }
        const bool ok = cv.wait_for(lk, std::chrono::seconds(60), [&] { return generation != gen || broken; });
        if (!ok || broken) {
            broken = true;
            cv.notify_all();
            return false;
        }
        return true;
    }
};

}  // namespace

struct b200la_comm {
    int rank = 0, size = 1, kind = 0;   // kind 0 NCCL, 1 local
    int device = -1;
    ncclComm_t nc = nullptr;
    std::shared_ptr<Fabric> fab;
    cudaEvent_t ev_ready = nullptr, ev_summed = nullptr;
    double *contrib = nullptr;          // local all-reduce contribution (8 doubles)
};

struct b200la_coupled {
    b200la_comm *comm = nullptr;
    const b200la_csr *diag = nullptr, *offd = nullptr;
    int n = 0, n_ghost = 0, n_border = 0, dtype = 0;
    std::vector<int> ghost_off, border_off;   // nranks + 1 each
    int *border_idx = nullptr;                // device
    void *border = nullptr, *ghost = nullptr; // device buffers
    cudaStream_t xs = nullptr;                // exchange stream
    cudaEvent_t packed = nullptr, arrived = nullptr;
};

namespace {

constexpr int kMaxRed = 8;   // doubles per all-reduce

// dst[k] = sum over ranks of their contributions, in rank order
__global__ void sum_contrib_kernel(int nranks, const double *const *src, int count, double *dst)
{
    const int k = threadIdx.x;
    if (k >= count) return;
    double s = 0.0;
    for (int q = 0; q < nranks; ++q) s += src[q][k];   // every rank adds in rank order
    dst[k] = s;
}

// x += alpha p; r -= alpha Ap; local partials of ||r||^2 and r.(D^-1 r)
// (r.r without a preconditioner), skipped once the solver stopped
template <typename T>
__global__ void __launch_bounds__(kBlock) coupled_update_kernel(int n, int jac, T *__restrict__ x, T *__restrict__ r,
                                                                const T *__restrict__ p, const T *__restrict__ Ap,
                                                                const T *__restrict__ invd, DevState *st,
                                                                double *out, Scratch sc)
{
    if (gate_closed(&st->status)) return;
    const T alpha = (T)cta_scalar(&st->alpha);
    double rr = 0.0, rz = 0.0;
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        T xi = x[i], ri = r[i];
        xi += alpha * p[i];
        ri -= alpha * Ap[i];
        x[i] = xi;
        r[i] = ri;
        rr += (double)(ri * ri);
        rz += jac ? (double)(ri * (ri * invd[i])) : (double)(ri * ri);
    }
    double v[2] = {rr, rz}, o[2];
    if (grid_reduce<2>(v, sc.partials, sc.ticket, o)) {
        out[0] = o[0];
        out[1] = o[1];
    }
}

// z = M r (Jacobi or none), p = z, local rho and rr partials
template <typename T>
__global__ void __launch_bounds__(kBlock) coupled_start_kernel(int n, int jac, const T *__restrict__ r,
                                                               const T *__restrict__ invd, T *__restrict__ p,
                                                               double *out, Scratch sc)
{
    double rho = 0.0, rr = 0.0;
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        const T ri = r[i];
        const T zi = jac ? ri * invd[i] : ri;
        p[i] = zi;
        rho += (double)(ri * zi);
        rr += (double)(ri * ri);
    }
    double v[2] = {rho, rr}, o[2];
    if (grid_reduce<2>(v, sc.partials, sc.ticket, o)) {
        out[0] = o[0];
        out[1] = o[1];
    }
}

// p = z (a block preconditioner's output), local rho = r.z and rr partials
template <typename T>
__global__ void __launch_bounds__(kBlock) coupled_start_z_kernel(int n, const T *__restrict__ r,
                                                                 const T *__restrict__ z, T *__restrict__ p,
                                                                 double *out, Scratch sc)
{
    double rho = 0.0, rr = 0.0;
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        const T ri = r[i], zi = z[i];
        p[i] = zi;
        rho += (double)(ri * zi);
        rr += (double)(ri * ri);
    }
    double v[2] = {rho, rr}, o[2];
    if (grid_reduce<2>(v, sc.partials, sc.ticket, o)) {
        out[0] = o[0];
        out[1] = o[1];
    }
}

// beta = rz / rho; rho = rz after a block preconditioner's apply: g = {r.z} (global)
__global__ void coupled_beta_kernel(DevState *st, const double *g)
{
    if (st->status != kIterate) return;
    st->beta = g[0] / st->rho;
    st->rho = g[0];
}

// r = b - t
template <typename T>
__global__ void sub_kernel(int n, const T *__restrict__ b, const T *__restrict__ t, T *__restrict__ r)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) r[i] = b[i] - t[i];
}

// Check(0, ||r||) after the start reductions: g = {rho, rr} (global)
__global__ void coupled_start_check_kernel(DevState *st, const double *g)
{
    st->rho = g[0];
    st->rr = g[1];
    const double res = sqrt(g[1]);
    st->res = res;
    st->iter = 0;
    if (st->hist && st->hist_len > 0) st->hist[0] = res;
    st->status = check_state(st, 0, res);
}

// alpha = rho / (p . Ap), g = {p . Ap} (global)
__global__ void coupled_alpha_kernel(DevState *st, const double *g)
{
    if (st->status != kIterate) return;
    st->pap = g[0];
    st->alpha = st->rho / g[0];
}

// iteration count, residual, Check, and (with_beta) beta: g = {rr, rz} (global)
__global__ void coupled_check_kernel(DevState *st, const double *g, int with_beta)
{
    if (st->status != kIterate) return;
    const int it = st->iter + 1;
    st->iter = it;
    st->rr = g[0];
    const double res = sqrt(g[0]);
    st->res = res;
    if (st->hist && it < st->hist_len) st->hist[it] = res;
    const int s = check_state(st, it, res);
    st->status = s;
    if (s == kIterate && with_beta) {
        st->beta = g[1] / st->rho;
        st->rho = g[1];
    }
}

int grid_for(const b200la_ctx *ctx, int n)
{
    int g = (n + kBlock * 4 - 1) / (kBlock * 4);
    g = std::min(g, std::min(ctx->num_sms * 4, kMaxGrid));
    return std::max(g, 1);
}

size_t esize(int dtype) { return dtype == B200LA_F64 ? 8 : 4; }

}  // namespace

// ------------------------------------------------------------------ communicator

static int comm_allreduce(b200la_ctx *ctx, b200la_comm *c, double *dev, int count)
{
    if (count < 1 || count > kMaxRed) return cfail(ctx, B200LA_ERR_ARG, "allreduce: 1..8 values");
    if (c->kind == 0) {
        ncclResult_t r = nccl()->AllReduce(dev, dev, count, ncclFloat64, ncclSum, c->nc, ctx->stream);
        if (r != ncclSuccess) return cfail(ctx, B200LA_ERR_COMM, std::string("ncclAllReduce: ") + nccl()->GetErrorString(r));
        return B200LA_OK;
    }
    Fabric &f = *c->fab;
    // the contribution buffer is free again once every peer summed the last one
    CCK(cudaMemcpyAsync(c->contrib, dev, sizeof(double) * count, cudaMemcpyDeviceToDevice, ctx->stream));
    CCK(cudaEventRecord(c->ev_ready, ctx->stream));
    f.contrib[c->rank] = c->contrib;
    f.ready[c->rank] = c->ev_ready;
    if (!f.barrier()) return cfail(ctx, B200LA_ERR_COMM, "local all-reduce: a rank did not arrive");
    std::vector<const double *> src(f.size);
    for (int q = 0; q < f.size; ++q) {
        CCK(cudaStreamWaitEvent(ctx->stream, f.ready[q], 0));
        src[q] = f.contrib[q];
    }
    // the pointer table travels by value in a small device copy
    double **tab = reinterpret_cast<double **>(ctx->dscal + 128);
    CCK(cudaMemcpyAsync(tab, src.data(), sizeof(double *) * f.size, cudaMemcpyHostToDevice, ctx->stream));
    sum_contrib_kernel<<<1, 32, 0, ctx->stream>>>(f.size, tab, count, dev);
    CCK(cudaGetLastError());
    CCK(cudaEventRecord(c->ev_summed, ctx->stream));
    f.done[c->rank] = c->ev_summed;
    if (!f.barrier()) return cfail(ctx, B200LA_ERR_COMM, "local all-reduce: a rank did not arrive");
    for (int q = 0; q < f.size; ++q) CCK(cudaStreamWaitEvent(ctx->stream, f.done[q], 0));
    // nobody records its events again before every rank has queued its waits
    if (!f.barrier()) return cfail(ctx, B200LA_ERR_COMM, "local all-reduce: a rank did not arrive");
    return B200LA_OK;
}

extern "C" int b200la_comm_unique_id(void *id)
{
    if (!id) return B200LA_ERR_ARG;
    const NcclApi *api = nccl();
    if (!api) return B200LA_ERR_COMM;
    ncclUniqueId u;
    if (api->GetUniqueId(&u) != ncclSuccess) return B200LA_ERR_COMM;
    static_assert(sizeof(ncclUniqueId) == B200LA_COMM_ID_BYTES, "NCCL unique id size");
    std::memcpy(id, &u, sizeof u);
    return B200LA_OK;
}

extern "C" int b200la_comm_create_nccl(b200la_ctx *ctx, const void *id, int rank, int nranks, b200la_comm **out)
{
    if (!ctx || !id || !out || nranks < 1 || rank < 0 || rank >= nranks)
        return cfail(ctx, B200LA_ERR_ARG, "comm_create_nccl: invalid argument");
    const NcclApi *api = nccl();
    if (!api) return cfail(ctx, B200LA_ERR_COMM, "comm_create_nccl: libnccl.so.2 could not be loaded");
    CCK(cudaSetDevice(ctx->device));
    ncclUniqueId u;
    std::memcpy(&u, id, sizeof u);
    ncclComm_t nc = nullptr;
    const ncclResult_t r = api->CommInitRank(&nc, nranks, u, rank);
    if (r != ncclSuccess) return cfail(ctx, B200LA_ERR_COMM, std::string("ncclCommInitRank: ") + api->GetErrorString(r));
    b200la_comm *c = new b200la_comm();
    c->rank = rank;
    c->size = nranks;
    c->kind = 0;
    c->device = ctx->device;
    c->nc = nc;
    *out = c;
    return B200LA_OK;
}

extern "C" int b200la_comm_create_local(int nranks, b200la_comm **out)
{
    if (nranks < 1 || !out) return B200LA_ERR_ARG;
    auto fab = std::make_shared<Fabric>(nranks);
    for (int q = 0; q < nranks; ++q) {
        b200la_comm *c = new b200la_comm();
        c->rank = q;
        c->size = nranks;
        c->kind = 1;
        c->fab = fab;
        out[q] = c;
    }
    return B200LA_OK;
}

// Device resources of a local communicator, made on the rank's own device at
// first use (the ranks' threads may drive different GPUs).
static int comm_local_setup(b200la_ctx *ctx, b200la_comm *c)
{
    if (c->kind != 1 || c->contrib) return B200LA_OK;
    c->device = ctx->device;
    CCK(cudaEventCreateWithFlags(&c->ev_ready, cudaEventDisableTiming));
    CCK(cudaEventCreateWithFlags(&c->ev_summed, cudaEventDisableTiming));
    CCK(cudaMalloc(&c->contrib, sizeof(double) * kMaxRed));
    return B200LA_OK;
}

extern "C" int b200la_comm_info(const b200la_comm *c, int *rank, int *nranks)
{
    if (!c) return B200LA_ERR_ARG;
    if (rank) *rank = c->rank;
    if (nranks) *nranks = c->size;
    return B200LA_OK;
}

extern "C" int b200la_comm_destroy(b200la_comm *c)
{
    if (!c) return B200LA_OK;
    if (c->device >= 0) cudaSetDevice(c->device);
    cudaDeviceSynchronize();
    if (c->nc && nccl()) nccl()->CommDestroy(c->nc);
    if (c->ev_ready) cudaEventDestroy(c->ev_ready);
    if (c->ev_summed) cudaEventDestroy(c->ev_summed);
    if (c->contrib) cudaFree(c->contrib);
    delete c;
    return B200LA_OK;
}

// ------------------------------------------------------------------ couplings and operator

extern "C" int b200la_coupled_create(b200la_ctx *ctx, b200la_comm *comm, const b200la_csr *diag,
                                     const b200la_csr *offdiag, const int *ghost_offsets, const int *border_offsets,
                                     const int *border_indices, b200la_coupled **out)
{
    if (!ctx || !comm || !diag || !ghost_offsets || !border_offsets || !out || diag->n != diag->m)
        return cfail(ctx, B200LA_ERR_ARG, "coupled_create: invalid argument");
    const int P = comm->size;
    const int n_ghost = ghost_offsets[P], n_border = border_offsets[P];
    if (ghost_offsets[0] != 0 || border_offsets[0] != 0 || n_ghost < 0 || n_border < 0 ||
        (n_border > 0 && !border_indices))
        return cfail(ctx, B200LA_ERR_ARG, "coupled_create: offsets must start at 0");
    for (int q = 0; q < P; ++q)
        if (ghost_offsets[q + 1] < ghost_offsets[q] || border_offsets[q + 1] < border_offsets[q] ||
            (q == comm->rank && (ghost_offsets[q + 1] != ghost_offsets[q] || border_offsets[q + 1] != border_offsets[q])))
            return cfail(ctx, B200LA_ERR_ARG, "coupled_create: offsets must ascend, none towards this rank");
    for (int k = 0; k < n_border; ++k)
        if (border_indices[k] < 0 || border_indices[k] >= diag->n)
            return cfail(ctx, B200LA_ERR_ARG, "coupled_create: border index outside the owned rows");
    if (n_ghost > 0 && (!offdiag || offdiag->n != diag->n || offdiag->m != n_ghost || offdiag->dtype != diag->dtype))
        return cfail(ctx, B200LA_ERR_ARG, "coupled_create: off-diagonal block must be n x n_ghost of the same dtype");
    int rc = comm_local_setup(ctx, comm);
    if (rc) return rc;
    b200la_coupled *M = new b200la_coupled();
    M->comm = comm;
    M->diag = diag;
    M->offd = n_ghost > 0 ? offdiag : nullptr;
    M->n = diag->n;
    M->n_ghost = n_ghost;
    M->n_border = n_border;
    M->dtype = diag->dtype;
    M->ghost_off.assign(ghost_offsets, ghost_offsets + P + 1);
    M->border_off.assign(border_offsets, border_offsets + P + 1);
    const size_t es = esize(M->dtype);
    cudaError_t e;
    if ((e = cudaMalloc(&M->border_idx, sizeof(int) * std::max(n_border, 1))) ||
        (e = cudaMalloc(&M->border, es * std::max(n_border, 1))) ||
        (e = cudaMalloc(&M->ghost, es * std::max(n_ghost, 1))) ||
        (n_border && (e = cudaMemcpy(M->border_idx, border_indices, sizeof(int) * n_border, cudaMemcpyHostToDevice))) ||
        (e = cudaMemset(M->ghost, 0, es * std::max(n_ghost, 1))) ||
        (e = cudaStreamCreateWithFlags(&M->xs, cudaStreamNonBlocking)) ||
        (e = cudaEventCreateWithFlags(&M->packed, cudaEventDisableTiming)) ||
        (e = cudaEventCreateWithFlags(&M->arrived, cudaEventDisableTiming))) {
        b200la_coupled_destroy(M);
        return ctx_fail(ctx, B200LA_ERR_ALLOC, "coupled_create", e);
    }
    *out = M;
    return B200LA_OK;
}

extern "C" int b200la_coupled_destroy(b200la_coupled *M)
{
    if (!M) return B200LA_OK;
    cudaDeviceSynchronize();
    if (M->border_idx) cudaFree(M->border_idx);
    if (M->border) cudaFree(M->border);
    if (M->ghost) cudaFree(M->ghost);
    if (M->xs) cudaStreamDestroy(M->xs);
    if (M->packed) cudaEventDestroy(M->packed);
    if (M->arrived) cudaEventDestroy(M->arrived);
    delete M;
    return B200LA_OK;
}

// Pack the border of x and start its exchange on the exchange stream; the
// ghosts are in place once the context's stream has waited on M->arrived.
static int exchange_begin(b200la_ctx *ctx, b200la_coupled *M, const void *x)
{
    b200la_comm *c = M->comm;
    if (M->n_border) {
        CCK(launch_gather(M->dtype, M->n_border, M->border_idx, x, M->border, ctx->stream));
        ctx->launches += 1;
    }
    CCK(cudaEventRecord(M->packed, ctx->stream));
    CCK(cudaStreamWaitEvent(M->xs, M->packed, 0));
    const size_t es = esize(M->dtype);
    const int P = c->size;
    if (c->kind == 0) {
        const NcclApi *api = nccl();
        const ncclDataType_t t = M->dtype == B200LA_F64 ? ncclFloat64 : ncclFloat32;
        ncclResult_t r = api->GroupStart();
        for (int q = 0; q < P && r == ncclSuccess; ++q) {
            const int nb = M->border_off[q + 1] - M->border_off[q], ng = M->ghost_off[q + 1] - M->ghost_off[q];
            if (nb) r = api->Send(static_cast<char *>(M->border) + es * M->border_off[q], nb, t, q, c->nc, M->xs);
            if (ng && r == ncclSuccess)
                r = api->Recv(static_cast<char *>(M->ghost) + es * M->ghost_off[q], ng, t, q, c->nc, M->xs);
        }
        const ncclResult_t r2 = api->GroupEnd();
        if (r != ncclSuccess || r2 != ncclSuccess)
            return cfail(ctx, B200LA_ERR_COMM, std::string("ghost exchange: ") +
                                                   api->GetErrorString(r != ncclSuccess ? r : r2));
        CCK(cudaEventRecord(M->arrived, M->xs));
        return B200LA_OK;
    }
    // local ranks: every receiver copies from its owners' border buffers
    Fabric &f = *c->fab;
    f.border[c->rank] = M->border;
    f.border_off[c->rank] = M->border_off.data();
    f.ready[c->rank] = M->packed;
    if (!f.barrier()) return cfail(ctx, B200LA_ERR_COMM, "ghost exchange: a rank did not arrive");
    for (int q = 0; q < P; ++q) {
        const int ng = M->ghost_off[q + 1] - M->ghost_off[q];
        if (!ng) continue;
        CCK(cudaStreamWaitEvent(M->xs, f.ready[q], 0));
        const char *src = static_cast<const char *>(f.border[q]) + es * f.border_off[q][c->rank];
        CCK(cudaMemcpyAsync(static_cast<char *>(M->ghost) + es * M->ghost_off[q], src, es * ng,
                            cudaMemcpyDeviceToDevice, M->xs));
    }
    CCK(cudaEventRecord(M->arrived, M->xs));
    f.done[c->rank] = M->arrived;
    if (!f.barrier()) return cfail(ctx, B200LA_ERR_COMM, "ghost exchange: a rank did not arrive");
    // the border is packed again only after every reader has copied it
    for (int q = 0; q < P; ++q)
        if (M->border_off[q + 1] > M->border_off[q]) CCK(cudaStreamWaitEvent(ctx->stream, f.done[q], 0));
    if (!f.barrier()) return cfail(ctx, B200LA_ERR_COMM, "ghost exchange: a rank did not arrive");
    return B200LA_OK;
}

static int exchange_end(b200la_ctx *ctx, b200la_coupled *M)
{
    CCK(cudaStreamWaitEvent(ctx->stream, M->arrived, 0));
    return B200LA_OK;
}

// y = A x over the coupled rows (diagonal block while the ghosts travel)
static int coupled_spmv_async(b200la_ctx *ctx, b200la_coupled *M, const void *x, void *y)
{
    int rc = exchange_begin(ctx, M, x);
    if (rc) return rc;
    SpmvOp op;
    op.epi = EPI_SET;
    op.x = x;
    op.y = y;
    if ((rc = spmv_run(ctx, M->diag, M->diag->all, op))) return rc;
    if ((rc = exchange_end(ctx, M))) return rc;
    if (M->offd) {
        SpmvOp o;
        o.epi = EPI_ADD;
        o.x = M->ghost;
        o.y = y;
        if ((rc = spmv_run(ctx, M->offd, M->offd->all, o))) return rc;
    }
    return B200LA_OK;
}

extern "C" int b200la_coupled_update_ghost(b200la_ctx *ctx, b200la_coupled *M, const void *x, void *ghost)
{
    if (!ctx || !M || !x) return cfail(ctx, B200LA_ERR_ARG, "coupled_update_ghost: invalid argument");
    int rc = exchange_begin(ctx, M, x);
    if (!rc) rc = exchange_end(ctx, M);
    if (!rc && ghost && M->n_ghost)
        CCK(cudaMemcpyAsync(ghost, M->ghost, esize(M->dtype) * M->n_ghost, cudaMemcpyDeviceToDevice, ctx->stream));
    if (!rc) CCK(cudaStreamSynchronize(ctx->stream));
    return rc;
}

extern "C" int b200la_coupled_spmv(b200la_ctx *ctx, b200la_coupled *M, const void *x, void *y)
{
    if (!ctx || !M || !x || !y || x == y) return cfail(ctx, B200LA_ERR_ARG, "coupled_spmv: invalid argument");
    return coupled_spmv_async(ctx, M, x, y);
}

extern "C" int b200la_coupled_dot(b200la_ctx *ctx, b200la_coupled *M, const void *x, const void *y, double *out)
{
    if (!ctx || !M || !x || !y || !out) return cfail(ctx, B200LA_ERR_ARG, "coupled_dot: invalid argument");
    CCK(launch_dot_to(ctx_scratch(ctx), M->dtype, M->n, x, y, ctx->dscal, nullptr, ctx->stream));
    ctx->launches += 1;
    int rc = comm_allreduce(ctx, M->comm, ctx->dscal, 1);
    if (rc) return rc;
    CCK(cudaMemcpyAsync(ctx->hscal, ctx->dscal, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CCK(cudaStreamSynchronize(ctx->stream));
    *out = ctx->hscal[0];
    return B200LA_OK;
}

// ------------------------------------------------------------------ coupled CG

extern "C" int b200la_coupled_cg(b200la_ctx *ctx, b200la_coupled *M, const b200la_precond *P, const void *b,
                                 void *x, const b200la_control *ctl, b200la_result *res)
{
    NvtxScope nvtx_range("b200la_coupled_cg");
    if (!ctx || !M || !b || !x || !ctl || ctl->maxits < 0)
        return cfail(ctx, B200LA_ERR_ARG, "coupled_cg: invalid argument");
    if (P && (P->n != M->n || P->dtype != M->dtype || (P->kind != B200LA_PRECOND_JACOBI && !P->perm_dev)))
        return cfail(ctx, B200LA_ERR_ARG,
                     "coupled_cg: the preconditioner must be built on this rank's diagonal block");
    // 0 none, 1 Jacobi (fused into the update), 2 a block preconditioner in
    // its own numbering: r gathered into it, applied, z scattered back
    const int pk = !P ? 0 : (P->kind == B200LA_PRECOND_JACOBI ? 1 : 2);
    const int n = M->n, dt = M->dtype, jac = pk == 1 ? 1 : 0;
    const void *invd = pk == 1 ? P->invd : nullptr;
    const size_t vb = ((esize(dt) * std::max(n, 1) + 255) / 256) * 256;
    void *wk;
    int rc = ctx_work(ctx, (pk == 2 ? 6 : 3) * vb, &wk);
    if (rc) return rc;
    char *base = static_cast<char *>(wk);
    void *r = base, *p = base + vb, *Ap = base + 2 * vb;
    void *z = base + 3 * vb, *rp = base + 4 * vb, *zp = base + 5 * vb;
    // z = P^T M^-1 P r on this rank's block (PreconditionerMultiColoring on op.diagonal())
    auto block_apply = [&](const int *gate) -> int {
        CCK(launch_gather(dt, n, P->perm_dev, r, rp, ctx->stream));
        int r2 = precond_apply_async(ctx, P, rp, zp, gate);
        if (r2) return r2;
        CCK(launch_scatter(dt, n, P->perm_dev, zp, z, ctx->stream));
        ctx->launches += 2;
        return B200LA_OK;
    };
    const Scratch sc = ctx_scratch(ctx);
    const int g = grid_for(ctx, n);
    double *red = ctx->dscal;      // [0..1] reductions
    const long long l0 = ctx->launches;

    DevState *hs = ctx->st_host;
    std::memset(hs, 0, sizeof(DevState));
    hs->maxits = ctl->maxits;
    hs->abstol = ctl->abstol;
    hs->reltol = ctl->reltol;
    hs->divtol = ctl->divtol;
    hs->status = kIterate;
    CCK(cudaMemcpyAsync(ctx->st, hs, sizeof(DevState), cudaMemcpyHostToDevice, ctx->stream));
    CCK(cudaEventRecord(ctx->ev0, ctx->stream));

    // r = b - A x; z = M r; p = z; rho = r.z; res = ||r||; Check(0)   (cg.cc:200-214)
    if ((rc = coupled_spmv_async(ctx, M, x, Ap))) return rc;
    if (dt == B200LA_F64) sub_kernel<double><<<g, kBlock, 0, ctx->stream>>>(n, (const double *)b, (const double *)Ap, (double *)r);
    else sub_kernel<float><<<g, kBlock, 0, ctx->stream>>>(n, (const float *)b, (const float *)Ap, (float *)r);
    CCK(cudaGetLastError());
    if (pk == 2) {
        if ((rc = block_apply(nullptr))) return rc;
        if (dt == B200LA_F64)
            coupled_start_z_kernel<double><<<g, kBlock, 0, ctx->stream>>>(n, (const double *)r, (const double *)z,
                                                                           (double *)p, red, sc);
        else
            coupled_start_z_kernel<float><<<g, kBlock, 0, ctx->stream>>>(n, (const float *)r, (const float *)z,
                                                                          (float *)p, red, sc);
    } else if (dt == B200LA_F64) {
        coupled_start_kernel<double><<<g, kBlock, 0, ctx->stream>>>(n, jac, (const double *)r, (const double *)invd,
                                                                     (double *)p, red, sc);
    } else {
        coupled_start_kernel<float><<<g, kBlock, 0, ctx->stream>>>(n, jac, (const float *)r, (const float *)invd,
                                                                    (float *)p, red, sc);
    }
    CCK(cudaGetLastError());
    ctx->launches += 2;
    if ((rc = comm_allreduce(ctx, M->comm, red, 2))) return rc;
    coupled_start_check_kernel<<<1, 1, 0, ctx->stream>>>(ctx->st, red);
    CCK(cudaGetLastError());
    ctx->launches += 1;

    auto iteration = [&]() -> int {
        // Ap = A p; alpha = rho / (p . Ap)                     (cg.cc:219-220)
        int r2 = coupled_spmv_async(ctx, M, p, Ap);
        if (r2) return r2;
        CCK(launch_dot_to(sc, dt, n, p, Ap, red, &ctx->st->status, ctx->stream));
        if ((r2 = comm_allreduce(ctx, M->comm, red, 1))) return r2;
        coupled_alpha_kernel<<<1, 1, 0, ctx->stream>>>(ctx->st, red);
        // x += alpha p; r -= alpha Ap; ||r||, r.z; Check; beta (cg.cc:221-240)
        if (dt == B200LA_F64)
            coupled_update_kernel<double><<<g, kBlock, 0, ctx->stream>>>(
                n, jac, (double *)x, (double *)r, (const double *)p, (const double *)Ap, (const double *)invd,
                ctx->st, red, sc);
        else
            coupled_update_kernel<float><<<g, kBlock, 0, ctx->stream>>>(n, jac, (float *)x, (float *)r,
                                                                        (const float *)p, (const float *)Ap,
                                                                        (const float *)invd, ctx->st, red, sc);
        CCK(cudaGetLastError());
        if ((r2 = comm_allreduce(ctx, M->comm, red, 2))) return r2;
        coupled_check_kernel<<<1, 1, 0, ctx->stream>>>(ctx->st, red, pk == 2 ? 0 : 1);
        if (pk == 2) {
            // z = M^-1 r on the block; rho = r.z across ranks; beta   (cg.cc:236-240)
            if ((r2 = block_apply(&ctx->st->status))) return r2;
            CCK(launch_dot_to(sc, dt, n, r, z, red, &ctx->st->status, ctx->stream));
            if ((r2 = comm_allreduce(ctx, M->comm, red, 1))) return r2;
            coupled_beta_kernel<<<1, 1, 0, ctx->stream>>>(ctx->st, red);
            ctx->launches += 2;
        }
        // p = beta p + z                                        (cg.cc:241)
        CCK(launch_cg_pupdate(dt, n, pk == 2 ? 2 : jac, p, r, invd, pk == 2 ? z : nullptr, ctx->st, ctx->stream));
        ctx->launches += 5;
        return B200LA_OK;
    };

    // batches of iterations; the host reads the (global) stop state after each
    const int K = 8;
    const long long max_batches = (long long)ctl->maxits / K + 2;
    CCK(cudaMemcpyAsync(hs, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
    CCK(cudaStreamSynchronize(ctx->stream));
    for (long long bt = 0; hs->status == kIterate && bt < max_batches; ++bt) {
        for (int k = 0; k < K; ++k)
            if ((rc = iteration())) return rc;
        CCK(cudaMemcpyAsync(hs, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
        CCK(cudaStreamSynchronize(ctx->stream));
    }
    CCK(cudaEventRecord(ctx->ev1, ctx->stream));
    CCK(cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    CCK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    rc = ctx_check_device_error(ctx);
    if (rc) return rc;
    if (res) {
        res->iters = hs->iter;
        res->status = hs->status;
        res->res0 = hs->res0;
        res->res = hs->res;
        res->outer = 0;
        res->launches = (int)(ctx->launches - l0);
        res->solve_ms = ms;
    }
    return B200LA_OK;
}
