// sweeps.cu -- diagonal kernels and the sync-free level-scheduled sweep.
//
// A level-scheduled triangular solve (lmp/lmatrix_csr_cpu.cc:2295-2392 gives
// the levels; lmp/lpreconditioner_mc_ilup.cc:208-262 the forward / backward
// recurrences) has as many dependent steps as levels -- about 1.5 thousand
// for a 512^2 Q1 grid -- with a few hundred rows each.  One launch per level
// would spend the solve in launch latency, so each sweep is ONE persistent
// launch: warps take chunks of rows in level order from an atomic ticket; a
// chunk never spans two levels, so its rows are independent of one another,
// and every row it depends on belongs to an earlier ticket that a running warp
// already holds.  A row waits (acquire loads, bounded) until the rows it reads
// are published, computes, stores, and publishes itself (release store of the
// sweep's epoch).  Epochs advance by two per apply, so flags never need
// clearing.
#include "b200la.h"
#include "b200la_internal.h"

#include <algorithm>
#include <cstdlib>
#include <string>
#include <vector>

using namespace b200;

namespace {

constexpr long long kFlagSpin = 1LL << 22;

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(unsigned *p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <typename T>
__global__ void invdiag_kernel(int n, const int *__restrict__ row, const int *__restrict__ col,
                               const T *__restrict__ val, T *__restrict__ out)
{
    // extract_invdiagelements (lmp/lmatrix_csr_cpu.cc:2414-2431)
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        T d = T(0);
        for (int j = row[i]; j < row[i + 1]; ++j)
            if (col[j] == i) d = val[j];
        out[i] = T(1) / d;
    }
}

template <typename T>
__global__ void jacobi_kernel(int n, const T *__restrict__ invd, const T *__restrict__ r, T *__restrict__ z,
                              const int *gate)
{
    if (gate_closed(gate)) return;
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) z[i] = r[i] * invd[i];
}

struct SyncFreeArgs {
    const int *row, *col;
    const void *val;
    const int2 *chunks;   // {first row, row count}, in dependency order
    int nchunks;
    int lg;               // log2 lanes per row
    const void *r;        // forward: the input
    void *z;              // output (in place)
    const void *d1, *d2;
    unsigned *flags;      // per-row published epoch
    unsigned *sync;       // [epoch base, fwd ticket, bwd ticket, done counter]
    int backward;         // 0 forward, 1 backward
    int sgs;              // 1 MC-SGS recurrences, 0 ILU
    const int *gate;
    int *err;
};

template <typename T>
__global__ void __launch_bounds__(kBlock) syncfree_sweep_kernel(SyncFreeArgs a)
{
    if (gate_closed(a.gate)) return;
    __shared__ unsigned s_epoch;
    if (threadIdx.x == 0) s_epoch = __ldcg(a.sync) + (a.backward ? 2u : 1u);
    __syncthreads();
    const unsigned epoch = s_epoch;
    unsigned *ticket = a.sync + 1 + a.backward;
    const int lane = threadIdx.x & 31;
    const int G = 1 << a.lg;
    const int grp = lane >> a.lg, lg_lane = lane & (G - 1);
    const T *__restrict__ val = static_cast<const T *>(a.val);
    T *z = static_cast<T *>(a.z);
    const T *r = static_cast<const T *>(a.r);
    const T *d1 = static_cast<const T *>(a.d1);
    const T *d2 = static_cast<const T *>(a.d2);
    bool timed_out = false;
    for (;;) {
        int c = 0;
        if (lane == 0) c = (int)atomicAdd(ticket, 1u);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (c >= a.nchunks) break;
        const int2 ch = a.chunks[c];
        const bool active = grp < ch.y;
        const int rr = ch.x + grp;
        T s = T(0);
        if (active) {
            const int j1 = __ldg(a.row + rr + 1);
            for (int j = __ldg(a.row + rr) + lg_lane; j < j1; j += G) {
                const int cc = __ldg(a.col + j);
                long long spin = 0;
                while (ld_acquire(a.flags + cc) != epoch) {
                    // give up (and make every other waiter give up) after a bound
                    if (++spin > kFlagSpin || ((spin & 1023) == 0 && *reinterpret_cast<volatile int *>(a.err))) {
                        timed_out = true;
                        break;
                    }
                }
                s += __ldg(val + j) * __ldcg(z + cc);
            }
        }
        for (int o = G >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (active && lg_lane == 0) {
            T out;
            if (!a.backward) out = a.sgs ? (-r[rr] + s) * d1[rr] : -(-r[rr] + s);
            else out = a.sgs ? (__ldcg(z + rr) * d2[rr] + s) * d1[rr] : (-__ldcg(z + rr) + s) * d1[rr];
            __stcg(z + rr, out);
            st_release(a.flags + rr, epoch);
        }
    }
    if (timed_out) atomicExch(a.err, kDevWaitTimeout);
    // the last block resets the ticket (and advances the epoch after the backward sweep)
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned t = atomicAdd(a.sync + 3, 1u);
        if (t == gridDim.x - 1) {
            a.sync[1 + a.backward] = 0u;
            a.sync[3] = 0u;
            if (a.backward) a.sync[0] = a.sync[0] + 2u;
            __threadfence();
        }
    }
}

}  // namespace

namespace b200 {

cudaError_t sweeps_configure() { return cudaSuccess; }

cudaError_t launch_invdiag(int dtype, int n, const int *row, const int *col, const void *val, void *out,
                           cudaStream_t st)
{
    const int g = std::max(1, std::min((n + kBlock - 1) / kBlock, 148 * 8));
    if (dtype == B200LA_F64)
        invdiag_kernel<double><<<g, kBlock, 0, st>>>(n, row, col, (const double *)val, (double *)out);
    else
        invdiag_kernel<float><<<g, kBlock, 0, st>>>(n, row, col, (const float *)val, (float *)out);
    return cudaGetLastError();
}

cudaError_t launch_jacobi(int dtype, int n, const void *invd, const void *r, void *z, const int *gate,
                          cudaStream_t st)
{
    const int g = std::max(1, std::min((n + kBlock * 4 - 1) / (kBlock * 4), 148 * 8));
    if (dtype == B200LA_F64)
        jacobi_kernel<double><<<g, kBlock, 0, st>>>(n, (const double *)invd, (const double *)r, (double *)z, gate);
    else
        jacobi_kernel<float><<<g, kBlock, 0, st>>>(n, (const float *)invd, (const float *)r, (float *)z, gate);
    return cudaGetLastError();
}

}  // namespace b200

// Host side: chunk lists and launches.

struct SyncFreePlan {
    int2 *fwd = nullptr, *bwd = nullptr;
    int nf = 0, nb = 0;
    int lg_l = 0, lg_u = 0;
};

static int lanes_for(const b200la_csr *M)
{
    const double mean = M->n ? (double)M->nnz / M->n : 0.0;
    int lg = 0;
    while (lg < 5 && (double)(1 << lg) < mean) ++lg;
    return lg;
}

int syncfree_setup(b200la_ctx *ctx, b200la_precond *P)
{
    const char *env = std::getenv("B200LA_SYNCFREE");
    bool use = P->nblocks > 64;
    if (env) use = std::atoi(env) != 0;
    if (!use) return B200LA_OK;
    const int lgL = lanes_for(P->L), lgU = lanes_for(P->U);
    // chunks of at most 32 >> lg rows, never crossing a block (level) boundary
    auto chunks = [&](int lg, bool reverse) {
        std::vector<int2> out;
        const int per = 32 >> lg;
        for (int k = 0; k < P->nblocks; ++k) {
            const int b = reverse ? P->nblocks - 1 - k : k;
            for (int r = P->block_off[b]; r < P->block_off[b + 1]; r += per)
                out.push_back(make_int2(r, std::min(per, P->block_off[b + 1] - r)));
        }
        return out;
    };
    std::vector<int2> f = chunks(lgL, false), bw = chunks(lgU, true);
    SyncFreePlan *plan = new SyncFreePlan();
    plan->nf = (int)f.size();
    plan->nb = (int)bw.size();
    plan->lg_l = lgL;
    plan->lg_u = lgU;
    cudaError_t e;
    if ((e = cudaMalloc(&plan->fwd, sizeof(int2) * f.size())) || (e = cudaMalloc(&plan->bwd, sizeof(int2) * bw.size())) ||
        (e = cudaMemcpy(plan->fwd, f.data(), sizeof(int2) * f.size(), cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(plan->bwd, bw.data(), sizeof(int2) * bw.size(), cudaMemcpyHostToDevice)) ||
        (e = cudaMalloc(&P->flags, sizeof(unsigned) * P->n)) || (e = cudaMemset(P->flags, 0, sizeof(unsigned) * P->n)) ||
        (e = cudaMalloc(&P->sync, sizeof(unsigned) * 4)) || (e = cudaMemset(P->sync, 0, sizeof(unsigned) * 4))) {
        if (plan->fwd) cudaFree(plan->fwd);
        if (plan->bwd) cudaFree(plan->bwd);
        delete plan;
        return ctx_fail(ctx, B200LA_ERR_ALLOC, "syncfree setup", e);
    }
    P->syncfree_plan = plan;
    P->use_syncfree = 1;
    return B200LA_OK;
}

void syncfree_free(b200la_precond *P)
{
    SyncFreePlan *plan = static_cast<SyncFreePlan *>(P->syncfree_plan);
    if (!plan) return;
    cudaFree(plan->fwd);
    cudaFree(plan->bwd);
    delete plan;
    P->syncfree_plan = nullptr;
}

int syncfree_apply(b200la_ctx *ctx, const b200la_precond *P, const void *r, void *z, const int *gate)
{
    const SyncFreePlan *plan = static_cast<const SyncFreePlan *>(P->syncfree_plan);
    SyncFreeArgs a;
    a.r = r;
    a.z = z;
    a.d1 = P->iDv;
    a.d2 = P->Dv;
    a.flags = P->flags;
    a.sync = P->sync;
    a.sgs = P->kind == B200LA_PRECOND_MCSGS;
    a.gate = gate;
    a.err = ctx->dev_err;
    const int grid = ctx->num_sms * 4;
    for (int dir = 0; dir < 2; ++dir) {
        const b200la_csr *M = dir ? P->U : P->L;
        a.row = M->row;
        a.col = M->col;
        a.val = M->val;
        a.chunks = dir ? plan->bwd : plan->fwd;
        a.nchunks = dir ? plan->nb : plan->nf;
        a.lg = dir ? plan->lg_u : plan->lg_l;
        a.backward = dir;
        if (P->dtype == B200LA_F64)
            syncfree_sweep_kernel<double><<<grid, kBlock, 0, ctx->stream>>>(a);
        else
            syncfree_sweep_kernel<float><<<grid, kBlock, 0, ctx->stream>>>(a);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "syncfree sweep", e);
        ctx->launches += 1;
    }
    return B200LA_OK;
}
