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
#include <cstring>
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

// Level sweep in one CTA, for operators with many small levels (the
// level-scheduled ILU(0) of a 2-D grid: ~1,500 levels of ~200 rows).  The
// levels are taken in dependency order, each level's rows by the CTA's 512
// threads, a CTA barrier between levels: no flags, no waits.  The most
// recently solved kLevelRing rows stay in a shared-memory ring, so the
// dependency gathers of a row (on the last few levels) come from shared
// memory; older columns are read from L2.  Forward: rows ascend, a column cc
// of the current level [r0, r1) is in the ring when cc >= r1 - ring (slots of
// rows >= r0 - ring are being rewritten by this level).  Backward: rows
// descend, cc is in the ring when cc < r0 + ring.
constexpr int kLevelRing = 8192;
constexpr int kLevelThreads = 512;
constexpr int kLevelMaxLevels = 24576;   // level offsets kept in shared memory

struct LevelSweepArgs {
    const int *row, *col;
    const void *val;
    const int *off;       // level offsets [nlev + 1] (rows of level l: [off[l], off[l+1]))
    int nlev;
    const void *r;
    void *z;
    const void *d1, *d2;
    int backward, sgs;
    const int *gate;
};

// Row data of one thread in one level, loaded ahead of the level (up to
// kLevelPre entries in registers; longer rows read the rest directly).
constexpr int kLevelPre = 8;
template <typename T>
struct LevelRow {
    int rr, j0, j1;
    int c[kLevelPre];
    T v[kLevelPre];
    T own, e1, e2;   // r_i (forward) or z_i (backward), d1_i, d2_i
};

template <typename T>
__global__ void __launch_bounds__(kLevelThreads) level_sweep_cta_kernel(LevelSweepArgs a)
{
    extern __shared__ __align__(16) unsigned char s_raw[];
    T *ring = reinterpret_cast<T *>(s_raw);
    int *s_off = reinterpret_cast<int *>(s_raw + kLevelRing * sizeof(T));
    if (gate_closed(a.gate)) return;
    for (int i = threadIdx.x; i <= a.nlev; i += kLevelThreads) {
        s_off[i] = __ldg(a.off + i);
    }
    __syncthreads();
    const T *__restrict__ val = static_cast<const T *>(a.val);
    const T *__restrict__ r = static_cast<const T *>(a.r);
    const T *__restrict__ d1 = static_cast<const T *>(a.d1);
    const T *__restrict__ d2 = static_cast<const T *>(a.d2);
    T *z = static_cast<T *>(a.z);
    const int tid = threadIdx.x, nlev = a.nlev;
    auto level_of = [&](int k) { return a.backward ? nlev - 1 - k : k; };
    // row of this thread in level k (or -1), its row-pointer pair, its entries
    auto first_row = [&](int k) {
        if (k >= nlev) return -1;
        const int l = level_of(k), rr = s_off[l] + tid;
        return rr < s_off[l + 1] ? rr : -1;
    };
    auto load_entries = [&](LevelRow<T> &q) {
#pragma unroll
        for (int e = 0; e < kLevelPre; ++e) {
            if (q.rr >= 0 && q.j0 + e < q.j1) {
                q.c[e] = __ldg(a.col + q.j0 + e);
                q.v[e] = __ldg(val + q.j0 + e);
            }
        }
        if (q.rr >= 0) {
            // the row's own inputs: r_i, or the forward result z_i (written by
            // the previous launch), and the diagonal scalings
            q.own = a.backward ? __ldcg(z + q.rr) : r[q.rr];
            q.e1 = d1 ? d1[q.rr] : T(0);
            q.e2 = (a.sgs && a.backward) ? d2[q.rr] : T(0);
        }
    };
    auto row_value = [&](int rr, int j0, int j1, const int *cp, const T *vp, int r0, int r1, T own, T e1, T e2) {
        T s = T(0);
#pragma unroll
        for (int e = 0; e < kLevelPre; ++e) {
            if (j0 + e < j1) {
                const int cc = cp[e];
                const bool in_ring = a.backward ? cc < r0 + kLevelRing : cc >= r1 - kLevelRing;
                s += vp[e] * (in_ring ? ring[cc & (kLevelRing - 1)] : __ldcg(z + cc));
            }
        }
        for (int j = j0 + kLevelPre; j < j1; ++j) {
            const int cc = __ldg(a.col + j);
            const bool in_ring = a.backward ? cc < r0 + kLevelRing : cc >= r1 - kLevelRing;
            s += __ldg(val + j) * (in_ring ? ring[cc & (kLevelRing - 1)] : __ldcg(z + cc));
        }
        T out;
        if (!a.backward) out = a.sgs ? (-own + s) * e1 : -(-own + s);
        else out = a.sgs ? (own * e2 + s) * e1 : (-own + s) * e1;
        ring[rr & (kLevelRing - 1)] = out;
        __stcg(z + rr, out);
    };
    // software pipeline: entries of level k + 1 and row pointers of level
    // k + 2 are in flight while level k is solved
    LevelRow<T> cur, nxt;
    cur.rr = first_row(0);
    cur.j0 = cur.rr >= 0 ? __ldg(a.row + cur.rr) : 0;
    cur.j1 = cur.rr >= 0 ? __ldg(a.row + cur.rr + 1) : 0;
    load_entries(cur);
    nxt.rr = first_row(1);
    nxt.j0 = nxt.rr >= 0 ? __ldg(a.row + nxt.rr) : 0;
    nxt.j1 = nxt.rr >= 0 ? __ldg(a.row + nxt.rr + 1) : 0;
    for (int k = 0; k < nlev; ++k) {
        const int l = level_of(k), r0 = s_off[l], r1 = s_off[l + 1];
        const int r2 = first_row(k + 2);
        const int p0 = r2 >= 0 ? __ldg(a.row + r2) : 0, p1 = r2 >= 0 ? __ldg(a.row + r2 + 1) : 0;
        load_entries(nxt);
        if (cur.rr >= 0) row_value(cur.rr, cur.j0, cur.j1, cur.c, cur.v, r0, r1, cur.own, cur.e1, cur.e2);
        // rows of a level beyond the first kLevelThreads (no look-ahead)
        for (int rr = r0 + tid + kLevelThreads; rr < r1; rr += kLevelThreads) {
            LevelRow<T> q;
            q.rr = rr;
            q.j0 = __ldg(a.row + rr);
            q.j1 = __ldg(a.row + rr + 1);
            load_entries(q);
            row_value(rr, q.j0, q.j1, q.c, q.v, r0, r1, q.own, q.e1, q.e2);
        }
        __syncthreads();
        cur = nxt;
        nxt.rr = r2;
        nxt.j0 = p0;
        nxt.j1 = p1;
    }
}

// The level sweep with a deeper look-ahead through the async-copy engine.
// At set-up every row of L / U is packed into kp fixed slots (columns and
// values, the entry count beside).  Each thread copies its row of level
// k + kStages - 1 (packed entries, count, own input and scalings) into a
// shared-memory stage with cp.async while level k is solved, so the loads of
// a level arrive kStages - 1 levels early and only the ring gathers, the
// solve and the level barrier remain on the critical path.
constexpr int kStages = 4;
constexpr int kRingStaged = 4096;
constexpr int kStagedMaxLevels = 4096;
constexpr int kStagedSlots = 4;    // packed entries per row (rows of L and U with at most this many)

struct LevelStagedArgs {
    const int *pcol;      // packed columns [n][kp]
    const void *pval;     // packed values [n][kp]
    const int *pcnt;      // entries per row
    const int *off;
    int nlev, n;
    const void *r;
    void *z;
    const void *d1, *d2;
    int backward, sgs;
    const int *gate;
};

__device__ __forceinline__ void cp_async(void *dst, const void *src, int bytes)
{
    const unsigned d = smem_u32(dst);
    if (bytes == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
    else if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <typename T, int KP>
struct StageRec {
    int col[KP];
    T val[KP];
    T own, e1, e2;
    int cnt;
};

template <typename T, int KP>
__global__ void __launch_bounds__(kLevelThreads) level_sweep_staged_kernel(LevelStagedArgs a)
{
    // one thread per row of the largest level (blockDim.x <= kLevelThreads):
    // idle warps would only lengthen every level's barrier
    const int NT = blockDim.x;
    extern __shared__ __align__(16) unsigned char s_raw[];
    using Rec = StageRec<T, KP>;
    Rec *stage = reinterpret_cast<Rec *>(s_raw);                             // [kStages][NT]
    T *ring = reinterpret_cast<T *>(s_raw + sizeof(Rec) * kStages * NT);
    int *s_off = reinterpret_cast<int *>(ring + kRingStaged);
    if (gate_closed(a.gate)) return;
    for (int i = threadIdx.x; i <= a.nlev; i += NT) s_off[i] = __ldg(a.off + i);
    __syncthreads();
    const int tid = threadIdx.x, nlev = a.nlev;
    const T *pval = static_cast<const T *>(a.pval);
    const T *r = static_cast<const T *>(a.r);
    const T *d1 = static_cast<const T *>(a.d1);
    const T *d2 = static_cast<const T *>(a.d2);
    T *z = static_cast<T *>(a.z);
    const bool need_e1 = a.backward || a.sgs, need_e2 = a.backward && a.sgs;
    auto level_of = [&](int k) { return a.backward ? nlev - 1 - k : k; };
    // this thread's row of level k into stage k % kStages (one commit group per level)
    auto issue = [&](int k) {
        if (k < nlev) {
            const int l = level_of(k), rr = s_off[l] + tid;
            if (rr < s_off[l + 1]) {
                Rec &q = stage[(k % kStages) * NT + tid];
#pragma unroll
                for (int b = 0; b < KP * 4; b += 16) cp_async(reinterpret_cast<char *>(q.col) + b,
                                                              reinterpret_cast<const char *>(a.pcol + (size_t)rr * KP) + b, 16);
#pragma unroll
                for (int b = 0; b < KP * (int)sizeof(T); b += 16)
                    cp_async(reinterpret_cast<char *>(q.val) + b, reinterpret_cast<const char *>(pval + (size_t)rr * KP) + b,
                             16);
                cp_async(&q.cnt, a.pcnt + rr, 4);
                cp_async(&q.own, (a.backward ? static_cast<const T *>(z) : r) + rr, (int)sizeof(T));
                if (need_e1) cp_async(&q.e1, d1 + rr, (int)sizeof(T));
                if (need_e2) cp_async(&q.e2, d2 + rr, (int)sizeof(T));
            }
        }
        cp_async_commit();
    };
    auto solve = [&](int rr, const int *cols, const T *vals, int cnt, T own, T e1, T e2, int r0, int r1) {
        T s = T(0);
#pragma unroll
        for (int e = 0; e < KP; ++e) {
            if (e < cnt) {
                const int cc = cols[e];
                const bool in_ring = a.backward ? cc < r0 + kRingStaged : cc >= r1 - kRingStaged;
                s += vals[e] * (in_ring ? ring[cc & (kRingStaged - 1)] : __ldcg(z + cc));
            }
        }
        T out;
        if (!a.backward) out = a.sgs ? (-own + s) * e1 : -(-own + s);
        else out = a.sgs ? (own * e2 + s) * e1 : (-own + s) * e1;
        ring[rr & (kRingStaged - 1)] = out;
        __stcg(z + rr, out);
    };
#pragma unroll
    for (int k = 0; k < kStages - 1; ++k) issue(k);
    for (int k = 0; k < nlev; ++k) {
        issue(k + kStages - 1);
        cp_async_wait<kStages - 1>();
        const int l = level_of(k), r0 = s_off[l], r1 = s_off[l + 1];
        const int rr = r0 + tid;
        if (rr < r1) {
            const Rec &q = stage[(k % kStages) * NT + tid];
            solve(rr, q.col, q.val, q.cnt, q.own, need_e1 ? q.e1 : T(0), need_e2 ? q.e2 : T(0), r0, r1);
        }
        // rows of a level beyond the first NT: read directly
        for (int r2 = rr + NT; r2 < r1; r2 += NT) {
            int cols[KP];
            T vals[KP];
#pragma unroll
            for (int e = 0; e < KP; ++e) {
                cols[e] = __ldg(a.pcol + (size_t)r2 * KP + e);
                vals[e] = __ldg(pval + (size_t)r2 * KP + e);
            }
            const T own = a.backward ? __ldcg(z + r2) : r[r2];
            solve(r2, cols, vals, __ldg(a.pcnt + r2), own, need_e1 ? d1[r2] : T(0), need_e2 ? d2[r2] : T(0), r0, r1);
        }
        __syncthreads();
    }
    cp_async_wait<0>();
}

// Pack the rows of a CSR into kp fixed slots (columns, values; unused slots
// column 0, value 0) with the entry count beside.
template <typename T>
__global__ void pack_rows_kernel(int n, int kp, const int *__restrict__ row, const int *__restrict__ col,
                                 const T *__restrict__ val, int *__restrict__ pcol, T *__restrict__ pval,
                                 int *__restrict__ pcnt)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int b = row[i], e = row[i + 1];
        for (int k = 0; k < kp; ++k) {
            const bool in = b + k < e;
            pcol[(size_t)i * kp + k] = in ? col[b + k] : 0;
            pval[(size_t)i * kp + k] = in ? val[b + k] : T(0);
        }
        pcnt[i] = e - b;
    }
}

constexpr size_t kStagedSmemCap = 226 * 1024;   // opt-in shared memory per CTA on sm_100 (227 KB), less the static part

template <typename T, int KP>
size_t staged_smem(int nlev, int NT = kLevelThreads)
{
    return sizeof(StageRec<T, KP>) * kStages * NT + sizeof(T) * kRingStaged + sizeof(int) * (nlev + 1);
}

}  // namespace

namespace b200 {

cudaError_t sweeps_configure()
{
    cudaError_t e;
    // the largest stage set a plan may use (its CTA size and level count are
    // checked against kStagedSmemCap at set-up)
    if ((e = cudaFuncSetAttribute(level_sweep_staged_kernel<double, kStagedSlots>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)std::min(staged_smem<double, kStagedSlots>(kStagedMaxLevels), kStagedSmemCap))) ||
        (e = cudaFuncSetAttribute(level_sweep_staged_kernel<float, kStagedSlots>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)std::min(staged_smem<float, kStagedSlots>(kStagedMaxLevels), kStagedSmemCap))))
        return e;
    e = cudaFuncSetAttribute(level_sweep_cta_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(kLevelRing * sizeof(double) + sizeof(int) * (kLevelMaxLevels + 1)));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(level_sweep_cta_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(kLevelRing * sizeof(float) + sizeof(int) * (kLevelMaxLevels + 1)));
}

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
    int *lev_off = nullptr;   // single-CTA level sweep: level offsets (null: chunk tickets)
    int nlev = 0;
    // staged variant: rows of L / U packed into kStagedSlots slots
    int staged = 0;
    int threads = kLevelThreads;   // the largest level's rows rounded up to a warp (at most kLevelThreads)
    int *pcol[2] = {nullptr, nullptr}, *pcnt[2] = {nullptr, nullptr};
    void *pval[2] = {nullptr, nullptr};
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
    // many small levels: one CTA walks them, with the async-copy look-ahead
    // when every row of L and U fits kStagedSlots slots (B200LA_SWEEP =
    // staged / cta / tickets to force a variant)
    auto maxlen = [](const b200la_csr *M) {
        int m = 0;
        for (int i = 0; i < M->n; ++i) m = std::max(m, M->h_row[i + 1] - M->h_row[i]);
        return m;
    };
    const bool few = P->nblocks > 64 && P->n / std::max(P->nblocks, 1) <= 4 * kLevelThreads;
    int widest = 1;
    for (int l = 0; l < P->nblocks; ++l) widest = std::max(widest, P->block_off[l + 1] - P->block_off[l]);
    const int nt = std::min(kLevelThreads, (widest + 31) / 32 * 32);
    const bool can_stage = P->nblocks <= kStagedMaxLevels && maxlen(P->L) <= kStagedSlots &&
                           maxlen(P->U) <= kStagedSlots &&
                           staged_smem<double, kStagedSlots>(P->nblocks, nt) <= kStagedSmemCap;
    bool cta = few && P->nblocks <= kLevelMaxLevels, staged = few && can_stage;
    if (const char *sw = std::getenv("B200LA_SWEEP")) {
        staged = std::strcmp(sw, "staged") == 0 && can_stage;
        cta = (std::strcmp(sw, "cta") == 0 || std::strcmp(sw, "staged") == 0) && P->nblocks <= kLevelMaxLevels;
    }
    if (cta) {
        SyncFreePlan *plan = new SyncFreePlan();
        plan->nlev = P->nblocks;
        plan->threads = nt;
        cudaError_t e;
        if ((e = cudaMalloc(&plan->lev_off, sizeof(int) * (P->nblocks + 1))) ||
            (e = cudaMemcpy(plan->lev_off, P->block_off.data(), sizeof(int) * (P->nblocks + 1),
                            cudaMemcpyHostToDevice))) {
            if (plan->lev_off) cudaFree(plan->lev_off);
            delete plan;
            return ctx_fail(ctx, B200LA_ERR_ALLOC, "level sweep setup", e);
        }
        if (staged) {
            const size_t es = P->dtype == B200LA_F64 ? 8 : 4, n = (size_t)P->n;
            for (int m = 0; m < 2 && e == cudaSuccess; ++m) {
                const b200la_csr *M = m ? P->U : P->L;
                if ((e = cudaMalloc(&plan->pcol[m], sizeof(int) * kStagedSlots * n)) ||
                    (e = cudaMalloc(&plan->pval[m], es * kStagedSlots * n)) ||
                    (e = cudaMalloc(&plan->pcnt[m], sizeof(int) * n)))
                    break;
                const int g = std::max(1, std::min((P->n + 255) / 256, 148 * 16));
                if (P->dtype == B200LA_F64)
                    pack_rows_kernel<double><<<g, 256, 0, ctx->stream>>>(P->n, kStagedSlots, M->row, M->col,
                                                                         (const double *)M->val, plan->pcol[m],
                                                                         (double *)plan->pval[m], plan->pcnt[m]);
                else
                    pack_rows_kernel<float><<<g, 256, 0, ctx->stream>>>(P->n, kStagedSlots, M->row, M->col,
                                                                        (const float *)M->val, plan->pcol[m],
                                                                        (float *)plan->pval[m], plan->pcnt[m]);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess) {
                P->syncfree_plan = plan;
                syncfree_free(P);
                return ctx_fail(ctx, B200LA_ERR_ALLOC, "staged level sweep setup", e);
            }
            plan->staged = 1;
        }
        P->syncfree_plan = plan;
        P->use_syncfree = 1;
        return B200LA_OK;
    }
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
    if (plan->fwd) cudaFree(plan->fwd);
    if (plan->bwd) cudaFree(plan->bwd);
    if (plan->lev_off) cudaFree(plan->lev_off);
    for (int m = 0; m < 2; ++m) {
        if (plan->pcol[m]) cudaFree(plan->pcol[m]);
        if (plan->pval[m]) cudaFree(plan->pval[m]);
        if (plan->pcnt[m]) cudaFree(plan->pcnt[m]);
    }
    delete plan;
    P->syncfree_plan = nullptr;
}

int syncfree_apply(b200la_ctx *ctx, const b200la_precond *P, const void *r, void *z, const int *gate)
{
    const SyncFreePlan *plan = static_cast<const SyncFreePlan *>(P->syncfree_plan);
    if (plan->staged) {
        LevelStagedArgs a;
        a.off = plan->lev_off;
        a.nlev = plan->nlev;
        a.n = P->n;
        a.r = r;
        a.z = z;
        a.d1 = P->iDv;
        a.d2 = P->Dv;
        a.sgs = P->kind == B200LA_PRECOND_MCSGS;
        a.gate = gate;
        for (int dir = 0; dir < 2; ++dir) {
            a.pcol = plan->pcol[dir];
            a.pval = plan->pval[dir];
            a.pcnt = plan->pcnt[dir];
            a.backward = dir;
            const int nt = plan->threads;
            if (P->dtype == B200LA_F64)
                level_sweep_staged_kernel<double, kStagedSlots>
                    <<<1, nt, staged_smem<double, kStagedSlots>(plan->nlev, nt), ctx->stream>>>(a);
            else
                level_sweep_staged_kernel<float, kStagedSlots>
                    <<<1, nt, staged_smem<float, kStagedSlots>(plan->nlev, nt), ctx->stream>>>(a);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "staged level sweep", e);
            ctx->launches += 1;
        }
        return B200LA_OK;
    }
    if (plan->lev_off) {
        LevelSweepArgs a;
        a.off = plan->lev_off;
        a.nlev = plan->nlev;
        a.r = r;
        a.z = z;
        a.d1 = P->iDv;
        a.d2 = P->Dv;
        a.sgs = P->kind == B200LA_PRECOND_MCSGS;
        a.gate = gate;
        for (int dir = 0; dir < 2; ++dir) {
            const b200la_csr *M = dir ? P->U : P->L;
            a.row = M->row;
            a.col = M->col;
            a.val = M->val;
            a.backward = dir;
            if (P->dtype == B200LA_F64)
                level_sweep_cta_kernel<double>
                    <<<1, kLevelThreads, kLevelRing * sizeof(double) + sizeof(int) * (plan->nlev + 1), ctx->stream>>>(a);
            else
                level_sweep_cta_kernel<float>
                    <<<1, kLevelThreads, kLevelRing * sizeof(float) + sizeof(int) * (plan->nlev + 1), ctx->stream>>>(a);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "level sweep", e);
            ctx->launches += 1;
        }
        return B200LA_OK;
    }
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
