// serve.cc -- the continuous-batching solve server (host side).
//
// Threads:
//   * admission: takes queued requests in arrival order, waits until the
//     memory budget and a slot are free, uploads (or assembles on the device)
//     the operator, builds the slot's chunk layout, Jacobi diagonal and
//     Krylov state on the copy stream, and hands the slot to the round
//     thread.  It also retires finished slots: result back to the host
//     array, memory back to the pool and the budget.
//   * rounds: tops the active set up from the admitted slots (arrival order,
//     bounded by max_active and by the bytes one batch iteration streams),
//     writes the tile table, replays the CUDA graph of iters_per_round batch
//     iterations, reads the per-slot final-status words, and passes finished
//     slots back for retirement.  Uploads of new requests overlap the rounds.
//   * gmres: nonsymmetric requests, one at a time on their own stream and
//     context, sharing the memory budget.
// Device memory comes from a pool owned by the server (stream-ordered
// allocations; freed blocks are kept for reuse).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "b200la.h"
#include "b200la_internal.h"
#include "serve.cuh"

using b200::srv::SysDesc;
using b200::srv::SysRun;
using b200::srv::SysState;

namespace {

constexpr int kTabCap = 1 << 16;    // systems one round may list
// The active set is split into lanes (3 by default, B200LA_SERVE_LANES from 1
// to kLanes), each with its own system table and its own chain of kernels in
// the round's graph: the chains run concurrently, so one lane's kernel tails
// and reduction chains overlap another lane's streaming.
constexpr int kLanes = 4;
constexpr size_t kTabWords = b200::srv::kTabHdrWords + sizeof(SysRun) / sizeof(int) * (size_t)kTabCap;

size_t al256(size_t b) { return (b + 255) & ~size_t(255); }

struct Req {
    long long id = 0;
    b200la_request r{};
    b200la_serve_result res{};
    bool done = false;
    // layout decided at submission
    int n = 0, fmt = 0, nchunks = 0;
    long long nnz = 0, slen = 0;      // stored entries (SELL: padded)
    long long slen32 = 0;             // stored FP32 entries (mixed; stencil: 32 L per chunk)
    int half = 0;                     // Q1 Poisson: half stencil layout (full-size storage kept for the fallback)
    long long hlen64 = 0, hlen32 = 0; // half stencil: FP64 / FP32 values streamed per product
    std::vector<int> sell_off;        // SELL chunk offsets
    size_t bytes = 0, temp_bytes = 0; // resident / admission scratch
    double iter_bytes = 0;            // streamed by one batch iteration
    double work = 0;                  // estimated bytes to convergence (iter_bytes x ~iterations)
    int w1 = 1, w2 = 1;               // chunk weights of the SpMV and update kernels (bytes per row)
};

struct Slot {
    int idx = -1;
    Req *req = nullptr;
    void *block = nullptr;
    SysDesc desc{};
};

// Row lengths of the structured Q1 operator: w(ix) w(iy) w(iz), w = 2 on the boundary.
inline int q1_rowlen(int dim, int N, long long i)
{
    const long long P = N + 1;
    const int ix = (int)(i % P), iy = (int)((i / P) % P), iz = dim == 3 ? (int)(i / (P * P)) : 1;
    auto w = [N](int t) { return (t == 0 || t == N) ? 2 : 3; };
    return w(ix) * w(iy) * (dim == 3 ? w(iz) : 1);
}

inline size_t q1_cells(int dim, int N) { return (size_t)N * N * (dim == 3 ? (size_t)N : 1); }

}  // namespace

struct b200la_server {
    b200la_serve_config cfg{};
    int device = 0, num_sms = 148;
    std::chrono::steady_clock::time_point t0;
    cudaMemPool_t pool = nullptr;
    cudaStream_t s_comp = nullptr, s_copy = nullptr, s_lane[kLanes] = {};   // s_lane[0] unused (lane 0: s_comp)
    cudaEvent_t ev_a = nullptr, ev_b = nullptr, ev_fork = nullptr, ev_join[kLanes] = {};
    int lanes = 3, lane_nt[kLanes] = {};
    bool lpt = false;                 // activate the ready system with the most estimated work first
    SysDesc *d_sys = nullptr;
    SysState *d_state = nullptr;
    unsigned *d_ticket = nullptr;
    int *d_done = nullptr, *h_done = nullptr;
    int *d_tiles = nullptr, *h_tiles = nullptr;
    // pinned staging of the admission thread's uploads: a copy from pageable
    // memory is staged by the driver, which may first wait for the copy
    // stream -- behind the admission kernels that share the GPU with the rounds
    struct AdmitStage {
        SysState hs;
        SysDesc d;
        unsigned asym;
    };
    AdmitStage *h_admit = nullptr;
    double *h_kc = nullptr;           // a request's cell field
    size_t h_kc_len = 0;
    cudaGraphExec_t graph = nullptr;
    // kernel shape
    int nw = 8, ctas_per_sm = 4, cpw = 4, iters = 16;
    double active_cap = 4096.0 * 1024 * 1024;
    int max_active = 1024;

    std::mutex mu;
    std::condition_variable cv_admit, cv_round, cv_done, cv_gm;
    std::deque<Req *> pending, gm_pending;
    std::deque<Slot *> ready, retire_q;
    std::vector<Slot *> active;
    std::vector<int> free_idx;
    std::unordered_map<long long, std::unique_ptr<Req>> reqs;
    long long next_id = 1, submitted = 0, completed = 0, failed = 0, rounds = 0, batch_iters = 0;
    double busy_ms = 0.0, resident = 0.0, peak_resident = 0.0;
    int peak_active = 0;
    bool quit = false;
    int fatal = 0;
    std::thread th_admit, th_round, th_gm;

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

// ------------------------------------------------------------- layout

int plan_request(b200la_server *S, Req *q)
{
    const b200la_request &r = q->r;
    const bool mixed = r.precision == B200LA_SERVE_MIXED;
    std::vector<int> len;
    if (r.row) {
        long long bad = 0;
        if (r.n <= 0 || r.nnz < 0 || !r.col || !r.val) return B200LA_ERR_ARG;
        if (b200::host::validate_csr(r.n, r.n, r.nnz, r.row, r.col, &bad)) return B200LA_ERR_CSR;
        q->n = r.n;
        q->nnz = r.nnz;
        len.resize(r.n);
        for (int i = 0; i < r.n; ++i) len[i] = r.row[i + 1] - r.row[i];
    } else {
        int n;
        int64_t nnz;
        if (b200::host::q1_sizes(r.q1_dim, r.q1_N, &n, &nnz) || (r.q1_kind != 0 && r.q1_kind != 1))
            return B200LA_ERR_ARG;
        q->n = n;
        q->nnz = nnz;
        len.resize(n);
        for (int i = 0; i < n; ++i) len[i] = q1_rowlen(r.q1_dim, r.q1_N, i);
    }
    const int n = q->n;
    q->nchunks = (n + b200::srv::kChunk - 1) / b200::srv::kChunk;
    if (!r.row) {
        // structured Q1 operator: stencil layout, no indices
        const int L = r.q1_dim == 3 ? 27 : 9;
        q->fmt = b200::srv::FMT_STENCIL;
        q->slen = (long long)q->nchunks * b200::srv::kChunk * L;
        q->slen32 = (long long)q->nchunks * b200::srv::kChunk * L;
        // Poisson operators are symmetric outside their identity rows: half
        // stencil (checked on the device at admission, full layout
        // otherwise).  B200LA_SERVE_HALF = 0: never; 1 (default): FP64
        // requests; 2: FP64 and mixed requests.
        const char *hv = std::getenv("B200LA_SERVE_HALF");
        const int hm = hv ? std::atoi(hv) : 1;
        q->half = r.q1_kind == 0 && (hm == 2 || (hm == 1 && !mixed));
        q->hlen64 = (long long)q->nchunks * b200::srv::kChunk * b200::srv::half_len64(r.q1_dim);
        q->hlen32 = (long long)q->nchunks * b200::srv::kChunk * b200::srv::half_len32(r.q1_dim);
    }
    int maxlen = 0;
    for (int v : len) maxlen = std::max(maxlen, v);
    long long slen = 0;
    if (q->fmt != b200::srv::FMT_STENCIL && maxlen <= b200::srv::kMaxRowSell) {
        q->sell_off.assign(q->nchunks + 1, 0);
        for (int c = 0; c < q->nchunks; ++c) {
            int L = 0;
            for (int i = c * 32; i < std::min(n, c * 32 + 32); ++i) L = std::max(L, len[i]);
            q->sell_off[c + 1] = q->sell_off[c] + 32 * L;
            slen += 32LL * L;
        }
    }
    if (q->fmt == b200::srv::FMT_STENCIL) {
        // layout fixed above
    } else if (maxlen <= b200::srv::kMaxRowSell && slen <= 2 * std::max<long long>(q->nnz, 1) &&
               slen < (1LL << 31)) {
        q->fmt = b200::srv::FMT_SELL;
        q->slen = q->slen32 = slen;
    } else {
        q->fmt = b200::srv::FMT_CSRW;
        q->slen = q->slen32 = q->nnz;
        q->sell_off.clear();
    }
    const size_t v8 = al256(8 * (size_t)n), v4 = al256(4 * (size_t)n);
    const bool stencil = q->fmt == b200::srv::FMT_STENCIL;
    const size_t offb = stencil ? 0
                        : q->fmt == b200::srv::FMT_SELL ? al256(4 * (size_t)(q->nchunks + 1))
                                                        : al256(4 * (size_t)(n + 1));
    const size_t colb = stencil ? 0 : al256(4 * (size_t)q->slen);
    const size_t pst = (size_t)((q->nchunks + 1) & ~1);
    const size_t ng = (size_t)((q->nchunks + b200::srv::kGroup - 1) / b200::srv::kGroup), gst = (ng + 1) & ~size_t(1);
    size_t b = offb + colb + al256(8 * (size_t)q->slen) + al256(24 * pst) + al256(24 * gst) + al256(4 * ng);
    if (stencil) b += al256(4 * (size_t)(q->nchunks + 1));   // identity-row mask and set-up check
    if (mixed) b += al256(4 * (size_t)q->slen32) + 2 * v8 + 7 * v4;
    else b += 8 * v8;
    q->bytes = b;
    q->temp_bytes = al256(4 * (size_t)(n + 1)) + al256(4 * (size_t)q->nnz) + al256(8 * (size_t)q->nnz) +
                    ((!r.row && r.q1_kcell) ? al256(8 * q1_cells(r.q1_dim, r.q1_N)) : 0);
    const double ib = stencil ? 0.0 : 4.0;   // index bytes per stored entry
    // values streamed per product (the half layout streams fewer than it stores)
    const double s64 = q->half ? (double)q->hlen64 : (double)q->slen, s32 = q->half ? (double)q->hlen32 : (double)q->slen32;
    q->iter_bytes = mixed ? 4.0 * s32 + ib * q->slen + 48.0 * n : (8.0 + ib) * s64 + 96.0 * n;   // vectors: 32n (SpMV) + 64n (update)
    // Jacobi-CG on a Q1 grid needs iterations in proportion to the nodes per line
    q->work = q->iter_bytes * (q->r.q1_N > 0 ? (double)q->r.q1_N : std::sqrt((double)n));
    // per-row costs of the two kernels: operator + gathers and stores (k1),
    // the update's vector traffic (k2); warp-per-row CSR counts double
    const double rows = 32.0 * q->nchunks;
    const double op = mixed ? (4.0 * s32 + ib * q->slen) / rows : (8.0 + ib) * s64 / rows;
    const double k1 = (op + (mixed ? 16.0 : 32.0)) * (q->fmt == b200::srv::FMT_CSRW ? 2.0 : 1.0);
    q->w1 = std::max(1, (int)std::lround(k1));
    q->w2 = mixed ? 32 : 64;
    // a system's weighted span stays below 2^30 (positions are int32)
    const long long wcap = std::max<long long>(1, (1LL << 30) / std::max(q->nchunks, 1));
    q->w1 = (int)std::min<long long>(q->w1, wcap);
    q->w2 = (int)std::min<long long>(q->w2, wcap);
    return B200LA_OK;
}

size_t gmres_bytes(const Req *q)
{
    const size_t n = q->n, nnz = q->nnz;
    const int m = std::max(q->r.gmres_m, 1);
    size_t b = 3 * al256(12 * nnz + 4 * (n + 1)) + (size_t)(m + 8) * al256(8 * n);
    return b;
}

// ------------------------------------------------------------- slots

int fail_all(b200la_server *S, int code);

#define SV(call)                                  \
    do {                                          \
        cudaError_t e_ = (call);                  \
        if (e_ != cudaSuccess) return -(int)e_;   \
    } while (0)

// Upload / assemble request q into slot sl (on the copy stream; synchronous).
int admit_slot(b200la_server *S, Req *q, Slot *sl)
{
    const b200la_request &r = q->r;
    const bool mixed = r.precision == B200LA_SERVE_MIXED;
    const int n = q->n;
    cudaStream_t st = S->s_copy;
    void *blk = nullptr, *tmp = nullptr;
    SV(cudaMallocFromPoolAsync(&blk, q->bytes, S->pool, st));
    SV(cudaMallocFromPoolAsync(&tmp, q->temp_bytes, S->pool, st));
    sl->block = blk;
    char *p = static_cast<char *>(blk);
    auto take = [&p](size_t b) {
        char *o = p;
        p += al256(b);
        return o;
    };
    SysDesc d{};
    d.n = n;
    d.nchunks = q->nchunks;
    d.mixed = mixed;
    d.fmt = q->fmt;
    d.pstride = (q->nchunks + 1) & ~1;
    d.ngroups = (q->nchunks + b200::srv::kGroup - 1) / b200::srv::kGroup;
    d.gstride = (d.ngroups + 1) & ~1;
    const bool sell = q->fmt == b200::srv::FMT_SELL;
    const bool stencil = q->fmt == b200::srv::FMT_STENCIL;
    if (stencil) {
        d.sdim = r.q1_dim;
        d.sP = r.q1_N + 1;
        d.sL = r.q1_dim == 3 ? 27 : 9;
        d.half = q->half;
        d.smask = reinterpret_cast<unsigned *>(take(4 * (size_t)(q->nchunks + 1)));
    } else {
        d.off = reinterpret_cast<int *>(take(sell ? 4 * (size_t)(q->nchunks + 1) : 4 * (size_t)(n + 1)));
        d.col = reinterpret_cast<int *>(take(4 * (size_t)q->slen));
    }
    d.val64 = reinterpret_cast<double *>(take(8 * (size_t)q->slen));
    d.val32 = mixed ? reinterpret_cast<float *>(take(4 * (size_t)q->slen32)) : nullptr;
    d.part = reinterpret_cast<double *>(take(24 * (size_t)d.pstride));
    d.gpart = reinterpret_cast<double *>(take(24 * (size_t)d.gstride));
    d.gcnt = reinterpret_cast<unsigned *>(take(4 * (size_t)d.ngroups));
    d.b = reinterpret_cast<double *>(take(8 * (size_t)n));
    char *vec0 = p;   // vectors that start at zero
    d.x = reinterpret_cast<double *>(take(8 * (size_t)n));
    const size_t ve = mixed ? 4 : 8;
    d.r = take(ve * n);
    d.z = take(ve * n);
    d.p0 = take(ve * n);
    d.p1 = take(ve * n);
    d.ap = take(ve * n);
    d.xl = mixed ? take(4 * (size_t)n) : nullptr;
    char *vec1 = p;
    d.invd = take(ve * n);
    d.ticket = S->d_ticket + (size_t)sl->idx * b200::srv::kTicketWords;
    d.done = S->d_done + sl->idx;

    // scratch CSR (and cell field)
    char *t = static_cast<char *>(tmp);
    int *trow = reinterpret_cast<int *>(t);
    t += al256(4 * (size_t)(n + 1));
    int *tcol = reinterpret_cast<int *>(t);
    t += al256(4 * (size_t)q->nnz);
    double *tval = reinterpret_cast<double *>(t);
    t += al256(8 * (size_t)q->nnz);
    if (r.row) {
        SV(cudaMemcpyAsync(trow, r.row, 4 * (size_t)(n + 1), cudaMemcpyHostToDevice, st));
        SV(cudaMemcpyAsync(tcol, r.col, 4 * (size_t)q->nnz, cudaMemcpyHostToDevice, st));
        SV(cudaMemcpyAsync(tval, r.val, 8 * (size_t)q->nnz, cudaMemcpyHostToDevice, st));
    } else {
        double *kc = nullptr;
        if (r.q1_kcell) {
            kc = reinterpret_cast<double *>(t);
            const size_t cells = q1_cells(r.q1_dim, r.q1_N);
            if (cells > S->h_kc_len) {
                // the staging buffer grows (the copy stream holds no copy from it: admissions end synchronised)
                if (S->h_kc) cudaFreeHost(S->h_kc);
                S->h_kc = nullptr;
                S->h_kc_len = 0;
                SV(cudaMallocHost(&S->h_kc, 8 * cells));
                S->h_kc_len = cells;
            }
            std::memcpy(S->h_kc, r.q1_kcell, 8 * cells);
            SV(cudaMemcpyAsync(kc, S->h_kc, 8 * cells, cudaMemcpyHostToDevice, st));
        }
        SV(b200::launch_q1_assemble(r.q1_dim, r.q1_N, r.q1_kind, kc, r.q1_nu, r.q1_beta, trow, tcol, tval, st));
    }
    if (stencil) {
        SV(cudaMemsetAsync(const_cast<double *>(d.val64), 0, 8 * (size_t)q->slen, st));
        if (mixed) SV(cudaMemsetAsync(const_cast<float *>(d.val32), 0, 4 * (size_t)q->slen32, st));
        SV(cudaMemsetAsync(const_cast<unsigned *>(d.smask), 0, 4 * (size_t)(q->nchunks + 1), st));
    } else if (sell) {
        SV(cudaMemcpyAsync(const_cast<int *>(d.off), q->sell_off.data(), 4 * (size_t)(q->nchunks + 1),
                           cudaMemcpyHostToDevice, st));
    } else {
        SV(cudaMemcpyAsync(const_cast<int *>(d.off), trow, 4 * (size_t)(n + 1), cudaMemcpyDeviceToDevice, st));
        SV(cudaMemcpyAsync(const_cast<int *>(d.col), tcol, 4 * (size_t)q->nnz, cudaMemcpyDeviceToDevice, st));
        SV(cudaMemcpyAsync(const_cast<double *>(d.val64), tval, 8 * (size_t)q->nnz, cudaMemcpyDeviceToDevice, st));
    }
    SV(b200::srv::launch_build_slot(d, trow, tcol, tval, st));
    if (stencil && d.half) {
        // the half layout needs a_ij == a_ji between rows that are not identity rows
        SV(cudaMemcpyAsync(&S->h_admit->asym, d.smask + q->nchunks, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        SV(cudaStreamSynchronize(st));
        if (S->h_admit->asym) {
            d.half = 0;
            SV(cudaMemsetAsync(const_cast<double *>(d.val64), 0, 8 * (size_t)q->slen, st));
            if (mixed) SV(cudaMemsetAsync(const_cast<float *>(d.val32), 0, 4 * (size_t)q->slen32, st));
            SV(b200::srv::launch_build_slot(d, trow, tcol, tval, st));
        }
    }
    if (r.b) SV(cudaMemcpyAsync(const_cast<double *>(d.b), r.b, 8 * (size_t)n, cudaMemcpyHostToDevice, st));
    else SV(b200::launch_q1_rhs(r.rhs_seed, r.q1_dim, r.q1_N, const_cast<double *>(d.b), st));
    SV(cudaMemsetAsync(vec0, 0, (size_t)(vec1 - vec0), st));
    SysState &hs = S->h_admit->hs;   // pinned: the copy below is asynchronous
    hs = SysState{};
    hs.abstol = r.ctl.abstol;
    hs.reltol = r.ctl.reltol;
    hs.divtol = r.ctl.divtol;
    hs.maxits = r.ctl.maxits;
    hs.in_abstol = r.inner.abstol;
    hs.in_reltol = r.inner.reltol;
    hs.in_divtol = r.inner.divtol;
    hs.in_maxits = r.inner.maxits;
    hs.max_outer = r.max_outer;
    hs.phase = mixed ? b200::srv::PH_OUTER : b200::srv::PH_CG_START;
    SV(cudaMemcpyAsync(S->d_state + sl->idx, &hs, sizeof hs, cudaMemcpyHostToDevice, st));
    SV(cudaMemsetAsync(d.ticket, 0, sizeof(unsigned) * b200::srv::kTicketWords, st));
    SV(cudaMemsetAsync(d.gcnt, 0, sizeof(unsigned) * (size_t)d.ngroups, st));
    SV(cudaMemsetAsync(d.done, 0, sizeof(int), st));
    S->h_admit->d = d;
    SV(cudaMemcpyAsync(S->d_sys + sl->idx, &S->h_admit->d, sizeof d, cudaMemcpyHostToDevice, st));
    SV(cudaFreeAsync(tmp, st));
    SV(cudaStreamSynchronize(st));   // the staging area is reused by the next admission
    sl->desc = d;
    return 0;
}

int retire_slot(b200la_server *S, Slot *sl)
{
    Req *q = sl->req;
    SysState hs{};
    cudaStream_t st = S->s_copy;
    SV(cudaMemcpyAsync(&hs, S->d_state + sl->idx, sizeof hs, cudaMemcpyDeviceToHost, st));
    SV(cudaMemcpyAsync(q->r.x, sl->desc.x, 8 * (size_t)q->n, cudaMemcpyDeviceToHost, st));
    SV(cudaStreamSynchronize(st));
    SV(cudaFreeAsync(sl->block, st));
    q->res.status = hs.status;
    q->res.iters = hs.iter;
    q->res.outer = hs.outer;
    q->res.res0 = hs.res0;
    q->res.res = hs.res;
    return 0;
}

void finish(b200la_server *S, Req *q, int status_if_error)
{
    // caller holds S->mu
    if (status_if_error) {
        q->res.status = -status_if_error;
        ++S->failed;
    } else {
        ++S->completed;
    }
    q->res.t_done = S->now();
    q->done = true;
    S->cv_done.notify_all();
}

int fail_all(b200la_server *S, int code)
{
    // caller holds S->mu; the round thread fails its own active set
    S->fatal = code;
    for (Req *q : S->pending) finish(S, q, code);
    S->pending.clear();
    for (Req *q : S->gm_pending) finish(S, q, code);
    S->gm_pending.clear();
    for (Slot *sl : S->ready) {
        finish(S, sl->req, code);
        delete sl;
    }
    S->ready.clear();
    for (Slot *sl : S->retire_q) {
        if (!sl->req->done) finish(S, sl->req, code);
        delete sl;
    }
    S->retire_q.clear();
    S->cv_round.notify_all();
    S->cv_admit.notify_all();
    S->cv_gm.notify_all();
    return code;
}

// ------------------------------------------------------------- threads

void admit_loop(b200la_server *S)
{
    cudaSetDevice(S->device);
    for (;;) {
        Slot *ret = nullptr;
        Req *q = nullptr;
        int idx = -1;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            auto fits = [S](const Req *r) {
                return !S->free_idx.empty() &&
                       S->resident + (double)(r->bytes + r->temp_bytes) <= S->cfg.budget_bytes;
            };
            S->cv_admit.wait(lk, [&] {
                return S->quit || !S->retire_q.empty() || (!S->pending.empty() && fits(S->pending.front()));
            });
            if (!S->retire_q.empty()) {
                ret = S->retire_q.front();
                S->retire_q.pop_front();
            } else if (!S->pending.empty() && fits(S->pending.front()) && !S->fatal) {
                q = S->pending.front();
                S->pending.pop_front();
                idx = S->free_idx.back();
                S->free_idx.pop_back();
                S->resident += (double)(q->bytes + q->temp_bytes);
                S->peak_resident = std::max(S->peak_resident, S->resident);
                q->res.t_admit = S->now();
            } else if (S->quit) {
                return;
            }
        }
        if (ret) {
            const int rc = retire_slot(S, ret);
            std::lock_guard<std::mutex> lk(S->mu);
            S->resident -= (double)ret->req->bytes;
            S->free_idx.push_back(ret->idx);
            if (rc) fail_all(S, B200LA_ERR_CUDA);
            else finish(S, ret->req, 0);
            delete ret;
            S->cv_gm.notify_all();
            continue;
        }
        if (!q) continue;
        Slot *sl = new Slot();
        sl->idx = idx;
        sl->req = q;
        q->res.bytes = (double)q->bytes;
        const int rc = admit_slot(S, q, sl);
        std::lock_guard<std::mutex> lk(S->mu);
        S->resident -= (double)q->temp_bytes;
        if (rc) {
            S->free_idx.push_back(idx);
            S->resident -= (double)q->bytes;
            delete sl;
            fail_all(S, B200LA_ERR_CUDA);
            continue;
        }
        q->res.t_ready = S->now();
        S->ready.push_back(sl);
        S->cv_round.notify_one();
    }
}

struct ActiveSys {
    int idx, nchunks, w1, w2;
    double ib;   // bytes streamed per batch iteration
};

// System table of the active set: header [systems, chunks, chunks per warp range].
// The lanes' system tables (host side): each system goes to the lane with
// the fewest bytes per batch iteration so far, in arrival order.
int write_table(b200la_server *S, const std::vector<ActiveSys> &act)
{
    double load[kLanes] = {};
    int nt[kLanes] = {}, tot[kLanes] = {}, W1[kLanes] = {}, W2[kLanes] = {};
    for (const ActiveSys &a : act) {
        int l = 0;
        for (int k = 1; k < S->lanes; ++k)
            if (load[k] < load[l]) l = k;
        load[l] += a.ib;
        SysRun *tab = reinterpret_cast<SysRun *>(S->h_tiles + (size_t)l * kTabWords + b200::srv::kTabHdrWords);
        tab[nt[l]++] = SysRun{a.idx, tot[l], a.nchunks, a.w1, a.w2, W1[l], W2[l], 0};
        tot[l] += a.nchunks;
        W1[l] += a.nchunks * a.w1;
        W2[l] += a.nchunks * a.w2;
    }
    int all = 0;
    for (int l = 0; l < S->lanes; ++l) {
        int *h = S->h_tiles + (size_t)l * kTabWords;
        h[0] = nt[l];
        h[1] = tot[l];
        h[2] = S->cpw;
        h[3] = 0;
        h[4] = W1[l];
        h[5] = W2[l];
        h[6] = h[7] = 0;
        S->lane_nt[l] = nt[l];
        all += nt[l];
    }
    return all;
}

// Copy the used part of every lane's table to the device.
cudaError_t upload_tables(b200la_server *S, cudaStream_t st)
{
    for (int l = 0; l < S->lanes; ++l) {
        const size_t off = (size_t)l * kTabWords;
        const cudaError_t e = cudaMemcpyAsync(S->d_tiles + off, S->h_tiles + off,
                                              sizeof(int) * b200::srv::kTabHdrWords + sizeof(SysRun) * (size_t)S->lane_nt[l],
                                              cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int run_round(b200la_server *S, const std::vector<ActiveSys> &act)
{
    NvtxScope nvtx_range("b200la_serve_round");
    write_table(S, act);
    cudaStream_t st = S->s_comp;
    SV(upload_tables(S, st));
    SV(cudaEventRecord(S->ev_a, st));
    SV(cudaGraphLaunch(S->graph, st));
    SV(cudaEventRecord(S->ev_b, st));
    SV(cudaMemcpyAsync(S->h_done, S->d_done, sizeof(int) * (size_t)S->cfg.max_slots, cudaMemcpyDeviceToHost, st));
    SV(cudaStreamSynchronize(st));
    float ms = 0.f;
    SV(cudaEventElapsedTime(&ms, S->ev_a, S->ev_b));
    S->busy_ms += ms;
    return 0;
}

void round_loop(b200la_server *S)
{
    cudaSetDevice(S->device);
    std::vector<ActiveSys> act;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_round.wait(lk, [S] { return S->quit || !S->ready.empty() || !S->active.empty(); });
            if (S->quit && S->active.empty() && S->ready.empty()) return;
            double wb = 0.0;
            long long wsum = 0;   // weighted chunk positions (int32 in the table)
            for (Slot *sl : S->active) {
                wb += sl->req->iter_bytes;
                wsum += (long long)sl->desc.nchunks * std::max(sl->req->w1, sl->req->w2);
            }
            while (!S->ready.empty() && (int)S->active.size() < std::min(S->max_active, kTabCap)) {
                auto it = S->ready.begin();
                if (S->lpt)
                    it = std::max_element(S->ready.begin(), S->ready.end(), [](const Slot *a, const Slot *b) {
                        return a->req->work < b->req->work;
                    });
                Slot *sl = *it;
                const bool room = S->active.empty() || wb + sl->req->iter_bytes <= S->active_cap;
                const long long ws = (long long)sl->desc.nchunks * std::max(sl->req->w1, sl->req->w2);
                if (!room || wsum + ws >= (1LL << 31)) break;
                wb += sl->req->iter_bytes;
                wsum += ws;
                S->ready.erase(it);
                S->active.push_back(sl);
            }
            S->peak_active = std::max(S->peak_active, (int)S->active.size());
            if (S->active.empty()) continue;
            act.clear();
            for (Slot *sl : S->active)
                act.push_back(ActiveSys{sl->idx, sl->desc.nchunks, sl->req->w1, sl->req->w2, sl->req->iter_bytes});
        }
        const int rc = S->fatal ? S->fatal : run_round(S, act);
        std::lock_guard<std::mutex> lk(S->mu);
        if (rc && !S->fatal) fail_all(S, B200LA_ERR_CUDA);
        if (S->fatal) {
            for (Slot *sl : S->active) {
                finish(S, sl->req, S->fatal);
                delete sl;
            }
            S->active.clear();
            continue;
        }
        ++S->rounds;
        S->batch_iters += S->iters;
        std::vector<Slot *> keep;
        keep.reserve(S->active.size());
        for (Slot *sl : S->active) {
            if (S->h_done[sl->idx] != 0) S->retire_q.push_back(sl);
            else keep.push_back(sl);
        }
        S->active.swap(keep);
        S->cv_admit.notify_one();
    }
}

void gmres_loop(b200la_server *S)
{
    cudaSetDevice(S->device);
    b200la_ctx *ctx = nullptr;
    const bool ok = b200la_create(S->device, &ctx) == B200LA_OK;
    for (;;) {
        Req *q = nullptr;
        size_t need = 0;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_gm.wait(lk, [&] {
                if (S->quit || S->gm_pending.empty()) return S->quit || false;
                return S->resident + (double)gmres_bytes(S->gm_pending.front()) <= S->cfg.budget_bytes;
            });
            if (S->gm_pending.empty()) {
                if (S->quit) break;
                continue;
            }
            q = S->gm_pending.front();
            S->gm_pending.pop_front();
            need = gmres_bytes(q);
            S->resident += (double)need;
            S->peak_resident = std::max(S->peak_resident, S->resident);
            q->res.t_admit = S->now();
        }
        q->res.bytes = (double)need;
        int rc = ok ? B200LA_OK : B200LA_ERR_DEVICE;
        const b200la_request &r = q->r;
        const int n = q->n;
        std::vector<int> hrow, hcol;
        std::vector<double> hval, hb(n), hx(n, 0.0);
        const int *row = r.row, *col = r.col;
        const double *val = r.val;
        if (!rc && !row) {
            hrow.resize(n + 1);
            hcol.resize(q->nnz);
            hval.resize(q->nnz);
            double beta[3] = {r.q1_beta[0], r.q1_beta[1], r.q1_beta[2]};
            if (b200::host::q1_assemble(r.q1_dim, r.q1_N, r.q1_kind, r.q1_kcell, r.q1_nu, beta, hrow.data(),
                                        hcol.data(), hval.data()))
                rc = B200LA_ERR_ARG;
            row = hrow.data();
            col = hcol.data();
            val = hval.data();
        }
        if (r.b) std::copy(r.b, r.b + n, hb.begin());
        else b200::host::q1_rhs(r.rhs_seed, r.q1_dim, r.q1_N, hb.data());
        b200la_csr *A = nullptr, *Ap = nullptr;
        b200la_precond *P = nullptr;
        void *db = nullptr, *dx = nullptr;
        std::vector<int> perm;
        b200la_result res{};
        const bool ilu = r.gmres_precond == B200LA_PRECOND_ILU0_LS;
        if (!rc) {
            if (ilu) {
                rc = b200la_precond_ilu0(ctx, n, row, col, val, B200LA_PRECOND_ILU0_LS, B200LA_F64, &P, &Ap);
                if (!rc) {
                    perm.resize(n);
                    std::vector<int> sizes(n);
                    int kind, nn, nb;
                    rc = b200la_precond_info(P, &kind, &nn, &nb, sizes.data(), perm.data());
                }
            } else {
                rc = b200la_csr_create(ctx, n, n, (int)q->nnz, row, col, val, B200LA_F64, &A);
                if (!rc && r.gmres_precond == B200LA_PRECOND_JACOBI) rc = b200la_precond_jacobi(ctx, A, &P);
            }
        }
        if (!rc) rc = b200la_malloc(ctx, 8 * (size_t)n, &db);
        if (!rc) rc = b200la_malloc(ctx, 8 * (size_t)n, &dx);
        if (!rc) {
            std::vector<double> bp(n);
            for (int i = 0; i < n; ++i) bp[i] = ilu ? hb[perm[i]] : hb[i];
            rc = b200la_memcpy_h2d(ctx, db, bp.data(), 8 * (size_t)n);
            if (!rc) rc = b200la_memset_zero(ctx, dx, 8 * (size_t)n);
            q->res.t_ready = S->now();
            if (!rc) rc = b200la_gmres(ctx, ilu ? Ap : A, P, std::max(r.gmres_m, 1), db, dx, &r.ctl, &res);
            if (!rc) {
                std::vector<double> xp(n);
                rc = b200la_memcpy_d2h(ctx, xp.data(), dx, 8 * (size_t)n);
                if (!rc) rc = b200la_sync(ctx);
                for (int i = 0; i < n && !rc; ++i) {
                    if (ilu) r.x[perm[i]] = xp[i];
                    else r.x[i] = xp[i];
                }
            }
        }
        if (db) b200la_free(ctx, db);
        if (dx) b200la_free(ctx, dx);
        if (P) b200la_precond_destroy(P);
        if (A) b200la_csr_destroy(A);
        if (Ap) b200la_csr_destroy(Ap);
        std::lock_guard<std::mutex> lk(S->mu);
        S->resident -= (double)need;
        q->res.status = res.status;
        q->res.iters = res.iters;
        q->res.res0 = res.res0;
        q->res.res = res.res;
        finish(S, q, rc);
        S->cv_admit.notify_all();
    }
    if (ctx) b200la_destroy(ctx);
}

// ------------------------------------------------------------- graph + tuning

int capture_graph(b200la_server *S)
{
    if (S->graph) {
        cudaGraphExecDestroy(S->graph);
        S->graph = nullptr;
    }
    const int grid = S->num_sms * S->ctas_per_sm;
    cudaGraph_t g = nullptr;
    SV(cudaStreamBeginCapture(S->s_comp, cudaStreamCaptureModeThreadLocal));
    // lane 0 on the capture stream, the others forked onto their own streams
    cudaError_t e = S->lanes > 1 ? cudaEventRecord(S->ev_fork, S->s_comp) : cudaSuccess;
    for (int l = 1; l < S->lanes && e == cudaSuccess; ++l) e = cudaStreamWaitEvent(S->s_lane[l], S->ev_fork, 0);
    for (int k = 0; k < S->iters && e == cudaSuccess; ++k)
        for (int l = 0; l < S->lanes && e == cudaSuccess; ++l)
            e = b200::srv::launch_round(S->nw, grid, S->d_sys, S->d_state, S->d_tiles + (size_t)l * kTabWords,
                                        l ? S->s_lane[l] : S->s_comp);
    for (int l = 1; l < S->lanes && e == cudaSuccess; ++l) {
        e = cudaEventRecord(S->ev_join[l], S->s_lane[l]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(S->s_comp, S->ev_join[l], 0);
    }
    const cudaError_t e2 = cudaStreamEndCapture(S->s_comp, &g);
    if (e != cudaSuccess) return -(int)e;
    if (e2 != cudaSuccess) return -(int)e2;
    e = cudaGraphInstantiate(&S->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return -(int)e;
    return 0;
}

// Time the candidate kernel shapes on a calibration batch of Q1 systems (one
// captured round each, lanes concurrent) and keep the fastest.  No shape
// changes any system's arithmetic.
int autotune(b200la_server *S)
{
    struct Cal {
        int dim, N;
    };
    const Cal cal[] = {{2, 512}, {2, 384}, {2, 256}, {2, 192}, {2, 128}, {2, 96}, {2, 64},
                       {2, 48},  {3, 64},  {3, 48},  {3, 32},  {3, 24},  {3, 16}};
    std::vector<std::unique_ptr<Req>> rq;
    std::vector<Slot *> slots;
    int rc = 0;
    for (size_t k = 0; k < sizeof cal / sizeof cal[0] && !rc; ++k) {
        auto q = std::make_unique<Req>();
        q->r.method = B200LA_SERVE_CG;
        q->r.precision = (k & 1) ? B200LA_SERVE_MIXED : B200LA_SERVE_F64;
        q->r.q1_dim = cal[k].dim;
        q->r.q1_N = cal[k].N;
        q->r.rhs_seed = 7 + k;
        q->r.ctl = b200la_control{1 << 30, 0.0, 0.0, 1e300};
        q->r.inner = b200la_control{1 << 30, 0.0, 1e-4, 1e300};
        q->r.max_outer = 1 << 30;
        rc = plan_request(S, q.get());
        if (rc) break;
        Slot *sl = new Slot();
        sl->idx = S->free_idx.back();
        S->free_idx.pop_back();
        sl->req = q.get();
        rc = admit_slot(S, q.get(), sl);
        slots.push_back(sl);
        rq.push_back(std::move(q));
    }
    struct Shape {
        int nw, cps, cpw;
    };
    const Shape shapes[] = {{8, 4, 4}, {8, 2, 4}, {8, 3, 4}, {8, 6, 4}, {4, 8, 4}, {4, 4, 4}};
    float best = 1e30f;
    Shape pick{S->nw, S->ctas_per_sm, S->cpw};
    std::vector<ActiveSys> act;
    for (Slot *sl : slots)
        act.push_back(ActiveSys{sl->idx, sl->desc.nchunks, sl->req->w1, sl->req->w2, sl->req->iter_bytes});
    for (const Shape &sh : shapes) {
        if (rc) break;
        S->nw = sh.nw;
        S->ctas_per_sm = sh.cps;
        S->cpw = sh.cpw;
        write_table(S, act);
        cudaStream_t st = S->s_comp;
        if (upload_tables(S, st) != cudaSuccess) {
            rc = -1;
            break;
        }
        // time the round exactly as it will run: the captured graph of this
        // shape, with the lanes' kernel chains concurrent
        if (capture_graph(S)) {
            rc = -1;
            break;
        }
        if (cudaGraphLaunch(S->graph, st) != cudaSuccess) rc = -1;
        cudaEventRecord(S->ev_a, st);
        for (int k = 0; k < 2 && !rc; ++k)
            if (cudaGraphLaunch(S->graph, st) != cudaSuccess) rc = -1;
        cudaEventRecord(S->ev_b, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, S->ev_a, S->ev_b);
        if (!rc && ms < best) {
            best = ms;
            pick = sh;
        }
    }
    S->nw = pick.nw;
    S->ctas_per_sm = pick.cps;
    S->cpw = pick.cpw;
    for (Slot *sl : slots) {
        cudaFreeAsync(sl->block, S->s_copy);
        S->free_idx.push_back(sl->idx);
        delete sl;
    }
    cudaStreamSynchronize(S->s_copy);
    return rc;
}

void destroy_server(b200la_server *S)
{
    if (S->graph) cudaGraphExecDestroy(S->graph);
    if (S->s_comp) cudaStreamSynchronize(S->s_comp);
    if (S->s_copy) cudaStreamSynchronize(S->s_copy);
    cudaFree(S->d_sys);
    cudaFree(S->d_state);
    cudaFree(S->d_ticket);
    cudaFree(S->d_done);
    cudaFree(S->d_tiles);
    cudaFreeHost(S->h_done);
    cudaFreeHost(S->h_tiles);
    if (S->h_admit) cudaFreeHost(S->h_admit);
    if (S->h_kc) cudaFreeHost(S->h_kc);
    if (S->ev_a) cudaEventDestroy(S->ev_a);
    if (S->ev_b) cudaEventDestroy(S->ev_b);
    if (S->ev_fork) cudaEventDestroy(S->ev_fork);
    for (int l = 1; l < kLanes; ++l) {
        if (S->ev_join[l]) cudaEventDestroy(S->ev_join[l]);
        if (S->s_lane[l]) cudaStreamDestroy(S->s_lane[l]);
    }
    if (S->s_comp) cudaStreamDestroy(S->s_comp);
    if (S->s_copy) cudaStreamDestroy(S->s_copy);
    if (S->pool) cudaMemPoolDestroy(S->pool);
    delete S;
}

}  // namespace

// ------------------------------------------------------------------ C ABI

extern "C" int b200la_serve_start(const b200la_serve_config *cfg, b200la_server **out)
{
    if (!out) return B200LA_ERR_ARG;
    *out = nullptr;
    b200la_server *S = new b200la_server();
    if (cfg) S->cfg = *cfg;
    b200la_serve_config &c = S->cfg;
    if (c.budget_bytes <= 0) c.budget_bytes = 60e9;
    if (c.max_slots <= 0) c.max_slots = 4096;
    if (c.max_active <= 0) c.max_active = 1024;
    if (c.iters_per_round <= 0) c.iters_per_round = 16;
    if (c.active_bytes <= 0) c.active_bytes = 4096.0 * 1024 * 1024;
    S->device = c.device;
    S->iters = c.iters_per_round;
    S->active_cap = c.active_bytes;
    S->max_active = std::min(c.max_active, c.max_slots);
    if (c.warps == 4 || c.warps == 8) S->nw = c.warps;
    if (c.ctas_per_sm > 0) S->ctas_per_sm = std::min(c.ctas_per_sm, S->nw == 4 ? 16 : 8);
    if (c.chunks_per_warp > 0) S->cpw = c.chunks_per_warp;
    S->t0 = std::chrono::steady_clock::now();
    cudaDeviceProp prop;
    if (cudaSetDevice(S->device) != cudaSuccess || cudaGetDeviceProperties(&prop, S->device) != cudaSuccess ||
        prop.major < 10) {
        delete S;
        return B200LA_ERR_DEVICE;
    }
    S->num_sms = prop.multiProcessorCount;
    cudaMemPoolProps pp{};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = S->device;
    bool ok = cudaMemPoolCreate(&S->pool, &pp) == cudaSuccess;
    if (ok) {
        uint64_t keep = ~0ULL;
        ok = cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep) == cudaSuccess;
    }
    if (const char *ln = std::getenv("B200LA_SERVE_LANES")) S->lanes = std::max(1, std::min(kLanes, std::atoi(ln)));
    if (const char *o = std::getenv("B200LA_SERVE_LPT")) S->lpt = std::atoi(o) != 0;
    ok = ok && cudaStreamCreateWithFlags(&S->s_comp, cudaStreamNonBlocking) == cudaSuccess &&
         cudaStreamCreateWithFlags(&S->s_copy, cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreate(&S->ev_a) == cudaSuccess && cudaEventCreate(&S->ev_b) == cudaSuccess &&
         cudaEventCreateWithFlags(&S->ev_fork, cudaEventDisableTiming) == cudaSuccess;
    for (int l = 1; l < kLanes; ++l)
        ok = ok && cudaStreamCreateWithFlags(&S->s_lane[l], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&S->ev_join[l], cudaEventDisableTiming) == cudaSuccess;
    const size_t ms = (size_t)c.max_slots;
    ok = ok && cudaMalloc(&S->d_sys, sizeof(SysDesc) * ms) == cudaSuccess &&
         cudaMalloc(&S->d_state, sizeof(SysState) * ms) == cudaSuccess &&
         cudaMalloc(&S->d_ticket, sizeof(unsigned) * b200::srv::kTicketWords * ms) == cudaSuccess &&
         cudaMalloc(&S->d_done, sizeof(int) * ms) == cudaSuccess &&
         cudaMalloc(&S->d_tiles, sizeof(int) * kTabWords * kLanes) == cudaSuccess &&
         cudaMallocHost(&S->h_done, sizeof(int) * ms) == cudaSuccess &&
         cudaMallocHost(&S->h_tiles, sizeof(int) * kTabWords * kLanes) == cudaSuccess &&
         cudaMallocHost(&S->h_admit, sizeof(b200la_server::AdmitStage)) == cudaSuccess;
    ok = ok && cudaMemset(S->d_done, 0, sizeof(int) * ms) == cudaSuccess &&
         cudaMemset(S->d_tiles, 0, sizeof(int) * kTabWords * kLanes) == cudaSuccess &&
         cudaMemset(S->d_sys, 0, sizeof(SysDesc) * ms) == cudaSuccess;
    if (!ok) {
        destroy_server(S);
        return B200LA_ERR_ALLOC;
    }
    for (int i = c.max_slots - 1; i >= 0; --i) S->free_idx.push_back(i);
    if (c.autotune && autotune(S)) {
        destroy_server(S);
        return B200LA_ERR_CUDA;
    }
    if (capture_graph(S)) {
        destroy_server(S);
        return B200LA_ERR_CUDA;
    }
    S->th_admit = std::thread(admit_loop, S);
    S->th_round = std::thread(round_loop, S);
    S->th_gm = std::thread(gmres_loop, S);
    *out = S;
    return B200LA_OK;
}

extern "C" int b200la_serve_submit(b200la_server *S, const b200la_request *req, long long *id)
{
    if (!S || !req || !id || !req->x) return B200LA_ERR_ARG;
    if (req->method != B200LA_SERVE_CG && req->method != B200LA_SERVE_GMRES) return B200LA_ERR_ARG;
    if (req->precision != B200LA_SERVE_F64 && req->precision != B200LA_SERVE_MIXED) return B200LA_ERR_ARG;
    if (req->method == B200LA_SERVE_GMRES && req->precision != B200LA_SERVE_F64) return B200LA_ERR_ARG;
    auto q = std::make_unique<Req>();
    q->r = *req;
    const int rc = plan_request(S, q.get());
    if (rc) return rc;
    const double need = req->method == B200LA_SERVE_GMRES ? (double)gmres_bytes(q.get())
                                                           : (double)(q->bytes + q->temp_bytes);
    if (need > S->cfg.budget_bytes) return B200LA_ERR_BUDGET;
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->fatal) return S->fatal;
    q->id = S->next_id++;
    q->res.t_submit = S->now();
    *id = q->id;
    Req *raw = q.get();
    S->reqs.emplace(q->id, std::move(q));
    ++S->submitted;
    if (req->method == B200LA_SERVE_GMRES) {
        S->gm_pending.push_back(raw);
        S->cv_gm.notify_all();
    } else {
        S->pending.push_back(raw);
        S->cv_admit.notify_one();
    }
    return B200LA_OK;
}

extern "C" int b200la_serve_poll(b200la_server *S, long long id, b200la_serve_result *res)
{
    if (!S) return B200LA_ERR_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return B200LA_ERR_NOTFOUND;
    if (!it->second->done) return B200LA_PENDING;
    if (res) *res = it->second->res;
    return B200LA_OK;
}

extern "C" int b200la_serve_wait(b200la_server *S, long long id, double timeout_s, b200la_serve_result *res)
{
    if (!S) return B200LA_ERR_ARG;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return B200LA_ERR_NOTFOUND;
    Req *q = it->second.get();
    S->cv_done.wait_for(lk, std::chrono::duration<double>(std::max(timeout_s, 0.0)), [q] { return q->done; });
    if (!q->done) return B200LA_PENDING;
    if (res) *res = q->res;
    return B200LA_OK;
}

extern "C" int b200la_serve_stats(b200la_server *S, b200la_serve_info *out)
{
    if (!S || !out) return B200LA_ERR_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    out->submitted = S->submitted;
    out->completed = S->completed;
    out->failed = S->failed;
    out->rounds = S->rounds;
    out->batch_iters = S->batch_iters;
    out->busy_ms = S->busy_ms;
    out->resident_bytes = S->resident;
    out->peak_resident_bytes = S->peak_resident;
    out->peak_active = S->peak_active;
    out->warps = S->nw;
    out->ctas_per_sm = S->ctas_per_sm;
    out->chunks_per_warp = S->cpw;
    out->iters_per_round = S->iters;
    out->active_bytes = S->active_cap;
    return B200LA_OK;
}

extern "C" int b200la_serve_stop(b200la_server *S)
{
    if (!S) return B200LA_ERR_ARG;
    {
        std::unique_lock<std::mutex> lk(S->mu);
        S->cv_done.wait(lk, [S] { return S->completed + S->failed >= S->submitted; });
        S->quit = true;
    }
    S->cv_admit.notify_all();
    S->cv_round.notify_all();
    S->cv_gm.notify_all();
    S->th_admit.join();
    S->th_round.join();
    S->th_gm.join();
    const int rc = S->fatal;
    destroy_server(S);
    return rc ? rc : B200LA_OK;
}
