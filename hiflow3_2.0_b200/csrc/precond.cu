// precond.cu -- preconditioners of the B200 lmp platform.
//
// Jacobi: z = r .* (1/a_ii)              (lmp/lpreconditioner.cc:127-165)
// Block sweeps in the permuted numbering (lmp/lpreconditioner_mc.cc:716-728):
//   MC symmetric Gauss-Seidel            (lmp/lpreconditioner_mc_sgs.cc, _gs.cc)
//   ILU(0), level-scheduled or coloured  (lmp/lpreconditioner_mc_ilup.cc)
// The reference stores the c(c-1) off-diagonal colour blocks as separate
// matrices and launches one SpMV per block; here the permuted factor is split
// once into L (columns in earlier blocks) and U (columns in later blocks), each
// with one tile schedule per block, so a sweep is one launch per block whose
// epilogue applies the diagonal scaling in the same pass.
#include "b200la.h"
#include "b200la_internal.h"

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <string>
#include <vector>

using namespace b200;

static int pfail(b200la_ctx *ctx, int code, const std::string &m)
{
    if (ctx) ctx->msg = m;
    return code;
}

extern "C" int b200la_precond_jacobi(b200la_ctx *ctx, const b200la_csr *A, b200la_precond **out)
{
    if (!ctx || !A || !out || A->n != A->m) return pfail(ctx, B200LA_ERR_ARG, "precond_jacobi: invalid argument");
    b200la_precond *P = new b200la_precond();
    P->kind = B200LA_PRECOND_JACOBI;
    P->n = A->n;
    P->dtype = A->dtype;
    const size_t es = A->dtype == B200LA_F64 ? 8 : 4;
    cudaError_t e = cudaMalloc(&P->invd, es * std::max(A->n, 1));
    if (e != cudaSuccess) {
        delete P;
        return ctx_fail(ctx, B200LA_ERR_ALLOC, "precond_jacobi", e);
    }
    if ((e = launch_invdiag(A->dtype, A->n, A->row, A->col, A->val, P->invd, ctx->stream)) ||
        (e = cudaStreamSynchronize(ctx->stream))) {
        b200la_precond_destroy(P);
        return ctx_fail(ctx, B200LA_ERR_CUDA, "precond_jacobi", e);
    }
    *out = P;
    return B200LA_OK;
}

// Upload a double-precision host vector in dtype.
static int upload_vec(b200la_ctx *ctx, const std::vector<double> &v, int dtype, void **out)
{
    const size_t n = v.size(), es = dtype == B200LA_F64 ? 8 : 4;
    cudaError_t e = cudaMalloc(out, es * std::max<size_t>(n, 1));
    if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_ALLOC, "precond upload", e);
    if (dtype == B200LA_F64) {
        e = cudaMemcpy(*out, v.data(), 8 * n, cudaMemcpyHostToDevice);
    } else {
        std::vector<float> f(v.begin(), v.end());
        e = cudaMemcpy(*out, f.data(), 4 * n, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "precond upload", e);
    return B200LA_OK;
}

static int upload_csr(b200la_ctx *ctx, const host::Csr &M, int dtype, const std::vector<int> &segs,
                      b200la_csr **out)
{
    const int nseg = (int)segs.size() - 1;
    if (dtype == B200LA_F64)
        return csr_upload(ctx, M.n, M.m, M.nnz(), M.row.data(), M.col.data(), M.val.data(), dtype, nseg,
                          nseg > 0 ? segs.data() : nullptr, out);
    std::vector<float> f(M.val.begin(), M.val.end());
    return csr_upload(ctx, M.n, M.m, M.nnz(), M.row.data(), M.col.data(), f.data(), dtype, nseg,
                      nseg > 0 ? segs.data() : nullptr, out);
}

static int build_block(b200la_ctx *ctx, int kind, int n, const int *row, const int *col, const double *val,
                       double omega, int dtype, b200la_precond **out, b200la_csr **A_perm, int ilu_p = 0,
                       int mat_power = 1)
{
    if (!ctx || n < 1 || !row || !col || !val || !out || (dtype != B200LA_F64 && dtype != B200LA_F32))
        return pfail(ctx, B200LA_ERR_ARG, "precond: invalid argument");
    if (!(omega > 0.0 && omega < 2.0)) return pfail(ctx, B200LA_ERR_ARG, "precond: omega must lie in (0, 2)");
    long long bad = -1;
    if (host::validate_csr(n, n, row[n], row, col, &bad)) return pfail(ctx, B200LA_ERR_CSR, "precond: malformed CSR");
    for (int i = 0; i < n; ++i) {
        bool d = false;
        for (int j = row[i]; j < row[i + 1]; ++j) d |= (col[j] == i && val[j] != 0.0);
        if (!d) return pfail(ctx, B200LA_ERR_SETUP, "precond: row " + std::to_string(i) + " has no nonzero diagonal");
    }
    host::Csr A;
    A.n = A.m = n;
    A.row.assign(row, row + n + 1);
    A.col.assign(col, col + row[n]);
    A.val.assign(val, val + row[n]);
    std::vector<int> sizes, perm;
    int nb = 0;
    host::Csr Ap, LU;
    if (kind == B200LA_PRECOND_ILU0_LS) {
        // ilu0 in natural order, level scheduling of the factor, permute_all
        // (lpreconditioner_mc.cc:176-192, 310-351)
        host::Csr F = A;
        if (ilu_p > 0) host::ilup(A, ilu_p, F);
        else host::ilu0(n, F.row.data(), F.col.data(), F.val.data());
        if (host::levelscheduling(n, F.row.data(), F.col.data(), &nb, sizes, perm))
            return pfail(ctx, B200LA_ERR_SETUP, "precond: level scheduling did not complete");
        host::reorder(A, perm, Ap);
        host::reorder(F, perm, LU);
    } else {
        // colours of the analysis matrix: the operator, or the pattern of its
        // mat_power-th power (build_aux_matrix, lpreconditioner_mc_ilup.cc:107-140)
        host::Csr aux;
        if (mat_power > 1) host::matrix_sup_power(A, mat_power, aux);
        const host::Csr &an = mat_power > 1 ? aux : A;
        if (host::multicoloring(n, an.row.data(), an.col.data(), &nb, sizes, perm))
            return pfail(ctx, B200LA_ERR_SETUP, "precond: multicolouring found no colours");
        host::reorder(A, perm, Ap);
        LU = Ap;
        if (kind == B200LA_PRECOND_ILU0_MC) {
            if (ilu_p > 0) host::ilup(Ap, ilu_p, LU);
            else host::ilu0(n, LU.row.data(), LU.col.data(), LU.val.data());
        }
    }
    std::vector<int> off(nb + 1, 0);
    for (int b = 0; b < nb; ++b) off[b + 1] = off[b] + sizes[b];
    host::dropoffs(LU, off);
    const bool sgs = (kind == B200LA_PRECOND_MCSGS);
    const double w = sgs ? omega : 1.0;
    // ScaleOffdiag(omega) and the scaled diagonal vectors (scale_D)
    std::vector<int> blk(n);
    for (int b = 0; b < nb; ++b)
        for (int i = off[b]; i < off[b + 1]; ++i) blk[i] = b;
    std::vector<double> Dv(n, 0.0), iDv(n, 0.0);
    host::Csr L, U;
    L.n = U.n = L.m = U.m = n;
    L.row.assign(n + 1, 0);
    U.row.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        for (int j = LU.row[i]; j < LU.row[i + 1]; ++j) {
            const int c = LU.col[j];
            if (c == i) {
                Dv[i] = LU.val[j];
                iDv[i] = 1 / LU.val[j];
                continue;
            }
            const double v = LU.val[j] * w;
            if (blk[c] < blk[i]) {
                L.col.push_back(c);
                L.val.push_back(v);
            } else if (blk[c] > blk[i]) {
                U.col.push_back(c);
                U.val.push_back(v);
            }
            // same-block couplings were dropped above
        }
        L.row[i + 1] = (int)L.col.size();
        U.row[i + 1] = (int)U.col.size();
    }
    for (int i = 0; i < n; ++i) {
        if (Dv[i] == 0.0) return pfail(ctx, B200LA_ERR_SETUP, "precond: zero pivot in row " + std::to_string(i));
        iDv[i] *= -1.0;
        if (sgs) {
            Dv[i] *= -1.0;
            Dv[i] *= 1.0 / (w * (2.0 - w));
        }
    }
    b200la_precond *P = new b200la_precond();
    P->kind = kind;
    P->n = n;
    P->dtype = dtype;
    P->nblocks = nb;
    P->block_off = off;
    P->perm = perm;
    int rc;
    if ((rc = upload_csr(ctx, L, dtype, off, &P->L)) || (rc = upload_csr(ctx, U, dtype, off, &P->U)) ||
        (rc = upload_vec(ctx, Dv, dtype, &P->Dv)) || (rc = upload_vec(ctx, iDv, dtype, &P->iDv))) {
        b200la_precond_destroy(P);
        return rc;
    }
    cudaError_t e = cudaMalloc(&P->perm_dev, sizeof(int) * n);
    if (e == cudaSuccess) e = cudaMemcpy(P->perm_dev, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        b200la_precond_destroy(P);
        return ctx_fail(ctx, B200LA_ERR_CUDA, "precond perm", e);
    }
    rc = syncfree_setup(ctx, P);
    if (rc) {
        b200la_precond_destroy(P);
        return rc;
    }
    if (A_perm) {
        rc = upload_csr(ctx, Ap, dtype, std::vector<int>(), A_perm);
        if (rc) {
            b200la_precond_destroy(P);
            return rc;
        }
    }
    // a parity-coloured structured Q1 grid: index-free lattice layouts of the
    // sweeps' two parts and of the coloured operator (the CSR stays for
    // everything else, and is used alone when any entry does not fit)
    int mx, my, mz;
    if (kind != B200LA_PRECOND_ILU0_LS && lattice::grid(n, row, col, &mx, &my, &mz) &&
        lattice::perm_ok(mx, my, mz, perm, off)) {
        if ((rc = lattice_attach(ctx, P->L, L, mx, my, mz, 0)) || (rc = lattice_attach(ctx, P->U, U, mx, my, mz, 1)) ||
            (A_perm && (rc = lattice_attach(ctx, *A_perm, Ap, mx, my, mz, 2)))) {
            if (A_perm) {
                b200la_csr_destroy(*A_perm);
                *A_perm = nullptr;
            }
            b200la_precond_destroy(P);
            return rc;
        }
    }
    *out = P;
    return B200LA_OK;
}

extern "C" int b200la_precond_mcsgs(b200la_ctx *ctx, int n, const int *row, const int *col, const double *val,
                                    double omega, int dtype, b200la_precond **out, b200la_csr **A_perm)
{
    return build_block(ctx, B200LA_PRECOND_MCSGS, n, row, col, val, omega, dtype, out, A_perm);
}

extern "C" int b200la_precond_ilu0(b200la_ctx *ctx, int n, const int *row, const int *col, const double *val,
                                   int mode, int dtype, b200la_precond **out, b200la_csr **A_perm)
{
    if (mode != B200LA_PRECOND_ILU0_LS && mode != B200LA_PRECOND_ILU0_MC)
        return pfail(ctx, B200LA_ERR_ARG, "precond_ilu0: mode must be ILU0_LS or ILU0_MC");
    return build_block(ctx, mode, n, row, col, val, 1.0, dtype, out, A_perm);
}

extern "C" int b200la_precond_ilup(b200la_ctx *ctx, int n, const int *row, const int *col, const double *val,
                                   int mode, int ilu_p, int mat_power, int dtype, b200la_precond **out,
                                   b200la_csr **A_perm)
{
    if (mode != B200LA_PRECOND_ILU0_LS && mode != B200LA_PRECOND_ILU0_MC)
        return pfail(ctx, B200LA_ERR_ARG, "precond_ilup: mode must be ILU0_LS or ILU0_MC");
    if (ilu_p < 0 || mat_power < 1 || (mode == B200LA_PRECOND_ILU0_LS && mat_power != 1))
        return pfail(ctx, B200LA_ERR_ARG, "precond_ilup: ilu_p >= 0, mat_power >= 1 (1 with level scheduling)");
    return build_block(ctx, mode, n, row, col, val, 1.0, dtype, out, A_perm, ilu_p, mat_power);
}

extern "C" int b200la_precond_info(const b200la_precond *P, int *kind, int *n, int *nblocks, int *block_sizes,
                                   int *perm)
{
    if (!P) return B200LA_ERR_ARG;
    if (kind) *kind = P->kind;
    if (n) *n = P->n;
    if (nblocks) *nblocks = P->nblocks;
    if (block_sizes)
        for (int b = 0; b < P->nblocks; ++b) block_sizes[b] = P->block_off[b + 1] - P->block_off[b];
    if (perm && !P->perm.empty()) std::copy(P->perm.begin(), P->perm.end(), perm);
    return B200LA_OK;
}

int precond_apply_async(b200la_ctx *ctx, const b200la_precond *P, const void *r, void *z, const int *gate)
{
    if (P->kind == B200LA_PRECOND_JACOBI) {
        cudaError_t e = launch_jacobi(P->dtype, P->n, P->invd, r, z, gate, ctx->stream);
        if (e != cudaSuccess) return ctx_fail(ctx, B200LA_ERR_CUDA, "jacobi apply", e);
        ctx->launches += 1;
        return B200LA_OK;
    }
    if (P->use_syncfree) return syncfree_apply(ctx, P, r, z, gate);
    const bool sgs = (P->kind == B200LA_PRECOND_MCSGS);
    // on the lattice layout the last block's backward step has no couplings:
    // it runs in the epilogue of that block's forward step (one launch less)
    const int nb = P->nblocks;
    int c0, c1;
    const bool fuse = nb > 1 && P->L->lt && P->U->lt && P->U->lt->ncol == nb && P->U->lt->col[nb - 1].nslot == 0 &&
                      lattice_segment(P->L, P->L->segs[nb], &c0, &c1) && !std::getenv("B200LA_NOFUSE_LAST");
    // lattice sweeps after the first launch as programmatic dependents of the
    // previous one (B200LA_PDL=0: plain stream order)
    const char *pe = std::getenv("B200LA_PDL");
    const int pdl = (P->L->lt && P->U->lt && (!pe || std::atoi(pe) != 0)) ? 1 : 0;
    // forward sweep over the blocks: z_i from r_i and the already-final z of earlier blocks
    for (int b = 0; b < nb; ++b) {
        SpmvOp op;
        op.epi = sgs ? EPI_SGS_F : EPI_ILU_F;
        if (fuse && b == nb - 1) op.epi = sgs ? EPI_SGS_FB : EPI_ILU_FB;
        op.pdl = b > 0 ? pdl : 0;   // the first waits for the whole stream (the gate is read before any wait)
        op.x = z;
        op.y = z;
        op.b = r;
        op.d1 = P->iDv;
        op.d2 = P->Dv;
        op.gate = gate;
        int rc = spmv_run(ctx, P->L, P->L->segs[1 + b], op);
        if (rc) return rc;
    }
    // diagonal step folded into the backward sweep, blocks in reverse order
    for (int b = nb - 1 - (fuse ? 1 : 0); b >= 0; --b) {
        SpmvOp op;
        op.epi = sgs ? EPI_SGS_B : EPI_ILU_B;
        op.pdl = pdl;
        op.x = z;
        op.y = z;
        op.d1 = P->iDv;
        op.d2 = P->Dv;
        op.gate = gate;
        int rc = spmv_run(ctx, P->U, P->U->segs[1 + b], op);
        if (rc) return rc;
    }
    return B200LA_OK;
}

extern "C" int b200la_precond_apply(b200la_ctx *ctx, const b200la_precond *P, const void *r, void *z)
{
    if (!ctx || !P || !r || !z || r == z) return pfail(ctx, B200LA_ERR_ARG, "precond_apply: invalid argument");
    return precond_apply_async(ctx, P, r, z, nullptr);
}

extern "C" int b200la_precond_destroy(b200la_precond *P)
{
    if (!P) return B200LA_OK;
    cudaDeviceSynchronize();
    if (P->invd) cudaFree(P->invd);
    if (P->L) b200la_csr_destroy(P->L);
    if (P->U) b200la_csr_destroy(P->U);
    if (P->Dv) cudaFree(P->Dv);
    if (P->iDv) cudaFree(P->iDv);
    if (P->perm_dev) cudaFree(P->perm_dev);
    syncfree_free(P);
    if (P->flags) cudaFree(P->flags);
    if (P->sync) cudaFree(P->sync);
    delete P;
    return B200LA_OK;
}
