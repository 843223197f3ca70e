// ref_driver.cc -- C entry points over HiFlow3's own CPU lmp classes.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the reference's unmodified CPU lmp sources (src/linear_algebra/lmp/*.cc,
// read from the reference tree at build time, never copied) into
// oracle/_ref/libhiflow_lmp_ref.so.  The library runs the reference code itself
// on small inputs to pin the C restatement (oracle.c) and, on the GPU host, as
// the timed CPU baseline.  Solver loops above lmp (src/linear_solver/cg.cc,
// gmres.cc) need MPI through CoupledVector, so they are restated here over the
// reference's lVector/lMatrix objects, statement by statement, with the
// reference's own kernels doing all the arithmetic.

#include "lmatrix_csr_cpu.h"
#include "lvector_cpu.h"
#include "lpreconditioner.h"
#include "lpreconditioner_mc.h"
#include "lpreconditioner_mc_sgs.h"
#include "lpreconditioner_mc_ilup.h"
#include "solvers/cg.h"

#include <chrono>
#include <cmath>
#include <cstring>
#include <omp.h>

#include "oracle.h"

using namespace hiflow::la;

namespace {

// CSR copy into a reference matrix object (impl 0: CPUsimple, 1: CPUopenmp).
lMatrix<double> *make_matrix(int impl, int n, int nnz, const int *row, const int *col,
                             const double *val, int nthreads)
{
    CPUsimple_CSR_lMatrix<double> *s = new CPUsimple_CSR_lMatrix<double>(nnz, n, n, "A");
    std::memcpy(s->matrix.row, row, sizeof(int) * (n + 1));
    std::memcpy(s->matrix.col, col, sizeof(int) * nnz);
    std::memcpy(s->matrix.val, val, sizeof(double) * nnz);
    if (impl == 0) return s;
    CPUopenmp_CSR_lMatrix<double> *o = new CPUopenmp_CSR_lMatrix<double>();
    o->CopyStructureFrom(*s);
    o->CopyFrom(*s);
    o->set_num_threads(nthreads > 0 ? nthreads : 1);
    delete s;
    return o;
}

lVector<double> *make_vector(int impl, int n, const double *v, int nthreads)
{
    if (impl == 0) {
        CPUsimple_lVector<double> *x = new CPUsimple_lVector<double>(n, "v");
        if (v) std::memcpy(x->buffer, v, sizeof(double) * n);
        else x->Zeros();
        return x;
    }
    CPUopenmp_lVector<double> *x = new CPUopenmp_lVector<double>(n, "v");
    x->set_num_threads(nthreads > 0 ? nthreads : 1);
    if (v) std::memcpy(x->buffer, v, sizeof(double) * n);
    else x->Zeros();
    return x;
}

void copy_out(const lVector<double> &v, double *out)
{
    const CPU_lVector<double> *c = dynamic_cast<const CPU_lVector<double> *>(&v);
    std::memcpy(out, c->buffer, sizeof(double) * c->get_size());
}

void csr_out(const lMatrix<double> &m, int *row, int *col, double *val)
{
    const CPU_CSR_lMatrix<double> *c = dynamic_cast<const CPU_CSR_lMatrix<double> *>(&m);
    std::memcpy(row, c->matrix.row, sizeof(int) * (c->get_num_row() + 1));
    std::memcpy(col, c->matrix.col, sizeof(int) * c->get_nnz());
    if (val) std::memcpy(val, c->matrix.val, sizeof(double) * c->get_nnz());
}

// Access to the colour/level bookkeeping of the reference preconditioners.
template <class Base>
struct Open : public Base {
    int ncolors() const { return this->ncolors_; }
    const int *sizes() const { return this->color_sizes_; }
};

// IterateControl::Check restated (src/common/iterate_control.cc:84-110).
struct Control {
    int maxits;
    double abstol, reltol, divtol, first;
    int check(int step, double value)
    {
        if (step == 0) first = value;
        if (value < abstol) return 1;
        if (value < reltol * first) return 2;
        if (value > divtol * first) return 3;
        if (step >= maxits) return 4;
        return 0;
    }
};

// Preconditioner adaptor: z = M^-1 r for the types driven below.
struct Precond {
    // 0 none, 1 Jacobi, 2 MC-SGS, 3 ILU(0) level-scheduled, 4 ILU(0) multicoloured,
    // 5 ILU(0) level-scheduled without the block split (factors applied by ilu_solve)
    int kind = 0;
    lPreconditioner<double> *lp = nullptr;
    lMatrix<double> *factors = nullptr;
    void apply(const lVector<double> &r, lVector<double> *z)
    {
        if (kind == 0) z->CopyFrom(r);
        else if (kind == 5) factors->ilu_solve(r, z);
        else lp->ApplylPreconditioner(r, z);
    }
};

}  // namespace

extern "C" {

int ref_coo_to_csr(int n, int nnz, const int *coo_row, const int *coo_col, const double *coo_val,
                   int *row, int *col, double *val)
{
    CPUsimple_CSR_lMatrix<double> A(nnz, n, n, "A");
    if (coo_val) A.TransformFromCOO(coo_row, coo_col, coo_val, n, n, nnz);
    else A.init_structure(coo_row, coo_col);
    csr_out(A, row, col, coo_val ? val : nullptr);
    return 0;
}

// Structured Q1 system assembled with the reference's init_structure,
// add_values and ZeroRows; element matrices from the oracle's weak-form
// restatement (the FEM stack itself is outside the path).
int ref_q1_assemble(int dim, int N, int kind, const double *kcell, double nu, const double *beta,
                    int *row, int *col, double *val)
{
    int n;
    int64_t nnz;
    if (orc_q1_sizes(dim, N, &n, &nnz)) return -1;
    std::vector<int> cr(nnz), cc(nnz);
    orc_q1_structure(dim, N, cr.data(), cc.data());
    CPUsimple_CSR_lMatrix<double> A((int)nnz, n, n, "A");
    A.init_structure(cr.data(), cc.data());
    A.Zeros();
    const int nv = 1 << dim, P = N + 1, CZ = dim == 3 ? N : 1;
    const double h = 1.0 / N;
    double Ke[64];
    if (!kcell) orc_q1_element(dim, h, kind, kind == 0 ? 1.0 : nu, beta, Ke);
    int dofs[8];
    for (int cz = 0; cz < CZ; ++cz)
        for (int cy = 0; cy < N; ++cy)
            for (int cx = 0; cx < N; ++cx) {
                const int64_t cell = cx + (int64_t)N * (cy + (int64_t)N * cz);
                for (int a = 0; a < nv; ++a)
                    dofs[a] = (cx + (a & 1)) + P * ((cy + ((a >> 1) & 1)) + P * (cz + ((a >> 2) & 1)));
                if (kcell) orc_q1_element(dim, h, kind, kcell[cell], beta, Ke);
                A.add_values(dofs, nv, dofs, nv, Ke);
            }
    std::vector<int> bnd(n);
    const int nb = orc_q1_dirichlet(dim, N, bnd.data());
    A.ZeroRows(bnd.data(), nb, 1.0);
    csr_out(A, row, col, val);
    return 0;
}

int ref_add_values(int n, int nnz, const int *row, const int *col, double *val,
                   const int *rows, int num_rows, const int *cols, int num_cols, const double *values)
{
    lMatrix<double> *A = make_matrix(0, n, nnz, row, col, val, 1);
    A->add_values(rows, num_rows, cols, num_cols, values);
    csr_out(*A, const_cast<int *>(row), const_cast<int *>(col), val);
    delete A;
    return 0;
}

int ref_spmv(int impl, int nthreads, int n, int nnz, const int *row, const int *col, const double *val,
             const double *x, double *y)
{
    lMatrix<double> *A = make_matrix(impl, n, nnz, row, col, val, nthreads);
    lVector<double> *vx = make_vector(impl, n, x, nthreads), *vy = make_vector(impl, n, nullptr, nthreads);
    A->VectorMult(*vx, vy);
    copy_out(*vy, y);
    delete A; delete vx; delete vy;
    return 0;
}

double ref_dot(int impl, int n, const double *x, const double *y)
{
    lVector<double> *a = make_vector(impl, n, x, 1), *b = make_vector(impl, n, y, 1);
    const double d = a->Dot(*b);
    delete a; delete b;
    return d;
}

int ref_multicoloring(int n, int nnz, const int *row, const int *col, const double *val,
                      int *ncolors, int *sizes, int *perm)
{
    lMatrix<double> *A = make_matrix(0, n, nnz, row, col, val, 1);
    int nc = 0, *cs = nullptr, *pi = nullptr;
    dynamic_cast<CPU_CSR_lMatrix<double> *>(A)->Multicoloring(nc, &cs, &pi);
    *ncolors = nc;
    std::memcpy(sizes, cs, sizeof(int) * nc);
    std::memcpy(perm, pi, sizeof(int) * n);
    delete[] cs; delete[] pi; delete A;
    return 0;
}

int ref_levelscheduling(int n, int nnz, const int *row, const int *col, const double *val,
                        int *nlevels, int *sizes, int *perm)
{
    lMatrix<double> *A = make_matrix(0, n, nnz, row, col, val, 1);
    int nl = 0, *ls = nullptr, *pi = nullptr;
    dynamic_cast<CPU_CSR_lMatrix<double> *>(A)->Levelscheduling(nl, &ls, &pi);
    *nlevels = nl;
    std::memcpy(sizes, ls, sizeof(int) * nl);
    std::memcpy(perm, pi, sizeof(int) * n);
    delete[] ls; delete[] pi; delete A;
    return 0;
}

int ref_reorder(int n, int nnz, const int *row, const int *col, const double *val, const int *perm,
                int *row_out, int *col_out, double *val_out)
{
    lMatrix<double> *A = make_matrix(0, n, nnz, row, col, val, 1);
    A->Reorder(perm);
    csr_out(*A, row_out, col_out, val_out);
    delete A;
    return 0;
}

int ref_ilu0(int n, int nnz, const int *row, const int *col, double *val)
{
    lMatrix<double> *A = make_matrix(0, n, nnz, row, col, val, 1);
    A->ilu0();
    csr_out(*A, const_cast<int *>(row), const_cast<int *>(col), val);
    delete A;
    return 0;
}

int ref_ilu_solve(int n, int nnz, const int *row, const int *col, const double *val,
                  const double *r, double *z)
{
    lMatrix<double> *A = make_matrix(0, n, nnz, row, col, val, 1);
    lVector<double> *vr = make_vector(0, n, r, 1), *vz = make_vector(0, n, nullptr, 1);
    A->ilu_solve(*vr, vz);
    copy_out(*vz, z);
    delete A; delete vr; delete vz;
    return 0;
}

// Build a block preconditioner with the reference class and apply it once.
// kind 2: MC symmetric Gauss-Seidel; 3: ILU(0) with level scheduling;
// 4: ILU(0) multicoloured.  r_perm is given in the permuted numbering.
// ILU(p) parameters of the kind 3 / 4 block preconditioners built below
// (ref_set_ilup; 0 and 1 give ILU(0) on the operator's own colouring).
static int g_ilu_p = 0, g_mat_power = 1;

static lPreconditioner_MultiColoring<double> *build_block(int kind, double omega, lMatrix<double> &A,
                                                          lMatrix<double> &Aperm, lVector<double> &x,
                                                          lVector<double> &rhs)
{
    lPreconditioner_MultiColoring<double> *p;
    if (kind == 2) {
        p = new Open<lPreconditioner_MultiColoring_SymmetricGaussSeidel<double>>();
    } else {
        Open<lPreconditioner_MultiColoring_ILUp<double>> *q = new Open<lPreconditioner_MultiColoring_ILUp<double>>();
        if (kind == 3) q->Init(g_ilu_p, 1, false, false, true);
        else q->Init(g_ilu_p, g_mat_power, true, true, false);
        p = q;
    }
    p->SetupOperator(A);
    p->SetupPermOperator(Aperm);
    p->SetupPermVectors(&x, &rhs);
    if (kind == 2 && omega != 1.0) p->SetRelax(omega);
    p->Build();
    return p;
}

static void block_info(int kind, lPreconditioner_MultiColoring<double> *p, int *nblocks, int *sizes)
{
    int nb;
    const int *s;
    if (kind == 2) {
        auto *o = static_cast<Open<lPreconditioner_MultiColoring_SymmetricGaussSeidel<double>> *>(p);
        nb = o->ncolors(); s = o->sizes();
    } else {
        auto *o = static_cast<Open<lPreconditioner_MultiColoring_ILUp<double>> *>(p);
        nb = o->ncolors(); s = o->sizes();
    }
    *nblocks = nb;
    if (sizes) std::memcpy(sizes, s, sizeof(int) * nb);
}

int ref_block_precond(int kind, double omega, int n, int nnz, const int *row, const int *col,
                      const double *val, const double *r_perm, double *z_perm, int *perm,
                      int *nblocks, int *sizes, int *Ap_row, int *Ap_col, double *Ap_val)
{
    lMatrix<double> *A = make_matrix(0, n, nnz, row, col, val, 1);
    lMatrix<double> *Ap = make_matrix(0, n, nnz, row, col, val, 1);
    lVector<double> *x = make_vector(0, n, nullptr, 1), *rhs = make_vector(0, n, nullptr, 1);
    lPreconditioner_MultiColoring<double> *p = build_block(kind, omega, *A, *Ap, *x, *rhs);
    std::memcpy(perm, p->get_permut(), sizeof(int) * n);
    block_info(kind, p, nblocks, sizes);
    csr_out(*Ap, Ap_row, Ap_col, Ap_val);
    lVector<double> *vr = make_vector(0, n, r_perm, 1), *vz = make_vector(0, n, nullptr, 1);
    p->ApplylPreconditioner(*vr, vz);
    copy_out(*vz, z_perm);
    delete p; delete A; delete Ap; delete x; delete rhs; delete vr; delete vz;
    return 0;
}

// lPreconditioner_MultiColoring_ILUp with ILU(ilu_p) and the colouring on the
// pattern of A^mat_power; mode 3 level scheduling, mode 4 multicolouring.
int ref_block_precond_ilup(int mode, int ilu_p, int mat_power, int n, int nnz, const int *row, const int *col,
                           const double *val, const double *r_perm, double *z_perm, int *perm, int *nblocks,
                           int *sizes, int *Ap_row, int *Ap_col, double *Ap_val)
{
    lMatrix<double> *A = make_matrix(0, n, nnz, row, col, val, 1);
    lMatrix<double> *Ap = make_matrix(0, n, nnz, row, col, val, 1);
    lVector<double> *x = make_vector(0, n, nullptr, 1), *rhs = make_vector(0, n, nullptr, 1);
    Open<lPreconditioner_MultiColoring_ILUp<double>> *q = new Open<lPreconditioner_MultiColoring_ILUp<double>>();
    if (mode == 3) q->Init(ilu_p, mat_power, false, false, true);
    else q->Init(ilu_p, mat_power, true, true, false);
    q->SetupOperator(*A);
    q->SetupPermOperator(*Ap);
    q->SetupPermVectors(x, rhs);
    q->Build();
    std::memcpy(perm, q->get_permut(), sizeof(int) * n);
    block_info(4, q, nblocks, sizes);
    csr_out(*Ap, Ap_row, Ap_col, Ap_val);
    lVector<double> *vr = make_vector(0, n, r_perm, 1), *vz = make_vector(0, n, nullptr, 1);
    q->ApplylPreconditioner(*vr, vz);
    copy_out(*vz, z_perm);
    delete q; delete A; delete Ap; delete x; delete rhs; delete vr; delete vz;
    return 0;
}

void ref_set_ilup(int ilu_p, int mat_power)
{
    g_ilu_p = ilu_p;
    g_mat_power = mat_power;
}

// CPU_CSR_lMatrix::ilup (lmatrix_csr_cpu.cc:1933-1952); returns nnz of the
// factors, -1 if cap is too small.
int ref_ilup(int n, int nnz, const int *row, const int *col, const double *val, int p, int cap, int *row_out,
             int *col_out, double *val_out)
{
    CPUsimple_CSR_lMatrix<double> A(nnz, n, n, "A");
    std::memcpy(A.matrix.row, row, sizeof(int) * (n + 1));
    std::memcpy(A.matrix.col, col, sizeof(int) * nnz);
    std::memcpy(A.matrix.val, val, sizeof(double) * nnz);
    A.ilup(p);
    const int m = A.get_nnz();
    if (m > cap) return -1;
    std::memcpy(row_out, A.matrix.row, sizeof(int) * (n + 1));
    std::memcpy(col_out, A.matrix.col, sizeof(int) * m);
    std::memcpy(val_out, A.matrix.val, sizeof(double) * m);
    return m;
}

// CPU_CSR_lMatrix::MatrixSupSPower (lmatrix_csr_cpu.cc:1641-1664).
int ref_power_pattern(int n, int nnz, const int *row, const int *col, int p, int cap, int *row_out, int *col_out)
{
    CPUsimple_CSR_lMatrix<double> A(nnz, n, n, "A");
    std::memcpy(A.matrix.row, row, sizeof(int) * (n + 1));
    std::memcpy(A.matrix.col, col, sizeof(int) * nnz);
    for (int j = 0; j < nnz; ++j) A.matrix.val[j] = 1.0;
    lMatrix<double> *P = A.MatrixSupSPower(p);
    CPU_CSR_lMatrix<double> *c = dynamic_cast<CPU_CSR_lMatrix<double> *>(P);
    const int m = c->get_nnz();
    if (m <= cap) {
        std::memcpy(row_out, c->matrix.row, sizeof(int) * (n + 1));
        std::memcpy(col_out, c->matrix.col, sizeof(int) * m);
    }
    delete P;
    return m <= cap ? m : -1;
}

// CG<LAD>::SolvePrecond / SolveNoPrecond restated over lmp objects
// (src/linear_solver/cg.cc:84-248).  precond: 0 none, 1 Jacobi, 2 MC-SGS.
// With a block preconditioner, b and x are in the permuted numbering of
// the operator returned by ref_block_precond.
static int pcg_loop(lMatrix<double> &A, Precond &P, lVector<double> &b, lVector<double> &x,
                    Control &ctl, int *iters, double *res_out, double *res_hist)
{
    lVector<double> *r = b.CloneWithoutContent(), *p = b.CloneWithoutContent();
    lVector<double> *z = b.CloneWithoutContent(), *Ap = b.CloneWithoutContent();
    int iter = 0;
    A.VectorMult(x, r);
    r->ScaleAdd(-1.0, b);
    double rr = r->Dot(*r), res = std::sqrt(rr), beta;
    int conv = ctl.check(iter, res);
    if (res_hist) res_hist[0] = res;
    if (P.kind) {
        z->Zeros();
        P.apply(*r, z);
        p->CopyFrom(*z);
        beta = r->Dot(*z);
    } else {
        p->CopyFrom(*r);
        beta = rr;
    }
    while (conv == 0) {
        ++iter;
        A.VectorMult(*p, Ap);
        const double alpha = beta / Ap->Dot(*p);
        x.Axpy(*p, alpha);
        r->Axpy(*Ap, -alpha);
        rr = r->Dot(*r);
        res = std::sqrt(rr);
        if (res_hist) res_hist[iter] = res;
        conv = ctl.check(iter, res);
        if (conv) break;
        if (P.kind) {
            z->Zeros();
            P.apply(*r, z);
            const double gamma = r->Dot(*z);
            beta = gamma / beta;
            p->ScaleAdd(beta, *z);
            beta = gamma;
        } else {
            beta = rr / beta;
            p->ScaleAdd(beta, *r);
            beta = rr;
        }
    }
    *iters = iter;
    *res_out = res;
    delete r; delete p; delete z; delete Ap;
    return conv;
}

int ref_pcg(int precond, int impl, int nthreads, int n, int nnz, const int *row, const int *col,
            const double *val, const double *b, double *x, int maxits, double abstol, double reltol,
            double divtol, int *iters, double *res, double *res_hist)
{
    lMatrix<double> *A = make_matrix(impl, n, nnz, row, col, val, nthreads);
    lVector<double> *vb = make_vector(impl, n, b, nthreads), *vx = make_vector(impl, n, x, nthreads);
    Precond P;
    P.kind = precond;
    lVector<double> *dcopy = nullptr;
    if (precond == 1) {
        lPreconditioner_Jacobi<double> *j = new lPreconditioner_Jacobi<double>();
        dcopy = vx->CloneWithoutContent();
        j->Init(*dcopy);
        j->SetupOperator(*A);
        j->Build();
        P.lp = j;
    } else if (precond == 2) {
        lMatrix<double> *Ap = make_matrix(0, n, nnz, row, col, val, 1);
        lVector<double> *xx = make_vector(0, n, nullptr, 1), *rr = make_vector(0, n, nullptr, 1);
        P.lp = build_block(2, 1.0, *A, *Ap, *xx, *rr);
        delete xx; delete rr;
        // the operator is used in the permuted numbering from here on
        delete A;
        A = make_matrix(impl, n, nnz, dynamic_cast<CPU_CSR_lMatrix<double> *>(Ap)->matrix.row,
                        dynamic_cast<CPU_CSR_lMatrix<double> *>(Ap)->matrix.col,
                        dynamic_cast<CPU_CSR_lMatrix<double> *>(Ap)->matrix.val, nthreads);
        delete Ap;
    }
    Control ctl{maxits, abstol, reltol, divtol, 0.0};
    const int conv = pcg_loop(*A, P, *vb, *vx, ctl, iters, res, res_hist);
    copy_out(*vx, x);
    delete P.lp; delete dcopy; delete A; delete vb; delete vx;
    return conv;
}

// GMRES<LAD>::SolveRight restated (src/linear_solver/gmres.cc:285-510).
// precond: 0 none, 3 ILU(0) level-scheduled, 4 ILU(0) multicoloured, 5 ILU(0)
// level-scheduled applied by ilu_solve; with a block preconditioner b and x
// are in its permuted numbering.
int ref_gmres(int precond, int impl, int nthreads, int m, int n, int nnz, const int *row,
              const int *col, const double *val, const double *b, double *x, int maxits,
              double abstol, double reltol, double divtol, int *iters, double *res_out)
{
    lMatrix<double> *A = make_matrix(impl, n, nnz, row, col, val, nthreads);
    Precond P;
    P.kind = precond;
    if (precond == 3 || precond == 4) {
        lMatrix<double> *Ap = make_matrix(0, n, nnz, row, col, val, 1);
        lVector<double> *xx = make_vector(0, n, nullptr, 1), *rr = make_vector(0, n, nullptr, 1);
        P.lp = build_block(precond, 1.0, *A, *Ap, *xx, *rr);
        delete xx; delete rr;
        delete A;
        CPU_CSR_lMatrix<double> *c = dynamic_cast<CPU_CSR_lMatrix<double> *>(Ap);
        A = make_matrix(impl, n, nnz, c->matrix.row, c->matrix.col, c->matrix.val, nthreads);
        delete Ap;
    }
    if (precond == 5) {
        // lPreconditioner_MultiColoring_ILUp with level scheduling, Build steps
        // (lpreconditioner_mc.cc:157-199): ilu0 of the operator in its own
        // order, Levelscheduling of the factors, the factors and the operator
        // reordered by that permutation.  The apply is the reference's
        // ilu_solve on the reordered factors (the same triangular solves that
        // the block apply performs level by level, without the per-level-pair
        // submatrices whose extraction costs O(levels^2 nnz) at set-up).
        lMatrix<double> *F = make_matrix(0, n, nnz, row, col, val, 1);
        F->ilu0();
        int nl = 0, *ls = nullptr, *pi = nullptr;
        dynamic_cast<CPU_CSR_lMatrix<double> *>(F)->Levelscheduling(nl, &ls, &pi);
        F->Reorder(pi);
        lMatrix<double> *Ap = make_matrix(0, n, nnz, row, col, val, 1);
        Ap->Reorder(pi);
        delete A;
        CPU_CSR_lMatrix<double> *c = dynamic_cast<CPU_CSR_lMatrix<double> *>(Ap);
        A = make_matrix(impl, n, nnz, c->matrix.row, c->matrix.col, c->matrix.val, nthreads);
        delete Ap;
        delete[] ls; delete[] pi;
        P.factors = F;
    }
    lVector<double> *vb = make_vector(impl, n, b, nthreads), *vx = make_vector(impl, n, x, nthreads);
    Control ctl{maxits, abstol, reltol, divtol, 0.0};
    const int mb = std::min(m, maxits);
    std::vector<lVector<double> *> V(mb + 1);
    for (auto &v : V) v = vb->CloneWithoutContent();
    lVector<double> *w = vb->CloneWithoutContent(), *z = vb->CloneWithoutContent();
    std::vector<double> H((size_t)mb * (mb + 1)), g(mb + 1), cs(mb + 1), sn(mb + 1);
    auto HH = [&](int j, int i) -> double & { return H[(size_t)j * (mb + 1) + i]; };
    auto rot = [](double c, double s, double *dx, double *dy) {
        const double t = c * (*dx) + s * (*dy);
        *dy = -s * (*dx) + c * (*dy);
        *dx = t;
    };
    int iter = 0;
    A->VectorMult(*vx, V[0]);
    V[0]->ScaleAdd(-1.0, *vb);
    double res = V[0]->Norm2();
    int conv = ctl.check(iter, res);
    auto update = [&](int k) {
        std::vector<double> y(g);
        for (int i = k + 1; i--;) {
            y[i] /= HH(i, i);
            const double t = y[i];
            for (int j = 0; j < i; ++j) y[j] -= HH(i, j) * t;
        }
        z->Zeros();
        for (int j = 0; j <= k; ++j) z->Axpy(*V[j], y[j]);
        w->Zeros();
        P.apply(*z, w);
        vx->Axpy(*w, 1.0);
    };
    while (conv == 0) {
        std::fill(g.begin(), g.end(), 0.0);
        std::fill(H.begin(), H.end(), 0.0);
        V[0]->Scale(1.0 / res);
        g[0] = res;
        for (int j = 0; j != mb; ++j) {
            ++iter;
            z->Zeros();
            P.apply(*V[j], z);
            A->VectorMult(*z, w);
            for (int i = 0; i <= j; ++i) {
                HH(j, i) = w->Dot(*V[i]);
                w->Axpy(*V[i], -1.0 * HH(j, i));
            }
            HH(j, j + 1) = w->Norm2();
            w->Scale(1.0 / HH(j, j + 1));
            V[j + 1]->CloneFrom(*w);
            for (int k = 0; k != j; ++k) rot(cs[k], sn[k], &HH(j, k), &HH(j, k + 1));
            const double beta = std::sqrt(HH(j, j) * HH(j, j) + HH(j, j + 1) * HH(j, j + 1));
            cs[j] = HH(j, j) / beta;
            sn[j] = HH(j, j + 1) / beta;
            rot(cs[j], sn[j], &HH(j, j), &HH(j, j + 1));
            rot(cs[j], sn[j], &g[j], &g[j + 1]);
            res = std::abs(g[j + 1]);
            conv = ctl.check(iter, res);
            if (conv) {
                update(j);
                break;
            }
        }
        if (conv == 0) {
            update(mb - 1);
            A->VectorMult(*vx, V[0]);
            V[0]->ScaleAdd(-1.0, *vb);
        }
    }
    copy_out(*vx, x);
    *iters = iter;
    *res_out = res;
    for (auto &v : V) delete v;
    delete w; delete z; delete vb; delete vx; delete A; delete P.lp; delete P.factors;
    return conv;
}

// The reference's lmp-level CG functor (src/linear_algebra/lmp/solvers/cg.h:103-221),
// as used by test/LinearAlgebra/cg.cc.
int ref_lmp_cg(int n, int nnz, const int *row, const int *col, const double *val, const double *b,
               double *x, double rel_eps, double abs_eps, int max_iter)
{
    lMatrix<double> *A = make_matrix(0, n, nnz, row, col, val, 1);
    lVector<double> *vb = make_vector(0, n, b, 1), *vx = make_vector(0, n, x, 1);
    int mi = max_iter;
    const int rc = cg(vx, vb, A, rel_eps, abs_eps, mi, -1, (lPreconditioner<double> *)nullptr);
    copy_out(*vx, x);
    delete A; delete vb; delete vx;
    return rc;
}

// The same functor (CGFunctor<double, true>, the harness of
// benchmark_local_solver) with or without lPreconditioner_Jacobi, reporting
// the iterations it ran (its max_iter argument on return).
int ref_lmp_cg_iters(int n, int nnz, const int *row, const int *col, const double *val, const double *b,
                     double *x, double rel_eps, double abs_eps, int max_iter, int jacobi, int *iters)
{
    lMatrix<double> *A = make_matrix(0, n, nnz, row, col, val, 1);
    lVector<double> *vb = make_vector(0, n, b, 1), *vx = make_vector(0, n, x, 1);
    lVector<double> *d = make_vector(0, n, nullptr, 1);
    lPreconditioner_Jacobi<double> J;
    if (jacobi) {
        J.Init(*d);
        J.SetupOperator(*A);
        J.Build();
    }
    CGFunctor<double, true> f;
    int mi = max_iter;
    const int rc = f(vx, vb, A, rel_eps, abs_eps, mi, -1, jacobi ? &J : (lPreconditioner<double> *)nullptr);
    *iters = mi;
    copy_out(*vx, x);
    delete A; delete vb; delete vx; delete d;
    return rc;
}

// Wall time of `reps` CPUopenmp_CSR_lMatrix::VectorMult calls
// (openmp/CPUopenmp_csr_lmatrix.cc:144-165), in seconds.
double ref_time_spmv(int nthreads, int reps, int n, int nnz, const int *row, const int *col,
                     const double *val, const double *x, double *y)
{
    lMatrix<double> *A = make_matrix(1, n, nnz, row, col, val, nthreads);
    lVector<double> *vx = make_vector(1, n, x, nthreads), *vy = make_vector(1, n, nullptr, nthreads);
    A->VectorMult(*vx, vy);
    const auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < reps; ++i) A->VectorMult(*vx, vy);
    const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    copy_out(*vy, y);
    delete A; delete vx; delete vy;
    return dt;
}

int ref_max_threads(void) { return omp_get_max_threads(); }

// CPU_CSR_lMatrix::ReadFile (lmp/lmatrix_csr_cpu.cc:1733-1749) on a
// MatrixMarket file the reference accepts; the CSR out (caps in entries).
// Returns nnz, or -1 when the caps are too small.
int ref_mm_read(const char *path, int *n, int *m, int *row, int *col, double *val, int cap_rows, int cap_nnz)
{
    CPUsimple_CSR_lMatrix<double> A;
    A.ReadFile(path);
    *n = A.get_num_row();
    *m = A.get_num_col();
    const int nnz = A.get_nnz();
    if (*n > cap_rows || nnz > cap_nnz) return -1;
    std::memcpy(row, A.matrix.row, sizeof(int) * (*n + 1));
    std::memcpy(col, A.matrix.col, sizeof(int) * nnz);
    std::memcpy(val, A.matrix.val, sizeof(double) * nnz);
    return nnz;
}

// CPU_CSR_lMatrix::WriteFile (lmp/lmatrix_csr_cpu.cc:1751-1765).
void ref_mm_write(const char *path, int n, int m, int nnz, const int *row, const int *col, const double *val)
{
    CPUsimple_CSR_lMatrix<double> A(nnz, n, m, "A");
    std::memcpy(A.matrix.row, row, sizeof(int) * (n + 1));
    std::memcpy(A.matrix.col, col, sizeof(int) * nnz);
    std::memcpy(A.matrix.val, val, sizeof(double) * nnz);
    A.WriteFile(path);
}

// CPU_lVector::ReadFile (lmp/lvector_cpu.cc:582-636): the values out, their
// count returned (-1 when cap is too small).
int ref_vec_read(const char *path, double *x, int cap)
{
    CPUsimple_lVector<double> v;
    v.ReadFile(path);
    const int n = v.get_size();
    if (n > cap) return -1;
    for (int i = 0; i < n; ++i) x[i] = v.buffer[i];
    return n;
}

// CPUsimple_lVector::ArgMin / ArgMax / Norm1 / NormMax (lmp/CPUsimple_lvector.cc:51-158).
void ref_vec_reduce(int n, const double *x, int *argmin, int *argmax, double *norm1, double *normmax)
{
    CPUsimple_lVector<double> v(n, "x");
    for (int i = 0; i < n; ++i) v.buffer[i] = x[i];
    *argmin = v.ArgMin();
    *argmax = v.ArgMax();
    *norm1 = v.Norm1();
    *normmax = v.NormMax();
}

// CPUsimple_lVector::Rot (:448-466) and Rotm (:540-600) with x the vector the
// method is called on and y its argument; both in place.
void ref_vec_rot(int n, double *x, double *y, double c, double s, const double *param)
{
    CPUsimple_lVector<double> vx(n, "x"), vy(n, "y");
    for (int i = 0; i < n; ++i) {
        vx.buffer[i] = x[i];
        vy.buffer[i] = y[i];
    }
    if (param) vx.Rotm(&vy, param[0]);
    else vx.Rot(&vy, c, s);
    for (int i = 0; i < n; ++i) {
        x[i] = vx.buffer[i];
        y[i] = vy.buffer[i];
    }
}

// CPUsimple_lVector::Rotg (:492-535) on host scalars.
void ref_rotg(double *a, double *b, double *c, double *s)
{
    CPUsimple_lVector<double> v(1, "x");
    v.Rotg(a, b, c, s);
}

// CPU_CSR_lMatrix::Scale / ScaleOffdiag / Zeros (lmp/lmatrix_csr_cpu.cc:100-103,
// 205-224) on an n x m CSR; the values in place.  mode 0 Scale, 1 ScaleOffdiag,
// 2 Zeros.
void ref_csr_scale(int n, int m, int nnz, const int *row, const int *col, double *val, double alpha, int mode)
{
    CPUsimple_CSR_lMatrix<double> A(nnz, n, m, "A");
    std::memcpy(A.matrix.row, row, sizeof(int) * (n + 1));
    std::memcpy(A.matrix.col, col, sizeof(int) * nnz);
    std::memcpy(A.matrix.val, val, sizeof(double) * nnz);
    if (mode == 0) A.Scale(alpha);
    else if (mode == 1) A.ScaleOffdiag(alpha);
    else A.Zeros();
    std::memcpy(val, A.matrix.val, sizeof(double) * nnz);
}

// CPU_CSR_lMatrix::extract_diagelements / extract_invdiagelements
// (lmp/lmatrix_csr_cpu.cc:2395-2431), rows [start, end) into out.
void ref_csr_diag(int n, int m, int nnz, const int *row, const int *col, const double *val, int start, int end,
                  int inverse, double *out)
{
    CPUsimple_CSR_lMatrix<double> A(nnz, n, m, "A");
    std::memcpy(A.matrix.row, row, sizeof(int) * (n + 1));
    std::memcpy(A.matrix.col, col, sizeof(int) * nnz);
    std::memcpy(A.matrix.val, val, sizeof(double) * nnz);
    CPUsimple_lVector<double> v(end - start, "d");
    if (inverse) A.extract_invdiagelements(start, end, &v);
    else A.extract_diagelements(start, end, &v);
    copy_out(v, out);
}

// CPU_CSR_lMatrix::extract_submatrix (lmp/lmatrix_csr_cpu.cc:1768-1843) and
// Compress (:142-202).  mode 0: the block [sr, er) x [sc, ec); mode 1: the
// matrix without its zero entries.  Returns the result's nnz (-1 when cap is
// too small), its row pointer (rows + 1 entries), columns and values out.
int ref_csr_extract(int n, int m, int nnz, const int *row, const int *col, const double *val, int mode, int sr,
                    int sc, int er, int ec, int cap, int *row_out, int *col_out, double *val_out)
{
    CPUsimple_CSR_lMatrix<double> A(nnz, n, m, "A");
    std::memcpy(A.matrix.row, row, sizeof(int) * (n + 1));
    std::memcpy(A.matrix.col, col, sizeof(int) * nnz);
    std::memcpy(A.matrix.val, val, sizeof(double) * nnz);
    const CPU_CSR_lMatrix<double> *c = &A;
    lMatrix<double> *S = nullptr;
    if (mode == 0) {
        S = A.extract_submatrix(sr, sc, er, ec);
        c = dynamic_cast<const CPU_CSR_lMatrix<double> *>(S);
    } else {
        A.Compress();
    }
    const int k = c->get_nnz(), rows = c->get_num_row();
    int rc = -1;
    if (k <= cap) {
        std::memcpy(row_out, c->matrix.row, sizeof(int) * (rows + 1));
        if (k) {
            std::memcpy(col_out, c->matrix.col, sizeof(int) * k);
            std::memcpy(val_out, c->matrix.val, sizeof(double) * k);
        }
        rc = k;
    }
    delete S;
    return rc;
}

// CPU_lVector::WriteFile (lmp/lvector_cpu.cc:638-663).
void ref_vec_write(const char *path, int n, const double *x)
{
    CPUsimple_lVector<double> v(n, "v");
    for (int i = 0; i < n; ++i) v.buffer[i] = x[i];
    v.WriteFile(path);
}

}  // extern "C"

namespace {

template <typename T>
lMatrix<T> *make_matrix_t(int impl, int n, int nnz, const int *row, const int *col, const double *val, int nthreads)
{
    CPUsimple_CSR_lMatrix<T> *s = new CPUsimple_CSR_lMatrix<T>(nnz, n, n, "A");
    std::memcpy(s->matrix.row, row, sizeof(int) * (n + 1));
    std::memcpy(s->matrix.col, col, sizeof(int) * nnz);
    for (int j = 0; j < nnz; ++j) s->matrix.val[j] = (T)val[j];
    if (impl == 0) return s;
    CPUopenmp_CSR_lMatrix<T> *o = new CPUopenmp_CSR_lMatrix<T>();
    o->CopyStructureFrom(*s);
    o->CopyFrom(*s);
    o->set_num_threads(nthreads > 0 ? nthreads : 1);
    delete s;
    return o;
}

template <typename T>
lVector<T> *make_vector_t(int impl, int n, int nthreads)
{
    if (impl == 0) {
        CPUsimple_lVector<T> *x = new CPUsimple_lVector<T>(n, "v");
        x->Zeros();
        return x;
    }
    CPUopenmp_lVector<T> *x = new CPUopenmp_lVector<T>(n, "v");
    x->set_num_threads(nthreads > 0 ? nthreads : 1);
    x->Zeros();
    return x;
}

// CG<LAD>::SolvePrecond with lPreconditioner_Jacobi, restated over lVector<T>
// (src/linear_solver/cg.cc:164-248); at most `cap` iterations when cap > 0.
template <typename T>
int pcg_t(lMatrix<T> &A, lPreconditioner<T> &P, lVector<T> &b, lVector<T> &x, Control &ctl, int cap, int *iters)
{
    lVector<T> *r = b.CloneWithoutContent(), *p = b.CloneWithoutContent();
    lVector<T> *z = b.CloneWithoutContent(), *Ap = b.CloneWithoutContent();
    int iter = 0;
    A.VectorMult(x, r);
    r->ScaleAdd((T)-1.0, b);
    T beta;
    double res = std::sqrt((double)r->Dot(*r));
    int conv = ctl.check(iter, res);
    z->Zeros();
    P.ApplylPreconditioner(*r, z);
    p->CopyFrom(*z);
    beta = r->Dot(*z);
    while (conv == 0 && (cap <= 0 || iter < cap)) {
        ++iter;
        A.VectorMult(*p, Ap);
        const T alpha = beta / Ap->Dot(*p);
        x.Axpy(*p, alpha);
        r->Axpy(*Ap, -alpha);
        res = std::sqrt((double)r->Dot(*r));
        conv = ctl.check(iter, res);
        if (conv) break;
        z->Zeros();
        P.ApplylPreconditioner(*r, z);
        const T gamma = r->Dot(*z);
        beta = gamma / beta;
        p->ScaleAdd(beta, *z);
        beta = gamma;
    }
    *iters = iter;
    delete r; delete p; delete z; delete Ap;
    return conv;
}

}  // namespace

extern "C" {

// MPIR<LAD_high, LAD_low>::Solve restated over the reference's lmp objects
// (src/linear_solver/mpir.cc:69-326): FP64 residual, CastFrom to FP32, FP32
// Jacobi-CG error correction, CastFrom back, FP64 update.  The relative stop
// uses the initial residual.  With sample_inner > 0 the run stops after that
// many inner iterations in total (a bounded timing sample).  Returns the wall
// time in seconds of the solve (setup excluded).
double ref_mpir(int impl, int nthreads, int n, int nnz, const int *row, const int *col, const double *val,
                const double *b, double *x, int max_outer, double reltol, double inner_reltol,
                int inner_maxits, int sample_inner, int *outer_done, int *inner_done, double *res_out)
{
    lMatrix<double> *Ah = make_matrix_t<double>(impl, n, nnz, row, col, val, nthreads);
    lMatrix<float> *Al = make_matrix_t<float>(impl, n, nnz, row, col, val, nthreads);
    lVector<double> *vb = make_vector_t<double>(impl, n, nthreads), *vx = make_vector_t<double>(impl, n, nthreads);
    std::memcpy(dynamic_cast<CPU_lVector<double> *>(vb)->buffer, b, sizeof(double) * n);
    std::memcpy(dynamic_cast<CPU_lVector<double> *>(vx)->buffer, x, sizeof(double) * n);
    lVector<double> *resh = vb->CloneWithoutContent(), *corh = vb->CloneWithoutContent();
    lVector<float> *resl = make_vector_t<float>(impl, n, nthreads), *corl = make_vector_t<float>(impl, n, nthreads);
    lVector<float> *dl = resl->CloneWithoutContent();
    lPreconditioner_Jacobi<float> J;
    J.Init(*dl);
    J.SetupOperator(*Al);
    J.Build();
    const auto t0 = std::chrono::steady_clock::now();
    Ah->VectorMult(*vx, resh);
    resh->ScaleAdd(-1.0, *vb);
    double res = resh->Norm2();
    const double res0 = res;
    int outer = 0, inner_total = 0;
    while (res > 0.0 && res > reltol * res0 && outer < max_outer &&
           (sample_inner <= 0 || inner_total < sample_inner)) {
        ++outer;
        resl->CastFrom(*resh);
        corl->Zeros();
        Control ic{inner_maxits, 0.0, inner_reltol, 1e6, 0.0};
        int it = 0;
        pcg_t<float>(*Al, J, *resl, *corl, ic, sample_inner > 0 ? sample_inner - inner_total : 0, &it);
        inner_total += it;
        corh->CastFrom(*corl);
        vx->Axpy(*corh, 1.0);
        Ah->VectorMult(*vx, resh);
        resh->ScaleAdd(-1.0, *vb);
        res = resh->Norm2();
    }
    const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::memcpy(x, dynamic_cast<CPU_lVector<double> *>(vx)->buffer, sizeof(double) * n);
    *outer_done = outer;
    *inner_done = inner_total;
    *res_out = res;
    delete Ah; delete Al; delete vb; delete vx; delete resh; delete corh; delete resl; delete corl; delete dl;
    return dt;
}

// The same MPIR over objects that persist between solves, so that repeated
// timed solves of one system do not rebuild the matrices: ref_mpir_create
// copies the CSR into the reference's FP64 and FP32 CPUopenmp matrices and
// builds the FP32 Jacobi preconditioner; ref_mpir_run solves once from x
// (seconds of the solve, as ref_mpir); ref_mpir_threads changes the OpenMP
// thread count of every object.
struct MpirSession {
    int n;
    lMatrix<double> *Ah;
    lMatrix<float> *Al;
    lVector<double> *vb, *vx, *resh, *corh;
    lVector<float> *resl, *corl, *dl;
    lPreconditioner_Jacobi<float> *J;
};

void *ref_mpir_create(int nthreads, int n, int nnz, const int *row, const int *col, const double *val)
{
    MpirSession *s = new MpirSession();
    s->n = n;
    s->Ah = make_matrix_t<double>(1, n, nnz, row, col, val, nthreads);
    s->Al = make_matrix_t<float>(1, n, nnz, row, col, val, nthreads);
    s->vb = make_vector_t<double>(1, n, nthreads);
    s->vx = make_vector_t<double>(1, n, nthreads);
    s->resh = s->vb->CloneWithoutContent();
    s->corh = s->vb->CloneWithoutContent();
    s->resl = make_vector_t<float>(1, n, nthreads);
    s->corl = make_vector_t<float>(1, n, nthreads);
    s->dl = s->resl->CloneWithoutContent();
    s->J = new lPreconditioner_Jacobi<float>();
    s->J->Init(*s->dl);
    s->J->SetupOperator(*s->Al);
    s->J->Build();
    return s;
}

void ref_mpir_threads(void *h, int nthreads)
{
    MpirSession *s = static_cast<MpirSession *>(h);
    const int t = nthreads > 0 ? nthreads : 1;
    dynamic_cast<CPUopenmp_CSR_lMatrix<double> *>(s->Ah)->set_num_threads(t);
    dynamic_cast<CPUopenmp_CSR_lMatrix<float> *>(s->Al)->set_num_threads(t);
    for (lVector<double> *v : {s->vb, s->vx, s->resh, s->corh})
        dynamic_cast<CPUopenmp_lVector<double> *>(v)->set_num_threads(t);
    for (lVector<float> *v : {s->resl, s->corl, s->dl})
        dynamic_cast<CPUopenmp_lVector<float> *>(v)->set_num_threads(t);
}

double ref_mpir_run(void *h, const double *b, double *x, int max_outer, double reltol, double inner_reltol,
                    int inner_maxits, int sample_inner, int *outer_done, int *inner_done, double *res_out)
{
    MpirSession *s = static_cast<MpirSession *>(h);
    const int n = s->n;
    std::memcpy(dynamic_cast<CPU_lVector<double> *>(s->vb)->buffer, b, sizeof(double) * n);
    std::memcpy(dynamic_cast<CPU_lVector<double> *>(s->vx)->buffer, x, sizeof(double) * n);
    const auto t0 = std::chrono::steady_clock::now();
    s->Ah->VectorMult(*s->vx, s->resh);
    s->resh->ScaleAdd(-1.0, *s->vb);
    double res = s->resh->Norm2();
    const double res0 = res;
    int outer = 0, inner_total = 0;
    while (res > 0.0 && res > reltol * res0 && outer < max_outer &&
           (sample_inner <= 0 || inner_total < sample_inner)) {
        ++outer;
        s->resl->CastFrom(*s->resh);
        s->corl->Zeros();
        Control ic{inner_maxits, 0.0, inner_reltol, 1e6, 0.0};
        int it = 0;
        pcg_t<float>(*s->Al, *s->J, *s->resl, *s->corl, ic, sample_inner > 0 ? sample_inner - inner_total : 0, &it);
        inner_total += it;
        s->corh->CastFrom(*s->corl);
        s->vx->Axpy(*s->corh, 1.0);
        s->Ah->VectorMult(*s->vx, s->resh);
        s->resh->ScaleAdd(-1.0, *s->vb);
        res = s->resh->Norm2();
    }
    const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::memcpy(x, dynamic_cast<CPU_lVector<double> *>(s->vx)->buffer, sizeof(double) * n);
    *outer_done = outer;
    *inner_done = inner_total;
    *res_out = res;
    return dt;
}

void ref_mpir_destroy(void *h)
{
    MpirSession *s = static_cast<MpirSession *>(h);
    delete s->J;
    delete s->Ah; delete s->Al; delete s->vb; delete s->vx; delete s->resh; delete s->corh;
    delete s->resl; delete s->corl; delete s->dl;
    delete s;
}

// FP64 Jacobi-CG over the reference's objects with an iteration cap, timed
// (seconds, setup excluded): the plain-precision comparison.
double ref_pcg_timed(int impl, int nthreads, int n, int nnz, const int *row, const int *col, const double *val,
                     const double *b, double *x, double reltol, int maxits, int *iters)
{
    lMatrix<double> *A = make_matrix_t<double>(impl, n, nnz, row, col, val, nthreads);
    lVector<double> *vb = make_vector_t<double>(impl, n, nthreads), *vx = make_vector_t<double>(impl, n, nthreads);
    std::memcpy(dynamic_cast<CPU_lVector<double> *>(vb)->buffer, b, sizeof(double) * n);
    lVector<double> *d = vb->CloneWithoutContent();
    lPreconditioner_Jacobi<double> J;
    J.Init(*d);
    J.SetupOperator(*A);
    J.Build();
    Control ctl{maxits, 0.0, reltol, 1e6, 0.0};
    const auto t0 = std::chrono::steady_clock::now();
    pcg_t<double>(*A, J, *vb, *vx, ctl, 0, iters);
    const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::memcpy(x, dynamic_cast<CPU_lVector<double> *>(vx)->buffer, sizeof(double) * n);
    delete A; delete vb; delete vx; delete d;
    return dt;
}

}  // extern "C"
