// adapter_drive.cc -- TEST HARNESS: HiFlow3's own lmp code run on the B200 classes.
//
// Compiled with the B200 lmp classes (hiflow3_2.0_b200/hiflow/b200_lmp.cc) and
// the reference's own CPU lmp objects into libb200_hiflow.so; the GPU tests
// call these entry points through ctypes and compare with the reference on
// CPU objects (oracle/_ref).  Every algorithm below is the reference's code,
// unmodified and instantiated on B200_lVector<double> / B200_CSR_lMatrix<double>:
//
//   ad_jacobi     lPreconditioner_Jacobi Init / SetupOperator / Build / Apply (lpreconditioner.cc:90-165)
//   ad_lmp_cg     CGFunctor<double, true> (lmp/solvers/cg.h:103-221), with or without that Jacobi
//   ad_mcsgs      lPreconditioner_MultiColoring_SymmetricGaussSeidel Build + Apply
//                 (lpreconditioner_mc.cc:157-777, lpreconditioner_mc_sgs.cc:46-90)
//   ad_benchmark  the Benchmark<VectorType, MatrixType> flow of
//                 examples/benchmark_local_solver/benchmark_local_solver.cc:113-190:
//                 files read into CPUsimple objects, Init + CopyStructureFrom + CopyFrom
//                 onto the platform (its GPU read path, :71-111), the functor solve, and
//                 the check dot(x - x_result), with CGFunctor
//   ad_members    lVector / lMatrix members on B200 objects and on CPUsimple objects
//
// The lmp GMRESFunctor (lmp/solvers/gmres.h) is not driven: it needs
// SeqDenseMatrix (linear_algebra/seq_dense_matrix.cc), which needs Boost.
//
// Host matrices enter the way the reference's GPU read path does: a CPUsimple
// matrix, then Init + CopyStructureFrom + CopyFrom on the platform's object.
#include "b200_lmp.h"

#include "lmatrix_csr_cpu.h"
#include "lpreconditioner.h"
#include "lpreconditioner_mc_sgs.h"
#include "lvector_cpu.h"
#include "solvers/cg.h"

#include <cstring>
#include <memory>
#include <string>

using namespace hiflow::la;

namespace {
std::string g_err;

void host_matrix(CPUsimple_CSR_lMatrix<double> &h, int n, int nnz, const int *row, const int *col, const double *val)
{
    h.Init(nnz, n, n, "A");
    std::memcpy(h.matrix.row, row, sizeof(int) * (n + 1));
    std::memcpy(h.matrix.col, col, sizeof(int) * nnz);
    std::memcpy(h.matrix.val, val, sizeof(double) * nnz);
}

// the reference's GPU read path (benchmark_local_solver.cc:71-111)
void to_platform(B200_CSR_lMatrix<double> &A, const CPUsimple_CSR_lMatrix<double> &h)
{
    A.Init(h.get_nnz(), h.get_num_row(), h.get_num_col(), "A");
    A.CopyStructureFrom(h);
    A.CopyFrom(h);
}

void to_platform(B200_lVector<double> &v, const double *x, int n, const char *name)
{
    CPUsimple_lVector<double> h(n, name);
    if (x) std::memcpy(h.buffer, x, sizeof(double) * n);
    else h.Zeros();
    v.Init(n, name);
    v.CopyFrom(h);
}

void to_host(const B200_lVector<double> &v, double *out)
{
    CPUsimple_lVector<double> h(v.get_size(), "out");
    v.CopyTo(h);
    std::memcpy(out, h.buffer, sizeof(double) * v.get_size());
}

template <typename F>
int guarded(F &&f)
{
    try {
        return f();
    } catch (const std::exception &e) {
        g_err = e.what();
        return -1;
    }
}
}  // namespace

extern "C" {

const char *ad_last_error(void) { return g_err.c_str(); }

void ad_select_device(int device) { b200_lmp_select_device(device); }

int ad_jacobi(int n, int nnz, const int *row, const int *col, const double *val, const double *r, double *z)
{
    return guarded([&] {
        CPUsimple_CSR_lMatrix<double> h;
        host_matrix(h, n, nnz, row, col, val);
        B200_CSR_lMatrix<double> A;
        to_platform(A, h);
        B200_lVector<double> vr, vz;
        to_platform(vr, r, n, "r");
        to_platform(vz, nullptr, n, "z");
        lPreconditioner_Jacobi<double> J;
        J.Init(vz);
        J.SetupOperator(A);
        J.Build();
        J.ApplylPreconditioner(vr, &vz);
        to_host(vz, z);
        return 0;
    });
}

int ad_lmp_cg(int n, int nnz, const int *row, const int *col, const double *val, const double *b, double *x,
              double rel_eps, double abs_eps, int max_iter, int jacobi, int *iters)
{
    return guarded([&] {
        CPUsimple_CSR_lMatrix<double> h;
        host_matrix(h, n, nnz, row, col, val);
        B200_CSR_lMatrix<double> A;
        to_platform(A, h);
        B200_lVector<double> vb, vx;
        to_platform(vb, b, n, "b");
        to_platform(vx, x, n, "x");
        std::unique_ptr<lPreconditioner_Jacobi<double>> J;
        B200_lVector<double> dj;
        if (jacobi) {
            to_platform(dj, nullptr, n, "d");
            J.reset(new lPreconditioner_Jacobi<double>());
            J->Init(dj);
            J->SetupOperator(A);
            J->Build();
        }
        CGFunctor<double, true> cg;
        int it = max_iter;
        const int rc = cg(&vx, &vb, &A, rel_eps, abs_eps, it, -1, J.get());
        *iters = it;
        to_host(vx, x);
        return rc;
    });
}

// The reference's multicoloured symmetric Gauss-Seidel on B200 objects: the
// operator, its permuted copy and the permuted vectors are B200 objects; the
// build clones to CPU objects where the reference does so for GPU platforms.
int ad_mcsgs(int n, int nnz, const int *row, const int *col, const double *val, const double *r_perm,
             double *z_perm, int *perm, int *ncolors)
{
    return guarded([&] {
        CPUsimple_CSR_lMatrix<double> h;
        host_matrix(h, n, nnz, row, col, val);
        B200_CSR_lMatrix<double> A, Ap;
        to_platform(A, h);
        to_platform(Ap, h);
        B200_lVector<double> xx, rhs;
        to_platform(xx, nullptr, n, "x");
        to_platform(rhs, nullptr, n, "rhs");
        lPreconditioner_MultiColoring_SymmetricGaussSeidel<double> P;
        P.SetupOperator(A);
        P.SetupPermOperator(Ap);
        P.SetupPermVectors(&xx, &rhs);
        P.Build();
        std::memcpy(perm, P.get_permut(), sizeof(int) * n);
        B200_lVector<double> vr, vz;
        to_platform(vr, r_perm, n, "r");
        to_platform(vz, nullptr, n, "z");
        P.ApplylPreconditioner(vr, &vz);
        to_host(vz, z_perm);
        (void)ncolors;
        return 0;
    });
}

// benchmark_local_solver.cc:113-190 with VectorType / MatrixType = the B200
// classes and its "cg" solver, CGFunctor<double, true>; rel_eps 1e-8, abs_eps
// 1e-14, max_iter 1000 as there.  Returns the solver's code; *dot =
// dot(x - x_result), *iters the iterations of the last solve.
int ad_benchmark(const char *file_A, const char *file_b, const char *file_x_result, const char *file_x_start,
                 int repetitions, double *dot, int *iters)
{
    return guarded([&] {
        auto read_vector = [](B200_lVector<double> &v, const char *f) {
            CPUsimple_lVector<double> s;
            s.ReadFile(f);
            v.Init(s.get_size(), "v");
            v.CopyFrom(s);
        };
        B200_lVector<double> b, x;
        read_vector(b, file_b);
        read_vector(x, file_x_start);
        B200_CSR_lMatrix<double> A;
        {
            CPUsimple_CSR_lMatrix<double> simpleA;
            simpleA.ReadFile(file_A);
            A.Init(simpleA.get_nnz(), simpleA.get_num_row(), simpleA.get_num_col(), "A");
            A.CopyStructureFrom(simpleA);
            A.CopyFrom(simpleA);
        }
        const double rel_eps = 1e-8, abs_eps = 1e-14;
        int rc = 0, it = 0;
        for (int k = 0; k < repetitions; ++k) {
            read_vector(x, file_x_start);
            it = 1000;
            CGFunctor<double, true> s;
            rc = s(&x, &b, &A, rel_eps, abs_eps, it, -1);
            if (rc != 0) return rc;
        }
        B200_lVector<double> x_result;
        read_vector(x_result, file_x_result);
        B200_lVector<double> r(x.get_size(), "r");
        r.CopyFrom(x_result);
        r.ScaleAdd(-1.0, x);
        *dot = r.Dot(r);
        *iters = it;
        return rc;
    });
}

// lVector / lMatrix members on B200 objects against the same calls on
// CPUsimple objects: a fixed script of operations, each result copied out
// (out must hold 16 n + 64 doubles).  Returns the number of values written.
int ad_members(int n, int nnz, const int *row, const int *col, const double *val, const double *x0,
               const double *y0, int platform, double *out)
{
    return guarded([&] {
        int k = 0;
        auto put = [&](const lVector<double> &v) {
            CPUsimple_lVector<double> h(v.get_size(), "o");
            h.CopyFrom(v);
            std::memcpy(out + k, h.buffer, sizeof(double) * v.get_size());
            k += v.get_size();
        };
        auto put1 = [&](double v) { out[k++] = v; };
        std::unique_ptr<lVector<double>> x, y;
        std::unique_ptr<lMatrix<double>> A;
        CPUsimple_CSR_lMatrix<double> h;
        host_matrix(h, n, nnz, row, col, val);
        if (platform) {
            B200_lVector<double> *bx = new B200_lVector<double>(), *by = new B200_lVector<double>();
            to_platform(*bx, x0, n, "x");
            to_platform(*by, y0, n, "y");
            x.reset(bx);
            y.reset(by);
            B200_CSR_lMatrix<double> *bA = new B200_CSR_lMatrix<double>();
            to_platform(*bA, h);
            A.reset(bA);
        } else {
            CPUsimple_lVector<double> *cx = new CPUsimple_lVector<double>(n, "x"), *cy = new CPUsimple_lVector<double>(n, "y");
            std::memcpy(cx->buffer, x0, sizeof(double) * n);
            std::memcpy(cy->buffer, y0, sizeof(double) * n);
            x.reset(cx);
            y.reset(cy);
            CPUsimple_CSR_lMatrix<double> *cA = new CPUsimple_CSR_lMatrix<double>();
            cA->CloneFrom(h);
            A.reset(cA);
        }
        std::unique_ptr<lVector<double>> t(x->CloneWithoutContent());
        A->VectorMult(*x, t.get());
        put(*t);                                         // A x
        A->VectorMultAdd(*y, t.get());
        put(*t);                                         // A x + A y
        put1(x->Dot(*y));
        put1(x->Norm2());
        put1(x->Norm1());
        put1(x->NormMax());
        put1(x->ArgMax());
        put1(x->ArgMin());
        t->CopyFrom(*x);
        t->Axpy(*y, 0.25);
        put(*t);                                         // x + y/4
        t->ScaleAdd(-2.0, *y);
        put(*t);                                         // -2 t + y
        t->Scale(3.0);
        put(*t);
        t->CopyFrom(*x);
        t->ElementWiseMult(*y);
        put(*t);                                         // x .* y
        std::unique_ptr<lVector<double>> s(x->extract_subvector(n / 4, n / 2));
        put(*s);
        t->CopyFrom(*y);
        t->partial_replace_subvector(0, 0, s->get_size(), *s);
        put(*t);
        t->partial_add_subvector(1, 0, s->get_size() - 1, 0.5, *s);
        put(*t);
        std::vector<int> idx;
        for (int i = 0; i < n; i += 3) idx.push_back(n - 1 - i);
        std::vector<double> v(idx.size());
        for (size_t i = 0; i < idx.size(); ++i) v[i] = 0.125 * (double)i;
        t->SetValues(idx.data(), (int)idx.size(), v.data());
        t->add_values(idx.data(), (int)idx.size(), v.data());
        put(*t);
        t->GetValues(idx.data(), 3, out + k);
        k += 3;
        t->set_indexset(idx.data(), (int)idx.size());
        t->GetIndexedValues(v.data());
        for (double e : v) put1(e);
        std::vector<int> p(n);
        for (int i = 0; i < n; ++i) p[i] = (i * 7 + 3) % n;   // a permutation when gcd(7, n) = 1
        t->CopyFrom(*x);
        t->Reorder(p.data());
        put(*t);
        std::unique_ptr<lVector<double>> dg(x->CloneWithoutContent());
        A->extract_diagelements(0, n, dg.get());
        put(*dg);
        A->extract_invdiagelements(0, n, dg.get());
        put(*dg);
        std::unique_ptr<lMatrix<double>> S(A->extract_submatrix(0, 0, n / 2, n / 2));
        std::unique_ptr<lVector<double>> xs(x->extract_subvector(0, n / 2)), ys(x->extract_subvector(0, n / 2));
        S->VectorMult(*xs, ys.get());
        put(*ys);
        A->Scale(0.5);
        A->VectorMult(*x, t.get());
        put(*t);
        A->ScaleOffdiag(2.0);
        A->VectorMult(*x, t.get());
        put(*t);
        return k;
    });
}

}  // extern "C"
