// host_setup.h -- one-time host algorithms of the B200 lmp platform.
//
// These restate the reference's host-side lmp routines that run once per
// operator (assembly into CSR, multicolouring, level scheduling, symmetric
// permutation, ILU(0) factorisation).  Their results (structure, colours,
// permutations, levels, factors) must equal the reference's bit for bit, so
// each keeps the reference's order of operations; the citations name the
// routine restated (paths relative to the HiFlow3 2.0 tree).
#pragma once

#include <cstdint>
#include <vector>

namespace b200 {
namespace host {

struct Csr {
    int n = 0, m = 0;
    std::vector<int> row, col;
    std::vector<double> val;
    int nnz() const { return row.empty() ? 0 : row[n]; }
};

// lmp/lmatrix_csr_cpu.cc:951-1044 (TransformFromCOO / init_structure)
void coo_to_csr(int n_rows, int nnz, const int *coo_row, const int *coo_col, const double *coo_val, int *row,
                int *col, double *val);
// lmp/lmatrix_csr_cpu.cc:1148-1181
void add_values(const int *row, const int *col, double *val, const int *rows, int num_rows, const int *cols,
                int num_cols, const double *values);
// lmp/lmatrix_csr_cpu.cc:1047-1068
void zero_rows(const int *row, const int *col, double *val, const int *idx, int size, double alpha);

// Structured Q1 systems: lexicographic DoFs (x fastest), element matrices of
// examples/poisson/poisson_tutorial.h:152-176 (kind 0) and
// examples/convection_diffusion/convdiff.cc:75-117 (kind 1) with 2-point Gauss.
// Quadrature tables of the Q1 element on a cell of side h: shape values,
// gradients, weights, gradient products and the Jacobian determinant.  The
// device assembler uploads these very numbers so that both assemblers round
// identically.
struct Q1Tables {
    int dim, nv, nq;
    double phi[8][8];       // [q][a]
    double grad[8][8][3];   // [q][a][d]
    double w[8];
    double gg[8][8][8];     // [q][i][j] = grad_j . grad_i
    double dJ;
};
void q1_tables(int dim, double h, Q1Tables &t);
int q1_sizes(int dim, int N, int *n, int64_t *nnz);
int q1_assemble(int dim, int N, int kind, const double *kcell, double nu, const double *beta, int *row, int *col,
                double *val);
int q1_dirichlet(int dim, int N, int *idx);
void q1_rhs(uint64_t seed, int dim, int N, double *b);

// lmp/lmatrix_csr_cpu.cc:2175-2290; perm[new] = old
int multicoloring(int n, const int *row, const int *col, int *ncolors, std::vector<int> &sizes,
                  std::vector<int> &perm);
// lmp/lmatrix_csr_cpu.cc:2295-2392; perm[new] = old
int levelscheduling(int n, const int *row, const int *col, int *nlevels, std::vector<int> &sizes,
                    std::vector<int> &perm);
// lmp/lmatrix_csr_cpu.cc:1847-1861 via COO (lmp/lmatrix_coo_cpu.cc:1019-1060)
void reorder(const Csr &A, const std::vector<int> &perm, Csr &B);
// lmp/lmatrix_csr_cpu.cc:1880-1930 (in place)
void ilu0(int n, const int *row, const int *col, double *val);
// lmp/lmatrix_csr_cpu.cc:1641-1664 (MatrixSupSPower) over :1520-1636
// (MatrixMultSupStructure): the pattern of A^p (p >= 1; p = 1 copies A);
// values are 1 for p > 1.
void matrix_sup_power(const Csr &A, int p, Csr &P);
// lmp/lmatrix_csr_cpu.cc:1933-2104 (ilup): ILU(p) by levels of fill on the
// pattern of A^(p+1), compressed to the entries of level <= p.
void ilup(const Csr &A, int p, Csr &LU);
// lmp/lpreconditioner_mc.cc:647-693 + lmp/lmatrix_csr_cpu.cc:2436-2495
void dropoffs(Csr &A, const std::vector<int> &block_off);

// Row-pattern dictionary of a CSR: rows whose column offsets relative to the
// row index (col - i, in column order) coincide share one pattern.  Fills
// pid[n], pattern offsets pat_off[npat+1] and the offsets themselves; returns
// false (leaving the outputs unspecified) when more than max_pat patterns or
// more than max_delta stored offsets would be needed.
bool row_patterns(int n, const int *row, const int *col, int max_pat, int max_delta, std::vector<uint16_t> &pid,
                  std::vector<int> &pat_off, std::vector<int> &pat_delta);

// Gather lines of a pattern table: the union of all pattern offsets, split
// into runs of consecutive integers [line_start[l], line_start[l] + line_span[l]].
// For every stored offset, its run (entry_line) and its position in the run
// (entry_lo).  A tile of R consecutive rows then reads x only on the lines
// shifted by the tile's first row, each R + span long.
void pattern_lines(const std::vector<int> &pat_delta, std::vector<int> &line_start, std::vector<int> &line_span,
                   std::vector<int> &entry_line, std::vector<int> &entry_lo);

// Validation of a CSR before upload: row monotone, row[0] == 0, columns in
// [0, n_cols).  Returns 0 or a negative code naming the first violation.
int validate_csr(int n_rows, int n_cols, int nnz, const int *row, const int *col, long long *bad_at);

}  // namespace host
}  // namespace b200
