// host_setup.cc -- one-time host algorithms (see host_setup.h).
//
// Built with -ffp-contract=off so that floating-point expressions evaluate in
// the written order, as the reference's host code does.
#include "host_setup.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace b200 {
namespace host {

void coo_to_csr(int n_rows, int nnz, const int *coo_row, const int *coo_col, const double *coo_val, int *row,
                int *col, double *val)
{
    // counting by row, exclusive scan, scatter in input order
    std::fill(row, row + n_rows + 1, 0);
    for (int e = 0; e < nnz; ++e) row[coo_row[e]] += 1;
    std::vector<int> fill(n_rows);
    int run = 0;
    for (int r = 0; r < n_rows; ++r) {
        const int cnt = row[r];
        row[r] = run;
        fill[r] = run;
        run += cnt;
    }
    row[n_rows] = nnz;
    for (int e = 0; e < nnz; ++e) {
        const int slot = fill[coo_row[e]]++;
        col[slot] = coo_col[e];
        if (coo_val) val[slot] = coo_val[e];
    }
    // per row: selection sort of the columns, each minimum swapped (with its
    // value) into place -- the reference's order, which fixes where duplicate
    // (row, col) pairs end up
    for (int r = 0; r < n_rows; ++r) {
        const int end = row[r + 1];
        for (int a = row[r]; a < end; ++a) {
            int best = a;
            for (int b = a + 1; b < end; ++b)
                if (col[b] < col[best]) best = b;
            std::swap(col[a], col[best]);
            if (coo_val) std::swap(val[a], val[best]);
        }
    }
}

void add_values(const int *row, const int *col, double *val, const int *rows, int num_rows, const int *cols,
                int num_cols, const double *values)
{
    // sorted merge of the element's columns into the stored row
    for (int i = 0; i < num_rows; ++i) {
        const double *v = values + (size_t)i * num_cols;
        int k = 0;
        const int end = row[rows[i] + 1];
        for (int j = row[rows[i]]; j != end && k < num_cols; ++j) {
            if (cols[k] < col[j]) {
                while (k < num_cols && cols[k] < col[j]) ++k;
                if (k >= num_cols) break;
            }
            if (cols[k] == col[j]) {
                val[j] += v[k];
                ++k;
            }
        }
    }
}

void zero_rows(const int *row, const int *col, double *val, const int *idx, int size, double alpha)
{
    for (int t = 0; t < size; ++t) {
        const int r = idx[t];
        for (int j = row[r]; j < row[r + 1]; ++j) val[j] = (col[j] == r) ? alpha : 0.0;
    }
}

int q1_sizes(int dim, int N, int *n, int64_t *nnz)
{
    if ((dim != 2 && dim != 3) || N < 1) return -1;
    const int64_t p = N + 1, s = 3 * (int64_t)N + 1;
    const int64_t nn = dim == 2 ? p * p : p * p * p;
    const int64_t nz = dim == 2 ? s * s : s * s * s;
    if (nn > 0x7fffffff || nz > 0x7fffffff) return -2;
    *n = (int)nn;
    *nnz = nz;
    return 0;
}

void q1_tables(int dim, double h, Q1Tables &t)
{
    t.dim = dim;
    t.nv = t.nq = 1 << dim;
    const double g = 1.0 / std::sqrt(3.0);
    const double pts[2] = {(1.0 - g) / 2.0, (1.0 + g) / 2.0};
    for (int q = 0; q < t.nq; ++q) {
        const double xi[3] = {pts[q & 1], pts[(q >> 1) & 1], pts[(q >> 2) & 1]};
        double w = 1.0;
        for (int d = 0; d < dim; ++d) w *= 0.5;
        t.w[q] = w;
        for (int a = 0; a < t.nv; ++a) {
            double f[3];
            for (int d = 0; d < dim; ++d) f[d] = ((a >> d) & 1) ? xi[d] : 1.0 - xi[d];
            double p = 1.0;
            for (int d = 0; d < dim; ++d) p *= f[d];
            t.phi[q][a] = p;
            for (int d = 0; d < dim; ++d) {
                double gd = ((a >> d) & 1) ? 1.0 : -1.0;
                for (int e = 0; e < dim; ++e)
                    if (e != d) gd *= f[e];
                t.grad[q][a][d] = gd / h;
            }
        }
    }
    for (int q = 0; q < t.nq; ++q)
        for (int i = 0; i < t.nv; ++i)
            for (int j = 0; j < t.nv; ++j) {
                double s = 0.0;
                for (int d = 0; d < dim; ++d) s += t.grad[q][j][d] * t.grad[q][i][d];
                t.gg[q][i][j] = s;
            }
    t.dJ = 1.0;
    for (int d = 0; d < dim; ++d) t.dJ *= h;
}

namespace {

void q1_element(const Q1Tables &t, int kind, double coef, const double *beta, double *Ke)
{
    const int nv = t.nv;
    std::fill(Ke, Ke + nv * nv, 0.0);
    for (int q = 0; q < t.nq; ++q) {
        for (int i = 0; i < nv; ++i)
            for (int j = 0; j < nv; ++j) Ke[i * nv + j] += t.w[q] * (coef * t.gg[q][i][j]) * t.dJ;
        if (kind == 1)
            for (int i = 0; i < nv; ++i)
                for (int j = 0; j < nv; ++j) {
                    double bg = 0.0;
                    for (int d = 0; d < t.dim; ++d) bg += beta[d] * t.grad[q][j][d];
                    Ke[i * nv + j] += t.w[q] * (bg * t.phi[q][i]) * t.dJ;
                }
    }
}

}  // namespace

int q1_dirichlet(int dim, int N, int *idx)
{
    const int P = N + 1, PZ = dim == 3 ? P : 1;
    int c = 0;
    for (int k = 0; k < PZ; ++k)
        for (int j = 0; j < P; ++j)
            for (int i = 0; i < P; ++i) {
                const bool on = i == 0 || i == N || j == 0 || j == N || (dim == 3 && (k == 0 || k == N));
                if (on) idx[c++] = i + P * (j + P * k);
            }
    return c;
}

int q1_assemble(int dim, int N, int kind, const double *kcell, double nu, const double *beta, int *row, int *col,
                double *val)
{
    int n;
    int64_t nnz;
    if (q1_sizes(dim, N, &n, &nnz)) return -1;
    const int P = N + 1, PZ = dim == 3 ? P : 1;
    // structure: the full Q1 stencil of every node, columns ascending
    // (the CSR init_structure would produce from these COO pairs)
    row[0] = 0;
    int64_t e = 0;
    for (int k = 0; k < PZ; ++k)
        for (int j = 0; j < P; ++j)
            for (int i = 0; i < P; ++i) {
                for (int dk = (dim == 3 ? -1 : 0); dk <= (dim == 3 ? 1 : 0); ++dk)
                    for (int dj = -1; dj <= 1; ++dj)
                        for (int di = -1; di <= 1; ++di) {
                            const int ii = i + di, jj = j + dj, kk = k + dk;
                            if (ii < 0 || ii >= P || jj < 0 || jj >= P || kk < 0 || kk >= PZ) continue;
                            col[e++] = ii + P * (jj + P * kk);
                        }
                row[i + P * (j + P * k) + 1] = (int)e;
            }
    std::memset(val, 0, sizeof(double) * nnz);
    Q1Tables t;
    q1_tables(dim, 1.0 / N, t);
    const int nv = t.nv, CZ = dim == 3 ? N : 1;
    double Ke[64];
    const double c0 = kind == 0 ? 1.0 : nu;
    if (!kcell) q1_element(t, kind, c0, beta, Ke);
    int dofs[8];
    for (int cz = 0; cz < CZ; ++cz)
        for (int cy = 0; cy < N; ++cy)
            for (int cx = 0; cx < N; ++cx) {
                for (int a = 0; a < nv; ++a)
                    dofs[a] = (cx + (a & 1)) + P * ((cy + ((a >> 1) & 1)) + P * (cz + ((a >> 2) & 1)));
                if (kcell) q1_element(t, kind, kcell[cx + (int64_t)N * (cy + (int64_t)N * cz)], beta, Ke);
                add_values(row, col, val, dofs, nv, dofs, nv, Ke);
            }
    std::vector<int> bnd(n);
    const int nb = q1_dirichlet(dim, N, bnd.data());
    zero_rows(row, col, val, bnd.data(), nb, 1.0);
    return 0;
}

void q1_rhs(uint64_t seed, int dim, int N, double *b)
{
    // splitmix64 stream: the k-th draw (k = DoF index + 1) mapped to [-1, 1)
    // with a 53-bit mantissa; 0 on Dirichlet DoFs
    const int P = N + 1, PZ = dim == 3 ? P : 1;
    int64_t i = 0;
    for (int k = 0; k < PZ; ++k)
        for (int j = 0; j < P; ++j)
            for (int ii = 0; ii < P; ++ii, ++i) {
                uint64_t z = seed + (uint64_t)(i + 1) * 0x9E3779B97F4A7C15ULL;
                z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
                z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
                z ^= z >> 31;
                const double u = 2.0 * ((double)(z >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
                const bool on = ii == 0 || ii == N || j == 0 || j == N || (dim == 3 && (k == 0 || k == N));
                b[i] = on ? 0.0 : u;
            }
}

int multicoloring(int n, const int *row, const int *col, int *ncolors, std::vector<int> &sizes,
                  std::vector<int> &perm)
{
    // Greedy colouring in row order: a node starts at colour 1 and, scanning
    // its row's columns (the whole scan repeated up to row-length times),
    // moves up one colour whenever a neighbour holds its current colour.  A
    // scan without a move ends the repetitions early: the rest would repeat it.
    std::vector<int> c(n, 0);
    int top = 0;
    for (int j = 0; j < n; ++j) {
        c[j] = 1;
        const int b = row[j], e = row[j + 1];
        for (int pass = b; pass < e; ++pass) {
            bool moved = false;
            for (int t = b; t < e; ++t) {
                const int nb = col[t];
                if (nb == j) continue;
                if (c[nb] == c[j]) {
                    ++c[j];
                    moved = true;
                }
                top = std::max(top, c[j]);
            }
            if (!moved) break;
        }
    }
    if (top == 0) return -1;
    *ncolors = top;
    sizes.assign(top, 0);
    for (int i = 0; i < n; ++i) ++sizes[c[i] - 1];
    std::vector<int> at(top, 0);
    for (int k = 1; k < top; ++k) at[k] = at[k - 1] + sizes[k - 1];
    perm.resize(n);
    for (int j = 0; j < n; ++j) perm[at[c[j] - 1]++] = j;
    return 0;
}

int levelscheduling(int n, const int *row, const int *col, int *nlevels, std::vector<int> &sizes,
                    std::vector<int> &perm)
{
    // For a structurally symmetric pattern the reference's sweep assigns
    // level(k) = 1 + max level over k's lower neighbours (0 if none), and
    // lists a level's nodes in index order.  Other patterns replay the sweep.
    auto present = [&](int r, int c) {
        const int *b = col + row[r], *e = col + row[r + 1];
        if (std::binary_search(b, e, c)) return true;
        return std::find(b, e, c) != e;
    };
    bool sym = true;
    for (int i = 0; i < n && sym; ++i)
        for (int j = row[i]; j < row[i + 1]; ++j)
            if (col[j] != i && !present(col[j], i)) {
                sym = false;
                break;
            }
    perm.resize(n);
    if (sym) {
        std::vector<int> lev(n);
        int top = -1;
        for (int k = 0; k < n; ++k) {
            int l = 0;
            for (int j = row[k]; j < row[k + 1]; ++j)
                if (col[j] < k) l = std::max(l, lev[col[j]] + 1);
            lev[k] = l;
            top = std::max(top, l);
        }
        sizes.assign(top + 1, 0);
        for (int k = 0; k < n; ++k) ++sizes[lev[k]];
        std::vector<int> at(top + 1, 0);
        for (int l = 1; l <= top; ++l) at[l] = at[l - 1] + sizes[l - 1];
        for (int k = 0; k < n; ++k) perm[at[lev[k]]++] = k;
        *nlevels = top + 1;
        return 0;
    }
    std::vector<int> depth(n, 0);
    std::vector<char> placed(n, 0);
    sizes.clear();
    int done = 0;
    for (int L = 0; L < n && done < n; ++L) {
        const int before = done;
        for (int k = 0; k < n; ++k) {
            if (placed[k] || depth[k] != L) continue;
            bool ready = true;
            for (int j = row[k]; j < row[k + 1]; ++j)
                if (col[j] < k && !placed[col[j]]) {
                    ready = false;
                    break;
                }
            if (!ready) continue;
            perm[done++] = k;
            placed[k] = 1;
            for (int j = row[k]; j < row[k + 1]; ++j)
                if (col[j] > k && depth[col[j]] <= depth[k]) depth[col[j]] = depth[k] + 1;
        }
        sizes.push_back(done - before);
    }
    if (done != n) {
        *nlevels = 0;
        return -1;
    }
    *nlevels = (int)sizes.size();
    return 0;
}

void reorder(const Csr &A, const std::vector<int> &perm, Csr &B)
{
    const int n = A.n, nnz = A.nnz();
    std::vector<int> inv(n), cr(nnz), cc(nnz);
    for (int i = 0; i < n; ++i) inv[perm[i]] = i;
    for (int i = 0; i < n; ++i)
        for (int j = A.row[i]; j < A.row[i + 1]; ++j) {
            cr[j] = inv[i];
            cc[j] = inv[A.col[j]];
        }
    B.n = n;
    B.m = A.m;
    B.row.assign(n + 1, 0);
    B.col.assign(nnz, 0);
    B.val.assign(nnz, 0.0);
    coo_to_csr(n, nnz, cr.data(), cc.data(), A.val.data(), B.row.data(), B.col.data(), B.val.data());
}

void ilu0(int n, const int *row, const int *col, double *val)
{
    // IKJ ILU(0) on the stored pattern; the pivot position is searched afresh
    // for every row k used (and kept from the previous search if absent)
    int piv = 0;
    for (int i = 1; i < n; ++i) {
        for (int ik = row[i]; col[ik] < i; ++ik) {
            const int k = col[ik];
            for (int p = row[k]; p < row[k + 1]; ++p)
                if (col[p] == k) piv = p;
            val[ik] = val[ik] / (1.0 * val[piv]);
            for (int ij = ik + 1; ij < row[i + 1]; ++ij) {
                double akj = 0.0;
                for (int p = row[k]; p < row[k + 1]; ++p)
                    if (col[p] == col[ij]) akj = val[p];
                val[ij] = val[ij] - val[ik] * akj;
            }
        }
    }
}

void matrix_sup_power(const Csr &A, int p, Csr &P)
{
    // row i of the product with A: the union of the rows of A named by the
    // columns of row i (the symbolic product of Bank & Douglas); columns in
    // ascending order, as the reference's COO round trip leaves them
    const int n = A.n;
    P = A;
    std::vector<int> mark(A.m > n ? A.m : n, -1), cols;
    for (int it = 1; it < p; ++it) {
        Csr Q;
        Q.n = n;
        Q.m = A.m;
        Q.row.assign(n + 1, 0);
        for (int i = 0; i < n; ++i) {
            cols.clear();
            for (int a = P.row[i]; a < P.row[i + 1]; ++a) {
                const int k = P.col[a];
                for (int b = A.row[k]; b < A.row[k + 1]; ++b) {
                    const int j = A.col[b];
                    if (mark[j] != i) {
                        mark[j] = i;
                        cols.push_back(j);
                    }
                }
            }
            std::sort(cols.begin(), cols.end());
            Q.col.insert(Q.col.end(), cols.begin(), cols.end());
            Q.row[i + 1] = (int)Q.col.size();
        }
        Q.val.assign(Q.col.size(), 1.0);
        std::fill(mark.begin(), mark.end(), -1);
        P = std::move(Q);
    }
}

void ilup(const Csr &A, int p, Csr &LU)
{
    const int n = A.n;
    // the pattern of A^(p+1) carrying A's values (zeros elsewhere)
    Csr F;
    matrix_sup_power(A, p + 1, F);
    for (int i = 0; i < n; ++i)
        for (int j = F.row[i]; j < F.row[i + 1]; ++j) {
            double v = 0.0;
            for (int k = A.row[i]; k < A.row[i + 1]; ++k)
                if (F.col[j] == A.col[k]) v += A.val[k];
            F.val[j] = v;
        }
    // level of fill: 0 for nonzero entries of A, 9999 for the rest
    std::vector<double> lev(F.col.size());
    for (size_t j = 0; j < lev.size(); ++j) lev[j] = F.val[j] * F.val[j] > 0.0 ? 0.0 : 9999.0;
    const double pp = (double)p;
    int kk = 0;
    for (int i = 1; i < n; ++i) {
        for (int ik = F.row[i]; F.col[ik] < i; ++ik) {
            if (!(lev[ik] <= pp)) continue;
            const int k = F.col[ik];
            for (int h = F.row[k]; h < F.row[k + 1]; ++h)
                if (F.col[h] == k) {
                    kk = h;
                    break;
                }
            F.val[ik] = F.val[ik] / (1.0 * F.val[kk]);
            for (int ij = ik + 1; ij < F.row[i + 1]; ++ij) {
                double vkj = 0.0, lkj = 9999;
                for (int h = F.row[k]; h < F.row[k + 1]; ++h)
                    if (F.col[h] == F.col[ij]) {
                        vkj = F.val[h];
                        lkj = lev[h];
                        break;
                    }
                const double lt = 1 + lkj + lev[ik];
                F.val[ij] = F.val[ij] - vkj * F.val[ik];
                if (lev[ij] > lt) lev[ij] = lt;
            }
        }
        for (int h = F.row[i]; h < F.row[i + 1]; ++h)
            if (lev[h] > pp) {
                F.val[h] = 0.0;
                lev[h] = 9999.0;
            }
    }
    // keep the entries of level <= p
    LU.n = n;
    LU.m = A.m;
    LU.row.assign(n + 1, 0);
    LU.col.clear();
    LU.val.clear();
    for (int i = 0; i < n; ++i) {
        for (int h = F.row[i]; h < F.row[i + 1]; ++h)
            if (lev[h] <= pp) {
                LU.col.push_back(F.col[h]);
                LU.val.push_back(F.val[h]);
            }
        LU.row[i + 1] = (int)LU.col.size();
    }
}

void dropoffs(Csr &A, const std::vector<int> &block_off)
{
    const int n = A.n;
    std::vector<int> blk(n);
    for (size_t b = 0; b + 1 < block_off.size(); ++b)
        for (int i = block_off[b]; i < block_off[b + 1]; ++i) blk[i] = (int)b;
    int dropped = 0;
    for (int i = 0; i < n; ++i)
        for (int j = A.row[i]; j < A.row[i + 1]; ++j)
            if (A.col[j] != i && blk[A.col[j]] == blk[i]) {
                A.val[j] = 0.0;
                ++dropped;
            }
    if (!dropped) return;
    // compress: keep only nonzero entries (all of them, as compress_me does)
    Csr B;
    B.n = n;
    B.m = A.m;
    B.row.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        for (int j = A.row[i]; j < A.row[i + 1]; ++j)
            if (A.val[j] != 0.0) {
                B.col.push_back(A.col[j]);
                B.val.push_back(A.val[j]);
            }
        B.row[i + 1] = (int)B.col.size();
    }
    A = std::move(B);
}

bool row_patterns(int n, const int *row, const int *col, int max_pat, int max_delta, std::vector<uint16_t> &pid,
                  std::vector<int> &pat_off, std::vector<int> &pat_delta)
{
    pid.assign(n, 0);
    pat_off.assign(1, 0);
    pat_delta.clear();
    // open-addressing table keyed by a 64-bit hash of the offset sequence
    const size_t cap = 4096;
    std::vector<long long> key(cap, -1);
    std::vector<int> slot_pat(cap, -1);
    for (int i = 0; i < n; ++i) {
        uint64_t h = 1469598103934665603ULL ^ (uint64_t)(row[i + 1] - row[i]);
        for (int j = row[i]; j < row[i + 1]; ++j) {
            h ^= (uint64_t)(uint32_t)(col[j] - i);
            h *= 1099511628211ULL;
        }
        size_t s = (size_t)(h % cap);
        int found = -1;
        for (size_t probe = 0; probe < cap; ++probe, s = (s + 1) % cap) {
            if (key[s] == -1) break;
            if (key[s] == (long long)(h >> 1)) {
                const int p = slot_pat[s];
                const int len = pat_off[p + 1] - pat_off[p];
                bool same = len == row[i + 1] - row[i];
                for (int k = 0; same && k < len; ++k) same = pat_delta[pat_off[p] + k] == col[row[i] + k] - i;
                if (same) {
                    found = p;
                    break;
                }
            }
        }
        if (found < 0) {
            found = (int)pat_off.size() - 1;
            if (found >= max_pat || (int)pat_delta.size() + (row[i + 1] - row[i]) > max_delta) return false;
            for (int j = row[i]; j < row[i + 1]; ++j) pat_delta.push_back(col[j] - i);
            pat_off.push_back((int)pat_delta.size());
            if (key[s] != -1) {
                // the probe stopped on a different key: find a free slot
                while (key[s] != -1) s = (s + 1) % cap;
            }
            key[s] = (long long)(h >> 1);
            slot_pat[s] = found;
        }
        pid[i] = (uint16_t)found;
    }
    return true;
}

void pattern_lines(const std::vector<int> &pat_delta, std::vector<int> &line_start, std::vector<int> &line_span,
                   std::vector<int> &entry_line, std::vector<int> &entry_lo)
{
    std::vector<int> d(pat_delta);
    std::sort(d.begin(), d.end());
    d.erase(std::unique(d.begin(), d.end()), d.end());
    line_start.clear();
    line_span.clear();
    for (size_t i = 0; i < d.size(); ++i) {
        if (i == 0 || d[i] != d[i - 1] + 1) {
            line_start.push_back(d[i]);
            line_span.push_back(0);
        } else {
            line_span.back() = d[i] - line_start.back();
        }
    }
    entry_line.resize(pat_delta.size());
    entry_lo.resize(pat_delta.size());
    for (size_t k = 0; k < pat_delta.size(); ++k) {
        const int l = (int)(std::upper_bound(line_start.begin(), line_start.end(), pat_delta[k]) - line_start.begin()) - 1;
        entry_line[k] = l;
        entry_lo[k] = pat_delta[k] - line_start[l];
    }
}

int validate_csr(int n_rows, int n_cols, int nnz, const int *row, const int *col, long long *bad_at)
{
    if (n_rows < 0 || n_cols < 0 || nnz < 0) return -1;
    if (row[0] != 0) {
        *bad_at = 0;
        return -2;
    }
    for (int i = 0; i < n_rows; ++i)
        if (row[i + 1] < row[i]) {
            *bad_at = i;
            return -3;
        }
    if (row[n_rows] != nnz) {
        *bad_at = n_rows;
        return -4;
    }
    for (int j = 0; j < nnz; ++j)
        if (col[j] < 0 || col[j] >= n_cols) {
            *bad_at = j;
            return -5;
        }
    return 0;
}

}  // namespace host
}  // namespace b200
