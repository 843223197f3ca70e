// mmio.cc -- MatrixMarket matrices and plain-text vectors, host side.
//
// The file formats and their reading rules follow HiFlow3's lmp I/O:
//   - CPU_CSR_lMatrix::ReadFile / WriteFile (lmp/lmatrix_csr_cpu.cc:1733-1765)
//     go through CPU_COO_lMatrix::ReadFile / WriteFile
//     (lmp/lmatrix_coo_cpu.cc:133-299) and the MatrixMarket banner and size
//     parsers of lmp/mmio.cc:103-219;
//   - CPU_lVector::ReadFile / WriteFile (lmp/lvector_cpu.cc:582-663).
// Matrices end up in CSR through the same COO -> CSR transformation as the
// reference (TransformFromCOO, host_setup.cc), so a file read here gives the
// reference's CSR entry for entry.
//
// Where the reference exits the process (unreadable file, unsupported type,
// short file), these functions return B200LA_ERR_IO / B200LA_ERR_FORMAT; an
// entry index outside the declared size is B200LA_ERR_CSR (the reference
// does not check it).  Everything else, quirks included, is kept:
//   - "symmetric" files are expanded, each off-diagonal entry followed by its
//     mirror; "skew-symmetric" and integer "hermitian" files are read as
//     general (no mirror entries, no sign change);
//   - the writer emits "column row value" per entry (lmatrix_coo_cpu.cc:293),
//     so a file written and read back holds the transpose;
//   - a vector file whose last value is not followed by a line break loses
//     that value (the reference's counting loop stops one short).
#include <cctype>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "b200la.h"
#include "host_setup.h"

namespace {

constexpr int kLine = 1025;   // line buffer of the banner and size parsers

struct MMFile {
    int rows = 0, cols = 0, entries = 0;
    bool symmetric = false;
};

// Banner line and size line (lmp/mmio.cc:103-219).
int read_header(FILE *f, MMFile &h)
{
    char line[kLine], banner[kLine], mtx[kLine], crd[kLine], type[kLine], sym[kLine];
    if (!std::fgets(line, kLine, f)) return B200LA_ERR_FORMAT;
    if (std::sscanf(line, "%s %s %s %s %s", banner, mtx, crd, type, sym) != 5) return B200LA_ERR_FORMAT;
    for (char *w : {mtx, crd, type, sym})
        for (char *p = w; *p; ++p) *p = (char)std::tolower((unsigned char)*p);
    if (std::strncmp(banner, "%%MatrixMarket", 14) != 0) return B200LA_ERR_FORMAT;
    if (std::strcmp(mtx, "matrix") != 0) return B200LA_ERR_FORMAT;
    // only sparse real / integer coordinate files are read
    if (std::strcmp(crd, "coordinate") != 0) return B200LA_ERR_FORMAT;
    const bool real = std::strcmp(type, "real") == 0, integer = std::strcmp(type, "integer") == 0;
    if (!real && !integer) return B200LA_ERR_FORMAT;
    const bool general = std::strcmp(sym, "general") == 0, symmetric = std::strcmp(sym, "symmetric") == 0;
    const bool herm = std::strcmp(sym, "hermitian") == 0, skew = std::strcmp(sym, "skew-symmetric") == 0;
    if (!general && !symmetric && !herm && !skew) return B200LA_ERR_FORMAT;
    if (real && herm) return B200LA_ERR_FORMAT;   // not a valid MatrixMarket type
    h.symmetric = symmetric;
    // comment lines, then "rows cols entries" (possibly after blank lines)
    do {
        if (!std::fgets(line, kLine, f)) return B200LA_ERR_FORMAT;
    } while (line[0] == '%');
    if (std::sscanf(line, "%d %d %d", &h.rows, &h.cols, &h.entries) != 3) {
        int got;
        do {
            got = std::fscanf(f, "%d %d %d", &h.rows, &h.cols, &h.entries);
            if (got == EOF) return B200LA_ERR_FORMAT;
        } while (got != 3);
    }
    if (h.rows < 0 || h.cols < 0 || h.entries < 0) return B200LA_ERR_FORMAT;
    return B200LA_OK;
}

// The file's entries as COO (0-based), symmetric files expanded in file order.
int read_coo(const char *path, MMFile &h, std::vector<int> &r, std::vector<int> &c, std::vector<double> &v)
{
    FILE *f = std::fopen(path, "r");
    if (!f) return B200LA_ERR_IO;
    int rc = read_header(f, h);
    if (!rc) {
        r.reserve(h.entries);
        c.reserve(h.entries);
        v.reserve(h.entries);
        for (int k = 0; k < h.entries; ++k) {
            int i, j;
            double x;   // integer files are read as doubles too
            if (std::fscanf(f, " %d %d %lf \n", &i, &j, &x) != 3) {
                rc = B200LA_ERR_FORMAT;
                break;
            }
            if (i < 1 || i > h.rows || j < 1 || j > h.cols) {
                rc = B200LA_ERR_CSR;
                break;
            }
            r.push_back(i - 1);
            c.push_back(j - 1);
            v.push_back(x);
            if (h.symmetric && i != j) {
                if (j > h.rows || i > h.cols) {
                    rc = B200LA_ERR_CSR;
                    break;
                }
                r.push_back(j - 1);
                c.push_back(i - 1);
                v.push_back(x);
            }
        }
    }
    std::fclose(f);
    return rc;
}

// CPU_lVector::ReadFile's two passes: count the values the stream delivers
// while it stays good (one more than there are, or exactly as many when
// the last value ends the file), then read that many.
int read_vec(const char *path, std::vector<double> *out, int *n_out)
{
    std::ifstream in(path, std::ifstream::in);
    if (!in.is_open()) return B200LA_ERR_IO;
    int count = 0;
    double v;
    while (in.good()) {
        in >> v;
        ++count;
    }
    in.close();
    const int n = count - 1;
    if (n_out) *n_out = n;
    if (!out) return B200LA_OK;
    out->assign(n > 0 ? n : 0, 0.0);
    std::ifstream in2(path);
    if (!in2.is_open()) return B200LA_ERR_IO;
    for (int i = 0; i < n && in2.good(); ++i) {
        in2 >> v;
        (*out)[i] = v;
    }
    return B200LA_OK;
}

}  // namespace

extern "C" int b200la_mm_read_info(const char *path, int *n_rows, int *n_cols, int *nnz)
{
    if (!path || !n_rows || !n_cols || !nnz) return B200LA_ERR_ARG;
    MMFile h;
    std::vector<int> r, c;
    std::vector<double> v;
    const int rc = read_coo(path, h, r, c, v);
    if (rc) return rc;
    *n_rows = h.rows;
    *n_cols = h.cols;
    *nnz = (int)r.size();
    return B200LA_OK;
}

extern "C" int b200la_mm_read_csr(const char *path, int n_rows, int nnz, int *row, int *col, double *val)
{
    if (!path || !row || n_rows < 0 || nnz < 0 || (nnz && (!col || !val))) return B200LA_ERR_ARG;
    MMFile h;
    std::vector<int> r, c;
    std::vector<double> v;
    const int rc = read_coo(path, h, r, c, v);
    if (rc) return rc;
    if (h.rows != n_rows || (int)r.size() != nnz) return B200LA_ERR_ARG;
    b200::host::coo_to_csr(n_rows, nnz, r.data(), c.data(), v.data(), row, col, val);
    return B200LA_OK;
}

extern "C" int b200la_mm_write_csr(const char *path, int n_rows, int n_cols, int nnz, const int *row, const int *col,
                                   const double *val)
{
    if (!path || !row || n_rows < 0 || n_cols < 0 || nnz < 0 || (nnz && (!col || !val))) return B200LA_ERR_ARG;
    if (row[0] != 0 || row[n_rows] != nnz) return B200LA_ERR_CSR;
    for (int i = 0; i < n_rows; ++i)
        if (row[i + 1] < row[i]) return B200LA_ERR_CSR;
    FILE *f = std::fopen(path, "w");
    if (!f) return B200LA_ERR_IO;
    bool ok = std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n") > 0 &&
              std::fprintf(f, "%d %d %d\n", n_rows, n_cols, nnz) > 0;
    for (int i = 0; ok && i < n_rows; ++i)
        for (int j = row[i]; ok && j < row[i + 1]; ++j)
            ok = std::fprintf(f, "%d %d %24.14e\n", col[j] + 1, i + 1, val[j]) > 0;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? B200LA_OK : B200LA_ERR_IO;
}

extern "C" int b200la_vec_read_info(const char *path, int *n)
{
    if (!path || !n) return B200LA_ERR_ARG;
    return read_vec(path, nullptr, n);
}

extern "C" int b200la_vec_read(const char *path, int n, double *x)
{
    if (!path || n < 0 || (n && !x)) return B200LA_ERR_ARG;
    std::vector<double> v;
    int m = 0;
    const int rc = read_vec(path, &v, &m);
    if (rc) return rc;
    if (m != n) return B200LA_ERR_ARG;
    for (int i = 0; i < n; ++i) x[i] = v[i];
    return B200LA_OK;
}

extern "C" int b200la_vec_write(const char *path, int n, const double *x)
{
    if (!path || n < 0 || (n && !x)) return B200LA_ERR_ARG;
    std::ofstream out(path, std::ifstream::out);
    if (!out.is_open()) return B200LA_ERR_IO;
    for (int i = 0; i < n; ++i) out << std::scientific << x[i] << std::endl;
    out.close();
    return out.fail() ? B200LA_ERR_IO : B200LA_OK;
}
