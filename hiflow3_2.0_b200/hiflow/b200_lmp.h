// b200_lmp.h -- the B200 platform as HiFlow3 lmp classes.
//
// B200_lVector<T> and B200_CSR_lMatrix<T> derive from HiFlow3's own
// hiflow::la::lVector<T> (src/linear_algebra/lmp/lvector.h:39-335) and
// CSR_lMatrix<T> (lmatrix_csr.h, over lmatrix.h:39-448), T = double or float,
// and forward every operation to the C ABI of libb200la (include/b200la.h).
// They are what a HiFlow3 build adds for the new platform: with the enum
// value and the two factory cases (la_global.h:40-48, init_vec_mat.cc:47-417)
// every lmp caller -- the CG / GMRES functors, the lPreconditioner classes,
// CoupledMatrix / CoupledVector -- runs on them unchanged.
//
// The data lives in device memory.  Operations that the reference's GPU
// classes perform on the host (the multicoloured preconditioner clones the
// operator to a CPUsimple matrix, lpreconditioner_mc.cc:309-356) reach these
// classes through CopyTo / CopyStructureTo, which fill CPU objects directly,
// as the CPU classes expect of a non-CPU peer (lmatrix_csr_cpu.cc:239-270,
// 406-443; lvector_cpu.cc:310-345).
//
// Errors: where the reference logs and calls exit(-1), these classes throw
// hiflow::la::B200Error with the library's message; a caller that does not
// catch it ends the process, as before.
//
// Until la_global.h gains its B200 value, get_platform() reports GPU and
// get_implementation_name() "B200".
#ifndef HIFLOW_B200_LMP_H
#define HIFLOW_B200_LMP_H

#include "lmatrix_csr.h"
#include "lvector.h"

#include "b200la.h"

#include <stdexcept>
#include <string>
#include <vector>

namespace hiflow {
namespace la {

class B200Error : public std::runtime_error {
  public:
    explicit B200Error(const std::string &what) : std::runtime_error(what) {}
};

// The process-wide library context of the B200 platform (one per device,
// created on first use on device b200_lmp_device(); init_platform_gpu's role,
// cuda/platform_management_gpu.cu:78-171).
void b200_lmp_select_device(int device);
int b200_lmp_device();
b200la_ctx *b200_lmp_context();
void b200_lmp_check(int rc, const char *what);

template <typename T>
class B200_lVector : public lVector<T> {
  public:
    B200_lVector();
    B200_lVector(int size, std::string name);
    virtual ~B200_lVector();

    // device buffer of get_size() values (null when empty)
    T *device() const { return d_; }

    virtual void Init(const int size, const std::string name);
    virtual void Clear(void);
    virtual void Zeros(void);
    virtual void Reorder(const int *index);

    virtual lVector<T> &operator=(const lVector<T> &vec2);
    virtual void CopyFrom(const lVector<T> &vec);
    virtual void CopyTo(lVector<T> &vec) const;
    virtual void CastFrom(const lVector<double> &vec);
    virtual void CastFrom(const lVector<float> &vec);
    virtual void CastTo(lVector<double> &vec) const;
    virtual void CastTo(lVector<float> &vec) const;
    virtual lVector<T> *CloneWithoutContent(void) const;
    virtual void Sync(void) const;

    virtual void add_value(const int i, T val);
    virtual void add_values(const int *indices, int length, const T *values);
    virtual void SetValues(const int *index, const int size, const T *values);
    virtual void GetValues(const int *index, const int size, T *values) const;
    virtual void SetBlockValues(const int start_i, const int end_i, const T *values);
    virtual void GetBlockValues(const int start_i, const int end_i, T *values) const;
    virtual void set_indexset(const int *indexset, const int size);
    virtual void get_indexset(int *indexset) const;
    virtual int get_indexset_size(void) const;
    virtual void GetIndexedValues(T *values) const;
    virtual void SetIndexedValues(const T *values);
    virtual lVector<T> *extract_subvector(const int start_i, const int end_i) const;
    virtual void partial_replace_subvector(const int start_i, const int start_sub_vec, const int size,
                                           const lVector<T> &sub_vec);
    virtual void partial_add_subvector(const int start_i, const int start_sub_vec, const int size, const T weight,
                                       const lVector<T> &sub_vec);
    virtual void ReadFile(const char *filename);
    virtual void WriteFile(const char *filename);

    virtual void ElementWiseMult(const lVector<T> &vec) const;
    virtual int ArgMin(void) const;
    virtual int ArgMax(void) const;
    virtual T Norm1(void) const;
    virtual T Norm2(void) const;
    virtual T NormMax(void) const;
    virtual T Dot(const lVector<T> &vec) const;
    virtual void Scale(const T scalar);
    virtual void Axpy(const lVector<T> &vec, const T scalar);
    virtual void ScaleAdd(const T scalar, const lVector<T> &vec);
    virtual void Rot(lVector<T> *vec, const T &sc, const T &ss);
    virtual void Rotg(T *sa, T *sb, T *sc, T *ss) const;
    virtual void Rotm(lVector<T> *vec, const T &sparam);
    virtual void Rotmg(T *sd1, T *sd2, T *x1, const T &x2, T *sparam) const;

  private:
    T *d_ = nullptr;
    std::vector<int> idx_;       // index set (host copy)
    int *idx_dev_ = nullptr;     // index set (device copy)
};

template <typename T>
class B200_CSR_lMatrix : public CSR_lMatrix<T> {
  public:
    B200_CSR_lMatrix();
    B200_CSR_lMatrix(int nnz, int num_row, int num_col, std::string name);
    virtual ~B200_CSR_lMatrix();

    // the library's matrix (null until values have been given)
    b200la_csr *handle() const;

    virtual void Init(const int init_nnz, const int init_num_row, const int init_num_col, const std::string init_name);
    virtual void Clear(void);
    virtual void Zeros(void);

    virtual lMatrix<T> &operator=(const lMatrix<T> &mat2);
    virtual void CopyFrom(const lMatrix<T> &mat2);
    virtual void CopyTo(lMatrix<T> &mat2) const;
    virtual void CastFrom(const lMatrix<double> &other);
    virtual void CastFrom(const lMatrix<float> &other);
    virtual void CastTo(lMatrix<double> &other) const;
    virtual void CastTo(lMatrix<float> &other) const;
    virtual void ConvertFrom(const lMatrix<T> &mat2);
    virtual void CopyStructureFrom(const lMatrix<T> &mat2);
    virtual void CopyStructureTo(lMatrix<T> &mat2) const;
    virtual lMatrix<T> *CloneWithoutContent(void) const;
    virtual void Sync(void) const;
    virtual void ReadFile(const char *filename);
    virtual void WriteFile(const char *filename) const;

    virtual void VectorMult(const lVector<T> &invec, lVector<T> *outvec) const;
    virtual void VectorMultAdd(const lVector<T> &invec, lVector<T> *outvec) const;
    virtual void VectorMultNoDiag(const lVector<T> &in, lVector<T> *out) const;
    virtual void SwapDiagElementsToRowFront(void);

    virtual void Compress(void);
    virtual void Scale(const T alpha);
    virtual void ScaleOffdiag(const T alpha);
    virtual void extract_diagelements(const int start_i, const int end_i, lVector<T> *vec) const;
    virtual void extract_invdiagelements(const int start_i, const int end_i, lVector<T> *vec) const;
    virtual lMatrix<T> *extract_submatrix(const int start_row, const int start_col, const int end_row,
                                          const int end_col) const;
    virtual void Reorder(const int *index);
    virtual void Multicoloring(int &ncolors, int **color_sizes, int **permut_index) const;
    virtual void Levelscheduling(int &nlevels, int **level_sizes, int **permut_index) const;
    virtual void ilu0(void);

    virtual void init_structure(const int *rows, const int *cols);
    virtual void add_value(const int row, const int col, const T val);
    virtual void add_values(const int *rows, int num_rows, const int *cols, int num_cols, const T *values);
    virtual void ZeroRows(const int *index_set, const int size, const T alpha);

  private:
    void set_sizes(int nnz, int nrow, int ncol, const std::string &name);
    void upload(const T *val);          // (re)create the device matrix from the host structure and val
    void download_values(std::vector<T> &val) const;
    void ensure() const;                // device matrix current (values staged on the host are uploaded)
    void stage() const;                 // values staged on the host for assembly
    void adopt(b200la_csr *A);          // take over a library matrix, structure mirrored on the host

    // structure mirror on the host (CSR row pointers and column indices)
    std::vector<int> row_, col_;
    // values staged on the host, in FP64, during assembly (init_structure / add_values / ZeroRows)
    mutable std::vector<double> stage_;
    mutable bool staged_ = false;
    mutable b200la_csr *A_ = nullptr;
};

}  // namespace la
}  // namespace hiflow

#endif
