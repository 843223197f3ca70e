// b200_lmp.cc -- B200_lVector<T> / B200_CSR_lMatrix<T>: HiFlow3 lmp classes
// over the C ABI of libb200la (declarations and conventions: b200_lmp.h).
#include "b200_lmp.h"

#include "lmatrix_csr_cpu.h"
#include "lvector_cpu.h"

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>

namespace hiflow {
namespace la {

// ------------------------------------------------------------------ context

namespace {
std::mutex g_ctx_mutex;
std::map<int, b200la_ctx *> g_ctx;
int g_device = 0;

template <typename T>
constexpr int dtype_of()
{
    return sizeof(T) == 8 ? B200LA_F64 : B200LA_F32;
}

template <typename T>
const B200_lVector<T> &b200(const lVector<T> &v, const char *what)
{
    const B200_lVector<T> *p = dynamic_cast<const B200_lVector<T> *>(&v);
    if (!p) throw B200Error(std::string(what) + ": the vector is not a B200_lVector");
    return *p;
}

template <typename T>
B200_lVector<T> &b200(lVector<T> &v, const char *what)
{
    B200_lVector<T> *p = dynamic_cast<B200_lVector<T> *>(&v);
    if (!p) throw B200Error(std::string(what) + ": the vector is not a B200_lVector");
    return *p;
}
}  // namespace

void b200_lmp_select_device(int device)
{
    std::lock_guard<std::mutex> lock(g_ctx_mutex);
    g_device = device;
}

int b200_lmp_device()
{
    std::lock_guard<std::mutex> lock(g_ctx_mutex);
    return g_device;
}

b200la_ctx *b200_lmp_context()
{
    std::lock_guard<std::mutex> lock(g_ctx_mutex);
    b200la_ctx *&c = g_ctx[g_device];
    if (!c) {
        const int rc = b200la_create(g_device, &c);
        if (rc != B200LA_OK) {
            c = nullptr;
            throw B200Error("b200la_create failed (" + std::to_string(rc) + ")");
        }
    }
    return c;
}

void b200_lmp_check(int rc, const char *what)
{
    if (rc == B200LA_OK) return;
    const char *msg = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_ctx_mutex);
        auto it = g_ctx.find(g_device);
        if (it != g_ctx.end() && it->second) msg = b200la_last_error(it->second);
    }
    throw B200Error(std::string(what) + ": " + std::to_string(rc) + (msg ? std::string(" ") + msg : ""));
}

#define CHECK(call, what) b200_lmp_check((call), what)

// ------------------------------------------------------------------- vector

template <typename T>
B200_lVector<T>::B200_lVector()
{
    this->platform_name_ = "B200";
    this->platform_id_ = GPU;
    this->implementation_name_ = "B200";
    this->implementation_id_ = SCALAR;
    this->size_ = 0;
    this->name_ = "";
}

template <typename T>
B200_lVector<T>::B200_lVector(int size, std::string name) : B200_lVector()
{
    Init(size, name);
}

template <typename T>
B200_lVector<T>::~B200_lVector()
{
    try {
        Clear();
    } catch (...) {
    }
}

template <typename T>
void B200_lVector<T>::Init(const int size, const std::string name)
{
    Clear();
    if (size < 0) throw B200Error("B200_lVector::Init: negative size");
    if (size > 0) {
        void *p = nullptr;
        CHECK(b200la_malloc(b200_lmp_context(), sizeof(T) * (size_t)size, &p), "B200_lVector::Init");
        d_ = static_cast<T *>(p);
    }
    this->size_ = size;
    this->name_ = name;
    Zeros();
}

template <typename T>
void B200_lVector<T>::Clear(void)
{
    if (d_) b200la_free(b200_lmp_context(), d_);
    if (idx_dev_) b200la_free(b200_lmp_context(), idx_dev_);
    d_ = nullptr;
    idx_dev_ = nullptr;
    idx_.clear();
    this->size_ = 0;
    this->name_ = "";
}

template <typename T>
void B200_lVector<T>::Zeros(void)
{
    if (this->size_ > 0)
        CHECK(b200la_memset_zero(b200_lmp_context(), d_, sizeof(T) * this->size_), "B200_lVector::Zeros");
}

// out[i] = in[index[i]] (lvector_cpu.cc:75-94), through a device copy of the index
template <typename T>
void B200_lVector<T>::Reorder(const int *index)
{
    const int n = this->size_;
    if (n == 0) return;
    b200la_ctx *c = b200_lmp_context();
    void *perm = nullptr, *tmp = nullptr;
    CHECK(b200la_malloc(c, sizeof(int) * n, &perm), "B200_lVector::Reorder");
    int rc = b200la_malloc(c, sizeof(T) * n, &tmp);
    if (!rc) rc = b200la_memcpy_h2d(c, perm, index, sizeof(int) * n);
    if (!rc) rc = b200la_permute(c, dtype_of<T>(), n, static_cast<int *>(perm), d_, tmp);
    if (!rc) rc = b200la_memcpy_d2d(c, d_, tmp, sizeof(T) * n);
    if (!rc) rc = b200la_sync(c);
    if (tmp) b200la_free(c, tmp);
    b200la_free(c, perm);
    CHECK(rc, "B200_lVector::Reorder");
}

template <typename T>
lVector<T> &B200_lVector<T>::operator=(const lVector<T> &vec2)
{
    if (this != &vec2) CopyFrom(vec2);
    return *this;
}

template <typename T>
void B200_lVector<T>::CopyFrom(const lVector<T> &vec)
{
    if (this == &vec) return;
    if (vec.get_size() != this->size_) throw B200Error("B200_lVector::CopyFrom: sizes differ");
    b200la_ctx *c = b200_lmp_context();
    if (const B200_lVector<T> *o = dynamic_cast<const B200_lVector<T> *>(&vec)) {
        if (this->size_) CHECK(b200la_memcpy_d2d(c, d_, o->d_, sizeof(T) * this->size_), "B200_lVector::CopyFrom");
    } else if (const CPU_lVector<T> *h = dynamic_cast<const CPU_lVector<T> *>(&vec)) {
        if (this->size_) {
            CHECK(b200la_memcpy_h2d(c, d_, h->buffer, sizeof(T) * this->size_), "B200_lVector::CopyFrom");
            CHECK(b200la_sync(c), "B200_lVector::CopyFrom");
        }
    } else {
        vec.CopyTo(*this);
    }
}

template <typename T>
void B200_lVector<T>::CopyTo(lVector<T> &vec) const
{
    if (CPU_lVector<T> *h = dynamic_cast<CPU_lVector<T> *>(&vec)) {
        if (vec.get_size() != this->size_) throw B200Error("B200_lVector::CopyTo: sizes differ");
        b200la_ctx *c = b200_lmp_context();
        if (this->size_) {
            CHECK(b200la_memcpy_d2h(c, h->buffer, d_, sizeof(T) * this->size_), "B200_lVector::CopyTo");
            CHECK(b200la_sync(c), "B200_lVector::CopyTo");
        }
    } else {
        vec.CopyFrom(*this);
    }
}

namespace {
// this (type T) from a vector of type S: device cast, host buffer converted, or the source's CastTo
template <typename T, typename S>
void cast_from(B200_lVector<T> &self, const lVector<S> &other)
{
    if (other.get_size() != self.get_size()) throw B200Error("B200_lVector::CastFrom: sizes differ");
    const int n = self.get_size();
    b200la_ctx *c = b200_lmp_context();
    if (const B200_lVector<S> *o = dynamic_cast<const B200_lVector<S> *>(&other)) {
        if (n) CHECK(b200la_cast(c, dtype_of<S>(), o->device(), dtype_of<T>(), self.device(), n), "CastFrom");
    } else if (const CPU_lVector<S> *h = dynamic_cast<const CPU_lVector<S> *>(&other)) {
        std::vector<T> tmp(n);
        for (int i = 0; i < n; ++i) tmp[i] = (T)h->buffer[i];
        if (n) {
            CHECK(b200la_memcpy_h2d(c, self.device(), tmp.data(), sizeof(T) * n), "CastFrom");
            CHECK(b200la_sync(c), "CastFrom");
        }
    } else {
        other.CastTo(self);
    }
}

// a vector of type S from this (type T)
template <typename T, typename S>
void cast_to(const B200_lVector<T> &self, lVector<S> &other)
{
    if (other.get_size() != self.get_size()) throw B200Error("B200_lVector::CastTo: sizes differ");
    const int n = self.get_size();
    if (CPU_lVector<S> *h = dynamic_cast<CPU_lVector<S> *>(&other)) {
        b200la_ctx *c = b200_lmp_context();
        std::vector<T> tmp(n);
        if (n) {
            CHECK(b200la_memcpy_d2h(c, tmp.data(), self.device(), sizeof(T) * n), "CastTo");
            CHECK(b200la_sync(c), "CastTo");
        }
        for (int i = 0; i < n; ++i) h->buffer[i] = (S)tmp[i];
    } else {
        other.CastFrom(self);
    }
}
}  // namespace

template <typename T>
void B200_lVector<T>::CastFrom(const lVector<double> &vec)
{
    cast_from<T, double>(*this, vec);
}
template <typename T>
void B200_lVector<T>::CastFrom(const lVector<float> &vec)
{
    cast_from<T, float>(*this, vec);
}
template <typename T>
void B200_lVector<T>::CastTo(lVector<double> &vec) const
{
    cast_to<T, double>(*this, vec);
}
template <typename T>
void B200_lVector<T>::CastTo(lVector<float> &vec) const
{
    cast_to<T, float>(*this, vec);
}

// a zeroed vector of the same size on this platform (lvector.cc:52-64 through the factory)
template <typename T>
lVector<T> *B200_lVector<T>::CloneWithoutContent(void) const
{
    return new B200_lVector<T>(this->size_, "clone from " + this->name_);
}

template <typename T>
void B200_lVector<T>::Sync(void) const
{
    CHECK(b200la_sync(b200_lmp_context()), "B200_lVector::Sync");
}

template <typename T>
void B200_lVector<T>::add_value(const int i, T val)
{
    add_values(&i, 1, &val);
}

template <typename T>
void B200_lVector<T>::add_values(const int *indices, int length, const T *values)
{
    if (length <= 0) return;
    b200la_ctx *c = b200_lmp_context();
    CHECK(b200la_vec_add_values(c, dtype_of<T>(), this->size_, d_, length, indices, values), "add_values");
    CHECK(b200la_sync(c), "add_values");
}

template <typename T>
void B200_lVector<T>::SetValues(const int *index, const int size, const T *values)
{
    if (size <= 0) return;
    b200la_ctx *c = b200_lmp_context();
    CHECK(b200la_vec_set_values(c, dtype_of<T>(), this->size_, d_, size, index, values), "SetValues");
    CHECK(b200la_sync(c), "SetValues");
}

template <typename T>
void B200_lVector<T>::GetValues(const int *index, const int size, T *values) const
{
    if (size <= 0) return;
    for (int k = 0; k < size; ++k)
        if (index[k] < 0 || index[k] >= this->size_) throw B200Error("GetValues: index out of range");
    b200la_ctx *c = b200_lmp_context();
    void *idx = nullptr, *out = nullptr;
    CHECK(b200la_malloc(c, sizeof(int) * size, &idx), "GetValues");
    int rc = b200la_malloc(c, sizeof(T) * size, &out);
    if (!rc) rc = b200la_memcpy_h2d(c, idx, index, sizeof(int) * size);
    if (!rc) rc = b200la_gather(c, dtype_of<T>(), size, static_cast<int *>(idx), d_, out);
    if (!rc) rc = b200la_memcpy_d2h(c, values, out, sizeof(T) * size);
    if (!rc) rc = b200la_sync(c);
    if (out) b200la_free(c, out);
    b200la_free(c, idx);
    CHECK(rc, "GetValues");
}

template <typename T>
void B200_lVector<T>::SetBlockValues(const int start_i, const int end_i, const T *values)
{
    if (start_i < 0 || end_i > this->size_ || end_i < start_i) throw B200Error("SetBlockValues: range");
    if (end_i == start_i) return;
    b200la_ctx *c = b200_lmp_context();
    CHECK(b200la_memcpy_h2d(c, d_ + start_i, values, sizeof(T) * (end_i - start_i)), "SetBlockValues");
    CHECK(b200la_sync(c), "SetBlockValues");
}

template <typename T>
void B200_lVector<T>::GetBlockValues(const int start_i, const int end_i, T *values) const
{
    if (start_i < 0 || end_i > this->size_ || end_i < start_i) throw B200Error("GetBlockValues: range");
    if (end_i == start_i) return;
    b200la_ctx *c = b200_lmp_context();
    CHECK(b200la_memcpy_d2h(c, values, d_ + start_i, sizeof(T) * (end_i - start_i)), "GetBlockValues");
    CHECK(b200la_sync(c), "GetBlockValues");
}

template <typename T>
void B200_lVector<T>::set_indexset(const int *indexset, const int size)
{
    for (int k = 0; k < size; ++k)
        if (indexset[k] < 0 || indexset[k] >= this->size_) throw B200Error("set_indexset: index out of range");
    b200la_ctx *c = b200_lmp_context();
    if (idx_dev_) b200la_free(c, idx_dev_);
    idx_dev_ = nullptr;
    idx_.assign(indexset, indexset + size);
    if (size > 0) {
        void *p = nullptr;
        CHECK(b200la_malloc(c, sizeof(int) * size, &p), "set_indexset");
        idx_dev_ = static_cast<int *>(p);
        CHECK(b200la_memcpy_h2d(c, idx_dev_, idx_.data(), sizeof(int) * size), "set_indexset");
        CHECK(b200la_sync(c), "set_indexset");
    }
}

template <typename T>
void B200_lVector<T>::get_indexset(int *indexset) const
{
    std::copy(idx_.begin(), idx_.end(), indexset);
}

template <typename T>
int B200_lVector<T>::get_indexset_size(void) const
{
    return (int)idx_.size();
}

template <typename T>
void B200_lVector<T>::GetIndexedValues(T *values) const
{
    const int m = (int)idx_.size();
    if (m == 0) return;
    b200la_ctx *c = b200_lmp_context();
    void *out = nullptr;
    CHECK(b200la_malloc(c, sizeof(T) * m, &out), "GetIndexedValues");
    int rc = b200la_gather(c, dtype_of<T>(), m, idx_dev_, d_, out);
    if (!rc) rc = b200la_memcpy_d2h(c, values, out, sizeof(T) * m);
    if (!rc) rc = b200la_sync(c);
    b200la_free(c, out);
    CHECK(rc, "GetIndexedValues");
}

template <typename T>
void B200_lVector<T>::SetIndexedValues(const T *values)
{
    const int m = (int)idx_.size();
    if (m == 0) return;
    b200la_ctx *c = b200_lmp_context();
    void *in = nullptr;
    CHECK(b200la_malloc(c, sizeof(T) * m, &in), "SetIndexedValues");
    int rc = b200la_memcpy_h2d(c, in, values, sizeof(T) * m);
    if (!rc) rc = b200la_scatter(c, dtype_of<T>(), m, idx_dev_, in, d_);
    if (!rc) rc = b200la_sync(c);
    b200la_free(c, in);
    CHECK(rc, "SetIndexedValues");
}

template <typename T>
lVector<T> *B200_lVector<T>::extract_subvector(const int start_i, const int end_i) const
{
    if (start_i < 0 || end_i > this->size_ || end_i < start_i) throw B200Error("extract_subvector: range");
    B200_lVector<T> *s = new B200_lVector<T>(end_i - start_i, "sub vecrix from " + this->name_);
    if (end_i > start_i)
        CHECK(b200la_memcpy_d2d(b200_lmp_context(), s->d_, d_ + start_i, sizeof(T) * (end_i - start_i)),
              "extract_subvector");
    return s;
}

template <typename T>
void B200_lVector<T>::partial_replace_subvector(const int start_i, const int start_sub_vec, const int size,
                                                const lVector<T> &sub_vec)
{
    const B200_lVector<T> &s = b200(sub_vec, "partial_replace_subvector");
    if (start_i < 0 || start_i + size > this->size_ || start_sub_vec < 0 || start_sub_vec + size > s.size_)
        throw B200Error("partial_replace_subvector: range");
    if (size > 0)
        CHECK(b200la_memcpy_d2d(b200_lmp_context(), d_ + start_i, s.d_ + start_sub_vec, sizeof(T) * size),
              "partial_replace_subvector");
}

template <typename T>
void B200_lVector<T>::partial_add_subvector(const int start_i, const int start_sub_vec, const int size,
                                            const T weight, const lVector<T> &sub_vec)
{
    const B200_lVector<T> &s = b200(sub_vec, "partial_add_subvector");
    if (start_i < 0 || start_i + size > this->size_ || start_sub_vec < 0 || start_sub_vec + size > s.size_)
        throw B200Error("partial_add_subvector: range");
    if (size > 0)
        CHECK(b200la_axpy(b200_lmp_context(), dtype_of<T>(), size, (double)weight, s.d_ + start_sub_vec,
                          d_ + start_i),
              "partial_add_subvector");
}

// the reference's vector file format (lvector_cpu.cc:582-663)
template <typename T>
void B200_lVector<T>::ReadFile(const char *filename)
{
    int n = 0;
    CHECK(b200la_vec_read_info(filename, &n), "B200_lVector::ReadFile");
    std::vector<double> v(n);
    CHECK(b200la_vec_read(filename, n, v.data()), "B200_lVector::ReadFile");
    Init(n, filename);
    std::vector<T> t(v.begin(), v.end());
    if (n) SetBlockValues(0, n, t.data());
}

template <typename T>
void B200_lVector<T>::WriteFile(const char *filename)
{
    std::vector<T> t(this->size_);
    if (this->size_) GetBlockValues(0, this->size_, t.data());
    std::vector<double> v(t.begin(), t.end());
    CHECK(b200la_vec_write(filename, this->size_, v.data()), "B200_lVector::WriteFile");
}

template <typename T>
void B200_lVector<T>::ElementWiseMult(const lVector<T> &vec) const
{
    const B200_lVector<T> &o = b200(vec, "ElementWiseMult");
    if (o.size_ != this->size_) throw B200Error("ElementWiseMult: sizes differ");
    if (this->size_)
        CHECK(b200la_ewmul(b200_lmp_context(), dtype_of<T>(), this->size_, o.d_, d_), "ElementWiseMult");
}

template <typename T>
int B200_lVector<T>::ArgMin(void) const
{
    int k = 0;
    CHECK(b200la_iamin(b200_lmp_context(), dtype_of<T>(), this->size_, d_, &k), "ArgMin");
    return k;
}

template <typename T>
int B200_lVector<T>::ArgMax(void) const
{
    int k = 0;
    CHECK(b200la_iamax(b200_lmp_context(), dtype_of<T>(), this->size_, d_, &k), "ArgMax");
    return k;
}

template <typename T>
T B200_lVector<T>::Norm1(void) const
{
    double r = 0.0;
    CHECK(b200la_asum(b200_lmp_context(), dtype_of<T>(), this->size_, d_, &r), "Norm1");
    return (T)r;
}

template <typename T>
T B200_lVector<T>::Norm2(void) const
{
    double r = 0.0;
    CHECK(b200la_nrm2(b200_lmp_context(), dtype_of<T>(), this->size_, d_, &r), "Norm2");
    return (T)r;
}

template <typename T>
T B200_lVector<T>::NormMax(void) const
{
    double r = 0.0;
    CHECK(b200la_normmax(b200_lmp_context(), dtype_of<T>(), this->size_, d_, &r), "NormMax");
    return (T)r;
}

template <typename T>
T B200_lVector<T>::Dot(const lVector<T> &vec) const
{
    const B200_lVector<T> &o = b200(vec, "Dot");
    if (o.size_ != this->size_) throw B200Error("Dot: sizes differ");
    double r = 0.0;
    CHECK(b200la_dot(b200_lmp_context(), dtype_of<T>(), this->size_, d_, o.d_, &r), "Dot");
    return (T)r;
}

template <typename T>
void B200_lVector<T>::Scale(const T scalar)
{
    if (this->size_) CHECK(b200la_scale(b200_lmp_context(), dtype_of<T>(), this->size_, (double)scalar, d_), "Scale");
}

template <typename T>
void B200_lVector<T>::Axpy(const lVector<T> &vec, const T scalar)
{
    const B200_lVector<T> &o = b200(vec, "Axpy");
    if (o.size_ != this->size_) throw B200Error("Axpy: sizes differ");
    if (this->size_)
        CHECK(b200la_axpy(b200_lmp_context(), dtype_of<T>(), this->size_, (double)scalar, o.d_, d_), "Axpy");
}

template <typename T>
void B200_lVector<T>::ScaleAdd(const T scalar, const lVector<T> &vec)
{
    const B200_lVector<T> &o = b200(vec, "ScaleAdd");
    if (o.size_ != this->size_) throw B200Error("ScaleAdd: sizes differ");
    if (this->size_)
        CHECK(b200la_scaleadd(b200_lmp_context(), dtype_of<T>(), this->size_, (double)scalar, o.d_, d_), "ScaleAdd");
}

template <typename T>
void B200_lVector<T>::Rot(lVector<T> *vec, const T &sc, const T &ss)
{
    B200_lVector<T> &o = b200(*vec, "Rot");
    if (o.size_ != this->size_) throw B200Error("Rot: sizes differ");
    if (this->size_)
        CHECK(b200la_rot(b200_lmp_context(), dtype_of<T>(), this->size_, d_, o.d_, (double)sc, (double)ss), "Rot");
}

template <typename T>
void B200_lVector<T>::Rotg(T *sa, T *sb, T *sc, T *ss) const
{
    CHECK(b200la_rotg(dtype_of<T>(), sa, sb, sc, ss), "Rotg");
}

// sparam is the first of five parameters (flag, h11, h21, h12, h22), as in
// the reference's CPUsimple_lVector::Rotm (CPUsimple_lvector.cc:540-600)
template <typename T>
void B200_lVector<T>::Rotm(lVector<T> *vec, const T &sparam)
{
    B200_lVector<T> &o = b200(*vec, "Rotm");
    if (o.size_ != this->size_) throw B200Error("Rotm: sizes differ");
    const T *p = &sparam;
    const double h[5] = {(double)p[0], (double)p[1], (double)p[2], (double)p[3], (double)p[4]};
    if (this->size_) CHECK(b200la_rotm(b200_lmp_context(), dtype_of<T>(), this->size_, d_, o.d_, h), "Rotm");
}

// not implemented by the reference's CPU and GPU vectors either (CPUsimple_lvector.cc:623-630)
template <typename T>
void B200_lVector<T>::Rotmg(T *, T *, T *, const T &, T *) const
{
    throw B200Error("B200_lVector::Rotmg is not implemented (nor in the reference's vectors)");
}

// ------------------------------------------------------------------- matrix

template <typename T>
B200_CSR_lMatrix<T>::B200_CSR_lMatrix()
{
    this->platform_name_ = "B200";
    this->platform_id_ = GPU;
    this->implementation_name_ = "B200";
    this->implementation_id_ = SCALAR;
    this->matrix_format_name_ = "CSR";
    this->matrix_format_id_ = CSR;
    this->symmetric_ = false;
    set_sizes(0, 0, 0, "");
}

template <typename T>
B200_CSR_lMatrix<T>::B200_CSR_lMatrix(int nnz, int num_row, int num_col, std::string name) : B200_CSR_lMatrix()
{
    Init(nnz, num_row, num_col, name);
}

template <typename T>
B200_CSR_lMatrix<T>::~B200_CSR_lMatrix()
{
    try {
        Clear();
    } catch (...) {
    }
}

template <typename T>
b200la_csr *B200_CSR_lMatrix<T>::handle() const
{
    ensure();
    return A_;
}

template <typename T>
void B200_CSR_lMatrix<T>::set_sizes(int nnz, int nrow, int ncol, const std::string &name)
{
    this->nnz_ = nnz;
    this->num_row_ = nrow;
    this->num_col_ = ncol;
    this->name_ = name;
}

// lMatrix::Init: the structure is given afterwards (CopyStructureFrom,
// init_structure, ReadFile); until then row pointers are zero
template <typename T>
void B200_CSR_lMatrix<T>::Init(const int init_nnz, const int init_num_row, const int init_num_col,
                               const std::string init_name)
{
    Clear();
    if (init_nnz < 0 || init_num_row < 0 || init_num_col < 0) throw B200Error("B200_CSR_lMatrix::Init: sizes");
    row_.assign(init_num_row + 1, 0);
    col_.assign(init_nnz, 0);
    set_sizes(init_nnz, init_num_row, init_num_col, init_name);
}

template <typename T>
void B200_CSR_lMatrix<T>::Clear(void)
{
    if (A_) b200la_csr_destroy(A_);
    A_ = nullptr;
    row_.clear();
    col_.clear();
    stage_.clear();
    staged_ = false;
    set_sizes(0, 0, 0, "");
}

template <typename T>
void B200_CSR_lMatrix<T>::upload(const T *val)
{
    b200la_ctx *c = b200_lmp_context();
    if (A_) b200la_csr_destroy(A_);
    A_ = nullptr;
    CHECK(b200la_csr_create(c, this->num_row_, this->num_col_, this->nnz_, row_.data(), col_.data(), val,
                            dtype_of<T>(), &A_),
          "B200_CSR_lMatrix: upload");
    staged_ = false;
    stage_.clear();
}

template <typename T>
void B200_CSR_lMatrix<T>::download_values(std::vector<T> &val) const
{
    val.resize(this->nnz_);
    if (staged_) {
        for (int j = 0; j < this->nnz_; ++j) val[j] = (T)stage_[j];
        return;
    }
    if (!A_) {
        std::fill(val.begin(), val.end(), T(0));
        return;
    }
    b200la_ctx *c = b200_lmp_context();
    CHECK(b200la_csr_download(c, A_, nullptr, nullptr, val.data()), "B200_CSR_lMatrix: download");
}

template <typename T>
void B200_CSR_lMatrix<T>::ensure() const
{
    if (staged_ || !A_) {
        std::vector<T> v(this->nnz_, T(0));
        if (staged_)
            for (int j = 0; j < this->nnz_; ++j) v[j] = (T)stage_[j];
        const_cast<B200_CSR_lMatrix<T> *>(this)->upload(v.data());
    }
}

template <typename T>
void B200_CSR_lMatrix<T>::adopt(b200la_csr *A)
{
    int n = 0, m = 0, nnz = 0;
    CHECK(b200la_csr_info(A, &n, &m, &nnz, nullptr, nullptr, nullptr, nullptr), "B200_CSR_lMatrix: info");
    const std::string name = this->name_;
    Clear();
    set_sizes(nnz, n, m, name);
    row_.resize(n + 1);
    col_.resize(nnz);
    CHECK(b200la_csr_download(b200_lmp_context(), A, row_.data(), col_.data(), nullptr), "B200_CSR_lMatrix: adopt");
    A_ = A;
}

template <typename T>
void B200_CSR_lMatrix<T>::Zeros(void)
{
    if (staged_) std::fill(stage_.begin(), stage_.end(), 0.0);
    else if (A_) CHECK(b200la_csr_scale(b200_lmp_context(), A_, 0.0, B200LA_SCALE_ZERO), "Zeros");
}

template <typename T>
lMatrix<T> &B200_CSR_lMatrix<T>::operator=(const lMatrix<T> &mat2)
{
    if (this != &mat2) CopyFrom(mat2);
    return *this;
}

// values of an equally structured matrix (lmatrix_csr_cpu.cc:239-270)
template <typename T>
void B200_CSR_lMatrix<T>::CopyFrom(const lMatrix<T> &mat2)
{
    if (this == &mat2) return;
    if (mat2.get_nnz() != this->nnz_ || mat2.get_num_row() != this->num_row_ || mat2.get_num_col() != this->num_col_)
        throw B200Error("B200_CSR_lMatrix::CopyFrom: sizes differ");
    if (const B200_CSR_lMatrix<T> *o = dynamic_cast<const B200_CSR_lMatrix<T> *>(&mat2)) {
        std::vector<T> v;
        o->download_values(v);
        upload(v.data());
    } else if (const CPU_CSR_lMatrix<T> *h = dynamic_cast<const CPU_CSR_lMatrix<T> *>(&mat2)) {
        upload(h->matrix.val);
    } else {
        mat2.CopyTo(*this);
    }
}

template <typename T>
void B200_CSR_lMatrix<T>::CopyTo(lMatrix<T> &mat2) const
{
    if (CPU_CSR_lMatrix<T> *h = dynamic_cast<CPU_CSR_lMatrix<T> *>(&mat2)) {
        if (mat2.get_nnz() != this->nnz_) throw B200Error("B200_CSR_lMatrix::CopyTo: sizes differ");
        std::vector<T> v;
        download_values(v);
        if (this->nnz_) std::memcpy(h->matrix.val, v.data(), sizeof(T) * this->nnz_);
    } else {
        mat2.CopyFrom(*this);
    }
}

template <typename T>
void B200_CSR_lMatrix<T>::CastFrom(const lMatrix<double> &other)
{
    if (const B200_CSR_lMatrix<double> *o = dynamic_cast<const B200_CSR_lMatrix<double> *>(&other)) {
        b200la_csr *B = nullptr;
        CHECK(b200la_csr_cast(b200_lmp_context(), o->handle(), dtype_of<T>(), &B), "CastFrom");
        this->name_ = other.get_name();
        adopt(B);
    } else if (const CPU_CSR_lMatrix<double> *h = dynamic_cast<const CPU_CSR_lMatrix<double> *>(&other)) {
        if (other.get_nnz() != this->nnz_) Init(other.get_nnz(), other.get_num_row(), other.get_num_col(), other.get_name());
        std::copy(h->matrix.row, h->matrix.row + other.get_num_row() + 1, row_.begin());
        std::copy(h->matrix.col, h->matrix.col + other.get_nnz(), col_.begin());
        std::vector<T> v(h->matrix.val, h->matrix.val + other.get_nnz());
        upload(v.data());
    } else {
        other.CastTo(*this);
    }
}

template <typename T>
void B200_CSR_lMatrix<T>::CastFrom(const lMatrix<float> &other)
{
    if (const B200_CSR_lMatrix<float> *o = dynamic_cast<const B200_CSR_lMatrix<float> *>(&other)) {
        b200la_csr *B = nullptr;
        CHECK(b200la_csr_cast(b200_lmp_context(), o->handle(), dtype_of<T>(), &B), "CastFrom");
        this->name_ = other.get_name();
        adopt(B);
    } else if (const CPU_CSR_lMatrix<float> *h = dynamic_cast<const CPU_CSR_lMatrix<float> *>(&other)) {
        if (other.get_nnz() != this->nnz_) Init(other.get_nnz(), other.get_num_row(), other.get_num_col(), other.get_name());
        std::copy(h->matrix.row, h->matrix.row + other.get_num_row() + 1, row_.begin());
        std::copy(h->matrix.col, h->matrix.col + other.get_nnz(), col_.begin());
        std::vector<T> v(h->matrix.val, h->matrix.val + other.get_nnz());
        upload(v.data());
    } else {
        other.CastTo(*this);
    }
}

namespace {
template <typename T, typename S>
void matrix_cast_to(const B200_CSR_lMatrix<T> &self, lMatrix<S> &other)
{
    if (CPU_CSR_lMatrix<S> *h = dynamic_cast<CPU_CSR_lMatrix<S> *>(&other)) {
        if (other.get_nnz() != self.get_nnz()) throw B200Error("B200_CSR_lMatrix::CastTo: sizes differ");
        std::vector<T> v(self.get_nnz());
        if (self.get_nnz())
            CHECK(b200la_csr_download(b200_lmp_context(), self.handle(), h->matrix.row, h->matrix.col, v.data()),
                  "CastTo");
        for (int j = 0; j < self.get_nnz(); ++j) h->matrix.val[j] = (S)v[j];
    } else {
        other.CastFrom(self);
    }
}
}  // namespace

template <typename T>
void B200_CSR_lMatrix<T>::CastTo(lMatrix<double> &other) const
{
    matrix_cast_to<T, double>(*this, other);
}

template <typename T>
void B200_CSR_lMatrix<T>::CastTo(lMatrix<float> &other) const
{
    matrix_cast_to<T, float>(*this, other);
}

template <typename T>
void B200_CSR_lMatrix<T>::ConvertFrom(const lMatrix<T> &mat2)
{
    if (mat2.get_matrix_format() != CSR)
        throw B200Error("B200_CSR_lMatrix::ConvertFrom: only CSR sources are supported");
    this->CloneFrom(mat2);
}

// lmatrix_csr_cpu.cc:406-438: Init with the source's sizes, then its row pointers and columns
template <typename T>
void B200_CSR_lMatrix<T>::CopyStructureFrom(const lMatrix<T> &mat2)
{
    if (this == &mat2) return;
    Init(mat2.get_nnz(), mat2.get_num_row(), mat2.get_num_col(), mat2.get_name());
    if (const B200_CSR_lMatrix<T> *o = dynamic_cast<const B200_CSR_lMatrix<T> *>(&mat2)) {
        row_ = o->row_;
        col_ = o->col_;
    } else if (const CPU_CSR_lMatrix<T> *h = dynamic_cast<const CPU_CSR_lMatrix<T> *>(&mat2)) {
        std::copy(h->matrix.row, h->matrix.row + this->num_row_ + 1, row_.begin());
        std::copy(h->matrix.col, h->matrix.col + this->nnz_, col_.begin());
    } else {
        mat2.CopyStructureTo(*this);
    }
}

template <typename T>
void B200_CSR_lMatrix<T>::CopyStructureTo(lMatrix<T> &mat2) const
{
    if (CPU_CSR_lMatrix<T> *h = dynamic_cast<CPU_CSR_lMatrix<T> *>(&mat2)) {
        // the CPU matrix has been Init'ed with this matrix's sizes by its CopyStructureFrom
        if (mat2.get_nnz() != this->nnz_ || mat2.get_num_row() != this->num_row_)
            throw B200Error("B200_CSR_lMatrix::CopyStructureTo: sizes differ");
        std::copy(row_.begin(), row_.end(), h->matrix.row);
        std::copy(col_.begin(), col_.end(), h->matrix.col);
    } else {
        mat2.CopyStructureFrom(*this);
    }
}

// same structure, zero values, on this platform (lmatrix.cc:64-79 through the factory)
template <typename T>
lMatrix<T> *B200_CSR_lMatrix<T>::CloneWithoutContent(void) const
{
    B200_CSR_lMatrix<T> *m = new B200_CSR_lMatrix<T>();
    m->CopyStructureFrom(*this);
    m->name_ = "clone from " + this->name_;
    return m;
}

template <typename T>
void B200_CSR_lMatrix<T>::Sync(void) const
{
    CHECK(b200la_sync(b200_lmp_context()), "B200_CSR_lMatrix::Sync");
}

// MatrixMarket (CPU_CSR_lMatrix::ReadFile / WriteFile, lmatrix_csr_cpu.cc:1733-1765)
template <typename T>
void B200_CSR_lMatrix<T>::ReadFile(const char *filename)
{
    int n = 0, m = 0, nnz = 0;
    CHECK(b200la_mm_read_info(filename, &n, &m, &nnz), "B200_CSR_lMatrix::ReadFile");
    Init(nnz, n, m, filename);
    std::vector<double> v(nnz);
    CHECK(b200la_mm_read_csr(filename, n, nnz, row_.data(), col_.data(), v.data()), "B200_CSR_lMatrix::ReadFile");
    std::vector<T> t(v.begin(), v.end());
    upload(t.data());
}

template <typename T>
void B200_CSR_lMatrix<T>::WriteFile(const char *filename) const
{
    std::vector<T> t;
    download_values(t);
    std::vector<double> v(t.begin(), t.end());
    CHECK(b200la_mm_write_csr(filename, this->num_row_, this->num_col_, this->nnz_, row_.data(), col_.data(),
                              v.data()),
          "B200_CSR_lMatrix::WriteFile");
}

template <typename T>
void B200_CSR_lMatrix<T>::VectorMult(const lVector<T> &invec, lVector<T> *outvec) const
{
    const B200_lVector<T> &x = b200(invec, "VectorMult");
    B200_lVector<T> &y = b200(*outvec, "VectorMult");
    if (x.get_size() != this->num_col_ || y.get_size() != this->num_row_) throw B200Error("VectorMult: sizes");
    CHECK(b200la_spmv(b200_lmp_context(), handle(), x.device(), y.device()), "VectorMult");
}

template <typename T>
void B200_CSR_lMatrix<T>::VectorMultAdd(const lVector<T> &invec, lVector<T> *outvec) const
{
    const B200_lVector<T> &x = b200(invec, "VectorMultAdd");
    B200_lVector<T> &y = b200(*outvec, "VectorMultAdd");
    if (x.get_size() != this->num_col_ || y.get_size() != this->num_row_) throw B200Error("VectorMultAdd: sizes");
    CHECK(b200la_spmv_add(b200_lmp_context(), handle(), x.device(), y.device()), "VectorMultAdd");
}

// out = (A - D) in: the product, then the diagonal's share taken away
template <typename T>
void B200_CSR_lMatrix<T>::VectorMultNoDiag(const lVector<T> &in, lVector<T> *out) const
{
    VectorMult(in, out);
    const int n = std::min(this->num_row_, this->num_col_);
    B200_lVector<T> d(n, "diag");
    extract_diagelements(0, n, &d);
    d.ElementWiseMult(b200(in, "VectorMultNoDiag"));
    B200_lVector<T> &y = b200(*out, "VectorMultNoDiag");
    CHECK(b200la_axpy(b200_lmp_context(), dtype_of<T>(), n, -1.0, d.device(), y.device()), "VectorMultNoDiag");
}

// each row's diagonal entry moved to the row's first position (the CPU
// matrices' SwapDiagElementsToRowFront, on the host mirror)
template <typename T>
void B200_CSR_lMatrix<T>::SwapDiagElementsToRowFront(void)
{
    std::vector<T> v;
    download_values(v);
    for (int i = 0; i < this->num_row_; ++i)
        for (int j = row_[i]; j < row_[i + 1]; ++j)
            if (col_[j] == i) {
                std::swap(col_[j], col_[row_[i]]);
                std::swap(v[j], v[row_[i]]);
                break;
            }
    upload(v.data());
}

template <typename T>
void B200_CSR_lMatrix<T>::Compress(void)
{
    b200la_csr *B = nullptr;
    CHECK(b200la_csr_compress(b200_lmp_context(), handle(), &B), "Compress");
    adopt(B);
}

template <typename T>
void B200_CSR_lMatrix<T>::Scale(const T alpha)
{
    CHECK(b200la_csr_scale(b200_lmp_context(), handle(), (double)alpha, B200LA_SCALE_ALL), "Scale");
}

template <typename T>
void B200_CSR_lMatrix<T>::ScaleOffdiag(const T alpha)
{
    CHECK(b200la_csr_scale(b200_lmp_context(), handle(), (double)alpha, B200LA_SCALE_OFFDIAG), "ScaleOffdiag");
}

template <typename T>
void B200_CSR_lMatrix<T>::extract_diagelements(const int start_i, const int end_i, lVector<T> *vec) const
{
    B200_lVector<T> &d = b200(*vec, "extract_diagelements");
    CHECK(b200la_csr_diag(b200_lmp_context(), handle(), start_i, end_i, 0, d.device()), "extract_diagelements");
}

template <typename T>
void B200_CSR_lMatrix<T>::extract_invdiagelements(const int start_i, const int end_i, lVector<T> *vec) const
{
    B200_lVector<T> &d = b200(*vec, "extract_invdiagelements");
    CHECK(b200la_csr_diag(b200_lmp_context(), handle(), start_i, end_i, 1, d.device()), "extract_invdiagelements");
}

template <typename T>
lMatrix<T> *B200_CSR_lMatrix<T>::extract_submatrix(const int start_row, const int start_col, const int end_row,
                                                   const int end_col) const
{
    b200la_csr *S = nullptr;
    CHECK(b200la_csr_extract_submatrix(b200_lmp_context(), handle(), start_row, start_col, end_row, end_col, &S),
          "extract_submatrix");
    B200_CSR_lMatrix<T> *m = new B200_CSR_lMatrix<T>();
    m->name_ = "sub matrix from " + this->name_;
    m->adopt(S);
    return m;
}

namespace {
template <typename T>
std::vector<double> as_double(const std::vector<T> &v)
{
    return std::vector<double>(v.begin(), v.end());
}
}  // namespace

// B = P A P^T on the host copy (lmatrix_csr_cpu.cc:1847-1861), then uploaded
template <typename T>
void B200_CSR_lMatrix<T>::Reorder(const int *index)
{
    std::vector<T> v;
    download_values(v);
    std::vector<double> vd = as_double(v), vo(this->nnz_);
    std::vector<int> r(this->num_row_ + 1), c(this->nnz_);
    CHECK(b200la_reorder_csr(this->num_row_, row_.data(), col_.data(), vd.data(), index, r.data(), c.data(),
                             vo.data()),
          "Reorder");
    row_ = r;
    col_ = c;
    std::vector<T> t(vo.begin(), vo.end());
    upload(t.data());
}

template <typename T>
void B200_CSR_lMatrix<T>::Multicoloring(int &ncolors, int **color_sizes, int **permut_index) const
{
    const int n = this->num_row_;
    std::vector<int> sizes(std::max(n, 1));
    *permut_index = new int[n];
    CHECK(b200la_multicoloring(n, row_.data(), col_.data(), &ncolors, sizes.data(), *permut_index), "Multicoloring");
    *color_sizes = new int[ncolors];
    std::copy(sizes.begin(), sizes.begin() + ncolors, *color_sizes);
}

template <typename T>
void B200_CSR_lMatrix<T>::Levelscheduling(int &nlevels, int **level_sizes, int **permut_index) const
{
    const int n = this->num_row_;
    std::vector<int> sizes(std::max(n, 1));
    *permut_index = new int[n];
    CHECK(b200la_levelscheduling(n, row_.data(), col_.data(), &nlevels, sizes.data(), *permut_index),
          "Levelscheduling");
    *level_sizes = new int[nlevels];
    std::copy(sizes.begin(), sizes.begin() + nlevels, *level_sizes);
}

// in-place ILU(0) (lmatrix_csr_cpu.cc:1880-1930) of the host copy, in FP64, then uploaded
template <typename T>
void B200_CSR_lMatrix<T>::ilu0(void)
{
    std::vector<T> v;
    download_values(v);
    std::vector<double> vd = as_double(v);
    CHECK(b200la_ilu0(this->num_row_, row_.data(), col_.data(), vd.data()), "ilu0");
    std::vector<T> t(vd.begin(), vd.end());
    upload(t.data());
}

// Assembly (init_structure / add_value(s) / ZeroRows, lmatrix_csr_cpu.cc:1047-1181)
// runs on values staged on the host; they move to the device at the next
// device operation.  FP32 matrices accumulate in FP64 and round once there.
template <typename T>
void B200_CSR_lMatrix<T>::init_structure(const int *rows, const int *cols)
{
    std::vector<int> r(this->num_row_ + 1), c(this->nnz_);
    CHECK(b200la_coo_to_csr(this->num_row_, this->nnz_, rows, cols, nullptr, r.data(), c.data(), nullptr),
          "init_structure");
    row_ = r;
    col_ = c;
    if (A_) b200la_csr_destroy(A_);
    A_ = nullptr;
    stage_.assign(this->nnz_, 0.0);
    staged_ = true;
}

template <typename T>
void B200_CSR_lMatrix<T>::add_value(const int row, const int col, const T val)
{
    add_values(&row, 1, &col, 1, &val);
}

template <typename T>
void B200_CSR_lMatrix<T>::stage() const
{
    if (staged_) return;
    std::vector<T> v;
    download_values(v);
    stage_.assign(v.begin(), v.end());
    staged_ = true;
}

template <typename T>
void B200_CSR_lMatrix<T>::add_values(const int *rows, int num_rows, const int *cols, int num_cols, const T *values)
{
    stage();
    if (sizeof(T) == 8) {
        CHECK(b200la_add_values(row_.data(), col_.data(), stage_.data(), rows, num_rows, cols, num_cols,
                                reinterpret_cast<const double *>(values)),
              "add_values");
    } else {
        std::vector<double> in(values, values + (size_t)num_rows * num_cols);
        CHECK(b200la_add_values(row_.data(), col_.data(), stage_.data(), rows, num_rows, cols, num_cols, in.data()),
              "add_values");
    }
}

template <typename T>
void B200_CSR_lMatrix<T>::ZeroRows(const int *index_set, const int size, const T alpha)
{
    stage();
    CHECK(b200la_zero_rows(row_.data(), col_.data(), stage_.data(), index_set, size, (double)alpha), "ZeroRows");
}

template class B200_lVector<double>;
template class B200_lVector<float>;
template class B200_CSR_lMatrix<double>;
template class B200_CSR_lMatrix<float>;

}  // namespace la
}  // namespace hiflow
