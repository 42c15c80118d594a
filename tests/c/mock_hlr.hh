// A minimal stand-in for the HLR / HLIBpro types that the HLR-side adapter
//  touches, so that the adapter can be compiled
// and run here: TMatrix / TBlockMatrix with index sets, dense_matrix and
// lrmatrix leaves whose blas::matrix copies are shallow views (as HLR's
// are), scalar_vector, matop_t and HLR_ERROR.  Only the members the adapter
// uses exist; the semantics follow the reference's headers
// (include/hlr/matrix/dense_matrix.hh, lrmatrix.hh, vector/scalar_vector.hh).
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#define HLR_ERROR(msg) throw std::runtime_error(std::string(msg))
#define cptrcast(ptr, type) (static_cast<const type*>(ptr))

using uint = unsigned int;

namespace Hpro {

enum matop_t { apply_normal = 'N', apply_transposed = 'T', apply_adjoint = 'C' };

struct TIndexSet {
    int64_t f = 0, l = -1;
    int64_t first() const { return f; }
    int64_t last() const { return l; }
    int64_t size() const { return l - f + 1; }
};

template <typename T>
struct TMatrix {
    TIndexSet r, c;
    virtual ~TMatrix() = default;
    TIndexSet row_is() const { return r; }
    TIndexSet col_is() const { return c; }
    size_t nrows() const { return size_t(r.size()); }
    size_t ncols() const { return size_t(c.size()); }
    virtual bool blocked() const { return false; }
    virtual bool dense() const { return false; }
};

template <typename T>
struct TBlockMatrix : TMatrix<T> {
    uint nbr = 0, nbc = 0;
    std::vector<std::unique_ptr<TMatrix<T>>> sub;   // column-major nbr x nbc
    uint nblock_rows() const { return nbr; }
    uint nblock_cols() const { return nbc; }
    const TMatrix<T>* block(uint i, uint j) const { return sub[i + j * nbr].get(); }
    bool blocked() const override { return true; }
};

}  // namespace Hpro

namespace hlr {

template <typename T> bool is_blocked(const Hpro::TMatrix<T>& M) { return M.blocked(); }
template <typename T> bool is_null(const T* p) { return p == nullptr; }

namespace blas {
// column-major matrix; copies share the storage (HLR's default copy is a view)
template <typename T>
struct matrix {
    std::shared_ptr<std::vector<T>> d;
    int64_t nr = 0, nc = 0;
    matrix() = default;
    matrix(int64_t r, int64_t c) : d(std::make_shared<std::vector<T>>(size_t(r * c))), nr(r), nc(c) {}
    T& operator()(int64_t i, int64_t j) { return (*d)[size_t(i + j * nr)]; }
    T operator()(int64_t i, int64_t j) const { return (*d)[size_t(i + j * nr)]; }
    T* data() const { return d ? d->data() : nullptr; }
    int64_t col_stride() const { return nr; }
};
template <typename T>
struct vector {
    std::vector<T> v;
    T* data() { return v.data(); }
    const T* data() const { return v.data(); }
};
}  // namespace blas

namespace matrix {
template <typename T>
struct dense_matrix : Hpro::TMatrix<T> {
    blas::matrix<T> M;
    const blas::matrix<T>& mat() const { return M; }
    bool dense() const override { return true; }
};
template <typename T>
struct lrmatrix : Hpro::TMatrix<T> {
    blas::matrix<T> u, v;   // M = U V^T
    uint rank() const { return uint(u.nc); }
    const blas::matrix<T>& U() const { return u; }
    const blas::matrix<T>& V() const { return v; }
};
template <typename T> bool is_dense(const Hpro::TMatrix<T>& M) { return M.dense(); }
}  // namespace matrix

namespace vector {
template <typename T>
struct scalar_vector {
    blas::vector<T> x;
};
}  // namespace vector

namespace blas {
template <typename T> vector<T>& vec(hlr::vector::scalar_vector<T>& s) { return s.x; }
template <typename T> const vector<T>& vec(const hlr::vector::scalar_vector<T>& s) { return s.x; }
}  // namespace blas

}  // namespace hlr
