// eigen_lite.h -- a small Eigen-API-compatible dense matrix subset for the VBD C++ surface.
//
// The reference's public C++ types are Eigen types (Types.h:26-64: Vec3, Matrix3r, TVerticesMat,
// ...).  Eigen 3 is not part of this project, so this header provides, under namespace Eigen, the
// subset those headers and their callers use:
//   Matrix<Scalar, Rows, Cols> (fixed or Dynamic sizes, column-major storage, data() layout as
//   Eigen's), Block views (col, row, block, segment), + - * / with scalars (a scalar of another
//   arithmetic type is converted to Scalar first), matrix products, transpose, determinant,
//   inverse (2x2, 3x3), trace, sum, prod, dot, cross, norm, array() coefficient-wise products,
//   asDiagonal, comma initialisation, Zero / Identity, JacobiSVD and SelfAdjointEigenSolver for
//   small matrices.
// Semantics: every expression is evaluated eagerly into a temporary, in source order; inner
// products accumulate left to right from the first term.  (Eigen's expression templates and
// summation order are not reproduced, so results can differ from real Eigen in the last bits.)
// When the real Eigen is available and VBD_USE_REAL_EIGEN is defined, include <Eigen/Dense>
// instead of this file.
#pragma once

#include <algorithm>
#include <array>
#include <cassert>
#include <cmath>
#include <cstddef>
#include <initializer_list>
#include <iostream>
#include <map>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace Eigen {

using Index = std::ptrdiff_t;
constexpr int Dynamic = -1;
enum DecompositionOptions { ComputeFullU = 0x04, ComputeThinU = 0x08, ComputeFullV = 0x10, ComputeThinV = 0x20 };

template <class S, int R, int C> class Matrix;
template <class X, int BR, int BC> class Block;

// Declared only (named in the reference's type aliases, never used on its VBD path).
template <class S, int Options = 0, class StorageIndex = int> class SparseMatrix;
template <class S, class StorageIndex = int> class Triplet;

namespace internal {

template <class T> struct is_dense : std::false_type {};
template <class S, int R, int C> struct is_dense<Matrix<S, R, C>> : std::true_type {};
template <class X, int R, int C> struct is_dense<Block<X, R, C>> : std::true_type {};

template <class T> struct traits;
template <class S, int R, int C> struct traits<Matrix<S, R, C>> {
    using Scalar = S;
    static constexpr int Rows = R, Cols = C;
};
template <class X, int R, int C> struct traits<Block<X, R, C>> {
    using Scalar = typename std::remove_const<X>::type::Scalar;
    static constexpr int Rows = R, Cols = C;
};

template <class T> using plain_t = Matrix<typename traits<T>::Scalar, traits<T>::Rows, traits<T>::Cols>;

// size of an expression result: a fixed size wins over Dynamic
constexpr int pick(int a, int b) { return a != Dynamic ? a : b; }

template <class T> constexpr bool is_scalar_v = std::is_arithmetic<T>::value;

}  // namespace internal

// Coefficient-wise view returned by array(): supports * (coefficient product) and sum().
template <class M> class ArrayView {
  public:
    explicit ArrayView(M m) : m_(std::move(m)) {}
    const M& matrix() const { return m_; }
    typename M::Scalar sum() const { return m_.sum(); }
    ArrayView operator*(const ArrayView& o) const { return ArrayView(m_.cwiseProduct(o.m_)); }

  private:
    M m_;
};

namespace internal {
// Coefficient storage: inline for fixed sizes (no heap traffic per temporary), heap otherwise.
template <class S, int R, int C, bool Fixed = (R != Dynamic && C != Dynamic)> struct Storage;
template <class S, int R, int C> struct Storage<S, R, C, true> {
    std::array<S, size_t(R* C > 0 ? R * C : 1)> a{};
    void assign(size_t, S v) { a.fill(v); }
    S* data() { return a.data(); }
    const S* data() const { return a.data(); }
    S& operator[](size_t i) { return a[i]; }
    const S& operator[](size_t i) const { return a[i]; }
    S* begin() { return a.data(); }
    S* end() { return a.data() + size_t(R * C); }
    const S* begin() const { return a.data(); }
    const S* end() const { return a.data() + size_t(R * C); }
};
template <class S, int R, int C> struct Storage<S, R, C, false> {
    std::vector<S> v;
    void assign(size_t n, S x) { v.assign(n, x); }
    S* data() { return v.data(); }
    const S* data() const { return v.data(); }
    S& operator[](size_t i) { return v[i]; }
    const S& operator[](size_t i) const { return v[i]; }
    S* begin() { return v.data(); }
    S* end() { return v.data() + v.size(); }
    const S* begin() const { return v.data(); }
    const S* end() const { return v.data() + v.size(); }
};
}  // namespace internal

template <class S, int R, int C> class Matrix {
    static_assert(R == Dynamic || R >= 0, "bad row count");
    static_assert(C == Dynamic || C >= 0, "bad column count");

  public:
    using Scalar = S;
    static constexpr int RowsAtCompileTime = R;
    static constexpr int ColsAtCompileTime = C;
    static constexpr bool IsVectorAtCompileTime = (R == 1 || C == 1);

    Matrix() : rows_(R == Dynamic ? 0 : R), cols_(C == Dynamic ? 0 : C) { d_.assign(size_t(rows_ * cols_), S(0)); }
    Matrix(Index rows, Index cols) : rows_(rows), cols_(cols) {
        check_shape(rows, cols);
        d_.assign(size_t(rows * cols), S(0));
    }
    // Vector of a given length (dynamic-length vectors), or of 2 / 3 / 4 given coefficients.
    template <class T, class = typename std::enable_if<internal::is_scalar_v<T> && (R == Dynamic || C == Dynamic) &&
                                                       IsVectorAtCompileTime>::type>
    explicit Matrix(T n) : Matrix(R == 1 ? 1 : Index(n), C == 1 ? 1 : Index(n)) {}
    // coefficient constructors of fixed-size 2-, 3- and 4-vectors
    template <int K = R * C, class = typename std::enable_if<K == 2 && IsVectorAtCompileTime>::type>
    Matrix(S a, S b) : Matrix(vec_rows(2), vec_cols(2)) {
        d_[0] = a;
        d_[1] = b;
    }
    template <int K = R * C, class = typename std::enable_if<K == 3 && IsVectorAtCompileTime>::type>
    Matrix(S a, S b, S c) : Matrix(vec_rows(3), vec_cols(3)) {
        d_[0] = a;
        d_[1] = b;
        d_[2] = c;
    }
    template <int K = R * C, class = typename std::enable_if<K == 4 && IsVectorAtCompileTime>::type>
    Matrix(S a, S b, S c, S e) : Matrix(vec_rows(4), vec_cols(4)) {
        d_[0] = a;
        d_[1] = b;
        d_[2] = c;
        d_[3] = e;
    }
    Matrix(const Matrix&) = default;
    Matrix(Matrix&&) = default;
    Matrix& operator=(const Matrix&) = default;
    Matrix& operator=(Matrix&&) = default;

    // From any dense expression of the same scalar (fixed <-> dynamic, blocks).
    template <class X, class = typename std::enable_if<internal::is_dense<X>::value>::type>
    Matrix(const X& o) : rows_(o.rows()), cols_(o.cols()) {
        check_shape(rows_, cols_);
        d_.assign(size_t(rows_ * cols_), S(0));
        for (Index j = 0; j < cols_; ++j)
            for (Index i = 0; i < rows_; ++i) (*this)(i, j) = o(i, j);
    }
    template <class X, class = typename std::enable_if<internal::is_dense<X>::value>::type>
    Matrix& operator=(const X& o) {
        Matrix tmp(o);
        *this = std::move(tmp);
        return *this;
    }

    Index rows() const { return rows_; }
    Index cols() const { return cols_; }
    Index size() const { return rows_ * cols_; }
    S* data() { return d_.data(); }
    const S* data() const { return d_.data(); }

    S& operator()(Index i, Index j) { return d_[size_t(i + j * rows_)]; }
    const S& operator()(Index i, Index j) const { return d_[size_t(i + j * rows_)]; }
    S& operator()(Index i) { return d_[size_t(i)]; }
    const S& operator()(Index i) const { return d_[size_t(i)]; }
    S& operator[](Index i) { return d_[size_t(i)]; }
    const S& operator[](Index i) const { return d_[size_t(i)]; }
    S coeff(Index i, Index j) const { return (*this)(i, j); }
    S& coeffRef(Index i, Index j) { return (*this)(i, j); }
    S coeff(Index i) const { return d_[size_t(i)]; }
    S& coeffRef(Index i) { return d_[size_t(i)]; }
    S& x() { return d_[0]; }
    S& y() { return d_[1]; }
    S& z() { return d_[2]; }
    S& w() { return d_[3]; }
    const S& x() const { return d_[0]; }
    const S& y() const { return d_[1]; }
    const S& z() const { return d_[2]; }
    const S& w() const { return d_[3]; }

    void resize(Index rows, Index cols) {
        check_shape(rows, cols);
        rows_ = rows;
        cols_ = cols;
        d_.assign(size_t(rows * cols), S(0));
    }
    void resize(Index n) {
        if (R == 1)
            resize(1, n);
        else
            resize(n, 1);
    }
    Matrix& setZero() {
        std::fill(d_.begin(), d_.end(), S(0));
        return *this;
    }
    Matrix& setConstant(S v) {
        std::fill(d_.begin(), d_.end(), v);
        return *this;
    }
    Matrix& setIdentity() {
        setZero();
        for (Index i = 0; i < std::min(rows_, cols_); ++i) (*this)(i, i) = S(1);
        return *this;
    }
    static Matrix Zero() { return Matrix(); }
    static Matrix Zero(Index n) {
        Matrix m;
        m.resize(n);
        return m;
    }
    static Matrix Zero(Index r, Index c) { return Matrix(r, c); }
    static Matrix Constant(S v) { return Matrix().setConstant(v); }
    static Matrix Identity() { return Matrix().setIdentity(); }
    static Matrix Identity(Index r, Index c) { return Matrix(r, c).setIdentity(); }

    // views
    Block<Matrix, R, 1> col(Index j) { return Block<Matrix, R, 1>(*this, 0, j, rows_, 1); }
    Block<const Matrix, R, 1> col(Index j) const { return Block<const Matrix, R, 1>(*this, 0, j, rows_, 1); }
    Block<Matrix, 1, C> row(Index i) { return Block<Matrix, 1, C>(*this, i, 0, 1, cols_); }
    Block<const Matrix, 1, C> row(Index i) const { return Block<const Matrix, 1, C>(*this, i, 0, 1, cols_); }
    template <int BR, int BC> Block<Matrix, BR, BC> block(Index i, Index j) {
        return Block<Matrix, BR, BC>(*this, i, j, BR, BC);
    }
    template <int BR, int BC> Block<const Matrix, BR, BC> block(Index i, Index j) const {
        return Block<const Matrix, BR, BC>(*this, i, j, BR, BC);
    }
    Block<Matrix, Dynamic, Dynamic> block(Index i, Index j, Index r, Index c) {
        return Block<Matrix, Dynamic, Dynamic>(*this, i, j, r, c);
    }
    Block<const Matrix, Dynamic, Dynamic> block(Index i, Index j, Index r, Index c) const {
        return Block<const Matrix, Dynamic, Dynamic>(*this, i, j, r, c);
    }
    template <int N> Block<Matrix, (C == 1 ? N : 1), (C == 1 ? 1 : N)> segment(Index i) {
        return Block<Matrix, (C == 1 ? N : 1), (C == 1 ? 1 : N)>(*this, C == 1 ? i : 0, C == 1 ? 0 : i,
                                                                    C == 1 ? N : 1, C == 1 ? 1 : N);
    }
    template <int N> Block<const Matrix, (C == 1 ? N : 1), (C == 1 ? 1 : N)> segment(Index i) const {
        return Block<const Matrix, (C == 1 ? N : 1), (C == 1 ? 1 : N)>(*this, C == 1 ? i : 0, C == 1 ? 0 : i,
                                                                          C == 1 ? N : 1, C == 1 ? 1 : N);
    }

    Matrix<S, C, R> transpose() const {
        Matrix<S, C, R> t(cols_, rows_);
        for (Index j = 0; j < cols_; ++j)
            for (Index i = 0; i < rows_; ++i) t(j, i) = (*this)(i, j);
        return t;
    }
    S sum() const {
        S s = S(0);
        for (const S& v : d_) s += v;
        return s;
    }
    S prod() const {
        S p = S(1);
        for (const S& v : d_) p *= v;
        return p;
    }
    S trace() const {
        S s = S(0);
        for (Index i = 0; i < std::min(rows_, cols_); ++i) s += (*this)(i, i);
        return s;
    }
    S squaredNorm() const {
        S s = S(0);
        for (const S& v : d_) s += v * v;
        return s;
    }
    S norm() const { return std::sqrt(squaredNorm()); }
    template <class X> S dot(const X& o) const {
        S s = d_[0] * o.coeff(0);
        for (Index i = 1; i < size(); ++i) s += d_[size_t(i)] * o.coeff(i);
        return s;
    }
    template <class X> Matrix cross(const X& o) const {
        Matrix r;
        r.resize(rows_, cols_);
        r[0] = (*this)[1] * o.coeff(2) - (*this)[2] * o.coeff(1);
        r[1] = (*this)[2] * o.coeff(0) - (*this)[0] * o.coeff(2);
        r[2] = (*this)[0] * o.coeff(1) - (*this)[1] * o.coeff(0);
        return r;
    }
    template <class X> Matrix cwiseProduct(const X& o) const {
        Matrix r(*this);
        for (Index j = 0; j < cols_; ++j)
            for (Index i = 0; i < rows_; ++i) r(i, j) *= o(i, j);
        return r;
    }
    ArrayView<Matrix> array() const { return ArrayView<Matrix>(*this); }
    Matrix<S, Dynamic, Dynamic> asDiagonal() const {
        Matrix<S, Dynamic, Dynamic> D(size(), size());
        for (Index i = 0; i < size(); ++i) D(i, i) = d_[size_t(i)];
        return D;
    }

    // cofactor expansion along the first row
    S determinant() const {
        const Matrix& a = *this;
        if (rows_ == 1) return a(0, 0);
        if (rows_ == 2) return a(0, 0) * a(1, 1) - a(0, 1) * a(1, 0);
        if (rows_ == 3)
            return a(0, 0) * (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) - a(0, 1) * (a(1, 0) * a(2, 2) - a(1, 2) * a(2, 0)) +
                   a(0, 2) * (a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0));
        throw std::logic_error("eigen_lite: determinant implemented up to 3x3");
    }
    // adjugate over determinant; 3x3 cofactors taken cyclically, det expanded along column 0
    Matrix inverse() const {
        const Matrix& a = *this;
        Matrix r(*this);
        if (rows_ == 2) {
            const S inv = S(1) / (a(0, 0) * a(1, 1) - a(0, 1) * a(1, 0));
            r(0, 0) = a(1, 1) * inv;
            r(0, 1) = -a(0, 1) * inv;
            r(1, 0) = -a(1, 0) * inv;
            r(1, 1) = a(0, 0) * inv;
            return r;
        }
        if (rows_ != 3) throw std::logic_error("eigen_lite: inverse implemented for 2x2 and 3x3");
        auto cof = [&](int i, int j) {
            const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            return a(i1, j1) * a(i2, j2) - a(i1, j2) * a(i2, j1);
        };
        const S c0 = cof(0, 0), c1 = cof(1, 0), c2 = cof(2, 0);
        S det = c0 * a(0, 0);
        det += c1 * a(1, 0);
        det += c2 * a(2, 0);
        const S inv = S(1) / det;
        r(0, 0) = c0 * inv;
        r(0, 1) = c1 * inv;
        r(0, 2) = c2 * inv;
        for (int i = 1; i < 3; ++i)
            for (int j = 0; j < 3; ++j) r(i, j) = cof(j, i) * inv;
        return r;
    }

    // in-place arithmetic
    template <class X, class = typename std::enable_if<internal::is_dense<X>::value>::type>
    Matrix& operator+=(const X& o) {
        for (Index j = 0; j < cols_; ++j)
            for (Index i = 0; i < rows_; ++i) (*this)(i, j) += o(i, j);
        return *this;
    }
    template <class X, class = typename std::enable_if<internal::is_dense<X>::value>::type>
    Matrix& operator-=(const X& o) {
        for (Index j = 0; j < cols_; ++j)
            for (Index i = 0; i < rows_; ++i) (*this)(i, j) -= o(i, j);
        return *this;
    }
    template <class T, class = typename std::enable_if<internal::is_scalar_v<T>>::type> Matrix& operator*=(T s) {
        const S v = S(s);
        for (S& x : d_) x *= v;
        return *this;
    }
    template <class T, class = typename std::enable_if<internal::is_scalar_v<T>>::type> Matrix& operator/=(T s) {
        const S v = S(s);
        for (S& x : d_) x /= v;
        return *this;
    }

    // comma initialiser, row by row
    class CommaInit {
      public:
        CommaInit(Matrix& m, S first) : m_(m), k_(0) { put(first); }
        template <class T> CommaInit& operator,(T v) {
            put(S(v));
            return *this;
        }

      private:
        void put(S v) {
            const Index i = k_ / m_.cols(), j = k_ % m_.cols();
            m_(i, j) = v;
            ++k_;
        }
        Matrix& m_;
        Index k_;
    };
    template <class T, class = typename std::enable_if<internal::is_scalar_v<T>>::type> CommaInit operator<<(T v) {
        return CommaInit(*this, S(v));
    }

  private:
    static constexpr Index vec_rows(Index n) { return R == 1 ? 1 : n; }
    static constexpr Index vec_cols(Index n) { return R == 1 ? n : 1; }
    static void check_shape(Index r, Index c) {
        if ((R != Dynamic && r != R) || (C != Dynamic && c != C))
            throw std::logic_error("eigen_lite: size does not match a fixed dimension");
    }
    Index rows_, cols_;
    internal::Storage<S, R, C> d_;
};

// Writable (or, for a const X, read-only) rectangular view of a matrix.
template <class X, int BR, int BC> class Block {
    using M = typename std::remove_const<X>::type;

  public:
    using Scalar = typename M::Scalar;
    using Ptr = typename std::conditional<std::is_const<X>::value, const Scalar*, Scalar*>::type;
    using Ref = typename std::conditional<std::is_const<X>::value, const Scalar&, Scalar&>::type;
    static constexpr int RowsAtCompileTime = BR;
    static constexpr int ColsAtCompileTime = BC;

    Block(X& m, Index i, Index j, Index r, Index c) : base_(m.data()), stride_(m.rows()), i_(i), j_(j), r_(r), c_(c) {}
    Block(const Block&) = default;

    Index rows() const { return r_; }
    Index cols() const { return c_; }
    Index size() const { return r_ * c_; }
    Ref operator()(Index i, Index j) const { return base_[(i_ + i) + (j_ + j) * stride_]; }
    Ref operator()(Index k) const { return r_ == 1 ? (*this)(0, k) : (*this)(k, 0); }
    Ref operator[](Index k) const { return (*this)(k); }
    Scalar coeff(Index i, Index j) const { return (*this)(i, j); }
    Scalar coeff(Index k) const { return (*this)(k); }
    Ref x() const { return (*this)(0); }
    Ref y() const { return (*this)(1); }
    Ref z() const { return (*this)(2); }

    // assignment copies coefficients into the viewed matrix
    Block& operator=(const Block& o) {
        Matrix<Scalar, BR, BC> tmp(o);
        assign(tmp);
        return *this;
    }
    template <class Y, class = typename std::enable_if<internal::is_dense<Y>::value>::type>
    Block& operator=(const Y& o) {
        Matrix<Scalar, BR, BC> tmp(o);
        assign(tmp);
        return *this;
    }
    template <class Y, class = typename std::enable_if<internal::is_dense<Y>::value>::type>
    Block& operator+=(const Y& o) {
        Matrix<Scalar, BR, BC> tmp(o);
        for (Index j = 0; j < c_; ++j)
            for (Index i = 0; i < r_; ++i) (*this)(i, j) += tmp(i, j);
        return *this;
    }
    template <class Y, class = typename std::enable_if<internal::is_dense<Y>::value>::type>
    Block& operator-=(const Y& o) {
        Matrix<Scalar, BR, BC> tmp(o);
        for (Index j = 0; j < c_; ++j)
            for (Index i = 0; i < r_; ++i) (*this)(i, j) -= tmp(i, j);
        return *this;
    }
    Block& setZero() {
        for (Index j = 0; j < c_; ++j)
            for (Index i = 0; i < r_; ++i) (*this)(i, j) = Scalar(0);
        return *this;
    }

    Matrix<Scalar, BR, BC> eval() const { return Matrix<Scalar, BR, BC>(*this); }
    Matrix<Scalar, BC, BR> transpose() const { return eval().transpose(); }
    Scalar sum() const { return eval().sum(); }
    Scalar squaredNorm() const { return eval().squaredNorm(); }
    Scalar norm() const { return eval().norm(); }
    template <class Y> Scalar dot(const Y& o) const { return eval().dot(o); }
    template <class Y> Matrix<Scalar, BR, BC> cross(const Y& o) const { return eval().cross(o); }
    ArrayView<Matrix<Scalar, BR, BC>> array() const { return eval().array(); }

  private:
    void assign(const Matrix<Scalar, BR, BC>& t) {
        if (t.rows() != r_ || t.cols() != c_) throw std::logic_error("eigen_lite: block assignment size mismatch");
        for (Index j = 0; j < c_; ++j)
            for (Index i = 0; i < r_; ++i) (*this)(i, j) = t(i, j);
    }
    Ptr base_;
    Index stride_, i_, j_, r_, c_;
};

// ---- free operators (eager) -----------------------------------------------------------------

template <class A, class B,
          class = typename std::enable_if<internal::is_dense<A>::value && internal::is_dense<B>::value>::type>
Matrix<typename internal::traits<A>::Scalar, internal::pick(internal::traits<A>::Rows, internal::traits<B>::Rows),
       internal::pick(internal::traits<A>::Cols, internal::traits<B>::Cols)>
operator+(const A& a, const B& b) {
    Matrix<typename internal::traits<A>::Scalar, internal::pick(internal::traits<A>::Rows, internal::traits<B>::Rows),
           internal::pick(internal::traits<A>::Cols, internal::traits<B>::Cols)>
        r(a.rows(), a.cols());
    for (Index j = 0; j < a.cols(); ++j)
        for (Index i = 0; i < a.rows(); ++i) r(i, j) = a(i, j) + b(i, j);
    return r;
}

template <class A, class B,
          class = typename std::enable_if<internal::is_dense<A>::value && internal::is_dense<B>::value>::type>
Matrix<typename internal::traits<A>::Scalar, internal::pick(internal::traits<A>::Rows, internal::traits<B>::Rows),
       internal::pick(internal::traits<A>::Cols, internal::traits<B>::Cols)>
operator-(const A& a, const B& b) {
    Matrix<typename internal::traits<A>::Scalar, internal::pick(internal::traits<A>::Rows, internal::traits<B>::Rows),
           internal::pick(internal::traits<A>::Cols, internal::traits<B>::Cols)>
        r(a.rows(), a.cols());
    for (Index j = 0; j < a.cols(); ++j)
        for (Index i = 0; i < a.rows(); ++i) r(i, j) = a(i, j) - b(i, j);
    return r;
}

template <class A, class = typename std::enable_if<internal::is_dense<A>::value>::type>
internal::plain_t<A> operator-(const A& a) {
    internal::plain_t<A> r(a);
    for (Index j = 0; j < r.cols(); ++j)
        for (Index i = 0; i < r.rows(); ++i) r(i, j) = -r(i, j);
    return r;
}

template <class T, class A,
          class = typename std::enable_if<internal::is_scalar_v<T> && internal::is_dense<A>::value>::type>
internal::plain_t<A> operator*(T s, const A& a) {
    using S = typename internal::traits<A>::Scalar;
    const S v = S(s);
    internal::plain_t<A> r(a);
    for (Index j = 0; j < r.cols(); ++j)
        for (Index i = 0; i < r.rows(); ++i) r(i, j) = v * r(i, j);
    return r;
}

template <class A, class T,
          class = typename std::enable_if<internal::is_scalar_v<T> && internal::is_dense<A>::value>::type>
internal::plain_t<A> operator*(const A& a, T s) {
    using S = typename internal::traits<A>::Scalar;
    const S v = S(s);
    internal::plain_t<A> r(a);
    for (Index j = 0; j < r.cols(); ++j)
        for (Index i = 0; i < r.rows(); ++i) r(i, j) = r(i, j) * v;
    return r;
}

template <class A, class T,
          class = typename std::enable_if<internal::is_scalar_v<T> && internal::is_dense<A>::value>::type>
internal::plain_t<A> operator/(const A& a, T s) {
    using S = typename internal::traits<A>::Scalar;
    const S v = S(s);
    internal::plain_t<A> r(a);
    for (Index j = 0; j < r.cols(); ++j)
        for (Index i = 0; i < r.rows(); ++i) r(i, j) = r(i, j) / v;
    return r;
}

// matrix product, inner sums accumulated left to right
template <class A, class B,
          class = typename std::enable_if<internal::is_dense<A>::value && internal::is_dense<B>::value>::type>
Matrix<typename internal::traits<A>::Scalar, internal::traits<A>::Rows, internal::traits<B>::Cols> operator*(
    const A& a, const B& b) {
    if (a.cols() != b.rows()) throw std::logic_error("eigen_lite: product size mismatch");
    Matrix<typename internal::traits<A>::Scalar, internal::traits<A>::Rows, internal::traits<B>::Cols> r(a.rows(),
                                                                                                         b.cols());
    for (Index i = 0; i < a.rows(); ++i)
        for (Index j = 0; j < b.cols(); ++j) {
            typename internal::traits<A>::Scalar s = a(i, 0) * b(0, j);
            for (Index k = 1; k < a.cols(); ++k) s += a(i, k) * b(k, j);
            r(i, j) = s;
        }
    return r;
}

template <class A, class = typename std::enable_if<internal::is_dense<A>::value>::type>
std::ostream& operator<<(std::ostream& os, const A& a) {
    for (Index i = 0; i < a.rows(); ++i) {
        for (Index j = 0; j < a.cols(); ++j) os << (j ? " " : "") << a(i, j);
        if (i + 1 < a.rows()) os << "\n";
    }
    return os;
}

// ---- small decompositions -------------------------------------------------------------------

// Symmetric eigen-decomposition by cyclic Jacobi rotations (in double); eigenvalues ascending.
template <class M> class SelfAdjointEigenSolver {
    using S = typename M::Scalar;
    static constexpr int N = M::RowsAtCompileTime;

  public:
    explicit SelfAdjointEigenSolver(const M& a) {
        const Index n = a.rows();
        std::vector<double> A(size_t(n * n)), V(size_t(n * n), 0.0);
        for (Index i = 0; i < n; ++i) {
            V[size_t(i * n + i)] = 1.0;
            for (Index j = 0; j < n; ++j) A[size_t(i * n + j)] = double(a(i, j));
        }
        for (int sweep = 0; sweep < 64; ++sweep) {
            double off = 0.0;
            for (Index p = 0; p < n; ++p)
                for (Index q = p + 1; q < n; ++q) off += A[size_t(p * n + q)] * A[size_t(p * n + q)];
            if (off < 1e-300) break;
            for (Index p = 0; p < n; ++p)
                for (Index q = p + 1; q < n; ++q) {
                    const double apq = A[size_t(p * n + q)];
                    if (apq == 0.0) continue;
                    const double theta = (A[size_t(q * n + q)] - A[size_t(p * n + p)]) / (2.0 * apq);
                    const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                    const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                    for (Index k = 0; k < n; ++k) {  // A <- J^T A J
                        const double akp = A[size_t(k * n + p)], akq = A[size_t(k * n + q)];
                        A[size_t(k * n + p)] = c * akp - s * akq;
                        A[size_t(k * n + q)] = s * akp + c * akq;
                    }
                    for (Index k = 0; k < n; ++k) {
                        const double apk = A[size_t(p * n + k)], aqk = A[size_t(q * n + k)];
                        A[size_t(p * n + k)] = c * apk - s * aqk;
                        A[size_t(q * n + k)] = s * apk + c * aqk;
                    }
                    for (Index k = 0; k < n; ++k) {
                        const double vkp = V[size_t(k * n + p)], vkq = V[size_t(k * n + q)];
                        V[size_t(k * n + p)] = c * vkp - s * vkq;
                        V[size_t(k * n + q)] = s * vkp + c * vkq;
                    }
                }
        }
        std::vector<Index> order(static_cast<size_t>(n));
        for (Index i = 0; i < n; ++i) order[size_t(i)] = i;
        std::sort(order.begin(), order.end(),
                  [&](Index x, Index y) { return A[size_t(x * n + x)] < A[size_t(y * n + y)]; });
        evals_.resize(n, 1);
        evecs_.resize(n, n);
        for (Index k = 0; k < n; ++k) {
            const Index c = order[size_t(k)];
            evals_(k) = S(A[size_t(c * n + c)]);
            for (Index i = 0; i < n; ++i) evecs_(i, k) = S(V[size_t(i * n + c)]);
        }
    }
    const Matrix<S, N, 1>& eigenvalues() const { return evals_; }
    const Matrix<S, N, N>& eigenvectors() const { return evecs_; }

  private:
    Matrix<S, N, 1> evals_;
    Matrix<S, N, N> evecs_;
};

// SVD of a small square matrix from the eigen-decomposition of A^T A (in double): singular values
// non-negative and descending, A = U diag(sigma) V^T.
template <class M> class JacobiSVD {
    using S = typename M::Scalar;
    static constexpr int N = M::RowsAtCompileTime;

  public:
    JacobiSVD(const M& a, unsigned = 0) {
        const Index n = a.rows();
        Matrix<double, N, N> A(n, n);
        for (Index i = 0; i < n; ++i)
            for (Index j = 0; j < n; ++j) A(i, j) = double(a(i, j));
        const Matrix<double, N, N> AtA = A.transpose() * A;
        SelfAdjointEigenSolver<Matrix<double, N, N>> es(AtA);
        sigma_.resize(n, 1);
        U_.resize(n, n);
        V_.resize(n, n);
        for (Index k = 0; k < n; ++k) {
            const Index c = n - 1 - k;  // descending
            const double lam = std::max(0.0, es.eigenvalues()(c));
            const double sg = std::sqrt(lam);
            sigma_(k) = S(sg);
            Matrix<double, N, 1> v(n, 1);
            for (Index i = 0; i < n; ++i) v(i) = es.eigenvectors()(i, c);
            const Matrix<double, N, 1> u = A * v;
            for (Index i = 0; i < n; ++i) {
                V_(i, k) = S(v(i));
                U_(i, k) = S(sg > 0 ? u(i) / sg : (i == k ? 1.0 : 0.0));
            }
        }
    }
    const Matrix<S, N, N>& matrixU() const { return U_; }
    const Matrix<S, N, N>& matrixV() const { return V_; }
    const Matrix<S, N, 1>& singularValues() const { return sigma_; }

  private:
    Matrix<S, N, 1> sigma_;
    Matrix<S, N, N> U_, V_;
};

// common typedefs
using Matrix3f = Matrix<float, 3, 3>;
using Matrix3d = Matrix<double, 3, 3>;
using Vector3f = Matrix<float, 3, 1>;
using Vector3d = Matrix<double, 3, 1>;
using Vector4i = Matrix<int, 4, 1>;
using MatrixXf = Matrix<float, Dynamic, Dynamic>;
using MatrixXd = Matrix<double, Dynamic, Dynamic>;
using VectorXf = Matrix<float, Dynamic, 1>;
using VectorXd = Matrix<double, Dynamic, 1>;

}  // namespace Eigen
