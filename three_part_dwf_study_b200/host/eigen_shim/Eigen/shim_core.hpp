// Project-written stand-in for the small part of the Eigen 3 API that the
// lattice study's C++ sources use. It exists so that, on a host without an
// Eigen installation, the unmodified reference headers (domain_wall/include/
// *.hpp, wilson/include/*.hpp) compile for the CPU oracle and the reference's
// mains compile against the drop-in headers (the drop-in build uses a system
// Eigen 3 instead wherever one is installed). The GPU hot path does not use it:
// there it only carries the host-side vector types across the C ABI. Nothing here is
// Eigen source; every operation is written from its mathematical definition:
//
//   dense  : column vectors / small matrices of std::complex<double>, eager
//            evaluation, a.dot(b) = sum_i conj(a_i) b_i, norm = sqrt(sum |a_i|^2)
//   sparse : compressed rows of (column, value) pairs sorted by column,
//            duplicate triplets summed in insertion order, products summed in
//            ascending inner index (the same order a column-major product uses)
//   CG     : Jacobi-preconditioned conjugate gradient (Saad, "Iterative Methods
//            for Sparse Linear Systems", 2nd ed., Alg. 9.1), started from x=0,
//            stopping when |r|^2 < tol^2 |b|^2 (Eigen's documented relative
//            residual criterion), iterations() counting completed updates of p.
//
// Summation order differs from a SIMD-vectorised Eigen build, so results agree
// with a real Eigen build to rounding, not bit for bit.
#pragma once

#include <array>
#include <cmath>
#include <complex>
#include <cstddef>
#include <limits>
#include <stdexcept>
#include <vector>

namespace Eigen {

using Index = std::ptrdiff_t;
constexpr int Dynamic = -1;
enum UpLoType { Lower = 1, Upper = 2 };

namespace shim {

template <typename S, int R, int C>
struct Storage
{
    std::array<S, R * C> a{};
    static constexpr Index rows() { return R; }
    static constexpr Index cols() { return C; }
    void resize(Index r, Index c)
    {
        if (r != R || c != C)
            throw std::runtime_error("shim: fixed-size resize");
    }
    S* data() { return a.data(); }
    const S* data() const { return a.data(); }
};

template <typename S>
struct Storage<S, Dynamic, 1>
{
    std::vector<S> v;
    Index rows() const { return static_cast<Index>(v.size()); }
    static constexpr Index cols() { return 1; }
    void resize(Index r, Index) { v.assign(static_cast<std::size_t>(r), S(0)); }
    S* data() { return v.data(); }
    const S* data() const { return v.data(); }
};

template <typename S>
struct Storage<S, Dynamic, Dynamic>
{
    std::vector<S> v;
    Index r = 0, c = 0;
    Index rows() const { return r; }
    Index cols() const { return c; }
    void resize(Index rr, Index cc)
    {
        r = rr;
        c = cc;
        v.assign(static_cast<std::size_t>(rr * cc), S(0));
    }
    S* data() { return v.data(); }
    const S* data() const { return v.data(); }
};

}  // namespace shim

template <typename S, int R, int C>
class Matrix;

template <typename M>
class CommaInit
{
public:
    CommaInit(M& m, const typename M::Scalar& first) : m_(m), k_(0) { put(first); }
    CommaInit& operator,(const typename M::Scalar& v)
    {
        put(v);
        return *this;
    }

private:
    void put(const typename M::Scalar& v)
    {
        // Comma initialisation fills row by row.
        const Index cols = m_.cols();
        m_(k_ / cols, k_ % cols) = v;
        ++k_;
    }
    M& m_;
    Index k_;
};

template <typename S, int R, int C>
class ColumnRef
{
public:
    ColumnRef(Matrix<S, R, C>& m, Index j) : m_(m), j_(j) {}
    template <typename V>
    ColumnRef& operator=(const V& v)
    {
        for (Index i = 0; i < m_.rows(); ++i)
            m_(i, j_) = v[i];
        return *this;
    }

private:
    Matrix<S, R, C>& m_;
    Index j_;
};

template <typename S, int R, int C>
class Matrix
{
public:
    using Scalar = S;
    using RealScalar = double;

    Matrix()
    {
        if constexpr (R != Dynamic && C != Dynamic)
            st_.a.fill(S(0));
    }
    explicit Matrix(Index n) { st_.resize(n, 1); }
    Matrix(Index r, Index c) { st_.resize(r, c); }

    static Matrix Zero(Index n)
    {
        Matrix m(n);
        return m;
    }
    static Matrix Zero(Index r, Index c)
    {
        Matrix m(r, c);
        return m;
    }
    static Matrix Zero() { return Matrix(); }
    static Matrix Identity()
    {
        Matrix m;
        for (Index i = 0; i < R && i < C; ++i)
            m(i, i) = S(1);
        return m;
    }

    Index rows() const { return st_.rows(); }
    Index cols() const { return st_.cols(); }
    Index size() const { return rows() * cols(); }
    S* data() { return st_.data(); }
    const S* data() const { return st_.data(); }

    S& operator[](Index i) { return st_.data()[i]; }
    const S& operator[](Index i) const { return st_.data()[i]; }
    S& operator()(Index i) { return st_.data()[i]; }
    const S& operator()(Index i) const { return st_.data()[i]; }
    // Column-major element storage.
    S& operator()(Index i, Index j) { return st_.data()[i + j * rows()]; }
    const S& operator()(Index i, Index j) const { return st_.data()[i + j * rows()]; }

    CommaInit<Matrix> operator<<(const S& v) { return CommaInit<Matrix>(*this, v); }

    ColumnRef<S, R, C> col(Index j) { return ColumnRef<S, R, C>(*this, j); }

    Matrix& operator+=(const Matrix& o)
    {
        check_same(o);
        for (Index i = 0; i < size(); ++i)
            (*this)[i] += o[i];
        return *this;
    }
    Matrix& operator-=(const Matrix& o)
    {
        check_same(o);
        for (Index i = 0; i < size(); ++i)
            (*this)[i] -= o[i];
        return *this;
    }

    S dot(const Matrix& o) const
    {
        check_same(o);
        S sum(0);
        for (Index i = 0; i < size(); ++i)
            sum += std::conj((*this)[i]) * o[i];
        return sum;
    }
    double squaredNorm() const
    {
        double sum = 0.0;
        for (Index i = 0; i < size(); ++i)
            sum += std::norm((*this)[i]);
        return sum;
    }
    double norm() const { return std::sqrt(squaredNorm()); }

    Matrix<S, C, R> adjoint() const
    {
        Matrix<S, C, R> out = make_sized<C, R>(cols(), rows());
        for (Index i = 0; i < rows(); ++i)
            for (Index j = 0; j < cols(); ++j)
                out(j, i) = std::conj((*this)(i, j));
        return out;
    }

    void check_same(const Matrix& o) const
    {
        if (o.rows() != rows() || o.cols() != cols())
            throw std::runtime_error("shim: dense size mismatch");
    }

    template <int R2, int C2>
    static Matrix<S, R2, C2> make_sized(Index r, Index c)
    {
        if constexpr (R2 != Dynamic && C2 != Dynamic)
            return Matrix<S, R2, C2>();
        else if constexpr (C2 == 1)
            return Matrix<S, R2, C2>(r);
        else
            return Matrix<S, R2, C2>(r, c);
    }

private:
    shim::Storage<S, R, C> st_;
};

template <typename S, int R, int C>
Matrix<S, R, C> operator+(Matrix<S, R, C> a, const Matrix<S, R, C>& b)
{
    a += b;
    return a;
}
template <typename S, int R, int C>
Matrix<S, R, C> operator-(Matrix<S, R, C> a, const Matrix<S, R, C>& b)
{
    a -= b;
    return a;
}
template <typename S, int R, int C>
Matrix<S, R, C> operator-(Matrix<S, R, C> a)
{
    for (Index i = 0; i < a.size(); ++i)
        a[i] = -a[i];
    return a;
}
template <typename S, int R, int C>
Matrix<S, R, C> operator*(double k, Matrix<S, R, C> a)
{
    for (Index i = 0; i < a.size(); ++i)
        a[i] = k * a[i];
    return a;
}
template <typename S, int R, int C>
Matrix<S, R, C> operator*(Matrix<S, R, C> a, double k)
{
    return k * a;
}
template <typename S, int R, int C>
Matrix<S, R, C> operator*(const std::complex<double>& k, Matrix<S, R, C> a)
{
    for (Index i = 0; i < a.size(); ++i)
        a[i] = k * a[i];
    return a;
}
template <typename S, int R, int C>
Matrix<S, R, C> operator*(Matrix<S, R, C> a, const std::complex<double>& k)
{
    return k * a;
}
template <typename S, int R, int C>
Matrix<S, R, C> operator/(Matrix<S, R, C> a, double k)
{
    for (Index i = 0; i < a.size(); ++i)
        a[i] = a[i] / k;
    return a;
}

// Dense matrix product (used for 2x2 spin matrices acting on 2-spinors).
template <typename S, int R, int K, int C>
Matrix<S, R, C> operator*(const Matrix<S, R, K>& a, const Matrix<S, K, C>& b)
{
    if (a.cols() != b.rows())
        throw std::runtime_error("shim: product size mismatch");
    Matrix<S, R, C> out = Matrix<S, R, K>::template make_sized<R, C>(a.rows(), b.cols());
    for (Index i = 0; i < a.rows(); ++i)
        for (Index j = 0; j < b.cols(); ++j)
        {
            S sum(0);
            for (Index k = 0; k < a.cols(); ++k)
                sum += a(i, k) * b(k, j);
            out(i, j) = sum;
        }
    return out;
}

using VectorXcd = Matrix<std::complex<double>, Dynamic, 1>;
using Vector2cd = Matrix<std::complex<double>, 2, 1>;
using Matrix2cd = Matrix<std::complex<double>, 2, 2>;
using MatrixXcd = Matrix<std::complex<double>, Dynamic, Dynamic>;

}  // namespace Eigen
