// Header-only stand-in for the subset of Eigen 3.4 that the reference's pressure-path sources
// use (amg.cpp, ldu_matrix.cpp, parallel_amg.cpp, mesh.cpp, mesh_builder.cpp, box_mesher.cpp,
// fv_geometry.cpp, flow_solver.cpp). TEST INFRASTRUCTURE ONLY: it lets those sources compile unchanged into the
// oracle's reference build (oracle/_ref) in an image without Eigen. Nothing in the product
// includes it.
//
// Arithmetic follows Eigen's published algorithms where they fix the result bits:
//   * dense reductions (sum, dot, squaredNorm, norm) in the order of Eigen's SSE2 reduction
//     (packets of two doubles; two packet accumulators for dynamic sizes, a packet tree for fixed
//     sizes, scalar tail last), which is what a default x86-64 build of the reference uses;
//   * element-wise operations one IEEE operation per element (no FMA contraction);
//   * sparse x sparse products in the order of Eigen's conservative_sparse_sparse_product
//     (row i of A*B accumulates A(i,k)*B(k,:) for k ascending over row i of A, columns of B(k,:)
//     in order, the first contribution assigning), with sorted inner indices;
//   * sparse x dense products row by row, each row summed from zero in storage order;
//   * setFromTriplets: duplicates summed in triplet order, inner indices sorted;
//   * prune(reference, eps): keeps entries with |v| > |reference| * eps (prune(0) drops exact
//     zeros); sparse + / - over the union of the two patterns, a missing side read as zero.
// Where this stand-in does NOT follow Eigen bit for bit:
//   * SimplicialLDLT factorises in the natural order (Eigen applies an AMD permutation first),
//     so coarse solves and the coarse inverse agree with Eigen's to round-off, not bitwise;
//   * small fixed-size matrix products (3x3 * 3x1, outer products) sum left to right;
//   * CompleteOrthogonalDecomposition, ConjugateGradient and IncompleteCholesky are declared so
//     that the sources compile; calling them throws std::logic_error (the pressure path with a
//     pinned reference cell never reaches them).
#pragma once

#include <algorithm>
#include <array>
#include <cassert>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <stdexcept>
#include <type_traits>
#include <utility>
#include <vector>

namespace Eigen {

using Index = std::ptrdiff_t;
inline constexpr int Dynamic = -1;
enum StorageOptions { ColMajor = 0, RowMajor = 1, AutoAlign = 0, DontAlign = 2 };
enum UpLoType { Lower = 1, Upper = 2 };
enum ComputationInfo { Success = 0, NumericalIssue = 1, NoConvergence = 2, InvalidInput = 3 };

namespace standin {

// Sum of e(0..n-1) in the order of Eigen's vectorised reduction of a dynamic-size expression
// with packets of two doubles and an aligned start: two packet accumulators over blocks of
// four, combined, one more packet if two elements remain, the horizontal add, then the last
// element of an odd size.
template <class E> double redux_dynamic(Index n, const E& e) {
    if (n <= 0) return 0.0;
    if (n < 2) return e(0);
    const Index aligned = (n / 2) * 2, aligned2 = (n / 4) * 4;
    double p0a = e(0), p0b = e(1);
    if (aligned > 2) {
        double p1a = e(2), p1b = e(3);
        for (Index i = 4; i < aligned2; i += 4) {
            p0a = p0a + e(i);
            p0b = p0b + e(i + 1);
            p1a = p1a + e(i + 2);
            p1b = p1b + e(i + 3);
        }
        p0a = p0a + p1a;
        p0b = p0b + p1b;
        if (aligned > aligned2) {
            p0a = p0a + e(aligned2);
            p0b = p0b + e(aligned2 + 1);
        }
    }
    double r = p0a + p0b;
    for (Index i = aligned; i < n; ++i) r = r + e(i);
    return r;
}

// Packet tree of Eigen's fully unrolled reduction over `len` packets of two starting at
// packet `start`; returns the two lanes.
template <class E> std::pair<double, double> redux_packets(Index start, Index len, const E& e) {
    if (len == 1) return {e(2 * start), e(2 * start + 1)};
    const Index half = len / 2;
    const auto a = redux_packets(start, half, e);
    const auto b = redux_packets(start + half, len - half, e);
    return {a.first + b.first, a.second + b.second};
}

// Scalar tree of Eigen's unrolled non-vectorised reduction: halves recursively.
template <class E> double redux_scalar_tree(Index start, Index len, const E& e) {
    if (len == 1) return e(start);
    const Index half = len / 2;
    return redux_scalar_tree(start, half, e) + redux_scalar_tree(start + half, len - half, e);
}

// Fixed-size reduction (complete unrolling): packets of two, then the scalar tail.
template <class E> double redux_fixed(Index n, const E& e) {
    const Index vec = (n / 2) * 2;
    if (vec == 0) return redux_scalar_tree(0, n, e);
    const auto p = redux_packets(0, vec / 2, e);
    double r = p.first + p.second;
    if (vec != n) r = r + redux_scalar_tree(vec, n - vec, e);
    return r;
}

template <typename S, int R, int C, bool Fixed = (R > 0 && C > 0)> struct DenseStorage;

template <typename S, int R, int C> struct DenseStorage<S, R, C, true> {
    S d[R * C] = {};
    static constexpr Index rows() { return R; }
    static constexpr Index cols() { return C; }
    void resize(Index r, Index c) {
        if (r != R || c != C) throw std::logic_error("Eigen stand-in: fixed-size resize");
    }
    S* data() { return d; }
    const S* data() const { return d; }
};

template <typename S, int R, int C> struct DenseStorage<S, R, C, false> {
    std::vector<S> d;
    Index r = R > 0 ? R : 0, c = C > 0 ? C : 0;
    Index rows() const { return r; }
    Index cols() const { return c; }
    void resize(Index rr, Index cc) {
        r = rr;
        c = cc;
        d.assign(static_cast<std::size_t>(rr * cc), S(0));
    }
    S* data() { return d.data(); }
    const S* data() const { return d.data(); }
};

} // namespace standin

template <typename S, int R, int C,
          int Opt = ((R == 1 && C != 1) ? RowMajor : ColMajor), int MR = R, int MC = C>
class Matrix;

template <typename M> class Map;
template <typename V> class DiagonalWrapper;
template <typename S, int Opt = ColMajor, typename I = int> class SparseMatrix;

template <typename T> struct is_dense : std::false_type {};
template <typename S, int R, int C, int O, int MR, int MC>
struct is_dense<Matrix<S, R, C, O, MR, MC>> : std::true_type {};
template <typename M> struct is_dense<Map<M>> : std::true_type {};
template <typename T> inline constexpr bool is_dense_v = is_dense<std::remove_cv_t<std::remove_reference_t<T>>>::value;

template <typename S, int R, int C, int Opt, int MR, int MC>
class Matrix : public standin::DenseStorage<S, R, C> {
    using Base = standin::DenseStorage<S, R, C>;

public:
    using Scalar = S;
    using PlainObject = Matrix;
    static constexpr int RowsAtCompileTime = R;
    static constexpr int ColsAtCompileTime = C;
    static constexpr int SizeAtCompileTime = (R > 0 && C > 0) ? R * C : Dynamic;
    static constexpr bool IsRowMajor = (Opt & RowMajor) != 0;
    static constexpr bool kFixed = R > 0 && C > 0;

    Matrix() {
        if constexpr (!kFixed) Base::resize(R > 0 ? R : 0, C > 0 ? C : 0);
    }
    // Vector size (or rows, cols) constructors of dynamic matrices; (x, y, z) of 3-vectors.
    template <typename T, typename = std::enable_if_t<std::is_integral_v<T> && !kFixed>>
    explicit Matrix(T n) {
        if constexpr (C == 1) Base::resize(static_cast<Index>(n), 1);
        else if constexpr (R == 1) Base::resize(1, static_cast<Index>(n));
        else throw std::logic_error("Eigen stand-in: size constructor of a matrix");
    }
    template <typename T1, typename T2,
              typename = std::enable_if_t<std::is_integral_v<T1> && std::is_integral_v<T2>>>
    Matrix(T1 r, T2 c) {
        Base::resize(static_cast<Index>(r), static_cast<Index>(c));
    }
    Matrix(double x, double y, double z) {
        static_assert(R * C == 3 || !kFixed, "3-coefficient constructor");
        if constexpr (!kFixed) Base::resize(C == 1 ? 3 : 1, C == 1 ? 1 : 3);
        Base::data()[0] = x;
        Base::data()[1] = y;
        Base::data()[2] = z;
    }
    Matrix(const Matrix&) = default;
    Matrix(Matrix&&) = default;
    Matrix& operator=(const Matrix&) = default;
    Matrix& operator=(Matrix&&) = default;
    // From another dense object (other storage order, a Map): coefficient-wise copy.
    template <typename Other, typename = std::enable_if_t<is_dense_v<Other> && !std::is_same_v<Other, Matrix>>>
    Matrix(const Other& o) {
        Base::resize(o.rows(), o.cols());
        for (Index i = 0; i < o.rows(); ++i)
            for (Index j = 0; j < o.cols(); ++j) coeffRef(i, j) = o.coeff(i, j);
    }
    // Dense copy of a sparse matrix.
    template <typename S2, int O2, typename I2> explicit Matrix(const SparseMatrix<S2, O2, I2>& a);
    template <typename Other, typename = std::enable_if_t<is_dense_v<Other> && !std::is_same_v<Other, Matrix>>>
    Matrix& operator=(const Other& o) {
        Matrix t(o);
        *this = std::move(t);
        return *this;
    }

    using Base::cols;
    using Base::data;
    using Base::rows;
    Index size() const { return rows() * cols(); }
    Index outerStride() const { return IsRowMajor ? cols() : rows(); }

    void resize(Index n) {
        if constexpr (C == 1) Base::resize(n, 1);
        else Base::resize(1, n);
    }
    void resize(Index r, Index c) { Base::resize(r, c); }
    void setZero() { std::fill(data(), data() + size(), S(0)); }

    Index lin(Index i, Index j) const { return IsRowMajor ? i * cols() + j : i + j * rows(); }
    S& coeffRef(Index i, Index j) { return data()[lin(i, j)]; }
    const S& coeff(Index i, Index j) const { return data()[lin(i, j)]; }
    S& coeffRef(Index i) { return data()[i]; }
    const S& coeff(Index i) const { return data()[i]; }
    S& operator()(Index i, Index j) { return coeffRef(i, j); }
    const S& operator()(Index i, Index j) const { return coeff(i, j); }
    S& operator()(Index i) { return data()[i]; }
    const S& operator()(Index i) const { return data()[i]; }
    S& operator[](Index i) { return data()[i]; }
    const S& operator[](Index i) const { return data()[i]; }
    S& x() { return data()[0]; }
    S& y() { return data()[1]; }
    S& z() { return data()[2]; }
    const S& x() const { return data()[0]; }
    const S& y() const { return data()[1]; }
    const S& z() const { return data()[2]; }

    static Matrix Constant(S v) {
        Matrix m;
        std::fill(m.data(), m.data() + m.size(), v);
        return m;
    }
    static Matrix Constant(Index n, S v) {
        Matrix m(n);
        std::fill(m.data(), m.data() + m.size(), v);
        return m;
    }
    static Matrix Constant(Index r, Index c, S v) {
        Matrix m(r, c);
        std::fill(m.data(), m.data() + m.size(), v);
        return m;
    }
    static Matrix Zero() { return Constant(S(0)); }
    static Matrix Zero(Index n) { return Constant(n, S(0)); }
    static Matrix Zero(Index r, Index c) { return Constant(r, c, S(0)); }
    static Matrix Ones() { return Constant(S(1)); }
    static Matrix Ones(Index n) { return Constant(n, S(1)); }
    static Matrix Identity() {
        Matrix m = Zero();
        for (Index i = 0; i < std::min(m.rows(), m.cols()); ++i) m(i, i) = S(1);
        return m;
    }

    // Reductions in Eigen's vectorised order (dynamic) or unrolled packet order (fixed).
    template <class E> S reduce(const E& e) const {
        if constexpr (kFixed) return standin::redux_fixed(size(), e);
        else return standin::redux_dynamic(size(), e);
    }
    S sum() const {
        return reduce([&](Index i) { return data()[i]; });
    }
    template <typename Other> S dot(const Other& o) const {
        return reduce([&](Index i) { return data()[i] * o.coeff(i); });
    }
    S squaredNorm() const {
        return reduce([&](Index i) { return data()[i] * data()[i]; });
    }
    S norm() const { return std::sqrt(squaredNorm()); }
    S minCoeff() const {
        S m = data()[0];
        for (Index i = 1; i < size(); ++i) m = std::min(m, data()[i]);
        return m;
    }
    S maxCoeff() const {
        S m = data()[0];
        for (Index i = 1; i < size(); ++i) m = std::max(m, data()[i]);
        return m;
    }
    Matrix normalized() const {
        Matrix r = *this;
        const S n = norm();
        if (n > S(0))
            for (Index i = 0; i < size(); ++i) r.data()[i] = r.data()[i] / n;
        return r;
    }
    template <typename Other> Matrix cwiseProduct(const Other& o) const {
        Matrix r = *this;
        for (Index i = 0; i < size(); ++i) r.data()[i] = data()[i] * o.coeff(i);
        return r;
    }
    Matrix cwiseAbs() const {
        Matrix r = *this;
        for (Index i = 0; i < size(); ++i) r.data()[i] = std::abs(data()[i]);
        return r;
    }
    // element-wise min / max (std::min / std::max per element, Eigen's default NaN handling)
    template <typename Other> Matrix cwiseMin(const Other& o) const {
        Matrix r = *this;
        for (Index i = 0; i < size(); ++i) r.data()[i] = std::min(data()[i], o.coeff(i));
        return r;
    }
    template <typename Other> Matrix cwiseMax(const Other& o) const {
        Matrix r = *this;
        for (Index i = 0; i < size(); ++i) r.data()[i] = std::max(data()[i], o.coeff(i));
        return r;
    }
    // mean = sum() / size(), the sum in the reduction order above
    S mean() const { return sum() / static_cast<S>(size()); }
    template <typename F> Matrix unaryExpr(F f) const {
        Matrix r = *this;
        for (Index i = 0; i < size(); ++i) r.data()[i] = f(data()[i]);
        return r;
    }
    Matrix cross(const Matrix& b) const {
        const Matrix& a = *this;
        return Matrix(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
    }
    Matrix<S, C, R> transpose() const {
        Matrix<S, C, R> t;
        if constexpr (!Matrix<S, C, R>::kFixed) t.resize(cols(), rows());
        for (Index i = 0; i < rows(); ++i)
            for (Index j = 0; j < cols(); ++j) t.coeffRef(j, i) = coeff(i, j);
        return t;
    }
    Matrix head(Index n) const {
        Matrix r(n);
        for (Index i = 0; i < n; ++i) r[i] = data()[i];
        return r;
    }
    DiagonalWrapper<Matrix> asDiagonal() const;

    // Column proxy: inv.col(j) = vector.
    struct ColRef {
        Matrix* m;
        Index j;
        template <typename V> ColRef& operator=(const V& v) {
            for (Index i = 0; i < m->rows(); ++i) m->coeffRef(i, j) = v.coeff(i);
            return *this;
        }
        Index size() const { return m->rows(); }
        S coeff(Index i) const { return m->coeff(i, j); }
    };
    ColRef col(Index j) { return ColRef{this, j}; }
    Matrix<S, R, 1> col(Index j) const {
        Matrix<S, R, 1> v;
        if constexpr (!Matrix<S, R, 1>::kFixed) v.resize(rows());
        for (Index i = 0; i < rows(); ++i) v[i] = coeff(i, j);
        return v;
    }
    const Matrix& eval() const { return *this; }

    Matrix inverse() const;

    template <typename Other> Matrix& operator+=(const Other& o) {
        for (Index i = 0; i < rows(); ++i)
            for (Index j = 0; j < cols(); ++j) coeffRef(i, j) = coeff(i, j) + o.coeff(i, j);
        return *this;
    }
    template <typename Other> Matrix& operator-=(const Other& o) {
        for (Index i = 0; i < rows(); ++i)
            for (Index j = 0; j < cols(); ++j) coeffRef(i, j) = coeff(i, j) - o.coeff(i, j);
        return *this;
    }
    Matrix& operator*=(S s) {
        for (Index i = 0; i < size(); ++i) data()[i] = data()[i] * s;
        return *this;
    }
    Matrix& operator/=(S s) {
        for (Index i = 0; i < size(); ++i) data()[i] = data()[i] / s;
        return *this;
    }
    Matrix operator-() const {
        Matrix r = *this;
        for (Index i = 0; i < size(); ++i) r.data()[i] = -data()[i];
        return r;
    }

    class CompleteOrthogonalDecomposition {
    public:
        Matrix pseudoInverse() const {
            throw std::logic_error("Eigen stand-in: CompleteOrthogonalDecomposition is not provided");
        }
    };
    CompleteOrthogonalDecomposition completeOrthogonalDecomposition() const { return {}; }
};

// Map: Map<const T> is a read-only copy of the mapped coefficients (reads only); Map<T> writes
// through to the caller's memory.
template <typename M> class Map;

template <typename S, int R, int C, int O, int MR, int MC>
class Map<const Matrix<S, R, C, O, MR, MC>> : public Matrix<S, R, C, O, MR, MC> {
public:
    using PlainObject = Matrix<S, R, C, O, MR, MC>;
    Map(const S* p, Index n) : PlainObject(n) { std::copy(p, p + n, this->data()); }
    Map(const S* p, Index r, Index c) : PlainObject(r, c) { std::copy(p, p + r * c, this->data()); }
};

template <typename S, int R, int C, int O, int MR, int MC> class Map<Matrix<S, R, C, O, MR, MC>> {
public:
    using PlainObject = Matrix<S, R, C, O, MR, MC>;
    using Scalar = S;
    Map(S* p, Index n) : p_(p), n_(n) {}
    Index size() const { return n_; }
    Index rows() const { return C == 1 ? n_ : 1; }
    Index cols() const { return C == 1 ? 1 : n_; }
    S coeff(Index i) const { return p_[i]; }
    S coeff(Index i, Index j) const { return p_[i + j]; }
    S& operator[](Index i) { return p_[i]; }
    const S& operator[](Index i) const { return p_[i]; }
    S* data() { return p_; }
    const S* data() const { return p_; }
    template <typename Other> Map& operator=(const Other& o) {
        for (Index i = 0; i < n_; ++i) p_[i] = o.coeff(i);
        return *this;
    }
    S norm() const { return PlainObject(*this).norm(); }
    S squaredNorm() const { return PlainObject(*this).squaredNorm(); }

private:
    S* p_;
    Index n_;
};

template <typename V> class DiagonalWrapper {
public:
    explicit DiagonalWrapper(const V& v) : v(v) {}
    const V& v;
};

template <typename S, int R, int C, int O, int MR, int MC>
DiagonalWrapper<Matrix<S, R, C, O, MR, MC>> Matrix<S, R, C, O, MR, MC>::asDiagonal() const {
    return DiagonalWrapper<Matrix>(*this);
}

// 3x3 inverse by cofactors: each cofactor as the difference of two products, the determinant
// as the reduction of column 0 times its cofactors, and the inverse as the transposed cofactor
// matrix times 1/det.
template <typename S, int R, int C, int O, int MR, int MC>
Matrix<S, R, C, O, MR, MC> Matrix<S, R, C, O, MR, MC>::inverse() const {
    if constexpr (R == 3 && C == 3) {
        const Matrix& m = *this;
        auto cof = [&](int i, int j) {
            const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            return m(i1, j1) * m(i2, j2) - m(i1, j2) * m(i2, j1);
        };
        const Matrix<S, 3, 1> c0(cof(0, 0), cof(1, 0), cof(2, 0));
        const S det = c0.cwiseProduct(m.col(0)).sum();
        const S inv = S(1) / det;
        Matrix r;
        r(1, 2) = cof(2, 1) * inv;
        r(2, 1) = cof(1, 2) * inv;
        r(2, 2) = cof(2, 2) * inv;
        r(1, 0) = cof(0, 1) * inv;
        r(1, 1) = cof(1, 1) * inv;
        r(2, 0) = cof(0, 2) * inv;
        r(0, 0) = c0[0] * inv;
        r(0, 1) = c0[1] * inv;
        r(0, 2) = c0[2] * inv;
        return r;
    } else {
        throw std::logic_error("Eigen stand-in: inverse() is provided for 3x3 matrices only");
    }
}

// ---- dense arithmetic (results are plain matrices) ----------------------------------------

template <typename A, typename B, typename = std::enable_if_t<is_dense_v<A> && is_dense_v<B>>>
typename A::PlainObject operator+(const A& a, const B& b) {
    typename A::PlainObject r(a);
    for (Index i = 0; i < r.rows(); ++i)
        for (Index j = 0; j < r.cols(); ++j) r.coeffRef(i, j) = a.coeff(i, j) + b.coeff(i, j);
    return r;
}
template <typename A, typename B, typename = std::enable_if_t<is_dense_v<A> && is_dense_v<B>>>
typename A::PlainObject operator-(const A& a, const B& b) {
    typename A::PlainObject r(a);
    for (Index i = 0; i < r.rows(); ++i)
        for (Index j = 0; j < r.cols(); ++j) r.coeffRef(i, j) = a.coeff(i, j) - b.coeff(i, j);
    return r;
}
template <typename A, typename = std::enable_if_t<is_dense_v<A>>>
typename A::PlainObject operator*(const A& a, double s) {
    typename A::PlainObject r(a);
    for (Index i = 0; i < r.size(); ++i) r.data()[i] = r.data()[i] * s;
    return r;
}
template <typename A, typename = std::enable_if_t<is_dense_v<A>>>
typename A::PlainObject operator*(double s, const A& a) {
    typename A::PlainObject r(a);
    for (Index i = 0; i < r.size(); ++i) r.data()[i] = s * r.data()[i];
    return r;
}
template <typename A, typename = std::enable_if_t<is_dense_v<A>>>
typename A::PlainObject operator/(const A& a, double s) {
    typename A::PlainObject r(a);
    for (Index i = 0; i < r.size(); ++i) r.data()[i] = r.data()[i] / s;
    return r;
}
// Small dense product (left-to-right sums; not Eigen's order for fixed sizes).
template <typename S, int R1, int C1, int O1, int MR1, int MC1, int R2, int C2, int O2, int MR2, int MC2>
Matrix<S, R1, C2> operator*(const Matrix<S, R1, C1, O1, MR1, MC1>& a, const Matrix<S, R2, C2, O2, MR2, MC2>& b) {
    Matrix<S, R1, C2> r;
    if constexpr (!Matrix<S, R1, C2>::kFixed) r.resize(a.rows(), b.cols());
    for (Index i = 0; i < a.rows(); ++i)
        for (Index j = 0; j < b.cols(); ++j) {
            S s = a.coeff(i, 0) * b.coeff(0, j);
            for (Index k = 1; k < a.cols(); ++k) s = s + a.coeff(i, k) * b.coeff(k, j);
            r.coeffRef(i, j) = s;
        }
    return r;
}

using MatrixXd = Matrix<double, Dynamic, Dynamic>;
using VectorXd = Matrix<double, Dynamic, 1>;
using Vector3d = Matrix<double, 3, 1>;
using Matrix3d = Matrix<double, 3, 3>;

// ---- sparse ---------------------------------------------------------------------------------

template <typename S, typename I = int> class Triplet {
public:
    Triplet() = default;
    Triplet(I r, I c, S v = S(0)) : r_(r), c_(c), v_(v) {}
    I row() const { return r_; }
    I col() const { return c_; }
    S value() const { return v_; }

private:
    I r_ = 0, c_ = 0;
    S v_ = S(0);
};

template <typename M> class SparseTranspose {
public:
    explicit SparseTranspose(const M& m) : m(m) {}
    const M& m;
};

template <typename S, int Opt, typename I> class SparseMatrix {
public:
    using Scalar = S;
    using StorageIndex = I;
    static constexpr bool IsRowMajor = (Opt & RowMajor) != 0;

    SparseMatrix() : outer_(1, 0) {}
    SparseMatrix(Index rows, Index cols) { resize(rows, cols); }
    SparseMatrix(const SparseMatrix&) = default;
    SparseMatrix(SparseMatrix&&) = default;
    SparseMatrix& operator=(const SparseMatrix&) = default;
    SparseMatrix& operator=(SparseMatrix&&) = default;
    // Storage-order conversion: counting sort by the other index (inner indices ascending).
    template <int O2, typename = std::enable_if_t<O2 != Opt>>
    SparseMatrix(const SparseMatrix<S, O2, I>& o) {
        resize(o.rows(), o.cols());
        transposed_copy(o.outerSize(), o.outerIndexPtr(), o.innerIndexPtr(), o.valuePtr(), o.nonZeros());
    }
    // From a transpose: same arrays if the storage orders differ, a counting sort otherwise.
    template <int O2> SparseMatrix(const SparseTranspose<SparseMatrix<S, O2, I>>& t) {
        const auto& o = t.m;
        resize(o.cols(), o.rows());
        if constexpr (O2 != Opt) {
            outer_.assign(o.outerIndexPtr(), o.outerIndexPtr() + o.outerSize() + 1);
            inner_.assign(o.innerIndexPtr(), o.innerIndexPtr() + o.nonZeros());
            val_.assign(o.valuePtr(), o.valuePtr() + o.nonZeros());
        } else {
            transposed_copy(o.outerSize(), o.outerIndexPtr(), o.innerIndexPtr(), o.valuePtr(), o.nonZeros());
        }
    }

    void resize(Index rows, Index cols) {
        rows_ = rows;
        cols_ = cols;
        outer_.assign(static_cast<std::size_t>(outerSize() + 1), I(0));
        inner_.clear();
        val_.clear();
    }
    void setZero() { resize(rows_, cols_); }
    void reserve(Index n) {
        inner_.reserve(static_cast<std::size_t>(n));
        val_.reserve(static_cast<std::size_t>(n));
    }
    Index rows() const { return rows_; }
    Index cols() const { return cols_; }
    Index outerSize() const { return IsRowMajor ? rows_ : cols_; }
    Index innerSize() const { return IsRowMajor ? cols_ : rows_; }
    Index nonZeros() const { return static_cast<Index>(val_.size()); }
    S* valuePtr() { return val_.data(); }
    const S* valuePtr() const { return val_.data(); }
    I* innerIndexPtr() { return inner_.data(); }
    const I* innerIndexPtr() const { return inner_.data(); }
    I* outerIndexPtr() { return outer_.data(); }
    const I* outerIndexPtr() const { return outer_.data(); }
    void makeCompressed() {}
    bool isCompressed() const { return true; }

    S coeff(Index r, Index c) const {
        const Index o = IsRowMajor ? r : c, in = IsRowMajor ? c : r;
        for (I k = outer_[o]; k < outer_[o + 1]; ++k)
            if (inner_[k] == in) return val_[k];
        return S(0);
    }

    class InnerIterator {
    public:
        InnerIterator(const SparseMatrix& m, Index outer)
            : m_(&m), o_(outer), k_(m.outer_[outer]), end_(m.outer_[outer + 1]) {}
        explicit operator bool() const { return k_ < end_; }
        InnerIterator& operator++() {
            ++k_;
            return *this;
        }
        S value() const { return m_->val_[k_]; }
        Index index() const { return m_->inner_[k_]; }
        Index col() const { return IsRowMajor ? index() : o_; }
        Index row() const { return IsRowMajor ? o_ : index(); }
        Index outer() const { return o_; }

    private:
        const SparseMatrix* m_;
        Index o_;
        I k_, end_;
    };

    // Duplicates summed in triplet order; inner indices sorted.
    template <typename It> void setFromTriplets(It b, It e) {
        std::vector<I> cnt(static_cast<std::size_t>(outerSize() + 1), I(0));
        std::vector<std::size_t> order;
        for (It it = b; it != e; ++it) ++cnt[static_cast<std::size_t>(outer_of(it->row(), it->col())) + 1];
        std::vector<I> start(cnt.size(), I(0));
        for (std::size_t o = 1; o < cnt.size(); ++o) start[o] = start[o - 1] + cnt[o];
        const std::size_t ntrip = static_cast<std::size_t>(start.back());
        std::vector<I> pos(start.begin(), start.end() - 1);
        std::vector<I> tin(ntrip);
        std::vector<S> tval(ntrip);
        for (It it = b; it != e; ++it) {
            const Index o = outer_of(it->row(), it->col());
            const I p = pos[static_cast<std::size_t>(o)]++;
            tin[static_cast<std::size_t>(p)] = static_cast<I>(inner_of(it->row(), it->col()));
            tval[static_cast<std::size_t>(p)] = it->value();
        }
        // per outer vector: stable sort by inner index, then collapse duplicates in order
        outer_.assign(static_cast<std::size_t>(outerSize() + 1), I(0));
        inner_.clear();
        val_.clear();
        std::vector<std::size_t> idx;
        for (Index o = 0; o < outerSize(); ++o) {
            idx.clear();
            for (I k = start[static_cast<std::size_t>(o)]; k < start[static_cast<std::size_t>(o) + 1]; ++k)
                idx.push_back(static_cast<std::size_t>(k));
            std::stable_sort(idx.begin(), idx.end(), [&](std::size_t a, std::size_t c) { return tin[a] < tin[c]; });
            for (std::size_t q = 0; q < idx.size(); ++q) {
                const std::size_t k = idx[q];
                if (q > 0 && tin[k] == tin[idx[q - 1]]) {
                    val_.back() = val_.back() + tval[k];
                } else {
                    inner_.push_back(tin[k]);
                    val_.push_back(tval[k]);
                }
            }
            outer_[static_cast<std::size_t>(o) + 1] = static_cast<I>(val_.size());
        }
    }

    void prune(const S& reference, double epsilon = 1e-12) {
        const double bound = std::abs(reference) * epsilon;
        std::size_t w = 0;
        I start = 0;
        for (Index o = 0; o < outerSize(); ++o) {
            const I end = outer_[static_cast<std::size_t>(o) + 1];
            for (I k = start; k < end; ++k) {
                if (!(std::abs(val_[static_cast<std::size_t>(k)]) <= bound)) {
                    inner_[w] = inner_[static_cast<std::size_t>(k)];
                    val_[w] = val_[static_cast<std::size_t>(k)];
                    ++w;
                }
            }
            start = end;
            outer_[static_cast<std::size_t>(o) + 1] = static_cast<I>(w);
        }
        inner_.resize(w);
        val_.resize(w);
    }

    SparseTranspose<SparseMatrix> transpose() const { return SparseTranspose<SparseMatrix>(*this); }

    // Leading rows / columns as a new matrix (the distributed paths use them).
    SparseMatrix topRows(Index n) const { return block_of(n, cols_); }
    SparseMatrix leftCols(Index n) const { return block_of(rows_, n); }
    SparseMatrix block_of(Index nr, Index nc) const {
        SparseMatrix r(nr, nc);
        for (Index o = 0; o < r.outerSize(); ++o) {
            for (I k = outer_[o]; k < outer_[o + 1]; ++k)
                if (inner_[k] < r.innerSize()) {
                    r.inner_.push_back(inner_[k]);
                    r.val_.push_back(val_[k]);
                }
            r.outer_[static_cast<std::size_t>(o) + 1] = static_cast<I>(r.val_.size());
        }
        return r;
    }

    // internal access for the free operators
    Index rows_ = 0, cols_ = 0;
    std::vector<I> outer_, inner_;
    std::vector<S> val_;

private:
    Index outer_of(Index r, Index c) const { return IsRowMajor ? r : c; }
    Index inner_of(Index r, Index c) const { return IsRowMajor ? c : r; }
    void transposed_copy(Index src_outer, const I* so, const I* si, const S* sv, Index nnz) {
        outer_.assign(static_cast<std::size_t>(outerSize() + 1), I(0));
        for (Index k = 0; k < nnz; ++k) ++outer_[static_cast<std::size_t>(si[k]) + 1];
        for (Index o = 0; o < outerSize(); ++o) outer_[o + 1] += outer_[o];
        std::vector<I> pos(outer_.begin(), outer_.end() - 1);
        inner_.assign(static_cast<std::size_t>(nnz), I(0));
        val_.assign(static_cast<std::size_t>(nnz), S(0));
        for (Index j = 0; j < src_outer; ++j)
            for (I k = so[j]; k < so[j + 1]; ++k) {
                const I p = pos[static_cast<std::size_t>(si[k])]++;
                inner_[static_cast<std::size_t>(p)] = static_cast<I>(j);
                val_[static_cast<std::size_t>(p)] = sv[k];
            }
    }
};

namespace standin {

// Gustavson product over outer vectors: for each outer vector of X, for each of its entries
// (k, y), for each entry (i, x) of outer vector k of Y: acc[i] = x*y on first touch, else
// acc[i] += x*y. Row-major C = A B takes (X, Y) = (A, B); column-major takes (B, A).
template <typename S, int O, typename I>
SparseMatrix<S, O, I> gustavson(const SparseMatrix<S, O, I>& X, const SparseMatrix<S, O, I>& Y, Index rows,
                                Index cols) {
    SparseMatrix<S, O, I> r(rows, cols);
    const Index inner = SparseMatrix<S, O, I>::IsRowMajor ? cols : rows;
    std::vector<char> mask(static_cast<std::size_t>(inner), 0);
    std::vector<S> acc(static_cast<std::size_t>(inner), S(0));
    std::vector<I> touched;
    for (Index o = 0; o < X.outerSize(); ++o) {
        touched.clear();
        for (I kx = X.outer_[o]; kx < X.outer_[o + 1]; ++kx) {
            const I k = X.inner_[static_cast<std::size_t>(kx)];
            const S y = X.val_[static_cast<std::size_t>(kx)];
            for (I ky = Y.outer_[k]; ky < Y.outer_[k + 1]; ++ky) {
                const I i = Y.inner_[static_cast<std::size_t>(ky)];
                const S x = Y.val_[static_cast<std::size_t>(ky)];
                if (!mask[static_cast<std::size_t>(i)]) {
                    mask[static_cast<std::size_t>(i)] = 1;
                    acc[static_cast<std::size_t>(i)] = x * y;
                    touched.push_back(i);
                } else {
                    acc[static_cast<std::size_t>(i)] += x * y;
                }
            }
        }
        std::sort(touched.begin(), touched.end());
        for (const I i : touched) {
            r.inner_.push_back(i);
            r.val_.push_back(acc[static_cast<std::size_t>(i)]);
            mask[static_cast<std::size_t>(i)] = 0;
        }
        r.outer_[static_cast<std::size_t>(o) + 1] = static_cast<I>(r.val_.size());
    }
    return r;
}

template <typename S, int O, typename I, typename F>
SparseMatrix<S, O, I> union_op(const SparseMatrix<S, O, I>& a, const SparseMatrix<S, O, I>& b, F f) {
    SparseMatrix<S, O, I> r(a.rows(), a.cols());
    for (Index o = 0; o < a.outerSize(); ++o) {
        I ka = a.outer_[o], kb = b.outer_[o];
        const I ea = a.outer_[o + 1], eb = b.outer_[o + 1];
        while (ka < ea || kb < eb) {
            if (ka < ea && kb < eb && a.inner_[ka] == b.inner_[kb]) {
                r.inner_.push_back(a.inner_[ka]);
                r.val_.push_back(f(a.val_[ka], b.val_[kb]));
                ++ka;
                ++kb;
            } else if (ka < ea && (kb >= eb || a.inner_[ka] < b.inner_[kb])) {
                r.inner_.push_back(a.inner_[ka]);
                r.val_.push_back(f(a.val_[ka], S(0)));
                ++ka;
            } else {
                r.inner_.push_back(b.inner_[kb]);
                r.val_.push_back(f(S(0), b.val_[kb]));
                ++kb;
            }
        }
        r.outer_[static_cast<std::size_t>(o) + 1] = static_cast<I>(r.val_.size());
    }
    return r;
}

} // namespace standin

template <typename S, int O, typename I>
SparseMatrix<S, O, I> operator*(const SparseMatrix<S, O, I>& a, const SparseMatrix<S, O, I>& b) {
    if (a.cols() != b.rows()) throw std::invalid_argument("Eigen stand-in: product size mismatch");
    if constexpr (SparseMatrix<S, O, I>::IsRowMajor) return standin::gustavson(a, b, a.rows(), b.cols());
    else return standin::gustavson(b, a, a.rows(), b.cols());
}

template <typename S, int O, typename I>
SparseMatrix<S, O, I> operator+(const SparseMatrix<S, O, I>& a, const SparseMatrix<S, O, I>& b) {
    return standin::union_op(a, b, [](S x, S y) { return x + y; });
}
template <typename S, int O, typename I>
SparseMatrix<S, O, I> operator-(const SparseMatrix<S, O, I>& a, const SparseMatrix<S, O, I>& b) {
    return standin::union_op(a, b, [](S x, S y) { return x - y; });
}
template <typename S, int O, typename I>
SparseMatrix<S, O, I> operator*(double s, const SparseMatrix<S, O, I>& a) {
    SparseMatrix<S, O, I> r = a;
    for (auto& v : r.val_) v = s * v;
    return r;
}
template <typename S, int O, typename I>
SparseMatrix<S, O, I> operator*(const SparseMatrix<S, O, I>& a, double s) {
    SparseMatrix<S, O, I> r = a;
    for (auto& v : r.val_) v = v * s;
    return r;
}

// diag(d) * A: every stored entry of row i times d[i] (the pattern is kept).
template <typename V, typename S, int O, typename I>
SparseMatrix<S, O, I> operator*(const DiagonalWrapper<V>& d, const SparseMatrix<S, O, I>& a) {
    SparseMatrix<S, O, I> r = a;
    for (Index o = 0; o < a.outerSize(); ++o)
        for (I k = a.outer_[o]; k < a.outer_[o + 1]; ++k) {
            const Index row = SparseMatrix<S, O, I>::IsRowMajor ? o : a.inner_[k];
            r.val_[k] = d.v.coeff(row) * a.val_[k];
        }
    return r;
}

// A * x for a dense vector x: row-major rows summed from zero in storage order; column-major
// accumulates column j times x[j] into the result.
template <typename S, int O, typename I, typename V, typename = std::enable_if_t<is_dense_v<V>>>
Matrix<S, Dynamic, 1> operator*(const SparseMatrix<S, O, I>& a, const V& x) {
    Matrix<S, Dynamic, 1> r = Matrix<S, Dynamic, 1>::Zero(a.rows());
    if constexpr (SparseMatrix<S, O, I>::IsRowMajor) {
        for (Index i = 0; i < a.rows(); ++i) {
            S t = S(0);
            for (I k = a.outer_[i]; k < a.outer_[i + 1]; ++k) t += a.val_[k] * x.coeff(a.inner_[k]);
            r[i] = r[i] + t;
        }
    } else {
        for (Index j = 0; j < a.cols(); ++j) {
            const S xj = x.coeff(j);
            for (I k = a.outer_[j]; k < a.outer_[j + 1]; ++k) r[a.inner_[k]] += a.val_[k] * xj;
        }
    }
    return r;
}

template <typename S, int R, int C, int O, int MR, int MC>
template <typename S2, int O2, typename I2>
Matrix<S, R, C, O, MR, MC>::Matrix(const SparseMatrix<S2, O2, I2>& a) {
    this->resize(a.rows(), a.cols());
    setZero();
    for (Index o = 0; o < a.outerSize(); ++o)
        for (I2 k = a.outer_[o]; k < a.outer_[o + 1]; ++k) {
            if constexpr (SparseMatrix<S2, O2, I2>::IsRowMajor) coeffRef(o, a.inner_[k]) = a.val_[k];
            else coeffRef(a.inner_[k], o) = a.val_[k];
        }
}

// ---- sparse Cholesky (natural ordering) ---------------------------------------------------

// LDL^T of the lower triangle in the natural order (Eigen's SimplicialLDLT permutes with AMD
// first); fails on a zero pivot as Eigen's does.
template <typename M, int UpLo = Lower> class SimplicialLDLT {
public:
    using S = typename M::Scalar;
    SimplicialLDLT() = default;
    explicit SimplicialLDLT(const M& a) { compute(a); }
    SimplicialLDLT& compute(const M& a) {
        n_ = a.rows();
        l_.assign(static_cast<std::size_t>(n_ * n_), S(0));
        d_.assign(static_cast<std::size_t>(n_), S(0));
        std::vector<S> lower(static_cast<std::size_t>(n_ * n_), S(0));
        for (Index o = 0; o < a.outerSize(); ++o)
            for (auto k = a.outer_[o]; k < a.outer_[o + 1]; ++k) {
                const Index r = M::IsRowMajor ? o : a.inner_[k], c = M::IsRowMajor ? a.inner_[k] : o;
                if (r >= c) lower[static_cast<std::size_t>(r * n_ + c)] = a.val_[k];
            }
        info_ = Success;
        for (Index j = 0; j < n_; ++j) {
            S dj = lower[static_cast<std::size_t>(j * n_ + j)];
            for (Index k = 0; k < j; ++k) {
                const S ljk = l_[static_cast<std::size_t>(j * n_ + k)];
                dj -= ljk * ljk * d_[static_cast<std::size_t>(k)];
            }
            if (dj == S(0)) {
                info_ = NumericalIssue;
                return *this;
            }
            d_[static_cast<std::size_t>(j)] = dj;
            l_[static_cast<std::size_t>(j * n_ + j)] = S(1);
            for (Index i = j + 1; i < n_; ++i) {
                S v = lower[static_cast<std::size_t>(i * n_ + j)];
                for (Index k = 0; k < j; ++k)
                    v -= l_[static_cast<std::size_t>(i * n_ + k)] * l_[static_cast<std::size_t>(j * n_ + k)] *
                         d_[static_cast<std::size_t>(k)];
                l_[static_cast<std::size_t>(i * n_ + j)] = v / dj;
            }
        }
        return *this;
    }
    ComputationInfo info() const { return info_; }
    template <typename V> Matrix<S, Dynamic, 1> solve(const V& b) const {
        if (info_ != Success) throw std::logic_error("SimplicialLDLT: solve after a failed factorisation");
        Matrix<S, Dynamic, 1> y(n_);
        for (Index i = 0; i < n_; ++i) {
            S v = b.coeff(i);
            for (Index k = 0; k < i; ++k) v -= l_[static_cast<std::size_t>(i * n_ + k)] * y[k];
            y[i] = v;
        }
        for (Index i = 0; i < n_; ++i) y[i] = y[i] / d_[static_cast<std::size_t>(i)];
        for (Index i = n_ - 1; i >= 0; --i) {
            S v = y[i];
            for (Index k = i + 1; k < n_; ++k) v -= l_[static_cast<std::size_t>(k * n_ + i)] * y[k];
            y[i] = v;
        }
        return y;
    }

private:
    Index n_ = 0;
    std::vector<S> l_, d_;
    ComputationInfo info_ = InvalidInput;
};

// ---- declared for compilation only ----------------------------------------------------------

template <typename S> class IncompleteCholesky {};

template <typename M, int UpLo = Lower, typename P = void> class ConjugateGradient {
public:
    void setTolerance(double) {}
    void setMaxIterations(Index) {}
    ConjugateGradient& compute(const M&) {
        throw std::logic_error("Eigen stand-in: ConjugateGradient is not provided");
    }
    template <typename B, typename X> Matrix<typename M::Scalar, Dynamic, 1> solveWithGuess(const B&, const X&) const {
        throw std::logic_error("Eigen stand-in: ConjugateGradient is not provided");
    }
    Index iterations() const { return 0; }
    ComputationInfo info() const { return InvalidInput; }
};

} // namespace Eigen
