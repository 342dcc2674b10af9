// mat3d_matrix.hpp -- the small dense-matrix type of the drop-in headers.
//
// The reference's classes expose Eigen dynamic matrices
// (typedef Matrix<double,Dynamic,Dynamic> MatrixDdd; Matrix<int,...> MatrixIdd,
// include/FFT_analysis3D.hpp:31-32).  Eigen is not a dependency of this
// library, so the drop-in headers ship this column-major stand-in with the
// subset callers of the reference use: (rows, cols) construction, resize,
// m(i) (linear, column-major) and m(i,j) access, the `m << a, b, ...` comma
// initializer (row by row), rows(), cols(), size(), data(), setZero(),
// setOnes(), sum(), row(i).sum(), col(j) copies, inverse() of small square
// matrices and printing.
#ifndef MAT3D_MATRIX_HPP
#define MAT3D_MATRIX_HPP

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <ostream>
#include <stdexcept>
#include <vector>

namespace m3d {

template <class T>
class DMatrix {
public:
    DMatrix() {}
    DMatrix(int r, int c) : r_(r), c_(c), d_((std::size_t)r * c, T()) {}

    int rows() const { return r_; }
    int cols() const { return c_; }
    int size() const { return r_ * c_; }
    void resize(int r, int c) {
        if (r == r_ && c == c_) return;
        r_ = r;
        c_ = c;
        d_.assign((std::size_t)r * c, T());
    }
    T* data() { return d_.data(); }
    const T* data() const { return d_.data(); }
    T& operator()(int i) { return d_[(std::size_t)i]; }
    const T& operator()(int i) const { return d_[(std::size_t)i]; }
    T& operator()(int i, int j) { return d_[(std::size_t)j * r_ + i]; }
    const T& operator()(int i, int j) const { return d_[(std::size_t)j * r_ + i]; }

    void setZero() { std::fill(d_.begin(), d_.end(), T(0)); }
    void setZero(int r, int c) { resize(r, c); setZero(); }
    void setOnes() { std::fill(d_.begin(), d_.end(), T(1)); }
    T sum() const {
        T s = T(0);
        for (const T& v : d_) s += v;
        return s;
    }

    struct RowRef {
        const DMatrix* m;
        int i;
        T sum() const {
            T s = T(0);
            for (int j = 0; j < m->c_; ++j) s += (*m)(i, j);
            return s;
        }
    };
    RowRef row(int i) const { return RowRef{this, i}; }
    DMatrix col(int j) const {
        DMatrix o(r_, 1);
        for (int i = 0; i < r_; ++i) o(i) = (*this)(i, j);
        return o;
    }

    DMatrix inverse() const {
        if (r_ != c_) throw std::invalid_argument("inverse of a non-square matrix");
        const int n = r_;
        DMatrix a = *this, inv(n, n);
        for (int i = 0; i < n; ++i) inv(i, i) = T(1);
        for (int c = 0; c < n; ++c) {
            int p = c;
            for (int r = c + 1; r < n; ++r)
                if (std::abs(a(r, c)) > std::abs(a(p, c))) p = r;
            for (int j = 0; j < n; ++j) { std::swap(a(c, j), a(p, j)); std::swap(inv(c, j), inv(p, j)); }
            const T pv = a(c, c);
            for (int j = 0; j < n; ++j) { a(c, j) /= pv; inv(c, j) /= pv; }
            for (int r = 0; r < n; ++r) {
                if (r == c) continue;
                const T f = a(r, c);
                for (int j = 0; j < n; ++j) { a(r, j) -= f * a(c, j); inv(r, j) -= f * inv(c, j); }
            }
        }
        return inv;
    }

    class Comma {
    public:
        Comma(DMatrix* m, int k) : m_(m), k_(k) {}
        Comma& operator,(T v) {
            m_->put(k_++, v);
            return *this;
        }
    private:
        DMatrix* m_;
        int k_;
    };
    Comma operator<<(T v) {
        put(0, v);
        return Comma(this, 1);
    }

private:
    void put(int k, T v) {
        if (c_ == 0 || k >= r_ * c_) throw std::out_of_range("too many coefficients in comma initializer");
        (*this)(k / c_, k % c_) = v;
    }
    int r_ = 0, c_ = 0;
    std::vector<T> d_;
};

template <class T>
inline std::ostream& operator<<(std::ostream& os, const DMatrix<T>& m) {
    for (int i = 0; i < m.rows(); ++i) {
        for (int j = 0; j < m.cols(); ++j) os << (j ? " " : "") << m(i, j);
        if (i + 1 < m.rows()) os << '\n';
    }
    return os;
}

}  // namespace m3d

typedef m3d::DMatrix<double> MatrixDdd;
typedef m3d::DMatrix<int> MatrixIdd;

#endif
