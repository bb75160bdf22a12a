// Test infrastructure, not product code.
//
// Stand-in for the Blasw BLAS/LAPACK wrapper (github.com/Mathific/Blasw), a
// git submodule of the reference at 3rd/blasw that is empty in the reference
// tree, so its pinned commit is not known here.  It provides only the calls
// that the reference's src/spyker/cpu/zca.cpp:67-118 makes, so that file
// compiles unmodified with SPYKER_USE_BLAS and its ZCA composition can be
// checked against the oracle's restatement (oracle/zca.py).
//
// Semantics restated from the BLAS/LAPACK routines the wrapper's names stand
// for (row-major storage throughout, as zca.cpp lays its arrays out):
//   rmat(p, r, c)             r x c row-major matrix view; .trans() its transpose
//   vec(p, n)                 vector view
//   rusym(p, n)               n x n symmetric matrix, upper triangle stored row-major
//   dot(A, x, y, a, b)        y = a A x + b y                      (gemv)
//   dot(A, B, C, a, b)        C = a A B + b C, B a matrix or a symmetric view (gemm / symm)
//   update(A, S, a, b)        S = a A A^T + b S on S's upper triangle (syrk)
//   eigen(S, w, true, true)   eigenvalues of S ascending in w and the matching
//                             unit eigenvectors in S's columns (syev, jobz = V):
//                             zca.cpp then forms U diag(f(w)) U^T from S's rows
//                             (zca.cpp:89-97), which needs exactly that layout.
//                             The meaning of the two flags is not known here;
//                             zca.cpp passes (true, true) and the shim always
//                             returns the eigenvectors.
// Sums are taken in FP64 and rounded once to the element type (the reference's
// BLAS rounds per operation; the checks allow for that difference).  The
// eigensolver is the cyclic Jacobi method (Golub and Van Loan, Matrix
// Computations, 4th ed., sec. 8.5.2-8.5.3) in FP64, swept until the
// off-diagonal mass is below 1e-30 of the matrix's squared Frobenius norm.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <numeric>
#include <stdexcept>
#include <vector>

// zca.cpp passes LAPACKE_sgesdd / LAPACKE_dgesdd as an argument it never calls
// (cpu/zca.cpp:67,161-164); these placeholders only give the names a type.
inline int LAPACKE_sgesdd() { return -1; }
inline int LAPACKE_dgesdd() { return -1; }

namespace Blasw
{
template <typename T>
struct Mat
{
    T *data;
    std::ptrdiff_t r, c;  // stored rows and columns (row-major)
    bool t;               // logical view is the transpose of the stored matrix

    std::ptrdiff_t rows() const { return t ? c : r; }
    std::ptrdiff_t cols() const { return t ? r : c; }
    T &at(std::ptrdiff_t i, std::ptrdiff_t j) const { return t ? data[j * c + i] : data[i * c + j]; }
    Mat trans() const { return Mat{data, r, c, !t}; }
};

template <typename T>
struct Sym
{
    T *data;
    std::ptrdiff_t n;

    std::ptrdiff_t rows() const { return n; }
    std::ptrdiff_t cols() const { return n; }
    T &at(std::ptrdiff_t i, std::ptrdiff_t j) const { return i <= j ? data[i * n + j] : data[j * n + i]; }
};

template <typename T>
struct Vec
{
    T *data;
    std::ptrdiff_t n;
};

template <typename T, typename I, typename J>
Mat<T> rmat(T *data, I rows, J cols)
{
    return Mat<T>{data, std::ptrdiff_t(rows), std::ptrdiff_t(cols), false};
}

template <typename T, typename I>
Sym<T> rusym(T *data, I n)
{
    return Sym<T>{data, std::ptrdiff_t(n)};
}

template <typename T, typename I>
Vec<T> vec(T *data, I n)
{
    return Vec<T>{data, std::ptrdiff_t(n)};
}

inline void need(bool ok, const char *what)
{
    if (!ok) throw std::runtime_error(what);
}

// y = alpha A x + beta y
template <typename T, typename A, typename B>
void dot(Mat<T> a, Vec<T> x, Vec<T> y, A alpha, B beta)
{
    need(a.cols() == x.n && a.rows() == y.n, "blasw shim: gemv shapes");
    std::vector<double> out(size_t(y.n));
    for (std::ptrdiff_t i = 0; i < a.rows(); ++i)
    {
        double s = 0;
        for (std::ptrdiff_t k = 0; k < a.cols(); ++k) s += double(a.at(i, k)) * double(x.data[k]);
        out[size_t(i)] = double(alpha) * s + (double(beta) != 0 ? double(beta) * double(y.data[i]) : 0.0);
    }
    for (std::ptrdiff_t i = 0; i < y.n; ++i) y.data[i] = T(out[size_t(i)]);
}

// C = alpha A B + beta C, B a general matrix view or a symmetric view
template <typename T, typename MB, typename A, typename B>
void dot(Mat<T> a, MB b, Mat<T> c, A alpha, B beta)
{
    need(a.cols() == b.rows() && a.rows() == c.rows() && b.cols() == c.cols(), "blasw shim: gemm shapes");
    const std::ptrdiff_t m = a.rows(), n = b.cols(), kk = a.cols();
    std::vector<double> bt(size_t(n * kk));  // B transposed, for unit-stride inner loops
    for (std::ptrdiff_t k = 0; k < kk; ++k)
        for (std::ptrdiff_t j = 0; j < n; ++j) bt[size_t(j * kk + k)] = double(b.at(k, j));
    std::vector<double> out(size_t(m * n));
#pragma omp parallel for
    for (std::ptrdiff_t i = 0; i < m; ++i)
    {
        std::vector<double> arow(static_cast<size_t>(kk));
        for (std::ptrdiff_t k = 0; k < kk; ++k) arow[size_t(k)] = double(a.at(i, k));
        for (std::ptrdiff_t j = 0; j < n; ++j)
        {
            double s = 0;
            const double *bj = bt.data() + j * kk;
            for (std::ptrdiff_t k = 0; k < kk; ++k) s += arow[size_t(k)] * bj[k];
            out[size_t(i * n + j)] = double(alpha) * s + (double(beta) != 0 ? double(beta) * double(c.at(i, j)) : 0.0);
        }
    }
    for (std::ptrdiff_t i = 0; i < m; ++i)
        for (std::ptrdiff_t j = 0; j < n; ++j) c.at(i, j) = T(out[size_t(i * n + j)]);
}

// S = alpha A A^T + beta S, upper triangle only
template <typename T, typename A, typename B>
void update(Mat<T> a, Sym<T> s, A alpha, B beta)
{
    need(a.rows() == s.n, "blasw shim: syrk shapes");
    const std::ptrdiff_t n = s.n, kk = a.cols();
    std::vector<double> rows(size_t(n * kk));
    for (std::ptrdiff_t i = 0; i < n; ++i)
        for (std::ptrdiff_t k = 0; k < kk; ++k) rows[size_t(i * kk + k)] = double(a.at(i, k));
#pragma omp parallel for
    for (std::ptrdiff_t i = 0; i < n; ++i)
        for (std::ptrdiff_t j = i; j < n; ++j)
        {
            double v = 0;
            const double *ri = rows.data() + i * kk, *rj = rows.data() + j * kk;
            for (std::ptrdiff_t k = 0; k < kk; ++k) v += ri[k] * rj[k];
            s.data[i * n + j] =
                T(double(alpha) * v + (double(beta) != 0 ? double(beta) * double(s.data[i * n + j]) : 0.0));
        }
}

// Eigenvalues ascending in w and unit eigenvectors in the columns of S's full
// row-major storage; only S's upper triangle is read.
template <typename T>
void eigen(Sym<T> s, Vec<T> w, bool, bool)
{
    const std::ptrdiff_t n = s.n;
    need(w.n == n, "blasw shim: eigen shapes");
    std::vector<double> a(size_t(n * n)), v(size_t(n * n), 0.0);
    for (std::ptrdiff_t i = 0; i < n; ++i)
        for (std::ptrdiff_t j = 0; j < n; ++j)
        {
            a[size_t(i * n + j)] = double(s.at(i, j));
        }
    for (std::ptrdiff_t i = 0; i < n; ++i) v[size_t(i * n + i)] = 1.0;
    auto A = [&](std::ptrdiff_t i, std::ptrdiff_t j) -> double & { return a[size_t(i * n + j)]; };
    auto V = [&](std::ptrdiff_t i, std::ptrdiff_t j) -> double & { return v[size_t(i * n + j)]; };

    double fro = 0;
    for (double x : a) fro += x * x;
    for (int sweep = 0; sweep < 100; ++sweep)
    {
        double off = 0;
        for (std::ptrdiff_t p = 0; p < n; ++p)
            for (std::ptrdiff_t q = p + 1; q < n; ++q) off += 2 * A(p, q) * A(p, q);
        if (off <= 1e-30 * fro) break;
        for (std::ptrdiff_t p = 0; p < n; ++p)
            for (std::ptrdiff_t q = p + 1; q < n; ++q)
            {
                const double apq = A(p, q);
                if (apq == 0) continue;
                // symmetric Schur 2x2: rotation (c, s) zeroing A(p, q)
                const double tau = (A(q, q) - A(p, p)) / (2 * apq);
                const double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1 + tau * tau));
                const double c = 1 / std::sqrt(1 + t * t), sn = t * c;
                for (std::ptrdiff_t k = 0; k < n; ++k)  // A <- A J
                {
                    const double akp = A(k, p), akq = A(k, q);
                    A(k, p) = c * akp - sn * akq;
                    A(k, q) = sn * akp + c * akq;
                }
                for (std::ptrdiff_t k = 0; k < n; ++k)  // A <- J^T A
                {
                    const double apk = A(p, k), aqk = A(q, k);
                    A(p, k) = c * apk - sn * aqk;
                    A(q, k) = sn * apk + c * aqk;
                }
                for (std::ptrdiff_t k = 0; k < n; ++k)  // V <- V J
                {
                    const double vkp = V(k, p), vkq = V(k, q);
                    V(k, p) = c * vkp - sn * vkq;
                    V(k, q) = sn * vkp + c * vkq;
                }
            }
    }
    std::vector<std::ptrdiff_t> order(static_cast<size_t>(n));
    std::iota(order.begin(), order.end(), std::ptrdiff_t(0));
    std::stable_sort(order.begin(), order.end(),
                     [&](std::ptrdiff_t x, std::ptrdiff_t y) { return A(x, x) < A(y, y); });
    for (std::ptrdiff_t j = 0; j < n; ++j) w.data[j] = T(A(order[size_t(j)], order[size_t(j)]));
    for (std::ptrdiff_t i = 0; i < n; ++i)
            for (std::ptrdiff_t j = 0; j < n; ++j) s.data[i * n + j] = T(V(i, order[size_t(j)]));
}
}  // namespace Blasw
