// Test infrastructure only: a minimal, project-written stand-in for the parts of Eigen3 that the
// reference solver uses, so that the reference's own headers (include/*.hpp of
// RikibabManos/Magnetohydrodynamics_Simulator) compile unmodified here without Eigen installed.
//
// Eigen3 is a third-party dependency of the reference (CMakeLists.txt:7, `find_package(Eigen3
// REQUIRED)`, no version pin, not vendored). It is absent from this machine, so this file restates
// the published behaviour of the few Eigen entities the reference touches:
//   solvers.hpp:150      Eigen::SparseMatrix<double> member, copy-assigned at :441
//   solvers.hpp:412-439  std::vector<Eigen::Triplet<double>>, setFromTriplets, makeCompressed
//   solvers.hpp:465-470  Eigen::Map<const Eigen::VectorXd>, Eigen::VectorXd, solver.solve(...)
//   integrator_main.cpp:48,60,92  ConjugateGradient<SparseMatrix<double>, Lower|Upper>::compute
//
// ConjugateGradient follows Eigen's documented defaults for this instantiation:
//   * DiagonalPreconditioner (Jacobi): z = r / diag(A), unit scaling where diag(A) == 0;
//   * solve(b) starts from x0 = 0;
//   * tolerance = NumTraits<double>::epsilon(); stop when |r|^2 < max(tol^2 |b|^2, DBL_MIN);
//   * at most 2 * cols iterations; b == 0 returns x = 0 immediately;
//   * with UpLo = Lower|Upper on a column-major matrix the full matrix is used and the product is
//     taken through the (row-major) transpose, i.e. each output entry is a dot product of one
//     column with p in increasing row order (the matrix here is symmetric).
// It is NOT Eigen: reductions are plain left-to-right sums, so results agree with a real Eigen
// build to rounding only (parity at this boundary is unpinned against real Eigen).
#pragma once
#include <vector>
#include <cstddef>
#include <cmath>
#include <limits>
#include <algorithm>
#include <utility>

namespace Eigen {

enum { Lower = 1, Upper = 2 };

template <typename Scalar>
class Triplet {
public:
    Triplet() : r_(0), c_(0), v_(0) {}
    Triplet(int r, int c, Scalar v) : r_(r), c_(c), v_(v) {}
    int row() const { return r_; }
    int col() const { return c_; }
    Scalar value() const { return v_; }
private:
    int r_, c_;
    Scalar v_;
};

class VectorXd {
public:
    VectorXd() {}
    explicit VectorXd(std::ptrdiff_t n) : d_(static_cast<size_t>(n), 0.0) {}
    std::ptrdiff_t size() const { return static_cast<std::ptrdiff_t>(d_.size()); }
    double& operator[](std::ptrdiff_t i) { return d_[static_cast<size_t>(i)]; }
    double operator[](std::ptrdiff_t i) const { return d_[static_cast<size_t>(i)]; }
    double& operator()(std::ptrdiff_t i) { return d_[static_cast<size_t>(i)]; }
    double operator()(std::ptrdiff_t i) const { return d_[static_cast<size_t>(i)]; }
    double* data() { return d_.data(); }
    const double* data() const { return d_.data(); }
    void resize(std::ptrdiff_t n) { d_.assign(static_cast<size_t>(n), 0.0); }
    template <typename Other>
    VectorXd& operator=(const Other& o) {
        std::vector<double> tmp(static_cast<size_t>(o.size()));
        for (std::ptrdiff_t i = 0; i < o.size(); ++i) tmp[static_cast<size_t>(i)] = o[i];
        d_.swap(tmp);
        return *this;
    }
    VectorXd& operator=(const VectorXd& o) { d_ = o.d_; return *this; }
    VectorXd(const VectorXd& o) = default;
private:
    std::vector<double> d_;
};

template <typename T>
class Map;

template <>
class Map<const VectorXd> {
public:
    Map(const double* p, std::ptrdiff_t n) : p_(p), n_(n) {}
    std::ptrdiff_t size() const { return n_; }
    double operator[](std::ptrdiff_t i) const { return p_[i]; }
    double operator()(std::ptrdiff_t i) const { return p_[i]; }
private:
    const double* p_;
    std::ptrdiff_t n_;
};

// Compressed column storage; row indices sorted inside each column, duplicates summed.
template <typename Scalar, int Options = 0, typename StorageIndex = int>
class SparseMatrix {
public:
    SparseMatrix() : rows_(0), cols_(0) {}
    SparseMatrix(std::ptrdiff_t r, std::ptrdiff_t c)
        : rows_(r), cols_(c), outer_(static_cast<size_t>(c) + 1, 0) {}
    std::ptrdiff_t rows() const { return rows_; }
    std::ptrdiff_t cols() const { return cols_; }

    template <typename It>
    void setFromTriplets(It begin, It end) {
        // counting sort by column (stable: triplets of one column keep their insertion order),
        // then a stable sort by row inside each column; duplicates are summed in that order
        const size_t nc = static_cast<size_t>(cols_);
        std::vector<size_t> start(nc + 1, 0);
        size_t total = 0;
        for (It it = begin; it != end; ++it) {
            ++start[static_cast<size_t>(it->col()) + 1];
            ++total;
        }
        for (size_t c = 0; c < nc; ++c) start[c + 1] += start[c];
        std::vector<std::pair<int, Scalar>> buf(total);
        std::vector<size_t> fill(start.begin(), start.end() - 1);
        for (It it = begin; it != end; ++it)
            buf[fill[static_cast<size_t>(it->col())]++] = std::make_pair(it->row(), it->value());
        outer_.assign(nc + 1, 0);
        inner_.clear();
        val_.clear();
        inner_.reserve(total);
        val_.reserve(total);
        for (size_t c = 0; c < nc; ++c) {
            std::stable_sort(buf.begin() + start[c], buf.begin() + start[c + 1],
                             [](const std::pair<int, Scalar>& a, const std::pair<int, Scalar>& b) {
                                 return a.first < b.first;
                             });
            for (size_t k = start[c]; k < start[c + 1]; ++k) {
                if (static_cast<StorageIndex>(inner_.size()) > outer_[c] &&
                    inner_.back() == buf[k].first) {
                    val_.back() += buf[k].second;  // duplicates are summed
                } else {
                    inner_.push_back(buf[k].first);
                    val_.push_back(buf[k].second);
                }
            }
            outer_[c + 1] = static_cast<StorageIndex>(inner_.size());
        }
    }
    void makeCompressed() {}

    // Accessors used by ConjugateGradient below.
    const std::vector<StorageIndex>& outer() const { return outer_; }
    const std::vector<int>& inner() const { return inner_; }
    const std::vector<Scalar>& values() const { return val_; }

private:
    std::ptrdiff_t rows_, cols_;
    std::vector<StorageIndex> outer_;
    std::vector<int> inner_;
    std::vector<Scalar> val_;
};

template <typename MatrixType, int UpLo>
class ConjugateGradient {
public:
    ConjugateGradient() : mat_(nullptr), iters_(0), error_(0), max_iters_(-1),
                          tol_(std::numeric_limits<double>::epsilon()) {}

    ConjugateGradient& compute(const MatrixType& A) {
        mat_ = &A;
        const std::ptrdiff_t n = A.cols();
        invdiag_.assign(static_cast<size_t>(n), 1.0);
        for (std::ptrdiff_t c = 0; c < n; ++c) {
            for (auto k = A.outer()[c]; k < A.outer()[c + 1]; ++k) {
                if (A.inner()[static_cast<size_t>(k)] == c) {
                    const double d = A.values()[static_cast<size_t>(k)];
                    invdiag_[static_cast<size_t>(c)] = (d == 0.0) ? 1.0 : 1.0 / d;
                }
            }
        }
        return *this;
    }

    void setMaxIterations(std::ptrdiff_t m) { max_iters_ = m; }
    void setTolerance(double t) { tol_ = t; }
    std::ptrdiff_t iterations() const { return iters_; }
    double error() const { return error_; }
    // Total matrix-vector products of the last solve (iterations() counts them Eigen's way).
    std::ptrdiff_t products() const { return products_; }
    // Products of every solve since the log was last cleared (test instrumentation).
    std::vector<std::ptrdiff_t> product_log;

    template <typename Rhs>
    VectorXd solve(const Rhs& b) {
        const std::ptrdiff_t n = mat_->cols();
        VectorXd x(n);  // x0 = 0
        products_ = 0;
        double rhsNorm2 = 0.0;
        for (std::ptrdiff_t i = 0; i < n; ++i) rhsNorm2 += b[i] * b[i];
        if (rhsNorm2 == 0.0) { iters_ = 0; error_ = 0.0; product_log.push_back(0); return x; }
        const double considerAsZero = std::numeric_limits<double>::min();
        const double threshold = std::max(tol_ * tol_ * rhsNorm2, considerAsZero);
        std::vector<double> r(static_cast<size_t>(n)), p(static_cast<size_t>(n)),
            z(static_cast<size_t>(n)), tmp(static_cast<size_t>(n));
        for (std::ptrdiff_t i = 0; i < n; ++i) r[i] = b[i] - 0.0;  // r = b - A*0
        double residualNorm2 = 0.0;
        for (std::ptrdiff_t i = 0; i < n; ++i) residualNorm2 += r[i] * r[i];
        if (residualNorm2 < threshold) {
            iters_ = 0; error_ = std::sqrt(residualNorm2 / rhsNorm2);
            product_log.push_back(0);
            return x;
        }
        for (std::ptrdiff_t i = 0; i < n; ++i) p[i] = invdiag_[i] * r[i];
        double absNew = 0.0;
        for (std::ptrdiff_t i = 0; i < n; ++i) absNew += r[i] * p[i];
        const std::ptrdiff_t maxIters = (max_iters_ < 0) ? 2 * n : max_iters_;
        std::ptrdiff_t i = 0;
        while (i < maxIters) {
            product(p, tmp);
            ++products_;
            double pt = 0.0;
            for (std::ptrdiff_t k = 0; k < n; ++k) pt += p[k] * tmp[k];
            const double alpha = absNew / pt;
            for (std::ptrdiff_t k = 0; k < n; ++k) x[k] += alpha * p[k];
            for (std::ptrdiff_t k = 0; k < n; ++k) r[k] -= alpha * tmp[k];
            residualNorm2 = 0.0;
            for (std::ptrdiff_t k = 0; k < n; ++k) residualNorm2 += r[k] * r[k];
            if (residualNorm2 < threshold) break;
            for (std::ptrdiff_t k = 0; k < n; ++k) z[k] = invdiag_[k] * r[k];
            const double absOld = absNew;
            absNew = 0.0;
            for (std::ptrdiff_t k = 0; k < n; ++k) absNew += r[k] * z[k];
            const double beta = absNew / absOld;
            for (std::ptrdiff_t k = 0; k < n; ++k) p[k] = z[k] + beta * p[k];
            ++i;
        }
        error_ = std::sqrt(residualNorm2 / rhsNorm2);
        iters_ = i;
        product_log.push_back(products_);
        return x;
    }

private:
    // out = A^T p, one dot product per output entry (A is symmetric here).
    void product(const std::vector<double>& p, std::vector<double>& out) const {
        const std::ptrdiff_t n = mat_->cols();
        for (std::ptrdiff_t c = 0; c < n; ++c) {
            double acc = 0.0;
            for (auto k = mat_->outer()[c]; k < mat_->outer()[c + 1]; ++k)
                acc += mat_->values()[static_cast<size_t>(k)] * p[mat_->inner()[static_cast<size_t>(k)]];
            out[static_cast<size_t>(c)] = 0.0 + acc;
        }
    }

    const MatrixType* mat_;
    std::vector<double> invdiag_;
    std::ptrdiff_t iters_;
    std::ptrdiff_t products_ = 0;
    double error_;
    std::ptrdiff_t max_iters_;
    double tol_;
};

}  // namespace Eigen
