// A small dense-matrix library exposing the subset of the Eigen API that the
// reference's integral and SCF sources use (MatrixXd / VectorXd storage and
// arithmetic, block/col access, a self-adjoint eigensolver and a
// column-pivoted Householder QR solve).  Eigen itself is not installed in
// this image; this file is written from the linear-algebra textbook methods
// (cyclic Jacobi rotations, Householder QR with column pivoting) and is only
// ever linked into the oracle build of the reference under oracle/_ref.
//
// The reference uses Eigen purely for storage on the ERI path
// (GaussianTwoElectrons.cpp:48-95, IntegralsRepository.cpp:396-421); on the
// SCF path it also multiplies, transposes and diagonalises
// (HartreeFockAlgorithm.cpp:48-59, RestrictedHartreeFock.cpp:121-153,
// DIIS.h:39-90).  Eigenvectors are unique only up to sign (and rotation in
// degenerate subspaces); densities and energies built from them are not.
#pragma once

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstddef>
#include <list>
#include <numeric>
#include <utility>
#include <vector>

namespace Eigen {

class MatrixXd;

// A column view used for `M.col(j) = N.col(k)` and `C.col(j) /= s`.
class ColRef {
 public:
  ColRef(MatrixXd &m, long j) : m_(m), j_(j) {}
  ColRef &operator=(const ColRef &o);
  ColRef &operator/=(double s);

 private:
  friend class MatrixXd;
  MatrixXd &m_;
  long j_;
};

class MatrixXd {
 public:
  MatrixXd() : r_(0), c_(0) {}
  MatrixXd(long r, long c) : r_(r), c_(c), d_(static_cast<size_t>(r * c), 0.0) {}
  MatrixXd(const MatrixXd &) = default;
  MatrixXd(MatrixXd &&) = default;
  MatrixXd &operator=(const MatrixXd &) = default;
  MatrixXd &operator=(MatrixXd &&) = default;

  static MatrixXd Zero(long r, long c) { return MatrixXd(r, c); }
  static MatrixXd Ones(long r, long c) {
    MatrixXd m(r, c);
    std::fill(m.d_.begin(), m.d_.end(), 1.0);
    return m;
  }
  static MatrixXd Identity(long r, long c) {
    MatrixXd m(r, c);
    for (long i = 0; i < std::min(r, c); ++i) m(i, i) = 1.0;
    return m;
  }

  long rows() const { return r_; }
  long cols() const { return c_; }
  long size() const { return r_ * c_; }
  void resize(long r, long c) {
    r_ = r;
    c_ = c;
    d_.assign(static_cast<size_t>(r * c), 0.0);
  }
  // column-major storage, as Eigen's default
  double &operator()(long i, long j) { return d_[static_cast<size_t>(j * r_ + i)]; }
  double operator()(long i, long j) const { return d_[static_cast<size_t>(j * r_ + i)]; }
  double &operator()(long i) { return d_[static_cast<size_t>(i)]; }
  double operator()(long i) const { return d_[static_cast<size_t>(i)]; }

  MatrixXd block(long i0, long j0, long nr, long nc) const {
    MatrixXd b(nr, nc);
    for (long j = 0; j < nc; ++j)
      for (long i = 0; i < nr; ++i) b(i, j) = (*this)(i0 + i, j0 + j);
    return b;
  }
  MatrixXd eval() const { return *this; }
  ColRef col(long j) { return ColRef(*this, j); }

  MatrixXd transpose() const {
    MatrixXd t(c_, r_);
    for (long j = 0; j < c_; ++j)
      for (long i = 0; i < r_; ++i) t(j, i) = (*this)(i, j);
    return t;
  }
  MatrixXd adjoint() const { return transpose(); }

  MatrixXd cwiseProduct(const MatrixXd &o) const {
    MatrixXd m(*this);
    for (size_t k = 0; k < d_.size(); ++k) m.d_[k] *= o.d_[k];
    return m;
  }
  MatrixXd cwiseInverse() const {
    MatrixXd m(*this);
    for (double &v : m.d_) v = 1.0 / v;
    return m;
  }
  MatrixXd cwiseSqrt() const {
    MatrixXd m(*this);
    for (double &v : m.d_) v = std::sqrt(v);
    return m;
  }
  // vector -> diagonal matrix
  MatrixXd asDiagonal() const {
    const long n = r_ * c_;
    MatrixXd m(n, n);
    for (long i = 0; i < n; ++i) m(i, i) = d_[static_cast<size_t>(i)];
    return m;
  }
  double sum() const { return std::accumulate(d_.begin(), d_.end(), 0.0); }
  double norm() const { return std::sqrt(cwiseProduct(*this).sum()); }

  MatrixXd &operator+=(const MatrixXd &o) {
    for (size_t k = 0; k < d_.size(); ++k) d_[k] += o.d_[k];
    return *this;
  }
  MatrixXd &operator-=(const MatrixXd &o) {
    for (size_t k = 0; k < d_.size(); ++k) d_[k] -= o.d_[k];
    return *this;
  }
  MatrixXd &operator*=(double s) {
    for (double &v : d_) v *= s;
    return *this;
  }
  MatrixXd &operator/=(double s) {
    for (double &v : d_) v /= s;
    return *this;
  }

  class QR;
  QR colPivHouseholderQr() const;

  const std::vector<double> &storage() const { return d_; }

 protected:
  long r_, c_;
  std::vector<double> d_;
};

inline ColRef &ColRef::operator=(const ColRef &o) {
  for (long i = 0; i < m_.rows(); ++i) m_(i, j_) = o.m_(i, o.j_);
  return *this;
}
inline ColRef &ColRef::operator/=(double s) {
  for (long i = 0; i < m_.rows(); ++i) m_(i, j_) /= s;
  return *this;
}

class VectorXd : public MatrixXd {
 public:
  VectorXd() : MatrixXd() {}
  explicit VectorXd(long n) : MatrixXd(n, 1) {}
  VectorXd(const MatrixXd &m) : MatrixXd(m) {}
  static VectorXd Zero(long n) { return VectorXd(n); }
  static VectorXd Ones(long n) { return VectorXd(MatrixXd::Ones(n, 1)); }
};

inline MatrixXd operator+(MatrixXd a, const MatrixXd &b) { return a += b; }
inline MatrixXd operator-(MatrixXd a, const MatrixXd &b) { return a -= b; }
inline MatrixXd operator*(MatrixXd a, double s) { return a *= s; }
inline MatrixXd operator*(double s, MatrixXd a) { return a *= s; }
inline MatrixXd operator/(MatrixXd a, double s) { return a /= s; }
inline MatrixXd operator*(const MatrixXd &a, const MatrixXd &b) {
  assert(a.cols() == b.rows());
  MatrixXd m(a.rows(), b.cols());
  for (long j = 0; j < b.cols(); ++j)
    for (long k = 0; k < a.cols(); ++k) {
      const double bkj = b(k, j);
      for (long i = 0; i < a.rows(); ++i) m(i, j) += a(i, k) * bkj;
    }
  return m;
}

// Householder QR with column pivoting, A P = Q R; solve() returns the
// least-squares / exact solution of A x = b.
class MatrixXd::QR {
 public:
  explicit QR(const MatrixXd &a) : qr_(a), perm_(static_cast<size_t>(a.cols())) {
    const long m = qr_.rows(), n = qr_.cols();
    std::iota(perm_.begin(), perm_.end(), 0L);
    std::vector<double> colnorm(static_cast<size_t>(n));
    for (long j = 0; j < n; ++j) {
      double s = 0;
      for (long i = 0; i < m; ++i) s += qr_(i, j) * qr_(i, j);
      colnorm[static_cast<size_t>(j)] = s;
    }
    const long kmax = std::min(m, n);
    beta_.assign(static_cast<size_t>(kmax), 0.0);
    for (long k = 0; k < kmax; ++k) {
      // pivot: remaining column with the largest norm
      long p = k;
      double best = -1;
      for (long j = k; j < n; ++j) {
        double s = 0;
        for (long i = k; i < m; ++i) s += qr_(i, j) * qr_(i, j);
        colnorm[static_cast<size_t>(j)] = s;
        if (s > best) { best = s; p = j; }
      }
      if (p != k) {
        for (long i = 0; i < m; ++i) std::swap(qr_(i, k), qr_(i, p));
        std::swap(perm_[static_cast<size_t>(k)], perm_[static_cast<size_t>(p)]);
      }
      // Householder vector for column k below the diagonal
      double alpha = 0;
      for (long i = k; i < m; ++i) alpha += qr_(i, k) * qr_(i, k);
      alpha = std::sqrt(alpha);
      if (alpha == 0) continue;
      if (qr_(k, k) > 0) alpha = -alpha;
      const double v0 = qr_(k, k) - alpha;
      // v = [v0, a_{k+1..m,k}], H = I - beta v v^T
      double vnorm2 = v0 * v0;
      for (long i = k + 1; i < m; ++i) vnorm2 += qr_(i, k) * qr_(i, k);
      const double beta = vnorm2 > 0 ? 2.0 / vnorm2 : 0.0;
      std::vector<double> v(static_cast<size_t>(m - k));
      v[0] = v0;
      for (long i = k + 1; i < m; ++i) v[static_cast<size_t>(i - k)] = qr_(i, k);
      for (long j = k + 1; j < n; ++j) {
        double s = 0;
        for (long i = k; i < m; ++i) s += v[static_cast<size_t>(i - k)] * qr_(i, j);
        s *= beta;
        for (long i = k; i < m; ++i) qr_(i, j) -= s * v[static_cast<size_t>(i - k)];
      }
      qr_(k, k) = alpha;
      for (long i = k + 1; i < m; ++i) qr_(i, k) = v[static_cast<size_t>(i - k)];
      vs_.push_back(std::move(v));
      beta_[static_cast<size_t>(k)] = beta;
      ks_.push_back(k);
    }
  }

  VectorXd solve(const MatrixXd &b) const {
    const long m = qr_.rows(), n = qr_.cols();
    std::vector<double> y(static_cast<size_t>(m));
    for (long i = 0; i < m; ++i) y[static_cast<size_t>(i)] = b(i);
    // y = Q^T b
    for (size_t t = 0; t < ks_.size(); ++t) {
      const long k = ks_[t];
      const std::vector<double> &v = vs_[t];
      double s = 0;
      for (long i = k; i < m; ++i) s += v[static_cast<size_t>(i - k)] * y[static_cast<size_t>(i)];
      s *= beta_[static_cast<size_t>(k)];
      for (long i = k; i < m; ++i) y[static_cast<size_t>(i)] -= s * v[static_cast<size_t>(i - k)];
    }
    // rank from |R_kk| relative to |R_00|
    const long kmax = std::min(m, n);
    const double tol = std::abs(kmax > 0 ? qr_(0, 0) : 0.0) * 1e-15 * static_cast<double>(std::max(m, n));
    long rank = 0;
    while (rank < kmax && std::abs(qr_(rank, rank)) > tol) ++rank;
    std::vector<double> z(static_cast<size_t>(n), 0.0);
    for (long i = rank - 1; i >= 0; --i) {
      double s = y[static_cast<size_t>(i)];
      for (long j = i + 1; j < rank; ++j) s -= qr_(i, j) * z[static_cast<size_t>(j)];
      z[static_cast<size_t>(i)] = s / qr_(i, i);
    }
    VectorXd x(n);
    for (long j = 0; j < n; ++j) x(perm_[static_cast<size_t>(j)]) = z[static_cast<size_t>(j)];
    return x;
  }

 private:
  MatrixXd qr_;
  std::vector<long> perm_;
  std::vector<std::vector<double>> vs_;
  std::vector<long> ks_;
  std::vector<double> beta_;
};

inline MatrixXd::QR MatrixXd::colPivHouseholderQr() const { return QR(*this); }

// Symmetric eigensolver by cyclic Jacobi rotations; eigenvalues ascending,
// eigenvectors as unit columns in the same order.
template <class M>
class SelfAdjointEigenSolver {
 public:
  explicit SelfAdjointEigenSolver(const MatrixXd &a) {
    const long n = a.rows();
    MatrixXd s = a;
    MatrixXd v = MatrixXd::Identity(n, n);
    const double total = s.cwiseProduct(s).sum();
    for (int sweep = 0; sweep < 60; ++sweep) {
      double off = 0;
      for (long j = 0; j < n; ++j)
        for (long i = 0; i < j; ++i) off += s(i, j) * s(i, j);
      if (off <= 1e-36 * total) break;
      for (long p = 0; p < n; ++p)
        for (long q = p + 1; q < n; ++q) {
          const double apq = s(p, q);
          if (apq == 0.0) continue;
          const double theta = (s(q, q) - s(p, p)) / (2.0 * apq);
          const double t = (theta >= 0 ? 1.0 : -1.0) / (std::abs(theta) + std::sqrt(theta * theta + 1.0));
          const double c = 1.0 / std::sqrt(t * t + 1.0);
          const double sn = t * c;
          for (long k = 0; k < n; ++k) {
            const double skp = s(k, p), skq = s(k, q);
            s(k, p) = c * skp - sn * skq;
            s(k, q) = sn * skp + c * skq;
          }
          for (long k = 0; k < n; ++k) {
            const double spk = s(p, k), sqk = s(q, k);
            s(p, k) = c * spk - sn * sqk;
            s(q, k) = sn * spk + c * sqk;
          }
          for (long k = 0; k < n; ++k) {
            const double vkp = v(k, p), vkq = v(k, q);
            v(k, p) = c * vkp - sn * vkq;
            v(k, q) = sn * vkp + c * vkq;
          }
        }
    }
    std::vector<long> order(static_cast<size_t>(n));
    std::iota(order.begin(), order.end(), 0L);
    std::stable_sort(order.begin(), order.end(), [&](long x, long y) { return s(x, x) < s(y, y); });
    values_ = VectorXd(n);
    vectors_ = MatrixXd(n, n);
    for (long k = 0; k < n; ++k) {
      const long o = order[static_cast<size_t>(k)];
      values_(k) = s(o, o);
      for (long i = 0; i < n; ++i) vectors_(i, k) = v(i, o);
    }
  }
  const VectorXd &eigenvalues() const { return values_; }
  const MatrixXd &eigenvectors() const { return vectors_; }

 private:
  VectorXd values_;
  MatrixXd vectors_;
};

// Declared so that DIIS.h's rank-4 tensor specialisation parses; the oracle
// build never instantiates it (it serves the CCSD code, which is not built).
template <class Scalar, int Rank>
class Tensor {
 public:
  void setZero() {}
  std::vector<long> dimensions() const { return {}; }
  double sum() const { return 0.0; }
  Tensor &operator+=(const Tensor &) { return *this; }
};
template <class Scalar, int Rank>
Tensor<Scalar, Rank> operator*(const Tensor<Scalar, Rank> &a, const Tensor<Scalar, Rank> &) { return a; }
template <class Scalar, int Rank>
Tensor<Scalar, Rank> operator*(double, const Tensor<Scalar, Rank> &a) { return a; }

}  // namespace Eigen

