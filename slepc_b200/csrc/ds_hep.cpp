// Host FP64 projected-problem solver; see ds_hep.h for the reference map.
#include "ds_hep.h"

#include <cmath>
#include <cstring>

// LAPACK / BLAS from the OpenBLAS bundled with scipy (symbols carry a scipy_ prefix).
extern "C" {
void scipy_dlartg_(const double *f, const double *g, double *c, double *s, double *r);
void scipy_drot_(const int *n, double *x, const int *incx, double *y, const int *incy, const double *c,
                 const double *s);
void scipy_dsteqr_(const char *compz, const int *n, double *d, double *e, double *z, const int *ldz, double *work,
                   int *info, size_t len);
}

namespace b200 {

void DsHep::allocate(int ld) {
  ld_ = ld;
  d_.assign((size_t)3 * ld, 0.0);
  Q_.assign((size_t)ld * ld, 0.0);
  rwork_.assign((size_t)2 * ld + 2, 0.0);
  perm_.assign(ld, 0);
  n_ = l_ = k_ = t_ = 0;
  state_ = kRaw;
}

int DsHep::compare(int which, double a, double b) {
  switch (which) {
    case B200_LARGEST_MAGNITUDE: {
      const double x = std::fabs(a), y = std::fabs(b);
      return (x < y) ? 1 : (x > y) ? -1 : 0;
    }
    case B200_SMALLEST_MAGNITUDE: {
      const double x = std::fabs(a), y = std::fabs(b);
      return (x > y) ? 1 : (x < y) ? -1 : 0;
    }
    case B200_LARGEST_REAL:
      return (a < b) ? 1 : (a > b) ? -1 : 0;
    case B200_SMALLEST_REAL:
      return (a > b) ? 1 : (a < b) ? -1 : 0;
    default:
      return 0;
  }
}

void DsHep::set_identity() {
  // Columns l..n-1 become the identity; locked columns keep their content.
  std::memset(Q_.data() + (size_t)l_ * ld_, 0, sizeof(double) * (size_t)ld_ * (n_ - l_));
  for (int i = l_; i < n_; ++i) Q_[i + (size_t)i * ld_] = 1.0;
}

// Rutishauser's reduction of a symmetric arrowhead to tridiagonal form with
// Givens rotations (LAPACK dlartg / BLAS drot), accumulating them into Q.
void DsHep::arrow_tridiag(int n, double *d, double *e, double *Q, int ld) {
  if (n <= 2) return;
  const int one = 1;
  for (int j = 0; j < n - 2; ++j) {
    double c, s, temp = e[j + 1];
    scipy_dlartg_(&temp, &e[j], &c, &s, &e[j + 1]);
    s = -s;
    temp = d[j + 1];
    e[j] = c * s * (temp - d[j]);
    d[j + 1] = s * s * d[j] + c * c * temp;
    d[j] = c * c * d[j] + s * s * temp;
    const int j2 = j + 2;
    scipy_drot_(&j2, Q + (size_t)j * ld, &one, Q + (size_t)(j + 1) * ld, &one, &c, &s);
    for (int i = j - 1; i >= 0; --i) {
      const double off = -s * e[i];
      e[i] = c * e[i];
      temp = e[i + 1];
      scipy_dlartg_(&temp, &off, &c, &s, &e[i + 1]);
      s = -s;
      temp = (d[i] - d[i + 1]) * s - 2.0 * c * e[i];
      const double p = s * temp;
      d[i + 1] += p;
      d[i] -= p;
      e[i] = -e[i] - c * temp;
      scipy_drot_(&j2, Q + (size_t)i * ld, &one, Q + (size_t)(i + 1) * ld, &one, &c, &s);
    }
  }
}

b200_status DsHep::solve(double *wr) {
  double *d = this->d(), *e = this->e();
  const size_t off = (size_t)l_ + (size_t)l_ * ld_;
  set_identity();
  if (state_ < kIntermediate) {
    int na = k_ - l_ + 1;
    if (na < 0) na = 0;
    arrow_tridiag(na, d + l_, e + l_, Q_.data() + off, ld_);
  }
  for (int i = 0; i < l_; ++i) wr[i] = d[i];
  int n1 = n_ - l_, info = 0, ld = ld_;
  if (n1 > 0) scipy_dsteqr_("V", &n1, d + l_, e + l_, Q_.data() + off, &ld, rwork_.data(), &info, 1);
  if (info) return B200_ERR_LAPACK;
  for (int i = l_; i < n_; ++i) wr[i] = d[i];
  if (n_ > 1) std::memset(e, 0, sizeof(double) * (size_t)(n_ - 1));
  state_ = kCondensed;
  return B200_OK;
}

void DsHep::sort(double *wr) {
  double *d = this->d();
  int *perm = perm_.data();
  for (int i = 0; i < n_; ++i) perm[i] = i;
  // insertion sort of d[l..t) with the comparator (stable for ties)
  for (int i = l_ + 1; i < t_; ++i) {
    const double re = d[perm[i]];
    int j = i - 1;
    int result = compare(which_, re, d[perm[j]]);
    while (result < 0 && j >= l_) {
      const int tmp = perm[j];
      perm[j] = perm[j + 1];
      perm[j + 1] = tmp;
      --j;
      if (j >= l_) result = compare(which_, re, d[perm[j]]);
    }
  }
  for (int i = l_; i < n_; ++i) wr[i] = d[perm[i]];
  // apply the permutation to the columns of Q (cycle walk with swaps)
  for (int i = l_; i < n_; ++i) {
    const int p = perm[i];
    if (p != i) {
      int j = i + 1;
      while (perm[j] != i) ++j;
      perm[j] = p;
      perm[i] = i;
      double *qp = Q_.data() + (size_t)p * ld_, *qi = Q_.data() + (size_t)i * ld_;
      for (int r = 0; r < n_; ++r) {
        const double tmp = qp[r];
        qp[r] = qi[r];
        qi[r] = tmp;
      }
    }
  }
  for (int i = l_; i < n_; ++i) d[i] = wr[i];
}

void DsHep::update_extra_row() {
  double *e = this->e();
  const double beta = e[n_ - 1];
  for (int i = 0; i < n_; ++i) e[i] = beta * Q_[n_ - 1 + (size_t)i * ld_];
  k_ = n_;
}

void DsHep::truncate(int n) {
  k_ = n;  // extra row present
  t_ = n_;
  n_ = n;
  state_ = kTruncated;
}

}  // namespace b200
