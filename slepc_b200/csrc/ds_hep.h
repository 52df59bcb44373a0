// Host FP64 solver of the projected Hermitian problem (DS of type HEP, compact
// arrowhead + tridiagonal storage), as used inside Krylov-Schur.
//
// Restates src/sys/classes/ds/impls/hep/dshep.c (DSArrowTridiag :221-265,
// DSIntermediate_HEP :267-321, DSSort_HEP :323-347, DSUpdateExtraRow_HEP
// :349-381, DSSolve_HEP_QR :383-427, DSTruncate_HEP :643-671) and
// src/sys/classes/ds/interface/dspriv.c (DSSortEigenvaluesReal_Private
// :254-273, DSPermuteColumns_Private :279-301, DSSetIdentity :407-426).
// The ncv x ncv problem stays on the host: it is O(ncv^3) ~ 0.5 Mflop per
// restart, far below a single GPU pass over the basis.
#pragma once

#include <vector>

#include "slepc_b200.h"

namespace b200 {

class DsHep {
 public:
  enum State { kRaw = 0, kIntermediate = 1, kCondensed = 2, kTruncated = 3 };

  void allocate(int ld);
  void set_dimensions(int n, int l, int k) {
    n_ = n;
    t_ = n;
    l_ = l;
    k_ = k;
  }
  void set_state(State s) { state_ = s; }
  void set_which(int which) { which_ = which; }

  // DSSolve (QR method): arrowhead reduction if RAW, then LAPACK dsteqr.
  b200_status solve(double *wr);
  // DSSort with the eigenvalue comparator of `which`.
  void sort(double *wr);
  // DSUpdateExtraRow: e_i = beta * Q(n-1, i), k = n.
  void update_extra_row();
  // DSTruncate(n, trim = false).
  void truncate(int n);

  int ld() const { return ld_; }
  int n() const { return n_; }
  double *d() { return d_.data(); }
  double *e() { return d_.data() + ld_; }
  double *Q() { return Q_.data(); }
  const double *Q() const { return Q_.data(); }

  // Comparator of SlepcCompare{Largest,Smallest}{Magnitude,Real}: <0 if a goes first.
  static int compare(int which, double a, double b);

 private:
  void set_identity();
  static void arrow_tridiag(int n, double *d, double *e, double *Q, int ld);

  int ld_ = 0, n_ = 0, l_ = 0, k_ = 0, t_ = 0;
  State state_ = kRaw;
  int which_ = B200_LARGEST_MAGNITUDE;
  std::vector<double> d_;  // d at [0,ld), e at [ld,2ld), third column unused
  std::vector<double> Q_;
  std::vector<double> rwork_;
  std::vector<int> perm_;
};

}  // namespace b200
