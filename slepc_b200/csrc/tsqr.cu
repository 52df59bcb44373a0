// Householder QR of a tall block of basis columns on the device, for the TSQR and TSQRCHOL block
// orthogonalizations of BVOrthogonalize.
//
// Replaces, on one process (one GPU), BVOrthogonalize_LAPACK_TSQR and
// BVOrthogonalize_LAPACK_TSQR_OnlyR (src/sys/classes/bv/interface/bvlapack.c:347-440, 510-560),
// which call LAPACK geqrf on the local rows, extract R and, for TSQR, form Q with orgqr (the MPI
// tree of R factors is empty with one process).  The kernels below restate the unblocked
// Householder algorithm (geqr2: for each column the reflector of dlarfg, beta = -sign(alpha) *
// ||x||, tau = (beta - alpha) / beta, v = x / (alpha - beta), then H = I - tau v v^T applied to
// the trailing columns; org2r: the reflectors applied backwards to the leading columns of the
// identity), so R carries LAPACK's signs.  The tiny-beta rescaling of dlarfg is not restated.
//
// Every reduction (column norms, v^T C) is a fixed-order tree over fixed row ranges, so repeated
// calls give the same bits.  Column-major blocks: element (r, c) at X[c * ld + r].
#include "common.h"
#include "kernels.h"

namespace b200 {
namespace {

constexpr int kHhThreads = 256;
constexpr int kHhRowsPerThread = 8;
constexpr int kHhRows = kHhThreads * kHhRowsPerThread;  // rows of one CTA in the reductions

// Fixed-order sum over the CTA: a shuffle tree per warp, then the warp sums in order by thread 0.
__device__ double block_sum(double v, double *red) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kHhThreads / 32; ++w) s += red[w];
  return s;  // valid on thread 0
}

// part[b] = sum of squares of X[r, j] over rows r in [j+1, n) of CTA b.
__global__ void __launch_bounds__(kHhThreads) hh_sumsq_kernel(const double *__restrict__ X, long long ld, int n,
                                                             int j, double *__restrict__ part) {
  __shared__ double red[kHhThreads / 32];
  const long long r0 = (long long)j + 1 + (long long)blockIdx.x * kHhRows;
  const double *x = X + (size_t)j * ld;
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < kHhRowsPerThread; ++i) {
    const long long r = r0 + threadIdx.x + (long long)i * kHhThreads;
    if (r < n) s = fma(x[r], x[r], s);
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// The reflector of column j (dlarfg): tau[j], scale[j] = 1 / (alpha - beta), and X[j, j] = beta.
__global__ void __launch_bounds__(kHhThreads) hh_reflector_kernel(double *__restrict__ X, long long ld, int j,
                                                                 const double *__restrict__ part, int nparts,
                                                                 double *__restrict__ tau,
                                                                 double *__restrict__ scale) {
  __shared__ double red[kHhThreads / 32];
  double s = 0.0;
  for (int b = threadIdx.x; b < nparts; b += kHhThreads) s += part[b];
  s = block_sum(s, red);
  if (threadIdx.x == 0) {
    double *xjj = X + (size_t)j * ld + j;
    const double alpha = *xjj, xnorm = sqrt(s);
    if (xnorm == 0.0) {
      tau[j] = 0.0;  // H = I, v left as it is
      scale[j] = 1.0;
    } else {
      const double beta = -copysign(hypot(alpha, xnorm), alpha);
      tau[j] = (beta - alpha) / beta;
      scale[j] = 1.0 / (alpha - beta);
      *xjj = beta;
    }
  }
}

// wpart[c * G + b] = sum over rows r in [j, n) of CTA b of v[r] * X[r, c], for c in (j, nc), with
// v = [1; X[j+1:n, j] * scale].  With store_v the scaled entries are written back (geqr2); without
// it X[j+1:n, j] already holds v (org2r) and scale is not read.
__global__ void __launch_bounds__(kHhThreads) hh_dot_kernel(double *__restrict__ X, long long ld, int n, int nc,
                                                           int j, const double *__restrict__ scale, int store_v,
                                                           double *__restrict__ wpart, int G) {
  __shared__ double red[kHhThreads / 32];
  const long long r0 = (long long)j + (long long)blockIdx.x * kHhRows;
  double *xj = X + (size_t)j * ld;
  const double sc = store_v ? scale[j] : 1.0;
  double v[kHhRowsPerThread];
#pragma unroll
  for (int i = 0; i < kHhRowsPerThread; ++i) {
    const long long r = r0 + threadIdx.x + (long long)i * kHhThreads;
    if (r == j) {
      v[i] = 1.0;
    } else if (r < n) {
      v[i] = store_v ? xj[r] * sc : xj[r];
      if (store_v) xj[r] = v[i];
    } else {
      v[i] = 0.0;
    }
  }
  for (int c = j + 1; c < nc; ++c) {
    const double *xc = X + (size_t)c * ld;
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < kHhRowsPerThread; ++i) {
      const long long r = r0 + threadIdx.x + (long long)i * kHhThreads;
      if (r < n) s = fma(v[i], xc[r], s);
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) wpart[(size_t)c * G + blockIdx.x] = s;
  }
}

// w[c] = sum of wpart[c * G + b] over b in order, for c in (j, nc).
__global__ void __launch_bounds__(kHhThreads) hh_w_kernel(const double *__restrict__ wpart, int G, int j, int nc,
                                                         double *__restrict__ w) {
  for (int c = j + 1 + threadIdx.x; c < nc; c += kHhThreads) {
    double s = 0.0;
    for (int b = 0; b < G; ++b) s += wpart[(size_t)c * G + b];
    w[c] = s;
  }
}

// X[r, c] -= tau v[r] w[c] for r in [j, n), c in (j, nc) (dlarf from the left; v[j] = 1).
__global__ void __launch_bounds__(kHhThreads) hh_update_kernel(double *__restrict__ X, long long ld, int n, int nc,
                                                              int j, const double *__restrict__ tau,
                                                              const double *__restrict__ w) {
  const long long r = (long long)j + (long long)blockIdx.x * kHhThreads + threadIdx.x;
  if (r >= n) return;
  const double t = tau[j];
  const double v = (r == j) ? 1.0 : X[(size_t)j * ld + r];
  for (int c = j + 1; c < nc; ++c) {
    double *x = X + (size_t)c * ld + r;
    *x = fma(v, -t * w[c], *x);
  }
}

// Column j of Q in org2r: rows above j zero, X[j, j] = 1 - tau, rows below scaled by -tau.
__global__ void __launch_bounds__(kHhThreads) hh_qcol_kernel(double *__restrict__ X, long long ld, int n, int j,
                                                            const double *__restrict__ tau) {
  const long long r = (long long)blockIdx.x * kHhThreads + threadIdx.x;
  if (r >= n) return;
  const double t = tau[j];
  double *x = X + (size_t)j * ld + r;
  if (r < j) *x = 0.0;
  else if (r == j) *x = 1.0 - t;
  else *x = -t * *x;
}

unsigned blocks_for(long long rows, int per) { return (unsigned)((rows + per - 1) / per); }

}  // namespace

int householder_qr_parts(int n) { return (int)blocks_for(n, kHhRows); }

// geqr2 of the n x nc block X (ld >= n), in place: R in the upper triangle, the reflectors below
// it, tau[0..nc).  work holds householder_qr_parts(n) * (nc + 1) + nc doubles and scale nc.
cudaError_t householder_qr_launch(double *X, long long ld, int n, int nc, double *tau, double *scale, double *work,
                                  cudaStream_t s) {
  const int P = householder_qr_parts(n);
  double *part = work, *wpart = work + P, *w = work + P + (size_t)P * nc;
  for (int j = 0; j < nc; ++j) {
    const int rows_below = n - j - 1;
    const int Gs = rows_below > 0 ? (int)blocks_for(rows_below, kHhRows) : 1;
    hh_sumsq_kernel<<<Gs, kHhThreads, 0, s>>>(X, ld, n, j, part);
    hh_reflector_kernel<<<1, kHhThreads, 0, s>>>(X, ld, j, part, Gs, tau, scale);
    count_launch();
    count_launch();
    if (j + 1 < nc) {
      const int G = (int)blocks_for((long long)n - j, kHhRows);
      hh_dot_kernel<<<G, kHhThreads, 0, s>>>(X, ld, n, nc, j, scale, 1, wpart, G);
      hh_w_kernel<<<1, kHhThreads, 0, s>>>(wpart, G, j, nc, w);
      hh_update_kernel<<<blocks_for((long long)n - j, kHhThreads), kHhThreads, 0, s>>>(X, ld, n, nc, j, tau, w);
      count_launch();
      count_launch();
      count_launch();
    } else {
      // the last column's v is still scaled into place (org2r reads it)
      const int G = (int)blocks_for((long long)n - j, kHhRows);
      hh_dot_kernel<<<G, kHhThreads, 0, s>>>(X, ld, n, nc, j, scale, 1, wpart, G);
      count_launch();
    }
  }
  return cudaGetLastError();
}

// org2r: overwrite the factored block with the n x nc orthonormal factor Q.
cudaError_t householder_q_launch(double *X, long long ld, int n, int nc, const double *tau, double *work,
                                 cudaStream_t s) {
  const int P = householder_qr_parts(n);
  double *wpart = work + P, *w = work + P + (size_t)P * nc;
  for (int j = nc - 1; j >= 0; --j) {
    if (j + 1 < nc) {
      const int G = (int)blocks_for((long long)n - j, kHhRows);
      hh_dot_kernel<<<G, kHhThreads, 0, s>>>(X, ld, n, nc, j, nullptr, 0, wpart, G);
      hh_w_kernel<<<1, kHhThreads, 0, s>>>(wpart, G, j, nc, w);
      hh_update_kernel<<<blocks_for((long long)n - j, kHhThreads), kHhThreads, 0, s>>>(X, ld, n, nc, j, tau, w);
      count_launch();
      count_launch();
      count_launch();
    }
    hh_qcol_kernel<<<blocks_for(n, kHhThreads), kHhThreads, 0, s>>>(X, ld, n, j, tau);
    count_launch();
  }
  return cudaGetLastError();
}

}  // namespace b200
