// Block SpMV with a fused three-term update for sm_100a, FP64:
//
//   Out(:,b) = alpha * (A Y(:,b) - shift * Y(:,b)) - beta * X(:,b),   b < nb
//
// One step of the scaled Chebyshev recurrence of a polynomial-filtered
// subspace iteration (Zhou and Saad, "A Chebyshev-Davidson algorithm for large
// symmetric eigenproblems", SIAM J. Matrix Anal. Appl. 29 (2007); the
// three-term form of their Algorithm "Chebyshev filter, scaled"), and with
// alpha = 1, shift = beta = 0 the plain block product A Y of a Rayleigh-Ritz
// step.  It is the FP64 refinement phase of the mixed-precision solver: the
// matrix is read once per group of 8 columns of the block instead of once per
// column.
//
// Layout: the sliced-ELL copy of the matrix (32-row slices, column-major in
// the slice) that the single-vector SpMV uses; lane i of a warp owns row
// 32s+i of slice s, sums its products in index order, and keeps the 8 column
// sums of its row in registers.  Rows longer than a slice admits are listed in
// rest_rows and done by one warp each (lanes stride the row, fixed shuffle
// tree per column).
#include "common.h"
#include "kernels.h"

namespace b200 {
namespace {

constexpr int kBlockThreads = 256;
constexpr int kGroup = 8;  // columns of the block per pass over a slice

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

template <typename VT>
__global__ void __launch_bounds__(kBlockThreads) spmm_sell_kernel(int nslices, int n, const long long *__restrict__ off,
                                                                  const int *__restrict__ width,
                                                                  const unsigned *__restrict__ mask,
                                                                  const VT *__restrict__ sval,
                                                                  const int *__restrict__ scol,
                                                                  const double *__restrict__ Y,
                                                                  const double *__restrict__ X,
                                                                  double *__restrict__ Out, int ld, int nb,
                                                                  double alpha, double shift, double beta) {
  const int lane = threadIdx.x & 31;
  const int nwarps = gridDim.x * (kBlockThreads / 32);
  for (int sl = blockIdx.x * (kBlockThreads / 32) + (threadIdx.x >> 5); sl < nslices; sl += nwarps) {
    const long long base = off[sl] + lane;
    const int w = width[sl];
    const int r = 32 * sl + lane;
    const bool mine = r < n && ((mask[sl] >> lane) & 1u);
    for (int g0 = 0; g0 < nb; g0 += kGroup) {
      const int gn = min(kGroup, nb - g0);
      const double *Yg = Y + (size_t)g0 * ld;
      double acc[kGroup];
#pragma unroll
      for (int b = 0; b < kGroup; ++b) acc[b] = 0.0;
      for (int k0 = 0; k0 < w; k0 += 8) {
        VT a[8];
        int c[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const bool in = k0 + u < w;
          c[u] = in ? __ldg(scol + base + 32ll * (k0 + u)) : -1;
          a[u] = in ? __ldg(sval + base + 32ll * (k0 + u)) : VT(0);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          if (c[u] < 0) continue;
          const double av = (double)a[u];
#pragma unroll
          for (int b = 0; b < kGroup; ++b)
            if (b < gn) acc[b] = __dadd_rn(acc[b], __dmul_rn(av, __ldg(Yg + (size_t)b * ld + c[u])));
        }
      }
      if (mine) {
#pragma unroll
        for (int b = 0; b < kGroup; ++b) {
          if (b >= gn) break;
          const size_t idx = (size_t)(g0 + b) * ld + r;
          double v = alpha * (acc[b] - shift * Y[idx]);
          if (X) v -= beta * X[idx];
          Out[idx] = v;
        }
      }
    }
  }
}

template <typename VT>
__global__ void __launch_bounds__(kBlockThreads) spmm_rows_kernel(int nrows, const int *__restrict__ rows,
                                                                  const int *__restrict__ rowptr,
                                                                  const int *__restrict__ colind,
                                                                  const VT *__restrict__ vals,
                                                                  const double *__restrict__ Y,
                                                                  const double *__restrict__ X,
                                                                  double *__restrict__ Out, int ld, int nb,
                                                                  double alpha, double shift, double beta) {
  const int lane = threadIdx.x & 31;
  const int nwarps = gridDim.x * (kBlockThreads / 32);
  for (int i = blockIdx.x * (kBlockThreads / 32) + (threadIdx.x >> 5); i < nrows; i += nwarps) {
    const int r = rows[i];
    const int p0 = rowptr[r], p1 = rowptr[r + 1];
    for (int g0 = 0; g0 < nb; g0 += kGroup) {
      const int gn = min(kGroup, nb - g0);
      const double *Yg = Y + (size_t)g0 * ld;
      double acc[kGroup];
#pragma unroll
      for (int b = 0; b < kGroup; ++b) acc[b] = 0.0;
      for (int p = p0 + lane; p < p1; p += 32) {
        const int c = __ldg(colind + p);
        const double av = (double)__ldg(vals + p);
#pragma unroll
        for (int b = 0; b < kGroup; ++b)
          if (b < gn) acc[b] = fma(av, __ldg(Yg + (size_t)b * ld + c), acc[b]);
      }
#pragma unroll
      for (int b = 0; b < kGroup; ++b) acc[b] = warp_sum(acc[b]);
      if (lane == 0) {
        for (int b = 0; b < gn; ++b) {
          const size_t idx = (size_t)(g0 + b) * ld + r;
          double v = alpha * (acc[b] - shift * Y[idx]);
          if (X) v -= beta * X[idx];
          Out[idx] = v;
        }
      }
    }
  }
}

template <typename VT>
cudaError_t spmm_sell_launch_t(const SpmvSell &S, int n, const int *rowptr, const int *colind, const VT *vals,
                               const double *Y, const double *X, double *Out, int ld, int nb, double alpha,
                               double shift, double beta, cudaStream_t stream) {
  static int sms = 0, per_sm = 0, rows_per_sm = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spmm_sell_kernel<VT>, kBlockThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rows_per_sm, spmm_rows_kernel<VT>, kBlockThreads, 0);
    if (per_sm <= 0) per_sm = 1;
    if (rows_per_sm <= 0) rows_per_sm = 1;
  }
  const int wpc = kBlockThreads / 32;
  if (S.nslices > 0) {
    int grid = (S.nslices + wpc - 1) / wpc;
    if (grid > sms * per_sm) grid = sms * per_sm;
    spmm_sell_kernel<VT><<<grid, kBlockThreads, 0, stream>>>(S.nslices, n, S.off, S.width, S.mask,
                                                             static_cast<const VT *>(S.vals), S.cols, Y, X, Out, ld,
                                                             nb, alpha, shift, beta);
    count_launch();
  }
  if (S.nrest > 0) {
    int grid = (S.nrest + wpc - 1) / wpc;
    if (grid > sms * rows_per_sm) grid = sms * rows_per_sm;
    spmm_rows_kernel<VT><<<grid, kBlockThreads, 0, stream>>>(S.nrest, S.rest_rows, rowptr, colind, vals, Y, X, Out, ld,
                                                             nb, alpha, shift, beta);
    count_launch();
  }
  return cudaGetLastError();
}

}  // namespace

cudaError_t spmm_sell_launch(const SpmvSell &S, int n, const int *rowptr, const int *colind, const void *vals, bool f32,
                             const double *Y, const double *X, double *Out, int ld, int nb, double alpha, double shift,
                             double beta, cudaStream_t stream) {
  if (nb <= 0 || n <= 0) return cudaSuccess;
  if (f32)
    return spmm_sell_launch_t<float>(S, n, rowptr, colind, static_cast<const float *>(vals), Y, X, Out, ld, nb, alpha,
                                     shift, beta, stream);
  return spmm_sell_launch_t<double>(S, n, rowptr, colind, static_cast<const double *>(vals), Y, X, Out, ld, nb, alpha,
                                    shift, beta, stream);
}

}  // namespace b200
