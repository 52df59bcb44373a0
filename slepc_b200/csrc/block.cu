// Block SpMV with a fused three-term update for sm_100a, FP64:
//
//   Out(:,b) = alpha * (A Y(:,b) - shift * Y(:,b)) - beta * X(:,b),   b < nb
//
// One step of the scaled Chebyshev recurrence of a polynomial-filtered
// subspace iteration (Zhou and Saad, "A Chebyshev-Davidson algorithm for large
// symmetric eigenproblems", SIAM J. Matrix Anal. Appl. 29 (2007); the
// three-term form of their Algorithm "Chebyshev filter, scaled"), and with
// alpha = 1, shift = beta = 0 the plain block product A Y of a Rayleigh-Ritz
// step.  It is the FP64 refinement phase of the mixed-precision solver.
//
// Layout: the sliced-ELL copy of the matrix (32-row slices, column-major in
// the slice) that the single-vector SpMV uses; lane i of a warp owns row
// 32s+i of slice s and sums its products in index order.  The matrix is read
// once per block.  Rows longer than a slice admits are listed in rest_rows and
// done by one warp each (lanes stride the row, fixed shuffle tree per column,
// 8 columns per pass over the row).
#include "common.h"
#include "kernels.h"

namespace b200 {
namespace {

constexpr int kBlockThreads = 256;
constexpr int kGroup = 8;  // columns of the block per pass over a long row
constexpr int kChunk = 8;  // nonzeros of a slice row held in registers
constexpr int kCols = 2;   // block columns whose gathers are issued together (80 registers, 3 CTAs per SM)

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Lane i of the warp owning slice s keeps the (up to kChunk) nonzeros of row 32s+i in registers and
// then streams over the columns of the block, CB columns at a time: the gathers of those columns
// are all issued before any sum, so a warp keeps CB * kChunk loads in flight.  Rows wider than
// kChunk take several chunks, the partial sums passing through Out (the same warp owns the row
// throughout).  Each row's products are rounded and summed in index order, as the single-vector
// sliced-ELL SpMV does, so a column of the result has the same bits as that SpMV.
template <typename VT, int CB>
__global__ void __launch_bounds__(kBlockThreads, 3) spmm_sell_kernel(int nslices, int n, const long long *__restrict__ off,
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
    const int rr = r < n ? r : n - 1;  // rows past n read a valid row (their results are not written)
    const int wc = w > 0 ? w : 1;      // an empty slice still writes its rows' affine part
    for (int k0 = 0; k0 < wc; k0 += kChunk) {
      double a[kChunk];
      int c[kChunk];
#pragma unroll
      for (int u = 0; u < kChunk; ++u) {
        const bool in = k0 + u < w;
        c[u] = in ? __ldcs(scol + base + 32ll * (k0 + u)) : -1;
        a[u] = in ? (double)__ldcs(sval + base + 32ll * (k0 + u)) : 0.0;
      }
      const bool first = k0 == 0, last = k0 + kChunk >= wc;
      for (int b0 = 0; b0 < nb; b0 += CB) {
        double y[CB][kChunk];
#pragma unroll
        for (int j = 0; j < CB; ++j) {
          const double *Yb = Y + (size_t)min(b0 + j, nb - 1) * ld;
#pragma unroll
          for (int u = 0; u < kChunk; ++u) y[j][u] = c[u] >= 0 ? __ldg(Yb + c[u]) : 0.0;
        }
#pragma unroll
        for (int j = 0; j < CB; ++j) {
          const int b = b0 + j;
          if (b >= nb) break;
          const size_t idx = (size_t)b * ld + rr;
          double acc = (!first && mine) ? Out[idx] : 0.0;
#pragma unroll
          for (int u = 0; u < kChunk; ++u)
            if (c[u] >= 0) acc = __dadd_rn(acc, __dmul_rn(a[u], y[j][u]));
          if (mine) {
            if (last) {
              double v = alpha * (acc - shift * Y[idx]);
              if (X) v -= beta * X[idx];
              Out[idx] = v;
            } else {
              Out[idx] = acc;
            }
          }
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
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spmm_sell_kernel<VT, kCols>, kBlockThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rows_per_sm, spmm_rows_kernel<VT>, kBlockThreads, 0);
    if (per_sm <= 0) per_sm = 1;
    if (rows_per_sm <= 0) rows_per_sm = 1;
  }
  const int wpc = kBlockThreads / 32;
  if (S.nslices > 0) {
    int grid = (S.nslices + wpc - 1) / wpc;
    if (grid > sms * per_sm) grid = sms * per_sm;
    spmm_sell_kernel<VT, kCols><<<grid, kBlockThreads, 0, stream>>>(S.nslices, n, S.off, S.width, S.mask,
                                                                    static_cast<const VT *>(S.vals), S.cols, Y, X,
                                                                    Out, ld, nb, alpha, shift, beta);
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
