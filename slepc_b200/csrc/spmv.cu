// CSR sparse matrix-vector product y = A x in FP64 for sm_100a.
//
// Replaces PETSc's MATAIJCUSPARSE MatMult behind BVMatMultColumn
// (src/sys/classes/bv/interface/bvops.c:862-890).  Scheduling: a group of
// LPR lanes (1..32, a power of two chosen from the mean row length) owns one
// row; consecutive groups own consecutive rows, so a warp streams one
// contiguous range of the value/column arrays.  Values and column indices
// are read once with streaming (evict-first) loads; x goes through the
// read-only path because every entry is reused by its neighbouring rows.
#include "common.h"
#include "kernels.h"

namespace b200 {

template <int LPR>
__global__ void __launch_bounds__(256) spmv_csr_kernel(int n, const int *__restrict__ rowptr,
                                                       const int *__restrict__ colind,
                                                       const double *__restrict__ vals,
                                                       const double *__restrict__ x, double *__restrict__ y,
                                                       const GsState *__restrict__ st, int step) {
  if (st && st->halt && st->halt_step < step) return;
  constexpr int kRowsPerWarp = 32 / LPR;
  const int lane = threadIdx.x & (LPR - 1);
  const int warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int sub = (threadIdx.x & 31) / LPR;
  for (long long base = (long long)warp_global * kRowsPerWarp; base < n; base += (long long)nwarps * kRowsPerWarp) {
    const long long row = base + sub;
    double sum = 0.0;
    if (row < n) {
      const int rs = __ldg(rowptr + row);
      const int re = __ldg(rowptr + row + 1);
      for (int p = rs + lane; p < re; p += LPR) {
        const double a = __ldcs(vals + p);
        const int c = __ldcs(colind + p);
        sum = fma(a, __ldg(x + c), sum);
      }
    }
#pragma unroll
    for (int off = LPR / 2; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off, LPR);
    if (lane == 0 && row < n) y[row] = sum;
  }
}

int spmv_choose_lanes(int n, int64_t nnz) {
  if (n <= 0) return 1;
  const double avg = (double)nnz / (double)n;
  int lanes = 1;
  while (lanes < 32 && lanes < avg) lanes <<= 1;
  return lanes;
}

cudaError_t spmv_launch(int n, const int *rowptr, const int *colind, const double *vals, const double *x, double *y,
                        int lanes, cudaStream_t stream, const GsState *st, int step) {
  if (n <= 0) return cudaSuccess;
  const int threads = 256;
  const long long rows_per_block = threads / lanes;
  long long blocks = (n + rows_per_block - 1) / rows_per_block;
  if (blocks > (1ll << 20)) blocks = 1ll << 20;
  switch (lanes) {
#define B200_SPMV_CASE(L)                                                                                 \
  case L:                                                                                                 \
    spmv_csr_kernel<L><<<(unsigned)blocks, threads, 0, stream>>>(n, rowptr, colind, vals, x, y, st, step); \
    break;
    B200_SPMV_CASE(1)
    B200_SPMV_CASE(2)
    B200_SPMV_CASE(4)
    B200_SPMV_CASE(8)
    B200_SPMV_CASE(16)
    B200_SPMV_CASE(32)
#undef B200_SPMV_CASE
    default:
      return cudaErrorInvalidValue;
  }
  count_launch();
  return cudaGetLastError();
}

}  // namespace b200
