// Explicit transpose of a CSR matrix in HBM, in the layout MatTranspose_SeqAIJ
// produces: row c of A^T lists the rows i of A with a nonzero in column c in
// ascending i.  Used for the A^T that SVDSetUp builds for the cross solver
// (src/svd/interface/svdsetup.c:300-314).
//
// The nonzeros of A are in row-major order, so a stable sort of the pairs
// (column, position) by column gives every row of A^T in ascending row order
// of A.  The sort is CUB's LSD radix sort (stable and deterministic); the
// row pointer of A^T is a column histogram plus a prefix sum, and the
// row index of each sorted nonzero is a binary search of A's row pointer.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "common.h"
#include "kernels.h"

namespace b200 {
namespace {

__global__ void iota_copy_kernel(long long nnz, const int *__restrict__ colind, int *__restrict__ keys,
                                 int *__restrict__ pos) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += (long long)gridDim.x * blockDim.x) {
    keys[p] = colind[p];
    pos[p] = (int)p;
  }
}

__global__ void column_count_kernel(long long nnz, const int *__restrict__ colind, int *__restrict__ counts) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += (long long)gridDim.x * blockDim.x)
    atomicAdd(counts + colind[p], 1);
}

// colind_t[k] = row of A holding nonzero pos[k]; vals_t[k] = vals[pos[k]]
template <typename VT>
__global__ void gather_transpose_kernel(long long nnz, int rows, const int *__restrict__ rowptr,
                                        const int *__restrict__ pos, const VT *__restrict__ vals,
                                        int *__restrict__ colind_t, VT *__restrict__ vals_t) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += (long long)gridDim.x * blockDim.x) {
    const int p = pos[k];
    // largest i with rowptr[i] <= p
    int lo = 0, hi = rows;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(rowptr + mid) <= p) lo = mid;
      else hi = mid;
    }
    colind_t[k] = lo;
    vals_t[k] = vals[p];
  }
}

unsigned grid_of(long long len) {
  const long long g = (len + 255) / 256;
  return (unsigned)(g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16);
}

int bits_for(int cols) {
  int b = 1;
  while (b < 31 && (1 << b) < cols) ++b;
  return b;
}

}  // namespace

cudaError_t csr_transpose_device(int rows, int cols, long long nnz, const int *rowptr, const int *colind,
                                 const void *vals, bool f32, int *rowptr_t, int *colind_t, void *vals_t,
                                 cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(rowptr_t, 0, sizeof(int) * ((size_t)cols + 1), s);
  if (e != cudaSuccess || nnz == 0) return e;
  int *keys[2] = {nullptr, nullptr}, *pos[2] = {nullptr, nullptr};
  void *temp = nullptr;
  size_t temp_bytes = 0, scan_bytes = 0;
  const unsigned grid = grid_of(nnz);
  do {
    if ((e = cudaMalloc(&keys[0], sizeof(int) * nnz)) != cudaSuccess) break;
    if ((e = cudaMalloc(&keys[1], sizeof(int) * nnz)) != cudaSuccess) break;
    if ((e = cudaMalloc(&pos[0], sizeof(int) * nnz)) != cudaSuccess) break;
    if ((e = cudaMalloc(&pos[1], sizeof(int) * nnz)) != cudaSuccess) break;
    iota_copy_kernel<<<grid, 256, 0, s>>>(nnz, colind, keys[0], pos[0]);
    count_launch();
    // counts in rowptr_t[1..cols], then an in-place inclusive scan gives the row pointer
    column_count_kernel<<<grid, 256, 0, s>>>(nnz, colind, rowptr_t + 1);
    count_launch();
    cub::DoubleBuffer<int> k(keys[0], keys[1]), v(pos[0], pos[1]);
    const int end_bit = bits_for(cols);
    if ((e = cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, k, v, (int)nnz, 0, end_bit, s)) != cudaSuccess)
      break;
    if ((e = cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, rowptr_t + 1, rowptr_t + 1, cols, s)) !=
        cudaSuccess)
      break;
    if (scan_bytes > temp_bytes) temp_bytes = scan_bytes;
    if ((e = cudaMalloc(&temp, temp_bytes)) != cudaSuccess) break;
    size_t tb = temp_bytes;
    if ((e = cub::DeviceRadixSort::SortPairs(temp, tb, k, v, (int)nnz, 0, end_bit, s)) != cudaSuccess) break;
    count_launch();
    tb = temp_bytes;
    if ((e = cub::DeviceScan::InclusiveSum(temp, tb, rowptr_t + 1, rowptr_t + 1, cols, s)) != cudaSuccess) break;
    count_launch();
    if (f32)
      gather_transpose_kernel<float><<<grid, 256, 0, s>>>(nnz, rows, rowptr, v.Current(),
                                                           static_cast<const float *>(vals), colind_t,
                                                           static_cast<float *>(vals_t));
    else
      gather_transpose_kernel<double><<<grid, 256, 0, s>>>(nnz, rows, rowptr, v.Current(),
                                                            static_cast<const double *>(vals), colind_t,
                                                            static_cast<double *>(vals_t));
    count_launch();
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  } while (0);
  cudaFree(keys[0]);
  cudaFree(keys[1]);
  cudaFree(pos[0]);
  cudaFree(pos[1]);
  cudaFree(temp);
  return e;
}

}  // namespace b200
