// Strided, batched FP32 GEMM on the tcgen05 tensor cores for the neural-operator kernels (learned.cu):
//
//   C[z] = alpha * A[z] B[z] + beta * C[z],  A: m x k, B: k x n, C: m x n, element (i, j) of matrix z of
//   a view at p + z * bs + i * rs + j * cs (any strides: the transposed views of the backward pass too).
//
// The larger output dimension goes on the 128-row MMA side (C or C^T is computed).  A CTA of 128
// threads owns a 128 x NT output tile (NT = 16..64).  For each 32-deep K chunk the threads stage the
// A and B tiles into shared memory in the K-major, non-swizzled core-matrix layout (8 rows x 16 bytes
// per core matrix; LBO = 128 bytes between core matrices along K, SBO = 1024 bytes between 8-row
// groups), each value split into a TF32 high part (round to nearest) and the FP32 remainder; one
// thread issues, per 8-deep K step, three tcgen05.mma kind::tf32 products hi*hi + hi*lo + lo*hi into
// the FP32 accumulator in TMEM (the split keeps about 21 bits of every product: FP32-level results
// from TF32 tensor cores, the three-product TF32 emulation of FP32 GEMM); the MMAs' commit releases
// the shared memory for the next chunk.  The four warps then read the accumulator (warp w owns TMEM
// lanes 32w..32w+31 = rows) and apply alpha and beta.  Every wait is bounded.
//
// When the tiles leave SMs idle and the depth is long (the weight gradients: 32 x 32 outputs over
// 262,144 grid points), the depth is split across CTAs into a workspace of partial tiles, and a
// second kernel sums them in a fixed order (optionally over the batch too): deterministic results.
#include <algorithm>
#include <utility>

#include <cuda.h>

#include "common.h"
#include "kernels.h"
#include "ptx.h"

namespace b200 {
namespace {

constexpr int kTcM = 128;       // rows of an output tile (MMA M)
constexpr int kTcK = 32;        // depth of a staged K chunk (4 MMA steps of 8)
constexpr int kTcThreads = 128;
constexpr int kCoreBytes = 128; // one core matrix: 8 rows x 16 bytes

struct View {
  const float *p;
  long long rs, cs, bs;
};

// Byte offset of element (row, kk) of a K-major, non-swizzled tile (K chunk of kTcK).
__device__ __forceinline__ uint32_t core_off(int row, int kk) {
  return (uint32_t)(((row >> 3) * (kTcK / 4) + (kk >> 2)) * kCoreBytes + (row & 7) * 16 + (kk & 3) * 4);
}

__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((kCoreBytes >> 4) & 0x3FFFu) << 16;                 // LBO: next core matrix along K
  d |= (uint64_t)(((kCoreBytes * kTcK / 4) >> 4) & 0x3FFFu) << 32;      // SBO: next 8-row group
  d |= (uint64_t)1 << 46;                                               // version; layout type 0 (no swizzle)
  return d;
}

__host__ __device__ constexpr uint32_t idesc_tf32_k(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Stages rows r0..r0+R-1 (of `rows`) and depths k0..kend-1 of the operand element (r, kk) at
// p[r * rs + kk * ks] into the hi / lo tiles, zero outside.  The loop runs along whichever of
// r and kk has unit stride, so the global reads coalesce for row- and column-major views.
template <int R>
__device__ __forceinline__ void stage_tile(const float *p, long long rs, long long ks, int r0, int rows, int k0,
                                           int kend, unsigned char *hi, unsigned char *lo) {
  const bool r_fast = rs == 1 && ks != 1;
  for (int e = threadIdx.x; e < R * kTcK; e += kTcThreads) {
    const int r = r_fast ? e % R : e / kTcK, kk = r_fast ? e / R : e % kTcK;
    const int gr = r0 + r, gk = k0 + kk;
    const float x = (gr < rows && gk < kend) ? __ldg(p + gr * rs + gk * ks) : 0.f;
    const float h = tf32_hi(x);
    const uint32_t o = core_off(r, kk);
    *reinterpret_cast<float *>(hi + o) = h;
    *reinterpret_cast<float *>(lo + o) = x - h;
  }
}


// One 128 x NT tile of the product for blockIdx.z = z * ksplit + part: depths [part * kper, +kper) of
// matrix z, written to C + blockIdx.z * bsc (ksplit = 1: the plain batched product).
template <int NT>
__global__ void __launch_bounds__(kTcThreads) tc_sgemm_kernel(int m, int n, int k, int ksplit, int kper, float alpha,
                                                              View A, View B, float beta, float *C, long long rsc,
                                                              long long csc, long long bsc, int *err) {
  constexpr int kABytes = kTcM * kTcK * 4, kBBytes = NT * kTcK * 4;
  constexpr uint32_t kCols = NT < 32 ? 32 : NT;  // TMEM columns (a power of two >= 32)
  extern __shared__ unsigned char raw[];
  __shared__ __align__(8) uint64_t done;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
  const uint32_t s0 = ptx::smem_u32(raw);
  unsigned char *sm = raw + ((128u - (s0 & 127u)) & 127u);
  unsigned char *Ahi = sm, *Alo = sm + kABytes, *Bhi = sm + 2 * kABytes, *Blo = sm + 2 * kABytes + kBBytes;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long zz = blockIdx.z, z = zz / ksplit;
  const int kbeg = (int)(zz % ksplit) * kper, kend = min(k, kbeg + kper);
  const int i0 = blockIdx.x * kTcM, j0 = blockIdx.y * NT;  // row tiles on x: up to 2^31 - 1
  const float *Ab = A.p + z * A.bs, *Bb = B.p + z * B.bs;
  if (threadIdx.x == 0) {
    ptx::mbar_init(&done, 1);
    abort_flag = 0;
    ptx::fence_mbar_init();
  }
  if (warp == 0) {
    ptx::tmem_alloc(&tmem_base, kCols);
    ptx::tmem_relinquish();
  }
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem = tmem_base;
  constexpr uint32_t idesc = idesc_tf32_k(kTcM, NT);
  int ch = 0;
  for (int k0 = kbeg; k0 < kend; k0 += kTcK, ++ch) {
    stage_tile<kTcM>(Ab, A.rs, A.cs, i0, m, k0, kend, Ahi, Alo);
    stage_tile<NT>(Bb, B.cs, B.rs, j0, n, k0, kend, Bhi, Blo);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic-proxy stores -> MMA reads
    __syncthreads();
    if (threadIdx.x == 0) {
      ptx::tc_fence_after();
      const uint32_t ah = ptx::smem_u32(Ahi), al = ptx::smem_u32(Alo), bh = ptx::smem_u32(Bhi), bl = ptx::smem_u32(Blo);
#pragma unroll
      for (int s = 0; s < kTcK / 8; ++s) {
        const uint32_t ko = (uint32_t)s * 2 * kCoreBytes;  // two core matrices per 8-deep step
        ptx::mma_tf32(tmem, desc_kmajor(ah + ko), desc_kmajor(bh + ko), idesc, ch > 0 || s > 0);
        ptx::mma_tf32(tmem, desc_kmajor(ah + ko), desc_kmajor(bl + ko), idesc, true);
        ptx::mma_tf32(tmem, desc_kmajor(al + ko), desc_kmajor(bh + ko), idesc, true);
      }
      ptx::mma_commit(&done);
    }
    if (!ptx::mbar_wait(&done, ch & 1)) abort_flag = 1;  // the MMAs have read the tiles
    __syncthreads();
    if (abort_flag) break;
  }
  ptx::tc_fence_after();
  const int row = i0 + warp * 32 + lane;
  const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
  float *Cr = C + zz * bsc + (long long)row * rsc;
  if (!abort_flag) {
#pragma unroll
    for (int c0 = 0; c0 < NT; c0 += 8) {
      float v[8];
      if (ch > 0) {
        ptx::tmem_ld8(tl + (uint32_t)c0, v);
        ptx::tmem_wait_ld();
      } else {
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = 0.f;  // an empty depth range: the product is zero
      }
      if (row < m) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int j = j0 + c0 + u;
          if (j < n) {
            float *cp = Cr + (long long)j * csc;
            *cp = beta != 0.f ? alpha * v[u] + beta * *cp : alpha * v[u];
          }
        }
      }
    }
  }
  if (abort_flag && threadIdx.x == 0) atomicOr(err, kDevErrTimeout);
  ptx::tc_fence_before();
  __syncthreads();
  if (warp == 0) ptx::tmem_dealloc(tmem, kCols);
}

// C[g] = alpha * sum_{s < per} W[g * per + s] + beta * C[g], W dense m x n slots summed in slot order.
__global__ void tc_reduce_kernel(const float *__restrict__ W, int m, int n, int groups, int per, float alpha,
                                 float beta, float *C, long long rsc, long long csc, long long bsc) {
  const long long mn = (long long)m * n, total = mn * groups;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const long long g = t / mn, e = t % mn;
    const float *w = W + g * per * mn + e;
    float acc = 0.f;
    for (int s = 0; s < per; ++s) acc += w[s * mn];
    float *cp = C + g * bsc + (e / n) * rsc + (e % n) * csc;
    *cp = beta != 0.f ? alpha * acc + beta * *cp : alpha * acc;
  }
}

template <int NT>
cudaError_t launch_nt(cudaStream_t s, int zcount, int m, int n, int k, int ksplit, int kper, float alpha, View A,
                      View B, float beta, float *C, long long rsc, long long csc, long long bsc, int *err) {
  const size_t smem = (size_t)(2 * kTcM * kTcK * 4 + 2 * NT * kTcK * 4) + 128;
  cudaError_t e = cudaFuncSetAttribute(tc_sgemm_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if ((n + NT - 1) / NT > 65535) return cudaErrorInvalidValue;
  const dim3 grid((m + kTcM - 1) / kTcM, (n + NT - 1) / NT, zcount);
  tc_sgemm_kernel<NT><<<grid, kTcThreads, smem, s>>>(m, n, k, ksplit, kper, alpha, A, B, beta, C, rsc, csc, bsc, err);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_any(cudaStream_t s, int zcount, int m, int n, int k, int ksplit, int kper, float alpha, View A,
                       View B, float beta, float *C, long long rsc, long long csc, long long bsc, int *err) {
  if (n <= 16) return launch_nt<16>(s, zcount, m, n, k, ksplit, kper, alpha, A, B, beta, C, rsc, csc, bsc, err);
  if (n <= 32) return launch_nt<32>(s, zcount, m, n, k, ksplit, kper, alpha, A, B, beta, C, rsc, csc, bsc, err);
  return launch_nt<64>(s, zcount, m, n, k, ksplit, kper, alpha, A, B, beta, C, rsc, csc, bsc, err);
}

}  // namespace

cudaError_t tc_sgemm(cudaStream_t s, int batch, int m, int n, int k, float alpha, const float *A, long long ars,
                     long long acs, long long abs_, const float *B, long long brs, long long bcs, long long bbs,
                     float beta, float *C, long long rsc, long long csc, long long bsc, int *err, float *ws,
                     size_t ws_floats, bool sum_batch) {
  if (batch <= 0 || m <= 0 || n <= 0) return cudaSuccess;
  if (!err || (sum_batch && !ws)) return cudaErrorInvalidValue;
  View Av{A, ars, acs, abs_}, Bv{B, brs, bcs, bbs};
  if (m < n) {  // C^T = B^T A^T: the larger output dimension on the 128-row side
    std::swap(m, n);
    std::swap(rsc, csc);
    const View t{Bv.p, Bv.cs, Bv.rs, Bv.bs};
    Bv = View{Av.p, Av.cs, Av.rs, Av.bs};
    Av = t;
  }
  const int NT = n <= 16 ? 16 : n <= 32 ? 32 : 64;
  const long long tiles = (long long)((m + kTcM - 1) / kTcM) * ((n + NT - 1) / NT) * batch;
  const long long mn = (long long)m * n;
  // Split the depth when the tiles leave SMs idle and the depth is long: about two CTAs per SM,
  // at least 128 deep per split, within the workspace.
  int ksplit = 1;
  if (ws && k >= 256 && tiles < 2 * 148) {
    ksplit = (int)std::min<long long>((2 * 148 + tiles - 1) / tiles, k / 128);
    ksplit = (int)std::min<long long>(ksplit, (long long)(ws_floats / (mn * batch)));
    if (ksplit < 1) ksplit = 1;
  }
  if (ksplit == 1 && !sum_batch) {
    if (batch > 65535) return cudaErrorInvalidValue;
    return launch_any(s, batch, m, n, k, 1, k, alpha, Av, Bv, beta, C, rsc, csc, bsc, err);
  }
  if ((long long)batch * ksplit > 65535 || (size_t)(mn * batch * ksplit) > ws_floats) return cudaErrorInvalidValue;
  const int kper = ((k + ksplit - 1) / ksplit + kTcK - 1) / kTcK * kTcK;
  cudaError_t e = launch_any(s, batch * ksplit, m, n, k, ksplit, kper, 1.f, Av, Bv, 0.f, ws, n, 1, mn, err);
  if (e != cudaSuccess) return e;
  const int groups = sum_batch ? 1 : batch, per = sum_batch ? batch * ksplit : ksplit;
  const long long total = mn * groups;
  const unsigned grid = (unsigned)std::min<long long>((total + 255) / 256, 148 * 8);
  tc_reduce_kernel<<<grid, 256, 0, s>>>(ws, m, n, groups, per, alpha, beta, C, rsc, csc, bsc);
  count_launch();
  return cudaGetLastError();
}

}  // namespace b200

using namespace b200;

extern "C" b200_status b200_tc_sgemm(int batch, int m, int n, int k, float alpha, const float *A, long long ars,
                                     long long acs, long long abs_, const float *B, long long brs, long long bcs,
                                     long long bbs, float beta, float *C, long long rsc, long long csc, long long bsc,
                                     int split, int sum_batch, void *stream) {
  B200_ARG_CHECK(batch > 0 && m > 0 && n > 0 && k >= 0 && A && B && C, "invalid GEMM arguments");
  B200_ARG_CHECK(batch <= 65535, "batch above 65535");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t ws_len = (split || sum_batch) ? (size_t)m * n * batch * 64 : 0;
  float *ws = nullptr;
  int *err = nullptr;
  B200_CUDA_CHECK(cudaMalloc(&err, sizeof(int)));
  if (ws_len && cudaMalloc(&ws, sizeof(float) * ws_len) != cudaSuccess) {
    cudaFree(err);
    b200_set_last_error(__FILE__, __LINE__, "cudaMalloc failed for the GEMM workspace");
    return B200_ERR_NOMEM;
  }
  cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), s);
  if (e == cudaSuccess)
    e = tc_sgemm(s, batch, m, n, k, alpha, A, ars, acs, abs_, B, brs, bcs, bbs, beta, C, rsc, csc, bsc, err, ws, ws_len,
                 sum_batch != 0);
  int herr = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(ws);
  cudaFree(err);
  B200_CUDA_CHECK(e);
  if (herr) {
    b200_set_last_error(__FILE__, __LINE__, "the GEMM kernel reported a device-side timeout");
    return B200_ERR_DEVICE;
  }
  return B200_OK;
}
