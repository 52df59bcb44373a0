// Strided, batched FP32 GEMM on the tcgen05 tensor cores for the neural-operator kernels (learned.cu):
//
//   C[z] = alpha * A[z] B[z] + beta * C[z],  A: m x k, B: k x n, C: m x n, element (i, j) of matrix z of
//   a view at p + z * bs + i * rs + j * cs (any strides: the transposed views of the backward pass too).
//
// The larger output dimension goes on the MMA's row side (C or C^T is computed).  A CTA of 128
// threads owns a TM x NT output tile (TM = 128, or 64 when the output has at most 64 rows; NT = 16,
// 32 or 64).  For each 32-deep K chunk the threads stage the A and B tiles into shared memory in the
// K-major, non-swizzled core-matrix layout (8 rows x 16 bytes per core matrix; LBO = 128 bytes
// between core matrices along K, SBO = 1024 bytes between 8-row groups; each warp store fills one
// whole core matrix, so the stores are free of bank conflicts), each value split into a TF32 high
// part (round to nearest) and the FP32 remainder; one thread issues, per 8-deep K step, three
// tcgen05.mma kind::tf32 products hi*hi + hi*lo + lo*hi into the FP32 accumulator in TMEM (the split
// keeps about 21 bits of every product: FP32-level results from TF32 tensor cores, the
// three-product TF32 emulation of FP32 GEMM).  Two shared stages: the next chunk is loaded into
// registers while the MMAs of the current one run, and split into the other stage once the MMAs
// two chunks back have committed.  The four warps then read the accumulator (tcgen05.ld) and apply
// alpha and beta.  Every wait is bounded.
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

// A thread's share of one operand chunk (R rows x kTcK depths) in registers.  The tile holds
// (R / 8) x (kTcK / 4) core matrices of 8 rows x 4 depths (128 contiguous bytes each); warp w takes
// core matrices q = 4 u + w, so each warp-wide store fills one whole core matrix (conflict-free),
// and lane l holds its element (rl, kl) -- rl = l % 8, kl = l / 8 when the rows have unit stride in
// global memory (8 consecutive rows = one 32-byte sector per depth), rl = l / 4, kl = l % 4 when the
// depths do (16 contiguous bytes per row).
template <int R>
struct Chunk {
  static constexpr int kKG = kTcK / 4;           // core matrices along the depth
  static constexpr int kPer = (R / 8) * kKG / 4;  // core matrices per warp
  float v[kPer];
  // global -> registers (zero outside rows x [k0, kend)); element (r, kk) at p[r * rs + kk * ks]
  __device__ __forceinline__ void load(const float *p, long long rs, long long ks, int r0, int rows, int k0,
                                       int kend) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool r_fast = rs == 1 && ks != 1;
    const int rl = r_fast ? (lane & 7) : (lane >> 2), kl = r_fast ? (lane >> 3) : (lane & 3);
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int q = 4 * u + warp;
      const int gr = r0 + (q / kKG) * 8 + rl, gk = k0 + (q % kKG) * 4 + kl;
      v[u] = (gr < rows && gk < kend) ? __ldg(p + gr * rs + gk * ks) : 0.f;
    }
  }
  // registers -> the hi / lo tiles (TF32 high part and FP32 remainder); byte offset of element
  // (rl, kl) of core matrix q: q * 128 + rl * 16 + kl * 4
  __device__ __forceinline__ void store(long long rs, long long ks, unsigned char *hi, unsigned char *lo) const {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool r_fast = rs == 1 && ks != 1;
    const int rl = r_fast ? (lane & 7) : (lane >> 2), kl = r_fast ? (lane >> 3) : (lane & 3);
    const uint32_t o0 = (uint32_t)(rl * 16 + kl * 4);
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const uint32_t o = (uint32_t)(4 * u + warp) * kCoreBytes + o0;
      const float h = tf32_hi(v[u]);
      *reinterpret_cast<float *>(hi + o) = h;
      *reinterpret_cast<float *>(lo + o) = v[u] - h;
    }
  }
};

// One TM x NT tile of the product for blockIdx.z = z * ksplit + part: depths [part * kper, +kper) of
// matrix z, written to C + blockIdx.z * bsc (ksplit = 1: the plain batched product).  Two shared
// stages: while the MMAs of chunk c read one stage, the threads load chunk c + 1 into registers and
// then (once the MMAs of chunk c - 1 have released it) split it into the other stage.  TM = 128: row
// i of the tile in TMEM lane i; TM = 64: rows 16w..16w+15 in lanes 32w..32w+15.
template <int TM, int NT>
__global__ void __launch_bounds__(kTcThreads) tc_sgemm_kernel(int m, int n, int k, int ksplit, int kper, float alpha,
                                                              View A, View B, float beta, float *C, long long rsc,
                                                              long long csc, long long bsc, int *err) {
  constexpr int kABytes = TM * kTcK * 4, kBBytes = NT * kTcK * 4, kStage = 2 * (kABytes + kBBytes);
  constexpr uint32_t kCols = NT < 32 ? 32 : NT;  // TMEM columns (a power of two >= 32)
  extern __shared__ unsigned char raw[];
  __shared__ __align__(8) uint64_t done[2];
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
  const uint32_t s0 = ptx::smem_u32(raw);
  unsigned char *sm = raw + ((128u - (s0 & 127u)) & 127u);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long zz = blockIdx.z, z = zz / ksplit;
  const int kbeg = (int)(zz % ksplit) * kper, kend = min(k, kbeg + kper);
  const int i0 = blockIdx.x * TM, j0 = blockIdx.y * NT;  // row tiles on x: up to 2^31 - 1
  const float *Ab = A.p + z * A.bs, *Bb = B.p + z * B.bs;
  if (threadIdx.x == 0) {
    ptx::mbar_init(&done[0], 1);
    ptx::mbar_init(&done[1], 1);
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
  constexpr uint32_t idesc = idesc_tf32_k(TM, NT);
  const int nch = kend > kbeg ? (kend - kbeg + kTcK - 1) / kTcK : 0;
  Chunk<TM> ra;
  Chunk<NT> rb;
  if (nch > 0) {
    ra.load(Ab, A.rs, A.cs, i0, m, kbeg, kend);
    rb.load(Bb, B.cs, B.rs, j0, n, kbeg, kend);
  }
  for (int ch = 0; ch < nch; ++ch) {
    const int st = ch & 1;
    unsigned char *Ahi = sm + st * kStage, *Alo = Ahi + kABytes, *Bhi = Alo + kABytes, *Blo = Bhi + kBBytes;
    if (ch >= 2 && !ptx::mbar_wait(&done[st], ((ch - 2) >> 1) & 1)) abort_flag = 1;  // chunk ch-2 released it
    __syncthreads();
    if (abort_flag) break;
    ra.store(A.rs, A.cs, Ahi, Alo);
    rb.store(B.cs, B.rs, Bhi, Blo);
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
      ptx::mma_commit(&done[st]);
    }
    if (ch + 1 < nch) {  // the next chunk's global loads overlap this chunk's MMAs
      const int k1 = kbeg + (ch + 1) * kTcK;
      ra.load(Ab, A.rs, A.cs, i0, m, k1, kend);
      rb.load(Bb, B.cs, B.rs, j0, n, k1, kend);
    }
  }
  // the last commit arrives after every earlier MMA of this thread has completed
  if (!abort_flag && nch > 0 && !ptx::mbar_wait(&done[(nch - 1) & 1], ((nch - 1) >> 1) & 1)) abort_flag = 1;
  __syncthreads();
  ptx::tc_fence_after();
  const bool live = TM == 128 || lane < 16;
  const int row = i0 + (TM == 128 ? warp * 32 + lane : warp * 16 + (lane & 15));
  const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
  float *Cr = C + zz * bsc + (long long)row * rsc;
  if (!abort_flag) {
#pragma unroll
    for (int c0 = 0; c0 < NT; c0 += 8) {
      float v[8];
      if (nch > 0) {
        ptx::tmem_ld8(tl + (uint32_t)c0, v);
        ptx::tmem_wait_ld();
      } else {
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = 0.f;  // an empty depth range: the product is zero
      }
      if (live && row < m) {
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

template <int TM, int NT>
cudaError_t launch_nt(cudaStream_t s, int zcount, int m, int n, int k, int ksplit, int kper, float alpha, View A,
                      View B, float beta, float *C, long long rsc, long long csc, long long bsc, int *err) {
  const int stages = kper <= kTcK ? 1 : 2;  // one chunk per CTA: the second stage would sit idle
  const size_t smem = (size_t)stages * 2 * (TM * kTcK * 4 + NT * kTcK * 4) + 128;
  cudaError_t e = cudaFuncSetAttribute(tc_sgemm_kernel<TM, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if ((n + NT - 1) / NT > 65535) return cudaErrorInvalidValue;
  const dim3 grid((m + TM - 1) / TM, (n + NT - 1) / NT, zcount);
  tc_sgemm_kernel<TM, NT><<<grid, kTcThreads, smem, s>>>(m, n, k, ksplit, kper, alpha, A, B, beta, C, rsc, csc, bsc,
                                                         err);
  count_launch();
  return cudaGetLastError();
}

template <int TM>
cudaError_t launch_tm(cudaStream_t s, int zcount, int m, int n, int k, int ksplit, int kper, float alpha, View A,
                      View B, float beta, float *C, long long rsc, long long csc, long long bsc, int *err) {
  if (n <= 16) return launch_nt<TM, 16>(s, zcount, m, n, k, ksplit, kper, alpha, A, B, beta, C, rsc, csc, bsc, err);
  if (n <= 32) return launch_nt<TM, 32>(s, zcount, m, n, k, ksplit, kper, alpha, A, B, beta, C, rsc, csc, bsc, err);
  return launch_nt<TM, 64>(s, zcount, m, n, k, ksplit, kper, alpha, A, B, beta, C, rsc, csc, bsc, err);
}

// 64-row tiles when the output has at most 64 rows (no MMA rows and staging spent on padding)
cudaError_t launch_any(cudaStream_t s, int zcount, int m, int n, int k, int ksplit, int kper, float alpha, View A,
                       View B, float beta, float *C, long long rsc, long long csc, long long bsc, int *err) {
  if (m <= 64) return launch_tm<64>(s, zcount, m, n, k, ksplit, kper, alpha, A, B, beta, C, rsc, csc, bsc, err);
  return launch_tm<128>(s, zcount, m, n, k, ksplit, kper, alpha, A, B, beta, C, rsc, csc, bsc, err);
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
  const int NT = n <= 16 ? 16 : n <= 32 ? 32 : 64, TM = m <= 64 ? 64 : kTcM;
  const long long tiles = (long long)((m + TM - 1) / TM) * ((n + NT - 1) / NT) * batch;
  const long long mn = (long long)m * n;
  // Split the depth when the tiles leave SMs idle and the depth is long: about four CTAs per SM,
  // at least 256 deep per split, within the workspace.
  int ksplit = 1;
  if (ws && k >= 512 && tiles < 4 * 148) {
    ksplit = (int)std::min<long long>((4 * 148 + tiles - 1) / tiles, k / 256);
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

extern "C" b200_status b200_tc_sgemm_async(int batch, int m, int n, int k, float alpha, const float *A, long long ars,
                                           long long acs, long long abs_, const float *B, long long brs, long long bcs,
                                           long long bbs, float beta, float *C, long long rsc, long long csc,
                                           long long bsc, int sum_batch, float *ws, size_t ws_floats, int *err,
                                           void *stream) {
  B200_ARG_CHECK(batch > 0 && m > 0 && n > 0 && k >= 0 && A && B && C && err, "invalid GEMM arguments");
  B200_ARG_CHECK(batch <= 65535 && (!sum_batch || ws), "batch above 65535, or sum_batch without a workspace");
  B200_CUDA_CHECK(tc_sgemm((cudaStream_t)stream, batch, m, n, k, alpha, A, ars, acs, abs_, B, brs, bcs, bbs, beta, C,
                           rsc, csc, bsc, err, ws, ws_floats, sum_batch != 0));
  return B200_OK;
}

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
