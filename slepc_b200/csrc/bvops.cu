// Dense tall-skinny BV operations in FP64 for sm_100a.
//
//   multinplace  BVMultInPlace   (src/sys/classes/bv/interface/bvops.c:220-245;
//                                 GPU reference bvcuda.cu:65-112: cudaMalloc of an
//                                 n x (e-s) temporary, cuBLAS DGEMM, cudaMemcpy2D back)
//                Here: a persistent row-blocked kernel.  Each CTA keeps Q(l:k,s:e) in
//                shared memory, loads a 64-row panel of V(:,l:k) into shared memory,
//                computes the 64 x (e-s) product with a register tile, and writes it
//                back over V(:,s:e) of the same rows.  Rows are disjoint across CTAs and
//                a panel is read completely before any of its rows is written, so the
//                update is safely in place with no temporary.
//   mult         BVMult          (bvops.c:47-85)
//   multvec      BVMultVec       (bvops.c:96-134)
//   dot          BVDot           (bvglobal.c)
//   sumsq        BVNorm(NORM_2 / NORM_FROBENIUS) building block, deterministic
//   residual     EPSComputeResidualNorm_Private (src/eps/interface/epssolve.c:666-722):
//                SpMV fused with r = Ax - lambda x and its sum of squares
//   random       stand-in for BVSetRandomColumn (bvops.c:360-379)
#include <cuda.h>
#include <cudaTypedefs.h>

#include <atomic>

#include "common.h"
#include "kernels.h"

namespace b200 {
namespace {

constexpr int kRB = 64;        // rows per panel of the in-place GEMM
constexpr int kGemmThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Y(:,0:nc) = X(:,0:kq) * Q(0:kq,0:nc) ; MAXJ = ceil(nc/16) <= 8.  X and Y may overlap (the
// in-place V(:,s:e) = V(:,l:k) Q(l:k,s:e) of BVMultInPlace): a panel of X is read completely before
// any of its rows is written.  TI / TO are the stored types of X and Y (double, or float for the
// FP32 basis of the mixed-precision solver); products and sums are FP64.
template <int MAXJ, typename TI, typename TO>
__global__ void __launch_bounds__(kGemmThreads) panel_gemm_kernel(const TI *X, int ldx, TO *Y, int ldy, int n, int kq,
                                                                  const double *__restrict__ Q, int ldq, int nc,
                                                                  double alpha, double beta) {
  extern __shared__ __align__(16) double sm[];
  double *Qs = sm;                          // [kq][nc] row-major by c: Qs[c*nc + j]
  double *As = sm + (size_t)kq * nc;        // input panel As[c*kRB + r]; then output tile Os[j*(kRB+1) + r]
  const int tid = threadIdx.x;
  for (int idx = tid; idx < kq * nc; idx += kGemmThreads) {
    const int c = idx / nc, j = idx - c * nc;
    Qs[idx] = Q[(size_t)c + (size_t)j * ldq];
  }
  const int cg = tid & 15;   // column group: columns cg + 16*jj
  const int rg = tid >> 4;   // row group: rows rg + 16*ii
  const int npanels = (n + kRB - 1) / kRB;
  for (int pnl = blockIdx.x; pnl < npanels; pnl += gridDim.x) {
    const long long r0 = (long long)pnl * kRB;
    const int rows = (int)min((long long)kRB, (long long)n - r0);
    __syncthreads();
    for (int idx = tid; idx < kq * kRB; idx += kGemmThreads) {
      const int c = idx / kRB, r = idx - c * kRB;
      As[idx] = (r < rows) ? (double)X[(size_t)c * ldx + r0 + r] : 0.0;
    }
    __syncthreads();
    double acc[4][MAXJ];
#pragma unroll
    for (int ii = 0; ii < 4; ++ii)
#pragma unroll
      for (int jj = 0; jj < MAXJ; ++jj) acc[ii][jj] = 0.0;
    for (int c = 0; c < kq; ++c) {
      double a[4], q[MAXJ];
#pragma unroll
      for (int ii = 0; ii < 4; ++ii) a[ii] = As[c * kRB + rg + 16 * ii];
#pragma unroll
      for (int jj = 0; jj < MAXJ; ++jj) {
        const int j = cg + 16 * jj;
        q[jj] = (j < nc) ? Qs[c * nc + j] : 0.0;
      }
#pragma unroll
      for (int ii = 0; ii < 4; ++ii)
#pragma unroll
        for (int jj = 0; jj < MAXJ; ++jj) acc[ii][jj] = fma(a[ii], q[jj], acc[ii][jj]);
    }
    __syncthreads();  // panel fully consumed: reuse its space as the output tile, padded to kRB+1 per column
#pragma unroll
    for (int ii = 0; ii < 4; ++ii)
#pragma unroll
      for (int jj = 0; jj < MAXJ; ++jj) {
        const int j = cg + 16 * jj;
        if (j < nc) As[j * (kRB + 1) + rg + 16 * ii] = acc[ii][jj];
      }
    __syncthreads();
    for (int idx = tid; idx < nc * kRB; idx += kGemmThreads) {
      const int j = idx / kRB, r = idx - j * kRB;
      if (r < rows) {
        TO *y = Y + (size_t)j * ldy + r0 + r;
        const double v = As[j * (kRB + 1) + r];
        *y = (TO)(beta == 0.0 ? alpha * v : alpha * v + beta * (double)*y);
      }
    }
  }
}

// The same product on the FP64 tensor cores: Y(:,0:nc) = X(:,0:kq) Q(0:kq,0:nc) with
// mma.sync.m8n8k4.f64 (tcgen05 has no FP64 kind).  A CTA loads a kRB-row panel of X (zero-padded to
// a multiple of 4 columns, converted to FP64) and Q (zero-padded to NT 8-column tiles) into shared
// memory; warp w computes rows 8w..8w+7 of the panel against all NT column tiles (lane (g, t) holds
// A(g, t), B(t, g) and D(g, 2t..2t+1) of each 8x8x4 step); the results are staged back through the
// panel's shared memory and written out column by column.  A panel is read completely before any of
// its rows is written, so X and Y may overlap (in-place BVMultInPlace).  Row strides of 72 and
// (8 mod 16) doubles keep each fragment load at two shared-memory wavefronts.
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

constexpr int kDmmaStride = kRB + 8;  // doubles between panel columns in shared memory

__host__ __device__ inline int dmma_q_stride(int ncp) { return (ncp % 16) ? ncp : ncp + 8; }

template <int NT, typename TI, typename TO>
__global__ void __launch_bounds__(kGemmThreads) panel_dmma_kernel(const TI *X, int ldx, TO *Y, int ldy, int n, int kq,
                                                                  const double *__restrict__ Q, int ldq, int nc,
                                                                  double alpha, double beta) {
  static_assert(kRB == 8 * (kGemmThreads / 32), "one 8-row strip per warp");
  extern __shared__ __align__(16) double sm[];
  const int kp = (kq + 3) & ~3;
  constexpr int ncp = NT * 8;
  const int SQ = dmma_q_stride(ncp);
  double *Qs = sm;                          // kp x SQ, Qs[k*SQ + j] = Q(k, j)
  double *Xs = sm + (size_t)kp * SQ;        // panel: Xs[c*kDmmaStride + r]; then the output tile
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  for (int idx = tid; idx < kp * ncp; idx += kGemmThreads) {
    const int k = idx / ncp, j = idx - k * ncp;
    Qs[k * SQ + j] = (k < kq && j < nc) ? Q[(size_t)k + (size_t)j * ldq] : 0.0;
  }
  const int npanels = (n + kRB - 1) / kRB;
  for (int pnl = blockIdx.x; pnl < npanels; pnl += gridDim.x) {
    const long long r0 = (long long)pnl * kRB;
    const int rows = (int)min((long long)kRB, (long long)n - r0);
    __syncthreads();  // the previous panel's output has been written out
    for (int idx = tid; idx < kp * kRB; idx += kGemmThreads) {
      const int c = idx / kRB, r = idx - c * kRB;
      Xs[c * kDmmaStride + r] = (c < kq && r < rows) ? (double)X[(size_t)c * ldx + r0 + r] : 0.0;
    }
    __syncthreads();
    double acc[NT][2];
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = 0.0;
    const double *xa = Xs + t * kDmmaStride + warp * 8 + g;
    const double *qb = Qs + t * SQ + g;
    for (int k0 = 0; k0 < kp; k0 += 4) {
      const double a = xa[k0 * kDmmaStride];
#pragma unroll
      for (int j = 0; j < NT; ++j) dmma_8x8x4(acc[j], a, qb[k0 * SQ + 8 * j]);
    }
    __syncthreads();  // every warp is done with the panel: its space takes the output tile
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      Xs[(8 * j + 2 * t) * kDmmaStride + warp * 8 + g] = acc[j][0];
      Xs[(8 * j + 2 * t + 1) * kDmmaStride + warp * 8 + g] = acc[j][1];
    }
    __syncthreads();
    for (int idx = tid; idx < nc * kRB; idx += kGemmThreads) {
      const int j = idx / kRB, r = idx - j * kRB;
      if (r < rows) {
        TO *y = Y + (size_t)j * ldy + r0 + r;
        const double v = Xs[j * kDmmaStride + r];
        *y = (TO)(beta == 0.0 ? alpha * v : alpha * v + beta * (double)*y);
      }
    }
  }
}

// The FP64 tensor-core product with the panel loads taken off the critical path (restart and BVMult):
// a producer warp streams each 64-row panel of X into a ring of shared-memory stages with one 2-D TMA
// load per panel, so the MMA k-loop of one panel overlaps the loads of the next ones.  In place is
// safe: a panel has landed in shared memory (its full barrier) before any of its rows is written,
// prefetches read other panels, and the only rows two CTAs touch at once are a box's extra rows past
// its panel, whose values are never used.  Waits are bounded; a timeout sets g_panel_err and the CTA
// stops (panel_gemm_error reads it).
constexpr int kTmaThreads = kGemmThreads + 32;
__device__ int g_panel_err;

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ bool mbar_wait_parity(uint64_t *bar, uint32_t parity) {
  for (long long it = 0; it < kSpinLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// The MMAs are the larger FP64 shapes (mma.sync.m16n8k16 .f64; m16n8k8 with KM = 8): 9% faster than
// m8n8k4 on the 128^3 restart (fewer fragment loads per flop; the shapes share one peak) with the
// same result bits.  TMA box of 68 rows: a column stride of 4 mod 16 doubles keeps every fragment
// load of a half warp on distinct banks.  Eight consumer warps as four 16-row strips times two
// halves of the 8-column tiles of Q.  Per KM-deep step a warp loads its A fragment once (KM/2
// doubles a lane) and reuses it across its tiles; Q's stride is also 4 mod 16.  Fragments
// (g = lane / 4, t = lane % 4): A element i at row g + 8 (i % 2), depth t + 4 (i / 2); B element i
// at depth t + 4 i, column g; D element i at row g + 8 (i / 2), column 2 t + i % 2.
constexpr int kM16Box = kRB + 4;  // rows of a panel's TMA box (column stride in shared memory)
__host__ __device__ inline int dmma16_q_stride(int ncp) { return ncp + ((4 - ncp % 16) + 16) % 16; }

template <int KM>
__device__ __forceinline__ void dmma_16x8(double (&d)[4], const double (&a)[KM / 2], const double (&b)[KM / 4]) {
  if constexpr (KM == 8) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
  } else {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
        "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
          "d"(b[1]), "d"(b[2]), "d"(b[3]));
  }
}

template <int NT, int KM>
__global__ void __launch_bounds__(kTmaThreads, 1) panel_dmma16_kernel(const __grid_constant__ CUtensorMap tx, double *Y,
                                                                      int ldy, int n, int kq,
                                                                      const double *__restrict__ Q, int ldq, int nc,
                                                                      double alpha, double beta, int stages) {
  extern __shared__ __align__(16) unsigned char tma_raw[];
  double *sm = reinterpret_cast<double *>(tma_raw + ((128u - (smem_addr(tma_raw) & 127u)) & 127u));
  __shared__ __align__(8) uint64_t full[8], empty[8];
  __shared__ int last_issue[8];
  __shared__ volatile int stop;
  constexpr int NTW = (NT + 1) / 2;  // 8-column tiles per consumer warp
  constexpr int ncp = NT * 8;
  const int kp = (kq + KM - 1) / KM * KM;
  const int SQ = dmma16_q_stride(ncp);
  const size_t stage_elems = (size_t)kp * kM16Box;
  double *Xst = sm;
  double *Qs = sm + (size_t)stages * stage_elems;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int npanels = (n + kRB - 1) / kRB;
  const int mine = blockIdx.x < npanels ? (npanels - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  if (tid == 0) {
    for (int s = 0; s < stages; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&full[s])), "r"(1) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&empty[s])), "r"(kGemmThreads / 32)
                   : "memory");
      last_issue[s] = -1;
    }
    stop = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int idx = tid; idx < kp * SQ; idx += kTmaThreads) {
    const int k = idx / SQ, j = idx - k * SQ;
    Qs[idx] = (k < kq && j < nc) ? Q[(size_t)k + (size_t)j * ldq] : 0.0;
  }
  __syncthreads();
  const uint32_t stage_bytes = (uint32_t)(stage_elems * sizeof(double));
  if (warp == kGemmThreads / 32) {
    if (lane == 0) {
      for (int i = 0; i < mine && !stop; ++i) {
        const int s = i % stages;
        if (i >= stages && !mbar_wait_parity(&empty[s], ((i / stages) - 1) & 1)) {
          atomicOr(&g_panel_err, kDevErrTimeout);
          stop = 1;
          break;
        }
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&full[s])),
                     "r"(stage_bytes)
                     : "memory");
        const int r0 = (blockIdx.x + i * gridDim.x) * kRB;
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
            "[%4];" ::"r"(smem_addr(Xst + (size_t)s * stage_elems)),
            "l"(reinterpret_cast<uint64_t>(&tx)), "r"(r0), "r"(0), "r"(smem_addr(&full[s]))
            : "memory");
        last_issue[s] = i;
      }
    }
  } else {
    const int g = lane >> 2, t = lane & 3;
    const int strip = warp & 3, half = warp >> 2;
    const int j0 = half * NTW, j1 = (half + 1) * NTW < NT ? (half + 1) * NTW : NT;
    for (int i = 0; i < mine && !stop; ++i) {
      const int s = i % stages;
      if (!mbar_wait_parity(&full[s], (i / stages) & 1)) {
        atomicOr(&g_panel_err, kDevErrTimeout);
        stop = 1;
        break;
      }
      const double *xa = Xst + (size_t)s * stage_elems + (size_t)t * kM16Box + strip * 16 + g;
      double acc[NTW][4];
#pragma unroll
      for (int j = 0; j < NTW; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
      for (int k0 = 0; k0 < kp; k0 += KM) {
        double a[KM / 2];
#pragma unroll
        for (int e = 0; e < KM / 2; ++e) a[e] = xa[(size_t)(k0 + 4 * (e / 2)) * kM16Box + 8 * (e % 2)];
#pragma unroll
        for (int jj = 0; jj < NTW; ++jj) {
          const int j = j0 + jj;
          if (j < j1) {
            double b[KM / 4];
#pragma unroll
            for (int e = 0; e < KM / 4; ++e) b[e] = Qs[(size_t)(k0 + t + 4 * e) * SQ + 8 * j + g];
            dmma_16x8<KM>(acc[jj], a, b);
          }
        }
      }
      __syncwarp();
      if (lane == 0)
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&empty[s])) : "memory");
      const long long rb = (long long)(blockIdx.x + i * gridDim.x) * kRB + strip * 16 + g;
#pragma unroll
      for (int jj = 0; jj < NTW; ++jj) {
        const int j = j0 + jj;
        if (j < j1) {
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const long long r = rb + 8 * (e / 2);
            const int c = 8 * j + 2 * t + (e % 2);
            if (r < n && c < nc) {
              double *y = Y + (size_t)c * ldy + r;
              *y = beta == 0.0 ? alpha * acc[jj][e] : alpha * acc[jj][e] + beta * *y;
            }
          }
        }
      }
    }
  }
  __syncthreads();
  if (tid == 0)
    for (int s = 0; s < stages; ++s)
      if (last_issue[s] >= 0) mbar_wait_parity(&full[s], (last_issue[s] / stages) & 1);
}

// Y(:,j) = alpha * X(:,0:nx) Q(0:nx,j) + beta * Y(:,j), one thread per row, Q column in registers-free loop.
__global__ void mult_kernel(double *Y, int ldy, const double *__restrict__ X, int ldx, int n, int nx, int ny,
                            const double *__restrict__ Q, int ldq, double alpha, double beta) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (r >= n) return;
  double acc = 0.0;
  for (int c = 0; c < nx; ++c) acc = fma(X[(size_t)c * ldx + r], Q[c + (size_t)j * ldq], acc);
  double *y = Y + (size_t)j * ldy + r;
  *y = (beta == 0.0) ? alpha * acc : alpha * acc + beta * (*y);
}

__global__ void multvec_kernel(const double *__restrict__ X, int ldx, int n, int k, const double *__restrict__ q,
                               double alpha, double beta, double *y) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double acc = 0.0;
  for (int c = 0; c < k; ++c) acc = fma(X[(size_t)c * ldx + r], q[c], acc);
  y[r] = (beta == 0.0) ? alpha * acc : beta * y[r] + alpha * acc;
}

// partial[blk * (nx*ny) + (i + j*ny)] over a persistent row split; one output pair per warp iteration.
__global__ void dot_partial_kernel(const double *__restrict__ X, int ldx, int nx, const double *__restrict__ Y,
                                   int ldy, int ny, int n, double *partial) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const long long rows_per = (n + gridDim.x - 1) / gridDim.x;
  const long long r0 = (long long)blockIdx.x * rows_per;
  const long long r1 = min((long long)n, r0 + rows_per);
  const int npairs = nx * ny;
  for (int pr = warp; pr < npairs; pr += nw) {
    const int i = pr % ny, j = pr / ny;
    const double *y = Y + (size_t)i * ldy, *x = X + (size_t)j * ldx;
    double acc = 0.0;
    for (long long r = r0 + lane; r < r1; r += 32) acc = fma(y[r], x[r], acc);
    acc = warp_sum(acc);
    if (lane == 0) partial[(size_t)blockIdx.x * npairs + pr] = acc;
  }
}

// Gram block M = Y^T X for up to T x T column pairs per CTA row, T = 16 TM (blockIdx.y, blockIdx.z
// select the T-column blocks of Y and X; TM is chosen from the block width so that narrow blocks do
// not pay for padding).  The CTA's rows are staged in 32-row panels in shared memory, the next panel
// is loaded into registers while the current one is consumed, and thread (ty, tx) of a 16 x 16 layout
// accumulates the TM x TM pairs (TM ty + a, TM tx + b) in row order.
// partial[blk * (nx*ny) + (i + j*ny)] as dot_partial_kernel writes it.
constexpr int kGramRows = 32;
template <int TM>
__global__ void __launch_bounds__(256) gram_partial_kernel(const double *__restrict__ X, int ldx, int nx,
                                                           const double *__restrict__ Y, int ldy, int ny, int n,
                                                           double *partial) {
  constexpr int T = 16 * TM;
  constexpr int kLoads = kGramRows * T / 256;  // elements of each operand a thread stages per panel
  __shared__ double Xs[kGramRows][T + 1], Ys[kGramRows][T + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int y0 = blockIdx.y * T, x0 = blockIdx.z * T;
  const int cy = min(T, ny - y0), cx = min(T, nx - x0);
  const long long rows_per = (n + gridDim.x - 1) / gridDim.x;
  const long long r0 = (long long)blockIdx.x * rows_per;
  const long long r1 = min((long long)n, r0 + rows_per);
  double acc[TM][TM];
#pragma unroll
  for (int a = 0; a < TM; ++a)
#pragma unroll
    for (int b = 0; b < TM; ++b) acc[a][b] = 0.0;
  double xr[kLoads], yr[kLoads];
  // column-major loads: 32 consecutive rows of one column per warp
  auto load = [&](long long p0, int pr) {
#pragma unroll
    for (int u = 0; u < kLoads; ++u) {
      const int e = threadIdx.x + 256 * u;
      const int r = e % kGramRows, c = e / kGramRows;
      xr[u] = (r < pr && c < cx) ? X[(size_t)(x0 + c) * ldx + p0 + r] : 0.0;
      yr[u] = (r < pr && c < cy) ? Y[(size_t)(y0 + c) * ldy + p0 + r] : 0.0;
    }
  };
  long long p0 = r0;
  int pr = p0 < r1 ? (int)min((long long)kGramRows, r1 - p0) : 0;
  if (pr > 0) load(p0, pr);
  while (pr > 0) {
#pragma unroll
    for (int u = 0; u < kLoads; ++u) {
      const int e = threadIdx.x + 256 * u;
      const int r = e % kGramRows, c = e / kGramRows;
      Xs[r][c] = xr[u];
      Ys[r][c] = yr[u];
    }
    __syncthreads();
    const long long pn = p0 + kGramRows;
    const int prn = pn < r1 ? (int)min((long long)kGramRows, r1 - pn) : 0;
    if (prn > 0) load(pn, prn);  // in flight while this panel is consumed
    for (int r = 0; r < pr; ++r) {
      double yv[TM], xv[TM];
#pragma unroll
      for (int a = 0; a < TM; ++a) yv[a] = Ys[r][TM * ty + a];
#pragma unroll
      for (int b = 0; b < TM; ++b) xv[b] = Xs[r][TM * tx + b];
#pragma unroll
      for (int a = 0; a < TM; ++a)
#pragma unroll
        for (int b = 0; b < TM; ++b) acc[a][b] = fma(yv[a], xv[b], acc[a][b]);
    }
    __syncthreads();
    p0 = pn;
    pr = prn;
  }
  const int npairs = nx * ny;
#pragma unroll
  for (int a = 0; a < TM; ++a)
#pragma unroll
    for (int b = 0; b < TM; ++b) {
      const int i = TM * ty + a, j = TM * tx + b;
      if (i < cy && j < cx) partial[(size_t)blockIdx.x * npairs + (y0 + i) + (size_t)(x0 + j) * ny] = acc[a][b];
    }
}

// The Gram pair on the FP64 MMA path (mma.sync.m16n8k16.f64), nc <= 64 columns: per 32-row chunk
// the CTA stages the columns of X and Y in shared memory (column stride 36 doubles, 4 mod 16: the
// fragment loads of a half warp hit distinct banks), the next chunk fetched into registers while the
// current one is consumed; warp w < 2 NMB accumulates the 16-row strip w % NMB of M1 = Y^T X
// (w < NMB) or of M2 = Y^T Y over its CTA's rows.  Fragments (g = lane / 4, t = lane % 4): A = Y^T,
// element e at row g + 8 (e % 2), depth t + 4 (e / 2); B element e at depth t + 4 e, column g; D
// element e at row g + 8 (e / 2), column 2 t + e % 2.  Partial sums partial[cta][M1 then M2], each (i + j nc).
constexpr int kDualRows = 32;  // rows per staged chunk
constexpr int kDualLd = 36;    // doubles per staged column
__device__ __forceinline__ void dmma_m16n8k16(double (&d)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
        "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

template <int NMB>
__global__ void __launch_bounds__(256) gram_dual_mma_kernel(const double *__restrict__ X, int ldx,
                                                            const double *__restrict__ Y, int ldy, int nc, int n,
                                                            double *partial) {
  constexpr int NC = 16 * NMB;  // staged columns (zero past nc)
  __shared__ double xs[NC * kDualLd], ys[NC * kDualLd];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const bool active = warp < 2 * NMB;
  const int mb = warp % NMB;
  const bool self = warp >= NMB;  // M2 = Y^T Y
  const double *bs = self ? ys : xs;
  const int nnb = (nc + 7) / 8;
  const long long rows_per = ((long long)(n + gridDim.x - 1) / gridDim.x + kDualRows - 1) / kDualRows * kDualRows;
  const long long r0 = (long long)blockIdx.x * rows_per;
  const long long r1 = min((long long)n, r0 + rows_per);
  double acc[2 * NMB][4];
#pragma unroll
  for (int j = 0; j < 2 * NMB; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
  constexpr int kPer = kDualRows * NC / 256;
  double px[kPer], py[kPer];
  auto fetch = [&](long long p0) {
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int e = threadIdx.x + 256 * u, c = e / kDualRows, r = e % kDualRows;
      const long long row = p0 + r;
      const bool in = row < r1 && c < nc;
      px[u] = in ? X[(size_t)c * ldx + row] : 0.0;
      py[u] = in ? Y[(size_t)c * ldy + row] : 0.0;
    }
  };
  if (r0 < r1) fetch(r0);
  for (long long p0 = r0; p0 < r1; p0 += kDualRows) {
    __syncthreads();  // the previous chunk is consumed
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int e = threadIdx.x + 256 * u, c = e / kDualRows, r = e % kDualRows;
      xs[c * kDualLd + r] = px[u];
      ys[c * kDualLd + r] = py[u];
    }
    __syncthreads();
    if (p0 + kDualRows < r1) fetch(p0 + kDualRows);
    if (active) {
#pragma unroll
      for (int k0 = 0; k0 < kDualRows; k0 += 16) {
        double a[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) a[e] = ys[(16 * mb + g + 8 * (e & 1)) * kDualLd + k0 + t + 4 * (e >> 1)];
#pragma unroll
        for (int j = 0; j < 2 * NMB; ++j) {
          if (j < nnb) {
            double b[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) b[e] = bs[(8 * j + g) * kDualLd + k0 + t + 4 * e];
            dmma_m16n8k16(acc[j], a, b);
          }
        }
      }
    }
  }
  if (!active) return;
  const size_t npairs = (size_t)nc * nc;
  double *pb = partial + (size_t)blockIdx.x * 2 * npairs + (self ? npairs : 0);
#pragma unroll
  for (int j = 0; j < 2 * NMB; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int i = 16 * mb + g + 8 * (e >> 1), col = 8 * j + 2 * t + (e & 1);
      if (i < nc && col < nc) pb[i + (size_t)col * nc] = acc[j][e];
    }
}

// M(i, j) = the sum over the row blocks of the partial sums.  A CTA takes 32 consecutive pairs (one
// per lane, so each load of a row block's partials is one coalesced 256-byte line); its 8 warps split
// the row blocks (warp g sums blocks g, g + 8, ...) and the 8 sums are added in a fixed order.
__global__ void __launch_bounds__(256) dot_final_kernel(const double *__restrict__ partial, int nblocks, int nx,
                                                        int ny, double *M, int ldm) {
  __shared__ double red[8][33];
  const int npairs = nx * ny;
  const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
  const int pr = blockIdx.x * 32 + lane;
  double acc = 0.0;
  if (pr < npairs)
    for (int b = g; b < nblocks; b += 8) acc += partial[(size_t)b * npairs + pr];
  red[g][lane] = acc;
  __syncthreads();
  if (g == 0 && pr < npairs) {
    double t = red[0][lane];
#pragma unroll
    for (int q = 1; q < 8; ++q) t += red[q][lane];
    M[(pr % ny) + (size_t)(pr / ny) * ldm] = t;
  }
}

__global__ void scale_kernel(double *x, long long len, double alpha) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    x[i] *= alpha;
}

__global__ void copy_kernel(double *dst, const double *__restrict__ src, long long len) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

__global__ void sumsq_partial_kernel(const double *__restrict__ x, long long len, double *partial) {
  __shared__ double red[32];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    acc = fma(x[i], x[i], acc);
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    partial[blockIdx.x] = s;
  }
}

__global__ void diff_sumsq_partial_kernel(const double *__restrict__ y, const double *__restrict__ x, double alpha,
                                          long long len, double *partial) {
  __shared__ double red[32];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x) {
    const double r = y[i] - alpha * x[i];
    acc = fma(r, r, acc);
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    partial[blockIdx.x] = s;
  }
}

// y -= alpha x (VecAXPY with -alpha), product and difference rounded separately
__global__ void axmy_kernel(double *y, const double *__restrict__ x, double alpha, long long len) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    y[i] = __dsub_rn(y[i], __dmul_rn(alpha, x[i]));
}

// columns c of V(:, 0:ncols): V(i,c) = d(i) * V(i,c)  (PCApply_Jacobi: pointwise product with diag^{-1})
__global__ void diag_scale_kernel(double *V, int ld, int n, int ncols, const double *__restrict__ d) {
  const long long total = (long long)n * ncols;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / n), i = (int)(t % n);
    V[i + (size_t)c * ld] = __dmul_rn(d[i], V[i + (size_t)c * ld]);
  }
}

// dinv(i) = 1 / a_ii (entries on the diagonal summed in index order; a zero diagonal counts as 1)
__global__ void inverse_diagonal_kernel(int n, const int *__restrict__ rowptr, const int *__restrict__ colind,
                                        const double *__restrict__ vals, double *dinv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = 0.0;
    for (int p = rowptr[i]; p < rowptr[i + 1]; ++p)
      if (colind[p] == i) d = __dadd_rn(d, vals[p]);
    dinv[i] = 1.0 / (d != 0.0 ? d : 1.0);
  }
}

// partial[c * gridDim.x + b] = sum of squares of column c over the block's row range
__global__ void colnorm_partial_kernel(const double *__restrict__ X, int ldx, int n, double *partial) {
  __shared__ double red[32];
  const int c = blockIdx.y;
  const long long rows_per = (n + gridDim.x - 1) / gridDim.x;
  const long long r0 = (long long)blockIdx.x * rows_per, r1 = min((long long)n, r0 + rows_per);
  const double *x = X + (size_t)c * ldx;
  double acc = 0.0;
  for (long long r = r0 + threadIdx.x; r < r1; r += blockDim.x) acc = fma(x[r], x[r], acc);
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    partial[(size_t)c * gridDim.x + blockIdx.x] = s;
  }
}

__global__ void colnorm_final_kernel(const double *__restrict__ partial, int nblocks, int k, double *out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= k) return;
  double s = 0.0;
  for (int b = 0; b < nblocks; ++b) s += partial[(size_t)c * nblocks + b];
  out[c] = sqrt(s);
}

// partial[c * gridDim.x + b] = sum over the block's rows of (AX(r,c) - theta[c] X(r,c))^2
__global__ void colresid_partial_kernel(const double *__restrict__ AX, const double *__restrict__ X, int ld, int n,
                                        const double *__restrict__ theta, double *partial) {
  __shared__ double red[32];
  const int c = blockIdx.y;
  const long long rows_per = (n + gridDim.x - 1) / gridDim.x;
  const long long r0 = (long long)blockIdx.x * rows_per, r1 = min((long long)n, r0 + rows_per);
  const double *ax = AX + (size_t)c * ld, *x = X + (size_t)c * ld;
  const double th = theta[c];
  double acc = 0.0;
  for (long long r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    const double d = ax[r] - th * x[r];
    acc = fma(d, d, acc);
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    partial[(size_t)c * gridDim.x + blockIdx.x] = t;
  }
}

__global__ void to_f32_kernel(float *dst, const double *__restrict__ src, long long len) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    dst[i] = __double2float_rn(src[i]);
}

// Gershgorin discs: partial[2b] = min_i (a_ii - sum_{j!=i} |a_ij|), partial[2b+1] = max_i (a_ii + ...)
// over the rows of block b (grid-stride).
template <typename VT>
__global__ void gershgorin_partial_kernel(int n, const int *__restrict__ rowptr, const int *__restrict__ colind,
                                          const VT *__restrict__ vals, double *partial) {
  __shared__ double rlo[32], rhi[32];
  double lo = 1.79769313486231571e+308, hi = -1.79769313486231571e+308;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = 0.0, rad = 0.0;
    for (int p = rowptr[i]; p < rowptr[i + 1]; ++p) {
      const double a = (double)vals[p];
      if (colind[p] == i) d += a;
      else rad += fabs(a);
    }
    lo = fmin(lo, d - rad);
    hi = fmax(hi, d + rad);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, off));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, off));
  }
  if ((threadIdx.x & 31) == 0) {
    rlo[threadIdx.x >> 5] = lo;
    rhi[threadIdx.x >> 5] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      lo = fmin(lo, rlo[w]);
      hi = fmax(hi, rhi[w]);
    }
    partial[2 * blockIdx.x] = lo;
    partial[2 * blockIdx.x + 1] = hi;
  }
}

__global__ void gershgorin_final_kernel(const double *__restrict__ partial, int nblocks, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double lo = 1.79769313486231571e+308, hi = -1.79769313486231571e+308;
  for (int b = 0; b < nblocks; ++b) {
    lo = fmin(lo, partial[2 * b]);
    hi = fmax(hi, partial[2 * b + 1]);
  }
  out[0] = lo;
  out[1] = hi;
}

__global__ void sum_final_kernel(const double *__restrict__ partial, int nblocks, double *out) {
  __shared__ double red[32];
  double acc = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) acc += partial[b];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    out[0] = s;
  }
}

template <int LPR>
__global__ void __launch_bounds__(256) residual_partial_kernel(int n, const int *__restrict__ rowptr,
                                                               const int *__restrict__ colind,
                                                               const double *__restrict__ vals,
                                                               const double *__restrict__ x, double lambda,
                                                               double *partial) {
  __shared__ double red[8];
  constexpr int kRowsPerWarp = 32 / LPR;
  const int lane = threadIdx.x & (LPR - 1);
  const int sub = (threadIdx.x & 31) / LPR;
  const int warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double acc = 0.0;
  for (long long base = (long long)warp_global * kRowsPerWarp; base < n; base += (long long)nwarps * kRowsPerWarp) {
    const long long row = base + sub;
    double sum = 0.0;
    if (row < n) {
      const int rs = rowptr[row], re = rowptr[row + 1];
      for (int p = rs + lane; p < re; p += LPR) sum = fma(vals[p], x[colind[p]], sum);
    }
#pragma unroll
    for (int off = LPR / 2; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off, LPR);
    if (lane == 0 && row < n) {
      const double r = sum - lambda * x[row];
      acc = fma(r, r, acc);
    }
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += red[w];
    partial[blockIdx.x] = s;
  }
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

__global__ void random_kernel(double *x, int n, uint64_t seed, uint64_t stream_id) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const uint64_t z = splitmix64(seed ^ splitmix64(stream_id * 0x100000001B3ULL + (uint64_t)i));
    x[i] = (double)(z >> 11) * (1.0 / 9007199254740992.0);
  }
}

int num_sms() {
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && cached[dev]) return cached[dev];
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  if (v <= 0) v = 1;
  if (dev < 64) cached[dev] = v;
  return v;
}

unsigned grid_for(long long len, int threads) {
  long long b = (len + threads - 1) / threads;
  const long long cap = (long long)num_sms() * 8;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

}  // namespace

std::atomic<bool> g_panel_launched{false};  // a pipelined product ran since the last error check

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      ptr = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  }();
  return fn;
}

// The pipelined FP64 product when X is FP64, 16-byte aligned with an even leading dimension, and two
// or more stages fit in shared memory beside Q; cudaErrorNotSupported otherwise (the caller falls back).
template <int KM>
cudaError_t panel_dmma16_launch(const double *X, int ldx, double *Y, int ldy, int n, int kq, const double *Q, int ldq,
                                int nc, cudaStream_t stream, double alpha, double beta) {
  const int kp = (kq + KM - 1) / KM * KM, nt = (nc + 7) / 8, ncp = 8 * nt;
  if (kp > 256 || ((uintptr_t)X & 15) || (ldx & 1) || nt < 1 || nt > 16) return cudaErrorNotSupported;
  const size_t stage = sizeof(double) * (size_t)kp * kM16Box;
  const size_t qbytes = sizeof(double) * (size_t)kp * dmma16_q_stride(ncp);
  const size_t avail = max_dynamic_smem() - 1024 - 128;
  if (avail < qbytes + 2 * stage) return cudaErrorNotSupported;
  int stages = (int)((avail - qbytes) / stage);
  if (stages > 8) stages = 8;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return cudaErrorNotSupported;
  CUtensorMap tm;
  const cuuint64_t dims[2] = {(cuuint64_t)n, (cuuint64_t)kq};
  const cuuint64_t strides[1] = {(cuuint64_t)ldx * sizeof(double)};
  const cuuint32_t box[2] = {(cuuint32_t)kM16Box, (cuuint32_t)kp};
  const cuuint32_t estr[2] = {1, 1};
  if (enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(X), dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorNotSupported;
  const size_t smem = qbytes + (size_t)stages * stage + 128;
  const int npanels = (n + kRB - 1) / kRB;
  int grid = num_sms();
  if (grid > npanels) grid = npanels;
  cudaError_t err = cudaSuccess;
  switch (nt) {
#define B200_M16_CASE(NT)                                                                                          \
  case NT:                                                                                                         \
    err = cudaFuncSetAttribute(panel_dmma16_kernel<NT, KM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
    if (err != cudaSuccess) return err;                                                                            \
    panel_dmma16_kernel<NT, KM><<<grid, kTmaThreads, smem, stream>>>(tm, Y, ldy, n, kq, Q, ldq, nc, alpha, beta,      \
                                                                     stages);                                      \
    break;
    B200_M16_CASE(1) B200_M16_CASE(2) B200_M16_CASE(3) B200_M16_CASE(4) B200_M16_CASE(5) B200_M16_CASE(6)
    B200_M16_CASE(7) B200_M16_CASE(8) B200_M16_CASE(9) B200_M16_CASE(10) B200_M16_CASE(11) B200_M16_CASE(12)
    B200_M16_CASE(13) B200_M16_CASE(14) B200_M16_CASE(15) B200_M16_CASE(16)
#undef B200_M16_CASE
    default:
      return cudaErrorNotSupported;
  }
  count_launch();
  g_panel_launched.store(true);
  return cudaGetLastError();
}


template <typename TI, typename TO>
cudaError_t panel_gemm_launch(const TI *X, int ldx, TO *Y, int ldy, int n, int kq, const double *Q, int ldq, int nc,
                              cudaStream_t stream, double alpha = 1.0, double beta = 0.0) {
  if (nc <= 0 || kq <= 0 || n <= 0) return cudaSuccess;
  if (nc > 16 * 8 || kq > kMaxCols) return cudaErrorInvalidValue;
  if constexpr (sizeof(TI) == sizeof(double) && sizeof(TO) == sizeof(double)) {
    const cudaError_t err = panel_dmma16_launch<16>(reinterpret_cast<const double *>(X), ldx,
                                                  reinterpret_cast<double *>(Y), ldy, n, kq, Q, ldq, nc, stream,
                                                  alpha, beta);
    if (err != cudaErrorNotSupported) return err;
  }
  {
    // FP64 tensor cores when the padded panel and Q fit in shared memory
    const int kp = (kq + 3) & ~3, nt = (nc + 7) / 8, ncp = 8 * nt;
    const size_t dsm = sizeof(double) * ((size_t)kp * dmma_q_stride(ncp) + (size_t)(kp > ncp ? kp : ncp) * kDmmaStride);
    if (dsm + 1024 <= max_dynamic_smem()) {
      const int npanels = (n + kRB - 1) / kRB;
      int grid = num_sms() * 2;
      if (grid > npanels) grid = npanels;
      cudaError_t err = cudaSuccess;
      switch (nt) {
#define B200_DMMA_CASE(NT)                                                                                  \
  case NT:                                                                                                  \
    err = allow_max_dynamic_smem(panel_dmma_kernel<NT, TI, TO>);                                            \
    if (err != cudaSuccess) return err;                                                                     \
    panel_dmma_kernel<NT, TI, TO><<<grid, kGemmThreads, dsm, stream>>>(X, ldx, Y, ldy, n, kq, Q, ldq, nc, alpha, \
                                                                       beta);                                  \
    break;
        B200_DMMA_CASE(1) B200_DMMA_CASE(2) B200_DMMA_CASE(3) B200_DMMA_CASE(4) B200_DMMA_CASE(5)
        B200_DMMA_CASE(6) B200_DMMA_CASE(7) B200_DMMA_CASE(8) B200_DMMA_CASE(9) B200_DMMA_CASE(10)
        B200_DMMA_CASE(11) B200_DMMA_CASE(12) B200_DMMA_CASE(13) B200_DMMA_CASE(14) B200_DMMA_CASE(15)
        B200_DMMA_CASE(16)
#undef B200_DMMA_CASE
        default:
          return cudaErrorInvalidValue;
      }
      count_launch();
      return cudaGetLastError();
    }
  }
  const size_t smem = sizeof(double) * ((size_t)kq * nc + (size_t)(kq > nc ? kq : nc) * (kRB + 1));
  if (smem + 1024 > max_dynamic_smem()) return cudaErrorInvalidValue;
  const int maxj = (nc + 15) / 16;
  const int npanels = (n + kRB - 1) / kRB;
  int grid = num_sms() * 2;
  if (grid > npanels) grid = npanels;
  cudaError_t err = cudaSuccess;
  switch (maxj) {
#define B200_MIP_CASE(J)                                                                                   \
  case J:                                                                                                  \
    err = allow_max_dynamic_smem(panel_gemm_kernel<J, TI, TO>);                                            \
    if (err != cudaSuccess) return err;                                                                    \
    panel_gemm_kernel<J, TI, TO><<<grid, kGemmThreads, smem, stream>>>(X, ldx, Y, ldy, n, kq, Q, ldq, nc, alpha, \
                                                                       beta);                                  \
    break;
    B200_MIP_CASE(1)
    B200_MIP_CASE(2)
    B200_MIP_CASE(3)
    B200_MIP_CASE(4)
    B200_MIP_CASE(5)
    B200_MIP_CASE(6)
    B200_MIP_CASE(7)
    B200_MIP_CASE(8)
#undef B200_MIP_CASE
    default:
      return cudaErrorInvalidValue;
  }
  count_launch();
  return cudaGetLastError();
}

cudaError_t panel_gemm_error(int *err, cudaStream_t stream) {
  int v = 0;
  *err = 0;
  if (!g_panel_launched.exchange(false)) return cudaSuccess;
  cudaError_t e = cudaMemcpyFromSymbolAsync(&v, g_panel_err, sizeof(int), 0, cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e == cudaSuccess && v) {
    const int zero = 0;
    e = cudaMemcpyToSymbolAsync(g_panel_err, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, stream);
  }
  *err = v;
  return e;
}

cudaError_t multinplace_launch(double *V, int ld, int n, int l, int k, const double *Q, int ldq, int s, int e,
                               cudaStream_t stream) {
  return panel_gemm_launch<double, double>(V + (size_t)l * ld, ld, V + (size_t)s * ld, ld, n, k - l, Q, ldq, e - s,
                                           stream);
}

cudaError_t multinplace_launch_f32(float *V, int ld, int n, int l, int k, const double *Q, int ldq, int s, int e,
                                   cudaStream_t stream) {
  return panel_gemm_launch<float, float>(V + (size_t)l * ld, ld, V + (size_t)s * ld, ld, n, k - l, Q, ldq, e - s,
                                         stream);
}

cudaError_t panel_mult_launch(double *Y, int ldy, const double *X, int ldx, int n, int nx, int ny, const double *Q,
                              int ldq, cudaStream_t stream) {
  return panel_gemm_launch<double, double>(X, ldx, Y, ldy, n, nx, Q, ldq, ny, stream);
}

cudaError_t panel_mult_launch_f32(double *Y, int ldy, const float *X, int ldx, int n, int nx, int ny, const double *Q,
                                  int ldq, cudaStream_t stream) {
  return panel_gemm_launch<float, double>(X, ldx, Y, ldy, n, nx, Q, ldq, ny, stream);
}

cudaError_t colresid_launch(const double *AX, const double *X, int ld, int n, int k, const double *theta, double *out,
                            double *work, int work_len, cudaStream_t stream) {
  if (k <= 0) return cudaSuccess;
  int blocks = num_sms();
  if (blocks * k > work_len) blocks = work_len / k;
  if (blocks < 1) return cudaErrorInvalidValue;
  colresid_partial_kernel<<<dim3(blocks, k), 256, 0, stream>>>(AX, X, ld, n, theta, work);
  count_launch();
  colnorm_final_kernel<<<(k + 127) / 128, 128, 0, stream>>>(work, blocks, k, out);
  count_launch();
  return cudaGetLastError();
}

cudaError_t to_f32_launch(float *dst, const double *src, long long len, cudaStream_t stream) {
  if (len <= 0) return cudaSuccess;
  to_f32_kernel<<<grid_for(len, 256), 256, 0, stream>>>(dst, src, len);
  count_launch();
  return cudaGetLastError();
}

cudaError_t gershgorin_launch(int n, const int *rowptr, const int *colind, const void *vals, bool f32, double *out,
                              double *work, int work_len, cudaStream_t stream) {
  int blocks = (int)grid_for(n, 256);
  if (2 * blocks > work_len) blocks = work_len / 2;
  if (blocks < 1) return cudaErrorInvalidValue;
  if (f32)
    gershgorin_partial_kernel<float><<<blocks, 256, 0, stream>>>(n, rowptr, colind, static_cast<const float *>(vals),
                                                                  work);
  else
    gershgorin_partial_kernel<double><<<blocks, 256, 0, stream>>>(n, rowptr, colind,
                                                                   static_cast<const double *>(vals), work);
  count_launch();
  gershgorin_final_kernel<<<1, 32, 0, stream>>>(work, blocks, out);
  count_launch();
  return cudaGetLastError();
}

cudaError_t mult_launch(double *Y, int ldy, const double *X, int ldx, int n, int nx, int ny, const double *Q, int ldq,
                        double alpha, double beta, cudaStream_t stream) {
  if (n <= 0 || ny <= 0) return cudaSuccess;
  // the row-panel product (X read once, FP64 tensor cores) when the block fits it; the simple
  // kernel below reads X once per output column
  if (nx > 0 && nx <= kMaxCols && ny <= 16 * 8) {
    const cudaError_t err = panel_gemm_launch<double, double>(X, ldx, Y, ldy, n, nx, Q, ldq, ny, stream, alpha, beta);
    if (err != cudaErrorInvalidValue) return err;  // otherwise the block does not fit shared memory
  }
  dim3 grid((unsigned)((n + 255) / 256), (unsigned)ny);
  mult_kernel<<<grid, 256, 0, stream>>>(Y, ldy, X, ldx, n, nx, ny, Q, ldq, alpha, beta);
  count_launch();
  return cudaGetLastError();
}

cudaError_t multvec_launch(const double *X, int ldx, int n, int k, const double *q, double alpha, double beta, double *y,
                           cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  multvec_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(X, ldx, n, k, q, alpha, beta, y);
  count_launch();
  return cudaGetLastError();
}

cudaError_t dot_launch(const double *X, int ldx, int nx, const double *Y, int ldy, int ny, int n, double *M, int ldm,
                       double *work, int work_len, cudaStream_t stream, int ctas_per_sm) {
  if (nx <= 0 || ny <= 0) return cudaSuccess;
  const int npairs = nx * ny;
  int blocks = num_sms() * (ctas_per_sm > 0 ? ctas_per_sm : 1);
  if (blocks * npairs > work_len) blocks = work_len / npairs;
  if (blocks < 1) return cudaErrorInvalidValue;
  if (npairs >= 64) {
    // register-tiled Gram blocks: both blocks of columns read once per CTA row range
    const int w = nx > ny ? nx : ny;
    const int tm = w > 48 ? 4 : (w + 15) / 16;
    const int T = 16 * tm;
    const dim3 grid(blocks, (ny + T - 1) / T, (nx + T - 1) / T);
    switch (tm) {
      case 1: gram_partial_kernel<1><<<grid, 256, 0, stream>>>(X, ldx, nx, Y, ldy, ny, n, work); break;
      case 2: gram_partial_kernel<2><<<grid, 256, 0, stream>>>(X, ldx, nx, Y, ldy, ny, n, work); break;
      case 3: gram_partial_kernel<3><<<grid, 256, 0, stream>>>(X, ldx, nx, Y, ldy, ny, n, work); break;
      default: gram_partial_kernel<4><<<grid, 256, 0, stream>>>(X, ldx, nx, Y, ldy, ny, n, work); break;
    }
  } else {
    dot_partial_kernel<<<blocks, 256, 0, stream>>>(X, ldx, nx, Y, ldy, ny, n, work);
  }
  count_launch();
  dot_final_kernel<<<(npairs + 31) / 32, 256, 0, stream>>>(work, blocks, nx, ny, M, ldm);
  count_launch();
  return cudaGetLastError();
}

cudaError_t dot_dual_launch(const double *X, int ldx, const double *Y, int ldy, int nc, int n, double *M, double *work,
                            int work_len, cudaStream_t stream, int ctas_per_sm) {
  if (nc <= 0) return cudaSuccess;
  if (nc > 64 || nc * nc < 64) return cudaErrorNotSupported;
  const int npairs2 = 2 * nc * nc;
  int blocks = num_sms() * (ctas_per_sm > 0 ? ctas_per_sm : 1);
  if (blocks * npairs2 > work_len) blocks = work_len / npairs2;
  if (blocks < 1) return cudaErrorInvalidValue;
  const int nmb = (nc + 15) / 16;  // the FP64 MMA form (16-row strips of both Gram blocks)
  switch (nmb) {
    case 1: gram_dual_mma_kernel<1><<<blocks, 256, 0, stream>>>(X, ldx, Y, ldy, nc, n, work); break;
    case 2: gram_dual_mma_kernel<2><<<blocks, 256, 0, stream>>>(X, ldx, Y, ldy, nc, n, work); break;
    case 3: gram_dual_mma_kernel<3><<<blocks, 256, 0, stream>>>(X, ldx, Y, ldy, nc, n, work); break;
    default: gram_dual_mma_kernel<4><<<blocks, 256, 0, stream>>>(X, ldx, Y, ldy, nc, n, work); break;
  }
  count_launch();
  dot_final_kernel<<<(npairs2 + 31) / 32, 256, 0, stream>>>(work, blocks, 2 * nc, nc, M, nc);
  count_launch();
  return cudaGetLastError();
}

// R(:, j) = AX(:, j) - theta[j] X(:, j), j < ncols (each element rounded as BVCopy + VecAXPY give it)
__global__ void resid_block_kernel(double *R, int ldr, const double *__restrict__ AX, int ldax,
                                   const double *__restrict__ X, int ldx, int n, int ncols, ThetaArg th) {
  const long long total = (long long)n * ncols;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t / n);
    const long long i = t - (long long)j * n;
    R[i + (size_t)j * ldr] = __dsub_rn(AX[i + (size_t)j * ldax], __dmul_rn(th.v[j], X[i + (size_t)j * ldx]));
  }
}

cudaError_t resid_block_launch(double *R, int ldr, const double *AX, int ldax, const double *X, int ldx, int n,
                               int ncols, const double *theta, cudaStream_t stream) {
  if (ncols <= 0 || n <= 0) return cudaSuccess;
  if (ncols > kThetaMax) return cudaErrorInvalidValue;
  ThetaArg th{};
  for (int j = 0; j < ncols; ++j) th.v[j] = theta[j];
  resid_block_kernel<<<grid_for((long long)n * ncols, 256), 256, 0, stream>>>(R, ldr, AX, ldax, X, ldx, n, ncols, th);
  count_launch();
  return cudaGetLastError();
}

cudaError_t scale_launch(double *x, long long len, double alpha, cudaStream_t stream) {
  if (len <= 0) return cudaSuccess;
  scale_kernel<<<grid_for(len, 256), 256, 0, stream>>>(x, len, alpha);
  count_launch();
  return cudaGetLastError();
}

cudaError_t copy_launch(double *dst, const double *src, long long len, cudaStream_t stream) {
  if (len <= 0) return cudaSuccess;
  copy_kernel<<<grid_for(len, 256), 256, 0, stream>>>(dst, src, len);
  count_launch();
  return cudaGetLastError();
}

cudaError_t colnorm_launch(const double *X, int ldx, int n, int k, double *out, double *work, int work_len,
                           cudaStream_t stream) {
  if (k <= 0) return cudaSuccess;
  int blocks = num_sms();
  if (blocks * k > work_len) blocks = work_len / k;
  if (blocks < 1) return cudaErrorInvalidValue;
  colnorm_partial_kernel<<<dim3(blocks, k), 256, 0, stream>>>(X, ldx, n, work);
  count_launch();
  colnorm_final_kernel<<<(k + 127) / 128, 128, 0, stream>>>(work, blocks, k, out);
  count_launch();
  return cudaGetLastError();
}

cudaError_t sumsq_launch(const double *x, long long len, double *out, double *work, int work_len, cudaStream_t stream) {
  int blocks = (int)grid_for(len, 256);
  if (blocks > work_len) blocks = work_len;
  sumsq_partial_kernel<<<blocks, 256, 0, stream>>>(x, len, work);
  count_launch();
  sum_final_kernel<<<1, 256, 0, stream>>>(work, blocks, out);
  count_launch();
  return cudaGetLastError();
}

cudaError_t diff_sumsq_launch(const double *y, const double *x, double alpha, long long len, double *out, double *work,
                              int work_len, cudaStream_t stream) {
  int blocks = (int)grid_for(len, 256);
  if (blocks > work_len) blocks = work_len;
  diff_sumsq_partial_kernel<<<blocks, 256, 0, stream>>>(y, x, alpha, len, work);
  count_launch();
  sum_final_kernel<<<1, 256, 0, stream>>>(work, blocks, out);
  count_launch();
  return cudaGetLastError();
}

cudaError_t residual_launch(int n, const int *rowptr, const int *colind, const double *vals, const double *x,
                            double lambda, double *out, double *work, int work_len, int lanes, cudaStream_t stream) {
  int blocks = num_sms() * 4;
  if (blocks > work_len) blocks = work_len;
  switch (lanes) {
#define B200_RES_CASE(L)                                                                                    \
  case L:                                                                                                   \
    residual_partial_kernel<L><<<blocks, 256, 0, stream>>>(n, rowptr, colind, vals, x, lambda, work); \
    break;
    B200_RES_CASE(1)
    B200_RES_CASE(2)
    B200_RES_CASE(4)
    B200_RES_CASE(8)
    B200_RES_CASE(16)
    B200_RES_CASE(32)
#undef B200_RES_CASE
    default:
      return cudaErrorInvalidValue;
  }
  count_launch();
  sum_final_kernel<<<1, 256, 0, stream>>>(work, blocks, out);
  count_launch();
  return cudaGetLastError();
}

cudaError_t axmy_launch(double *y, const double *x, double alpha, long long len, cudaStream_t stream) {
  if (len <= 0) return cudaSuccess;
  axmy_kernel<<<grid_for(len, 256), 256, 0, stream>>>(y, x, alpha, len);
  count_launch();
  return cudaGetLastError();
}

cudaError_t diag_scale_launch(double *V, int ld, int n, int ncols, const double *d, cudaStream_t stream) {
  if (ncols <= 0 || n <= 0) return cudaSuccess;
  diag_scale_kernel<<<grid_for((long long)n * ncols, 256), 256, 0, stream>>>(V, ld, n, ncols, d);
  count_launch();
  return cudaGetLastError();
}

cudaError_t inverse_diagonal_launch(int n, const int *rowptr, const int *colind, const double *vals, double *dinv,
                                    cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  inverse_diagonal_kernel<<<grid_for(n, 256), 256, 0, stream>>>(n, rowptr, colind, vals, dinv);
  count_launch();
  return cudaGetLastError();
}

cudaError_t random_launch(double *x, int n, uint64_t seed, uint64_t stream_id, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  random_kernel<<<grid_for(n, 256), 256, 0, stream>>>(x, n, seed, stream_id);
  count_launch();
  return cudaGetLastError();
}

}  // namespace b200
