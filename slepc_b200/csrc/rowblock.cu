// Row-major block kernels for sm_100a: the Chebyshev-filter step (block SpMV with a fused
// three-term update), Gram products (tcgen05 TF32 tensor cores for the orthonormalisation, FP64 for
// the Rayleigh quotients), the block rotation Y = X M, column residual norms and layout
// conversions.  Layout: rowblock.h.  No SLEPc counterpart as kernels: they serve the
// mixed-precision form of the Hermitian eigensolver (mixed.cu), whose FP64 result replaces the
// EPSSolve eigenpairs.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>

#include "common.h"
#include "internal.h"
#include "kernels.h"
#include "ptx.h"
#include "rowblock.h"

namespace b200 {
namespace {

constexpr int kRbThreads = 256;
constexpr int kChunk = 8;  // nonzeros of a row whose gathers are issued together

// Lane mapping of a block row: 16-byte vector accesses (4 floats or 2 doubles), LPR lanes per row,
// CPL vectors per lane, RPI rows per warp iteration.
template <typename TX, int BP>
struct Map {
  static constexpr int VEC = 16 / (int)sizeof(TX);
  static constexpr int NVEC = BP / VEC;
  // 64-column blocks: FP32 with 8 lanes per row and two vectors each (4 rows per warp iteration:
  // twice the gathers in flight per warp, 7% faster than 16 lanes x one vector on the 128^3
  // Laplacian), FP64 with 16 lanes per row and two vectors each (2 rows per warp iteration)
  static constexpr int LPR = (BP == 64) ? (sizeof(TX) == 4 ? 8 : 16) : (NVEC < 32 ? NVEC : 32);
  static constexpr int CPL = NVEC / LPR;
  static constexpr int RPI = 32 / LPR;
};

__device__ __forceinline__ void vld(const float *p, float (&v)[4]) {
  const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
  v[0] = t.x;
  v[1] = t.y;
  v[2] = t.z;
  v[3] = t.w;
}
__device__ __forceinline__ void vld(const double *p, double (&v)[2]) {
  const double2 t = __ldg(reinterpret_cast<const double2 *>(p));
  v[0] = t.x;
  v[1] = t.y;
}
__device__ __forceinline__ void vst(float *p, const float (&v)[4]) {
  *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void vst(double *p, const double (&v)[2]) {
  *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
}

// Y = alpha (A X - shift X) - beta Z over the rows of the sliced-ELL copy.  One warp per 32-row
// slice: the slice's column indices and values are staged in the warp's shared memory with
// coalesced loads, then LPR lanes per row gather whole rows of X (16-byte vectors) for every
// nonzero of the row and accumulate in TX.
template <typename TV, typename TX, int BP>
__global__ void __launch_bounds__(kRbThreads) rb_spmm_kernel(int nslices, int n, const long long *__restrict__ off,
                                                             const int *__restrict__ width,
                                                             const unsigned *__restrict__ mask,
                                                             const TV *__restrict__ sval, const int *__restrict__ scol,
                                                             int wmax, const TX *__restrict__ X,
                                                             const TX *__restrict__ Z, TX *__restrict__ Y,
                                                             double alpha, double shift, double beta) {
  using M = Map<TX, BP>;
  extern __shared__ __align__(16) unsigned char sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int per_warp = 32 * wmax;
  int *wc = reinterpret_cast<int *>(sm) + (size_t)warp * per_warp;
  TV *wv = reinterpret_cast<TV *>(sm + (size_t)(kRbThreads / 32) * per_warp * sizeof(int)) + (size_t)warp * per_warp;
  const int sub = lane / M::LPR, li = lane % M::LPR;
  const int nwarps = gridDim.x * (kRbThreads / 32);
  for (int sl = blockIdx.x * (kRbThreads / 32) + warp; sl < nslices; sl += nwarps) {
    const int w = width[sl];
    const long long base = off[sl];
    const unsigned m = mask[sl];
    for (int k = 0; k < w; ++k) {
      wc[k * 32 + lane] = __ldg(scol + base + 32ll * k + lane);
      wv[k * 32 + lane] = __ldg(sval + base + 32ll * k + lane);
    }
    __syncwarp();
    for (int it = 0; it < 32; it += M::RPI) {
      const int i = it + sub;
      const int r = 32 * sl + i;
      if (r < n && ((m >> i) & 1u)) {
        // the row's own X and Z first, then every gather of a chunk of kChunk nonzeros before any
        // product: kChunk independent 16-byte loads per lane in flight (padding entries read the row
        // itself, already cached, with a zero coefficient)
        TX xr[M::CPL][M::VEC], z[M::CPL][M::VEC], acc[M::CPL][M::VEC];
#pragma unroll
        for (int cv = 0; cv < M::CPL; ++cv) {
          const size_t o = (size_t)r * BP + (size_t)(li + cv * M::LPR) * M::VEC;
          vld(X + o, xr[cv]);
          if (Z) vld(Z + o, z[cv]);
#pragma unroll
          for (int e = 0; e < M::VEC; ++e) acc[cv][e] = TX(0);
        }
        for (int k0 = 0; k0 < w; k0 += kChunk) {
          int cc[kChunk];
          TX aa[kChunk];
#pragma unroll
          for (int u = 0; u < kChunk; ++u) {
            const int k = k0 + u;
            const int c = k < w ? wc[k * 32 + i] : -1;
            cc[u] = c >= 0 ? c : r;
            aa[u] = c >= 0 ? (TX)wv[k * 32 + i] : TX(0);
          }
          TX xv[kChunk][M::CPL][M::VEC];
#pragma unroll
          for (int u = 0; u < kChunk; ++u)
#pragma unroll
            for (int cv = 0; cv < M::CPL; ++cv)
              vld(X + (size_t)cc[u] * BP + (size_t)(li + cv * M::LPR) * M::VEC, xv[u][cv]);
#pragma unroll
          for (int u = 0; u < kChunk; ++u)
#pragma unroll
            for (int cv = 0; cv < M::CPL; ++cv)
#pragma unroll
              for (int e = 0; e < M::VEC; ++e) acc[cv][e] = fma(aa[u], xv[u][cv][e], acc[cv][e]);
        }
#pragma unroll
        for (int cv = 0; cv < M::CPL; ++cv) {
          const size_t o = (size_t)r * BP + (size_t)(li + cv * M::LPR) * M::VEC;
          TX out[M::VEC];
#pragma unroll
          for (int e = 0; e < M::VEC; ++e) {
            double v = alpha * ((double)acc[cv][e] - shift * (double)xr[cv][e]);
            if (Z) v -= beta * (double)z[cv][e];
            out[e] = (TX)v;
          }
          vst(Y + o, out);
        }
      }
    }
    __syncwarp();
  }
}

// The rows the slices leave out (more nonzeros than a slice admits): one warp per row, the RPI
// lane groups taking every RPI-th nonzero, their sums combined by a shuffle tree.
template <typename TV, typename TX, int BP>
__global__ void __launch_bounds__(kRbThreads) rb_spmm_rest_kernel(int nrest, int n, const int *__restrict__ rows,
                                                                  const int *__restrict__ rowptr,
                                                                  const int *__restrict__ colind,
                                                                  const TV *__restrict__ vals,
                                                                  const TX *__restrict__ X, const TX *__restrict__ Z,
                                                                  TX *__restrict__ Y, double alpha, double shift,
                                                                  double beta) {
  using M = Map<TX, BP>;
  const int lane = threadIdx.x & 31;
  const int sub = lane / M::LPR, li = lane % M::LPR;
  const int nwarps = gridDim.x * (kRbThreads / 32);
  for (int q = blockIdx.x * (kRbThreads / 32) + (threadIdx.x >> 5); q < nrest; q += nwarps) {
    const int r = rows[q];
    if (r < 0 || r >= n) continue;
    const int p0 = rowptr[r], p1 = rowptr[r + 1];
    TX acc[M::CPL][M::VEC];
#pragma unroll
    for (int cv = 0; cv < M::CPL; ++cv)
#pragma unroll
      for (int e = 0; e < M::VEC; ++e) acc[cv][e] = TX(0);
    for (int p = p0 + sub; p < p1; p += M::RPI) {
      const int c = __ldg(colind + p);
      const TX a = (TX)__ldg(vals + p);
#pragma unroll
      for (int cv = 0; cv < M::CPL; ++cv) {
        TX x[M::VEC];
        vld(X + (size_t)c * BP + (size_t)(li + cv * M::LPR) * M::VEC, x);
#pragma unroll
        for (int e = 0; e < M::VEC; ++e) acc[cv][e] = fma(a, x[e], acc[cv][e]);
      }
    }
#pragma unroll
    for (int o = M::LPR; o < 32; o <<= 1)
#pragma unroll
      for (int cv = 0; cv < M::CPL; ++cv)
#pragma unroll
        for (int e = 0; e < M::VEC; ++e) acc[cv][e] += __shfl_xor_sync(0xffffffffu, acc[cv][e], o);
    if (sub == 0) {
#pragma unroll
      for (int cv = 0; cv < M::CPL; ++cv) {
        const size_t o = (size_t)r * BP + (size_t)(li + cv * M::LPR) * M::VEC;
        TX xr[M::VEC], z[M::VEC], out[M::VEC];
        vld(X + o, xr);
        if (Z) vld(Z + o, z);
#pragma unroll
        for (int e = 0; e < M::VEC; ++e) {
          double v = alpha * ((double)acc[cv][e] - shift * (double)xr[e]);
          if (Z) v -= beta * (double)z[e];
          out[e] = (TX)v;
        }
        vst(Y + o, out);
      }
    }
  }
}

// ---------------------------------------------------------------- tensor-core Gram (TF32)
//
// G = X^T Y over row tiles of KT rows.  Warp 0 (one lane) streams each tile of X (and Y) into a
// ring of shared-memory stages with 2-D TMA loads (128-byte swizzle with 32-byte atoms, the only
// layout the tensor cores take for MN-major TF32; one box per 32-column strip);
// warp 1 (one lane) issues, for every 8 rows of the tile, one tcgen05.mma kind::tf32 of shape
// BP x BP x 8 with both operands MN-major (the strips are the MN blocks, LBO apart), accumulating in
// TMEM, and commits each stage back to the producer; at the end all four warps read the BP x BP FP32
// accumulator out of TMEM (warp w owns TMEM lanes 32w..32w+31) into the CTA's partial-sum slot.
// Every wait is bounded; a timeout is reported through err and the CTA writes zeros.
template <int BP, bool CROSS>
struct GramTc {
  static constexpr int KT = BP == 64 ? 128 : 64;  // rows of a tile (the K extent)
  static constexpr int STRIP = KT * 128;          // bytes of one 32-column strip of a tile
  static constexpr int TILE = STRIP * (BP / 32);  // bytes of one operand tile
  static constexpr int STAGE = TILE * (CROSS ? 2 : 1);
  static constexpr int STAGES = CROSS ? 3 : 6;
  static constexpr size_t SMEM = (size_t)STAGE * STAGES + 1024;  // + alignment slack for the 1024-byte atoms
};

template <int BP, bool CROSS>
__global__ void __launch_bounds__(128, 1) rb_gram_tf32_kernel(const __grid_constant__ CUtensorMap tx,
                                                              const __grid_constant__ CUtensorMap ty, int ntiles,
                                                              float *__restrict__ partials, int *__restrict__ err) {
  using C = GramTc<BP, CROSS>;
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full[C::STAGES], empty[C::STAGES], done;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
  __shared__ int consumed, issued;
  const uint32_t s0 = ptx::smem_u32(smem_raw);
  unsigned char *smem = smem_raw + ((1024u - (s0 & 1023u)) & 1023u);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t0 = (int)((long long)ntiles * blockIdx.x / gridDim.x);
  const int t1 = (int)((long long)ntiles * (blockIdx.x + 1) / gridDim.x);
  const int nt = t1 - t0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < C::STAGES; ++s) {
      ptx::mbar_init(&full[s], 1);
      ptx::mbar_init(&empty[s], 1);
    }
    ptx::mbar_init(&done, 1);
    abort_flag = 0;
    consumed = 0;
    issued = 0;
    ptx::fence_mbar_init();
  }
  if (warp == 2) {
    ptx::tmem_alloc(&tmem_base, BP);
    ptx::tmem_relinquish();
  }
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem = tmem_base;

  if (warp == 0 && lane == 0) {
    int t = 0;
    for (; t < nt; ++t) {
      const int s = t % C::STAGES;
      if (t >= C::STAGES && !ptx::mbar_wait(&empty[s], ((t / C::STAGES) - 1) & 1)) {
        abort_flag = 1;
        break;
      }
      if (abort_flag) break;
      unsigned char *st = smem + (size_t)s * C::STAGE;
      ptx::mbar_arrive_expect_tx(&full[s], C::STAGE);
      const int row = (t0 + t) * C::KT;
#pragma unroll
      for (int h = 0; h < BP / 32; ++h) ptx::tma_load_2d(st + h * C::STRIP, &tx, h * 32, row, &full[s]);
      if (CROSS)
#pragma unroll
        for (int h = 0; h < BP / 32; ++h) ptx::tma_load_2d(st + C::TILE + h * C::STRIP, &ty, h * 32, row, &full[s]);
    }
    issued = t;
  } else if (warp == 1 && lane == 0) {
    constexpr uint32_t idesc = ptx::idesc_tf32_mn(BP, BP);
    int t = 0;
    for (; t < nt; ++t) {
      const int s = t % C::STAGES;
      if (!ptx::mbar_wait(&full[s], (t / C::STAGES) & 1)) {
        abort_flag = 1;
        break;
      }
      ptx::tc_fence_after();
      const uint32_t a0 = ptx::smem_u32(smem + (size_t)s * C::STAGE);
      const uint32_t b0 = CROSS ? a0 + C::TILE : a0;
#pragma unroll
      for (int k = 0; k < C::KT / 8; ++k)
        ptx::mma_tf32(tmem, ptx::smem_desc_sw128_32b(a0 + 1024u * k, C::STRIP, 512),
                      ptx::smem_desc_sw128_32b(b0 + 1024u * k, C::STRIP, 512), idesc, t > 0 || k > 0);
      ptx::mma_commit(&empty[s]);  // the stage is free once these MMAs have read it
    }
    consumed = t;
    ptx::mma_commit(&done);  // every MMA issued above
  }
  __syncwarp();
  if (!ptx::mbar_wait(&done, 0)) abort_flag = 1;
  __syncthreads();
  ptx::tc_fence_after();
  float *out = partials + (size_t)blockIdx.x * BP * BP;
  if (nt > 0 && !abort_flag) {
    // M = 64: rows 16w..16w+15 in lanes 32w..32w+15; M = 128: row 32w + t in lane 32w + t
    const int row = BP == 64 ? warp * 16 + (lane & 15) : warp * 32 + lane;
    const bool write = BP == 64 ? lane < 16 : true;
    const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < BP; c0 += 8) {
      float v[8];
      ptx::tmem_ld8(tl + (uint32_t)c0, v);
      ptx::tmem_wait_ld();
      if (write) {
        float4 *o = reinterpret_cast<float4 *>(out + (size_t)row * BP + c0);
        o[0] = make_float4(v[0], v[1], v[2], v[3]);
        o[1] = make_float4(v[4], v[5], v[6], v[7]);
      }
    }
  } else {
    for (int e = threadIdx.x; e < BP * BP; e += blockDim.x) out[e] = 0.f;
  }
  if (threadIdx.x == 0) {
    if (abort_flag) atomicOr(err, kDevErrTimeout);
    // copies that were issued but never consumed (only after a timeout) land before the CTA exits
    for (int t = consumed; t < issued; ++t) ptx::mbar_wait(&full[t % C::STAGES], (t / C::STAGES) & 1);
  }
  ptx::tc_fence_before();
  __syncthreads();
  if (warp == 2) ptx::tmem_dealloc(tmem, BP);
}

// G[e] = sum over the CTAs of partials[cta][e] in CTA order (FP64), e < bp * bp.
template <typename TP>
__global__ void rb_reduce_kernel(const TP *__restrict__ partials, int nparts, int len, double *__restrict__ G) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= len) return;
  double s = 0.0;
  for (int b = 0; b < nparts; ++b) s += (double)partials[(size_t)b * len + e];
  G[e] = s;
}

// ---------------------------------------------------------------- FP64 Gram pair
//
// G = X^T X and H = X^T W, every product and sum in FP64 (FP32 inputs are exact in FP64).  Grid
// (row ranges) x (64 x 64 quadrants of the bp x bp result); 256 threads, a 4 x 4 register tile of
// G and of H per thread; 16-row slabs of the three column strips staged in shared memory, the next
// slab fetched into registers while the current one is consumed.
constexpr int kSlab = 16;
constexpr int kQ = 64;
template <typename TX, int BP>
__global__ void __launch_bounds__(256) rb_gram2_kernel(const TX *__restrict__ X, const TX *__restrict__ W, int n,
                                                       int rows_per_cta, double *__restrict__ partials) {
  __shared__ double xa[kSlab][kQ + 2], xb[kSlab][kQ + 2], wb[kSlab][kQ + 2];
  constexpr int NQ = BP / kQ;
  const int qi = blockIdx.y / NQ, qj = blockIdx.y % NQ;
  const int ti = threadIdx.x / 16, tj = threadIdx.x % 16;
  double g[4][4], h[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) g[a][b] = h[a][b] = 0.0;
  const int r0 = blockIdx.x * rows_per_cta, r1 = min(n, r0 + rows_per_cta);
  // the next slab is fetched into registers while the current one is consumed from shared memory
  constexpr int kPer = kSlab * kQ / 256;
  double pa[kPer], pb[kPer], pw[kPer];
  auto fetch = [&](int slab) {
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int e = threadIdx.x + 256 * u, rr = e / kQ, c = e % kQ, r = slab + rr;
      const bool in = r < r1;
      pa[u] = in ? (double)X[(size_t)r * BP + qi * kQ + c] : 0.0;
      pb[u] = in ? (double)X[(size_t)r * BP + qj * kQ + c] : 0.0;
      pw[u] = in ? (double)W[(size_t)r * BP + qj * kQ + c] : 0.0;
    }
  };
  if (r0 < r1) fetch(r0);
  for (int slab = r0; slab < r1; slab += kSlab) {
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int e = threadIdx.x + 256 * u, rr = e / kQ, c = e % kQ;
      xa[rr][c] = pa[u];
      xb[rr][c] = pb[u];
      wb[rr][c] = pw[u];
    }
    __syncthreads();
    if (slab + kSlab < r1) fetch(slab + kSlab);
#pragma unroll 4
    for (int rr = 0; rr < kSlab; ++rr) {
      double a[4], b[4], w[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        a[u] = xa[rr][ti * 4 + u];
        b[u] = xb[rr][tj * 4 + u];
        w[u] = wb[rr][tj * 4 + u];
      }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          g[p][q] = fma(a[p], b[q], g[p][q]);
          h[p][q] = fma(a[p], w[q], h[p][q]);
        }
    }
    __syncthreads();
  }
  double *pg = partials + (size_t)blockIdx.x * 2 * BP * BP;
  double *ph = pg + (size_t)BP * BP;
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const size_t e = (size_t)(qi * kQ + ti * 4 + p) * BP + qj * kQ + tj * 4 + q;
      pg[e] = g[p][q];
      ph[e] = h[p][q];
    }
}

// ---------------------------------------------------------------- FP64 Gram pair on the FP64 MMA path
//
// The same G = X^T X and H = X^T W (64-column row-major blocks, products and sums in FP64) with
// mma.sync.m16n8k16 f64: per 32-row chunk the CTA converts X and W to FP64 in shared memory (row
// stride 68 doubles, 4 mod 16: every fragment load of a half warp hits distinct banks); warp w
// accumulates the 16 x 64 strip 16 (w % 4).. of G (w < 4) or of H (w >= 4) over its CTA's rows,
// the next chunk fetched into registers while the current one is consumed.  Fragments (g = lane / 4,
// t = lane % 4): A = X^T, element e at row g + 8 (e % 2), depth t + 4 (e / 2); B element e at depth
// t + 4 e, column g; D element e at row g + 8 (e / 2), column 2 t + e % 2.  The CTA's partial sums
// go to partials[cta][G then H] as rb_gram2_kernel writes them.
constexpr int kMmaRows = 32;   // rows per shared chunk (two 16-deep MMA steps)
constexpr int kMmaLd = 68;     // doubles per chunk row in shared memory
__device__ __forceinline__ void dmma16816(double (&d)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
        "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

template <typename TX>
__global__ void __launch_bounds__(256) rb_gram2_mma_kernel(const TX *__restrict__ X, const TX *__restrict__ W, int n,
                                                           int rows_per_cta, double *__restrict__ partials) {
  constexpr int BP = 64;
  __shared__ double xs[kMmaRows * kMmaLd], ws[kMmaRows * kMmaLd];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int mb = warp & 3;          // 16-row strip of the output
  const bool hw = warp >= 4;        // H = X^T W (else G = X^T X)
  const double *bsrc = hw ? ws : xs;
  double acc[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
  const int r0 = blockIdx.x * rows_per_cta, r1 = min(n, r0 + rows_per_cta);
  // a chunk: kMmaRows x 64 values of X and of W, 8 of each per thread; element e = tid + 256 u, so a
  // warp reads 32 consecutive values of a row and writes 32 consecutive doubles (no bank conflicts)
  constexpr int kPer = kMmaRows * BP / 256;
  TX px[kPer], pw[kPer];
  auto fetch = [&](int c0) {
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int e = threadIdx.x + 256 * u, rr = e / BP, c = e % BP, r = c0 + rr;
      const bool in = r < r1;
      px[u] = in ? X[(size_t)r * BP + c] : TX(0);
      pw[u] = in ? W[(size_t)r * BP + c] : TX(0);
    }
  };
  if (r0 < r1) fetch(r0);
  for (int c0 = r0; c0 < r1; c0 += kMmaRows) {
    __syncthreads();  // the previous chunk is consumed
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int e = threadIdx.x + 256 * u, rr = e / BP, c = e % BP;
      xs[rr * kMmaLd + c] = (double)px[u];
      ws[rr * kMmaLd + c] = (double)pw[u];
    }
    __syncthreads();
    if (c0 + kMmaRows < r1) fetch(c0 + kMmaRows);
#pragma unroll
    for (int k0 = 0; k0 < kMmaRows; k0 += 16) {
      double a[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) a[e] = xs[(k0 + t + 4 * (e >> 1)) * kMmaLd + 16 * mb + g + 8 * (e & 1)];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        double b[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) b[e] = bsrc[(k0 + t + 4 * e) * kMmaLd + 8 * j + g];
        dmma16816(acc[j], a, b);
      }
    }
  }
  double *out = partials + (size_t)blockIdx.x * 2 * BP * BP + (hw ? (size_t)BP * BP : 0);
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int row = 16 * mb + g + 8 * (e >> 1), col = 8 * j + 2 * t + (e & 1);
      out[(size_t)row * BP + col] = acc[j][e];
    }
}

// ---------------------------------------------------------------- rotation Y = X M
//
// 256 threads; a tile of RT = 16 TR rows of X in shared memory (row stride BP + 1), M (converted to
// TX) in shared memory; thread (tr, tc) computes rows tr*TR..+TR-1, columns tc*TC..+TC-1 (TC =
// BP/16) and writes them with 16-byte stores.
template <typename TX, int BP>
struct Rot {
  static constexpr int TR = sizeof(TX) == 4 ? 8 : 4;
  static constexpr int TC = BP / 16;
  static constexpr int RT = 16 * TR;
  static constexpr size_t SMEM = sizeof(TX) * ((size_t)RT * (BP + 1) + (size_t)BP * BP);
};

template <typename TX, int BP>
__global__ void __launch_bounds__(256) rb_rotate_kernel(const TX *__restrict__ X, TX *__restrict__ Y, int n,
                                                        const double *__restrict__ Mg) {
  using R = Rot<TX, BP>;
  extern __shared__ __align__(16) unsigned char sm[];
  TX *Ms = reinterpret_cast<TX *>(sm);
  TX *Xs = Ms + (size_t)BP * BP;
  for (int e = threadIdx.x; e < BP * BP; e += 256) Ms[e] = (TX)Mg[e];
  const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
  const int ntiles = (n + R::RT - 1) / R::RT;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int row0 = tile * R::RT;
    __syncthreads();
    for (int e = threadIdx.x; e < R::RT * BP; e += 256) {
      const int rr = e / BP, c = e % BP, r = row0 + rr;
      Xs[rr * (BP + 1) + c] = r < n ? X[(size_t)r * BP + c] : TX(0);
    }
    __syncthreads();
    TX acc[R::TR][R::TC];
#pragma unroll
    for (int i = 0; i < R::TR; ++i)
#pragma unroll
      for (int j = 0; j < R::TC; ++j) acc[i][j] = TX(0);
#pragma unroll 2
    for (int k = 0; k < BP; ++k) {
      TX x[R::TR], m[R::TC];
#pragma unroll
      for (int i = 0; i < R::TR; ++i) x[i] = Xs[(tr * R::TR + i) * (BP + 1) + k];
#pragma unroll
      for (int j = 0; j < R::TC; ++j) m[j] = Ms[k * BP + tc * R::TC + j];
#pragma unroll
      for (int i = 0; i < R::TR; ++i)
#pragma unroll
        for (int j = 0; j < R::TC; ++j) acc[i][j] = fma(x[i], m[j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < R::TR; ++i) {
      const int r = row0 + tr * R::TR + i;
      if (r < n) {
        TX *dst = Y + (size_t)r * BP + tc * R::TC;
        constexpr int V = 16 / (int)sizeof(TX);
#pragma unroll
        for (int j = 0; j < R::TC; j += V) {
          TX v[V];
#pragma unroll
          for (int u = 0; u < V; ++u) v[u] = acc[i][j + u];
          vst(dst + j, v);
        }
      }
    }
  }
}

// ---------------------------------------------------------------- residual norms
template <typename TX, int BP>
__global__ void __launch_bounds__(256) rb_resid_kernel(const TX *__restrict__ W, const TX *__restrict__ X, int n,
                                                       const double *__restrict__ theta, double *__restrict__ work) {
  constexpr int RPB = 256 / BP;  // rows a block covers per step
  __shared__ double red[256];
  const int c = threadIdx.x % BP, rs = threadIdx.x / BP;
  const double th = theta[c];
  double acc = 0.0;
  for (long long r = (long long)blockIdx.x * RPB + rs; r < n; r += (long long)gridDim.x * RPB) {
    const double d = (double)W[(size_t)r * BP + c] - th * (double)X[(size_t)r * BP + c];
    acc = fma(d, d, acc);
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < BP) {
    double s = 0.0;
    for (int q = 0; q < RPB; ++q) s += red[q * BP + threadIdx.x];
    work[(size_t)blockIdx.x * BP + threadIdx.x] = s;
  }
}

__global__ void rb_resid_final_kernel(const double *__restrict__ work, int nparts, int bp, double *__restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= bp) return;
  double s = 0.0;
  for (int b = 0; b < nparts; ++b) s += work[(size_t)b * bp + c];
  out[c] = sqrt(s);
}

// ---------------------------------------------------------------- conversions
__global__ void rb_widen_kernel(const float *__restrict__ X, double *__restrict__ Y, long long count) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x)
    Y[i] = (double)X[i];
}

// 32 x 32 tiles through shared memory: rows of the block -> columns of V.
template <typename TX>
__global__ void rb_to_colmajor_kernel(const TX *__restrict__ X, int n, int bp, int ncols, double *__restrict__ V,
                                      int ld) {
  __shared__ double t[32][33];
  const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  for (int q = threadIdx.y; q < 32; q += blockDim.y) {
    const int r = r0 + q, c = c0 + threadIdx.x;
    t[q][threadIdx.x] = (r < n && c < bp) ? (double)X[(size_t)r * bp + c] : 0.0;
  }
  __syncthreads();
  for (int q = threadIdx.y; q < 32; q += blockDim.y) {
    const int c = c0 + q, r = r0 + threadIdx.x;
    if (c < ncols && r < n) V[(size_t)c * ld + r] = t[threadIdx.x][q];
  }
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Counter-based N(0,1) entries (Box-Muller on two 53-bit uniforms of a hash of seed, row, column).
template <typename TX>
__global__ void rb_init_kernel(TX *__restrict__ X, int n, int bp, const double *__restrict__ src, int lds, int nsrc,
                               uint64_t seed) {
  const long long count = (long long)n * bp;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / bp), c = (int)(i % bp);
    double v;
    if (c < nsrc) {
      v = src[(size_t)c * lds + r];
    } else {
      const uint64_t h1 = mix64(seed ^ mix64(((uint64_t)r << 20) ^ (uint64_t)c));
      const uint64_t h2 = mix64(h1 ^ 0xD1B54A32D192ED03ull);
      const double u1 = ((h1 >> 11) + 1) * (1.0 / 9007199254740993.0);  // (0, 1]
      const double u2 = (h2 >> 11) * (1.0 / 9007199254740992.0);
      v = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    }
    X[i] = (TX)v;
  }
}

int grid_for(long long count, int threads) {
  long long g = (count + threads - 1) / threads;
  const long long cap = (long long)num_sms_host() * 8;
  if (g > cap) g = cap;
  return (int)(g > 0 ? g : 1);
}

template <typename K>
cudaError_t ensure_smem(K kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename TV, typename TX, int BP>
cudaError_t spmm_t(const SpmvSell &S, int n, const int *rowptr, const int *colind, const TV *cvals, const TV *svals,
                   const TX *X, const TX *Z, TX *Y, double alpha, double shift, double beta, cudaStream_t s) {
  const int wmax = S.max_width > 0 ? S.max_width : 1;
  const size_t smem = (size_t)(kRbThreads / 32) * 32 * wmax * (sizeof(int) + sizeof(TV));
  cudaError_t e = ensure_smem(rb_spmm_kernel<TV, TX, BP>, smem);
  if (e != cudaSuccess) return e;
  if (S.nslices > 0) {
    // one resident wave: the grid-stride loop then spreads the slices evenly over the CTAs
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rb_spmm_kernel<TV, TX, BP>, kRbThreads, smem);
    if (e != cudaSuccess) return e;
    per_sm = per_sm < 1 ? 1 : per_sm;
    long long g = (S.nslices + (kRbThreads / 32) - 1) / (kRbThreads / 32);
    const long long cap = (long long)num_sms_host() * per_sm;
    if (g > cap) g = cap;
    rb_spmm_kernel<TV, TX, BP><<<(int)g, kRbThreads, smem, s>>>(S.nslices, n, S.off, S.width, S.mask, svals, S.cols,
                                                                 wmax, X, Z, Y, alpha, shift, beta);
    count_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (S.nrest > 0) {
    rb_spmm_rest_kernel<TV, TX, BP><<<grid_for((long long)S.nrest * 32, kRbThreads), kRbThreads, 0, s>>>(
        S.nrest, n, S.rest_rows, rowptr, colind, cvals, X, Z, Y, alpha, shift, beta);
    count_launch();
    e = cudaGetLastError();
  }
  return e;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
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

template <int BP, bool CROSS>
cudaError_t gram_tc_t(const CUtensorMap &tx, const CUtensorMap &ty, int n, double *G, float *work, int *err,
                      cudaStream_t s) {
  using C = GramTc<BP, CROSS>;
  cudaError_t e = cudaFuncSetAttribute(rb_gram_tf32_kernel<BP, CROSS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)C::SMEM);
  if (e != cudaSuccess) return e;
  const int ntiles = (n + C::KT - 1) / C::KT;
  const int grid = rb_gram_ctas(n, BP);
  rb_gram_tf32_kernel<BP, CROSS><<<grid, 128, C::SMEM, s>>>(tx, ty, ntiles, work, err);
  count_launch();
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  rb_reduce_kernel<float><<<(BP * BP + 255) / 256, 256, 0, s>>>(work, grid, BP * BP, G);
  count_launch();
  return cudaGetLastError();
}

template <typename TX, int BP>
cudaError_t gram2_t(const TX *X, const TX *W, int n, double *GH, double *work, cudaStream_t s) {
  const int ctas = rb_gram_ctas(n, BP);
  if constexpr (BP == 64) {  // the FP64 MMA path
    int rows = (n + ctas - 1) / ctas;
    rows = (rows + kMmaRows - 1) / kMmaRows * kMmaRows;
    const int gx = (n + rows - 1) / rows;
    rb_gram2_mma_kernel<TX><<<gx > 0 ? gx : 1, 256, 0, s>>>(X, W, n, rows, work);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    rb_reduce_kernel<double><<<(2 * BP * BP + 255) / 256, 256, 0, s>>>(work, gx > 0 ? gx : 1, 2 * BP * BP, GH);
    count_launch();
    return cudaGetLastError();
  }
  int rows = (n + ctas - 1) / ctas;
  rows = (rows + kSlab - 1) / kSlab * kSlab;
  const int gx = (n + rows - 1) / rows;
  dim3 grid(gx > 0 ? gx : 1, (BP / kQ) * (BP / kQ));
  rb_gram2_kernel<TX, BP><<<grid, 256, 0, s>>>(X, W, n, rows, work);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // the partials hold G then H per row range: reduce both in one pass over 2 bp^2 entries
  rb_reduce_kernel<double><<<(2 * BP * BP + 255) / 256, 256, 0, s>>>(work, grid.x, 2 * BP * BP, GH);
  count_launch();
  return cudaGetLastError();
}

template <typename TX, int BP>
cudaError_t rotate_t(const TX *X, TX *Y, int n, const double *M, cudaStream_t s) {
  using R = Rot<TX, BP>;
  cudaError_t e = ensure_smem(rb_rotate_kernel<TX, BP>, R::SMEM);
  if (e != cudaSuccess) return e;
  const int ntiles = (n + R::RT - 1) / R::RT;
  int per_sm = (int)((220 * 1024) / R::SMEM);
  per_sm = per_sm < 1 ? 1 : per_sm;
  int grid = num_sms_host() * per_sm;
  if (grid > ntiles) grid = ntiles;
  rb_rotate_kernel<TX, BP><<<grid > 0 ? grid : 1, 256, R::SMEM, s>>>(X, Y, n, M);
  count_launch();
  return cudaGetLastError();
}

template <typename TX, int BP>
cudaError_t resid_t(const TX *W, const TX *X, int n, const double *theta, double *out, double *work, cudaStream_t s) {
  constexpr int RPB = 256 / BP;
  long long g = ((long long)n + RPB - 1) / RPB;
  if (g > 1024) g = 1024;
  if (g < 1) g = 1;
  rb_resid_kernel<TX, BP><<<(int)g, 256, 0, s>>>(W, X, n, theta, work);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  rb_resid_final_kernel<<<1, BP, 0, s>>>(work, (int)g, BP, out);
  count_launch();
  return cudaGetLastError();
}

}  // namespace

int rb_gram_ctas(int n, int bp) {
  const int kt = bp == 64 ? 128 : 64;
  const int tiles = (n + kt - 1) / kt;
  const int sms = num_sms_host();
  return tiles < sms ? (tiles > 0 ? tiles : 1) : sms;
}

cudaError_t rb_spmm_launch(const SpmvSell &S, int n, const int *rowptr, const int *colind, const void *cvals,
                           const void *svals, bool vals_f32, bool x32, int bp, const void *X, const void *Z, void *Y,
                           double alpha, double shift, double beta, cudaStream_t s) {
#define RB_SPMM(TV, TX, BPV)                                                                                       \
  return spmm_t<TV, TX, BPV>(S, n, rowptr, colind, static_cast<const TV *>(cvals), static_cast<const TV *>(svals), \
                             static_cast<const TX *>(X), static_cast<const TX *>(Z), static_cast<TX *>(Y), alpha,  \
                             shift, beta, s)
  if (bp == 64) {
    if (x32) {
      if (vals_f32) RB_SPMM(float, float, 64);
      RB_SPMM(double, float, 64);
    }
    if (vals_f32) RB_SPMM(float, double, 64);
    RB_SPMM(double, double, 64);
  }
  if (bp == 128) {
    if (x32) {
      if (vals_f32) RB_SPMM(float, float, 128);
      RB_SPMM(double, float, 128);
    }
    if (vals_f32) RB_SPMM(float, double, 128);
    RB_SPMM(double, double, 128);
  }
#undef RB_SPMM
  return cudaErrorInvalidValue;
}

cudaError_t rb_make_tmap_f32(CUtensorMap *tm, const float *X, int n, int bp) {
  memset(tm, 0, sizeof(*tm));
  if ((bp != 64 && bp != 128) || n <= 0 || ((uintptr_t)X & 15)) return cudaErrorInvalidValue;
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_tiled();
  if (!enc) return cudaErrorNotSupported;
  const int kt = bp == 64 ? 128 : 64;
  const cuuint64_t dims[2] = {(cuuint64_t)bp, (cuuint64_t)n};
  const cuuint64_t strides[1] = {(cuuint64_t)bp * sizeof(float)};
  const cuuint32_t box[2] = {32, (cuuint32_t)kt};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(X), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t rb_gram_tf32_launch(const CUtensorMap &tx, const CUtensorMap *ty, int n, int bp, double *G, float *work,
                                int *err, cudaStream_t s) {
  if (bp == 64) return ty ? gram_tc_t<64, true>(tx, *ty, n, G, work, err, s) : gram_tc_t<64, false>(tx, tx, n, G, work, err, s);
  if (bp == 128)
    return ty ? gram_tc_t<128, true>(tx, *ty, n, G, work, err, s) : gram_tc_t<128, false>(tx, tx, n, G, work, err, s);
  return cudaErrorInvalidValue;
}

cudaError_t rb_gram2_f64_launch(const void *X, const void *W, bool x32, int n, int bp, double *GH, double *work,
                                cudaStream_t s) {
  if (bp == 64)
    return x32 ? gram2_t<float, 64>(static_cast<const float *>(X), static_cast<const float *>(W), n, GH, work, s)
               : gram2_t<double, 64>(static_cast<const double *>(X), static_cast<const double *>(W), n, GH, work, s);
  if (bp == 128)
    return x32 ? gram2_t<float, 128>(static_cast<const float *>(X), static_cast<const float *>(W), n, GH, work, s)
               : gram2_t<double, 128>(static_cast<const double *>(X), static_cast<const double *>(W), n, GH, work, s);
  return cudaErrorInvalidValue;
}

cudaError_t rb_rotate_launch(const void *X, void *Y, bool x32, int n, int bp, const double *M, cudaStream_t s) {
  if (bp == 64)
    return x32 ? rotate_t<float, 64>(static_cast<const float *>(X), static_cast<float *>(Y), n, M, s)
               : rotate_t<double, 64>(static_cast<const double *>(X), static_cast<double *>(Y), n, M, s);
  if (bp == 128)
    return x32 ? rotate_t<float, 128>(static_cast<const float *>(X), static_cast<float *>(Y), n, M, s)
               : rotate_t<double, 128>(static_cast<const double *>(X), static_cast<double *>(Y), n, M, s);
  return cudaErrorInvalidValue;
}

cudaError_t rb_resid_launch(const void *W, const void *X, bool x32, int n, int bp, const double *theta, double *out,
                            double *work, cudaStream_t s) {
  if (bp == 64)
    return x32 ? resid_t<float, 64>(static_cast<const float *>(W), static_cast<const float *>(X), n, theta, out, work, s)
               : resid_t<double, 64>(static_cast<const double *>(W), static_cast<const double *>(X), n, theta, out,
                                     work, s);
  if (bp == 128)
    return x32 ? resid_t<float, 128>(static_cast<const float *>(W), static_cast<const float *>(X), n, theta, out, work,
                                     s)
               : resid_t<double, 128>(static_cast<const double *>(W), static_cast<const double *>(X), n, theta, out,
                                      work, s);
  return cudaErrorInvalidValue;
}

cudaError_t rb_widen_launch(const float *X, double *Y, long long count, cudaStream_t s) {
  rb_widen_kernel<<<grid_for(count, 256), 256, 0, s>>>(X, Y, count);
  count_launch();
  return cudaGetLastError();
}

cudaError_t rb_to_colmajor_launch(const void *X, bool x32, int n, int bp, int ncols, double *V, int ld,
                                  cudaStream_t s) {
  dim3 grid((n + 31) / 32, (bp + 31) / 32), block(32, 8);
  if (x32) rb_to_colmajor_kernel<float><<<grid, block, 0, s>>>(static_cast<const float *>(X), n, bp, ncols, V, ld);
  else rb_to_colmajor_kernel<double><<<grid, block, 0, s>>>(static_cast<const double *>(X), n, bp, ncols, V, ld);
  count_launch();
  return cudaGetLastError();
}

cudaError_t rb_init_launch(void *X, bool x32, int n, int bp, const double *src, int lds, int nsrc, uint64_t seed,
                           cudaStream_t s) {
  const long long count = (long long)n * bp;
  if (x32) rb_init_kernel<float><<<grid_for(count, 256), 256, 0, s>>>(static_cast<float *>(X), n, bp, src, lds, nsrc, seed);
  else rb_init_kernel<double><<<grid_for(count, 256), 256, 0, s>>>(static_cast<double *>(X), n, bp, src, lds, nsrc, seed);
  count_launch();
  return cudaGetLastError();
}

}  // namespace b200

using namespace b200;

extern "C" b200_status b200_rowblock_gram(int n, int bp, const float *X, const float *Y, int tensor_cores, double *G,
                                          void *stream) {
  B200_ARG_CHECK(n > 0 && (bp == 64 || bp == 128) && X && G, "n > 0, bp = 64 or 128, X and G required");
  B200_ARG_CHECK((((uintptr_t)X | (uintptr_t)(Y ? Y : X)) & 15) == 0, "X and Y must be 16-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  const int ctas = rb_gram_ctas(n, bp);
  const size_t sq = (size_t)bp * bp;
  double *work = nullptr, *gh = nullptr;
  int *err = nullptr;
  const size_t wbytes = std::max(sizeof(double) * 2 * sq * ctas, sizeof(float) * sq * ctas);
  B200_CUDA_CHECK(cudaMalloc(&work, wbytes));
  if (cudaMalloc(&gh, sizeof(double) * 2 * sq) != cudaSuccess || cudaMalloc(&err, sizeof(int)) != cudaSuccess) {
    cudaFree(work);
    cudaFree(gh);
    b200_set_last_error(__FILE__, __LINE__, "cudaMalloc failed");
    return B200_ERR_NOMEM;
  }
  cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), s);
  if (e == cudaSuccess) {
    if (tensor_cores) {
      CUtensorMap tx, ty;
      e = rb_make_tmap_f32(&tx, X, n, bp);
      if (e == cudaSuccess && Y) e = rb_make_tmap_f32(&ty, Y, n, bp);
      if (e == cudaSuccess) e = rb_gram_tf32_launch(tx, Y ? &ty : nullptr, n, bp, G, reinterpret_cast<float *>(work), err, s);
    } else {
      e = rb_gram2_f64_launch(X, Y ? Y : X, true, n, bp, gh, work, s);
      if (e == cudaSuccess) e = cudaMemcpyAsync(G, gh + sq, sizeof(double) * sq, cudaMemcpyDeviceToDevice, s);
    }
  }
  int herr = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(work);
  cudaFree(gh);
  cudaFree(err);
  B200_CUDA_CHECK(e);
  if (herr) {
    b200_set_last_error(__FILE__, __LINE__, "the Gram kernel reported a device-side timeout");
    return B200_ERR_DEVICE;
  }
  return B200_OK;
}
