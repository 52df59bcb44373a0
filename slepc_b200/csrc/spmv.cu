// CSR sparse matrix-vector product y = A x in FP64 for sm_100a.
//
// Replaces PETSc's MATAIJCUSPARSE MatMult behind BVMatMultColumn
// (src/sys/classes/bv/interface/bvops.c:862-890) and STApply
// (src/sys/classes/st/interface/stsolve.c:45-60).
//
// Two schedules:
//  * spmv_rowblock_kernel (used by b200_mat): rows are grouped on the host
//    into blocks of at most kTileNnz nonzeros and kTileRows rows.  A CTA
//    streams its block's values and column indices with coalesced,
//    independent loads (many in flight per thread), multiplies by the
//    gathered x (read-only path: neighbouring rows reuse x), keeps the
//    rounded products in shared memory, then sums every row in index order
//    with plain adds -- the order of PETSc's MatMult_SeqAIJ, so short rows
//    give the same bits as a sequential CPU loop.  A row longer than
//    kTileNnz gets a block of its own and a CTA-wide tree reduction.
//  * spmv_csr_kernel (the stateless b200_csr_spmv entry): LPR lanes per row.
#include "common.h"
#include "kernels.h"

namespace b200 {

namespace {

constexpr int kSpmvThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

__global__ void __launch_bounds__(kSpmvThreads) spmv_rowblock_kernel(const int *__restrict__ blocks,
                                                                     const int *__restrict__ rowptr,
                                                                     const int *__restrict__ colind,
                                                                     const double *__restrict__ vals,
                                                                     const double *__restrict__ x,
                                                                     double *__restrict__ y,
                                                                     const GsState *__restrict__ st, int step) {
  if (st && st->halt && st->halt_step < step) return;
  __shared__ double prod[kTileNnz];
  __shared__ int rp[kTileRows + 1];
  __shared__ double red[kSpmvThreads / 32];
  const int tid = threadIdx.x;
  const int r0 = blocks[blockIdx.x], r1 = blocks[blockIdx.x + 1];
  const int nrows = r1 - r0;
  const int p0 = rowptr[r0], p1 = rowptr[r1];
  const int cnt = p1 - p0;
  if (cnt > kTileNnz) {
    // one long row: strided partial sums, then a fixed-order tree
    double s = 0.0;
    for (int p = p0 + tid; p < p1; p += kSpmvThreads) s = __dadd_rn(s, __dmul_rn(__ldcs(vals + p), __ldg(x + __ldcs(colind + p))));
    s = warp_sum(s);
    if ((tid & 31) == 0) red[tid >> 5] = s;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int w = 0; w < kSpmvThreads / 32; ++w) t += red[w];
      y[r0] = t;
    }
    return;
  }
  for (int r = tid; r <= nrows; r += kSpmvThreads) rp[r] = rowptr[r0 + r] - p0;
  // stream the block's nonzeros: four independent (value, index, x) loads per thread in flight
  int p = tid;
  for (; p + 3 * kSpmvThreads < cnt; p += 4 * kSpmvThreads) {
    double a[4];
    int c[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a[u] = __ldcs(vals + p0 + p + u * kSpmvThreads);
      c[u] = __ldcs(colind + p0 + p + u * kSpmvThreads);
    }
    double xv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) xv[u] = __ldg(x + c[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u) prod[p + u * kSpmvThreads] = __dmul_rn(a[u], xv[u]);
  }
  for (; p < cnt; p += kSpmvThreads) prod[p] = __dmul_rn(__ldcs(vals + p0 + p), __ldg(x + __ldcs(colind + p0 + p)));
  __syncthreads();
  for (int r = tid; r < nrows; r += kSpmvThreads) {
    double s = 0.0;
    for (int q = rp[r]; q < rp[r + 1]; ++q) s = __dadd_rn(s, prod[q]);
    y[r0 + r] = s;
  }
}

// Warp tiles.  A tile {r0, r1, p0, p1} is <= 32 rows and <= kWarpTileNnz nonzeros; lane i of the owning
// warp streams nonzeros i, i+32, ... (kWarpTileNnz/32 value, index and x loads in flight per
// lane), keeps the rounded products in warp-private shared memory, and after a __syncwarp sums
// row i of the tile in index order (the order of a sequential CSR loop).  Full occupancy (2048
// threads per SM): the short loads of many warps hide the gather latency.
// VT is the stored value type (double, or float for FP32 storage); products and sums are FP64.
template <typename VT, typename XT>
__global__ void __launch_bounds__(kSpmvThreads) spmv_warptile_kernel(int ntiles, const int4 *__restrict__ tiles,
                                                                     const int *__restrict__ rowptr,
                                                                     const int *__restrict__ colind,
                                                                     const VT *__restrict__ vals,
                                                                     const XT *__restrict__ x,
                                                                     double *__restrict__ y,
                                                                     const GsState *__restrict__ st, int step) {
  if (st && st->halt && st->halt_step < step) return;
  __shared__ double prod_all[kSpmvThreads / 32][kWarpTileNnz];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double *prod = prod_all[wib];
  const int nwarps = gridDim.x * (kSpmvThreads / 32);
  for (int t = blockIdx.x * (kSpmvThreads / 32) + wib; t < ntiles; t += nwarps) {
    const int4 tile = tiles[t];
    const int r0 = tile.x, r1 = tile.y, p0 = tile.z, p1 = tile.w;
    const int nrows = r1 - r0;  // 1..32
    const int cnt = p1 - p0;
    // the nonzero range comes with the tile, so the value and index loads below do not wait
    // for the row pointer; the row boundaries are needed only for the sums
    const int myrow_start = (lane < nrows) ? __ldg(rowptr + r0 + lane) : 0;
    const int next = __shfl_down_sync(0xffffffffu, myrow_start, 1);
    const int myrow_end = (lane + 1 < nrows) ? next : p1;
    VT a[kWarpTileNnz / 32];  // kept in the stored type until the multiply (fewer registers for FP32)
    int c[kWarpTileNnz / 32];
#pragma unroll
    for (int u = 0; u < kWarpTileNnz / 32; ++u) {
      const int q = lane + 32 * u;
      a[u] = (q < cnt) ? __ldcs(vals + p0 + q) : VT(0);
      c[u] = (q < cnt) ? __ldcs(colind + p0 + q) : 0;
    }
#pragma unroll
    for (int u = 0; u < kWarpTileNnz / 32; ++u) {
      const int q = lane + 32 * u;
      if (q < cnt) prod[q] = __dmul_rn((double)a[u], (double)__ldg(x + c[u]));
    }
    __syncwarp();
    if (lane < nrows) {
      double sacc = 0.0;
      for (int q = myrow_start - p0; q < myrow_end - p0; ++q) sacc = __dadd_rn(sacc, prod[q]);
      y[r0 + lane] = sacc;
    }
    __syncwarp();
  }
}

// The same warp tiles with a two-tile software pipeline: while a warp gathers x for tile t it
// already has the values and column indices of its next tile in flight (half occupancy, twice
// the loads in flight per warp).  Same sums in the same order as spmv_warptile_kernel.
template <typename VT, typename XT>
__global__ void __launch_bounds__(kSpmvThreads, sizeof(VT) == 4 ? 4 : 3)
    spmv_warptile_pipelined_kernel(int ntiles, const int4 *__restrict__ tiles, const int *__restrict__ rowptr,
                                   const int *__restrict__ colind, const VT *__restrict__ vals,
                                   const XT *__restrict__ x, double *__restrict__ y,
                                   const GsState *__restrict__ st, int step) {
  if (st && st->halt && st->halt_step < step) return;
  __shared__ double prod_all[kSpmvThreads / 32][kWarpTileNnz];
  constexpr int U = kWarpTileNnz / 32;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double *prod = prod_all[wib];
  const int nwarps = gridDim.x * (kSpmvThreads / 32);
  int t = blockIdx.x * (kSpmvThreads / 32) + wib;
  if (t >= ntiles) return;
  int4 tile = tiles[t];
  VT a[U];
  int c[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int q = lane + 32 * u;
    a[u] = (q < tile.w - tile.z) ? __ldcs(vals + tile.z + q) : VT(0);
    c[u] = (q < tile.w - tile.z) ? __ldcs(colind + tile.z + q) : 0;
  }
  while (true) {
    const int tn = t + nwarps;
    int4 ntile = make_int4(0, 0, 0, 0);
    VT an[U];
    int cn[U];
    if (tn < ntiles) {
      ntile = tiles[tn];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int q = lane + 32 * u;
        an[u] = (q < ntile.w - ntile.z) ? __ldcs(vals + ntile.z + q) : VT(0);
        cn[u] = (q < ntile.w - ntile.z) ? __ldcs(colind + ntile.z + q) : 0;
      }
    }
    const int r0 = tile.x, nrows = tile.y - tile.x, p0 = tile.z, p1 = tile.w, cnt = p1 - p0;
    const int myrow_start = (lane < nrows) ? __ldg(rowptr + r0 + lane) : 0;
    const int nextb = __shfl_down_sync(0xffffffffu, myrow_start, 1);
    const int myrow_end = (lane + 1 < nrows) ? nextb : p1;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int q = lane + 32 * u;
      if (q < cnt) prod[q] = __dmul_rn((double)a[u], (double)__ldg(x + c[u]));
    }
    __syncwarp();
    if (lane < nrows) {
      double sacc = 0.0;
      for (int q = myrow_start - p0; q < myrow_end - p0; ++q) sacc = __dadd_rn(sacc, prod[q]);
      y[r0 + lane] = sacc;
    }
    __syncwarp();
    if (tn >= ntiles) break;
    t = tn;
    tile = ntile;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      a[u] = an[u];
      c[u] = cn[u];
    }
  }
}

// Sliced ELL (32-row slices): slice s stores its rows column-major in kSellWidth-padded chunks,
// entry (row 32s+i, k) at off[s] + 32k + i, column -1 for padding; lane i of the owning warp sums
// row 32s+i in index order (the same bits as a sequential CSR loop) with loads of 32 consecutive
// entries per instruction.  Rows with more than kSellMaxRow nonzeros are not in the slices
// (their mask bit is 0) and are computed by the tile or segment kernels.
template <typename VT, typename XT>
__global__ void __launch_bounds__(kSpmvThreads) spmv_sell_kernel(int nslices, int n, const long long *__restrict__ off,
                                                                 const int *__restrict__ width,
                                                                 const unsigned *__restrict__ mask,
                                                                 const VT *__restrict__ sval,
                                                                 const int *__restrict__ scol,
                                                                 const XT *__restrict__ x, double *__restrict__ y,
                                                                 const GsState *__restrict__ st, int step) {
  // Launched as a programmatic dependent of the previous kernel (the Gram-Schmidt pass that wrote
  // x): wait for that grid and its writes, then let the next kernel be launched.
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" :::);
  if (st && st->halt && st->halt_step < step) return;
  const int lane = threadIdx.x & 31;
  const int nwarps = gridDim.x * (kSpmvThreads / 32);
  for (int sl = blockIdx.x * (kSpmvThreads / 32) + (threadIdx.x >> 5); sl < nslices; sl += nwarps) {
    const long long base = off[sl] + lane;
    const int w = width[sl];
    double sacc = 0.0;
    for (int k0 = 0; k0 < w; k0 += 8) {
      VT a[8];
      int c[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const bool in = k0 + u < w;
        c[u] = in ? __ldcs(scol + base + 32ll * (k0 + u)) : -1;
        a[u] = in ? __ldcs(sval + base + 32ll * (k0 + u)) : VT(0);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (c[u] >= 0) sacc = __dadd_rn(sacc, __dmul_rn((double)a[u], (double)__ldg(x + c[u])));
    }
    const int r = 32 * sl + lane;
    if (r < n && ((mask[sl] >> lane) & 1u)) y[r] = sacc;
  }
}

// Segments of rows longer than a warp tile: segs[s] = {p_begin, p_end} (at most kSegmentNnz
// nonzeros).  A warp streams its segment in chunks of kWarpTileNnz nonzeros with 8 independent
// value/index loads and then 8 x gathers in flight per lane, adds each lane's products in a
// fixed order, reduces the warp with a fixed shuffle tree and writes partials[s].  Half
// occupancy buys the registers for the loads in flight; long dense-like rows (the power-law
// columns of a transposed matrix) stream at full width.
template <typename VT, typename XT>
__global__ void __launch_bounds__(kSpmvThreads, sizeof(VT) == 4 ? 4 : 3) spmv_segment_kernel(int nsegs, const int2 *__restrict__ segs,
                                                                       const int *__restrict__ colind,
                                                                       const VT *__restrict__ vals,
                                                                       const XT *__restrict__ x,
                                                                       double *__restrict__ partials,
                                                                       const GsState *__restrict__ st, int step) {
  if (st && st->halt && st->halt_step < step) return;
  const int lane = threadIdx.x & 31;
  const int nwarps = gridDim.x * (kSpmvThreads / 32);
  for (int sg = blockIdx.x * (kSpmvThreads / 32) + (threadIdx.x >> 5); sg < nsegs; sg += nwarps) {
    const int2 seg = segs[sg];
    constexpr int U = kWarpTileNnz / 32;
    double sacc = 0.0;
    const int nfull = (seg.y - seg.x) / kWarpTileNnz;
    VT a[U];
    int c[U];
    if (nfull > 0) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        a[u] = __ldcs(vals + seg.x + lane + 32 * u);
        c[u] = __ldcs(colind + seg.x + lane + 32 * u);
      }
    }
    // software pipeline: the values and indices of chunk k+1 are in flight while chunk k gathers x
    for (int k = 0; k < nfull; ++k) {
      double xv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) xv[u] = (double)__ldg(x + c[u]);
      VT an[U];
      int cn[U];
      if (k + 1 < nfull) {
        const int pn = seg.x + (k + 1) * kWarpTileNnz + lane;
#pragma unroll
        for (int u = 0; u < U; ++u) {
          an[u] = __ldcs(vals + pn + 32 * u);
          cn[u] = __ldcs(colind + pn + 32 * u);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) sacc = __dadd_rn(sacc, __dmul_rn((double)a[u], xv[u]));
#pragma unroll
      for (int u = 0; u < U; ++u) {
        a[u] = an[u];
        c[u] = cn[u];
      }
    }
    const int p = seg.x + nfull * kWarpTileNnz;
    for (int q = p + lane; q < seg.y; q += 32)
      sacc = __dadd_rn(sacc, __dmul_rn((double)__ldcs(vals + q), (double)__ldg(x + __ldcs(colind + q))));
    sacc = warp_sum(sacc);
    if (lane == 0) partials[sg] = sacc;
  }
}

// y[row] of every long row from its segment partials: one warp per row, lane l adds partials
// l, l+32, ... in order, then a fixed shuffle tree.  longrows[i] = {row, first slot, slot count}.
__global__ void __launch_bounds__(256) spmv_fixup_kernel(int nlong, const int3 *__restrict__ longrows,
                                                         const double *__restrict__ partials,
                                                         double *__restrict__ y, const GsState *__restrict__ st,
                                                         int step) {
  if (st && st->halt && st->halt_step < step) return;
  const int lane = threadIdx.x & 31;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= nlong) return;
  const int3 lr = longrows[i];
  double sacc = 0.0;
  for (int k = lane; k < lr.z; k += 32) sacc += partials[lr.y + k];
  sacc = warp_sum(sacc);
  if (lane == 0) y[lr.x] = sacc;
}

template <int LPR>
__global__ void __launch_bounds__(256) spmv_csr_kernel(int n, const int *__restrict__ rowptr,
                                                       const int *__restrict__ colind,
                                                       const double *__restrict__ vals,
                                                       const double *__restrict__ x, double *__restrict__ y) {
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

}  // namespace

int spmv_choose_lanes(int n, int64_t nnz) {
  if (n <= 0) return 1;
  const double avg = (double)nnz / (double)n;
  int lanes = 1;
  while (lanes < 32 && lanes < avg) lanes <<= 1;
  return lanes;
}

std::vector<int> spmv_row_blocks(int n, const int *rowptr) {
  std::vector<int> b;
  b.reserve(n / 64 + 2);
  int r = 0;
  b.push_back(0);
  while (r < n) {
    const int start = r;
    const int base = rowptr[start];
    while (r < n && r - start < kTileRows && rowptr[r + 1] - base <= kTileNnz) ++r;
    if (r == start) ++r;  // a single row longer than the tile: a block of its own
    b.push_back(r);
  }
  return b;
}

SellPlan spmv_sell_plan(int n, const int *rowptr) {
  SellPlan sp;
  const int nslices = (n + 31) / 32;
  sp.off.resize(nslices);
  sp.width.resize(nslices);
  sp.mask.resize(nslices);
  long long total = 0;
  for (int sl = 0; sl < nslices; ++sl) {
    int w = 0;
    unsigned m = 0;
    for (int i = 0; i < 32 && 32 * sl + i < n; ++i) {
      const int r = 32 * sl + i, len = rowptr[r + 1] - rowptr[r];
      if (len <= kSellMaxRow) {
        m |= 1u << i;
        if (len > w) w = len;
      } else {
        sp.rest_rows.push_back(r);
      }
    }
    sp.off[sl] = total;
    sp.width[sl] = w;
    sp.mask[sl] = m;
    total += 32ll * w;
  }
  sp.entries = total;
  // warp tiles and segments for the rows left out of the slices
  for (int r = 0; r < n;) {
    if (rowptr[r + 1] - rowptr[r] <= kSellMaxRow) {
      ++r;
      continue;
    }
    const int start = r;
    const int base = rowptr[start];
    while (r < n && r - start < 32 && rowptr[r + 1] - rowptr[r] > kSellMaxRow && rowptr[r + 1] - base <= kWarpTileNnz)
      ++r;
    if (r > start) {
      sp.rest.tiles.push_back({start, r, rowptr[start], rowptr[r]});
      continue;
    }
    const int p0 = rowptr[r], p1 = rowptr[r + 1];
    const int first = (int)sp.rest.segs.size();
    for (int p = p0; p < p1; p += kSegmentNnz)
      sp.rest.segs.push_back({p, (p1 - p > kSegmentNnz) ? p + kSegmentNnz : p1});
    sp.rest.longrows.push_back({r, first, (int)sp.rest.segs.size() - first});
    ++r;
  }
  return sp;
}

WarpTiles spmv_warp_tiles(int n, const int *rowptr) {
  WarpTiles wt;
  wt.tiles.reserve(n / 16 + 2);
  int r = 0;
  while (r < n) {
    const int start = r;
    const int base = rowptr[start];
    while (r < n && r - start < 32 && rowptr[r + 1] - base <= kWarpTileNnz) ++r;
    if (r > start) {
      wt.tiles.push_back({start, r, rowptr[start], rowptr[r]});
      continue;
    }
    // a single row longer than a tile: segments of kSegmentNnz nonzeros
    const int p0 = rowptr[r], p1 = rowptr[r + 1];
    const int first = (int)wt.segs.size();
    for (int p = p0; p < p1; p += kSegmentNnz) wt.segs.push_back({p, (p1 - p > kSegmentNnz) ? p + kSegmentNnz : p1});
    wt.longrows.push_back({r, first, (int)wt.segs.size() - first});
    ++r;
  }
  return wt;
}

template <typename VT, typename XT>
cudaError_t spmv_warptile_launch_t(const SpmvTiles &T, const int *rowptr, const int *colind, const VT *vals,
                                   const XT *x, double *y, cudaStream_t stream, const GsState *st, int step,
                                   bool pipelined) {
  static int sms = 0, tile_per_sm = 0, seg_per_sm = 0, pipe_per_sm = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tile_per_sm, spmv_warptile_kernel<VT, XT>, kSpmvThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&seg_per_sm, spmv_segment_kernel<VT, XT>, kSpmvThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pipe_per_sm, spmv_warptile_pipelined_kernel<VT, XT>, kSpmvThreads, 0);
    if (tile_per_sm <= 0) tile_per_sm = 1;
    if (seg_per_sm <= 0) seg_per_sm = 1;
    if (pipe_per_sm <= 0) pipe_per_sm = 1;
  }
  const int warps_per_cta = kSpmvThreads / 32;
  // persistent grids: every CTA resident at once
  if (T.nsegs > 0) {
    int grid = (T.nsegs + warps_per_cta - 1) / warps_per_cta;
    if (grid > sms * seg_per_sm) grid = sms * seg_per_sm;
    spmv_segment_kernel<VT, XT><<<grid, kSpmvThreads, 0, stream>>>(T.nsegs, T.segs, colind, vals, x, T.partials, st,
                                                               step);
    count_launch();
  }
  if (T.ntiles > 0) {
    int grid = (T.ntiles + warps_per_cta - 1) / warps_per_cta;
    if (pipelined) {
      if (grid > sms * pipe_per_sm) grid = sms * pipe_per_sm;
      spmv_warptile_pipelined_kernel<VT, XT><<<grid, kSpmvThreads, 0, stream>>>(T.ntiles, T.tiles, rowptr, colind, vals,
                                                                            x, y, st, step);
    } else {
      if (grid > sms * tile_per_sm) grid = sms * tile_per_sm;
      spmv_warptile_kernel<VT, XT><<<grid, kSpmvThreads, 0, stream>>>(T.ntiles, T.tiles, rowptr, colind, vals, x, y,
                                                                  st, step);
    }
    count_launch();
  }
  if (T.nlong > 0) {
    spmv_fixup_kernel<<<(T.nlong * 32 + 255) / 256, 256, 0, stream>>>(T.nlong, T.longrows, T.partials, y, st, step);
    count_launch();
  }
  return cudaGetLastError();
}

// one thread per row: entries k < width of row 32s+i at off[s] + 32k + i, padding (-1, 0) past the
// row's end and for rows outside the slices
template <typename VT>
__global__ void sell_gather_kernel(int n, int nslices, const long long *__restrict__ off, const int *__restrict__ width,
                                   const unsigned *__restrict__ mask, const int *__restrict__ rowptr,
                                   const int *__restrict__ colind, const VT *__restrict__ vals, int *__restrict__ scol,
                                   VT *__restrict__ sval) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < 32ll * nslices;
       t += (long long)gridDim.x * blockDim.x) {
    const int sl = (int)(t >> 5), i = (int)(t & 31), r = 32 * sl + i;
    const bool in = r < n && ((mask[sl] >> i) & 1u);
    const int p0 = in ? rowptr[r] : 0, len = in ? rowptr[r + 1] - p0 : 0;
    const long long base = off[sl] + i;
    for (int k = 0; k < width[sl]; ++k) {
      scol[base + 32ll * k] = k < len ? colind[p0 + k] : -1;
      sval[base + 32ll * k] = k < len ? vals[p0 + k] : VT(0);
    }
  }
}

cudaError_t sell_gather(int n, const SpmvSell &S, const int *rowptr, const int *colind, const void *vals, bool f32,
                        cudaStream_t stream) {
  if (S.nslices <= 0) return cudaSuccess;
  long long g = (32ll * S.nslices + 255) / 256;
  if (g > 148 * 32) g = 148 * 32;
  if (f32)
    sell_gather_kernel<float><<<(unsigned)g, 256, 0, stream>>>(n, S.nslices, S.off, S.width, S.mask, rowptr, colind,
                                                               static_cast<const float *>(vals), S.cols,
                                                               static_cast<float *>(S.vals));
  else
    sell_gather_kernel<double><<<(unsigned)g, 256, 0, stream>>>(n, S.nslices, S.off, S.width, S.mask, rowptr, colind,
                                                                static_cast<const double *>(vals), S.cols,
                                                                static_cast<double *>(S.vals));
  count_launch();
  return cudaGetLastError();
}

template <typename VT, typename XT>
cudaError_t spmv_sell_launch_t(const SpmvSell &S, const VT *svals, int n, const SpmvTiles &rest, const int *rowptr,
                               const int *colind, const VT *vals, const XT *x, double *y, cudaStream_t stream,
                               const GsState *st, int step) {
  static int sms = 0, per_sm = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spmv_sell_kernel<VT, XT>, kSpmvThreads, 0);
    if (per_sm <= 0) per_sm = 1;
  }
  if (S.nslices > 0) {
    int grid = (S.nslices + kSpmvThreads / 32 - 1) / (kSpmvThreads / 32);
    if (grid > sms * per_sm) grid = sms * per_sm;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kSpmvThreads);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, spmv_sell_kernel<VT, XT>, S.nslices, n, (const long long *)S.off,
                                       (const int *)S.width, (const unsigned *)S.mask, svals, (const int *)S.cols, x,
                                       y, st, step);
    if (e != cudaSuccess) return e;
    count_launch();
  }
  if (rest.ntiles > 0 || rest.nsegs > 0) {
    cudaError_t e = spmv_warptile_launch_t<VT, XT>(rest, rowptr, colind, vals, x, y, stream, st, step, false);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

cudaError_t spmv_sell_launch(const SpmvSell &S, int n, const SpmvTiles &rest, const int *rowptr, const int *colind,
                             const double *vals, const double *x, double *y, cudaStream_t stream, const GsState *st,
                             int step) {
  return spmv_sell_launch_t<double, double>(S, static_cast<const double *>(S.vals), n, rest, rowptr, colind, vals, x,
                                            y, stream, st, step);
}

cudaError_t spmv_sell_launch_f32(const SpmvSell &S, int n, const SpmvTiles &rest, const int *rowptr,
                                 const int *colind, const float *vals, const double *x, double *y,
                                 cudaStream_t stream, const GsState *st, int step) {
  return spmv_sell_launch_t<float, double>(S, static_cast<const float *>(S.vals), n, rest, rowptr, colind, vals, x, y,
                                           stream, st, step);
}

cudaError_t spmv_sell_launch_x32(const SpmvSell &S, const float *svals, int n, const SpmvTiles &rest,
                                 const int *rowptr, const int *colind, const float *vals, const float *x, double *y,
                                 cudaStream_t stream, const GsState *st, int step) {
  return spmv_sell_launch_t<float, float>(S, svals, n, rest, rowptr, colind, vals, x, y, stream, st, step);
}

cudaError_t spmv_warptile_launch(const SpmvTiles &T, const int *rowptr, const int *colind, const double *vals,
                                 const double *x, double *y, cudaStream_t stream, const GsState *st, int step,
                                 bool pipelined) {
  return spmv_warptile_launch_t<double, double>(T, rowptr, colind, vals, x, y, stream, st, step, pipelined);
}

cudaError_t spmv_warptile_launch_f32(const SpmvTiles &T, const int *rowptr, const int *colind, const float *vals,
                                     const double *x, double *y, cudaStream_t stream, const GsState *st, int step,
                                     bool pipelined) {
  return spmv_warptile_launch_t<float, double>(T, rowptr, colind, vals, x, y, stream, st, step, pipelined);
}

cudaError_t spmv_rowblock_launch(int nblocks, const int *blocks, const int *rowptr, const int *colind,
                                 const double *vals, const double *x, double *y, cudaStream_t stream,
                                 const GsState *st, int step) {
  if (nblocks <= 0) return cudaSuccess;
  spmv_rowblock_kernel<<<nblocks, kSpmvThreads, 0, stream>>>(blocks, rowptr, colind, vals, x, y, st, step);
  count_launch();
  return cudaGetLastError();
}

cudaError_t spmv_launch(int n, const int *rowptr, const int *colind, const double *vals, const double *x, double *y,
                        int lanes, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  const int threads = 256;
  const long long rows_per_block = threads / lanes;
  long long blocks = (n + rows_per_block - 1) / rows_per_block;
  if (blocks > (1ll << 20)) blocks = 1ll << 20;
  switch (lanes) {
#define B200_SPMV_CASE(L)                                                                         \
  case L:                                                                                         \
    spmv_csr_kernel<L><<<(unsigned)blocks, threads, 0, stream>>>(n, rowptr, colind, vals, x, y); \
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
