// Launch wrappers of the device kernels (internal to the library).
#pragma once

#include <vector>

#include "common.h"

namespace b200 {

// Allow a kernel the largest dynamic shared memory the device grants per
// block (the opt-in maximum less the kernel's static shared memory).
template <typename K>
cudaError_t allow_max_dynamic_smem(K kernel) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa;
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kernel);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
  return e;
}

// Largest dynamic shared memory a block may request on the current device.
inline size_t max_dynamic_smem() {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return (size_t)optin;
}

void count_launch();
uint64_t launch_count();

// ---- SpMV (spmv.cu)
constexpr int kTileNnz = 4096;   // nonzeros staged per CTA of the row-block SpMV
constexpr int kTileRows = 1024;  // rows per CTA of the row-block SpMV
int spmv_choose_lanes(int n, int64_t nnz);
constexpr int kWarpTileNnz = 256;   // nonzeros staged per warp tile of the warp-tile SpMV
constexpr int kSegmentNnz = 1024;   // nonzeros per segment of a row longer than a warp tile
// Row blocks for the row-block SpMV: block b covers rows [b[i], b[i+1]).
std::vector<int> spmv_row_blocks(int n, const int *rowptr_host);
// Warp tiles for the warp-tile SpMV: {r0, r1, p0, p1} (rows and their nonzeros) for up to 32
// short rows; a row longer than
// kWarpTileNnz becomes segments {p_begin, p_end} of at most kSegmentNnz nonzeros, and
// longrows = {row, first segment, segment count}.
struct WarpTiles {
  std::vector<int4> tiles;
  std::vector<int2> segs;
  std::vector<int3> longrows;
};
WarpTiles spmv_warp_tiles(int n, const int *rowptr_host);
// Device copies of a WarpTiles plan plus one partial-sum slot per segment.
struct SpmvTiles {
  int4 *tiles = nullptr;
  int ntiles = 0;
  int2 *segs = nullptr;
  int nsegs = 0;
  int3 *longrows = nullptr;
  int nlong = 0;
  double *partials = nullptr;
};
// Sliced ELL with 32-row slices for rows of at most kSellMaxRow nonzeros; the other rows go to
// warp tiles and segments (rest).
constexpr int kSellMaxRow = 32;
struct SellPlan {
  std::vector<long long> off;
  std::vector<int> width;
  std::vector<unsigned> mask;
  long long entries = 0;
  WarpTiles rest;
  std::vector<int> rest_rows;  // the rows left out of the slices, ascending
};
SellPlan spmv_sell_plan(int n, const int *rowptr_host);
struct SpmvSell {
  int nslices = 0;
  long long *off = nullptr;
  int *width = nullptr;
  unsigned *mask = nullptr;
  void *vals = nullptr;  // double or float, like the matrix
  int *cols = nullptr;
  SpmvTiles rest;
  long long entries = 0;     // slice entries (padding included)
  int *rest_rows = nullptr;  // rows left out of the slices (block SpMV: one warp per row)
  int nrest = 0;
  float *vals32 = nullptr;   // FP32 copy of vals for the mixed-precision solver (FP64 matrices only)
  int max_width = 0;         // widest slice (host copy; sizes the row-block SpMM's staging)
};
cudaError_t spmv_sell_launch(const SpmvSell &S, int n, const SpmvTiles &rest, const int *rowptr, const int *colind,
                             const double *vals, const double *x, double *y, cudaStream_t stream,
                             const GsState *st = nullptr, int step = 0);
cudaError_t spmv_sell_launch_f32(const SpmvSell &S, int n, const SpmvTiles &rest, const int *rowptr,
                                 const int *colind, const float *vals, const double *x, double *y,
                                 cudaStream_t stream, const GsState *st = nullptr, int step = 0);
// FP32 values and FP32 x (the FP32 basis of the mixed-precision solver); products and sums FP64.
// svals: the slices' FP32 values; vals: FP32 CSR values for the rows outside the slices.
cudaError_t spmv_sell_launch_x32(const SpmvSell &S, const float *svals, int n, const SpmvTiles &rest,
                                 const int *rowptr, const int *colind, const float *vals, const float *x, double *y,
                                 cudaStream_t stream, const GsState *st = nullptr, int step = 0);
// Block SpMV with a fused three-term update (block.cu), FP64:
//   Out(:,b) = alpha * (A Y(:,b) - shift * Y(:,b)) - beta * X(:,b),  b < nb
// (X may be null: no beta term).  Y, X and Out are column-major with leading dimension ld; Out
// must not overlap Y or X.  The slices are read once per block.
cudaError_t spmm_sell_launch(const SpmvSell &S, int n, const int *rowptr, const int *colind, const void *vals, bool f32,
                             const double *Y, const double *X, double *Out, int ld, int nb, double alpha, double shift,
                             double beta, cudaStream_t stream);
// The slices' columns and values from the CSR arrays in HBM (S.off/width/mask already on the device).
cudaError_t sell_gather(int n, const SpmvSell &S, const int *rowptr, const int *colind, const void *vals, bool f32,
                        cudaStream_t stream);
// pipelined: the two-tile software-pipelined variant of the tile kernel (same result bits).
cudaError_t spmv_warptile_launch(const SpmvTiles &T, const int *rowptr, const int *colind, const double *vals,
                                 const double *x, double *y, cudaStream_t stream, const GsState *st = nullptr,
                                 int step = 0, bool pipelined = false);
// Same with FP32 stored values (products and sums in FP64).
cudaError_t spmv_warptile_launch_f32(const SpmvTiles &T, const int *rowptr, const int *colind, const float *vals,
                                     const double *x, double *y, cudaStream_t stream, const GsState *st = nullptr,
                                     int step = 0, bool pipelined = false);
// st/step: when st is given, the launch is skipped on the device if a
// Lanczos run halted (breakdown) at an earlier step.
cudaError_t spmv_rowblock_launch(int nblocks, const int *blocks, const int *rowptr, const int *colind,
                                 const double *vals, const double *x, double *y, cudaStream_t stream,
                                 const GsState *st = nullptr, int step = 0);
cudaError_t spmv_launch(int n, const int *rowptr, const int *colind, const double *vals, const double *x, double *y,
                        int lanes, cudaStream_t stream);

// ---- Fused Gram-Schmidt passes (gs.cu)
// Device workspace of one BV for the Gram-Schmidt kernels.
struct GsWork {
  GsState *st;        // control block
  double *coef;       // [kMaxCols] coefficients applied by the next UPDATE
  double *cnew;       // [kMaxCols+1] result of the last reduced dot
  double *partials;   // [(kMaxCols+1) * max_ctas] per-CTA partial dots
  int max_ctas;
  int num_sms;
};

struct GsPassArgs {
  double *V;      // basis, column-major
  int ld, n;
  int jb;         // basis columns 0..jb-1
  int wcol;       // column holding the vector being orthogonalised
  double *hacc;   // accumulated coefficients (jb + 1 entries: coefficients then norm)
  double *T;      // optional Lanczos output: T[step] = alpha, T[ldt+step] = beta
  int ldt;
  int step;       // Lanczos step index (halt gating), or -1
  int normalize;  // scale by 1/norm at the end
  int column;     // 1: column variant (BV_SafeSqrt check on w^T w)
  int total_cols; // columns allocated from V (bounds of the tile loads)
  // FP32 basis (mixed-precision solver): when V32 is set the basis columns are read from V32
  // (leading dimension ld32) and the vector being orthogonalised is the FP64 vector wvec (n + 2
  // entries allocated); wvec may also be set with an FP64 basis.
  const float *V32;
  int ld32;
  double *wvec;
  // with V32: the first CGS pass (its dot and the update applying its coefficients) in FP32
  // arithmetic, and the FP64 DGKS correction pass always taken
  int fast32;
};

// Enqueue the full CGS + DGKS("if needed") orthogonalisation of one column:
// a first dot pass plus the follow-up passes the device decides on.
cudaError_t gs_orthogonalize_launch(const GsPassArgs &a, const GsWork &w, cudaStream_t stream);
// Initialise the control block (eta, deftol, clears halt/err) -- once per run.
cudaError_t gs_state_reset(const GsWork &w, double eta, cudaStream_t stream);
// out[0..2] = norm, lindep flag and error bits of the last orthogonalisation (no host sync).
cudaError_t gs_record_launch(const GsWork &w, double *out, cudaStream_t stream);
// Plain dots q = V(:,0:jb)^T w (no decision), result in w.cnew.
cudaError_t gs_dot_launch(const GsPassArgs &a, const GsWork &w, cudaStream_t stream);

// Explicit transpose of a device CSR matrix (transpose.cu): rowptr_t (cols+1), colind_t and
// vals_t (nnz) in HBM, each row of A^T in ascending row order of A.  Synchronises the stream.
cudaError_t csr_transpose_device(int rows, int cols, long long nnz, const int *rowptr, const int *colind,
                                 const void *vals, bool f32, int *rowptr_t, int *colind_t, void *vals_t,
                                 cudaStream_t s);

// ---- Dense tall-skinny operations (bvops.cu)
// Device error bits of the TMA-pipelined panel product since the last call (read, then cleared;
// synchronises the stream when such a product ran since then): kDevErrTimeout when a bounded wait
// gave up.
cudaError_t panel_gemm_error(int *err, cudaStream_t stream);
// V(:,s:e) = V(:,l:k) * Q(l:k,s:e), row-blocked, in place; Q points at element (l,s).
// Householder QR of an n x nc column-major block (tsqr.cu): geqr2 in place (R above the diagonal,
// reflectors below, tau), and org2r (the block overwritten with Q).  work: householder_qr_parts(n)
// * (nc + 1) + nc doubles; scale: nc doubles.
int householder_qr_parts(int n);
cudaError_t householder_qr_launch(double *X, long long ld, int n, int nc, double *tau, double *scale, double *work,
                                  cudaStream_t s);
cudaError_t householder_q_launch(double *X, long long ld, int n, int nc, const double *tau, double *work,
                                 cudaStream_t s);
cudaError_t multinplace_launch(double *V, int ld, int n, int l, int k, const double *Q, int ldq, int s, int e,
                               cudaStream_t stream);
// The same on an FP32 basis (products and sums FP64, results rounded to FP32).
cudaError_t multinplace_launch_f32(float *V, int ld, int n, int l, int k, const double *Q, int ldq, int s, int e,
                                   cudaStream_t stream);
// Y(:,0:ny) = X(:,0:nx) Q(0:nx,0:ny) with the row-panel kernel (ny <= 128, X and Y distinct).
cudaError_t panel_mult_launch(double *Y, int ldy, const double *X, int ldx, int n, int nx, int ny, const double *Q,
                              int ldq, cudaStream_t stream);
cudaError_t panel_mult_launch_f32(double *Y, int ldy, const float *X, int ldx, int n, int nx, int ny, const double *Q,
                                  int ldq, cudaStream_t stream);
// out[c] = ||AX(:,c) - theta[c] X(:,c)||_2 for c < k (theta and out on the device), deterministic.
cudaError_t colresid_launch(const double *AX, const double *X, int ld, int n, int k, const double *theta, double *out,
                            double *work, int work_len, cudaStream_t stream);
// dst = src rounded to FP32.
cudaError_t to_f32_launch(float *dst, const double *src, long long len, cudaStream_t stream);
// out[0], out[1] = the smallest left and largest right end of the Gershgorin discs (device).
cudaError_t gershgorin_launch(int n, const int *rowptr, const int *colind, const void *vals, bool f32, double *out,
                              double *work, int work_len, cudaStream_t stream);
// Y(:,0:ny) = alpha * X(:,0:nx) * Q(0:nx,0:ny) + beta * Y(:,0:ny)   (X != Y storage)
cudaError_t mult_launch(double *Y, int ldy, const double *X, int ldx, int n, int nx, int ny, const double *Q, int ldq,
                        double alpha, double beta, cudaStream_t stream);
// y = beta*y + alpha*X(:,0:k) q
cudaError_t multvec_launch(const double *X, int ldx, int n, int k, const double *q, double alpha, double beta, double *y,
                           cudaStream_t stream);
// Row blocks per SM of BVDot and the block orthogonalisations: 4 for blocks of up to 64 x 64 pairs
// (one CTA column of Gram tiles, so the rows must supply the parallelism), 1 above that (the tiles
// do, and the partial sums would take npairs * 4 * SMs doubles).
inline int dot_ctas_per_sm(int nx, int ny) { return (long long)nx * ny <= 64 * 64 ? 4 : 1; }
// M(0:ny,0:nx) = Y(:,0:ny)^T X(:,0:nx), M column-major ldm (device), deterministic for a given
// ctas_per_sm (row blocks per SM of the partial sums).
cudaError_t dot_launch(const double *X, int ldx, int nx, const double *Y, int ldy, int ny, int n, double *M, int ldm,
                       double *work, int work_len, cudaStream_t stream, int ctas_per_sm = 1);
// M (nc x 2nc, ld nc) = [Y^T X | Y^T Y] from one pass over X and Y on the FP64 MMA path (8 <= nc <= 64
// columns each; FP64 products and sums, in the MMA's order); cudaErrorNotSupported outside that range.
cudaError_t dot_dual_launch(const double *X, int ldx, const double *Y, int ldy, int nc, int n, double *M, double *work,
                            int work_len, cudaStream_t stream, int ctas_per_sm);
// R(:, j) = AX(:, j) - theta[j] X(:, j) for j < ncols <= kThetaMax (theta on the host).
constexpr int kThetaMax = 128;
struct ThetaArg {
  double v[kThetaMax];
};
cudaError_t resid_block_launch(double *R, int ldr, const double *AX, int ldax, const double *X, int ldx, int n,
                               int ncols, const double *theta, cudaStream_t stream);
cudaError_t scale_launch(double *x, long long len, double alpha, cudaStream_t stream);
cudaError_t copy_launch(double *dst, const double *src, long long len, cudaStream_t stream);
// out[c] = ||X(:,c)||_2 for c < k (device), deterministic (fixed row split, fixed order).
cudaError_t colnorm_launch(const double *X, int ldx, int n, int k, double *out, double *work, int work_len,
                           cudaStream_t stream);
// Sum of squares of x (len) into out[0] (device), deterministic two-level reduction.
cudaError_t sumsq_launch(const double *x, long long len, double *out, double *work, int work_len, cudaStream_t stream);
// out[0] = ||y - alpha x||^2, deterministic two-level reduction.
cudaError_t diff_sumsq_launch(const double *y, const double *x, double alpha, long long len, double *out, double *work,
                              int work_len, cudaStream_t stream);
// out[0] = ||A x - lambda x||^2 (fused SpMV + residual), deterministic.
cudaError_t residual_launch(int n, const int *rowptr, const int *colind, const double *vals, const double *x,
                            double lambda, double *out, double *work, int work_len, int lanes, cudaStream_t stream);
// y -= alpha x, with the product and the difference rounded separately (VecAXPY(y,-alpha,x)).
cudaError_t axmy_launch(double *y, const double *x, double alpha, long long len, cudaStream_t stream);
// V(i,c) = d(i) V(i,c) for columns 0..ncols-1 (Jacobi preconditioner application).
cudaError_t diag_scale_launch(double *V, int ld, int n, int ncols, const double *d, cudaStream_t stream);
// dinv(i) = 1 / a_ii of a square FP64 CSR matrix (1 where the diagonal is zero).
cudaError_t inverse_diagonal_launch(int n, const int *rowptr, const int *colind, const double *vals, double *dinv,
                                    cudaStream_t stream);
// Counter-based uniform [0,1) column (stands in for PETSc's VecSetRandom).
cudaError_t random_launch(double *x, int n, uint64_t seed, uint64_t stream_id, cudaStream_t stream);

// ---- Strided batched FP32 GEMM on the tensor cores (tcgemm.cu)
// C[z] = alpha A[z] B[z] + beta C[z] for z < batch (A m x k, B k x n; element (i, j) of a view at
// p + z * bs + i * rs + j * cs), three-product TF32 (FP32-level accuracy).  With a workspace of
// ws_floats floats the depth may be split across CTAs and summed in a fixed order; sum_batch (needs
// ws) writes the single sum over z into C.  err collects kDevErrTimeout from bounded waits.
cudaError_t tc_sgemm(cudaStream_t s, int batch, int m, int n, int k, float alpha, const float *A, long long ars,
                     long long acs, long long abs_, const float *B, long long brs, long long bcs, long long bbs,
                     float beta, float *C, long long rsc, long long csc, long long bsc, int *err, float *ws,
                     size_t ws_floats, bool sum_batch);

}  // namespace b200
