// Row-major blocks of vectors for the Chebyshev-filtered subspace form of the mixed-precision solver.
//
// A block of BP vectors of length n (BP = 64 or 128) is stored row-major: row r (the r-th entry of
// every vector) is BP consecutive values at X + r * BP.  A sparse row then gathers whole 256- or
// 512-byte rows of the block, and a 32-column strip of a tile of rows is one 128-byte-wide TMA box.
#pragma once

#include <cuda.h>

#include "common.h"
#include "kernels.h"

namespace b200 {

// Y = alpha * (A X - shift * X) - beta * Z on row-major blocks of width bp (Z nullable: no beta
// term).  A is the square CSR operand given by its sliced-ELL copy (slice values svals: float or
// double as vals_f32 says) and, for rows the slices leave out, its CSR arrays (values cvals of the
// same type).  TX = float (x32) or double.  Y must not overlap X or Z.
cudaError_t rb_spmm_launch(const SpmvSell &S, int n, const int *rowptr, const int *colind, const void *cvals,
                           const void *svals, bool vals_f32, bool x32, int bp, const void *X, const void *Z, void *Y,
                           double alpha, double shift, double beta, cudaStream_t stream);

// Tensor map of a row-major FP32 block (n rows of bp floats) for the tensor-core Gram kernel.
cudaError_t rb_make_tmap_f32(CUtensorMap *tm, const float *X, int n, int bp);
// Partial-sum slots the Gram kernels need: blocks * bp * bp values.
int rb_gram_ctas(int n, int bp);
// G (bp x bp, FP64, device, row-major) = X^T Y of FP32 row-major blocks on the tensor cores
// (tcgen05 kind::tf32, accumulation in TMEM in FP32, the per-CTA partials summed in FP64 in a fixed
// order).  tx and ty are tensor maps of X and Y (ty == tx for X^T X).  work: rb_gram_ctas * bp * bp
// floats.  err (device int) receives kDevErrTimeout if a bounded wait gave up.
cudaError_t rb_gram_tf32_launch(const CUtensorMap &tx, const CUtensorMap *ty, int n, int bp, double *G, float *work,
                                int *err, cudaStream_t stream);
// GH[0 : bp^2] = X^T X and GH[bp^2 : 2 bp^2] = X^T W (bp x bp each, FP64, row-major, device) of
// row-major blocks X and W (float or double as x32 says), every product and sum in FP64, per-CTA
// partials summed in a fixed order (deterministic).  work: rb_gram_ctas * 2 * bp * bp doubles.
cudaError_t rb_gram2_f64_launch(const void *X, const void *W, bool x32, int n, int bp, double *GH, double *work,
                                cudaStream_t stream);
// Y = X M: M is bp x bp FP64 row-major (device), X and Y row-major blocks (float or double), Y != X.
cudaError_t rb_rotate_launch(const void *X, void *Y, bool x32, int n, int bp, const double *M, cudaStream_t stream);
// out[c] = ||W(:,c) - theta[c] X(:,c)||_2 for c < bp (FP64 sums, fixed order); work: bp * 1024 doubles.
cudaError_t rb_resid_launch(const void *W, const void *X, bool x32, int n, int bp, const double *theta, double *out,
                            double *work, cudaStream_t stream);
// Y (double, row-major) = X (float, row-major), n * bp entries.
cudaError_t rb_widen_launch(const float *X, double *Y, long long count, cudaStream_t stream);
// V(:, c) = X(:, c) for c < ncols: row-major block (float or double) into a column-major FP64
// array with leading dimension ld.
cudaError_t rb_to_colmajor_launch(const void *X, bool x32, int n, int bp, int ncols, double *V, int ld,
                                  cudaStream_t stream);
// Start block: columns c < nsrc from the column-major FP64 array src (leading dimension lds), the
// others N(0,1) from a counter-based generator (seed, row, column); float or double.
cudaError_t rb_init_launch(void *X, bool x32, int n, int bp, const double *src, int lds, int nsrc, uint64_t seed,
                           cudaStream_t stream);

}  // namespace b200
