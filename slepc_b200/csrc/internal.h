// Entry points shared between the object layer (lib.cu) and the SVD solver (svd.cu).
#pragma once
#include <cuda_runtime.h>

#include "slepc_b200.h"
#include "kernels.h"

namespace b200 {
// The cross shell of A: A^T A, or A A^T when swapped (the m < n case, which
// SVDSetUp handles by exchanging A and A^T, src/svd/interface/svdsetup.c:300-314).
b200_status mat_create_cross_ex(b200_mat A, bool swapped, b200_mat *C);
// y = A x, or y = A^T x (transpose; matrices from b200_mat_create_aij), on the given stream.
cudaError_t mat_apply(b200_mat A, const double *x, double *y, cudaStream_t stream, bool transpose);
// BVOrthogonalizeColumn / BVOrthonormalizeColumn (normalize = 1) of column j against columns 0..j-1.
b200_status bv_orth_column(b200_bv bv, int j, int normalize, double *H, double *norm, int *lindep);
// EPSSetUp's BVInsertVecs of the initial space into columns 0..k-1 (sets eps->nini_eff).
b200_status eps_insert_initial_space(b200_eps eps, b200_bv V, int max_cols);
// BVOrthogonalize (no R) with one host synchronisation for the whole block.
b200_status bv_orthogonalize_block(b200_bv bv);
// BVOrthogonalizeVec + scale by 1/norm for several device vectors, one synchronisation.
b200_status bv_orthonormalize_vecs(b200_bv bv, double *const *vecs, int count, int *breakdown);
// BVDot(W, Z, MA) and BVDot(Z, Z, MB) over the same active column count, one pass over both blocks
// (FP64 MMAs) and one synchronisation: the Gram pair of a Rayleigh-Ritz step.
b200_status bv_dot_pair(b200_bv W, b200_bv Z, double *MA, double *MB, int ldm);
// BVOrthogonalize of two independent blocks (no R) with the Cholesky or SVQB block types: both
// Gram products read back in one synchronisation (otherwise one block after the other).
b200_status bv_orthogonalize_pair(b200_bv a, b200_bv b);
// Column norms of the active columns, one synchronisation.
b200_status bv_column_norms(b200_bv bv, double *nrm);
// Stream-ordered device allocation from the library's per-device pool (freed memory is kept for
// reuse by the process) and its release on the same stream.
cudaError_t pool_alloc(void **p, size_t bytes, cudaStream_t s);
cudaError_t pool_free(void *p, cudaStream_t s);
// Buffers of the Mat, BV and EPS objects, from the same pool through a library stream: the
// allocation has completed when dev_malloc returns and dev_free first waits for the device, so
// both keep cudaMalloc/cudaFree's synchronous meaning for buffers used on any stream, while a
// create/destroy per call (the one-call host solve) reuses memory instead of mapping and unmapping
// it each time.
cudaError_t dev_malloc(void **p, size_t bytes);
void dev_free(void *p);
template <typename T>
inline cudaError_t dev_malloc(T **p, size_t bytes) {
  return dev_malloc(reinterpret_cast<void **>(p), bytes);
}
// Streaming multiprocessors of the current device.
int num_sms_host();
// EPSSolve with EPSLOBPCG (lobpcg.cu).
b200_status lobpcg_solve(b200_eps eps);
// BVMatMult: Y(:, Y.l+j) = A V(:, V.l+j) over the active columns (block SpMV for square CSR).
b200_status bv_mat_mult(b200_bv V, b200_mat A, b200_bv Y);
// EPSMonitor (epsmon.c:39): run the monitors of eps; B200_ERR_STATE when one returns nonzero.
b200_status eps_monitor(b200_eps eps, int its, int nconv, const double *eigr, const double *errest, int nest);
// Start the monitor clock of a solve.
void eps_monitor_start(b200_eps eps);
// Krylov-Schur with b200_eps_set_precision(MIXED) after the setup (mixed.cu).
b200_status mixed_solve(b200_eps eps);
// Read the Gram-Schmidt control block after a stream synchronisation (maps device errors).
b200_status bv_state(b200_bv bv, GsState *out);
// Sliced-ELL copy and FP32 value copies of a square CSR operator for the mixed solver.
b200_status mat_mixed_prepare(b200_mat A, cudaStream_t s);
// y = A x with FP32 values and FP32 x (products and sums FP64); gated on st/step like the SpMV.
cudaError_t mat_spmv_x32(b200_mat A, const float *x, double *y, cudaStream_t stream, const GsState *st, int step);
// Out(:,b) = alpha (A Y(:,b) - shift Y(:,b)) - beta X(:,b), b < nb, with the operator's own values.
cudaError_t mat_spmm(b200_mat A, const double *Y, const double *X, double *Out, int ld, int nb, double alpha,
                     double shift, double beta, cudaStream_t stream);
// out[0..1] (device) = Gershgorin bounds of the spectrum of A.
cudaError_t mat_gershgorin(b200_mat A, double *out, double *work, int work_len, cudaStream_t stream);
}  // namespace b200
