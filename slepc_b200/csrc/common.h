// Shared definitions for the B200 Krylov-Schur library (host and device).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "slepc_b200.h"

namespace b200 {

// Largest number of basis columns a BV may hold (ncv+1 plus the internal
// work column).  Bounded by the per-CTA column accumulators of the
// Gram-Schmidt kernels (one per thread of a 256-thread block).
constexpr int kMaxCols = 255;

// Number of spin iterations after which a device-side wait gives up.
constexpr long long kSpinLimit = 1ll << 22;

// Device error flags (bitmask written by kernels, read by the host).
enum DeviceError : int {
  kDevErrNone = 0,
  kDevErrInnerProduct = 1,   // BV_SafeSqrt rejected a negative inner product
  kDevErrTimeout = 2,        // a bounded wait (mbarrier / ticket) gave up
  kDevErrNonFinite = 4,      // NaN or Inf met in a reduction
};

// Gram-Schmidt pass actions (bitmask), decided on the device.
enum GsAction : int {
  kActNone = 0,
  kActUpdate = 1,   // w <- w - V(:,0:j) coef
  kActDot = 2,      // partial dots V(:,0:j)^T w and w^T w
  kActScale = 4,    // w <- w * scale (normalisation)
};

// Stages of the DGKS state machine (what the pending dot result means).
enum GsStage : int {
  kStageDotOfPass = 0,     // c holds the dot of pass `pass`
  kStageExplicitNorm = 1,  // c holds V^T w' after pass `pass`; c[j] = ||w'||^2 gives the explicit norm
  kStageDone = 2,
};

// Per-BV device control block for one column orthogonalisation.  Written by
// the host before the first pass, then advanced on the device by the last
// CTA of every Gram-Schmidt pass.
struct GsState {
  int action;        // GsAction bits for the next pass kernel
  int stage;         // GsStage
  int pass;          // CGS passes applied so far (1..3)
  int j;             // column being orthogonalised (columns 0..j-1 are the basis)
  int normalize;     // 1: scale the result by 1/norm (BVOrthonormalizeColumn)
  int want_self;     // 1: include w^T w in the dot (column variant); 0: vector variant
  int lindep;        // linear dependence flag of the last finished column
  int halt;          // set when a Lanczos run broke down: later steps are skipped
  int halt_step;     // Lanczos step index at which the breakdown happened
  int err;           // DeviceError bits
  int lanczos_step;  // index j of the Lanczos step in flight (for T output)
  int t_base;        // offset of T output, -1 = none
  unsigned int ticket;  // CTA arrival counter of the running pass
  int pad0;
  double eta;        // DGKS threshold (0.7071)
  double deftol;     // 10*eps for BV_SafeSqrt
  double onrm, nrm;  // norms of the current pass
  double scale;      // multiplier applied by the kScale action
  double beta_out;   // norm returned to the caller (BVOrthonormalizeColumn's norm)
  unsigned long long bytes;  // algorithmic bytes moved by the passes since the reset
  int passes;        // pass kernels that did work since the reset
  int pad1;
};

}  // namespace b200

#define B200_CUDA_CHECK(expr)                                                         \
  do {                                                                                \
    cudaError_t _e = (expr);                                                          \
    if (_e != cudaSuccess) {                                                          \
      b200_set_last_error(__FILE__, __LINE__, cudaGetErrorString(_e));               \
      return B200_ERR_CUDA;                                                           \
    }                                                                                 \
  } while (0)

#define B200_CHECK(expr)                \
  do {                                  \
    b200_status _s = (expr);            \
    if (_s != B200_OK) return _s;       \
  } while (0)

#define B200_ARG_CHECK(cond, msg)                                 \
  do {                                                            \
    if (!(cond)) {                                                \
      b200_set_last_error(__FILE__, __LINE__, msg);               \
      return B200_ERR_ARG;                                        \
    }                                                             \
  } while (0)

extern "C" void b200_set_last_error(const char *file, int line, const char *msg);
