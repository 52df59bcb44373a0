// Fused classical Gram-Schmidt with DGKS refinement for sm_100a.
//
// Replaces the BV Gram-Schmidt path of SLEPc:
//   BVOrthogonalizeGS (src/sys/classes/bv/interface/bvorthog.c:145-217)
//   BVOrthogonalizeCGS1 (bvorthog.c:91-132) with BVDotColumnInc (:32-47),
//   BVMultColumn (bvops.c:165), BV_SquareRoot / BV_SquareSum / BV_AddCoefficients
//   (include/slepc/private/bvimpl.h:121-141, 289-415)
// whose GPU form (bvcuda.cu:204-264, 45-60, 420-548) issues a cuBLAS gemv per
// half-pass plus 2-4 synchronous device-to-host scalar copies per pass.
//
// Here one kernel, gs_pass_kernel, performs any combination of
//   UPDATE  w <- w - V(:,0:jb) coef      (the second half of CGS pass p)
//   SCALE   w <- w * scale               (BVOrthonormalizeColumn's 1/norm)
//   DOT     c <- [V(:,0:jb) w', w'^T w'] (the first half of CGS pass p+1)
// in one streaming read of V: each CTA of a persistent grid (one per SM)
// pulls row chunks of all jb columns plus w into shared memory with
// cp.async.bulk copies completing on an mbarrier (two stages, so the next
// chunk is in flight while the current one is computed), applies the update
// row-wise and the dot column-wise from shared memory, and accumulates
// per-CTA column sums.  The last CTA to finish (atomic ticket) reduces the
// per-CTA sums in a fixed order (deterministic result), then runs the DGKS
// decision of BVOrthogonalizeGS on the device and writes the action of the
// next pass.  The host enqueues a fixed sequence of passes without waiting;
// passes the device decides against return immediately.
//
// A CGS pass of the reference reads V twice (dot, then update); fusing the
// update of pass p with the dot of pass p+1 reads V three times per column
// with one DGKS refinement instead of four, and no host round trip.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.h"
#include "kernels.h"

namespace b200 {
namespace {

constexpr int kConsumerWarps = 8;                     // warps that compute
constexpr int kConsumers = kConsumerWarps * 32;        // 256 consumer threads
constexpr int kThreads = kConsumers + 32;              // + one producer warp issuing the bulk copies
constexpr int kWarps = kThreads / 32;
constexpr int kMaxStages = 8;
constexpr int kMaxChunk = 256;                         // rows per chunk (tile box limit)
constexpr size_t kStageTarget = 64 * 1024;            // bytes of one pipeline stage (target)
constexpr size_t kStageBudget = 196 * 1024;           // bytes of all stages together
// FP32 basis: two CTAs per SM (twice the consumer warps for the same bytes), each with about half
// the stage budget; chunks of 128 rows (512-byte runs per column) whenever two stages fit, which
// measured well ahead of 64 rows with more stages
constexpr size_t kStageBudget32 = 100 * 1024;
template <typename TS>
constexpr int ctas_per_sm() { return sizeof(TS) == sizeof(float) ? 2 : 1; }

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait: returns false if the phase did not complete within kSpinLimit polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  for (long long it = 0; it < kSpinLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// 2-D tile load through a tensor map: box at (x = first row, y = first column).
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *tmap, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Barrier 1 over the consumer warps only (the producer warp never joins it), with an OR-vote:
// true on every consumer thread if any passed true.
__device__ __forceinline__ bool consumer_sync_or(bool v) {
  uint32_t out;
  asm volatile(
      "{\n"
      " .reg .pred pi, po;\n"
      " setp.ne.u32 pi, %1, 0;\n"
      " bar.red.or.pred po, 1, %2, pi;\n"
      " selp.u32 %0, 1, 0, po;\n"
      "}\n"
      : "=r"(out)
      : "r"((uint32_t)v), "n"(kConsumers)
      : "memory");
  return out != 0;
}
// Barrier 1 over the consumer warps only, without a vote.
__device__ __forceinline__ void consumer_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(kConsumers) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

struct PassParams {
  GsPassArgs a;
  GsState *st;
  double *coef;
  double *cnew;
  double *partials;
  int first;       // first pass of a column: action = DOT, coefficients start from zero
  int plain_dot;   // plain BVDotVec: DOT only, no decision
  int chunk;       // rows per chunk (power of two, 32..256)
  int stages;      // pipeline stages (2..kMaxStages)
  int box_cols;    // columns fetched by the 2-D tile load (jb, or jb+1 when w is column jb)
  int stage_bytes; // bytes of one stage: CH rows of the jb basis columns (stored type) and of w (FP64)
  int nchunks;
  int G;           // CTAs in the grid
};

// Shared scalars of the decision step.
struct DecideShared {
  int stage, pass, action, cont, lindep, err;
  double onrm, nrm, scale;
  double red[kWarps];
};

// BVOrthogonalizeGS's "finish a pass" logic (bvorthog.c:176-187, 209-214), run by thread 0.
__device__ void finish_pass(DecideShared &d, const PassParams &p, double onrm, double nrm, bool have_next) {
  const GsState *st = p.st;
  const GsPassArgs &a = p.a;
  // fast32: the first pass ran in FP32 arithmetic, so the FP64 correction pass is always taken
  const bool refine =
      d.pass < 3 && nrm != 0.0 && (fabs(nrm) < st->eta * fabs(onrm) || (a.fast32 && d.pass == 1));
  if (refine) {
    if (have_next) {
      // The dot just reduced is already the dot of the next pass.
      d.stage = kStageDotOfPass;
      d.cont = 1;
    } else {
      d.action = kActUpdate | kActDot;
      d.stage = kStageDotOfPass;
      d.cont = 0;
    }
    return;
  }
  const int lindep = !(nrm != 0.0 && fabs(nrm) >= st->eta * fabs(onrm));
  d.lindep = lindep;
  d.nrm = nrm;
  d.scale = (a.normalize && nrm != 1.0 && nrm != 0.0) ? 1.0 / nrm : 1.0;
  d.action = (have_next ? 0 : kActUpdate) | (d.scale != 1.0 ? kActScale : 0);
  d.stage = kStageDone;
  d.cont = 0;
  if (a.hacc) a.hacc[a.jb] = lindep ? 0.0 : nrm;  // BV_SetValue(bv,k,k,h,...)
  if (a.T) {
    a.T[a.step] = (a.jb > 0) ? a.hacc[a.jb - 1] : 0.0;
    a.T[a.ldt + a.step] = lindep ? 0.0 : nrm;
  }
}

// DGKS decision on the reduced dot (cnew_s), run by the whole last CTA.
__device__ void decide(const PassParams &p, const double *cnew_s, DecideShared &d) {
  const GsPassArgs &a = p.a;
  GsState *st = p.st;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    d.stage = p.first ? kStageDotOfPass : st->stage;
    d.pass = p.first ? 0 : st->pass;
    d.onrm = st->onrm;
    d.action = kActNone;
    d.lindep = 0;
    d.err = 0;
    d.nrm = 0.0;
    d.scale = 1.0;
  }
  __syncthreads();
  bool fresh = p.first != 0;
  for (int iter = 0; iter < 4; ++iter) {
    if (d.stage == kStageDotOfPass) {
      // Coefficients of this pass: applied by the next UPDATE and accumulated (BV_AddCoefficients).
      double local = 0.0;
      for (int i = tid; i < a.jb; i += kThreads) {
        const double c = cnew_s[i];
        p.coef[i] = c;
        if (a.hacc) a.hacc[i] = fresh ? c : a.hacc[i] + c;
        local = fma(c, c, local);
      }
      local = warp_sum(local);
      if (lane == 0) d.red[warp] = local;
      __syncthreads();
      if (tid == 0) {
        double sum = 0.0;
        for (int w = 0; w < kWarps; ++w) sum += d.red[w];  // BV_SquareSum
        d.pass += 1;
        const double self = cnew_s[a.jb];
        if (a.column && !(self > -st->deftol)) d.err |= kDevErrInnerProduct;  // BV_SafeSqrt
        const double onrm = (self < 0.0) ? 0.0 : sqrt(self);
        const double t = onrm * onrm - sum;  // estimate |v'| from |v| (bvorthog.c:124-127)
        if (t > 0.0) {
          finish_pass(d, p, onrm, sqrt(t), false);
        } else {
          d.onrm = onrm;
          d.action = kActUpdate | kActDot;  // explicit norm of the updated vector next
          d.stage = kStageExplicitNorm;
          d.cont = 0;
        }
      }
    } else if (d.stage == kStageExplicitNorm) {
      if (tid == 0) {
        const double self = cnew_s[a.jb];
        finish_pass(d, p, d.onrm, (self < 0.0) ? 0.0 : sqrt(self), true);  // BV_NormVecOrColumn
      }
    } else {
      if (tid == 0) d.cont = 0;
    }
    fresh = false;
    __syncthreads();
    if (!d.cont) break;
    __syncthreads();
  }
  if (tid == 0) {
    st->action = d.action;
    st->stage = d.stage;
    st->pass = d.pass;
    st->onrm = d.onrm;
    st->err |= d.err;
    if (d.stage == kStageDone) {
      st->nrm = d.nrm;
      st->scale = d.scale;
      st->beta_out = d.nrm;
      st->lindep = d.lindep;
      if (d.lindep && a.step >= 0) {
        st->halt = 1;
        st->halt_step = a.step;
      }
    } else {
      st->scale = 1.0;
    }
  }
}

// MAXCPW: largest number of dot columns one consumer warp owns (columns warp, warp+8, ...).
//
// Warp roles: warps 0..7 consume (update, scale, dot), warp 8 produces.  The
// producer streams row chunks (w and the jb basis columns, one bulk copy per
// column) into `stages` shared-memory stages; full[s] completes when a
// stage's bytes have landed, empty[s] when the 8 consumer warps are done with
// it.  Consumers synchronise among themselves only between the update (which
// rewrites w) and the dot (which reads the new w).
//
// TS is the stored type of the basis: double, or float for the FP32 basis of the mixed-precision
// solver (w, the coefficients and every product and sum stay FP64).
template <int MAXCPW, typename TS>
__global__ void __launch_bounds__(kThreads, ctas_per_sm<TS>()) gs_pass_kernel(PassParams p,
                                                                             const __grid_constant__ CUtensorMap tmap) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // Launched as a programmatic dependent of the previous kernel in the stream: wait until that
  // grid has finished and its writes (the control block, coefficients, w) are visible, then let
  // the next pass be launched at once (its CTAs take each SM as this grid's CTA leaves it).
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" :::);
  GsState *st = p.st;
  const GsPassArgs &a = p.a;
  if (a.step >= 0 && st->halt && st->halt_step < a.step) return;
  const int action = (p.first || p.plain_dot) ? (int)kActDot : st->action;
  if (action == kActNone) return;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool producer = (warp == kConsumerWarps);
  const int CH = p.chunk;
  const int S = p.stages;
  const int jb = a.jb;
  const bool do_update = (action & kActUpdate) != 0;
  const bool do_dot = (action & kActDot) != 0;
  const bool do_scale = (action & kActScale) != 0;
  const int ncl = (do_update || do_dot) ? jb : 0;  // basis columns streamed
  const double scale = do_scale ? st->scale : 1.0;
  // FP32 basis with fast32: the dot of the first pass and the update that applies its coefficients
  // run in FP32 arithmetic (products and sums), the correction pass in FP64
  const int passno = p.first ? 0 : st->pass;
  const bool fast_dot = sizeof(TS) == sizeof(float) && a.fast32 && p.first && do_dot;
  const bool fast_update = sizeof(TS) == sizeof(float) && a.fast32 && do_update && passno == 1;

  // shared memory carve-up
  uint64_t *full = reinterpret_cast<uint64_t *>(smem_raw);
  uint64_t *empty = full + kMaxStages;
  double *coef_s = reinterpret_cast<double *>(smem_raw + 128);
  double *cacc = coef_s + kMaxCols;           // [kMaxCols + 1]
  DecideShared *dsh = reinterpret_cast<DecideShared *>(cacc + kMaxCols + 1);
  __shared__ int is_last, timed_out, n_issued;
  __shared__ double upd[2 * kConsumers];      // partial update sums (TPR*CH = kConsumers per chunk), by chunk parity
  __shared__ double wps[kMaxChunk];           // w' of the current chunk (updated and scaled), read by the dot
  __shared__ float coef32_s[sizeof(TS) == sizeof(float) ? kMaxCols : 1];  // FP32 coefficients (fast update)
  const size_t head = 128 + sizeof(double) * (2 * kMaxCols + 1) + ((sizeof(DecideShared) + 127) / 128) * 128;
  unsigned char *stage_base = smem_raw + ((head + 127) / 128) * 128;
  const size_t stage_bytes = (size_t)p.stage_bytes;
  const size_t w_offset = (size_t)CH * jb * sizeof(TS);  // w follows the basis columns in a stage

  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumerWarps);
    }
    fence_mbar_init();
    timed_out = 0;
    n_issued = 0;
  }
  for (int i = tid; i < jb; i += kThreads) coef_s[i] = do_update ? p.coef[i] : 0.0;
  if constexpr (sizeof(TS) == sizeof(float))
    if (fast_update)
      for (int i = tid; i < jb; i += kThreads) coef32_s[i] = __double2float_rn(p.coef[i]);
  __syncthreads();

  const int G = p.G;
  const int nmine = (p.nchunks > (int)blockIdx.x) ? (p.nchunks - 1 - (int)blockIdx.x) / G + 1 : 0;
  double *Vw = a.wvec ? a.wvec : a.V + (size_t)a.wcol * a.ld;
  int consumed = 0;

  // dot accumulators: lane-private partial sums of the columns this warp owns, across all chunks
  double acc[MAXCPW];
#pragma unroll
  for (int t = 0; t < MAXCPW; ++t) acc[t] = 0.0;

  if (producer) {
    for (int i = 0; i < nmine; ++i) {
      const int s = i % S;
      if (i >= S) {
        const bool ok = mbar_wait_bounded(&empty[s], (uint32_t)(((i / S) - 1) & 1));
        if (!__all_sync(0xffffffffu, ok)) {
          if (lane == 0) timed_out = 1;
          break;
        }
      }
      const long long r0 = ((long long)blockIdx.x + (long long)i * G) * CH;
      const int rows = (int)min((long long)CH, (long long)a.n - r0);
      unsigned char *buf = stage_base + (size_t)s * stage_bytes;
      if (lane == 0) {
        // one tile load brings the basis columns (and w when it is column jb); rows past n read as zeros
        const bool tile = ncl > 0;
        const bool w_in_tile = tile && p.box_cols == jb + 1;
        const uint32_t wbytes = w_in_tile ? 0u : (uint32_t)(((rows * 8) + 15) & ~15);
        const uint32_t tbytes = tile ? (uint32_t)CH * (uint32_t)sizeof(TS) * (uint32_t)p.box_cols : 0u;
        mbar_arrive_expect_tx(&full[s], tbytes + wbytes);
        if (tile) tma_load_2d(buf, &tmap, (int)r0, 0, &full[s]);
        if (!w_in_tile) bulk_load(buf + w_offset, Vw + r0, wbytes, &full[s]);
        n_issued = i + 1;
      }
      __syncwarp();
    }
  } else {
    // Update mapping: the chunk's rows form CH/32 groups of 32; the 8 consumer warps split into
    // TPR = 8/(CH/32) parts, warp w taking row group w % (CH/32) and columns part, part+TPR, ...
    // (one column, 32 consecutive rows per instruction: no bank conflicts).  Partial sums meet
    // in upd[part][row] behind the chunk's barrier; consumer thread r then folds them into row r
    // of w' (fixed order), keeps it in wps for the dot and writes it back to global memory, and
    // a second barrier hands wps to the dot.
    const int groups = CH / 32;  // 1..8
    const int TPR = kConsumerWarps / groups;
    const int part = warp / groups;
    const int urow = (warp % groups) * 32 + lane;
    for (int i = 0; i < nmine; ++i) {
      const int s = i % S;
      const bool ok = mbar_wait_bounded(&full[s], (uint32_t)((i / S) & 1));
      const long long r0 = ((long long)blockIdx.x + (long long)i * G) * CH;
      const int rows = (int)min((long long)CH, (long long)a.n - r0);
      const unsigned char *sbuf = stage_base + (size_t)s * stage_bytes;
      const TS *Vs = reinterpret_cast<const TS *>(sbuf);  // column c at Vs + c*CH, w after the basis
      const double *wsrc = reinterpret_cast<const double *>(sbuf + w_offset);
      double *up = upd + (i & 1) * kConsumers;  // partial update sums of this chunk
      const bool rewrite = do_update || do_scale;
      if (rewrite) {
        if (ok && do_update) {
          if constexpr (sizeof(TS) == sizeof(double)) {
            double s0 = 0.0, s1 = 0.0;
            int c = part;
            for (; c + TPR < jb; c += 2 * TPR) {
              s0 = fma(Vs[(size_t)c * CH + urow], coef_s[c], s0);
              s1 = fma(Vs[(size_t)(c + TPR) * CH + urow], coef_s[c + TPR], s1);
            }
            if (c < jb) s0 = fma(Vs[(size_t)c * CH + urow], coef_s[c], s0);
            up[part * CH + urow] = s0 + s1;
          } else if (fast_update) {
            float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
            int c = part;
            for (; c + 3 * TPR < jb; c += 4 * TPR) {
              s0 = fmaf((float)Vs[(size_t)c * CH + urow], coef32_s[c], s0);
              s1 = fmaf((float)Vs[(size_t)(c + TPR) * CH + urow], coef32_s[c + TPR], s1);
              s2 = fmaf((float)Vs[(size_t)(c + 2 * TPR) * CH + urow], coef32_s[c + 2 * TPR], s2);
              s3 = fmaf((float)Vs[(size_t)(c + 3 * TPR) * CH + urow], coef32_s[c + 3 * TPR], s3);
            }
            for (; c < jb; c += TPR) s0 = fmaf((float)Vs[(size_t)c * CH + urow], coef32_s[c], s0);
            up[part * CH + urow] = (double)((s0 + s1) + (s2 + s3));
          } else {
            // four independent chains: the FP32 basis doubles the columns a chunk holds per byte
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
            int c = part;
            for (; c + 3 * TPR < jb; c += 4 * TPR) {
              s0 = fma((double)Vs[(size_t)c * CH + urow], coef_s[c], s0);
              s1 = fma((double)Vs[(size_t)(c + TPR) * CH + urow], coef_s[c + TPR], s1);
              s2 = fma((double)Vs[(size_t)(c + 2 * TPR) * CH + urow], coef_s[c + 2 * TPR], s2);
              s3 = fma((double)Vs[(size_t)(c + 3 * TPR) * CH + urow], coef_s[c + 3 * TPR], s3);
            }
            for (; c < jb; c += TPR) s0 = fma((double)Vs[(size_t)c * CH + urow], coef_s[c], s0);
            up[part * CH + urow] = (s0 + s1) + (s2 + s3);
          }
        }
        if (consumer_sync_or(!ok)) break;  // partial sums complete (and a timed-out wait is agreed on)
      } else if (!ok) {
        break;
      }
      // w' = w - sum of the parts (fixed order), scaled: once per row, for the dot and global memory
      if (rewrite) {
        for (int r = tid; r < rows; r += kConsumers) {
          double wv = wsrc[r];
          if (do_update) {
            double tot = 0.0;
            for (int q = 0; q < TPR; ++q) tot += up[q * CH + r];
            wv -= tot;
          }
          if (do_scale) wv *= scale;
          wps[r] = wv;
          Vw[r0 + r] = wv;
        }
        if (do_dot) consumer_sync();
      }
      const double *wd = rewrite ? wps : wsrc;  // the vector the dot multiplies
      if (do_dot && fast_dot) {
        // FP32 products summed in FP32 over the chunk's rows of this lane, then added in FP64
        float facc[MAXCPW];
#pragma unroll
        for (int t = 0; t < MAXCPW; ++t) facc[t] = 0.f;
        for (int r = lane; r < rows; r += 32) {
          const float wr = __double2float_rn(wd[r]);
#pragma unroll
          for (int t = 0; t < MAXCPW; ++t) {
            const int c = warp + kConsumerWarps * t;
            if (c < jb) facc[t] = fmaf((float)Vs[(size_t)c * CH + r], wr, facc[t]);
            else if (c == jb) facc[t] = fmaf(wr, wr, facc[t]);
          }
        }
#pragma unroll
        for (int t = 0; t < MAXCPW; ++t) acc[t] += (double)facc[t];
      } else if (do_dot) {
        for (int r = lane; r < rows; r += 32) {
          const double wr = wd[r];
#pragma unroll
          for (int t = 0; t < MAXCPW; ++t) {
            const int c = warp + kConsumerWarps * t;
            if (c < jb) acc[t] = fma((double)Vs[(size_t)c * CH + r], wr, acc[t]);
            else if (c == jb) acc[t] = fma(wr, wr, acc[t]);
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);  // stage only read here: the next bulk copy may overwrite it
      consumed = i + 1;
    }
    if (lane == 0 && consumed < nmine) timed_out = 1;
  }
  __syncthreads();
  if (timed_out) {
    // Drain the copies still in flight (bounded), report, and leave.
    if (tid == 0) {
      atomicOr(&st->err, (int)kDevErrTimeout);
      for (int i = consumed; i < n_issued; ++i) (void)mbar_wait_bounded(&full[i % S], (uint32_t)((i / S) & 1));
    }
    __syncthreads();
    return;
  }

  // per-CTA column sums -> partials[c * G + cta]
  if (do_dot && !producer) {
#pragma unroll
    for (int t = 0; t < MAXCPW; ++t) {
      const int c = warp + kConsumerWarps * t;
      const double v = warp_sum(acc[t]);
      if (lane == 0 && c <= jb) p.partials[(size_t)c * G + blockIdx.x] = v;
    }
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) is_last = (atomicAdd(&st->ticket, 1u) == (unsigned)(G - 1));
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  if (tid == 0) {
    // algorithmic traffic of this pass: streamed columns + w read, w written back if changed
    st->bytes += (unsigned long long)a.n *
                 ((unsigned long long)sizeof(TS) * ncl + 8ull * (1ull + ((do_update || do_scale) ? 1ull : 0ull)));
    st->passes += 1;
  }
  if (!do_dot) {
    // The final UPDATE/SCALE of a column is done: later follow-up launches idle.
    if (tid == 0) {
      st->ticket = 0u;
      st->action = kActNone;
    }
    return;
  }

  // Fixed-order reduction across CTAs: lane b sums CTAs b, b+32, ...; then a fixed shuffle tree.
  double *cnew_s = cacc;
  for (int c = warp; c <= jb; c += kWarps) {
    double sacc = 0.0;
    for (int b = lane; b < G; b += 32) sacc += __ldcg(p.partials + (size_t)c * G + b);
    sacc = warp_sum(sacc);
    if (lane == 0) {
      cnew_s[c] = sacc;
      p.cnew[c] = sacc;
    }
  }
  __syncthreads();
  if (tid == 0) st->ticket = 0u;
  if (p.plain_dot) return;
  decide(p, cnew_s, *dsh);
}

// bytes of one pipeline stage: CH rows of jb basis columns of ts bytes each, then CH rows of w (FP64)
size_t pass_stage_bytes(int jb, int CH, size_t ts) { return (size_t)CH * ((size_t)jb * ts + sizeof(double)); }

size_t pass_smem_bytes(int jb, int CH, int stages, size_t ts) {
  const size_t head = 128 + sizeof(double) * (2 * kMaxCols + 1) + ((sizeof(DecideShared) + 127) / 128) * 128;
  return ((head + 127) / 128) * 128 + (size_t)stages * pass_stage_bytes(jb, CH, ts);
}

// Rows per chunk: the largest power of two (32..256, the tile box limit) whose stage fits the target size.
int pass_chunk_rows(int jb, size_t ts) {
  if (ts == sizeof(float)) {
    int ch = kMaxChunk / 2;
    while (ch > 32 && 2 * pass_stage_bytes(jb, ch, ts) > kStageBudget32) ch /= 2;
    return ch;
  }
  const size_t rows = kStageTarget / ((size_t)jb * ts + sizeof(double));
  int ch = 32;
  while (ch < kMaxChunk && (size_t)(2 * ch) <= rows) ch *= 2;
  return ch;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  }
  return fn;
}

// Tensor map over the basis: dim 0 = rows (n, contiguous), dim 1 = columns (stride ld), box CH x box_cols.
cudaError_t make_tmap(CUtensorMap *tm, const GsPassArgs &a, int CH, int box_cols, int total_cols) {
  const bool f32 = a.V32 != nullptr;
  memset(tm, 0, sizeof(*tm));
  if (box_cols <= 0) return cudaSuccess;  // no tile load in this pass
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  const cuuint64_t dims[2] = {(cuuint64_t)a.n, (cuuint64_t)total_cols};
  const cuuint64_t strides[1] = {f32 ? (cuuint64_t)a.ld32 * sizeof(float) : (cuuint64_t)a.ld * sizeof(double)};
  const cuuint32_t box[2] = {(cuuint32_t)CH, (cuuint32_t)box_cols};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(tm, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2,
                   f32 ? (void *)a.V32 : (void *)a.V, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

int pass_stages(int jb, int CH, size_t ts) {
  const size_t stage = pass_stage_bytes(jb, CH, ts);
  size_t s = (ts == sizeof(double) ? kStageBudget : kStageBudget32) / stage;
  if (s > (size_t)kMaxStages) s = kMaxStages;
  return (int)s;
}

template <int M, typename TS>
cudaError_t launch_pass_t(const PassParams &p, const CUtensorMap &tm, size_t smem, cudaStream_t stream) {
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr_set[dev]) {
    cudaError_t e = allow_max_dynamic_smem(gs_pass_kernel<M, TS>);
    if (e != cudaSuccess) return e;
    attr_set[dev] = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)p.G);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, gs_pass_kernel<M, TS>, p, tm);
}

cudaError_t launch_pass(const GsPassArgs &a, const GsWork &w, int first, int plain_dot, cudaStream_t stream) {
  PassParams p;
  p.a = a;
  p.st = w.st;
  p.coef = w.coef;
  p.cnew = w.cnew;
  p.partials = w.partials;
  p.first = first;
  p.plain_dot = plain_dot;
  const bool f32 = a.V32 != nullptr;
  const size_t ts = f32 ? sizeof(float) : sizeof(double);
  if (f32 && !a.wvec) return cudaErrorInvalidValue;  // w is FP64 and kept apart from an FP32 basis
  p.chunk = pass_chunk_rows(a.jb, ts);
  p.stages = pass_stages(a.jb, p.chunk, ts);
  p.stage_bytes = (int)pass_stage_bytes(a.jb, p.chunk, ts);
  if (p.stages < 2) return cudaErrorInvalidValue;
  p.nchunks = (a.n + p.chunk - 1) / p.chunk;
  int G = w.num_sms * (f32 ? ctas_per_sm<float>() : 1);
  if (G > w.max_ctas) G = w.max_ctas;
  if (G > p.nchunks) G = p.nchunks;
  if (G < 1) G = 1;
  p.G = G;
  const size_t smem = pass_smem_bytes(a.jb, p.chunk, p.stages, ts);
  if (smem + 4096 > max_dynamic_smem()) return cudaErrorInvalidValue;
  // w is column jb in the column variant: one box covers basis and w
  p.box_cols = (a.wcol == a.jb && !a.wvec && !f32) ? a.jb + 1 : a.jb;
  CUtensorMap tm;
  cudaError_t e = make_tmap(&tm, a, p.chunk, p.box_cols, a.total_cols);
  if (e != cudaSuccess) return e;
  const int cpw = (a.jb + 1 + kConsumerWarps - 1) / kConsumerWarps;  // dot columns per consumer warp (basis + self)
  if (f32) {
    if (cpw <= 2) e = launch_pass_t<2, float>(p, tm, smem, stream);
    else if (cpw <= 4) e = launch_pass_t<4, float>(p, tm, smem, stream);
    else if (cpw <= 8) e = launch_pass_t<8, float>(p, tm, smem, stream);
    else if (cpw <= 12) e = launch_pass_t<12, float>(p, tm, smem, stream);
    else if (cpw <= 16) e = launch_pass_t<16, float>(p, tm, smem, stream);
    else if (cpw <= 32) e = launch_pass_t<32, float>(p, tm, smem, stream);
    else return cudaErrorInvalidValue;
  } else if (cpw <= 2) e = launch_pass_t<2, double>(p, tm, smem, stream);
  else if (cpw <= 4) e = launch_pass_t<4, double>(p, tm, smem, stream);
  else if (cpw <= 8) e = launch_pass_t<8, double>(p, tm, smem, stream);
  else if (cpw <= 12) e = launch_pass_t<12, double>(p, tm, smem, stream);
  else if (cpw <= 16) e = launch_pass_t<16, double>(p, tm, smem, stream);
  else if (cpw <= 32) e = launch_pass_t<32, double>(p, tm, smem, stream);
  else return cudaErrorInvalidValue;
  count_launch();
  return e;
}

}  // namespace

namespace {
__global__ void gs_reset_kernel(GsState *st, double eta) {
  GsState h;
  memset(&h, 0, sizeof(h));
  h.eta = eta;
  h.deftol = 10.0 * 2.220446049250313e-16;  // BV deftol = 10*PETSC_MACHINE_EPSILON (bvfunc.c:184)
  h.halt_step = -1;
  h.scale = 1.0;
  *st = h;
}
}  // namespace

cudaError_t gs_state_reset(const GsWork &w, double eta, cudaStream_t stream) {
  gs_reset_kernel<<<1, 1, 0, stream>>>(w.st, eta);
  count_launch();
  return cudaGetLastError();
}

cudaError_t gs_orthogonalize_launch(const GsPassArgs &a, const GsWork &w, cudaStream_t stream) {
  if (a.jb < 0 || a.jb >= kMaxCols) return cudaErrorInvalidValue;
  cudaError_t e = launch_pass(a, w, 1, 0, stream);
  // Worst case: three passes whose norm estimates all need the explicit norm,
  // then a final scale: four follow-up launches (idle ones return at once).
  for (int k = 0; k < 4 && e == cudaSuccess; ++k) e = launch_pass(a, w, 0, 0, stream);
  return e;
}

// out[0] = the norm, out[1] = the lindep flag, out[2] = the device error bits of the last column
// orthogonalisation (read back once for a block of columns)
__global__ void gs_record_kernel(const GsState *__restrict__ st, double *out) {
  out[0] = st->beta_out;
  out[1] = (double)st->lindep;
  out[2] = (double)st->err;
}

cudaError_t gs_record_launch(const GsWork &w, double *out, cudaStream_t stream) {
  gs_record_kernel<<<1, 1, 0, stream>>>(w.st, out);
  count_launch();
  return cudaGetLastError();
}

cudaError_t gs_dot_launch(const GsPassArgs &a, const GsWork &w, cudaStream_t stream) {
  if (a.jb < 0 || a.jb >= kMaxCols) return cudaErrorInvalidValue;
  return launch_pass(a, w, 0, 1, stream);
}

}  // namespace b200
