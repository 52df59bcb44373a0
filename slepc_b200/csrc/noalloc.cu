// Allocation-free Gram-Schmidt entry point.
//
// b200_orthogonalize_column_noalloc runs the same fused CGS + DGKS passes as
// b200_bv_orthogonalize_column on a basis the caller owns, but takes every
// piece of working memory from one fixed array compiled into this library
// instead of allocating device memory.  It exists for callers that cannot
// call cudaMalloc: code running where device allocation is forbidden or
// unavailable to it, such as a host that has handed all device memory to its
// own pool allocator, or a plugin loaded into a process whose memory budget
// must not grow after start-up.
//
// The scratch array lives in device global memory for the life of the
// process on every GPU that loads this library.  Its address is looked up
// once per (device, context) pair, on the first call made with that device
// and context current: a caller that makes its own contexts with cuCtxCreate
// gets the array of its own context, not the primary context's.  The lookup
// is not repeated after cudaDeviceReset (the primary context keeps its
// handle across a reset while the module, and with it the array, may be
// reloaded elsewhere), so a process that resets a device must not call this
// entry point on that device afterwards.  All calls share the one array, so
// two calls whose work overlaps on the GPU (different streams, or different
// host threads) overwrite each other's scratch and give wrong results:
// serialise them.
#include <cuda.h>

#include <mutex>

#include "common.h"
#include "kernels.h"

namespace b200 {
namespace {

// Capacity of the scratch: the control block, the coefficient vectors and the
// per-CTA partial dot products of up to kNoAllocMaxCtas CTAs.
constexpr int kNoAllocMaxCtas = 160;
constexpr size_t kScratchDoubles =
    (sizeof(GsState) + 7) / 8 + 32 + kMaxCols + (kMaxCols + 1) + (size_t)(kMaxCols + 1) * kNoAllocMaxCtas;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

struct ScratchView {
  int dev = -1;
  CUcontext ctx = nullptr;  // context the address belongs to
  double *base = nullptr;   // device address of g_noalloc_scratch in that context
};

constexpr int kMaxViews = 64;
std::mutex g_setup_mutex;
ScratchView g_views[kMaxViews];
int g_nviews = 0;

using CtxGetCurrent = CUresult (*)(CUcontext *);

// The calling thread's current context through the driver entry point (no link against libcuda;
// nothing is allocated).  Null when no context is current yet.
CUcontext current_context() {
  static CtxGetCurrent fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<CtxGetCurrent>(p);
  }();
  CUcontext c = nullptr;
  if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
  return c;
}

// Device address of the scratch for the current device and context, looked up once per pair.
cudaError_t scratch_address(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  CUcontext ctx = current_context();
  for (int i = 0; ctx && i < g_nviews; ++i)
    if (g_views[i].dev == dev && g_views[i].ctx == ctx) {
      *out = g_views[i].base;
      return cudaSuccess;
    }
  // first call in this context (or no context current yet: the lookup makes the primary one current)
  void *p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  ctx = current_context();
  bool known = false;
  for (int i = 0; ctx && i < g_nviews; ++i) known = known || (g_views[i].dev == dev && g_views[i].ctx == ctx);
  if (ctx && !known && g_nviews < kMaxViews) g_views[g_nviews++] = ScratchView{dev, ctx, static_cast<double *>(p)};
  *out = static_cast<double *>(p);
  return cudaSuccess;
}

}  // namespace
}  // namespace b200

using namespace b200;

extern "C" b200_status b200_orthogonalize_column_noalloc(int n, int ld, int ncols, double *V, int j, double *H,
                                                         double *norm, int *lindep, void *stream) {
  B200_ARG_CHECK(V && H && n > 0 && ld >= n && ld % 2 == 0, "V must be n x ncols column-major with an even ld >= n");
  B200_ARG_CHECK(j >= 0 && j < ncols, "column index j out of range");
  B200_ARG_CHECK(j + 1 < kMaxCols, "j too large for the fixed scratch: j must be at most 253");
  B200_ARG_CHECK(((uintptr_t)V & 15) == 0, "V must be 16-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  double *base = nullptr;
  B200_CUDA_CHECK(scratch_address(&base));

  // carve the scratch: control block, coefficients, reduced dot, per-CTA partials
  GsWork w{};
  double *q = base;
  w.st = reinterpret_cast<GsState *>(q);
  q += (sizeof(GsState) + 7) / 8 + 32;
  w.coef = q;
  q += kMaxCols;
  w.cnew = q;
  q += kMaxCols + 1;
  w.partials = q;
  int sms = 0, dev = 0;
  B200_CUDA_CHECK(cudaGetDevice(&dev));
  B200_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  w.num_sms = sms;
  w.max_ctas = sms < kNoAllocMaxCtas ? sms : kNoAllocMaxCtas;

  // the control block carries over from the last call: start it from zero
  B200_CUDA_CHECK(gs_state_reset(w, 0.7071, s));
  GsPassArgs a{};
  a.V = V;
  a.ld = ld;
  a.n = n;
  a.jb = j;
  a.wcol = j;
  a.total_cols = ncols;
  a.hacc = H;
  a.T = nullptr;
  a.ldt = 0;
  a.step = -1;
  a.normalize = 0;
  a.column = 1;
  B200_CUDA_CHECK(gs_orthogonalize_launch(a, w, s));
  GsState st;
  B200_CUDA_CHECK(cudaMemcpyAsync(&st, w.st, sizeof(GsState), cudaMemcpyDeviceToHost, s));
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  if (st.err & kDevErrInnerProduct) {
    b200_set_last_error(__FILE__, __LINE__, "invalid inner product (negative self dot product)");
    return B200_ERR_INNER;
  }
  if (st.err) {
    b200_set_last_error(__FILE__, __LINE__, "a Gram-Schmidt kernel reported a device-side error");
    return B200_ERR_DEVICE;
  }
  if (norm) *norm = st.beta_out;
  if (lindep) *lindep = st.lindep;
  return B200_OK;
}
