// Host objects (Mat, BV, EPS), the Krylov-Schur driver and the C ABI.
//
// The driver restates EPSSolve_KrylovSchur_Default
// (src/eps/impls/krylov/krylovschur/krylovschur.c:227-348) for Hermitian
// problems with Ritz extraction and locking, together with EPSSetUp's
// defaults (krylovschur.c:93-194, src/eps/interface/epssetup.c:669-713),
// EPSGetStartVector (epssolve.c:841-870), EPSKrylovConvergence
// (src/eps/impls/krylov/epskrylov.c:207-295), EPSConvergedRelative and
// EPSStoppingBasic (epsdefault.c:224-232, 290-305), and SlepcSortEigenvalues
// (src/sys/slepcsc.c:89-149).  All vector work runs on the GPU; a Lanczos
// run of BVMatLanczos (bvkrylov.c:165-226) is enqueued as one asynchronous
// sequence of kernels with a single host synchronisation at its end.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.h"
#include "ds_hep.h"
#include "internal.h"
#include "kernels.h"
#include "rowblock.h"
#include "objects.h"

using namespace b200;

// --------------------------------------------------------------- errors ---
static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

// LAPACK from the OpenBLAS bundled with scipy (symbols carry a scipy_ prefix)
extern "C" void scipy_dpotrf_(const char *uplo, const int *n, double *a, const int *lda, int *info, size_t);
extern "C" void scipy_dtrtri_(const char *uplo, const char *diag, const int *n, double *a, const int *lda, int *info,
                              size_t, size_t);
extern "C" void scipy_dsyev_(const char *jobz, const char *uplo, const int *n, double *a, const int *lda, double *w,
                             double *work, const int *lwork, int *info, size_t, size_t);

extern "C" void b200_set_last_error(const char *file, int line, const char *msg) {
  const char *base = strrchr(file, '/');
  g_last_error = std::string(msg) + " (" + (base ? base + 1 : file) + ":" + std::to_string(line) + ")";
}
extern "C" const char *b200_last_error(void) { return g_last_error.c_str(); }
extern "C" const char *b200_version(void) { return "slepc_b200 0.1 (sm_100a, FP64 Krylov-Schur)"; }
extern "C" uint64_t b200_kernel_launch_count(void) { return g_launches.load(); }

namespace b200 {
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(); }
// Stream-ordered allocations from one pool per device that keeps up to kPoolKeep bytes of what is
// freed for the next allocation of the process (the mixed form's gigabyte blocks, the basis and
// matrix arrays of a repeated solve); beyond that the driver returns memory at the next
// synchronisation.
static constexpr uint64_t kPoolKeep = 16ull << 30;
static std::mutex g_pool_mu;
static cudaMemPool_t g_pools[64] = {};
static cudaStream_t g_alloc_streams[64] = {};

static cudaMemPool_t device_pool(int dev) {
  if (dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  cudaMemPool_t *pools = g_pools;
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    uint64_t keep = kPoolKeep;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = p;
  }
  return pools[dev];
}

// The library's own non-blocking stream on device dev, on which object buffers are allocated and
// freed (so that every reuse of a freed block by a later object is ordered on one stream).
static cudaStream_t alloc_stream(int dev) {
  if (dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (!g_alloc_streams[dev]) {
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    g_alloc_streams[dev] = st;
  }
  return g_alloc_streams[dev];
}

cudaError_t pool_alloc(void **p, size_t bytes, cudaStream_t s) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  cudaMemPool_t pool = device_pool(dev);
  if (!pool) return cudaErrorMemoryAllocation;
  return cudaMallocFromPoolAsync(p, bytes, pool, s);
}

cudaError_t pool_free(void *p, cudaStream_t s) { return p ? cudaFreeAsync(p, s) : cudaSuccess; }

cudaError_t dev_malloc(void **p, size_t bytes) {
  *p = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  cudaMemPool_t pool = device_pool(dev);
  cudaStream_t s = alloc_stream(dev);
  if (!pool || !s) return cudaErrorMemoryAllocation;
  e = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    if (*p) cudaFreeAsync(*p, s);
    *p = nullptr;
    // an allocation that the kept memory blocks: hand the pool's unused memory back and retry once
    if (e == cudaErrorMemoryAllocation) {
      cudaGetLastError();
      cudaStreamSynchronize(s);
      cudaMemPoolTrimTo(pool, 0);
      e = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) *p = nullptr;
    }
  }
  return e;
}

void dev_free(void *p) {
  if (!p) return;
  // the buffer's own device (an object may be destroyed while another device is current)
  int cur = 0, dev = 0;
  cudaGetDevice(&cur);
  dev = cur;
  cudaPointerAttributes pa;
  if (cudaPointerGetAttributes(&pa, p) == cudaSuccess && pa.type == cudaMemoryTypeDevice) dev = pa.device;
  else cudaGetLastError();
  if (dev != cur) cudaSetDevice(dev);
  cudaDeviceSynchronize();
  cudaFreeAsync(p, alloc_stream(dev));
  if (dev != cur) cudaSetDevice(cur);
}

int num_sms_host() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  return v > 0 ? v : 1;
}
}  // namespace b200

#define B200_DEV_ERR(msg)                             \
  do {                                                \
    b200_set_last_error(__FILE__, __LINE__, msg);     \
    return B200_ERR_DEVICE;                           \
  } while (0)

// ------------------------------------------------------------------ Mat ---
static void part_free(CsrPart &P) {
  dev_free(P.rowptr);
  dev_free(P.colind);
  dev_free(P.vals);
  dev_free(P.blocks);
  dev_free(P.wt.tiles);
  dev_free(P.wt.segs);
  dev_free(P.wt.longrows);
  dev_free(P.wt.partials);
  dev_free(P.sell.off);
  dev_free(P.sell.width);
  dev_free(P.sell.mask);
  dev_free(P.sell.vals);
  dev_free(P.sell.cols);
  dev_free(P.sell.rest.tiles);
  dev_free(P.sell.rest.segs);
  dev_free(P.sell.rest.longrows);
  dev_free(P.sell.rest.partials);
  dev_free(P.sell.rest_rows);
  dev_free(P.sell.vals32);
  dev_free(P.vals32);
  P = CsrPart{};
}

static b200_status part_alloc(CsrPart &P, int rows, int cols, int64_t nnz, bool f32) {
  P.rows = rows;
  P.cols = cols;
  P.nnz = nnz;
  P.f32 = f32;
  P.lanes = spmv_choose_lanes(rows, nnz);
  const size_t vsz = f32 ? sizeof(float) : sizeof(double);
  if (dev_malloc(&P.rowptr, sizeof(int) * ((size_t)rows + 1)) != cudaSuccess ||
      dev_malloc(&P.colind, sizeof(int) * (size_t)(nnz > 0 ? nnz : 1)) != cudaSuccess ||
      dev_malloc(&P.vals, vsz * (size_t)(nnz > 0 ? nnz : 1)) != cudaSuccess) {
    part_free(P);
    b200_set_last_error(__FILE__, __LINE__, "device allocation failed for the CSR arrays");
    return B200_ERR_NOMEM;
  }
  return B200_OK;
}

static b200_status part_upload(CsrPart &P, const int *rowptr, const int *colind, const void *vals, cudaMemcpyKind kind,
                               cudaStream_t s) {
  const size_t vsz = P.f32 ? sizeof(float) : sizeof(double);
  cudaError_t e = cudaMemcpyAsync(P.rowptr, rowptr, sizeof(int) * ((size_t)P.rows + 1), kind, s);
  if (e == cudaSuccess && P.nnz) e = cudaMemcpyAsync(P.colind, colind, sizeof(int) * (size_t)P.nnz, kind, s);
  if (e == cudaSuccess && P.nnz) e = cudaMemcpyAsync(P.vals, vals, vsz * (size_t)P.nnz, kind, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    b200_set_last_error(__FILE__, __LINE__, cudaGetErrorString(e));
    return B200_ERR_CUDA;
  }
  return B200_OK;
}

static b200_status part_build_sell(CsrPart &P, const int *rowptr_host, cudaStream_t s);

// Row blocks (FP64 only), warp tiles and the sliced-ELL copy (the default schedule) from a host
// copy of rowptr, uploaded to the device.
static b200_status part_set_schedules(CsrPart &P, const int *rowptr_host, cudaStream_t s) {
  if (!P.f32) {
    std::vector<int> b = spmv_row_blocks(P.rows, rowptr_host);
    P.nblocks = (int)b.size() - 1;
    B200_CUDA_CHECK(dev_malloc(&P.blocks, sizeof(int) * b.size()));
    B200_CUDA_CHECK(cudaMemcpyAsync(P.blocks, b.data(), sizeof(int) * b.size(), cudaMemcpyHostToDevice, s));
  }
  WarpTiles wt = spmv_warp_tiles(P.rows, rowptr_host);
  P.wt.ntiles = (int)wt.tiles.size();
  P.wt.nsegs = (int)wt.segs.size();
  P.wt.nlong = (int)wt.longrows.size();
  if (P.wt.ntiles) {
    B200_CUDA_CHECK(dev_malloc(&P.wt.tiles, sizeof(int4) * wt.tiles.size()));
    B200_CUDA_CHECK(
        cudaMemcpyAsync(P.wt.tiles, wt.tiles.data(), sizeof(int4) * wt.tiles.size(), cudaMemcpyHostToDevice, s));
  }
  if (P.wt.nsegs) {
    B200_CUDA_CHECK(dev_malloc(&P.wt.segs, sizeof(int2) * wt.segs.size()));
    B200_CUDA_CHECK(dev_malloc(&P.wt.partials, sizeof(double) * wt.segs.size()));
    B200_CUDA_CHECK(dev_malloc(&P.wt.longrows, sizeof(int3) * wt.longrows.size()));
    B200_CUDA_CHECK(
        cudaMemcpyAsync(P.wt.segs, wt.segs.data(), sizeof(int2) * wt.segs.size(), cudaMemcpyHostToDevice, s));
    B200_CUDA_CHECK(cudaMemcpyAsync(P.wt.longrows, wt.longrows.data(), sizeof(int3) * wt.longrows.size(),
                                    cudaMemcpyHostToDevice, s));
  }
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  return part_build_sell(P, rowptr_host, s);
}

// Sliced-ELL copy of a CSR operand, built in HBM from the device CSR arrays.
static b200_status part_build_sell(CsrPart &P, const int *rowptr_host, cudaStream_t s) {
  if (P.sell_ready) return B200_OK;
  std::vector<int> rp;
  if (!rowptr_host) {
    rp.resize((size_t)P.rows + 1);
    B200_CUDA_CHECK(cudaMemcpyAsync(rp.data(), P.rowptr, sizeof(int) * rp.size(), cudaMemcpyDeviceToHost, s));
    B200_CUDA_CHECK(cudaStreamSynchronize(s));
    rowptr_host = rp.data();
  }
  SellPlan sp = spmv_sell_plan(P.rows, rowptr_host);
  SpmvSell &S = P.sell;
  S.nslices = (int)sp.off.size();
  const size_t vsz = P.f32 ? sizeof(float) : sizeof(double);
  B200_CUDA_CHECK(dev_malloc(&S.off, sizeof(long long) * (S.nslices ? S.nslices : 1)));
  B200_CUDA_CHECK(dev_malloc(&S.width, sizeof(int) * (S.nslices ? S.nslices : 1)));
  B200_CUDA_CHECK(dev_malloc(&S.mask, sizeof(unsigned) * (S.nslices ? S.nslices : 1)));
  B200_CUDA_CHECK(dev_malloc(&S.vals, vsz * (size_t)(sp.entries ? sp.entries : 1)));
  B200_CUDA_CHECK(dev_malloc(&S.cols, sizeof(int) * (size_t)(sp.entries ? sp.entries : 1)));
  if (S.nslices) {
    B200_CUDA_CHECK(cudaMemcpyAsync(S.off, sp.off.data(), sizeof(long long) * S.nslices, cudaMemcpyHostToDevice, s));
    B200_CUDA_CHECK(cudaMemcpyAsync(S.width, sp.width.data(), sizeof(int) * S.nslices, cudaMemcpyHostToDevice, s));
    B200_CUDA_CHECK(cudaMemcpyAsync(S.mask, sp.mask.data(), sizeof(unsigned) * S.nslices, cudaMemcpyHostToDevice, s));
    B200_CUDA_CHECK(sell_gather(P.rows, S, P.rowptr, P.colind, P.vals, P.f32, s));
  }
  S.entries = sp.entries;
  S.max_width = 0;
  for (int w : sp.width) S.max_width = w > S.max_width ? w : S.max_width;
  S.nrest = (int)sp.rest_rows.size();
  if (S.nrest) {
    B200_CUDA_CHECK(dev_malloc(&S.rest_rows, sizeof(int) * sp.rest_rows.size()));
    B200_CUDA_CHECK(cudaMemcpyAsync(S.rest_rows, sp.rest_rows.data(), sizeof(int) * sp.rest_rows.size(),
                                    cudaMemcpyHostToDevice, s));
  }
  WarpTiles &wt = sp.rest;
  S.rest.ntiles = (int)wt.tiles.size();
  S.rest.nsegs = (int)wt.segs.size();
  S.rest.nlong = (int)wt.longrows.size();
  if (S.rest.ntiles) {
    B200_CUDA_CHECK(dev_malloc(&S.rest.tiles, sizeof(int4) * wt.tiles.size()));
    B200_CUDA_CHECK(
        cudaMemcpyAsync(S.rest.tiles, wt.tiles.data(), sizeof(int4) * wt.tiles.size(), cudaMemcpyHostToDevice, s));
  }
  if (S.rest.nsegs) {
    B200_CUDA_CHECK(dev_malloc(&S.rest.segs, sizeof(int2) * wt.segs.size()));
    B200_CUDA_CHECK(dev_malloc(&S.rest.partials, sizeof(double) * wt.segs.size()));
    B200_CUDA_CHECK(dev_malloc(&S.rest.longrows, sizeof(int3) * wt.longrows.size()));
    B200_CUDA_CHECK(
        cudaMemcpyAsync(S.rest.segs, wt.segs.data(), sizeof(int2) * wt.segs.size(), cudaMemcpyHostToDevice, s));
    B200_CUDA_CHECK(cudaMemcpyAsync(S.rest.longrows, wt.longrows.data(), sizeof(int3) * wt.longrows.size(),
                                    cudaMemcpyHostToDevice, s));
  }
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  P.sell_ready = true;
  return B200_OK;
}

static cudaError_t part_spmv(const CsrPart &P, int schedule, const double *x, double *y, cudaStream_t stream,
                             const GsState *st, int step) {
  if (schedule == B200_SPMV_SELL && P.sell_ready) {
    if (P.f32)
      return spmv_sell_launch_f32(P.sell, P.rows, P.sell.rest, P.rowptr, P.colind, static_cast<const float *>(P.vals),
                                  x, y, stream, st, step);
    return spmv_sell_launch(P.sell, P.rows, P.sell.rest, P.rowptr, P.colind, static_cast<const double *>(P.vals), x,
                            y, stream, st, step);
  }
  const bool pipelined = schedule == B200_SPMV_PIPELINED;
  if (P.f32)
    return spmv_warptile_launch_f32(P.wt, P.rowptr, P.colind, static_cast<const float *>(P.vals), x, y, stream, st,
                                    step, pipelined);
  if (schedule == B200_SPMV_ROWBLOCK)
    return spmv_rowblock_launch(P.nblocks, P.blocks, P.rowptr, P.colind, static_cast<const double *>(P.vals), x, y,
                                stream, st, step);
  return spmv_warptile_launch(P.wt, P.rowptr, P.colind, static_cast<const double *>(P.vals), x, y, stream, st, step,
                              pipelined);
}

// y = Op x for the operator of A (the EPS operator: A itself, or A^T A).
static cudaError_t mat_spmv(b200_mat A, const double *x, double *y, cudaStream_t stream, const GsState *st = nullptr,
                            int step = 0) {
  if (A->kind == kMatCross) {
    const CsrPart &first = A->swapped ? A->base->at : A->base->a;
    const CsrPart &second = A->swapped ? A->base->a : A->base->at;
    cudaError_t e = part_spmv(first, A->base->schedule, x, A->work, stream, st, step);
    if (e != cudaSuccess) return e;
    return part_spmv(second, A->base->schedule, A->work, y, stream, st, step);
  }
  return part_spmv(A->a, A->schedule, x, y, stream, st, step);
}

template <typename VT>
static double csr_norm_inf_host(int rows, const int *rowptr, const VT *vals) {
  double nrm = 0.0;
  for (int i = 0; i < rows; ++i) {
    double sacc = 0.0;
    for (int p = rowptr[i]; p < rowptr[i + 1]; ++p) sacc += std::fabs((double)vals[p]);
    if (sacc > nrm) nrm = sacc;
  }
  return nrm;
}

extern "C" b200_status b200_mat_create_csr(int n, int64_t nnz, const int *rowptr, const int *colind, const double *vals,
                                           void *stream, b200_mat *A) {
  B200_ARG_CHECK(A && n > 0 && nnz >= 0 && rowptr && (nnz == 0 || (colind && vals)), "invalid CSR arguments");
  B200_ARG_CHECK(rowptr[0] == 0 && rowptr[n] == nnz, "rowptr must start at 0 and end at nnz");
  B200_ARG_CHECK(nnz <= 0x7fffffff, "nnz must fit a 32-bit index (PETSc default int size)");
  cudaStream_t s = (cudaStream_t)stream;
  b200_mat M = new b200_mat_s;
  M->m = M->n = n;
  M->nnz = nnz;
  M->stream = s;
  b200_status st = part_alloc(M->a, n, n, nnz, false);
  if (st == B200_OK) st = part_upload(M->a, rowptr, colind, vals, cudaMemcpyHostToDevice, s);
  if (st == B200_OK) st = part_set_schedules(M->a, rowptr, s);
  if (st != B200_OK) {
    b200_mat_destroy(M);
    return st;
  }
  M->norm_inf = csr_norm_inf_host(n, rowptr, vals);
  *A = M;
  return B200_OK;
}

extern "C" b200_status b200_mat_create_csr_device(int n, int64_t nnz, const int *rowptr, const int *colind,
                                                  const double *vals, void *stream, b200_mat *A) {
  B200_ARG_CHECK(A && n > 0 && nnz >= 0 && rowptr && (nnz == 0 || (colind && vals)), "invalid CSR arguments");
  B200_ARG_CHECK(nnz <= 0x7fffffff, "nnz must fit a 32-bit index");
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<int> hrow((size_t)n + 1);
  B200_CUDA_CHECK(cudaMemcpyAsync(hrow.data(), rowptr, sizeof(int) * ((size_t)n + 1), cudaMemcpyDeviceToHost, s));
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  B200_ARG_CHECK(hrow[0] == 0 && hrow[n] == nnz, "rowptr must start at 0 and end at nnz");
  b200_mat M = new b200_mat_s;
  M->m = M->n = n;
  M->nnz = nnz;
  M->stream = s;
  b200_status st = part_alloc(M->a, n, n, nnz, false);
  if (st == B200_OK) st = part_upload(M->a, rowptr, colind, vals, cudaMemcpyDeviceToDevice, s);
  if (st == B200_OK) st = part_set_schedules(M->a, hrow.data(), s);
  if (st != B200_OK) {
    b200_mat_destroy(M);
    return st;
  }
  *A = M;
  return B200_OK;
}

template <typename VT>
static b200_status mat_create_aij(int m, int n, int64_t nnz, const int *rowptr, const int *colind, const VT *vals,
                                  cudaStream_t s, b200_mat *A) {
  for (int64_t p = 0; p < nnz; ++p)
    B200_ARG_CHECK(colind[p] >= 0 && colind[p] < n, "column index out of range");
  for (int i = 0; i < m; ++i) B200_ARG_CHECK(rowptr[i] <= rowptr[i + 1], "rowptr must be nondecreasing");
  const bool f32 = sizeof(VT) == sizeof(float);
  b200_mat M = new b200_mat_s;
  M->m = m;
  M->n = n;
  M->nnz = nnz;
  M->stream = s;
  b200_status st = part_alloc(M->a, m, n, nnz, f32);
  if (st == B200_OK) st = part_upload(M->a, rowptr, colind, vals, cudaMemcpyHostToDevice, s);
  if (st == B200_OK) st = part_set_schedules(M->a, rowptr, s);
  // the explicit transpose, built in HBM from the uploaded A
  if (st == B200_OK) st = part_alloc(M->at, n, m, nnz, f32);
  std::vector<int> rp;
  if (st == B200_OK) {
    cudaError_t e = csr_transpose_device(m, n, nnz, M->a.rowptr, M->a.colind, M->a.vals, f32, M->at.rowptr,
                                         M->at.colind, M->at.vals, s);
    rp.resize((size_t)n + 1);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(rp.data(), M->at.rowptr, sizeof(int) * ((size_t)n + 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      b200_set_last_error(__FILE__, __LINE__, cudaGetErrorString(e));
      st = e == cudaErrorMemoryAllocation ? B200_ERR_NOMEM : B200_ERR_CUDA;
    }
  }
  if (st == B200_OK) st = part_set_schedules(M->at, rp.data(), s);
  if (st != B200_OK) {
    b200_mat_destroy(M);
    return st;
  }
  M->norm_inf = csr_norm_inf_host(m, rowptr, vals);
  *A = M;
  return B200_OK;
}

extern "C" b200_status b200_mat_create_aij(int m, int n, int64_t nnz, const int *rowptr, const int *colind,
                                           const void *vals, int scalar_type, void *stream, b200_mat *A) {
  B200_ARG_CHECK(A && m > 0 && n > 0 && nnz >= 0 && rowptr && (nnz == 0 || (colind && vals)), "invalid CSR arguments");
  B200_ARG_CHECK(rowptr[0] == 0 && rowptr[m] == nnz, "rowptr must start at 0 and end at nnz");
  B200_ARG_CHECK(nnz <= 0x7fffffff, "nnz must fit a 32-bit index (PETSc default int size)");
  B200_ARG_CHECK(scalar_type == B200_SCALAR_F64 || scalar_type == B200_SCALAR_F32, "unknown scalar type");
  if (scalar_type == B200_SCALAR_F32)
    return mat_create_aij(m, n, nnz, rowptr, colind, static_cast<const float *>(vals), (cudaStream_t)stream, A);
  return mat_create_aij(m, n, nnz, rowptr, colind, static_cast<const double *>(vals), (cudaStream_t)stream, A);
}

namespace b200 {
b200_status mat_create_cross_ex(b200_mat A, bool swapped, b200_mat *C) {
  B200_ARG_CHECK(A && C && A->kind == kMatCsr && A->at.rows == A->n, "A must be a matrix from b200_mat_create_aij");
  b200_mat M = new b200_mat_s;
  M->kind = kMatCross;
  M->swapped = swapped;
  M->m = M->n = swapped ? A->m : A->n;
  M->nnz = A->nnz;
  M->base = A;
  M->stream = A->stream;
  const int wlen = swapped ? A->n : A->m;
  if (dev_malloc(&M->work, sizeof(double) * (size_t)wlen) != cudaSuccess) {
    delete M;
    b200_set_last_error(__FILE__, __LINE__, "device allocation failed for the cross-product work vector");
    return B200_ERR_NOMEM;
  }
  *C = M;
  return B200_OK;
}

cudaError_t mat_apply(b200_mat A, const double *x, double *y, cudaStream_t stream, bool transpose) {
  if (!transpose) return mat_spmv(A, x, y, stream);
  return part_spmv(A->at, A->schedule, x, y, stream, nullptr, 0);
}
}  // namespace b200

extern "C" b200_status b200_mat_create_cross(b200_mat A, b200_mat *C) { return mat_create_cross_ex(A, false, C); }

// The sliced-ELL copy of a square CSR operator and, for FP64 values, FP32 copies of its values
// (CSR and slices) for the FP32 phase of the mixed-precision solver.
b200_status b200::mat_mixed_prepare(b200_mat A, cudaStream_t s) {
  B200_ARG_CHECK(A->kind == kMatCsr && A->m == A->n, "the mixed-precision solver needs a square CSR operator");
  CsrPart &P = A->a;
  B200_CHECK(part_build_sell(P, nullptr, s));
  if (!P.f32 && !P.vals32) {
    B200_CUDA_CHECK(dev_malloc(&P.vals32, sizeof(float) * (size_t)(P.nnz > 0 ? P.nnz : 1)));
    B200_CUDA_CHECK(dev_malloc(&P.sell.vals32, sizeof(float) * (size_t)(P.sell.entries > 0 ? P.sell.entries : 1)));
    B200_CUDA_CHECK(to_f32_launch(P.vals32, static_cast<const double *>(P.vals), P.nnz, s));
    B200_CUDA_CHECK(to_f32_launch(P.sell.vals32, static_cast<const double *>(P.sell.vals), P.sell.entries, s));
  }
  return B200_OK;
}

extern "C" b200_status b200_rowblock_spmm(b200_mat A, int bp, int x32, const void *X, const void *Z, void *Y,
                                          double alpha, double shift, double beta, void *stream) {
  B200_ARG_CHECK(A && X && Y && (bp == 64 || bp == 128), "A, X, Y required; bp = 64 or 128");
  B200_ARG_CHECK(A->kind == kMatCsr && A->m == A->n, "the block SpMV needs a square CSR operator");
  B200_ARG_CHECK((((uintptr_t)X | (uintptr_t)Y | (uintptr_t)(Z ? Z : X)) & 15) == 0, "blocks must be 16-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  B200_CHECK(mat_mixed_prepare(A, s));
  const CsrPart &P = A->a;
  const bool vf32 = x32 ? true : P.f32;
  const void *sv = x32 ? (P.f32 ? P.sell.vals : (const void *)P.sell.vals32) : P.sell.vals;
  const void *cv = x32 ? (P.f32 ? P.vals : (const void *)P.vals32) : P.vals;
  B200_CUDA_CHECK(rb_spmm_launch(P.sell, P.rows, P.rowptr, P.colind, cv, sv, vf32, x32 != 0, bp, X, Z, Y, alpha, shift,
                                 beta, s));
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  return B200_OK;
}

cudaError_t b200::mat_spmv_x32(b200_mat A, const float *x, double *y, cudaStream_t stream, const GsState *st,
                               int step) {
  const CsrPart &P = A->a;
  const float *svals = P.f32 ? static_cast<const float *>(P.sell.vals) : P.sell.vals32;
  const float *cvals = P.f32 ? static_cast<const float *>(P.vals) : P.vals32;
  return spmv_sell_launch_x32(P.sell, svals, P.rows, P.sell.rest, P.rowptr, P.colind, cvals, x, y, stream, st, step);
}

cudaError_t b200::mat_spmm(b200_mat A, const double *Y, const double *X, double *Out, int ld, int nb, double alpha,
                           double shift, double beta, cudaStream_t stream) {
  const CsrPart &P = A->a;
  return spmm_sell_launch(P.sell, P.rows, P.rowptr, P.colind, P.vals, P.f32, Y, X, Out, ld, nb, alpha, shift, beta,
                          stream);
}

cudaError_t b200::mat_gershgorin(b200_mat A, double *out, double *work, int work_len, cudaStream_t stream) {
  const CsrPart &P = A->a;
  return gershgorin_launch(P.rows, P.rowptr, P.colind, P.vals, P.f32, out, work, work_len, stream);
}

extern "C" b200_status b200_mat_mult(b200_mat A, const double *x, double *y) {
  B200_ARG_CHECK(A && x && y, "null argument");
  B200_CUDA_CHECK(mat_spmv(A, x, y, A->stream));
  return B200_OK;
}

extern "C" b200_status b200_mat_mult_transpose(b200_mat A, const double *x, double *y) {
  B200_ARG_CHECK(A && x && y, "null argument");
  B200_ARG_CHECK(A->kind == kMatCsr && A->at.rows == A->n, "only a rectangular AIJ matrix stores its transpose");
  B200_CUDA_CHECK(part_spmv(A->at, A->schedule, x, y, A->stream, nullptr, 0));
  return B200_OK;
}

extern "C" b200_status b200_mat_get_size(b200_mat A, int *n, int64_t *nnz) {
  B200_ARG_CHECK(A, "null matrix");
  if (n) *n = A->n;
  if (nnz) *nnz = A->nnz;
  return B200_OK;
}

extern "C" b200_status b200_mat_get_sizes(b200_mat A, int *m, int *n) {
  B200_ARG_CHECK(A, "null matrix");
  if (m) *m = A->m;
  if (n) *n = A->n;
  return B200_OK;
}

extern "C" b200_status b200_mat_norm_inf(b200_mat A, double *nrm) {
  B200_ARG_CHECK(A && nrm, "null argument");
  B200_ARG_CHECK(A->norm_inf >= 0.0, "the infinity norm is known only for matrices created from host arrays");
  *nrm = A->norm_inf;
  return B200_OK;
}

extern "C" b200_status b200_mat_set_spmv_schedule(b200_mat A, int schedule) {
  B200_ARG_CHECK(A && (schedule == B200_SPMV_ROWBLOCK || schedule == B200_SPMV_WARPTILE ||
                       schedule == B200_SPMV_PIPELINED || schedule == B200_SPMV_SELL),
                 "unknown SpMV schedule");
  B200_ARG_CHECK(schedule != B200_SPMV_ROWBLOCK || (A->kind == kMatCsr && !A->a.f32),
                 "the row-block schedule is available for FP64 CSR matrices only");
  B200_ARG_CHECK(A->kind == kMatCsr, "set the schedule on the matrix of a cross shell");
  if (schedule == B200_SPMV_SELL) {
    B200_CHECK(part_build_sell(A->a, nullptr, A->stream));
    if (A->at.rows) B200_CHECK(part_build_sell(A->at, nullptr, A->stream));
  }
  A->schedule = schedule;
  return B200_OK;
}

extern "C" b200_status b200_mat_get_lanes(b200_mat A, int *lanes) {
  B200_ARG_CHECK(A && lanes, "null argument");
  *lanes = A->kind == kMatCross ? A->base->a.lanes : A->a.lanes;
  return B200_OK;
}

// MatLoad: the next Mat object of a PETSc binary file as a square CSR operator
// (storage B200_MAT_OPERATOR) or as a general AIJ matrix with its transpose
// (storage B200_SCALAR_F64 / B200_SCALAR_F32).
extern "C" b200_status b200_mat_load(b200_viewer v, int storage, void *stream, b200_mat *A) {
  B200_ARG_CHECK(v && A, "null argument");
  B200_ARG_CHECK(storage == B200_MAT_OPERATOR || storage == B200_SCALAR_F64 || storage == B200_SCALAR_F32,
                 "unknown storage");
  int classid = 0, m = 0, n = 0;
  int64_t nnz = 0;
  B200_CHECK(b200_viewer_peek(v, &classid, &m, &n, &nnz));
  B200_ARG_CHECK(classid == B200_MAT_FILE_CLASSID, "the next object in the file is not a Mat");
  B200_ARG_CHECK(storage != B200_MAT_OPERATOR || m == n, "an operator must be square");
  std::vector<int> rp((size_t)m + 1), ci((size_t)(nnz > 0 ? nnz : 1));
  std::vector<double> va((size_t)(nnz > 0 ? nnz : 1));
  B200_CHECK(b200_mat_read_csr(v, rp.data(), ci.data(), va.data()));
  if (storage == B200_MAT_OPERATOR) return b200_mat_create_csr(n, nnz, rp.data(), ci.data(), va.data(), stream, A);
  if (storage == B200_SCALAR_F32) {
    std::vector<float> vf(va.begin(), va.end());
    return b200_mat_create_aij(m, n, nnz, rp.data(), ci.data(), vf.data(), B200_SCALAR_F32, stream, A);
  }
  return b200_mat_create_aij(m, n, nnz, rp.data(), ci.data(), va.data(), B200_SCALAR_F64, stream, A);
}

// MatView to a PETSc binary file (FP32-stored values are written widened to double).
extern "C" b200_status b200_mat_view(b200_mat A, b200_viewer v) {
  B200_ARG_CHECK(A && v, "null argument");
  B200_ARG_CHECK(A->kind == kMatCsr, "a cross shell has no stored entries to view");
  const CsrPart &P = A->a;
  std::vector<int> rp((size_t)P.rows + 1), ci((size_t)(P.nnz > 0 ? P.nnz : 1));
  std::vector<double> va((size_t)(P.nnz > 0 ? P.nnz : 1));
  B200_CUDA_CHECK(cudaMemcpyAsync(rp.data(), P.rowptr, sizeof(int) * rp.size(), cudaMemcpyDeviceToHost, A->stream));
  if (P.nnz) {
    B200_CUDA_CHECK(
        cudaMemcpyAsync(ci.data(), P.colind, sizeof(int) * (size_t)P.nnz, cudaMemcpyDeviceToHost, A->stream));
    if (P.f32) {
      std::vector<float> vf((size_t)P.nnz);
      B200_CUDA_CHECK(
          cudaMemcpyAsync(vf.data(), P.vals, sizeof(float) * (size_t)P.nnz, cudaMemcpyDeviceToHost, A->stream));
      B200_CUDA_CHECK(cudaStreamSynchronize(A->stream));
      for (size_t i = 0; i < vf.size(); ++i) va[i] = vf[i];
    } else {
      B200_CUDA_CHECK(
          cudaMemcpyAsync(va.data(), P.vals, sizeof(double) * (size_t)P.nnz, cudaMemcpyDeviceToHost, A->stream));
    }
  }
  B200_CUDA_CHECK(cudaStreamSynchronize(A->stream));
  return b200_mat_write_csr(v, P.rows, P.cols, P.nnz, rp.data(), ci.data(), va.data());
}

extern "C" b200_status b200_mat_destroy(b200_mat A) {
  if (!A) return B200_OK;
  part_free(A->a);
  part_free(A->at);
  dev_free(A->work);
  delete A;
  return B200_OK;
}

extern "C" b200_status b200_csr_spmv(int n, const int *rowptr, const int *colind, const double *vals, const double *x,
                                     double *y, int lanes, void *stream) {
  B200_ARG_CHECK(n >= 0 && rowptr && colind && vals && x && y, "null argument");
  B200_ARG_CHECK(lanes == 1 || lanes == 2 || lanes == 4 || lanes == 8 || lanes == 16 || lanes == 32,
                 "lanes must be a power of two in [1,32]");
  B200_CUDA_CHECK(spmv_launch(n, rowptr, colind, vals, x, y, lanes, (cudaStream_t)stream));
  return B200_OK;
}

// ------------------------------------------------------------------- BV ---
// hpin is written by the host only after the host-to-device copies out of it have run: those
// copies record hpin_ev, and a writer waits for that event instead of draining the stream.
static cudaError_t hpin_acquire(b200_bv bv) { return bv->hpin_ev ? cudaEventSynchronize(bv->hpin_ev) : cudaSuccess; }
static cudaError_t hpin_release(b200_bv bv) {
  if (!bv->hpin_ev) {
    cudaError_t e = cudaEventCreateWithFlags(&bv->hpin_ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
  }
  return cudaEventRecord(bv->hpin_ev, bv->stream);
}

static void bv_free(b200_bv bv) {
  if (!bv) return;
  dev_free(bv->V);
  dev_free(bv->gs.st);
  dev_free(bv->gs.coef);
  dev_free(bv->gs.cnew);
  dev_free(bv->gs.partials);
  dev_free(bv->coefbuf);
  dev_free(bv->hvec);
  dev_free(bv->T);
  dev_free(bv->red);
  dev_free(bv->scal);
  dev_free(bv->qbuf);
  if (bv->hpin_ev) {
    cudaEventSynchronize(bv->hpin_ev);
    cudaEventDestroy(bv->hpin_ev);
  }
  cudaFreeHost(bv->hpin);
  delete bv;
}

// Grow the coefficient staging (device qbuf, pinned hpin) to hold q doubles and the reduction
// workspace to hold red doubles; block operations between BVs of different widths need more
// than a BV's own (m+1)^2.
static b200_status bv_reserve(b200_bv bv, size_t q, size_t red) {
  if (q > bv->qbuf_len || q + 64 > bv->hpin_len) {
    B200_CUDA_CHECK(cudaStreamSynchronize(bv->stream));
    double *nq = nullptr, *nh = nullptr;
    B200_CUDA_CHECK(dev_malloc(&nq, sizeof(double) * q));
    if (cudaMallocHost(&nh, sizeof(double) * (q + 64)) != cudaSuccess) {
      dev_free(nq);
      b200_set_last_error(__FILE__, __LINE__, "pinned host allocation failed");
      return B200_ERR_NOMEM;
    }
    hpin_acquire(bv);
    dev_free(bv->qbuf);
    cudaFreeHost(bv->hpin);
    bv->qbuf = nq;
    bv->hpin = nh;
    bv->qbuf_len = q;
    bv->hpin_len = q + 64;
  }
  if (red > (size_t)bv->red_len) {
    B200_CUDA_CHECK(cudaStreamSynchronize(bv->stream));
    double *nr = nullptr;
    B200_CUDA_CHECK(dev_malloc(&nr, sizeof(double) * red));
    dev_free(bv->red);
    bv->red = nr;
    bv->red_len = (int)red;
  }
  return B200_OK;
}

extern "C" b200_status b200_bv_create(int n, int m, void *stream, b200_bv *out) {
  B200_ARG_CHECK(out && n > 0 && m > 0, "invalid BV sizes");
  B200_ARG_CHECK(m + 1 < kMaxCols, "too many BV columns for the Gram-Schmidt kernels (m <= 253)");
  b200_bv bv = new b200_bv_s;
  bv->n = n;
  bv->m = m;
  bv->ld = ((n + 31) / 32) * 32;
  bv->k = m;
  bv->stream = (cudaStream_t)stream;
  bv->ldc = m + 1;
  bv->ldt = m + 1;
  const int sms = num_sms_host();
  bv->gs.num_sms = sms;
  bv->gs.max_ctas = 2 * sms;  // the FP32-basis passes of the mixed solver run two CTAs per SM
  bv->red_len = sms * 8 > 4096 ? sms * 8 : 4096;
  bv->qbuf_len = (size_t)(m + 1) * (m + 1);
  bv->hpin_len = (size_t)(m + 1) * (m + 1) + 4 * (size_t)(m + 1) + 64;
  bool ok = true;
  // one spare chunk of rows past the last column: the bulk copies of a ragged
  // final chunk round up to 16 bytes
  ok = ok && dev_malloc(&bv->V, sizeof(double) * ((size_t)bv->ld * (m + 1) + 32)) == cudaSuccess;
  ok = ok && dev_malloc(&bv->gs.st, sizeof(GsState)) == cudaSuccess;
  ok = ok && dev_malloc(&bv->gs.coef, sizeof(double) * kMaxCols) == cudaSuccess;
  ok = ok && dev_malloc(&bv->gs.cnew, sizeof(double) * (kMaxCols + 1)) == cudaSuccess;
  ok = ok && dev_malloc(&bv->gs.partials, sizeof(double) * (size_t)(kMaxCols + 1) * 2 * sms) == cudaSuccess;
  ok = ok && dev_malloc(&bv->coefbuf, sizeof(double) * (size_t)bv->ldc * (m + 1)) == cudaSuccess;
  ok = ok && dev_malloc(&bv->hvec, sizeof(double) * (kMaxCols + 1)) == cudaSuccess;
  ok = ok && dev_malloc(&bv->T, sizeof(double) * 2 * (size_t)bv->ldt) == cudaSuccess;
  ok = ok && dev_malloc(&bv->red, sizeof(double) * (size_t)bv->red_len) == cudaSuccess;
  ok = ok && dev_malloc(&bv->scal, sizeof(double) * 16) == cudaSuccess;
  ok = ok && dev_malloc(&bv->qbuf, sizeof(double) * bv->qbuf_len) == cudaSuccess;
  ok = ok && cudaMallocHost(&bv->hpin, sizeof(double) * bv->hpin_len) == cudaSuccess;
  if (!ok) {
    bv_free(bv);
    b200_set_last_error(__FILE__, __LINE__, "device allocation failed for the BV");
    return B200_ERR_NOMEM;
  }
  cudaError_t e = cudaMemsetAsync(bv->V, 0, sizeof(double) * ((size_t)bv->ld * (m + 1) + 32), bv->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(bv->coefbuf, 0, sizeof(double) * (size_t)bv->ldc * (m + 1), bv->stream);
  if (e == cudaSuccess) e = gs_state_reset(bv->gs, bv->eta, bv->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(bv->stream);
  if (e != cudaSuccess) {
    bv_free(bv);
    b200_set_last_error(__FILE__, __LINE__, cudaGetErrorString(e));
    return B200_ERR_CUDA;
  }
  *out = bv;
  return B200_OK;
}

extern "C" b200_status b200_bv_destroy(b200_bv bv) {
  bv_free(bv);
  return B200_OK;
}

extern "C" b200_status b200_bv_get_sizes(b200_bv bv, int *n, int *m, int *ld) {
  B200_ARG_CHECK(bv, "null BV");
  if (n) *n = bv->n;
  if (m) *m = bv->m;
  if (ld) *ld = bv->ld;
  return B200_OK;
}

extern "C" b200_status b200_bv_get_array(b200_bv bv, double **V) {
  B200_ARG_CHECK(bv && V, "null argument");
  *V = bv->V;
  return B200_OK;
}

extern "C" b200_status b200_bv_set_active_columns(b200_bv bv, int l, int k) {
  B200_ARG_CHECK(bv && 0 <= k && k <= bv->m && 0 <= l && l <= k, "active columns out of range");
  bv->l = l;
  bv->k = k;
  return B200_OK;
}

extern "C" b200_status b200_bv_get_active_columns(b200_bv bv, int *l, int *k) {
  B200_ARG_CHECK(bv, "null BV");
  if (l) *l = bv->l;
  if (k) *k = bv->k;
  return B200_OK;
}

extern "C" b200_status b200_bv_set_orthog_eta(b200_bv bv, double eta) {
  B200_ARG_CHECK(bv && eta > 0.0, "eta must be positive");
  bv->eta = eta;
  return B200_OK;
}

extern "C" b200_status b200_bv_set_orthog_block(b200_bv bv, int type) {
  B200_ARG_CHECK(bv, "null BV");
  B200_ARG_CHECK(type >= B200_ORTHOG_BLOCK_GS && type <= B200_ORTHOG_BLOCK_SVQB, "unknown block orthogonalization type");
  bv->orthog_block = type;
  return B200_OK;
}

extern "C" b200_status b200_bv_get_orthog_block(b200_bv bv, int *type) {
  B200_ARG_CHECK(bv && type, "null argument");
  *type = bv->orthog_block;
  return B200_OK;
}


extern "C" b200_status b200_bv_set_column(b200_bv bv, int j, const double *x) {
  B200_ARG_CHECK(bv && x && j >= 0 && j < bv->m, "column index out of range");
  B200_CUDA_CHECK(cudaMemcpyAsync(col(bv, j), x, sizeof(double) * bv->n, cudaMemcpyHostToDevice, bv->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(bv->stream));
  return B200_OK;
}

extern "C" b200_status b200_bv_get_column(b200_bv bv, int j, double *x) {
  B200_ARG_CHECK(bv && x && j >= 0 && j < bv->m, "column index out of range");
  B200_CUDA_CHECK(cudaMemcpyAsync(x, col(bv, j), sizeof(double) * bv->n, cudaMemcpyDeviceToHost, bv->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(bv->stream));
  return B200_OK;
}

extern "C" b200_status b200_bv_copy_vec(b200_bv bv, int j, double *x) {
  B200_ARG_CHECK(bv && x && j >= 0 && j < bv->m, "column index out of range");
  B200_CUDA_CHECK(copy_launch(x, col(bv, j), bv->n, bv->stream));
  return B200_OK;
}

extern "C" b200_status b200_bv_insert_vec(b200_bv bv, int j, const double *x) {
  B200_ARG_CHECK(bv && x && j >= 0 && j < bv->m, "column index out of range");
  B200_CUDA_CHECK(copy_launch(col(bv, j), x, bv->n, bv->stream));
  return B200_OK;
}

// Read back the control block after a synchronisation; map device errors.
static b200_status bv_read_state(b200_bv bv, GsState *out) {
  GsState *h = reinterpret_cast<GsState *>(bv->hpin);
  B200_CUDA_CHECK(cudaMemcpyAsync(h, bv->gs.st, sizeof(GsState), cudaMemcpyDeviceToHost, bv->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(bv->stream));
  *out = *h;
  if (out->err & kDevErrInnerProduct) {
    b200_set_last_error(__FILE__, __LINE__, "invalid inner product (negative self dot product)");
    return B200_ERR_INNER;
  }
  if (out->err) B200_DEV_ERR("a Gram-Schmidt kernel reported a device-side error (bounded wait expired)");
  int perr = 0;
  B200_CUDA_CHECK(panel_gemm_error(&perr, bv->stream));
  if (perr) B200_DEV_ERR("the panel product kernel reported a device-side error (bounded wait expired)");
  return B200_OK;
}

b200_status b200::bv_state(b200_bv bv, GsState *out) { return bv_read_state(bv, out); }

// Orthogonalise column j against columns 0..j-1 (column variant).
b200_status b200::bv_orth_column(b200_bv bv, int j, int normalize, double *H, double *norm, int *lindep) {
  B200_CUDA_CHECK(gs_state_reset(bv->gs, bv->eta, bv->stream));
  GsPassArgs a{};
  a.V = bv->V;
  a.ld = bv->ld;
  a.total_cols = bv->m + 1;
  a.n = bv->n;
  a.jb = j;
  a.wcol = j;
  a.hacc = bv->coefbuf + (size_t)j * bv->ldc;
  a.T = nullptr;
  a.ldt = 0;
  a.step = -1;
  a.normalize = normalize;
  a.column = 1;
  B200_CUDA_CHECK(gs_orthogonalize_launch(a, bv->gs, bv->stream));
  if (H) {
    B200_CUDA_CHECK(cudaMemcpyAsync(bv->hpin + 64, a.hacc, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, bv->stream));
  }
  GsState st;
  B200_CHECK(bv_read_state(bv, &st));
  if (H) memcpy(H, bv->hpin + 64, sizeof(double) * (j + 1));
  if (norm) *norm = st.beta_out;
  if (lindep) *lindep = st.lindep;
  return B200_OK;
}

extern "C" b200_status b200_bv_orthogonalize_column(b200_bv bv, int j, double *H, double *norm, int *lindep) {
  B200_ARG_CHECK(bv && j >= 0 && j < bv->m, "column index out of range");
  return bv_orth_column(bv, j, 0, H, norm, lindep);
}

extern "C" b200_status b200_bv_orthonormalize_column(b200_bv bv, int j, double *norm, int *lindep) {
  B200_ARG_CHECK(bv && j >= 0 && j < bv->m, "column index out of range");
  return bv_orth_column(bv, j, 1, nullptr, norm, lindep);
}

extern "C" b200_status b200_bv_orthogonalize_vec(b200_bv bv, double *v, double *H, double *norm, int *lindep) {
  B200_ARG_CHECK(bv && v, "null argument");
  const int k = bv->k;
  // the vector is staged in the work column (column m) so every bulk copy stays inside the BV storage
  B200_CUDA_CHECK(copy_launch(col(bv, bv->m), v, bv->n, bv->stream));
  B200_CUDA_CHECK(gs_state_reset(bv->gs, bv->eta, bv->stream));
  GsPassArgs a{};
  a.V = bv->V;
  a.ld = bv->ld;
  a.total_cols = bv->m + 1;
  a.n = bv->n;
  a.jb = k;
  a.wcol = bv->m;
  a.hacc = bv->hvec;
  a.step = -1;
  a.normalize = 0;
  a.column = 0;
  B200_CUDA_CHECK(gs_orthogonalize_launch(a, bv->gs, bv->stream));
  B200_CUDA_CHECK(copy_launch(v, col(bv, bv->m), bv->n, bv->stream));
  if (H && k > 0)
    B200_CUDA_CHECK(cudaMemcpyAsync(bv->hpin + 64, bv->hvec, sizeof(double) * k, cudaMemcpyDeviceToHost, bv->stream));
  GsState st;
  B200_CHECK(bv_read_state(bv, &st));
  if (H && k > 0) memcpy(H, bv->hpin + 64, sizeof(double) * k);
  if (norm) *norm = st.beta_out;
  if (lindep) *lindep = st.lindep;
  return B200_OK;
}

// One classical Gram-Schmidt pass with the contract of the BV gramschmidt op
// (include/slepc/private/bvimpl.h:53, used in place of BVOrthogonalizeCGS1, bvorthog.c:91-132):
// c = V^T w with c[jb] = w^T w (BVDotColumnInc / BVDotVec), w -= V c (BVMultColumn / BVMultVec),
// h += c (BV_AddCoefficients), onorm = sqrt(w^T w) before the pass (BV_SquareRoot / BVNormVec),
// norm = sqrt(onorm^2 - c^T c), or the explicit norm of the updated vector when that estimate is
// not positive.  The DOT is the fused pass kernel's plain-dot mode; the update is BVMultVec's kernel.
extern "C" b200_status b200_bv_gram_schmidt(b200_bv bv, int j, double *v, double *h, double *c, double *onorm,
                                            double *norm) {
  B200_ARG_CHECK(bv, "null argument");
  const bool column = v == nullptr;
  const int jb = column ? j : bv->k;
  B200_ARG_CHECK(jb >= 0 && jb < bv->m + (column ? 0 : 1) && (!column || j < bv->m), "column index out of range");
  cudaStream_t s = bv->stream;
  const int wcol = column ? j : bv->m;
  if (!column) B200_CUDA_CHECK(copy_launch(col(bv, bv->m), v, bv->n, s));  // staged in the work column
  double *w = col(bv, wcol);
  GsPassArgs a{};
  a.V = bv->V;
  a.ld = bv->ld;
  a.total_cols = bv->m + 1;
  a.n = bv->n;
  a.jb = jb;
  a.wcol = wcol;
  a.step = -1;
  B200_CUDA_CHECK(gs_dot_launch(a, bv->gs, s));  // cnew[0..jb-1] = V^T w, cnew[jb] = w^T w
  const double *cnew = bv->gs.cnew;
  if (jb > 0) B200_CUDA_CHECK(multvec_launch(bv->V, bv->ld, bv->n, jb, cnew, -1.0, 1.0, w, s));
  if (c) B200_CUDA_CHECK(cudaMemcpyAsync(c, cnew, sizeof(double) * (jb + 1), cudaMemcpyDeviceToDevice, s));
  double *hh = h ? h : bv->coefbuf + (size_t)j * bv->ldc;
  if (jb > 0 && (h || column)) B200_CUDA_CHECK(axmy_launch(hh, cnew, -1.0, jb, s));  // h += c
  if (!column) B200_CUDA_CHECK(copy_launch(v, w, bv->n, s));
  if (!onorm && !norm) return B200_OK;
  B200_CHECK(bv_reserve(bv, 0, 0));
  B200_CUDA_CHECK(cudaMemcpyAsync(bv->hpin + 64, cnew, sizeof(double) * (jb + 1), cudaMemcpyDeviceToHost, s));
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  const double *hc = bv->hpin + 64;
  const double self = hc[jb];
  if (column && !(self > -10.0 * 2.220446049250313e-16)) {  // BV_SafeSqrt
    b200_set_last_error(__FILE__, __LINE__, "invalid inner product (negative self dot product)");
    return B200_ERR_INNER;
  }
  const double beta = self < 0.0 ? 0.0 : std::sqrt(self);
  if (onorm) *onorm = beta;
  if (norm) {
    double sum = 0.0;
    for (int i = 0; i < jb; ++i) sum += hc[i] * hc[i];  // BV_SquareSum
    const double t = beta * beta - sum;
    if (t > 0.0) {
      *norm = std::sqrt(t);
    } else {  // BV_NormVecOrColumn
      double ss = 0.0;
      B200_CUDA_CHECK(sumsq_launch(w, bv->n, bv->scal, bv->red, bv->red_len, s));
      B200_CUDA_CHECK(cudaMemcpyAsync(&ss, bv->scal, sizeof(double), cudaMemcpyDeviceToHost, s));
      B200_CUDA_CHECK(cudaStreamSynchronize(s));
      *norm = std::sqrt(ss);
    }
  }
  return B200_OK;
}

// BVResize (bvbasic.c:338-388, BVResize_Svec svec.c:261-300): new storage of m columns, the first
// min(m, old m) columns copied when copy is set; l and k are clipped to m.
extern "C" b200_status b200_bv_resize(b200_bv bv, int m, int copy) {
  B200_ARG_CHECK(bv && m > 0, "the number of columns must be positive");
  if (m == bv->m) return B200_OK;
  b200_bv nb = nullptr;
  B200_CHECK(b200_bv_create(bv->n, m, bv->stream, &nb));
  if (copy) {
    const int keep = std::min(m, bv->m);
    B200_CUDA_CHECK(cudaMemcpyAsync(nb->V, bv->V, sizeof(double) * (size_t)bv->ld * keep, cudaMemcpyDeviceToDevice,
                                    bv->stream));
  }
  nb->eta = bv->eta;
  nb->orthog_block = bv->orthog_block;
  nb->seed = bv->seed;
  nb->nrand = bv->nrand;
  nb->l = std::min(bv->l, m);
  nb->k = std::min(bv->k, m);
  B200_CUDA_CHECK(cudaStreamSynchronize(bv->stream));
  std::swap(*bv, *nb);  // the caller's handle keeps its identity and gets the new storage
  return b200_bv_destroy(nb);
}

// BVCopy (bvbasic.c:1779-1808, BVCopy_Svec svec.c:233-247): Y(:, Y.l + j) = X(:, X.l + j) for the
// k - l active columns of X; Y needs as many columns from its l.
extern "C" b200_status b200_bv_copy(b200_bv X, b200_bv Y) {
  B200_ARG_CHECK(X && Y && X->n == Y->n, "mismatching local dimension");
  const int nc = X->k - X->l;
  B200_ARG_CHECK(nc <= Y->m - Y->l, "Y has not enough non-leading columns");
  if (X == Y || nc <= 0) return B200_OK;
  B200_CUDA_CHECK(cudaMemcpy2DAsync(col(Y, Y->l), sizeof(double) * Y->ld, col(X, X->l), sizeof(double) * X->ld,
                                    sizeof(double) * X->n, nc, cudaMemcpyDeviceToDevice, X->stream));
  if (Y->stream != X->stream) B200_CUDA_CHECK(cudaStreamSynchronize(X->stream));
  return B200_OK;
}

// BVNormalize (bvglobal.c:829-866) for real scalars (eigi NULL): every active column scaled to unit
// 2-norm (a zero column is left as it is); norms_host (nullable, k - l values) receives the norms.
extern "C" b200_status b200_bv_normalize(b200_bv bv, double *norms_host) {
  B200_ARG_CHECK(bv, "null argument");
  const int nc = bv->k - bv->l;
  if (nc <= 0) return B200_OK;
  std::vector<double> nrm((size_t)nc);
  B200_CHECK(bv_column_norms(bv, nrm.data()));
  for (int i = 0; i < nc; ++i)
    if (nrm[i] != 0.0 && nrm[i] != 1.0) B200_CUDA_CHECK(scale_launch(col(bv, bv->l + i), bv->n, 1.0 / nrm[i], bv->stream));
  if (norms_host) memcpy(norms_host, nrm.data(), sizeof(double) * nc);
  return B200_OK;
}

// BVMultInPlaceHermitianTranspose (bvops.c:268-296) for real scalars: V(:,s:e) = V(:,l:k) Q(s:e,l:k)^T,
// i.e. the in-place product with the transpose of the host matrix Q (leading dimension ldq >= e).
extern "C" b200_status b200_bv_mult_inplace_trans(b200_bv bv, const double *Q, int ldq, int s, int e) {
  B200_ARG_CHECK(bv && Q && 0 <= s && s <= e && e <= bv->m && ldq >= e, "invalid arguments");
  const int k = bv->k;
  std::vector<double> Qt((size_t)k * std::max(e, 1));  // Qt(i, c) = Q(c, i): leading dimension k
  for (int c = s; c < e; ++c)
    for (int i = 0; i < k; ++i) Qt[(size_t)c * k + i] = Q[(size_t)i * ldq + c];
  return b200_bv_mult_inplace(bv, Qt.data(), k, s, e);
}

extern "C" b200_status b200_bv_scale_column(b200_bv bv, int j, double alpha) {
  B200_ARG_CHECK(bv && j < bv->m, "column index out of range");
  if (j < 0) {
    for (int c = bv->l; c < bv->k; ++c) B200_CUDA_CHECK(scale_launch(col(bv, c), bv->n, alpha, bv->stream));
  } else if (alpha != 1.0) {
    B200_CUDA_CHECK(scale_launch(col(bv, j), bv->n, alpha, bv->stream));
  }
  return B200_OK;
}

// BVOrthogonalize_GS without R: every column of [l,k) orthogonalised against all previous columns
// and scaled by 1/norm on the device, the norms recorded on the device and read back once.  A
// dependent column is found only at that read-back, after the later columns have been
// orthogonalised against it, so V(:,l:k) is undefined when B200_ERR_BREAKDOWN is returned (the
// reference stops at the first zero norm, bvorthog.c:546, with the same status).
b200_status b200::bv_orthogonalize_block(b200_bv bv) {
  const int nc = bv->k - bv->l;
  if (nc <= 0) return B200_OK;
  B200_CHECK(bv_reserve(bv, (size_t)3 * nc, 0));
  for (int j = bv->l; j < bv->k; ++j) {
    B200_CUDA_CHECK(gs_state_reset(bv->gs, bv->eta, bv->stream));
    GsPassArgs a{};
    a.V = bv->V;
    a.ld = bv->ld;
    a.total_cols = bv->m + 1;
    a.n = bv->n;
    a.jb = j;
    a.wcol = j;
    a.hacc = bv->coefbuf + (size_t)j * bv->ldc;
    a.step = -1;
    a.normalize = 1;
    a.column = 1;
    B200_CUDA_CHECK(gs_orthogonalize_launch(a, bv->gs, bv->stream));
    B200_CUDA_CHECK(gs_record_launch(bv->gs, bv->qbuf + 3 * (size_t)(j - bv->l), bv->stream));
  }
  B200_CUDA_CHECK(
      cudaMemcpyAsync(bv->hpin, bv->qbuf, sizeof(double) * 3 * (size_t)nc, cudaMemcpyDeviceToHost, bv->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(bv->stream));
  for (int c = 0; c < nc; ++c) {
    const int err = (int)bv->hpin[3 * c + 2];
    if (err & kDevErrInnerProduct) {
      b200_set_last_error(__FILE__, __LINE__, "invalid inner product (negative self dot product)");
      return B200_ERR_INNER;
    }
    if (err) B200_DEV_ERR("a Gram-Schmidt kernel reported a device-side error");
    if (bv->hpin[3 * c] == 0.0) {
      b200_set_last_error(__FILE__, __LINE__, "breakdown in BVOrthogonalize due to a linearly dependent column");
      return B200_ERR_BREAKDOWN;
    }
  }
  return B200_OK;
}

// BVOrthogonalizeVec of `count` device vectors against the active columns of bv, each scaled by
// 1/norm on the device; one read-back at the end.  *breakdown: some vector had norm 0 or was
// linearly dependent (the caller stops, as LOBPCG does).
b200_status b200::bv_orthonormalize_vecs(b200_bv bv, double *const *vecs, int count, int *breakdown) {
  *breakdown = 0;
  if (count <= 0) return B200_OK;
  B200_CHECK(bv_reserve(bv, (size_t)3 * count, 0));
  for (int i = 0; i < count; ++i) {
    B200_CUDA_CHECK(copy_launch(col(bv, bv->m), vecs[i], bv->n, bv->stream));
    B200_CUDA_CHECK(gs_state_reset(bv->gs, bv->eta, bv->stream));
    GsPassArgs a{};
    a.V = bv->V;
    a.ld = bv->ld;
    a.total_cols = bv->m + 1;
    a.n = bv->n;
    a.jb = bv->k;
    a.wcol = bv->m;
    a.hacc = bv->hvec;
    a.step = -1;
    a.normalize = 1;
    a.column = 0;
    B200_CUDA_CHECK(gs_orthogonalize_launch(a, bv->gs, bv->stream));
    B200_CUDA_CHECK(copy_launch(vecs[i], col(bv, bv->m), bv->n, bv->stream));
    B200_CUDA_CHECK(gs_record_launch(bv->gs, bv->qbuf + 3 * (size_t)i, bv->stream));
  }
  B200_CUDA_CHECK(
      cudaMemcpyAsync(bv->hpin, bv->qbuf, sizeof(double) * 3 * (size_t)count, cudaMemcpyDeviceToHost, bv->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(bv->stream));
  for (int i = 0; i < count; ++i) {
    const int err = (int)bv->hpin[3 * i + 2];
    if (err) B200_DEV_ERR("a Gram-Schmidt kernel reported a device-side error");
    if (!(bv->hpin[3 * i] > 0.0) || bv->hpin[3 * i + 1] != 0.0) *breakdown = 1;
  }
  return B200_OK;
}

// Norms of columns [l,k) into host nrm[0..k-l), one reduction and one read-back.
b200_status b200::bv_column_norms(b200_bv bv, double *nrm) {
  const int nc = bv->k - bv->l;
  if (nc <= 0) return B200_OK;
  B200_CHECK(bv_reserve(bv, (size_t)nc, (size_t)nc * num_sms_host()));
  B200_CUDA_CHECK(colnorm_launch(col(bv, bv->l), bv->ld, bv->n, nc, bv->qbuf, bv->red, bv->red_len, bv->stream));
  B200_CUDA_CHECK(cudaMemcpyAsync(bv->hpin, bv->qbuf, sizeof(double) * nc, cudaMemcpyDeviceToHost, bv->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(bv->stream));
  memcpy(nrm, bv->hpin, sizeof(double) * nc);
  return B200_OK;
}

// BVOrthogonalize_Chol (bvorthog.c:595-613) and BVOrthogonalize_SVQB (:665-684) on the active
// columns [l,k): one Gram-Schmidt pass against the leading columns (BVOrthogonalize_BlockGS,
// :492-501: C = V1^T V2, V2 -= V1 C), the Gram matrix G = V2^T V2 on the device, its
// factorisation on the host in FP64 (BVMatCholInv_LAPACK_Private, bvlapack.c:136-213: dpotrf "U",
// once more with 50 eps on the diagonal if it fails, dtrtri; BVMatSVQB_LAPACK_Private, :261-340:
// D = diag(G)^{-1/2}, dsyev "V" "L" of D G D = U Lambda U^T, S = D U Lambda^{-1/2}), then
// V2 := V2 S with the row-panel in-place product.  Six kernel launches and one read-back instead
// of a Gram-Schmidt sweep per column.  R (nullable): R(0:l, l:k) = C and R(l:k, l:k) = the
// Cholesky factor or Lambda^{1/2} U^T D^{-1}, so that V_in = V_out R.  A zero column or a
// non-positive eigenvalue of the SVQB Gram matrix (a numerically rank-deficient block, for which
// the reference would divide by zero or take the square root of a negative number) is reported as
// a breakdown.
// The device half: C, V2 -= V1 C and G queued on the stream with their read-back into bv->hpin.
static b200_status bv_gram_enqueue(b200_bv bv) {
  const int l = bv->l, k = bv->k, nc = k - l, n = bv->n, ld = bv->ld;
  if (nc <= 0) return B200_OK;
  const size_t nC = (size_t)l * nc, nG = (size_t)nc * nc;
  const int cps_c = dot_ctas_per_sm(nc, l), cps_g = dot_ctas_per_sm(nc, nc);
  B200_CHECK(bv_reserve(bv, nC + nG, std::max(nC * cps_c, nG * cps_g) * num_sms_host()));
  cudaStream_t s = bv->stream;
  double *Cdev = bv->qbuf, *Gdev = bv->qbuf + nC;
  if (l > 0) {
    B200_CUDA_CHECK(dot_launch(col(bv, l), ld, nc, bv->V, ld, l, n, Cdev, l, bv->red, bv->red_len, s, cps_c));
    B200_CUDA_CHECK(mult_launch(col(bv, l), ld, bv->V, ld, n, l, nc, Cdev, l, -1.0, 1.0, s));
  }
  B200_CUDA_CHECK(
      dot_launch(col(bv, l), ld, nc, col(bv, l), ld, nc, n, Gdev, nc, bv->red, bv->red_len, s, cps_g));
  B200_CUDA_CHECK(cudaMemcpyAsync(bv->hpin, bv->qbuf, sizeof(double) * (nC + nG), cudaMemcpyDeviceToHost, s));
  return B200_OK;
}

// The host half, after a synchronisation of the stream: factor G, then queue V2 := V2 S.
static b200_status bv_gram_finish(b200_bv bv, double *R, int ldr) {
  const int l = bv->l, k = bv->k, nc = k - l, n = bv->n, ld = bv->ld;
  if (nc <= 0) return B200_OK;
  const size_t nC = (size_t)l * nc, nG = (size_t)nc * nc;
  cudaStream_t s = bv->stream;
  double *Gdev = bv->qbuf + nC;
  std::vector<double> C(bv->hpin, bv->hpin + nC), G(bv->hpin + nC, bv->hpin + nC + nG), Rf(nG, 0.0), S(nG, 0.0);
  int info = 0;
  if (bv->orthog_block == B200_ORTHOG_BLOCK_CHOL) {
    Rf = G;
    scipy_dpotrf_("U", &nc, Rf.data(), &nc, &info, 1);
    if (info) {
      Rf = G;
      for (int i = 0; i < nc; ++i) Rf[(size_t)i * nc + i] += 50.0 * 2.220446049250313e-16;
      info = 0;
      scipy_dpotrf_("U", &nc, Rf.data(), &nc, &info, 1);
      if (info) {
        b200_set_last_error(__FILE__, __LINE__, "LAPACK dpotrf failed in BVOrthogonalize (Cholesky)");
        return B200_ERR_LAPACK;
      }
    }
    for (int j = 0; j < nc; ++j)
      for (int i = j + 1; i < nc; ++i) Rf[(size_t)j * nc + i] = 0.0;
    S = Rf;
    scipy_dtrtri_("U", "N", &nc, S.data(), &nc, &info, 1, 1);
    if (info) {
      b200_set_last_error(__FILE__, __LINE__, "LAPACK dtrtri failed in BVOrthogonalize (Cholesky)");
      return B200_ERR_LAPACK;
    }
  } else {
    std::vector<double> D(nc), eig(nc);
    for (int i = 0; i < nc; ++i) {
      if (!(G[(size_t)i * nc + i] > 0.0)) {
        b200_set_last_error(__FILE__, __LINE__, "breakdown in BVOrthogonalize (SVQB): zero column");
        return B200_ERR_BREAKDOWN;
      }
      D[i] = 1.0 / std::sqrt(G[(size_t)i * nc + i]);
    }
    for (int j = 0; j < nc; ++j)
      for (int i = 0; i < nc; ++i) S[(size_t)j * nc + i] = G[(size_t)j * nc + i] * D[i] * D[j];
    int lwork = -1;
    double q = 0.0;
    scipy_dsyev_("V", "L", &nc, S.data(), &nc, eig.data(), &q, &lwork, &info, 1, 1);
    lwork = std::max(1, (int)q);
    std::vector<double> work(lwork);
    scipy_dsyev_("V", "L", &nc, S.data(), &nc, eig.data(), work.data(), &lwork, &info, 1, 1);
    if (info) {
      b200_set_last_error(__FILE__, __LINE__, "LAPACK dsyev failed in BVOrthogonalize (SVQB)");
      return B200_ERR_LAPACK;
    }
    for (int i = 0; i < nc; ++i)
      if (!(eig[i] > 0.0)) {
        b200_set_last_error(__FILE__, __LINE__, "breakdown in BVOrthogonalize (SVQB): rank-deficient block");
        return B200_ERR_BREAKDOWN;
      }
    for (int j = 0; j < nc; ++j)
      for (int i = 0; i < nc; ++i) Rf[(size_t)j * nc + i] = S[(size_t)i * nc + j] * std::sqrt(eig[i]) / D[j];
    for (int j = 0; j < nc; ++j)
      for (int i = 0; i < nc; ++i) S[(size_t)j * nc + i] *= D[i] / std::sqrt(eig[j]);
  }
  B200_CUDA_CHECK(hpin_acquire(bv));
  memcpy(bv->hpin, S.data(), sizeof(double) * nG);
  B200_CUDA_CHECK(cudaMemcpyAsync(Gdev, bv->hpin, sizeof(double) * nG, cudaMemcpyHostToDevice, s));
  B200_CUDA_CHECK(hpin_release(bv));
  B200_CUDA_CHECK(multinplace_launch(bv->V, ld, n, l, k, Gdev, nc, l, k, s));
  if (R) {
    for (int j = 0; j < nc; ++j) {
      for (int i = 0; i < l; ++i) R[i + (size_t)(l + j) * ldr] = C[i + (size_t)j * l];
      for (int i = 0; i < nc; ++i) R[l + i + (size_t)(l + j) * ldr] = Rf[i + (size_t)j * nc];
    }
  }
  return B200_OK;
}

static b200_status bv_orthogonalize_gram(b200_bv bv, double *R, int ldr) {
  B200_CHECK(bv_gram_enqueue(bv));
  B200_CUDA_CHECK(cudaStreamSynchronize(bv->stream));
  return bv_gram_finish(bv, R, ldr);
}

// BVOrthogonalize_TSQR / _TSQRCHOL (bvorthog.c:615-660) on one process: block Gram-Schmidt
// against the leading l columns (BVOrthogonalize_BlockGS, bvorthog.c:492-502), then the
// Householder QR of V(:, l:k) on the device (bvlapack.c:347-440 with one rank: geqrf + orgqr; for
// TSQRCHOL only R, from a copy, then V(:, l:k) := V(:, l:k) R^{-1} as BVMatTriInv_LAPACK_Private
// and BVMultInPlace do).  R(0:l, l:k) holds the Gram-Schmidt coefficients, R(l:k, l:k) the
// triangular factor with LAPACK's signs.
static b200_status bv_orthogonalize_tsqr(b200_bv bv, double *R, int ldr) {
  const int l = bv->l, k = bv->k, nc = k - l, n = bv->n, ld = bv->ld;
  if (nc <= 0) return B200_OK;
  if (n < nc) {
    b200_set_last_error(__FILE__, __LINE__, "TSQR needs at least as many rows as active columns");
    return B200_ERR_SUP;
  }
  const bool chol = bv->orthog_block == B200_ORTHOG_BLOCK_TSQRCHOL;
  cudaStream_t s = bv->stream;
  std::vector<double> C((size_t)l * nc);
  if (l > 0) {
    const size_t nC = (size_t)l * nc;
    const int cps_c = dot_ctas_per_sm(nc, l);
    B200_CHECK(bv_reserve(bv, nC, nC * cps_c * num_sms_host()));
    B200_CUDA_CHECK(dot_launch(col(bv, l), ld, nc, bv->V, ld, l, n, bv->qbuf, l, bv->red, bv->red_len, s, cps_c));
    B200_CUDA_CHECK(mult_launch(col(bv, l), ld, bv->V, ld, n, l, nc, bv->qbuf, l, -1.0, 1.0, s));
    B200_CUDA_CHECK(cudaMemcpyAsync(C.data(), bv->qbuf, sizeof(double) * nC, cudaMemcpyDeviceToHost, s));
  }
  const size_t wlen = (size_t)householder_qr_parts(n) * (nc + 1) + 3 * (size_t)nc;
  double *work = nullptr, *copy = nullptr;
  B200_CUDA_CHECK(dev_malloc(&work, sizeof(double) * wlen));
  double *tau = work + (wlen - 2 * (size_t)nc), *scale = work + (wlen - (size_t)nc);
  if (chol && dev_malloc(&copy, sizeof(double) * (size_t)ld * nc) != cudaSuccess) {
    dev_free(work);
    b200_set_last_error(__FILE__, __LINE__, "device allocation failed for the TSQRCHOL copy");
    return B200_ERR_NOMEM;
  }
  double *X = chol ? copy : col(bv, l);
  cudaError_t e = cudaSuccess;
  if (chol) e = cudaMemcpyAsync(copy, col(bv, l), sizeof(double) * (size_t)ld * nc, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = householder_qr_launch(X, ld, n, nc, tau, scale, work, s);
  std::vector<double> Rf((size_t)nc * nc, 0.0);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(Rf.data(), sizeof(double) * nc, X, sizeof(double) * ld, sizeof(double) * nc, nc,
                          cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && !chol) e = householder_q_launch(X, ld, n, nc, tau, work, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  dev_free(copy);
  dev_free(work);
  if (e != cudaSuccess) {
    b200_set_last_error(__FILE__, __LINE__, cudaGetErrorString(e));
    return B200_ERR_CUDA;
  }
  for (int j = 0; j < nc; ++j)
    for (int i = j + 1; i < nc; ++i) Rf[(size_t)j * nc + i] = 0.0;
  if (chol) {
    std::vector<double> S = Rf;
    int info = 0;
    scipy_dtrtri_("U", "N", &nc, S.data(), &nc, &info, 1, 1);
    if (info) {
      b200_set_last_error(__FILE__, __LINE__, "LAPACK dtrtri failed in BVOrthogonalize (TSQRCHOL)");
      return B200_ERR_LAPACK;
    }
    B200_CHECK(bv_reserve(bv, (size_t)nc * nc, 0));
    B200_CUDA_CHECK(hpin_acquire(bv));
    memcpy(bv->hpin, S.data(), sizeof(double) * (size_t)nc * nc);
    B200_CUDA_CHECK(cudaMemcpyAsync(bv->qbuf, bv->hpin, sizeof(double) * (size_t)nc * nc, cudaMemcpyHostToDevice, s));
    B200_CUDA_CHECK(hpin_release(bv));
    B200_CUDA_CHECK(multinplace_launch(bv->V, ld, n, l, k, bv->qbuf, nc, l, k, s));
  }
  if (R) {
    for (int j = 0; j < nc; ++j) {
      for (int i = 0; i < l; ++i) R[i + (size_t)(l + j) * ldr] = C[i + (size_t)j * l];
      for (int i = 0; i < nc; ++i) R[l + i + (size_t)(l + j) * ldr] = Rf[i + (size_t)j * nc];
    }
  }
  return B200_OK;
}

namespace b200 {
b200_status bv_orthogonalize_pair(b200_bv a, b200_bv b) {
  B200_ARG_CHECK(a && b && a != b, "invalid BVOrthogonalize pair");
  auto is_gram = [](int t) { return t == B200_ORTHOG_BLOCK_CHOL || t == B200_ORTHOG_BLOCK_SVQB; };
  const bool gram = is_gram(a->orthog_block) && is_gram(b->orthog_block);
  if (!gram || a->stream != b->stream) {
    B200_CHECK(b200_bv_orthogonalize(a, nullptr, 0));
    return b200_bv_orthogonalize(b, nullptr, 0);
  }
  B200_CHECK(bv_gram_enqueue(a));
  B200_CHECK(bv_gram_enqueue(b));
  B200_CUDA_CHECK(cudaStreamSynchronize(a->stream));
  B200_CHECK(bv_gram_finish(a, nullptr, 0));
  return bv_gram_finish(b, nullptr, 0);
}
}  // namespace b200

extern "C" b200_status b200_bv_orthogonalize(b200_bv bv, double *R, int ldr) {
  B200_ARG_CHECK(bv && (!R || ldr >= bv->k), "R leading dimension too small");
  if (bv->orthog_block == B200_ORTHOG_BLOCK_TSQR || bv->orthog_block == B200_ORTHOG_BLOCK_TSQRCHOL)
    return bv_orthogonalize_tsqr(bv, R, ldr);
  if (bv->orthog_block != B200_ORTHOG_BLOCK_GS) return bv_orthogonalize_gram(bv, R, ldr);
  if (!R) return bv_orthogonalize_block(bv);
  for (int j = bv->l; j < bv->k; ++j) {
    double norm = 0.0;
    std::vector<double> H(j + 1);
    B200_CHECK(bv_orth_column(bv, j, 0, R ? H.data() : nullptr, &norm, nullptr));
    if (norm == 0.0) {
      b200_set_last_error(__FILE__, __LINE__, "breakdown in BVOrthogonalize due to a linearly dependent column");
      return B200_ERR_BREAKDOWN;
    }
    if (R) {
      for (int i = 0; i < j; ++i) R[i + (size_t)j * ldr] = H[i];
      R[j + (size_t)j * ldr] = norm;
    }
    B200_CHECK(b200_bv_scale_column(bv, j, 1.0 / norm));
  }
  return B200_OK;
}

static b200_status bv_multinplace_dev(b200_bv bv, const double *Qdev_ls, int ldq, int s, int e) {
  if (s >= e || bv->k <= bv->l) return B200_OK;
  B200_CUDA_CHECK(multinplace_launch(bv->V, bv->ld, bv->n, bv->l, bv->k, Qdev_ls, ldq, s, e, bv->stream));
  return B200_OK;
}

extern "C" b200_status b200_bv_mult_inplace(b200_bv bv, const double *Q, int ldq, int s, int e) {
  B200_ARG_CHECK(bv && Q && ldq >= bv->k, "invalid Q");
  B200_ARG_CHECK(s >= bv->l && s <= bv->m && e >= bv->l && e <= bv->m, "s/e out of range");
  if (s >= e) return B200_OK;
  const int kq = bv->k - bv->l, nc = e - s;
  B200_CHECK(bv_reserve(bv, (size_t)kq * nc, 0));
  // pack Q(l:k, s:e) into pinned memory, then one host-to-device copy
  B200_CUDA_CHECK(hpin_acquire(bv));
  for (int j = 0; j < nc; ++j)
    memcpy(bv->hpin + (size_t)j * kq, Q + (size_t)bv->l + (size_t)(s + j) * ldq, sizeof(double) * kq);
  B200_CUDA_CHECK(
      cudaMemcpyAsync(bv->qbuf, bv->hpin, sizeof(double) * (size_t)kq * nc, cudaMemcpyHostToDevice, bv->stream));
  B200_CUDA_CHECK(hpin_release(bv));
  return bv_multinplace_dev(bv, bv->qbuf, kq, s, e);
}

extern "C" b200_status b200_bv_mult_inplace_device(b200_bv bv, const double *Q, int ldq, int s, int e) {
  B200_ARG_CHECK(bv && Q && ldq >= bv->k, "invalid Q");
  B200_ARG_CHECK(s >= bv->l && s <= bv->m && e >= bv->l && e <= bv->m, "s/e out of range");
  return bv_multinplace_dev(bv, Q + (size_t)bv->l + (size_t)s * ldq, ldq, s, e);
}

extern "C" b200_status b200_bv_mult(b200_bv Y, double alpha, double beta, b200_bv X, const double *Q, int ldq) {
  B200_ARG_CHECK(X && Y && X != Y && Q && X->n == Y->n, "invalid BVMult arguments");
  const int nx = X->k - X->l, ny = Y->k - Y->l;
  B200_ARG_CHECK(ldq >= X->k, "Q leading dimension too small");
  if (ny <= 0) return B200_OK;
  B200_CHECK(bv_reserve(Y, (size_t)nx * ny, 0));
  B200_CUDA_CHECK(hpin_acquire(Y));
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) Y->hpin[i + (size_t)j * nx] = Q[(size_t)(X->l + i) + (size_t)(Y->l + j) * ldq];
  B200_CUDA_CHECK(
      cudaMemcpyAsync(Y->qbuf, Y->hpin, sizeof(double) * (size_t)nx * ny, cudaMemcpyHostToDevice, Y->stream));
  B200_CUDA_CHECK(hpin_release(Y));
  B200_CUDA_CHECK(mult_launch(col(Y, Y->l), Y->ld, col(X, X->l), X->ld, X->n, nx, ny, Y->qbuf, nx, alpha, beta, Y->stream));
  return B200_OK;
}

extern "C" b200_status b200_bv_mult_vec(b200_bv X, double alpha, double beta, double *y, const double *q) {
  B200_ARG_CHECK(X && y && (q || X->k == X->l), "null argument");
  const int k = X->k - X->l;
  B200_CUDA_CHECK(cudaStreamSynchronize(X->stream));
  if (k > 0) memcpy(X->hpin, q, sizeof(double) * k);
  B200_CUDA_CHECK(cudaMemcpyAsync(X->scal, X->hpin, sizeof(double) * (k > 0 ? k : 1), cudaMemcpyHostToDevice, X->stream));
  if (k > 16) {
    B200_ARG_CHECK((size_t)k <= X->qbuf_len, "too many columns");
    B200_CUDA_CHECK(cudaMemcpyAsync(X->qbuf, X->hpin, sizeof(double) * k, cudaMemcpyHostToDevice, X->stream));
  }
  B200_CUDA_CHECK(multvec_launch(col(X, X->l), X->ld, X->n, k, k > 16 ? X->qbuf : X->scal, alpha, beta, y, X->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(X->stream));
  return B200_OK;
}

extern "C" b200_status b200_bv_dot(b200_bv X, b200_bv Y, double *M, int ldm) {
  B200_ARG_CHECK(X && Y && M && X->n == Y->n, "invalid BVDot arguments");
  const int nx = X->k - X->l, ny = Y->k - Y->l;
  B200_ARG_CHECK(ldm >= Y->k, "M leading dimension too small");
  if (nx <= 0 || ny <= 0) return B200_OK;
  const int cps = dot_ctas_per_sm(nx, ny);
  B200_CHECK(bv_reserve(X, (size_t)nx * ny, (size_t)nx * ny * num_sms_host() * cps));
  B200_CUDA_CHECK(dot_launch(col(X, X->l), X->ld, nx, col(Y, Y->l), Y->ld, ny, X->n, X->qbuf, ny, X->red, X->red_len,
                             X->stream, cps));
  B200_CUDA_CHECK(
      cudaMemcpyAsync(X->hpin, X->qbuf, sizeof(double) * (size_t)nx * ny, cudaMemcpyDeviceToHost, X->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(X->stream));
  for (int j = 0; j < nx; ++j)
    for (int i = 0; i < ny; ++i) M[(size_t)(Y->l + i) + (size_t)(X->l + j) * ldm] = X->hpin[i + (size_t)j * ny];
  return B200_OK;
}

namespace b200 {
b200_status bv_dot_pair(b200_bv W, b200_bv Z, double *MA, double *MB, int ldm) {
  B200_ARG_CHECK(W && Z && MA && MB && W->n == Z->n, "invalid BVDot pair arguments");
  const int nc = Z->k - Z->l;
  B200_ARG_CHECK(W->k - W->l == nc && ldm >= Z->k && ldm >= W->k, "BVDot pair: column ranges differ");
  if (nc <= 0) return B200_OK;
  const size_t sq = (size_t)nc * nc;
  const int cps = dot_ctas_per_sm(nc, nc);
  B200_CHECK(bv_reserve(Z, 2 * sq, 2 * sq * num_sms_host() * cps));
  cudaError_t e = dot_dual_launch(col(W, W->l), W->ld, col(Z, Z->l), Z->ld, nc, Z->n, Z->qbuf, Z->red, Z->red_len,
                                  Z->stream, cps);
  if (e == cudaErrorNotSupported) {  // more than 64 columns: the two products one after the other
    e = dot_launch(col(W, W->l), W->ld, nc, col(Z, Z->l), Z->ld, nc, Z->n, Z->qbuf, nc, Z->red, Z->red_len, Z->stream,
                   cps);
    if (e == cudaSuccess)
      e = dot_launch(col(Z, Z->l), Z->ld, nc, col(Z, Z->l), Z->ld, nc, Z->n, Z->qbuf + sq, nc, Z->red, Z->red_len,
                     Z->stream, cps);
  }
  B200_CUDA_CHECK(e);
  B200_CUDA_CHECK(cudaMemcpyAsync(Z->hpin, Z->qbuf, sizeof(double) * 2 * sq, cudaMemcpyDeviceToHost, Z->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(Z->stream));
  for (int j = 0; j < nc; ++j)
    for (int i = 0; i < nc; ++i) {
      MA[(size_t)(Z->l + i) + (size_t)(W->l + j) * ldm] = Z->hpin[i + (size_t)j * nc];
      MB[(size_t)(Z->l + i) + (size_t)(Z->l + j) * ldm] = Z->hpin[sq + i + (size_t)j * nc];
    }
  return B200_OK;
}
}  // namespace b200

extern "C" b200_status b200_bv_dot_vec(b200_bv X, const double *y, double *q) {
  B200_ARG_CHECK(X && y && q, "null argument");
  const int k = X->k - X->l;
  if (k <= 0) return B200_OK;
  B200_CUDA_CHECK(copy_launch(col(X, X->m), y, X->n, X->stream));
  GsPassArgs a{};
  a.V = col(X, X->l);
  a.ld = X->ld;
  a.total_cols = X->m + 1 - X->l;
  a.n = X->n;
  a.jb = k;
  a.wcol = X->m - X->l;
  a.step = -1;
  B200_CUDA_CHECK(gs_dot_launch(a, X->gs, X->stream));
  B200_CUDA_CHECK(cudaMemcpyAsync(X->hpin, X->gs.cnew, sizeof(double) * k, cudaMemcpyDeviceToHost, X->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(X->stream));
  memcpy(q, X->hpin, sizeof(double) * k);
  return B200_OK;
}

static b200_status bv_sumsq(b200_bv bv, const double *x, long long len, double *out) {
  B200_CUDA_CHECK(sumsq_launch(x, len, bv->scal, bv->red, bv->red_len, bv->stream));
  B200_CUDA_CHECK(cudaMemcpyAsync(bv->hpin, bv->scal, sizeof(double), cudaMemcpyDeviceToHost, bv->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(bv->stream));
  *out = bv->hpin[0];
  return B200_OK;
}

extern "C" b200_status b200_bv_norm_column(b200_bv bv, int j, double *nrm) {
  B200_ARG_CHECK(bv && nrm && j >= 0 && j < bv->m, "column index out of range");
  double s = 0.0;
  B200_CHECK(bv_sumsq(bv, col(bv, j), bv->n, &s));
  *nrm = std::sqrt(s);
  return B200_OK;
}

extern "C" b200_status b200_bv_norm(b200_bv bv, double *nrm) {
  B200_ARG_CHECK(bv && nrm, "null argument");
  double tot = 0.0;
  for (int c = bv->l; c < bv->k; ++c) {
    double s = 0.0;
    B200_CHECK(bv_sumsq(bv, col(bv, c), bv->n, &s));
    tot += s;
  }
  *nrm = std::sqrt(tot);
  return B200_OK;
}

extern "C" b200_status b200_bv_copy_column(b200_bv bv, int j, int i) {
  B200_ARG_CHECK(bv && j >= 0 && j < bv->m && i >= 0 && i < bv->m, "column index out of range");
  if (i == j) return B200_OK;
  B200_CUDA_CHECK(copy_launch(col(bv, i), col(bv, j), bv->n, bv->stream));
  return B200_OK;
}

extern "C" b200_status b200_bv_mat_mult_column(b200_bv bv, b200_mat A, int j) {
  B200_ARG_CHECK(bv && A && A->n == bv->n && j >= 0 && j + 1 < bv->m, "invalid BVMatMultColumn arguments");
  B200_CUDA_CHECK(mat_spmv(A, col(bv, j), col(bv, j + 1), bv->stream));
  return B200_OK;
}

// BVMatMult (bvops.c:692-730) with the matrix-product path of BVMatMult_Svec (svec.c:203-219):
// Y(:, Y.l + j) = A V(:, V.l + j) for the active columns.  A square CSR operator takes the block
// SpMV (the matrix read once for all columns); other operators go column by column.
b200_status b200::bv_mat_mult(b200_bv V, b200_mat A, b200_bv Y) {
  const int nc = V->k - V->l;
  if (nc <= 0) return B200_OK;
  if (A->kind == kMatCsr && A->m == A->n && V->ld == Y->ld && A->a.sell_ready) {
    const CsrPart &P = A->a;
    B200_CUDA_CHECK(spmm_sell_launch(P.sell, P.rows, P.rowptr, P.colind, P.vals, P.f32, col(V, V->l), nullptr,
                                     col(Y, Y->l), V->ld, nc, 1.0, 0.0, 0.0, Y->stream));
    return B200_OK;
  }
  for (int j = 0; j < nc; ++j) B200_CUDA_CHECK(mat_spmv(A, col(V, V->l + j), col(Y, Y->l + j), Y->stream));
  return B200_OK;
}

extern "C" b200_status b200_bv_mat_mult(b200_bv V, b200_mat A, b200_bv Y) {
  B200_ARG_CHECK(V && A && Y && V != Y, "invalid BVMatMult arguments (V and Y must differ)");
  B200_ARG_CHECK(A->n == V->n && A->m == Y->n, "mismatching dimensions of A, V and Y");
  B200_ARG_CHECK(V->k - V->l == Y->k - Y->l, "V and Y must have the same number of active columns");
  return bv_mat_mult(V, A, Y);
}

// Timing of a Lanczos run (optional): event pairs around each SpMV and each column orthogonalisation.
struct RunTimer {
  bool on = false;
  std::vector<cudaEvent_t> ev;
  size_t used = 0;
  double ms_spmv = 0.0, ms_orth = 0.0;
  void reserve(size_t count) {
    while (ev.size() < count) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) break;
      ev.push_back(e);
    }
  }
  cudaEvent_t next() { return used < ev.size() ? ev[used++] : nullptr; }
  ~RunTimer() {
    for (auto e : ev) cudaEventDestroy(e);
  }
};

// BVMatLanczos: steps j = k..m-1 enqueued back to back; one synchronisation at the end.
static b200_status bv_lanczos(b200_bv bv, b200_mat A, int k, int *m, double *alpha, double *beta_h, double *beta,
                              int *breakdown, RunTimer *timer, GsState *st_out) {
  const int m0 = *m;
  B200_CUDA_CHECK(gs_state_reset(bv->gs, bv->eta, bv->stream));
  const bool timing = timer && timer->on;
  if (timing) {
    timer->reserve((size_t)4 * (m0 - k) + 4);
    timer->used = 0;
  }
  for (int j = k; j < m0; ++j) {
    cudaEvent_t e0 = timing ? timer->next() : nullptr, e1 = timing ? timer->next() : nullptr;
    cudaEvent_t e2 = timing ? timer->next() : nullptr, e3 = timing ? timer->next() : nullptr;
    if (e0) cudaEventRecord(e0, bv->stream);
    B200_CUDA_CHECK(mat_spmv(A, col(bv, j), col(bv, j + 1), bv->stream, bv->gs.st, j));
    if (e1) cudaEventRecord(e1, bv->stream);
    GsPassArgs a{};
    a.V = bv->V;
    a.ld = bv->ld;
    a.total_cols = bv->m + 1;
    a.n = bv->n;
    a.jb = j + 1;
    a.wcol = j + 1;
    a.hacc = bv->coefbuf + (size_t)(j + 1) * bv->ldc;
    a.T = bv->T;
    a.ldt = bv->ldt;
    a.step = j;
    a.normalize = 1;
    a.column = 1;
    if (e2) cudaEventRecord(e2, bv->stream);
    B200_CUDA_CHECK(gs_orthogonalize_launch(a, bv->gs, bv->stream));
    if (e3) cudaEventRecord(e3, bv->stream);
  }
  // one device-to-host copy of T and of the control block
  double *hT = bv->hpin + 64;
  B200_CUDA_CHECK(cudaMemcpyAsync(hT, bv->T, sizeof(double) * 2 * (size_t)bv->ldt, cudaMemcpyDeviceToHost, bv->stream));
  GsState st;
  B200_CHECK(bv_read_state(bv, &st));
  if (st_out) *st_out = st;
  int mm = m0;
  int bd = 0;
  if (st.halt) {
    mm = st.halt_step + 1;
    bd = 1;
  }
  for (int j = k; j < mm; ++j) {
    if (alpha) alpha[j] = hT[j];
    if (beta_h) beta_h[j] = hT[bv->ldt + j];
  }
  *m = mm;
  if (beta) *beta = st.beta_out;
  if (breakdown) *breakdown = bd;
  if (timing) {
    for (int j = k; j < m0; ++j) {
      const size_t base = (size_t)4 * (j - k);
      if (base + 3 >= timer->ev.size()) break;
      float t = 0.f;
      if (cudaEventElapsedTime(&t, timer->ev[base], timer->ev[base + 1]) == cudaSuccess) timer->ms_spmv += t;
      if (cudaEventElapsedTime(&t, timer->ev[base + 2], timer->ev[base + 3]) == cudaSuccess) timer->ms_orth += t;
    }
  }
  return B200_OK;
}

extern "C" b200_status b200_bv_mat_lanczos(b200_bv bv, b200_mat A, int k, int *m, double *alpha, double *beta_h,
                                           double *beta, int *breakdown) {
  B200_ARG_CHECK(bv && A && m && A->n == bv->n, "invalid BVMatLanczos arguments");
  B200_ARG_CHECK(k >= 0 && *m > k && *m < bv->m, "k/m out of range (need k < m < columns)");
  return bv_lanczos(bv, A, k, m, alpha, beta_h, beta, breakdown, nullptr, nullptr);
}

// ------------------------------------------------------------------ EPS ---
extern "C" b200_status b200_eps_create(void *stream, b200_eps *eps) {
  B200_ARG_CHECK(eps, "null argument");
  b200_eps E = new b200_eps_s;
  E->stream = (cudaStream_t)stream;
  *eps = E;
  return B200_OK;
}

extern "C" b200_status b200_eps_destroy(b200_eps eps) {
  if (!eps) return B200_OK;
  b200_bv_destroy(eps->V);
  dev_free(eps->resid_buf);
  dev_free(eps->op_buf);
  dev_free(eps->dinv);
  if (eps->rb32 || eps->rb64 || eps->mred) cudaStreamSynchronize(eps->stream);  // no kernel still reads them
  if (eps->rb32) pool_free(eps->rb32, eps->stream);
  if (eps->rb64) pool_free(eps->rb64, eps->stream);
  if (eps->mred) pool_free(eps->mred, eps->stream);
  if (eps->monitor_jsonl) fclose(eps->monitor_jsonl);
  delete eps;
  return B200_OK;
}

extern "C" b200_status b200_eps_set_operators(b200_eps eps, b200_mat A) {
  B200_ARG_CHECK(eps && A, "null argument");
  B200_ARG_CHECK(A->m == A->n, "the operator of an eigenproblem must be square");
  dev_free(eps->op_buf);
  eps->op_buf = nullptr;
  eps->A = A;
  eps->solved = false;
  return B200_OK;
}

extern "C" b200_status b200_eps_set_dimensions(b200_eps eps, int nev, int ncv, int mpd) {
  B200_ARG_CHECK(eps && nev > 0, "nev must be positive");
  eps->nev = nev;
  eps->ncv = ncv;
  eps->mpd = mpd;
  eps->solved = false;
  return B200_OK;
}

extern "C" b200_status b200_eps_set_tolerances(b200_eps eps, double tol, int max_it) {
  B200_ARG_CHECK(eps, "null argument");
  eps->tol = tol;
  eps->max_it = max_it;
  eps->solved = false;
  return B200_OK;
}

extern "C" b200_status b200_eps_set_which_eigenpairs(b200_eps eps, int which) {
  B200_ARG_CHECK(eps && which >= B200_LARGEST_MAGNITUDE && which <= B200_SMALLEST_REAL, "unsupported which");
  eps->which = which;
  eps->which_set = true;
  eps->solved = false;
  return B200_OK;
}

extern "C" b200_status b200_eps_krylovschur_set_locking(b200_eps eps, int lock) {
  B200_ARG_CHECK(eps, "null argument");
  eps->lock = lock ? 1 : 0;
  return B200_OK;
}

extern "C" b200_status b200_eps_krylovschur_get_locking(b200_eps eps, int *lock) {
  B200_ARG_CHECK(eps && lock, "null argument");
  *lock = eps->lock;
  return B200_OK;
}

extern "C" b200_status b200_eps_krylovschur_set_restart(b200_eps eps, double keep) {
  B200_ARG_CHECK(eps && keep >= 0.1 && keep <= 0.9, "keep must be in [0.1,0.9]");
  eps->keep = keep;
  return B200_OK;
}

extern "C" b200_status b200_eps_set_initial_space(b200_eps eps, const double *v0) {
  B200_ARG_CHECK(eps && v0 && eps->A, "set the operator before the initial space");
  eps->v0.assign(v0, v0 + eps->A->n);
  eps->v0_dev = nullptr;
  eps->X0.clear();
  eps->nini_block = 0;
  eps->nini = 1;
  eps->solved = false;
  return B200_OK;
}

extern "C" b200_status b200_eps_set_initial_space_device(b200_eps eps, const double *v0) {
  B200_ARG_CHECK(eps && v0 && eps->A, "set the operator before the initial space");
  eps->v0.clear();
  eps->v0_dev = v0;
  eps->X0.clear();
  eps->nini_block = 0;
  eps->nini = 1;
  eps->solved = false;
  return B200_OK;
}

extern "C" b200_status b200_eps_set_initial_space_block(b200_eps eps, int k, const double *X) {
  B200_ARG_CHECK(eps && eps->A && k >= 0 && (k == 0 || X), "set the operator before the initial space");
  eps->v0.clear();
  eps->v0_dev = nullptr;
  eps->X0.assign(X, X + (size_t)k * eps->A->n);
  eps->nini_block = k;
  eps->nini = k;
  eps->solved = false;
  return B200_OK;
}

extern "C" b200_status b200_eps_set_precision(b200_eps eps, int precision) {
  B200_ARG_CHECK(eps, "null argument");
  B200_ARG_CHECK(precision == B200_PRECISION_FP64 || precision == B200_PRECISION_MIXED, "unknown precision");
  eps->precision = precision;
  return B200_OK;
}

extern "C" b200_status b200_eps_set_mixed_options(b200_eps eps, double tol_low, int degree, int guard,
                                                  int max_sweeps, int fp64_gram) {
  B200_ARG_CHECK(eps, "null argument");
  B200_ARG_CHECK(degree <= 4096 && max_sweeps <= 100000, "degree or max_sweeps too large");
  B200_ARG_CHECK(guard <= 127, "guard too large: the block holds at most 128 vectors");
  eps->mixed_tol_low = tol_low > 0.0 ? tol_low : 0.0;
  eps->mixed_degree = degree > 0 ? degree : 0;
  eps->mixed_guard = guard >= 0 ? guard : -1;
  eps->mixed_max_sweeps = max_sweeps > 0 ? max_sweeps : 0;
  eps->mixed_fp64_gram = fp64_gram ? 1 : 0;
  return B200_OK;
}

extern "C" b200_status b200_eps_set_type(b200_eps eps, int type) {
  B200_ARG_CHECK(eps && (type == B200_EPS_KRYLOVSCHUR || type == B200_EPS_LOBPCG), "unknown EPS type");
  eps->type = type;
  eps->solved = false;
  return B200_OK;
}

extern "C" b200_status b200_eps_lobpcg_set_block_size(b200_eps eps, int bs) {
  B200_ARG_CHECK(eps && bs >= 0, "the block size must be positive");
  eps->lobpcg_bs = bs;
  return B200_OK;
}

extern "C" b200_status b200_eps_lobpcg_set_restart(b200_eps eps, double restart) {
  B200_ARG_CHECK(eps && restart >= 0.1 && restart <= 1.0, "the restart argument must be in [0.1,1.0]");
  eps->lobpcg_restart = restart;
  return B200_OK;
}

extern "C" b200_status b200_eps_lobpcg_set_locking(b200_eps eps, int lock) {
  B200_ARG_CHECK(eps, "null argument");
  eps->lobpcg_lock = lock ? 1 : 0;
  return B200_OK;
}

extern "C" b200_status b200_eps_set_preconditioner(b200_eps eps, int pc) {
  B200_ARG_CHECK(eps && (pc == B200_PC_NONE || pc == B200_PC_JACOBI), "unknown preconditioner");
  eps->pc = pc;
  return B200_OK;
}

extern "C" b200_status b200_eps_set_bv_orthog_block(b200_eps eps, int type) {
  B200_ARG_CHECK(eps, "null EPS");
  B200_ARG_CHECK(type >= B200_ORTHOG_BLOCK_GS && type <= B200_ORTHOG_BLOCK_SVQB, "unknown block orthogonalization type");
  eps->orthog_block = type;
  if (eps->V) eps->V->orthog_block = type;
  return B200_OK;
}

// EPSSetUp's BVInsertVecs(V,0,&k,IS,TRUE) (epssetup.c:421-427, bvfunc.c:331-374): the initial
// space into columns 0..k-1, orthonormalised, linearly dependent vectors dropped.
b200_status b200::eps_insert_initial_space(b200_eps eps, b200_bv V, int max_cols) {
  const int nin = eps->nini_block > 0 ? eps->nini_block : (eps->nini ? 1 : 0);
  B200_ARG_CHECK(nin <= max_cols, "the number of initial vectors is larger than ncv");
  int ndep = 0;
  for (int i = 0; i < nin; ++i) {
    double *dst = col(V, i - ndep);
    if (eps->nini_block > 0)
      B200_CUDA_CHECK(cudaMemcpyAsync(dst, eps->X0.data() + (size_t)i * V->n, sizeof(double) * V->n,
                                      cudaMemcpyHostToDevice, V->stream));
    else if (eps->v0_dev)
      B200_CUDA_CHECK(copy_launch(dst, eps->v0_dev, V->n, V->stream));
    else
      B200_CUDA_CHECK(cudaMemcpyAsync(dst, eps->v0.data(), sizeof(double) * V->n, cudaMemcpyHostToDevice, V->stream));
    double norm = 0.0;
    int lindep = 0;
    B200_CHECK(bv_orth_column(V, i - ndep, 0, nullptr, &norm, &lindep));
    if (norm == 0.0 || lindep) ++ndep;
    else B200_CHECK(b200_bv_scale_column(V, i - ndep, 1.0 / norm));
  }
  eps->nini_eff = nin - ndep;
  return B200_OK;
}

extern "C" b200_status b200_eps_set_max_restarts(b200_eps eps, int max_restarts) {
  B200_ARG_CHECK(eps && max_restarts >= 0, "invalid argument");
  eps->max_restarts = max_restarts;
  return B200_OK;
}

// ---- EPSMonitor (src/eps/interface/epsmon.c:39-60, 96-130)
static double host_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void b200::eps_monitor_start(b200_eps eps) { eps->monitor_t0 = host_ms(); }

b200_status b200::eps_monitor(b200_eps eps, int its, int nconv, const double *eigr, const double *errest, int nest) {
  for (auto &m : eps->monitors)
    if (m.first(eps, its, nconv, eigr, errest, nest, m.second) != 0) {
      b200_set_last_error(__FILE__, __LINE__, "a monitor returned an error");
      return B200_ERR_STATE;
    }
  if (eps->monitor_jsonl) {
    FILE *f = eps->monitor_jsonl;
    fprintf(f, "{\"its\": %d, \"nconv\": %d, \"nest\": %d, \"ms\": %.3f, \"gs_bytes\": %lld, \"eigr\": [", its, nconv,
            nest, host_ms() - eps->monitor_t0, (long long)eps->stats.gs_bytes);
    for (int i = 0; i < nest; ++i) fprintf(f, "%s%.17g", i ? ", " : "", eigr[i]);
    fprintf(f, "], \"errest\": [");
    for (int i = 0; i < nest; ++i) fprintf(f, "%s%.6e", i ? ", " : "", errest[i]);
    fprintf(f, "]}\n");
    fflush(f);
  }
  return B200_OK;
}

extern "C" b200_status b200_eps_monitor_set(b200_eps eps, b200_eps_monitor_fn fn, void *ctx) {
  B200_ARG_CHECK(eps, "null argument");
  if (!fn) return b200_eps_monitor_cancel(eps);
  B200_ARG_CHECK(eps->monitors.size() < 8, "too many monitors (at most 8)");
  eps->monitors.emplace_back(fn, ctx);
  return B200_OK;
}

extern "C" b200_status b200_eps_monitor_cancel(b200_eps eps) {
  B200_ARG_CHECK(eps, "null argument");
  eps->monitors.clear();
  if (eps->monitor_jsonl) fclose(eps->monitor_jsonl);
  eps->monitor_jsonl = nullptr;
  return B200_OK;
}

extern "C" b200_status b200_eps_monitor_jsonl(b200_eps eps, const char *path) {
  B200_ARG_CHECK(eps && path, "null argument");
  FILE *f = fopen(path, "w");
  if (!f) {
    b200_set_last_error(__FILE__, __LINE__, "cannot open the monitor file");
    return B200_ERR_IO;
  }
  if (eps->monitor_jsonl) fclose(eps->monitor_jsonl);
  eps->monitor_jsonl = f;
  return B200_OK;
}

extern "C" b200_status b200_eps_set_timing(b200_eps eps, int on) {
  B200_ARG_CHECK(eps, "null argument");
  eps->timing = on;
  return B200_OK;
}

// EPSSetDimensions_Default (epssetup.c:669-713) + EPSSetUp_KrylovSchur checks (krylovschur.c:105-112).
static b200_status eps_setup(b200_eps eps) {
  B200_ARG_CHECK(eps->A, "EPSSetOperators must be called first");
  const int n = eps->A->n;
  int nev = eps->nev, ncv = eps->ncv, mpd = eps->mpd;
  if (ncv > 0) {
    B200_ARG_CHECK(ncv >= nev + 1 || (ncv == nev && ncv == n), "the value of ncv must be at least nev+1");
  } else if (mpd > 0) {
    ncv = std::min(n, nev + mpd);
  } else {
    if (nev < 500) ncv = std::min(n, std::max(2 * nev, nev + 15));
    else {
      mpd = 500;
      ncv = std::min(n, nev + mpd);
    }
  }
  if (mpd <= 0) mpd = ncv;
  B200_ARG_CHECK(ncv <= nev + mpd, "the value of ncv must not be larger than nev+mpd");
  if (!eps->lock && mpd < ncv) {  // krylovschur.c:116
    b200_set_last_error(__FILE__, __LINE__, "should not use the mpd parameter in the non-locking variant");
    return B200_ERR_SUP;
  }
  B200_ARG_CHECK(ncv <= n, "ncv cannot exceed the problem size");
  B200_ARG_CHECK(ncv + 2 < kMaxCols, "ncv too large for this build (ncv <= 251)");
  eps->n_ = n;
  eps->ncv_ = ncv;
  eps->mpd_ = mpd;
  eps->max_it_ = eps->max_it > 0 ? eps->max_it : std::max(100, 2 * n / ncv);
  eps->tol_ = eps->tol > 0.0 ? eps->tol : 1e-8;  // SLEPC_DEFAULT_TOL (slepcmath.h:25)
  if (eps->V) {
    int bn, bm, bld;
    b200_bv_get_sizes(eps->V, &bn, &bm, &bld);
    if (bn != n || bm != ncv + 1 || eps->V->stream != eps->stream) {
      b200_bv_destroy(eps->V);
      eps->V = nullptr;
    }
  }
  if (!eps->V) B200_CHECK(b200_bv_create(n, ncv + 1, eps->stream, &eps->V));  // EPSAllocateSolution(eps,1)
  eps->ds.allocate(ncv + 1);  // DSAllocate(ds, ncv+1)
  eps->ds.set_which(eps->which);
  eps->eigr.assign(ncv + 1, 0.0);
  eps->errest.assign(ncv + 1, 0.0);
  eps->perm.assign(ncv + 1, 0);
  for (int i = 0; i <= ncv; ++i) eps->perm[i] = i;
  if (!eps->resid_buf) B200_CUDA_CHECK(dev_malloc(&eps->resid_buf, sizeof(double) * 8));
  return B200_OK;
}

// EPSGetStartVector (epssolve.c:841-870): column i, random unless i == 0 and an initial vector exists.
static b200_status eps_start_vector(b200_eps eps, int i, int *breakdown) {
  b200_bv bv = eps->V;
  if (i > 0 || eps->nini_eff == 0) B200_CUDA_CHECK(random_launch(col(bv, i), bv->n, bv->seed, bv->nrand++, bv->stream));
  double norm = 0.0;
  int lindep = 0;
  B200_CHECK(bv_orth_column(bv, i, 0, nullptr, &norm, &lindep));
  if (breakdown) *breakdown = lindep;
  else if (lindep || norm == 0.0) {
    b200_set_last_error(__FILE__, __LINE__,
                        i ? "unable to generate more start vectors" : "initial vector is zero or in the deflation space");
    return B200_ERR_BREAKDOWN;
  }
  if (norm != 0.0) B200_CHECK(b200_bv_scale_column(bv, i, 1.0 / norm));
  return B200_OK;
}

extern "C" b200_status b200_eps_solve(b200_eps eps) {
  B200_ARG_CHECK(eps, "null argument");
  if (eps->type == B200_EPS_LOBPCG) return lobpcg_solve(eps);
  B200_CHECK(eps_setup(eps));
  if (eps->precision == B200_PRECISION_MIXED) return mixed_solve(eps);
  b200_bv V = eps->V;
  DsHep &ds = eps->ds;
  const int ncv = eps->ncv_, mpd = eps->mpd_, nev = eps->nev;
  const double tol = eps->tol_;
  memset(&eps->stats, 0, sizeof(eps->stats));
  const uint64_t launches0 = launch_count();
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, eps->stream);
  eps_monitor_start(eps);
  RunTimer timer;
  timer.on = eps->timing != 0;
  double ms_restart = 0.0;
  cudaEvent_t r0 = nullptr, r1 = nullptr;
  if (timer.on) {
    cudaEventCreate(&r0);
    cudaEventCreate(&r1);
  }

  eps->nconv = 0;
  eps->its = 0;
  eps->reason = B200_CONVERGED_ITERATING;
  eps->solved = false;
  V->nrand = 0;
  b200_bv_set_active_columns(V, 0, V->m);

  // EPSSetUp: BVInsertVecs(V,0,&k,IS,TRUE); then EPSGetStartVector(eps,0,NULL)
  B200_CHECK(eps_insert_initial_space(eps, V, ncv));
  B200_CHECK(eps_start_vector(eps, 0, nullptr));

  int l = 0;
  double beta = 0.0;
  while (eps->reason == B200_CONVERGED_ITERATING) {
    eps->its++;
    int nv = std::min(eps->nconv + mpd, ncv);
    ds.set_dimensions(nv, eps->nconv, eps->nconv + l);
    int breakdown = 0;
    GsState st{};
    B200_CHECK(bv_lanczos(V, eps->A, eps->nconv + l, &nv, ds.d(), ds.e(), &beta, &breakdown, &timer, &st));
    eps->stats.lanczos_steps += nv - (eps->nconv + l);
    for (int j = eps->nconv + l; j < nv; ++j) eps->stats.column_visits += j + 2;
    eps->stats.gs_passes += st.passes;
    eps->stats.gs_bytes += (int64_t)st.bytes;
    ds.set_dimensions(nv, eps->nconv, eps->nconv + l);
    ds.set_state(l ? DsHep::kRaw : DsHep::kIntermediate);
    b200_bv_set_active_columns(V, eps->nconv, nv);

    B200_CHECK(ds.solve(eps->eigr.data()));
    ds.sort(eps->eigr.data());
    ds.update_extra_row();

    // EPSKrylovConvergence: errest_i = beta*|Q(n-1,i)| / |theta_i|, stop at the first failure
    int k = nv;
    for (int kk = eps->nconv; kk < nv; ++kk) {
      const double re = eps->eigr[kk];
      const double resnorm = std::fabs(ds.Q()[ds.n() - 1 + (size_t)kk * ds.ld()]) * beta;
      const double w = std::fabs(re);
      eps->errest[kk] = (w != 0.0) ? resnorm / w : 1.79769313486231571e+308;
      if (eps->errest[kk] >= tol) {
        k = kk;
        break;
      }
    }
    // EPSStoppingBasic
    if (k >= nev) eps->reason = B200_CONVERGED_TOL;
    else if (eps->its >= eps->max_it_) eps->reason = B200_DIVERGED_ITS;

    if (eps->reason != B200_CONVERGED_ITERATING || breakdown || k == nv) l = 0;
    else l = std::max(1, (int)((nv - k) * eps->keep));
    const int nconv_mon = k;   // what EPSMonitor reports (before the non-locking reset)
    if (!eps->lock && l > 0) {  // non-locking variant (krylovschur.c:295): reset the converged count
      l += k;
      k = 0;
    }

    if (eps->reason == B200_CONVERGED_ITERATING) {
      if (breakdown || k == nv) {
        if (k < nev) {
          int bd = 0;
          B200_CHECK(eps_start_vector(eps, k, &bd));
          if (bd) eps->reason = B200_DIVERGED_BREAKDOWN;
        }
      } else {
        ds.truncate(k + l);
      }
    }
    // BVMultInPlace(V,Q,nconv,k+l) over the active columns [nconv,nv)
    if (timer.on) cudaEventRecord(r0, V->stream);
    B200_CHECK(b200_bv_mult_inplace(V, ds.Q(), ds.ld(), eps->nconv, k + l));
    if (timer.on) cudaEventRecord(r1, V->stream);
    if (eps->reason == B200_CONVERGED_ITERATING && !breakdown) B200_CHECK(b200_bv_copy_column(V, nv, k + l));
    if (timer.on) {
      cudaEventSynchronize(r1);
      float t = 0.f;
      if (cudaEventElapsedTime(&t, r0, r1) == cudaSuccess) ms_restart += t;
    }
    eps->nconv = k;
    eps->stats.restarts++;
    if (!eps->monitors.empty() || eps->monitor_jsonl)  // krylovschur.c:339
      B200_CHECK(eps_monitor(eps, eps->its, nconv_mon, eps->eigr.data(), eps->errest.data(), nv));
    if (eps->max_restarts > 0 && eps->stats.restarts >= eps->max_restarts &&
        eps->reason == B200_CONVERGED_ITERATING)
      break;
  }
  B200_CUDA_CHECK(cudaStreamSynchronize(V->stream));
  // SlepcSortEigenvalues (slepcsc.c:89-149) over the converged pairs
  for (int i = 0; i <= ncv; ++i) eps->perm[i] = i;
  for (int i = eps->nconv - 1; i >= 0; --i) {
    const double re = eps->eigr[eps->perm[i]];
    int j = i + 1;
    while (j < eps->nconv) {
      if (DsHep::compare(eps->which, re, eps->eigr[eps->perm[j]]) <= 0) break;
      std::swap(eps->perm[j - 1], eps->perm[j]);
      ++j;
    }
  }
  cudaEventRecord(t1, eps->stream);
  cudaEventSynchronize(t1);
  float total = 0.f;
  cudaEventElapsedTime(&total, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (r0) cudaEventDestroy(r0);
  if (r1) cudaEventDestroy(r1);
  eps->stats.ms_total = total;
  eps->stats.ms_spmv = timer.ms_spmv;
  eps->stats.ms_orth = timer.ms_orth;
  eps->stats.ms_restart = ms_restart;
  eps->stats.kernel_launches = (int64_t)(launch_count() - launches0);
  eps->solved = true;
  return B200_OK;
}

extern "C" b200_status b200_eps_get_converged(b200_eps eps, int *nconv) {
  B200_ARG_CHECK(eps && nconv, "null argument");
  if (!eps->solved) {
    b200_set_last_error(__FILE__, __LINE__, "EPSSolve must be called first");
    return B200_ERR_STATE;
  }
  *nconv = eps->nconv;
  return B200_OK;
}

extern "C" b200_status b200_eps_get_iteration_number(b200_eps eps, int *its) {
  B200_ARG_CHECK(eps && its, "null argument");
  *its = eps->its;
  return B200_OK;
}

extern "C" b200_status b200_eps_get_converged_reason(b200_eps eps, int *reason) {
  B200_ARG_CHECK(eps && reason, "null argument");
  *reason = eps->reason;
  return B200_OK;
}

static b200_status eps_check_index(b200_eps eps, int i) {
  if (!eps->solved) {
    b200_set_last_error(__FILE__, __LINE__, "EPSSolve must be called first");
    return B200_ERR_STATE;
  }
  B200_ARG_CHECK(i >= 0 && i < eps->nconv, "eigenpair index out of range");
  return B200_OK;
}

extern "C" b200_status b200_eps_get_eigenpair(b200_eps eps, int i, double *eigr, double *x) {
  B200_ARG_CHECK(eps, "null argument");
  B200_CHECK(eps_check_index(eps, i));
  const int p = eps->perm[i];
  if (eigr) *eigr = eps->eigr[p];
  if (x) {
    B200_CUDA_CHECK(
        cudaMemcpyAsync(x, col(eps->V, p), sizeof(double) * eps->n_, cudaMemcpyDeviceToHost, eps->V->stream));
    B200_CUDA_CHECK(cudaStreamSynchronize(eps->V->stream));
  }
  return B200_OK;
}

extern "C" b200_status b200_eps_get_eigenvector_device(b200_eps eps, int i, const double **x) {
  B200_ARG_CHECK(eps && x, "null argument");
  B200_CHECK(eps_check_index(eps, i));
  *x = col(eps->V, eps->perm[i]);
  return B200_OK;
}

extern "C" b200_status b200_eps_get_error_estimate(b200_eps eps, int i, double *errest) {
  B200_ARG_CHECK(eps && errest, "null argument");
  B200_CHECK(eps_check_index(eps, i));
  *errest = eps->errest[eps->perm[i]];
  return B200_OK;
}

extern "C" b200_status b200_eps_compute_error(b200_eps eps, int i, int type, double *error) {
  B200_ARG_CHECK(eps && error, "null argument");
  B200_CHECK(eps_check_index(eps, i));
  const int p = eps->perm[i];
  const double lam = eps->eigr[p];
  b200_mat A = eps->A;
  b200_bv V = eps->V;
  // ||A x - lambda x||_2, with the shift skipped for |lambda| <= eps (epssolve.c:689-694)
  const double shift = (std::fabs(lam) > 2.220446049250313e-16) ? lam : 0.0;
  if (A->kind == kMatCsr && !A->a.f32) {
    B200_CUDA_CHECK(residual_launch(A->n, A->a.rowptr, A->a.colind, static_cast<const double *>(A->a.vals), col(V, p),
                                    shift, eps->resid_buf, V->red, V->red_len, A->a.lanes, V->stream));
  } else {
    if (!eps->op_buf) B200_CUDA_CHECK(dev_malloc(&eps->op_buf, sizeof(double) * (size_t)A->n));
    B200_CUDA_CHECK(mat_spmv(A, col(V, p), eps->op_buf, V->stream));
    B200_CUDA_CHECK(diff_sumsq_launch(eps->op_buf, col(V, p), shift, A->n, eps->resid_buf, V->red, V->red_len,
                                      V->stream));
  }
  B200_CUDA_CHECK(cudaMemcpyAsync(V->hpin, eps->resid_buf, sizeof(double), cudaMemcpyDeviceToHost, V->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(V->stream));
  double r = std::sqrt(V->hpin[0]);
  if (type == B200_ERROR_RELATIVE) r /= std::fabs(lam);
  *error = r;
  return B200_OK;
}

extern "C" b200_status b200_eps_get_stats(b200_eps eps, b200_eps_stats *stats) {
  B200_ARG_CHECK(eps && stats, "null argument");
  *stats = eps->stats;
  return B200_OK;
}

extern "C" b200_status b200_eps_solve_csr_host(int n, int64_t nnz, const int *rowptr, const int *colind,
                                               const double *vals, const double *v0, int nev, int ncv, int mpd,
                                               double tol, int max_it, int which, double *evals, double *X,
                                               double *errest, int *info, void *stream) {
  return b200_eps_solve_csr_host_ex(n, nnz, rowptr, colind, vals, v0, nev, ncv, mpd, tol, max_it, which,
                                    B200_PRECISION_FP64, evals, X, errest, info, stream);
}

extern "C" b200_status b200_eps_solve_csr_host_ex(int n, int64_t nnz, const int *rowptr, const int *colind,
                                                  const double *vals, const double *v0, int nev, int ncv, int mpd,
                                                  double tol, int max_it, int which, int precision, double *evals,
                                                  double *X, double *errest, int *info, void *stream) {
  b200_mat A = nullptr;
  b200_eps E = nullptr;
  B200_CHECK(b200_mat_create_csr(n, nnz, rowptr, colind, vals, stream, &A));
  b200_status s = b200_eps_create(stream, &E);
  if (s == B200_OK) s = b200_eps_set_operators(E, A);
  if (s == B200_OK && precision != B200_PRECISION_FP64) s = b200_eps_set_precision(E, precision);
  if (s == B200_OK) s = b200_eps_set_dimensions(E, nev, ncv, mpd);
  if (s == B200_OK) s = b200_eps_set_tolerances(E, tol, max_it);
  if (s == B200_OK) s = b200_eps_set_which_eigenpairs(E, which);
  if (s == B200_OK && v0) s = b200_eps_set_initial_space(E, v0);
  if (s == B200_OK) s = b200_eps_solve(E);
  if (s == B200_OK) {
    for (int i = 0; i < E->nconv && s == B200_OK; ++i) {
      double lam = 0.0;
      s = b200_eps_get_eigenpair(E, i, &lam, X ? X + (size_t)i * n : nullptr);
      if (evals) evals[i] = lam;
      if (errest) errest[i] = E->errest[E->perm[i]];
    }
    if (info) {
      info[0] = E->nconv;
      info[1] = E->its;
      info[2] = E->reason;
      info[3] = (int)E->stats.lanczos_steps;
      info[4] = (int)E->stats.restarts;
    }
  }
  b200_eps_destroy(E);
  b200_mat_destroy(A);
  return s;
}
