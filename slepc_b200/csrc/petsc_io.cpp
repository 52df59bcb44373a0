// PETSc binary viewer format for Mat (AIJ) and Vec objects, host side.
//
// The format PetscViewerBinary writes for MatView / VecView and reads for
// MatLoad / VecLoad (used by SLEPc drivers such as
// src/eps/tutorials/ex4.c:45-48 and ex31.c:551-562), with 32-bit PetscInt and
// real double PetscScalar, every number big-endian:
//   Mat: int32 classid 1211216, int32 M, int32 N, int32 nz,
//        int32 row lengths[M], int32 column indices[nz], float64 values[nz]
//   Vec: int32 classid 1211214, int32 N, float64 values[N]
// Objects follow one another in a file; a viewer reads or appends them in order.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.h"

struct b200_viewer_s {
  FILE *f = nullptr;
  int mode = 0;  // B200_FILE_MODE_READ / WRITE / APPEND
  std::string path;
};

namespace {

uint32_t bswap32(uint32_t v) {
  return (v >> 24) | ((v >> 8) & 0x0000ff00u) | ((v << 8) & 0x00ff0000u) | (v << 24);
}

uint64_t bswap64(uint64_t v) {
  return ((uint64_t)bswap32((uint32_t)v) << 32) | bswap32((uint32_t)(v >> 32));
}

bool host_is_little() {
  const uint16_t probe = 1;
  return *reinterpret_cast<const uint8_t *>(&probe) == 1;
}

bool read_i32(FILE *f, int32_t *out, size_t count) {
  if (count == 0) return true;
  if (fread(out, sizeof(int32_t), count, f) != count) return false;
  if (host_is_little())
    for (size_t i = 0; i < count; ++i) out[i] = (int32_t)bswap32((uint32_t)out[i]);
  return true;
}

bool read_f64(FILE *f, double *out, size_t count) {
  if (count == 0) return true;
  if (fread(out, sizeof(double), count, f) != count) return false;
  if (host_is_little())
    for (size_t i = 0; i < count; ++i) {
      uint64_t u;
      memcpy(&u, out + i, 8);
      u = bswap64(u);
      memcpy(out + i, &u, 8);
    }
  return true;
}

bool write_i32(FILE *f, const int32_t *in, size_t count) {
  std::vector<int32_t> buf(in, in + count);
  if (host_is_little())
    for (auto &v : buf) v = (int32_t)bswap32((uint32_t)v);
  return count == 0 || fwrite(buf.data(), sizeof(int32_t), count, f) == count;
}

bool write_f64(FILE *f, const double *in, size_t count) {
  std::vector<uint64_t> buf(count);
  for (size_t i = 0; i < count; ++i) {
    memcpy(&buf[i], in + i, 8);
    if (host_is_little()) buf[i] = bswap64(buf[i]);
  }
  return count == 0 || fwrite(buf.data(), sizeof(uint64_t), count, f) == count;
}

constexpr int32_t kMatClassid = B200_MAT_FILE_CLASSID;
constexpr int32_t kVecClassid = B200_VEC_FILE_CLASSID;

#define B200_IO_FAIL(msg)                          \
  do {                                             \
    b200_set_last_error(__FILE__, __LINE__, msg);  \
    return B200_ERR_IO;                            \
  } while (0)

}  // namespace

extern "C" b200_status b200_viewer_binary_open(const char *path, int mode, b200_viewer *v) {
  B200_ARG_CHECK(path && v, "null argument");
  B200_ARG_CHECK(mode == B200_FILE_MODE_READ || mode == B200_FILE_MODE_WRITE || mode == B200_FILE_MODE_APPEND,
                 "unknown file mode");
  const char *m = mode == B200_FILE_MODE_READ ? "rb" : (mode == B200_FILE_MODE_WRITE ? "wb" : "ab");
  FILE *f = fopen(path, m);
  if (!f) B200_IO_FAIL("cannot open the binary file");
  b200_viewer V = new b200_viewer_s;
  V->f = f;
  V->mode = mode;
  V->path = path;
  *v = V;
  return B200_OK;
}

extern "C" b200_status b200_viewer_destroy(b200_viewer v) {
  if (!v) return B200_OK;
  const bool ok = !v->f || fclose(v->f) == 0;
  delete v;
  if (!ok) B200_IO_FAIL("closing the binary file failed");
  return B200_OK;
}

extern "C" b200_status b200_viewer_peek(b200_viewer v, int *classid, int *m, int *n, int64_t *nnz) {
  B200_ARG_CHECK(v && v->f && v->mode == B200_FILE_MODE_READ, "viewer not open for reading");
  const long pos = ftell(v->f);
  int32_t h[4] = {0, 0, 0, 0};
  if (!read_i32(v->f, h, 2)) {
    fseek(v->f, pos, SEEK_SET);
    B200_IO_FAIL("end of file: no further object");
  }
  if (h[0] == kMatClassid && !read_i32(v->f, h + 2, 2)) {
    fseek(v->f, pos, SEEK_SET);
    B200_IO_FAIL("truncated Mat header");
  }
  fseek(v->f, pos, SEEK_SET);
  if (h[0] != kMatClassid && h[0] != kVecClassid) B200_IO_FAIL("not a PETSc binary Mat or Vec object");
  if (classid) *classid = h[0];
  if (h[0] == kMatClassid) {
    if (m) *m = h[1];
    if (n) *n = h[2];
    if (nnz) *nnz = h[3];
  } else {
    if (m) *m = h[1];
    if (n) *n = 1;
    if (nnz) *nnz = h[1];
  }
  return B200_OK;
}

extern "C" b200_status b200_mat_read_csr(b200_viewer v, int *rowptr, int *colind, double *vals) {
  B200_ARG_CHECK(v && v->f && v->mode == B200_FILE_MODE_READ, "viewer not open for reading");
  B200_ARG_CHECK(rowptr, "null rowptr");
  int32_t h[4];
  if (!read_i32(v->f, h, 4)) B200_IO_FAIL("truncated Mat header");
  if (h[0] != kMatClassid) B200_IO_FAIL("the next object is not a Mat");
  const int32_t M = h[1], N = h[2], nz = h[3];
  if (M < 0 || N < 0 || nz < 0) B200_IO_FAIL("negative Mat sizes (64-bit PetscInt files are not read)");
  B200_ARG_CHECK(nz == 0 || (colind && vals), "null colind/vals");
  std::vector<int32_t> lens((size_t)M);
  if (!read_i32(v->f, lens.data(), (size_t)M)) B200_IO_FAIL("truncated row lengths");
  rowptr[0] = 0;
  for (int32_t i = 0; i < M; ++i) {
    if (lens[i] < 0) B200_IO_FAIL("negative row length");
    rowptr[i + 1] = rowptr[i] + lens[i];
  }
  if (rowptr[M] != nz) B200_IO_FAIL("row lengths do not add up to nz");
  if (!read_i32(v->f, colind, (size_t)nz)) B200_IO_FAIL("truncated column indices");
  for (int32_t p = 0; p < nz; ++p)
    if (colind[p] < 0 || colind[p] >= N) B200_IO_FAIL("column index out of range");
  if (!read_f64(v->f, vals, (size_t)nz)) B200_IO_FAIL("truncated values");
  return B200_OK;
}

extern "C" b200_status b200_mat_write_csr(b200_viewer v, int m, int n, int64_t nnz, const int *rowptr,
                                          const int *colind, const double *vals) {
  B200_ARG_CHECK(v && v->f && v->mode != B200_FILE_MODE_READ, "viewer not open for writing");
  B200_ARG_CHECK(m >= 0 && n >= 0 && nnz >= 0 && nnz <= 0x7fffffff && rowptr && (nnz == 0 || (colind && vals)),
                 "invalid CSR arguments");
  B200_ARG_CHECK(rowptr[0] == 0 && rowptr[m] == nnz, "rowptr must start at 0 and end at nnz");
  const int32_t h[4] = {kMatClassid, m, n, (int32_t)nnz};
  std::vector<int32_t> lens((size_t)m);
  for (int i = 0; i < m; ++i) lens[i] = rowptr[i + 1] - rowptr[i];
  if (!write_i32(v->f, h, 4) || !write_i32(v->f, lens.data(), lens.size()) ||
      !write_i32(v->f, colind, (size_t)nnz) || !write_f64(v->f, vals, (size_t)nnz) || fflush(v->f) != 0)
    B200_IO_FAIL("writing the Mat failed");
  return B200_OK;
}

extern "C" b200_status b200_vec_read(b200_viewer v, int nmax, int *n, double *x) {
  B200_ARG_CHECK(v && v->f && v->mode == B200_FILE_MODE_READ, "viewer not open for reading");
  int32_t h[2];
  const long pos = ftell(v->f);
  if (!read_i32(v->f, h, 2)) B200_IO_FAIL("truncated Vec header");
  if (h[0] != kVecClassid) {
    fseek(v->f, pos, SEEK_SET);
    B200_IO_FAIL("the next object is not a Vec");
  }
  if (h[1] < 0) B200_IO_FAIL("negative Vec size");
  if (h[1] > nmax || (h[1] > 0 && !x)) {
    fseek(v->f, pos, SEEK_SET);
    b200_set_last_error(__FILE__, __LINE__, "the Vec is longer than the buffer");
    return B200_ERR_ARG;
  }
  if (!read_f64(v->f, x, (size_t)h[1])) B200_IO_FAIL("truncated Vec values");
  if (n) *n = h[1];
  return B200_OK;
}

extern "C" b200_status b200_vec_write(b200_viewer v, int n, const double *x) {
  B200_ARG_CHECK(v && v->f && v->mode != B200_FILE_MODE_READ, "viewer not open for writing");
  B200_ARG_CHECK(n >= 0 && (n == 0 || x), "invalid Vec arguments");
  const int32_t h[2] = {kVecClassid, n};
  if (!write_i32(v->f, h, 2) || !write_f64(v->f, x, (size_t)n) || fflush(v->f) != 0)
    B200_IO_FAIL("writing the Vec failed");
  return B200_OK;
}
