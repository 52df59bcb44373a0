/*
 * gen_powerlaw.c -- generator of the rectangular sparse test matrix of the
 * SVD cross workload (host code; not part of the GPU library).
 *
 * Row i of the m x n matrix holds k = min(nnz_row, n) distinct columns: the
 * first k distinct values of a stream of draws c = floor(x) - 1, where x has
 * the density proportional to x^-alpha on [1, n+1) and is drawn by inverse
 * CDF, x = (1 - u (1 - (n+1)^(1-alpha)))^(-1/(alpha-1)).  Column c is thus
 * drawn with probability proportional to the integral of x^-alpha over
 * [c+1, c+2): a power law with exponent alpha in the column index, so that a
 * few columns appear in almost every row.  The columns of a row are sorted
 * ascending and the value in slot j of row i is a standard normal
 * (Box-Muller) rounded to float32.
 *
 * Every uniform comes from splitmix64 on a counter (seed, stream, row, draw),
 * so the matrix depends only on (m, n, nnz_row, alpha, seed) and rows can be
 * generated in parallel.  gen_uniform / gen_normal expose the streams so a
 * pure-Python restatement can be checked against this file.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

static uint64_t mix(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

static uint64_t draw_bits(uint64_t seed, int stream, int64_t row, int64_t t)
{
  const uint64_t key = ((uint64_t)row << 24) ^ (uint64_t)t;
  return mix(mix(seed * 4 + (uint64_t)stream) ^ key);
}

/* uniform in [0,1) */
double gen_uniform(uint64_t seed, int stream, int64_t row, int64_t t)
{
  return (double)(draw_bits(seed, stream, row, t) >> 11) * (1.0 / 9007199254740992.0);
}

/* standard normal from two uniforms of stream 1 (draws 2j and 2j+1) */
double gen_normal(uint64_t seed, int64_t row, int64_t j)
{
  const double u1 = ((double)(draw_bits(seed, 1, row, 2 * j) >> 11) + 1.0) * (1.0 / 9007199254740992.0);
  const double u2 = gen_uniform(seed, 1, row, 2 * j + 1);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

static int cmp_int(const void *a, const void *b)
{
  const int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

/* rowptr: m+1 entries; colind, vals: m * min(nnz_row, n) entries.  Returns 0,
 * or 1 for invalid arguments. */
int gen_powerlaw(int m, int n, int nnz_row, double alpha, uint64_t seed, int *rowptr, int *colind, float *vals)
{
  if (m <= 0 || n <= 0 || nnz_row <= 0 || !(alpha > 1.0)) return 1;
  const int k = nnz_row < n ? nnz_row : n;
  const double a1 = alpha - 1.0;
  const double tail = 1.0 - pow((double)n + 1.0, -a1);
  int64_t i;
  for (i = 0; i <= m; i++) rowptr[i] = (int)(i * k);
#pragma omp parallel for schedule(dynamic, 256)
  for (i = 0; i < m; i++) {
    int *cols = colind + i * k;
    int cnt = 0;
    for (int64_t t = 0; cnt < k && t < (1 << 24); t++) {
      const double u = gen_uniform(seed, 0, i, t);
      const double x = pow(1.0 - u * tail, -1.0 / a1);
      int c = (int)floor(x) - 1;
      if (c < 0) c = 0;
      if (c > n - 1) c = n - 1;
      int seen = 0;
      for (int q = 0; q < cnt; q++)
        if (cols[q] == c) { seen = 1; break; }
      if (!seen) cols[cnt++] = c;
    }
    /* draw budget exhausted (only for tiny n with a huge alpha): the smallest unused columns */
    for (int c = 0; cnt < k && c < n; c++) {
      int seen = 0;
      for (int q = 0; q < cnt; q++)
        if (cols[q] == c) { seen = 1; break; }
      if (!seen) cols[cnt++] = c;
    }
    qsort(cols, (size_t)cnt, sizeof(int), cmp_int);
    for (int j = 0; j < k; j++) vals[i * k + j] = (float)gen_normal(seed, i, j);
  }
  return 0;
}
