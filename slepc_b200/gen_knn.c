/*
 * gen_knn.c -- generator of the batched workload's matrices (host code; not
 * part of the GPU library).
 *
 * Problem p has n points drawn uniformly in the unit square from a
 * counter-based stream (seed, p, i), sorted by the cell of a g x g grid
 * (g = ceil(sqrt(n / 2)), row-major cells, point index breaking ties), so that
 * neighbouring rows are near in space.  Every point is joined to its k
 * nearest other points (exact: the grid is searched in growing square rings
 * until no unsearched cell can hold a closer point; distance ties broken by
 * the smaller index), the graph is symmetrised (W = max(W, W^T), unit
 * weights) and the operator is 2 I - L_norm = I + D^{-1/2} W D^{-1/2}, with
 * D the degrees of W: CSR with sorted column indices, diagonal 1, entries
 * 1/sqrt(d_i d_j).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static uint64_t mix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

/* uniform [0,1) for (seed, problem, i, coordinate) */
double knn_uniform(uint64_t seed, int64_t problem, int64_t i, int coord)
{
  const uint64_t key = ((uint64_t)problem << 40) ^ ((uint64_t)i << 1) ^ (uint64_t)coord;
  return (double)(mix64(mix64(seed ^ 0x6b6e6eULL) ^ key) >> 11) * (1.0 / 9007199254740992.0);
}

typedef struct {
  double x, y;
  int cell;
  int id;
} pt;

static int cmp_pt(const void *a, const void *b)
{
  const pt *p = (const pt *)a, *q = (const pt *)b;
  if (p->cell != q->cell) return p->cell < q->cell ? -1 : 1;
  return (p->id > q->id) - (p->id < q->id);
}

static int cmp_int(const void *a, const void *b)
{
  const int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

/* nonzeros of the problem's matrix, for sizing (calls the full build with no output) */
int64_t knn_nnz(int n, int k, uint64_t seed, int64_t problem);

/* Builds problem p: rowptr (n+1), colind / vals (capacity cap, returns nnz or -1). */
int64_t knn_build(int n, int k, uint64_t seed, int64_t problem, int *rowptr, int *colind, double *vals, int64_t cap)
{
  if (n <= k || k <= 0) return -1;
  const int g = (int)ceil(sqrt((double)n / 2.0));
  pt *P = (pt *)malloc(sizeof(pt) * (size_t)n);
  for (int i = 0; i < n; i++) {
    P[i].x = knn_uniform(seed, problem, i, 0);
    P[i].y = knn_uniform(seed, problem, i, 1);
    int cx = (int)(P[i].x * g), cy = (int)(P[i].y * g);
    if (cx >= g) cx = g - 1;
    if (cy >= g) cy = g - 1;
    P[i].cell = cy * g + cx;
    P[i].id = i;
  }
  qsort(P, (size_t)n, sizeof(pt), cmp_pt);
  int *cstart = (int *)calloc((size_t)g * g + 1, sizeof(int));
  for (int i = 0; i < n; i++) cstart[P[i].cell + 1]++;
  for (int c = 0; c < g * g; c++) cstart[c + 1] += cstart[c];
  /* k nearest of every point (indices into the sorted order) */
  int *nb = (int *)malloc(sizeof(int) * (size_t)n * k);
  double *bd = (double *)malloc(sizeof(double) * (size_t)k);
  int *bi = (int *)malloc(sizeof(int) * (size_t)k);
  const double h = 1.0 / g;
  for (int i = 0; i < n; i++) {
    const int cx = P[i].cell % g, cy = P[i].cell / g;
    int cnt = 0;
    for (int ring = 0;; ring++) {
      for (int yy = cy - ring; yy <= cy + ring; yy++) {
        if (yy < 0 || yy >= g) continue;
        for (int xx = cx - ring; xx <= cx + ring; xx++) {
          if (xx < 0 || xx >= g) continue;
          if (yy != cy - ring && yy != cy + ring && xx != cx - ring && xx != cx + ring) continue;
          const int c = yy * g + xx;
          for (int q = cstart[c]; q < cstart[c + 1]; q++) {
            if (q == i) continue;
            const double dx = P[q].x - P[i].x, dy = P[q].y - P[i].y, d2 = dx * dx + dy * dy;
            /* insert into the sorted best list (distance, then index) */
            if (cnt == k && (d2 > bd[k - 1] || (d2 == bd[k - 1] && q > bi[k - 1]))) continue;
            int pos = cnt < k ? cnt++ : k - 1;
            while (pos > 0 && (bd[pos - 1] > d2 || (bd[pos - 1] == d2 && bi[pos - 1] > q))) {
              bd[pos] = bd[pos - 1];
              bi[pos] = bi[pos - 1];
              pos--;
            }
            bd[pos] = d2;
            bi[pos] = q;
          }
        }
      }
      /* every unsearched cell is at least ring*h away in x or y from the point's cell */
      const double fx = P[i].x - cx * h, fy = P[i].y - cy * h;
      double edge = fx;
      if (h - fx < edge) edge = h - fx;
      if (fy < edge) edge = fy;
      if (h - fy < edge) edge = h - fy;
      const double reach = ring * h + edge;
      const int covers_all = (cx - ring <= 0 && cy - ring <= 0 && cx + ring >= g - 1 && cy + ring >= g - 1);
      if (covers_all || (cnt == k && reach * reach >= bd[k - 1])) break;
    }
    for (int t = 0; t < k; t++) nb[(size_t)i * k + t] = bi[t];
  }
  /* symmetrise: union of i->j and j->i */
  int *deg = (int *)calloc((size_t)n, sizeof(int));
  for (int i = 0; i < n; i++)
    for (int t = 0; t < k; t++) {
      deg[i]++;
      deg[nb[(size_t)i * k + t]]++;
    }
  int *start = (int *)malloc(sizeof(int) * ((size_t)n + 1));
  start[0] = 0;
  for (int i = 0; i < n; i++) start[i + 1] = start[i] + deg[i];
  int *adj = (int *)malloc(sizeof(int) * (size_t)start[n]);
  int *fill = (int *)calloc((size_t)n, sizeof(int));
  for (int i = 0; i < n; i++)
    for (int t = 0; t < k; t++) {
      const int j = nb[(size_t)i * k + t];
      adj[start[i] + fill[i]++] = j;
      adj[start[j] + fill[j]++] = i;
    }
  int *ulen = (int *)malloc(sizeof(int) * (size_t)n);
  for (int i = 0; i < n; i++) {
    int *a = adj + start[i];
    qsort(a, (size_t)deg[i], sizeof(int), cmp_int);
    int u = 0;
    for (int t = 0; t < deg[i]; t++)
      if (u == 0 || a[u - 1] != a[t]) a[u++] = a[t];
    ulen[i] = u;  /* the symmetric degree d_i */
  }
  int64_t nnz = 0;
  for (int i = 0; i < n; i++) nnz += ulen[i] + 1;
  if (rowptr && nnz <= cap) {
    int64_t p = 0;
    rowptr[0] = 0;
    for (int i = 0; i < n; i++) {
      const int *a = adj + start[i];
      int placed = 0;
      for (int t = 0; t < ulen[i]; t++) {
        if (!placed && a[t] > i) {
          colind[p] = i;
          vals[p++] = 1.0;
          placed = 1;
        }
        colind[p] = a[t];
        vals[p++] = 1.0 / sqrt((double)ulen[i] * (double)ulen[a[t]]);
      }
      if (!placed) {
        colind[p] = i;
        vals[p++] = 1.0;
      }
      rowptr[i + 1] = (int)p;
    }
  }
  free(P); free(cstart); free(nb); free(bd); free(bi); free(deg); free(start); free(adj); free(fill); free(ulen);
  return nnz;
}

int64_t knn_nnz(int n, int k, uint64_t seed, int64_t problem)
{
  return knn_build(n, k, seed, problem, NULL, NULL, NULL, 0);
}

/* coordinates of problem p's points in the sorted (row) order, for tests */
int knn_points(int n, uint64_t seed, int64_t problem, double *xy)
{
  const int g = (int)ceil(sqrt((double)n / 2.0));
  pt *P = (pt *)malloc(sizeof(pt) * (size_t)n);
  for (int i = 0; i < n; i++) {
    P[i].x = knn_uniform(seed, problem, i, 0);
    P[i].y = knn_uniform(seed, problem, i, 1);
    int cx = (int)(P[i].x * g), cy = (int)(P[i].y * g);
    if (cx >= g) cx = g - 1;
    if (cy >= g) cy = g - 1;
    P[i].cell = cy * g + cx;
    P[i].id = i;
  }
  qsort(P, (size_t)n, sizeof(pt), cmp_pt);
  for (int i = 0; i < n; i++) {
    xy[2 * i] = P[i].x;
    xy[2 * i + 1] = P[i].y;
  }
  free(P);
  return 0;
}

/*
 * All problems of a batch, concatenated: problem p has ns[p] rows starting at global row
 * row_off[p] and nonzeros starting at nnz_off[p]; its column indices are local (0..ns[p]-1).
 * Phase 1 (nnz_out == NULL): fills counts[p] with each problem's nonzeros.
 * Phase 2: writes rowptr (local, per problem: ns[p]+1 entries at row_off[p]+p), colind, vals.
 */
int knn_build_batch(int nprob, const int *ns, int k, uint64_t seed, int64_t *counts, const int64_t *row_off,
                    const int64_t *nnz_off, int *rowptr, int *colind, double *vals)
{
  int bad = 0;
  int p;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : bad)
  for (p = 0; p < nprob; p++) {
    const int n = ns[p];
    if (!rowptr) {
      counts[p] = knn_nnz(n, k, seed, p);
      if (counts[p] < 0) bad++;
    } else {
      const int64_t got = knn_build(n, k, seed, p, rowptr + row_off[p] + p, colind + nnz_off[p], vals + nnz_off[p],
                                    counts[p]);
      if (got != counts[p]) bad++;
    }
  }
  return bad;
}
