/*
 * CPU restatement of RVPoint's scalar hot path -- TEST INFRASTRUCTURE ONLY.
 * See rvp_oracle.h. Reference citations are paths inside Mumu-kun/rvpoint.
 *
 * Arithmetic is written in the reference's evaluation order; the Makefile
 * compiles with -ffp-contract=off so that no FMA changes a rounding.
 */
#define _GNU_SOURCE
#include "rvp_oracle.h"

#include <float.h>
#include <pthread.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ------------------------------------------------------------------------ */
/* SpatialHash                                                              */
/* ------------------------------------------------------------------------ */

typedef struct {
  float min_x, min_y, min_z, max_x, max_y, max_z, cell;
  int64_t p1, p2;
  size_t nb;         /* number of buckets */
  int64_t *bkey;     /* sorted distinct bucket keys */
  size_t *bstart;    /* bucket b holds order[bstart[b] .. bstart[b+1]) */
  int *order;        /* point indices grouped by bucket, input order inside */
} rvo_hash;

typedef struct {
  int64_t key;
  int idx;
} key_idx;

static int cmp_key_idx(const void *a, const void *b) {
  const key_idx *p = (const key_idx *)a, *q = (const key_idx *)b;
  if (p->key != q->key) return p->key < q->key ? -1 : 1;
  return p->idx < q->idx ? -1 : (p->idx > q->idx);
}

/* getCellIndices: spatial_hashing.h:47-52 (float divide, floor, int cast). */
static void cell_of(const rvo_hash *h, float x, float y, float z, int *ix,
                    int *iy, int *iz) {
  *ix = (int)floorf((x - h->min_x) / h->cell);
  *iy = (int)floorf((y - h->min_y) / h->cell);
  *iz = (int)floorf((z - h->min_z) / h->cell);
}

/* hashCell: spatial_hashing.h:43-45. */
static int64_t hash_cell(const rvo_hash *h, int ix, int iy, int iz) {
  return (int64_t)ix + (int64_t)iy * h->p1 + (int64_t)iz * h->p2;
}

/* setInputCloud (spatial_hashing.cpp:21-96, scalar branch :76-83) and
 * build (:98-108). Buckets keep input order, like push_back. */
static void hash_build(rvo_hash *h, const float *x, const float *y,
                       const float *z, size_t n, float cell, int64_t p1,
                       int64_t p2) {
  memset(h, 0, sizeof(*h));
  h->cell = cell;
  h->p1 = p1;
  h->p2 = p2;
  if (n == 0) return;
  h->min_x = h->min_y = h->min_z = FLT_MAX;
  h->max_x = h->max_y = h->max_z = -FLT_MAX;
  for (size_t j = 0; j < n; ++j) {
    if (x[j] < h->min_x) h->min_x = x[j];
    if (x[j] > h->max_x) h->max_x = x[j];
    if (y[j] < h->min_y) h->min_y = y[j];
    if (y[j] > h->max_y) h->max_y = y[j];
    if (z[j] < h->min_z) h->min_z = z[j];
    if (z[j] > h->max_z) h->max_z = z[j];
  }
  const float eps = cell * 0.01f; /* eps_scale_ = 0.01f, spatial_hashing.h:32 */
  h->min_x -= eps;
  h->min_y -= eps;
  h->min_z -= eps;
  h->max_x += eps;
  h->max_y += eps;
  h->max_z += eps;

  key_idx *ki = (key_idx *)malloc(n * sizeof(key_idx));
  for (size_t i = 0; i < n; ++i) {
    int ix, iy, iz;
    cell_of(h, x[i], y[i], z[i], &ix, &iy, &iz);
    ki[i].key = hash_cell(h, ix, iy, iz);
    ki[i].idx = (int)i;
  }
  qsort(ki, n, sizeof(key_idx), cmp_key_idx);
  h->order = (int *)malloc(n * sizeof(int));
  h->bkey = (int64_t *)malloc(n * sizeof(int64_t));
  h->bstart = (size_t *)malloc((n + 1) * sizeof(size_t));
  size_t nb = 0;
  for (size_t i = 0; i < n; ++i) {
    h->order[i] = ki[i].idx;
    if (i == 0 || ki[i].key != ki[i - 1].key) {
      h->bkey[nb] = ki[i].key;
      h->bstart[nb] = i;
      ++nb;
    }
  }
  h->bstart[nb] = n;
  h->nb = nb;
  free(ki);
}

static void hash_free(rvo_hash *h) {
  free(h->order);
  free(h->bkey);
  free(h->bstart);
  memset(h, 0, sizeof(*h));
}

static long find_bucket(const rvo_hash *h, int64_t key) {
  size_t lo = 0, hi = h->nb;
  while (lo < hi) {
    size_t mid = (lo + hi) / 2;
    if (h->bkey[mid] < key) lo = mid + 1; else hi = mid;
  }
  if (lo < h->nb && h->bkey[lo] == key) return (long)lo;
  return -1;
}

typedef struct {
  float d2;
  int idx;
} nbr;

/* std::pair<float,int> operator< : spatial_hashing.cpp:149-154. */
static int cmp_nbr(const void *a, const void *b) {
  const nbr *p = (const nbr *)a, *q = (const nbr *)b;
  if (p->d2 < q->d2) return -1;
  if (q->d2 < p->d2) return 1;
  return p->idx < q->idx ? -1 : (p->idx > q->idx);
}

typedef struct {
  nbr *v;
  size_t n, cap;
} nbr_vec;

static void nv_push(nbr_vec *v, float d2, int idx) {
  if (v->n == v->cap) {
    v->cap = v->cap ? 2 * v->cap : 64;
    v->v = (nbr *)realloc(v->v, v->cap * sizeof(nbr));
  }
  v->v[v->n].d2 = d2;
  v->v[v->n].idx = idx;
  v->n++;
}

/* radiusSearch: spatial_hashing.cpp:110-168, with the gather-filter of
 * rvv_common.cpp:49-68 (d2 = dx*dx + dy*dy + dz*dz, keep d2 <= r2). */
static size_t hash_radius(const rvo_hash *h, const float *x, const float *y,
                          const float *z, float qx, float qy, float qz,
                          float radius, int max_nn, nbr_vec *out) {
  out->n = 0;
  if (h->nb == 0) return 0;
  const float r2 = radius * radius;
  int qix, qiy, qiz;
  cell_of(h, qx, qy, qz, &qix, &qiy, &qiz);
  const int R = (int)ceilf(radius / h->cell) + 1;
  for (int dx = -R; dx <= R; ++dx)
    for (int dy = -R; dy <= R; ++dy)
      for (int dz = -R; dz <= R; ++dz) {
        long b = find_bucket(h, hash_cell(h, qix + dx, qiy + dy, qiz + dz));
        if (b < 0) continue;
        for (size_t t = h->bstart[b]; t < h->bstart[b + 1]; ++t) {
          int j = h->order[t];
          float ex = x[j] - qx, ey = y[j] - qy, ez = z[j] - qz;
          float d2 = ex * ex + ey * ey + ez * ez;
          if (d2 <= r2) nv_push(out, d2, j);
        }
      }
  if (out->n) qsort(out->v, out->n, sizeof(nbr), cmp_nbr);
  if (max_nn > 0 && out->n > (size_t)max_nn) out->n = (size_t)max_nn;
  return out->n;
}

long long rvo_hash_radius_search(const float *x, const float *y, const float *z,
                                 size_t n, float cell, int64_t p1, int64_t p2,
                                 const float *qx, const float *qy,
                                 const float *qz, size_t nq, float radius,
                                 int max_nn, long long *offsets, int *idx,
                                 float *d2, long long cap) {
  rvo_hash h;
  hash_build(&h, x, y, z, n, cell, p1, p2);
  nbr_vec v = {0, 0, 0};
  long long tot = 0;
  int overflow = 0;
  offsets[0] = 0;
  for (size_t q = 0; q < nq; ++q) {
    size_t c = hash_radius(&h, x, y, z, qx[q], qy[q], qz[q], radius, max_nn, &v);
    if (!overflow && tot + (long long)c <= cap) {
      for (size_t t = 0; t < c; ++t) {
        idx[tot + t] = v.v[t].idx;
        d2[tot + t] = v.v[t].d2;
      }
    } else {
      overflow = 1;
    }
    tot += (long long)c;
    offsets[q + 1] = tot;
  }
  free(v.v);
  hash_free(&h);
  return overflow ? -1 : tot;
}

/* ------------------------------------------------------------------------ */
/* Voxel grid: voxel_grid_downsamp_sc (voxel_grid_downsamp.cpp:183-213)     */
/* ------------------------------------------------------------------------ */

typedef struct {
  int vx, vy, vz, idx;
} vkey;

/* std::map<std::tuple<int,int,int>> order, then input order (stable). */
static int cmp_vkey(const void *a, const void *b) {
  const vkey *p = (const vkey *)a, *q = (const vkey *)b;
  if (p->vx != q->vx) return p->vx < q->vx ? -1 : 1;
  if (p->vy != q->vy) return p->vy < q->vy ? -1 : 1;
  if (p->vz != q->vz) return p->vz < q->vz ? -1 : 1;
  return p->idx < q->idx ? -1 : (p->idx > q->idx);
}

size_t rvo_voxel_grid(const float *x, const float *y, const float *z, size_t n,
                      float leaf, float *out, int *keys) {
  if (n == 0) return 0;
  const float inv_leaf = 1.0f / leaf;
  vkey *k = (vkey *)malloc(n * sizeof(vkey));
  for (size_t i = 0; i < n; ++i) {
    k[i].vx = (int)floorf(x[i] * inv_leaf);
    k[i].vy = (int)floorf(y[i] * inv_leaf);
    k[i].vz = (int)floorf(z[i] * inv_leaf);
    k[i].idx = (int)i;
  }
  qsort(k, n, sizeof(vkey), cmp_vkey);
  size_t count = 0;
  size_t s = 0;
  while (s < n) {
    size_t e = s + 1;
    while (e < n && k[e].vx == k[s].vx && k[e].vy == k[s].vy && k[e].vz == k[s].vz) ++e;
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    for (size_t t = s; t < e; ++t) {
      sx += x[k[t].idx];
      sy += y[k[t].idx];
      sz += z[k[t].idx];
    }
    const float f = 1.0f / (float)(int)(e - s);
    out[3 * count + 0] = sx * f;
    out[3 * count + 1] = sy * f;
    out[3 * count + 2] = sz * f;
    if (keys) {
      keys[3 * count + 0] = k[s].vx;
      keys[3 * count + 1] = k[s].vy;
      keys[3 * count + 2] = k[s].vz;
    }
    ++count;
    s = e;
  }
  free(k);
  return count;
}

/* ------------------------------------------------------------------------ */
/* Statistical outlier removal                                              */
/* ------------------------------------------------------------------------ */

/* Global statistics and ordered copy-out: statistical_outlier_removal.cpp
 * :43-62 (sor_sc) and :193-218 (filter_by_mean_dists); both evaluate the
 * same float expressions, sequentially over i. */
static size_t sor_filter(const float *x, const float *y, const float *z,
                         size_t n, const float *mean_dists, float alpha,
                         float *out, unsigned char *keep) {
  float global_sum = 0.0f;
  for (size_t i = 0; i < n; ++i) global_sum += mean_dists[i];
  const float global_mean = global_sum / (float)n;
  float variance_sum = 0.0f;
  for (size_t i = 0; i < n; ++i) {
    const float diff = mean_dists[i] - global_mean;
    variance_sum += diff * diff;
  }
  const float global_std = sqrtf(variance_sum / (float)n);
  const float thresh = global_mean + alpha * global_std;
  size_t count = 0;
  for (size_t i = 0; i < n; ++i) {
    const int kp = mean_dists[i] <= thresh;
    if (keep) keep[i] = (unsigned char)kp;
    if (kp) {
      if (out) {
        out[3 * count + 0] = x[i];
        out[3 * count + 1] = y[i];
        out[3 * count + 2] = z[i];
      }
      ++count;
    }
  }
  return count;
}

/* ------------------------------------------------------------------------ */
/* Row-parallel driver for the brute-force searches: every query's result is  */
/* independent of the others, so the rows are split over threads (count from  */
/* RVO_THREADS, else the online cores); the arithmetic of each row stays the  */
/* sequential restatement.                                                    */
/* ------------------------------------------------------------------------ */
typedef void (*row_fn)(void *job, size_t lo, size_t hi);
typedef struct {
  row_fn fn;
  void *job;
  size_t n;
  size_t next; /* next unclaimed row, taken in chunks under the lock */
  pthread_mutex_t lock;
} par_ctx;

static void *par_worker(void *arg) {
  par_ctx *c = (par_ctx *)arg;
  const size_t chunk = 64;
  for (;;) {
    pthread_mutex_lock(&c->lock);
    const size_t lo = c->next;
    c->next = lo + chunk < c->n ? lo + chunk : c->n;
    const size_t hi = c->next;
    pthread_mutex_unlock(&c->lock);
    if (lo >= hi) return NULL;
    c->fn(c->job, lo, hi);
  }
}

static void run_parallel(size_t n, row_fn fn, void *job) {
  long t = 0;
  const char *env = getenv("RVO_THREADS");
  if (env) t = strtol(env, NULL, 10);
  if (t <= 0) t = sysconf(_SC_NPROCESSORS_ONLN);
  if (t < 1) t = 1;
  if (t > 256) t = 256;
  if ((size_t)t > n / 64 + 1) t = (long)(n / 64 + 1);
  par_ctx c = {fn, job, n, 0, PTHREAD_MUTEX_INITIALIZER};
  pthread_t th[256];
  long started = 0;
  for (long i = 1; i < t; ++i)
    if (pthread_create(&th[started], NULL, par_worker, &c) == 0) ++started;
  par_worker(&c);
  for (long i = 0; i < started; ++i) pthread_join(th[i], NULL);
}

typedef struct {
  const float *x, *y, *z;
  size_t n;
  int k;
  float *md;
} sor_job;

static void sor_rows(void *arg, size_t lo, size_t hi) {
  const sor_job *J = (const sor_job *)arg;
  const float *x = J->x, *y = J->y, *z = J->z;
  const size_t n = J->n;
  const int k = J->k, kk = k + 1;
  float *best = (float *)malloc((size_t)kk * sizeof(float));
  for (size_t i = lo; i < hi; ++i) {
    int cnt = 0;
    for (size_t j = 0; j < n; ++j) {
      const float dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
      const float d = dx * dx + dy * dy + dz * dz;
      if (cnt == kk && !(d < best[kk - 1])) continue;
      int p = cnt < kk ? cnt++ : kk - 1;
      while (p > 0 && d < best[p - 1]) {
        best[p] = best[p - 1];
        --p;
      }
      best[p] = d;
    }
    float sum = 0.0f;
    for (int j = 1; j <= k; ++j) sum += sqrtf(best[j]);
    J->md[i] = sum / (float)k;
  }
  free(best);
}

/* sor_sc (statistical_outlier_removal.cpp:19-63): the k+1 smallest d2 over
 * all n points (self included), then mean of sqrt over ranks 1..k. */
size_t rvo_sor_exact(const float *x, const float *y, const float *z, size_t n,
                     int k, float alpha, float *out, float *mean_dists,
                     unsigned char *keep) {
  if (n == 0) return 0;
  if (k < 1 || (size_t)k + 1 > n) return 0; /* reference: partial_sort past end */
  float *md = mean_dists ? mean_dists : (float *)malloc(n * sizeof(float));
  sor_job job = {x, y, z, n, k, md};
  run_parallel(n, sor_rows, &job);
  size_t c = sor_filter(x, y, z, n, md, alpha, out, keep);
  if (!mean_dists) free(md);
  return c;
}

/* sor_spatial_hash (statistical_outlier_removal.cpp:246-270). */
size_t rvo_sor_radius(const float *x, const float *y, const float *z, size_t n,
                      float cell, int k, float alpha, float search_radius,
                      float *out, float *mean_dists, unsigned char *keep) {
  if (n == 0) return 0;
  rvo_hash h;
  hash_build(&h, x, y, z, n, cell, 73856093LL, 19349663LL);
  float *md = mean_dists ? mean_dists : (float *)malloc(n * sizeof(float));
  nbr_vec v = {0, 0, 0};
  for (size_t i = 0; i < n; ++i) {
    size_t c = hash_radius(&h, x, y, z, x[i], y[i], z[i], search_radius, k + 1, &v);
    if (c > 1) {
      const int valid_k = k < (int)c - 1 ? k : (int)c - 1;
      float sum = 0.0f;
      for (int j = 1; j <= valid_k; ++j) sum += sqrtf(v.v[j].d2);
      md[i] = sum / (float)valid_k;
    } else {
      md[i] = search_radius;
    }
  }
  free(v.v);
  hash_free(&h);
  size_t c = sor_filter(x, y, z, n, md, alpha, out, keep);
  if (!mean_dists) free(md);
  return c;
}

/* ------------------------------------------------------------------------ */
/* Normals                                                                  */
/* ------------------------------------------------------------------------ */

/* simple_eigen3x3_smallest (normal_estimation.cpp:16-52), float. The
 * rotation updates only A[p][p], A[q][q] and A[p][q], as the reference does. */
static void eigen_smallest_f(float cov[3][3], float *nx, float *ny, float *nz,
                             int iters) {
  float A[3][3], V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  memcpy(A, cov, sizeof(A));
  for (int it = 0; it < iters; ++it) {
    int p = 0, q = 1;
    float max_off = fabsf(A[0][1]);
    if (fabsf(A[0][2]) > max_off) { p = 0; q = 2; max_off = fabsf(A[0][2]); }
    if (fabsf(A[1][2]) > max_off) { p = 1; q = 2; }
    const float phi = 0.5f * atan2f(2 * A[p][q], A[p][p] - A[q][q]);
    const float c = cosf(phi), s = sinf(phi);
    const float app = A[p][p], aqq = A[q][q], apq = A[p][q];
    A[p][p] = c * c * app - 2 * s * c * apq + s * s * aqq;
    A[q][q] = s * s * app + 2 * s * c * apq + c * c * aqq;
    A[p][q] = 0;
    for (int r = 0; r < 3; ++r) {
      const float vip = V[r][p], viq = V[r][q];
      V[r][p] = c * vip - s * viq;
      V[r][q] = s * vip + c * viq;
    }
  }
  int m = 0;
  if (A[1][1] < A[m][m]) m = 1;
  if (A[2][2] < A[m][m]) m = 2;
  *nx = V[0][m];
  *ny = V[1][m];
  *nz = V[2][m];
}

static void eigen_smallest_d(double cov[3][3], double *nx, double *ny,
                             double *nz, int iters) {
  double A[3][3], V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  memcpy(A, cov, sizeof(A));
  for (int it = 0; it < iters; ++it) {
    int p = 0, q = 1;
    double max_off = fabs(A[0][1]);
    if (fabs(A[0][2]) > max_off) { p = 0; q = 2; max_off = fabs(A[0][2]); }
    if (fabs(A[1][2]) > max_off) { p = 1; q = 2; }
    const double phi = 0.5 * atan2(2 * A[p][q], A[p][p] - A[q][q]);
    const double c = cos(phi), s = sin(phi);
    const double app = A[p][p], aqq = A[q][q], apq = A[p][q];
    A[p][p] = c * c * app - 2 * s * c * apq + s * s * aqq;
    A[q][q] = s * s * app + 2 * s * c * apq + c * c * aqq;
    A[p][q] = 0;
    for (int r = 0; r < 3; ++r) {
      const double vip = V[r][p], viq = V[r][q];
      V[r][p] = c * vip - s * viq;
      V[r][q] = s * vip + c * viq;
    }
  }
  int m = 0;
  if (A[1][1] < A[m][m]) m = 1;
  if (A[2][2] < A[m][m]) m = 2;
  *nx = V[0][m];
  *ny = V[1][m];
  *nz = V[2][m];
}

/* flipNormalTowardsViewpoint (normal_estimation.cpp:55-67). */
static void flip_f(float px, float py, float pz, float vpx, float vpy,
                   float vpz, float *nx, float *ny, float *nz) {
  const float vx = vpx - px, vy = vpy - py, vz = vpz - pz;
  const float dot = vx * *nx + vy * *ny + vz * *nz;
  if (dot < 0) {
    *nx = -*nx;
    *ny = -*ny;
    *nz = -*nz;
  }
}

static void flip_d(double px, double py, double pz, double vpx, double vpy,
                   double vpz, double *nx, double *ny, double *nz) {
  const double vx = vpx - px, vy = vpy - py, vz = vpz - pz;
  const double dot = vx * *nx + vy * *ny + vz * *nz;
  if (dot < 0) {
    *nx = -*nx;
    *ny = -*ny;
    *nz = -*nz;
  }
}

/* Covariance of a neighbour list: compute_covariance_rvv
 * (normal_estimation.cpp:117-142) when div_centroid == 0 (centroid scaled by
 * 1.0f/n), normal_estimation_sc (:141-158) when div_centroid != 0 (divided by
 * n). Then eigen + flip. */
static void normal_from_list_f(const float *x, const float *y, const float *z,
                               const nbr *l, size_t m, int div_centroid,
                               float px, float py, float pz, float vpx,
                               float vpy, float vpz, int iters, float *nx,
                               float *ny, float *nz) {
  float cx = 0, cy = 0, cz = 0;
  for (size_t t = 0; t < m; ++t) {
    cx += x[l[t].idx];
    cy += y[l[t].idx];
    cz += z[l[t].idx];
  }
  if (div_centroid) {
    cx /= (float)(int)m;
    cy /= (float)(int)m;
    cz /= (float)(int)m;
  } else {
    const float inv_n = 1.0f / (float)m;
    cx *= inv_n;
    cy *= inv_n;
    cz *= inv_n;
  }
  float c00 = 0, c01 = 0, c02 = 0, c11 = 0, c12 = 0, c22 = 0;
  for (size_t t = 0; t < m; ++t) {
    const float dx = x[l[t].idx] - cx, dy = y[l[t].idx] - cy, dz = z[l[t].idx] - cz;
    c00 += dx * dx; c01 += dx * dy; c02 += dx * dz;
    c11 += dy * dy; c12 += dy * dz;
    c22 += dz * dz;
  }
  float cov[3][3] = {{c00, c01, c02}, {c01, c11, c12}, {c02, c12, c22}};
  eigen_smallest_f(cov, nx, ny, nz, iters);
  flip_f(px, py, pz, vpx, vpy, vpz, nx, ny, nz);
}

static void normal_from_list_d(const float *x, const float *y, const float *z,
                               const nbr *l, size_t m, int div_centroid,
                               float px, float py, float pz, float vpx,
                               float vpy, float vpz, int iters, float *nx,
                               float *ny, float *nz) {
  double cx = 0, cy = 0, cz = 0;
  for (size_t t = 0; t < m; ++t) {
    cx += x[l[t].idx];
    cy += y[l[t].idx];
    cz += z[l[t].idx];
  }
  (void)div_centroid;
  cx /= (double)m;
  cy /= (double)m;
  cz /= (double)m;
  double c00 = 0, c01 = 0, c02 = 0, c11 = 0, c12 = 0, c22 = 0;
  for (size_t t = 0; t < m; ++t) {
    const double dx = x[l[t].idx] - cx, dy = y[l[t].idx] - cy, dz = z[l[t].idx] - cz;
    c00 += dx * dx; c01 += dx * dy; c02 += dx * dz;
    c11 += dy * dy; c12 += dy * dz;
    c22 += dz * dz;
  }
  double cov[3][3] = {{c00, c01, c02}, {c01, c11, c12}, {c02, c12, c22}};
  double ax, ay, az;
  eigen_smallest_d(cov, &ax, &ay, &az, iters);
  flip_d(px, py, pz, vpx, vpy, vpz, &ax, &ay, &az);
  *nx = (float)ax;
  *ny = (float)ay;
  *nz = (float)az;
}

/* normal_estimation_rvv(in, const SpatialHash&, ...) (normal_estimation.cpp
 * :189-214): radius neighbours sorted by (d2, idx); fewer than 3 -> zero. */
void rvo_normals_radius(const float *x, const float *y, const float *z,
                        size_t n, float cell, float radius, float vpx,
                        float vpy, float vpz, int iters, int use_f64,
                        float *nx, float *ny, float *nz) {
  if (n == 0) return;
  rvo_hash h;
  hash_build(&h, x, y, z, n, cell, 73856093LL, 19349663LL);
  nbr_vec v = {0, 0, 0};
  for (size_t i = 0; i < n; ++i) {
    size_t m = hash_radius(&h, x, y, z, x[i], y[i], z[i], radius, 0, &v);
    if (m < 3) {
      nx[i] = ny[i] = nz[i] = 0;
      continue;
    }
    if (use_f64)
      normal_from_list_d(x, y, z, v.v, m, 0, x[i], y[i], z[i], vpx, vpy, vpz,
                         iters, nx + i, ny + i, nz + i);
    else
      normal_from_list_f(x, y, z, v.v, m, 0, x[i], y[i], z[i], vpx, vpy, vpz,
                         iters, nx + i, ny + i, nz + i);
  }
  free(v.v);
  hash_free(&h);
}

/* k+1 nearest of point i over all points, ordered by (d2, idx). */
static void knn_brute(const float *x, const float *y, const float *z, size_t n,
                      size_t i, int kk, nbr *best) {
  int cnt = 0;
  for (size_t j = 0; j < n; ++j) {
    const float dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
    nbr c;
    c.d2 = dx * dx + dy * dy + dz * dz;
    c.idx = (int)j;
    if (cnt == kk && cmp_nbr(&c, &best[kk - 1]) >= 0) continue;
    int p = cnt < kk ? cnt++ : kk - 1;
    while (p > 0 && cmp_nbr(&c, &best[p - 1]) < 0) {
      best[p] = best[p - 1];
      --p;
    }
    best[p] = c;
  }
}

typedef struct {
  const float *x, *y, *z;
  size_t n;
  int kk;
  float vpx, vpy, vpz;
  int iters, use_f64;
  float *nx, *ny, *nz; /* normals, or */
  int *idx;            /* the lists themselves (n * kk) */
  float *d2;
} normals_job;

static void normals_rows(void *arg, size_t lo, size_t hi) {
  const normals_job *J = (const normals_job *)arg;
  const float *x = J->x, *y = J->y, *z = J->z;
  const int kk = J->kk;
  nbr *best = (nbr *)malloc((size_t)kk * sizeof(nbr));
  for (size_t i = lo; i < hi; ++i) {
    knn_brute(x, y, z, J->n, i, kk, best);
    if (J->idx) {
      for (int t = 0; t < kk; ++t) {
        J->idx[i * (size_t)kk + t] = best[t].idx;
        J->d2[i * (size_t)kk + t] = best[t].d2;
      }
    } else if (J->use_f64) {
      normal_from_list_d(x, y, z, best, (size_t)kk, 1, x[i], y[i], z[i], J->vpx, J->vpy,
                         J->vpz, J->iters, J->nx + i, J->ny + i, J->nz + i);
    } else {
      normal_from_list_f(x, y, z, best, (size_t)kk, 1, x[i], y[i], z[i], J->vpx, J->vpy,
                         J->vpz, J->iters, J->nx + i, J->ny + i, J->nz + i);
    }
  }
  free(best);
}

/* normal_estimation_sc (normal_estimation.cpp:72-112). The reference's
 * partial_sort leaves the order of equal distances unspecified; this
 * restatement (and the GPU path) breaks ties by index. */
void rvo_normals_knn(const float *x, const float *y, const float *z, size_t n,
                     int k, float vpx, float vpy, float vpz, int iters,
                     int use_f64, float *nx, float *ny, float *nz) {
  if (n == 0) return;
  const int kk = k + 1;
  if ((size_t)kk > n) return;
  normals_job job = {x, y, z, n, kk, vpx, vpy, vpz, iters, use_f64, nx, ny, nz, NULL, NULL};
  run_parallel(n, normals_rows, &job);
}

/* The k+1 nearest of every point (self included) by brute force, ordered by
 * (d2, idx): the neighbour sets normal_estimation_sc (normal_estimation.cpp:
 * 79-88) selects, with ties broken by index. idx/d2: n * (k+1) each. */
void rvo_knn_lists(const float *x, const float *y, const float *z, size_t n,
                   int kk, int *idx, float *d2) {
  if (n == 0 || kk < 1 || (size_t)kk > n) return;
  normals_job job = {x, y, z, n, kk, 0, 0, 0, 0, 0, NULL, NULL, NULL, idx, d2};
  run_parallel(n, normals_rows, &job);
}

/* Cyclic Jacobi on a symmetric 3x3 (double), iterated until the off-diagonal
 * mass is negligible; the textbook two-sided rotation (all entries updated). */
static void jacobi_converged(double A[3][3], double V[3][3], double ev[3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) V[i][j] = (i == j);
  for (int sweep = 0; sweep < 64; ++sweep) {
    const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    const double dia = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
    if (off <= 1e-36 * dia || off == 0.0) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (A[p][q] == 0.0) continue;
        const double theta = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
        const double t = (theta >= 0 ? 1.0 : -1.0) /
                         (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int r = 0; r < 3; ++r) {
          const double arp = A[r][p], arq = A[r][q];
          A[r][p] = c * arp - s * arq;
          A[r][q] = s * arp + c * arq;
        }
        for (int r = 0; r < 3; ++r) {
          const double apr = A[p][r], aqr = A[q][r];
          A[p][r] = c * apr - s * aqr;
          A[q][r] = s * apr + c * aqr;
        }
        for (int r = 0; r < 3; ++r) {
          const double vrp = V[r][p], vrq = V[r][q];
          V[r][p] = c * vrp - s * vrq;
          V[r][q] = s * vrp + c * vrq;
        }
      }
  }
  for (int i = 0; i < 3; ++i) ev[i] = A[i][i];
}

void rvo_normals_knn_exact_f64(const float *x, const float *y, const float *z,
                               size_t n, const int *nbr_idx, int kk, float vpx,
                               float vpy, float vpz, double *nx, double *ny,
                               double *nz, double *cond) {
  for (size_t i = 0; i < n; ++i) {
    const int *l = nbr_idx + i * (size_t)kk;
    double cx = 0, cy = 0, cz = 0;
    for (int t = 0; t < kk; ++t) {
      cx += x[l[t]];
      cy += y[l[t]];
      cz += z[l[t]];
    }
    cx /= kk;
    cy /= kk;
    cz /= kk;
    double A[3][3] = {{0}};
    for (int t = 0; t < kk; ++t) {
      const double d[3] = {x[l[t]] - cx, y[l[t]] - cy, z[l[t]] - cz};
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) A[a][b] += d[a] * d[b];
    }
    double V[3][3], ev[3];
    jacobi_converged(A, V, ev);
    int m = 0, M = 0;
    for (int a = 1; a < 3; ++a) {
      if (ev[a] < ev[m]) m = a;
      if (ev[a] > ev[M]) M = a;
    }
    double ax = V[0][m], ay = V[1][m], az = V[2][m];
    const double nrm = sqrt(ax * ax + ay * ay + az * az);
    ax /= nrm;
    ay /= nrm;
    az /= nrm;
    flip_d(x[i], y[i], z[i], vpx, vpy, vpz, &ax, &ay, &az);
    nx[i] = ax;
    ny[i] = ay;
    nz[i] = az;
    if (cond) {
      const double lo = fabs(ev[m]);
      cond[i] = lo > 0 ? fabs(ev[M]) / lo : INFINITY;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* RANSAC plane                                                             */
/* ------------------------------------------------------------------------ */

/* compute_plane_coefficients (ransac_plane.cpp:18-50). */
static int plane_coeffs(float x1, float y1, float z1, float x2, float y2,
                        float z2, float x3, float y3, float z3, float *m,
                        float collinear) {
  const float v1x = x2 - x1, v1y = y2 - y1, v1z = z2 - z1;
  const float v2x = x3 - x1, v2y = y3 - y1, v2z = z3 - z1;
  float a = v1y * v2z - v1z * v2y;
  float b = v1z * v2x - v1x * v2z;
  float c = v1x * v2y - v1y * v2x;
  const float norm = sqrtf(a * a + b * b + c * c);
  if (norm < collinear) return 0;
  a /= norm;
  b /= norm;
  c /= norm;
  const float d = -(a * x1 + b * y1 + c * z1);
  m[0] = a;
  m[1] = b;
  m[2] = c;
  m[3] = d;
  return 1;
}

/* ransac_plane_sc (ransac_plane.cpp:55-111). rand_stream replaces the
 * srand(0)/rand() calls (three per iteration, consumed even when the
 * iteration is skipped). */
int rvo_ransac_plane(const float *x, const float *y, const float *z, size_t n,
                     float thresh, int max_iters, float collinear, float prob,
                     const int *rand_stream, float *model, int *counts,
                     float *models, int *iters_run) {
  if (iters_run) *iters_run = 0;
  if (n < 3) return 0;
  double pc = (double)prob;
  if (pc < 0.5) pc = 0.5;
  if (pc > 0.9999) pc = 0.9999;
  const double log_p = log(1.0 - pc);
  int best = 0;
  float best_model[4] = {0, 0, 0, 0};
  int k_iters = max_iters;
  int iter = 0;
  /* Per-hypothesis counts are evaluated for all max_iters hypotheses so a
   * caller can compare them; the replay below reads them in order. */
  if (counts || models) {
    for (int it = 0; it < max_iters; ++it) {
      const int i1 = (int)((size_t)rand_stream[3 * it + 0] % n);
      const int i2 = (int)((size_t)rand_stream[3 * it + 1] % n);
      const int i3 = (int)((size_t)rand_stream[3 * it + 2] % n);
      float m[4] = {0, 0, 0, 0};
      int cnt;
      if (i1 == i2 || i1 == i3 || i2 == i3) {
        cnt = -1;
      } else if (!plane_coeffs(x[i1], y[i1], z[i1], x[i2], y[i2], z[i2], x[i3],
                               y[i3], z[i3], m, collinear)) {
        cnt = -2;
      } else {
        cnt = 0;
        for (size_t i = 0; i < n; ++i) {
          const float dist = fabsf(m[0] * x[i] + m[1] * y[i] + m[2] * z[i] + m[3]);
          if (dist <= thresh) cnt++;
        }
      }
      if (counts) counts[it] = cnt;
      if (models) memcpy(models + 4 * it, m, sizeof(m));
    }
  }
  for (iter = 0; iter < k_iters && iter < max_iters; ++iter) {
    const int i1 = (int)((size_t)rand_stream[3 * iter + 0] % n);
    const int i2 = (int)((size_t)rand_stream[3 * iter + 1] % n);
    const int i3 = (int)((size_t)rand_stream[3 * iter + 2] % n);
    if (i1 == i2 || i1 == i3 || i2 == i3) continue;
    float m[4];
    if (!plane_coeffs(x[i1], y[i1], z[i1], x[i2], y[i2], z[i2], x[i3], y[i3],
                      z[i3], m, collinear))
      continue;
    int cur = 0;
    for (size_t i = 0; i < n; ++i) {
      const float dist = fabsf(m[0] * x[i] + m[1] * y[i] + m[2] * z[i] + m[3]);
      if (dist <= thresh) cur++;
    }
    if (cur > best) {
      best = cur;
      memcpy(best_model, m, sizeof(m));
      const double w = (double)best / (double)n;
      double p_no = 1.0 - pow(w, 3.0);
      if (p_no < DBL_EPSILON) p_no = DBL_EPSILON;
      if (p_no > 1.0 - DBL_EPSILON) p_no = 1.0 - DBL_EPSILON;
      const double log_no = log(p_no);
      if (fabs(log_no) > 1e-7) {
        const int dyn = (int)ceil(log_p / log_no);
        if (dyn > 0 && dyn < k_iters) k_iters = dyn;
      }
    }
  }
  if (iters_run) *iters_run = iter;
  memcpy(model, best_model, sizeof(best_model));
  return best;
}

/* extract_plane_inliers_outliers_rvv, scalar branch (ransac_plane.cpp
 * :373-381): inlier iff -t <= a*x + b*y + c*z + d <= t. */
void rvo_extract_plane(const float *x, const float *y, const float *z,
                       size_t n, const float *model, float thresh,
                       float *inliers, float *outliers, size_t *n_in,
                       size_t *n_out) {
  const float a = model[0], b = model[1], c = model[2], d = model[3];
  size_t ni = 0, no = 0;
  for (size_t j = 0; j < n; ++j) {
    const float dist = a * x[j] + b * y[j] + c * z[j] + d;
    float *dst;
    if (dist >= -thresh && dist <= thresh)
      dst = inliers ? inliers + 3 * ni : 0, ++ni;
    else
      dst = outliers ? outliers + 3 * no : 0, ++no;
    if (dst) {
      dst[0] = x[j];
      dst[1] = y[j];
      dst[2] = z[j];
    }
  }
  *n_in = ni;
  *n_out = no;
}

/* ------------------------------------------------------------------------ */
/* Euclidean clustering                                                     */
/* ------------------------------------------------------------------------ */
static int cmp_int(const void *a, const void *b) {
  const int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

/* euclidean_clustering.cpp:113-189 with radiusQueryUnvisited's scalar branch
 * (:88-98): neighbours of the current point are the unvisited points with
 * ((px - qx)^2 + (py - qy)^2) + (pz - qz)^2 <= tol^2, in index order, pushed
 * to a FIFO queue; a cluster is every point the BFS from a seed reaches. */
long rvo_euclidean_clusters(const float *x, const float *y, const float *z, size_t n,
                            float tolerance, int min_size, int max_size, long long *offsets,
                            int *indices) {
  const float tol_sq = tolerance * tolerance;
  unsigned char *visited = calloc(n ? n : 1, 1);
  int *queue = malloc(sizeof(int) * (n ? n : 1));
  long n_cl = 0;
  long long o = 0;
  offsets[0] = 0;
  for (size_t seed = 0; seed < n; ++seed) {
    if (visited[seed]) continue;
    size_t head = 0, tail = 0;
    visited[seed] = 1;
    queue[tail++] = (int)seed;
    while (head < tail) {
      const int cur = queue[head++];
      const float qx = x[cur], qy = y[cur], qz = z[cur];
      for (size_t i = 0; i < n; ++i) {
        if (visited[i]) continue;
        const float dx = x[i] - qx, dy = y[i] - qy, dz = z[i] - qz;
        if (dx * dx + dy * dy + dz * dz <= tol_sq) {
          visited[i] = 1;
          queue[tail++] = (int)i;
        }
      }
    }
    /* the BFS order (queue[0..tail)) is the cluster's membership */
    const int sz = (int)tail;
    if (sz >= min_size && sz <= max_size) {
      memcpy(indices + o, queue, sizeof(int) * tail);
      qsort(indices + o, tail, sizeof(int), cmp_int);
      o += (long long)tail;
      offsets[++n_cl] = o;
    }
  }
  free(visited);
  free(queue);
  return n_cl;
}

/* ------------------------------------------------------------------------ */
/* Octree / PointerOctree                                                   */
/* ------------------------------------------------------------------------ */

/* Root box: octree.cpp:36-53 (min, max + eps) and pointer_octree.cpp:36-63
 * (min - eps, max + eps). */
static void oct_root(int kind, const float *x, const float *y, const float *z, size_t n,
                     float eps, float b[6]) {
  const float *c[3] = {x, y, z};
  for (int a = 0; a < 3; ++a) {
    float lo = FLT_MAX, hi = -FLT_MAX;
    for (size_t i = 0; i < n; ++i) {
      if (c[a][i] < lo) lo = c[a][i];
      if (c[a][i] > hi) hi = c[a][i];
    }
    b[a] = kind == 0 ? lo : lo - eps;
    b[3 + a] = hi + eps;
  }
}

/* buildParams (octree.cpp:59-94): a node with <= cap points, or at
 * max_depth, is a leaf; otherwise its points go to child
 * (x >= mid) | (y >= mid) << 1 | (z >= mid) << 2 in index order, with
 * mid = (min + max) * 0.5f per axis, and the children are visited 0..7. */
static void oct_split(const float *x, const float *y, const float *z, int *idx, int *tmp,
                      size_t cnt, const float b[6], int depth, size_t cap, int max_depth,
                      int *out, size_t *pos) {
  if (cnt <= cap || depth >= max_depth) {
    memcpy(out + *pos, idx, cnt * sizeof(int));
    *pos += cnt;
    return;
  }
  const float mx = (b[0] + b[3]) * 0.5f, my = (b[1] + b[4]) * 0.5f,
              mz = (b[2] + b[5]) * 0.5f;
  size_t count[8] = {0}, start[8];
  for (size_t t = 0; t < cnt; ++t) {
    const int i = idx[t];
    const int code = (x[i] >= mx) | ((y[i] >= my) << 1) | ((z[i] >= mz) << 2);
    count[code]++;
  }
  start[0] = 0;
  for (int c = 1; c < 8; ++c) start[c] = start[c - 1] + count[c - 1];
  size_t fill[8];
  memcpy(fill, start, sizeof(fill));
  for (size_t t = 0; t < cnt; ++t) {
    const int i = idx[t];
    const int code = (x[i] >= mx) | ((y[i] >= my) << 1) | ((z[i] >= mz) << 2);
    tmp[fill[code]++] = i;
  }
  memcpy(idx, tmp, cnt * sizeof(int));
  for (int c = 0; c < 8; ++c) {
    if (!count[c]) continue;
    float cb[6];
    cb[0] = (c & 1) ? mx : b[0];
    cb[3] = (c & 1) ? b[3] : mx;
    cb[1] = (c & 2) ? my : b[1];
    cb[4] = (c & 2) ? b[4] : my;
    cb[2] = (c & 4) ? mz : b[2];
    cb[5] = (c & 4) ? b[5] : mz;
    oct_split(x, y, z, idx + start[c], tmp + start[c], count[c], cb, depth + 1, cap,
              max_depth, out, pos);
  }
}

void rvo_octree_order(int kind, const float *x, const float *y, const float *z, size_t n,
                      int cap, int max_depth, float eps, int *order) {
  if (n == 0) return;
  float b[6];
  oct_root(kind, x, y, z, n, eps, b);
  int *idx = (int *)malloc(n * sizeof(int)), *tmp = (int *)malloc(n * sizeof(int));
  for (size_t i = 0; i < n; ++i) idx[i] = (int)i;
  size_t pos = 0;
  /* (size_t)max_points_per_leaf_, as the reference compares */
  oct_split(x, y, z, idx, tmp, n, b, 0, (size_t)(long long)cap, max_depth, order, &pos);
  free(idx);
  free(tmp);
}

long long rvo_octree_radius_search(int kind, const float *x, const float *y, const float *z,
                                   size_t n, int cap_leaf, int max_depth, float eps,
                                   const float *qx, const float *qy, const float *qz,
                                   size_t nq, float radius, long long *offsets, int *idx,
                                   float *d2, long long cap) {
  int *order = (int *)malloc((n ? n : 1) * sizeof(int));
  rvo_octree_order(kind, x, y, z, n, cap_leaf, max_depth, eps, order);
  const float r2 = radius * radius;
  long long tot = 0;
  offsets[0] = 0;
  for (size_t q = 0; q < nq; ++q) {
    for (size_t p = 0; p < n; ++p) {
      const int j = order[p];
      const float dx = x[j] - qx[q], dy = y[j] - qy[q], dz = z[j] - qz[q];
      const float d = dx * dx + dy * dy + dz * dz;
      if (d <= r2) {
        if (tot < cap) {
          idx[tot] = j;
          d2[tot] = d;
        }
        ++tot;
      }
    }
    offsets[q + 1] = tot;
  }
  free(order);
  return tot > cap ? -1 : tot;
}

/* --- std::nth_element (libstdc++ 13, bits/stl_algo.h / stl_heap.h) -------
 * Introselect: while the range holds more than 3 elements, move the median
 * of (first + 1, middle, last - 1) to first, partition the rest around it
 * (Hoare, unguarded) and keep the side holding nth; after 2 * floor(log2 n)
 * rounds fall back to a binary-heap selection of the nth + 1 smallest.
 * The last range is insertion-sorted. Only operator< is used. */
static void fswap(float *a, long i, long j) {
  const float t = a[i];
  a[i] = a[j];
  a[j] = t;
}

/* percolate v up from hole towards top in the max-heap a */
static void heap_up(float *a, long hole, long top, float v) {
  long parent = (hole - 1) / 2;
  while (hole > top && a[parent] < v) {
    a[hole] = a[parent];
    hole = parent;
    parent = (hole - 1) / 2;
  }
  a[hole] = v;
}

/* move the hole down to a leaf along the larger children, then put v in
 * by percolating it up (the bottom-up sift of libstdc++'s __adjust_heap) */
static void heap_adjust(float *a, long hole, long len, float v) {
  const long top = hole;
  long child = hole;
  while (child < (len - 1) / 2) {
    child = 2 * (child + 1);
    if (a[child] < a[child - 1]) child--;
    a[hole] = a[child];
    hole = child;
  }
  if ((len & 1) == 0 && child == (len - 2) / 2) {
    child = 2 * (child + 1);
    a[hole] = a[child - 1];
    hole = child - 1;
  }
  heap_up(a, hole, top, v);
}

static void heap_select(float *a, long middle, long last) {
  if (middle >= 2) {
    for (long parent = (middle - 2) / 2;; --parent) {
      heap_adjust(a, parent, middle, a[parent]);
      if (parent == 0) break;
    }
  }
  for (long i = middle; i < last; ++i) {
    if (a[i] < a[0]) {
      const float v = a[i];
      a[i] = a[0];
      heap_adjust(a, 0, middle, v);
    }
  }
}

int rvo_nth_element(float *a, size_t n, size_t nth) {
  if (n == 0 || nth >= n) return 0;
  long first = 0, last = (long)n;
  int lg = 0;
  while (((size_t)1 << (lg + 1)) <= n) ++lg;
  int depth = 2 * lg;
  while (last - first > 3) {
    if (depth == 0) {
      heap_select(a + first, (long)nth + 1 - first, last - first);
      fswap(a, first, (long)nth);
      return 1;
    }
    --depth;
    /* median of three to first */
    const long x = first + 1, y = first + (last - first) / 2, z = last - 1;
    if (a[x] < a[y]) {
      if (a[y] < a[z]) fswap(a, first, y);
      else if (a[x] < a[z]) fswap(a, first, z);
      else fswap(a, first, x);
    } else if (a[x] < a[z]) {
      fswap(a, first, x);
    } else if (a[y] < a[z]) {
      fswap(a, first, z);
    } else {
      fswap(a, first, y);
    }
    /* unguarded partition of [first + 1, last) around a[first] */
    long lo = first + 1, hi = last;
    for (;;) {
      while (a[lo] < a[first]) ++lo;
      --hi;
      while (a[first] < a[hi]) --hi;
      if (!(lo < hi)) break;
      fswap(a, lo, hi);
      ++lo;
    }
    if (lo <= (long)nth) first = lo;
    else last = lo;
  }
  for (long i = first + 1; i < last; ++i) {
    const float v = a[i];
    if (v < a[first]) {
      memmove(a + first + 1, a + first, (size_t)(i - first) * sizeof(float));
      a[first] = v;
    } else {
      long j = i;
      while (v < a[j - 1]) {
        a[j] = a[j - 1];
        --j;
      }
      a[j] = v;
    }
  }
  return 0;
}

static int cmp_f32(const void *a, const void *b) {
  const float p = *(const float *)a, q = *(const float *)b;
  return (p > q) - (p < q);
}

size_t rvo_sor_octree(int kind, const float *x, const float *y, const float *z, size_t n,
                      int cap_leaf, int max_depth, float eps, int k, float alpha,
                      float search_radius, float *out, float *mean_dists, unsigned char *keep) {
  if (n == 0) return 0;
  int *order = (int *)malloc(n * sizeof(int));
  rvo_octree_order(kind, x, y, z, n, cap_leaf, max_depth, eps, order);
  float *md = mean_dists ? mean_dists : (float *)malloc(n * sizeof(float));
  float *d = (float *)malloc(n * sizeof(float));
  const float r2 = search_radius * search_radius;
  for (size_t i = 0; i < n; ++i) {
    size_t c = 0;
    for (size_t p = 0; p < n; ++p) {
      const int j = order[p];
      const float dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
      const float v = dx * dx + dy * dy + dz * dz;
      if (v <= r2) d[c++] = v;
    }
    if (c > 1) {
      const int valid_k = k < (int)c - 1 ? k : (int)c - 1;
      if (kind == 0) qsort(d, c, sizeof(float), cmp_f32);
      else rvo_nth_element(d, c, (size_t)valid_k);
      float sum = 0.0f;
      for (int j = 1; j <= valid_k; ++j) sum += sqrtf(d[j]);
      md[i] = sum / (float)valid_k;
    } else {
      md[i] = search_radius;
    }
  }
  free(d);
  free(order);
  size_t kept = sor_filter(x, y, z, n, md, alpha, out, keep);
  if (!mean_dists) free(md);
  return kept;
}

void rvo_normals_octree(int kind, const float *x, const float *y, const float *z, size_t n,
                        int cap_leaf, int max_depth, float eps, float radius, float vpx,
                        float vpy, float vpz, int iters, float *nx, float *ny, float *nz) {
  if (n == 0) return;
  int *order = (int *)malloc(n * sizeof(int));
  rvo_octree_order(kind, x, y, z, n, cap_leaf, max_depth, eps, order);
  nbr *l = (nbr *)malloc(n * sizeof(nbr));
  const float r2 = radius * radius;
  for (size_t i = 0; i < n; ++i) {
    size_t m = 0;
    for (size_t p = 0; p < n; ++p) {
      const int j = order[p];
      const float dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
      const float v = dx * dx + dy * dy + dz * dz;
      if (v <= r2) {
        l[m].d2 = v;
        l[m].idx = j;
        ++m;
      }
    }
    if (m < 3) {
      nx[i] = ny[i] = nz[i] = 0;
      continue;
    }
    normal_from_list_f(x, y, z, l, m, 0, x[i], y[i], z[i], vpx, vpy, vpz, iters, nx + i,
                       ny + i, nz + i);
  }
  free(l);
  free(order);
}
