/*
 * psod_oracle.c -- CPU oracle for the SOD stage of Psod (test infrastructure).
 *
 * TEST INFRASTRUCTURE ONLY: the checker that tests/, smoke() and the CPU
 * baseline run against.  The product (psod_b200) never links it.
 *
 * A single-threaded C restatement of the 1-rank path of
 * sod/sod_profile_rdfof_parallel_hdf5.f90 ("main" below).  Every step
 * cites the Fortran lines it follows.  Parity is UNPINNED: the reference
 * has no golden vectors for this path and cannot be built here.
 *
 * Build with -O2 -ffp-contract=off -fno-fast-math: the Fortran reference
 * is built at -O0 (sod/Makefile_v2save:4) and never fuses multiply-adds.
 */
#include "psod_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define FIX_ONE ((double)(1ULL << PSOD_FIX_SHIFT))

/* ------------------------------------------------------------------ */
/* quick_sort  (main:2477-2571), 0-based.                              */
/* ------------------------------------------------------------------ */
static void qs_swap(double *list, int64_t *order, int64_t a, int64_t b) {
  double t = list[a];
  list[a] = list[b];
  list[b] = t;
  int64_t it = order[a];
  order[a] = order[b];
  order[b] = it;
}

/* interchange_sort (main:2552-2569) */
static void qs_interchange(double *list, int64_t *order, int64_t l,
                           int64_t r) {
  for (int64_t i = l; i <= r - 1; i++)
    for (int64_t j = i + 1; j <= r; j++)
      if (list[i] > list[j]) qs_swap(list, order, i, j);
}

/* quick_sort_1 (main:2502-2549).  The two recursive calls work on
 * disjoint ranges, so an explicit stack gives the same permutation. */
static void qs_range(double *list, int64_t *order, int64_t left,
                     int64_t right) {
  int64_t cap = 128, top = 0;
  int64_t *stk = (int64_t *)malloc(sizeof(int64_t) * 2 * cap);
  stk[top++] = left;
  stk[top++] = right;
  while (top > 0) {
    int64_t r = stk[--top];
    int64_t l = stk[--top];
    if (r < l + 6) { /* max_simple_sort_size = 6, main:2509-2513 */
      qs_interchange(list, order, l, r);
      continue;
    }
    /* 1-based (L+R)/2 maps to 0-based (l+r)/2 for l,r >= 0 */
    double reference = list[(l + r) / 2];
    int64_t i = l - 1, j = r + 1;
    for (;;) {
      do { i++; } while (!(list[i] >= reference));
      do { j--; } while (!(list[j] <= reference));
      if (i < j) {
        qs_swap(list, order, i, j);
      } else if (i == j) {
        i++;
        break;
      } else {
        break;
      }
    }
    if (top + 4 > 2 * cap) {
      cap *= 2;
      stk = (int64_t *)realloc(stk, sizeof(int64_t) * 2 * cap);
    }
    if (l < j) {
      stk[top++] = l;
      stk[top++] = j;
    }
    if (i < r) {
      stk[top++] = i;
      stk[top++] = r;
    }
  }
  free(stk);
}

void psod_oracle_quick_sort(double *list, int64_t *order, int64_t n) {
  for (int64_t i = 0; i < n; i++) order[i] = i;
  if (n > 0) qs_range(list, order, 0, n - 1);
}

/* Canonical order: ascending key, ties by ascending tie value (the
 * particle's original index), which is unique. */
typedef struct {
  double key;
  int64_t tie;
  int64_t pos;
} keytie_t;

static int keytie_cmp(const void *a, const void *b) {
  const keytie_t *x = (const keytie_t *)a, *y = (const keytie_t *)b;
  if (x->key < y->key) return -1;
  if (x->key > y->key) return 1;
  if (x->tie < y->tie) return -1;
  if (x->tie > y->tie) return 1;
  return 0;
}

/* Sort list[] in place and write the permutation (original positions) to
 * order[]: with the reference quicksort, or canonically by (key, tie[i])
 * where tie == NULL means tie[i] = i. */
static void sort_with_order(double *list, int64_t *order, int64_t n, int mode,
                            const int64_t *tie) {
  if (mode == PSOD_ORACLE_REFERENCE) {
    psod_oracle_quick_sort(list, order, n);
    return;
  }
  keytie_t *kt = (keytie_t *)malloc(sizeof(keytie_t) * (size_t)(n > 0 ? n : 1));
  for (int64_t i = 0; i < n; i++) {
    kt[i].key = list[i];
    kt[i].tie = tie ? tie[i] : i;
    kt[i].pos = i;
  }
  qsort(kt, (size_t)n, sizeof(keytie_t), keytie_cmp);
  for (int64_t i = 0; i < n; i++) {
    list[i] = kt[i].key;
    order[i] = kt[i].pos;
  }
  free(kt);
}

/* ------------------------------------------------------------------ */
/* Zone geometry (main:321-441, 665-668, 689-698, 738-739): zone nzone  */
/* of nxcpu^3, with its buffer.                                        */
/* ------------------------------------------------------------------ */
typedef struct {
  int32_t nx;       /* grid cells per side */
  int32_t nxcpu;    /* zones per axis */
  int32_t nxzone;   /* nx / nxcpu */
  int32_t nxbuffer; /* resolved buffer */
  double xmin[3], xmax[3]; /* zone + buffer per axis, box units */
  double xminzone[3], xmaxzone[3]; /* utile zone per axis, grid units (after *scale) */
  int64_t local_nx; /* spherover's local_nx = nxzone + 2*nxbuffer */
  int32_t nxcic;    /* 2*nx */
  double scale;     /* nx */
  float mpf;        /* 1/nparttotal as real(4), main:662 */
  float munit;      /* mpf*nparttotal back to real(4), main:685 */
} zone_t;

static int zone_setup(const psod_oracle_params *p, zone_t *z) {
  if (p->nx < 5 || p->ncut < 1 || 2 * p->ncut + 1 > p->nx || p->nmin < 10 ||
      p->nbins < 1 || p->nsel < 1 || p->npart_total < 1)
    return PSOD_ORACLE_ERR_ARG;
  const int32_t ncpu = p->nxcpu <= 0 ? 1 : p->nxcpu;
  if (p->nx % ncpu != 0 || p->nzone < 0 || (int64_t)p->nzone >= (int64_t)ncpu * ncpu * ncpu)
    return PSOD_ORACLE_ERR_ARG;
  z->nx = p->nx;
  z->nxcpu = ncpu;
  z->nxzone = p->nx / ncpu; /* main:349 */
  z->nxbuffer = p->nxbuffer;
  if (z->nxbuffer == 0) z->nxbuffer = z->nxzone / 2; /* main:380-381 */
  if (z->nxbuffer < p->ncut) return PSOD_ORACLE_ERR_ARG;     /* main:386 */
  if (ncpu == 1) {
    /* main:392 allows nxbuffer == nxzone; the CIC indices of the last half
     * cell then land in the reference's padding past the periodic grid,
     * which is not restated here */
    if (z->nxbuffer >= z->nxzone) return PSOD_ORACLE_ERR_ARG;
  } else {
    if (z->nxbuffer > z->nxzone) return PSOD_ORACLE_ERR_ARG; /* main:392 */
    /* a local grid shorter than the box by fewer than max(ncut, 2) cells
     * would let the wrapped cell walks land on its far side (refused, as
     * by the library) */
    const int64_t local = (int64_t)z->nxzone + 2 * (int64_t)z->nxbuffer;
    const int32_t reach = p->ncut > 2 ? p->ncut : 2;
    if (local < p->nx && local > p->nx - reach) return PSOD_ORACLE_ERR_ARG;
  }
  /* zone indices, main:344-346 */
  const int32_t iz3[3] = {p->nzone / (ncpu * ncpu), (p->nzone - (p->nzone / (ncpu * ncpu)) * ncpu * ncpu) / ncpu,
                          p->nzone % ncpu};
  double q = (double)z->nxbuffer / (double)z->nxzone;
  z->scale = (double)p->nx;                 /* main:689 */
  for (int a = 0; a < 3; a++) {
    z->xmin[a] = ((double)iz3[a] - q) / (double)ncpu;       /* main:401 */
    z->xmax[a] = ((double)iz3[a] + 1.0 + q) / (double)ncpu; /* main:402 */
    z->xminzone[a] = ((double)iz3[a] / (double)ncpu) * z->scale;         /* main:420, 691 */
    z->xmaxzone[a] = (((double)iz3[a] + 1.0) / (double)ncpu) * z->scale; /* main:421, 692 */
  }
  z->local_nx = (int64_t)z->nxzone + 2 * (int64_t)z->nxbuffer; /* main:739 */
  z->nxcic = 2 * p->nx;                     /* main:667 */
  z->mpf = (float)(1.0 / (double)p->npart_total);              /* main:662 */
  z->munit = (float)((double)z->mpf * (double)p->npart_total); /* main:685 */
  return PSOD_ORACLE_OK;
}

/* Periodic selection test of cic/cicm1 (main:1140-1148, 1309-1317). */
static int in_zone_periodic(double x, double lo, double hi) {
  return (x >= lo && x <= hi) || (x >= lo + 1.0 && x <= hi + 1.0) ||
         (x >= lo - 1.0 && x <= hi - 1.0);
}

/* CIC cell index and weights along one axis (main:1154-1190). */
static int cic_axis(float xf, double xxmin, double dx, int32_t nc, int32_t *i0,
                    int32_t *i1, double *dd, double *de) {
  double d = ((double)xf - xxmin) / dx;
  int32_t ix = (int32_t)d; /* Fortran int(): truncation */
  if (d < 0.0) ix = ix - 1;
  d = d - (double)ix;
  double e = 1.0 - d;
  int32_t ixp1 = ix + 1;
  if (ixp1 < 0) ixp1 = ixp1 + nc;
  if (ix < 0) ix = ix + nc;
  if (ixp1 >= nc) ixp1 = ixp1 - nc;
  if (ix >= nc) ix = ix - nc;
  if (ix < 0 || ix >= nc || ixp1 < 0 || ixp1 >= nc) return 0;
  *i0 = ix;
  *i1 = ixp1;
  *dd = d;
  *de = e;
  return 1;
}

/* ------------------------------------------------------------------ */
/* cic (main:1077-1265)                                                */
/* ------------------------------------------------------------------ */
int psod_oracle_cic(const psod_oracle_params *p, int64_t n, const float *pos,
                    int mode, double *grid) {
  zone_t z;
  int st = zone_setup(p, &z);
  if (st) return st;
  const int64_t nc = z.nxcic;
  const int64_t nnode = nc * nc * nc;
  const double dx = 1.0 / (double)nc; /* main:1126 */
  const double *xxmin = z.xmin;       /* main:665 */
  int64_t *fix = NULL;
  if (mode == PSOD_ORACLE_CANONICAL) {
    fix = (int64_t *)calloc((size_t)nnode, sizeof(int64_t));
    if (!fix) return PSOD_ORACLE_ERR_ARG;
  } else {
    memset(grid, 0, sizeof(double) * (size_t)nnode); /* main:1124 */
  }
  const double mpf = (double)z.mpf;
  for (int64_t i = 0; i < n; i++) {
    const float *x = pos + 3 * i;
    if (!(in_zone_periodic(x[0], z.xmin[0], z.xmax[0]) &&
          in_zone_periodic(x[1], z.xmin[1], z.xmax[1]) &&
          in_zone_periodic(x[2], z.xmin[2], z.xmax[2])))
      continue;
    int32_t ix, ixp, iy, iyp, iz, izp;
    double ddx, dex, ddy, dey, ddz, dez;
    if (!cic_axis(x[0], xxmin[0], dx, (int32_t)nc, &ix, &ixp, &ddx, &dex) ||
        !cic_axis(x[1], xxmin[1], dx, (int32_t)nc, &iy, &iyp, &ddy, &dey) ||
        !cic_axis(x[2], xxmin[2], dx, (int32_t)nc, &iz, &izp, &ddz, &dez)) {
      free(fix);
      return PSOD_ORACLE_ERR_ARG;
    }
    /* the eight corners in the reference's order, main:1196-1211 */
    const int32_t cx[8] = {ix, ixp, ix, ixp, ix, ixp, ix, ixp};
    const int32_t cy[8] = {iy, iy, iyp, iyp, iy, iy, iyp, iyp};
    const int32_t cz[8] = {iz, iz, iz, iz, izp, izp, izp, izp};
    const double wx[8] = {dex, ddx, dex, ddx, dex, ddx, dex, ddx};
    const double wy[8] = {dey, dey, ddy, ddy, dey, dey, ddy, ddy};
    const double wz[8] = {dez, dez, dez, dez, ddz, ddz, ddz, ddz};
    for (int c = 0; c < 8; c++) {
      int64_t node = (int64_t)cx[c] + nc * ((int64_t)cy[c] + nc * cz[c]);
      if (mode == PSOD_ORACLE_CANONICAL) {
        double w = (wx[c] * wy[c]) * wz[c];
        fix[node] += (int64_t)llrint(w * FIX_ONE);
      } else {
        grid[node] = grid[node] + ((mpf * wx[c]) * wy[c]) * wz[c];
      }
    }
  }
  const double vol = (dx * dx) * dx; /* dx*dy*dz, main:1263 */
  if (mode == PSOD_ORACLE_CANONICAL) {
    const double kc = (mpf / FIX_ONE) / vol;
    for (int64_t k = 0; k < nnode; k++) grid[k] = (double)fix[k] * kc;
    free(fix);
  } else {
    for (int64_t k = 0; k < nnode; k++) grid[k] = grid[k] / vol;
  }
  return PSOD_ORACLE_OK;
}

/* ------------------------------------------------------------------ */
/* cicm1 (main:1268-1390)                                              */
/* ------------------------------------------------------------------ */
int psod_oracle_cicm1(const psod_oracle_params *p, int64_t n,
                      const float *pos, const double *grid, double *rho) {
  zone_t z;
  int st = zone_setup(p, &z);
  if (st) return st;
  const int64_t nc = z.nxcic;
  const double dx = 1.0 / (double)nc;
  const double *xxmin = z.xmin;
  for (int64_t i = 0; i < n; i++) {
    const float *x = pos + 3 * i;
    rho[i] = 0.0;
    if (!(in_zone_periodic(x[0], z.xmin[0], z.xmax[0]) &&
          in_zone_periodic(x[1], z.xmin[1], z.xmax[1]) &&
          in_zone_periodic(x[2], z.xmin[2], z.xmax[2])))
      continue;
    int32_t ix, ixp, iy, iyp, iz, izp;
    double ddx, dex, ddy, dey, ddz, dez;
    if (!cic_axis(x[0], xxmin[0], dx, (int32_t)nc, &ix, &ixp, &ddx, &dex) ||
        !cic_axis(x[1], xxmin[1], dx, (int32_t)nc, &iy, &iyp, &ddy, &dey) ||
        !cic_axis(x[2], xxmin[2], dx, (int32_t)nc, &iz, &izp, &ddz, &dez))
      return PSOD_ORACLE_ERR_ARG;
    const int32_t cx[8] = {ix, ixp, ix, ixp, ix, ixp, ix, ixp};
    const int32_t cy[8] = {iy, iy, iyp, iyp, iy, iy, iyp, iyp};
    const int32_t cz[8] = {iz, iz, iz, iz, izp, izp, izp, izp};
    const double wx[8] = {dex, ddx, dex, ddx, dex, ddx, dex, ddx};
    const double wy[8] = {dey, dey, ddy, ddy, dey, dey, ddy, ddy};
    const double wz[8] = {dez, dez, dez, dez, ddz, ddz, ddz, ddz};
    double r = 0.0;
    for (int c = 0; c < 8; c++) { /* main:1368-1383, fixed term order */
      int64_t node = (int64_t)cx[c] + nc * ((int64_t)cy[c] + nc * cz[c]);
      r = r + ((grid[node] * wx[c]) * wy[c]) * wz[c];
    }
    rho[i] = r;
  }
  return PSOD_ORACLE_OK;
}

/* ------------------------------------------------------------------ */
/* tri_cic (main:998-1037)                                             */
/* ------------------------------------------------------------------ */
int psod_oracle_tri_cic(int64_t n, const double *rho, int mode,
                        int64_t *isort, int64_t *npart_new) {
  double *pdens = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  for (int64_t i = 0; i < n; i++) pdens[i] = 1.0 / rho[i]; /* main:1022 */
  sort_with_order(pdens, isort, n, mode, NULL);             /* main:1025 */
  int64_t i = 0;
  while (i < n && pdens[i] < 1.0 / 100.0) i++; /* main:1029-1031 */
  /* npart_new counts the first particle with 1/rho >= 0.01 (main:1032);
   * when every particle is denser the reference reads past the end, and
   * the count is clamped to n here. */
  *npart_new = (i < n) ? i + 1 : n;
  free(pdens);
  return PSOD_ORACLE_OK;
}

/* ------------------------------------------------------------------ */
/* spherover (main:1396-2201)                                          */
/* ------------------------------------------------------------------ */
typedef struct {
  int64_t n, cap;
  int64_t *v;
} vec64_t;

static void vpush(vec64_t *a, int64_t x) {
  if (a->n == a->cap) {
    a->cap = a->cap ? 2 * a->cap : 1024;
    a->v = (int64_t *)realloc(a->v, sizeof(int64_t) * a->cap);
  }
  a->v[a->n++] = x;
}

typedef struct {
  int64_t n, cap;
  double *v;
} vecd_t;

static void vpushd(vecd_t *a, double x) {
  if (a->n == a->cap) {
    a->cap = a->cap ? 2 * a->cap : 1024;
    a->v = (double *)realloc(a->v, sizeof(double) * a->cap);
  }
  a->v[a->n++] = x;
}

typedef struct {
  int64_t n, cap;
  float *v;
} vecf_t;

static void vpushf(vecf_t *a, float x) {
  if (a->n == a->cap) {
    a->cap = a->cap ? 2 * a->cap : 1024;
    a->v = (float *)realloc(a->v, sizeof(float) * a->cap);
  }
  a->v[a->n++] = x;
}

/* minimum-image squared distance (main:2014-2020, 1844-1850) */
static inline double dist2(double xx, double yy, double zz, double xc,
                           double yc, double zc, double tx, double ty,
                           double tz) {
  double dx = fabs(xx - xc);
  dx = (dx < tx - dx) ? dx : tx - dx;
  double dy = fabs(yy - yc);
  dy = (dy < ty - dy) ? dy : ty - dy;
  double dz = fabs(zz - zc);
  dz = (dz < tz - dz) ? dz : tz - dz;
  return (dx * dx + dy * dy) + dz * dz;
}

/* Records stored in the cells of the preselect cube (half-width ncut around
 * cell c0) that meet the ball of radius rb around (xc, yc, zc): the
 * algorithmic read volume of one crossing search.  A cell i of an axis
 * spans [i + xs, i + xs + 1); the ball meets row (dj, dk) when
 * rb^2 - gy^2 - gz^2 >= 0 with g the gap from the centre to the row's cells,
 * and the row's cells t0..t1 around the centre's x offset.  Every operation
 * is rounded separately, as in the GPU's counter. */
static double cell_rel(double x, int64_t i, double xs, double nxd) {
  double d = x - (((double)i + xs) + 0.5);
  d = d - nxd * floor(d / nxd + 0.5);
  return d;
}
static double cell_gap(double t0, int t, double nxd) {
  double d = fabs((double)t - t0);
  d = fmin(d, nxd - d);
  return fmax(d - 0.5, 0.0);
}
static int64_t ball_touch(const int64_t *num, int32_t nx, int32_t ncut, const int64_t c0[3], double xc,
                          double yc, double zc, const double xs[3], double rb) {
  const double nxd = (double)nx;
  const double tx = cell_rel(xc, c0[0], xs[0], nxd), ty = cell_rel(yc, c0[1], xs[1], nxd),
               tz = cell_rel(zc, c0[2], xs[2], nxd);
  const double rm2 = rb * rb;
  int64_t sum = 0;
  for (int dk = -ncut; dk <= ncut; dk++)
    for (int dj = -ncut; dj <= ncut; dj++) {
      const double gy = cell_gap(ty, dj, nxd), gz = cell_gap(tz, dk, nxd);
      const double gy2 = gy * gy, gz2 = gz * gz;
      const double rem = (rm2 - gy2) - gz2;
      if (rem < 0.0) continue;
      const double wx = sqrt(rem);
      int t0 = (int)ceil((tx - 0.5) - wx), t1 = (int)floor((tx + 0.5) + wx);
      if (t0 < -ncut) t0 = -ncut;
      if (t1 > ncut) t1 = ncut;
      int64_t jj = (c0[1] + dj) % nx, kk = (c0[2] + dk) % nx;
      if (jj < 0) jj += nx;
      if (kk < 0) kk += nx;
      for (int t = t0; t <= t1; t++) {
        int64_t ii = (c0[0] + t) % nx;
        if (ii < 0) ii += nx;
        sum += num[ii + (int64_t)nx * (jj + (int64_t)nx * kk)];
      }
    }
  return sum;
}

/* Crossing scan of main:2040-2100 for one threshold.  dist is sorted.
 * Returns i (1-based stop index); *ovd_out gets overdens at exit. */
static int64_t crossing_scan(const double *dist, int64_t npart_sel,
                             double seuil, double seuil2, double munit,
                             int32_t ncut, double *ovd_out, int64_t *masse2) {
  const double twopi = 6.283185307179586; /* main:1424 */
  const double c = (2.0 / 3.0) * twopi;
  const double dc0 = 0.0; /* always 0 before refinement, main:1765-1771 */
  int64_t i = 1;
  double overdens = 2.0 * seuil;
  double amass = munit;
  double rayon = 0.0;
  while (i < 10 || (overdens > seuil && i < npart_sel &&
                    rayon < ((double)ncut - sqrt(dc0)))) {
    i = i + 1;
    rayon = sqrt(dist[i - 1]);
    double volume = c * ((rayon * rayon) * rayon);
    amass = amass + munit;
    overdens = amass / volume;
    if (masse2 && overdens > seuil2) *masse2 = i; /* main:2062-2069 */
  }
  *ovd_out = overdens;
  return i;
}

/* spherover; when au is given, the arithmetic audit counters are filled
 * along the way (see psod_oracle_audit_spherover). */
static int spherover_impl(const psod_oracle_params *p, int64_t n,
                          const float *pos, const int64_t *ids,
                          const int64_t *isort, int64_t npart_new, int mode,
                          psod_oracle_result *res, psod_oracle_audit *au) {
  memset(res, 0, sizeof(*res));
  if (au) memset(au, 0, sizeof(*au));
  res->fail_rank = -1;
  res->npart_new = npart_new;
  zone_t z;
  int st = zone_setup(p, &z);
  if (st) {
    res->status = st;
    return st;
  }
  const int32_t nx = z.nx;
  const double scale = z.scale;
  const double *xxmin = z.xmin; /* main:738 */
  const int64_t local_nx = z.local_nx; /* main:739 */
  const double Mmin = (double)p->nmin;
  const double munit = (double)z.munit;
  const double tx = (double)nx; /* taillex, main:1517 */
  const double rmin2 = (scale / nx) * (scale / nx); /* rayon_min**2 */
  const double eps = scale / nx / 64.0;            /* main:1527 */
  const double eps2 = eps * eps;
  const int nbins = p->nbins;

  /* posf = posf*scale, stored back to real(4) (main:690) */
  float *pg = (float *)malloc(sizeof(float) * 3 * (size_t)(n > 0 ? n : 1));
  for (int64_t i = 0; i < 3 * n; i++) pg[i] = (float)((double)pos[i] * scale);

  /* linked list, main:1564-1604.  Cells are kept compact (stride nx): the
   * reference's stride local_nx orders cells identically. */
  const int64_t ncell = (int64_t)nx * nx * nx;
  double *ckey = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  int64_t *cell_of = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
  for (int64_t i = 0; i < n; i++) {
    int64_t c3[3];
    for (int a = 0; a < 3; a++) {
      int64_t ia = (int64_t)floor((double)pg[3 * i + a] - xxmin[a] * scale);
      if (ia < 0) ia = ia + nx;
      if (ia >= nx) ia = ia - nx;
      c3[a] = ia;
    }
    cell_of[i] = c3[0] + (int64_t)nx * (c3[1] + (int64_t)nx * c3[2]);
    ckey[i] = (double)cell_of[i];
  }
  int64_t *isort_ngp = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
  sort_with_order(ckey, isort_ngp, n, mode, NULL);
  int64_t *first = (int64_t *)calloc((size_t)ncell, sizeof(int64_t));
  int64_t *num = (int64_t *)calloc((size_t)ncell, sizeof(int64_t));
  {
    /* literal run scan of main:1591-1604, including its handling of the
     * final run: a last cell holding a single particle is folded into the
     * previous run. */
    int64_t imin = 0;
    while (imin < n) {
      int64_t ind = (int64_t)ckey[imin];
      int64_t i = imin;
      first[ind] = imin;
      while (ckey[i] == (double)ind && i < n - 1) i = i + 1;
      if (i == n - 1) i = n;
      int64_t imax = i - 1;
      num[ind] = i - imin;
      imin = imax + 1;
    }
  }
  free(ckey);

  unsigned char *alive = (unsigned char *)malloc((size_t)(n > 0 ? n : 1));
  memset(alive, 1, (size_t)n); /* xsort = 1.0, main:1619 */

  vec64_t sel = {0}, sel2 = {0};
  vecd_t dist = {0};
  vec64_t h_id = {0}, h_mass = {0}, h_rank = {0}, h_cidx = {0}, h_m2 = {0},
          h_prof = {0}, h_mext = {0}, m_off = {0}, m_idx = {0};
  vecf_t h_c = {0};
  vecd_t h_r = {0};
  vpush(&m_off, 0);
  int64_t *perm = NULL;
  int64_t perm_cap = 0;
  double *edges = (double *)malloc(sizeof(double) * nbins);
  int status = PSOD_ORACLE_OK;

  for (int64_t ipart = 0; ipart < npart_new; ipart++) { /* main:1624 */
    const int64_t s = isort[ipart];
    if (!alive[s]) continue; /* main:1628 */
    double xc = pg[3 * s], yc = pg[3 * s + 1], zc = pg[3 * s + 2];
    int64_t iamas = ids[s];
    int64_t cidx = s;
    int64_t c0[3];
    {
      double xs[3] = {xc, yc, zc};
      for (int a = 0; a < 3; a++) { /* main:1644-1654 */
        int64_t ia = (int64_t)floor(xs[a] - xxmin[a] * scale);
        if (ia < 0) ia = ia + nx;
        if (ia >= nx) ia = ia - nx;
        c0[a] = ia;
      }
    }
    /* preselect, main:1657-1716 */
    sel.n = 0;
    double mtotsel = 0.0;
    for (int di = -p->ncut; di <= p->ncut && !status; di++) {
      int64_t ii = di + c0[0];
      if (ii >= nx) ii -= nx;
      if (ii < 0) ii += nx;
      if (ii >= local_nx) continue; /* outside the local grid */
      for (int dj = -p->ncut; dj <= p->ncut && !status; dj++) {
        int64_t jj = dj + c0[1];
        if (jj >= nx) jj -= nx;
        if (jj < 0) jj += nx;
        if (jj >= local_nx) continue; /* outside the local grid */
        for (int dk = -p->ncut; dk <= p->ncut && !status; dk++) {
          int64_t kk = dk + c0[2];
          if (kk >= nx) kk -= nx;
          if (kk < 0) kk += nx;
          if (kk >= local_nx) continue; /* outside the local grid */
          int64_t ind = ii + (int64_t)nx * (jj + (int64_t)nx * kk);
          for (int64_t ip = first[ind]; ip < first[ind] + num[ind]; ip++) {
            int64_t q = isort_ngp[ip];
            if (!alive[q]) continue;
            if (sel.n + 1 > p->nsel) { /* main:1681-1693 */
              status = PSOD_ORACLE_ERR_NSEL;
              break;
            }
            vpush(&sel, q);
            mtotsel = mtotsel + munit;
          }
        }
      }
    }
    if (status) {
      res->fail_rank = ipart;
      break;
    }
    /* ncut2 = 2 set, main:1720-1755 */
    sel2.n = 0;
    for (int di = -2; di <= 2; di++) {
      int64_t ii = di + c0[0];
      if (ii >= nx) ii -= nx;
      if (ii < 0) ii += nx;
      if (ii >= local_nx) continue; /* outside the local grid */
      for (int dj = -2; dj <= 2; dj++) {
        int64_t jj = dj + c0[1];
        if (jj >= nx) jj -= nx;
        if (jj < 0) jj += nx;
        if (jj >= local_nx) continue; /* outside the local grid */
        for (int dk = -2; dk <= 2; dk++) {
          int64_t kk = dk + c0[2];
          if (kk >= nx) kk -= nx;
          if (kk < 0) kk += nx;
          if (kk >= local_nx) continue; /* outside the local grid */
          int64_t ind = ii + (int64_t)nx * (jj + (int64_t)nx * kk);
          for (int64_t ip = first[ind]; ip < first[ind] + num[ind]; ip++) {
            int64_t q = isort_ngp[ip];
            if (alive[q]) vpush(&sel2, q);
          }
        }
      }
    }
    if (!(mtotsel >= Mmin)) continue; /* main:1759 */
    res->nprocessed++;

    /* centre refinement, ncut3 = 1, main:1799-1909 */
    {
      double smax = 0.0;
      int64_t sqmax = 0;
      /* audit: the argmax of each arithmetic over the same candidates in
       * the same scan order, and the runner-up of the fixed-point sums */
      double a_smax = 0.0;
      int64_t a_sqmax = 0, a_sq2 = 0, a_cr = -1, a_cc = -1;
      for (int di = -1; di <= 1; di++) {
        int64_t ii = di + c0[0];
        if (ii >= nx) ii -= nx;
        if (ii < 0) ii += nx;
        if (ii >= local_nx) continue; /* outside the local grid */
        for (int dj = -1; dj <= 1; dj++) {
          int64_t jj = dj + c0[1];
          if (jj >= nx) jj -= nx;
          if (jj < 0) jj += nx;
          if (jj >= local_nx) continue; /* outside the local grid */
          for (int dk = -1; dk <= 1; dk++) {
            int64_t kk = dk + c0[2];
            if (kk >= nx) kk -= nx;
            if (kk < 0) kk += nx;
            if (kk >= local_nx) continue; /* outside the local grid */
            int64_t ind = ii + (int64_t)nx * (jj + (int64_t)nx * kk);
            for (int64_t ip = first[ind]; ip < first[ind] + num[ind]; ip++) {
              int64_t q = isort_ngp[ip];
              if (!alive[q]) continue;
              double xcn = pg[3 * q], ycn = pg[3 * q + 1], zcn = pg[3 * q + 2];
              double sum = 0.0;
              int64_t sq = 0;
              for (int64_t jjj = 0; jjj < sel2.n; jjj++) {
                int64_t r = sel2.v[jjj];
                double d2 = dist2(pg[3 * r], pg[3 * r + 1], pg[3 * r + 2], xcn,
                                  ycn, zcn, tx, tx, tx);
                if (d2 <= rmin2) {
                  double t = 1.0 / sqrt(d2 + eps2); /* main:1854-1855 */
                  if (mode == PSOD_ORACLE_CANONICAL || au)
                    sq += (int64_t)llrint(t * FIX_ONE);
                  if (mode == PSOD_ORACLE_REFERENCE || au)
                    sum = sum + t;
                }
              }
              if (au) {
                if (sum > a_smax) {
                  a_smax = sum;
                  a_cr = q;
                }
                if (sq > a_sqmax) {
                  a_sq2 = a_sqmax;
                  a_sqmax = sq;
                  a_cc = q;
                } else if (sq > a_sq2) {
                  a_sq2 = sq;
                }
              }
              int better = (mode == PSOD_ORACLE_CANONICAL) ? (sq > sqmax)
                                                           : (sum > smax);
              if (better) { /* strict >, main:1865 */
                xc = xcn;
                yc = ycn;
                zc = zcn;
                iamas = ids[q];
                cidx = q;
                smax = sum;
                sqmax = sq;
              }
            }
          }
        }
      }
      if (au) {
        au->refine_seeds++;
        if (a_cr != a_cc) au->refine_flips++;
        if (a_sqmax > 0 && (double)(a_sqmax - a_sq2) < 1e-9 * (double)a_sqmax) au->refine_near++;
      }
    }

    /* distances, main:2002-2026 */
    const int64_t npart_sel = sel.n;
    dist.n = 0;
    for (int64_t i = 0; i < npart_sel; i++) {
      int64_t q = sel.v[i];
      vpushd(&dist, dist2(pg[3 * q], pg[3 * q + 1], pg[3 * q + 2], xc, yc, zc,
                          tx, tx, tx));
    }
    if (perm_cap < npart_sel) {
      perm_cap = npart_sel;
      perm = (int64_t *)realloc(perm, sizeof(int64_t) * perm_cap);
    }
    sort_with_order(dist.v, perm, npart_sel, mode, sel.v); /* main:2030 */

    /* crossing, main:2040-2100 */
    double ovd;
    /* masse2 keeps its previous value in the reference when no step is
     * above seuil2 (it is only printed there); here it restarts at 0 */
    int64_t masse2 = 0;
    int64_t i = crossing_scan(dist.v, npart_sel, p->delta, p->delta2, munit,
                              p->ncut, &ovd, &masse2);
    if (ovd > p->delta) { /* main:2072-2089 */
      status = PSOD_ORACLE_ERR_SELRADIUS;
      res->fail_rank = ipart;
      break;
    }
    const double rayon = sqrt(dist.v[i - 2]); /* distance(i-1), 1-based */
    const int64_t masse = i - 1;
    if (au) {
      /* the masse-th and (masse+1)-th sorted distances equal: which of the
       * tied particles become members depends on the sort's tie order */
      if (masse < npart_sel && dist.v[masse - 1] == dist.v[masse]) {
        au->dist_tie_cut++;
        if (masse > au->dist_tie_cut_nmax) au->dist_tie_cut_nmax = masse;
      }
      for (int64_t k = 1; k < masse; k++)
        if (dist.v[k - 1] == dist.v[k]) {
          au->dist_tie_members++;
          break;
        }
    }
    /* algorithmic reads: the cells meeting the ball out to the stopping
     * particle (the i-th, 1-based) */
    {
      const double xs3[3] = {xxmin[0] * scale, xxmin[1] * scale, xxmin[2] * scale};
      res->cross_touch += ball_touch(num, nx, p->ncut, c0, xc, yc, zc, xs3, sqrt(dist.v[i - 1]));
    }
    const double amass = (double)masse * munit;

    /* profile edges and cumulative counts, main:2103-2115 */
    for (int j = 0; j < nbins; j++) {
      double denom = (double)nbins - 1.0;
      double f = (denom > 0.0)
                     ? exp(log(p->rbin_lo) +
                           ((double)j * (log(p->rbin_hi) - log(p->rbin_lo))) /
                               denom)
                     : p->rbin_hi;
      edges[j] = rayon * f;
    }

    /* keep test, main:2118-2120 */
    const int keep = amass >= Mmin && xc <= z.xmaxzone[0] && xc > z.xminzone[0] &&
                     yc <= z.xmaxzone[1] && yc > z.xminzone[1] &&
                     zc <= z.xmaxzone[2] && zc > z.xminzone[2];
    if (keep) {
      vpush(&h_id, iamas);
      vpush(&h_mass, masse);
      vpush(&h_rank, ipart);
      vpush(&h_cidx, cidx);
      vpushf(&h_c, (float)(xc / scale));
      vpushf(&h_c, (float)(yc / scale));
      vpushf(&h_c, (float)(zc / scale));
      vpushd(&h_r, rayon);
      vpush(&h_m2, masse2);
      /* edges increase with j, so each bin resumes where the last one
       * stopped, as main:2106-2114 does */
      int64_t cnt = 0;
      for (int j = 0; j < nbins; j++) {
        while (cnt < npart_sel && sqrt(dist.v[cnt]) < edges[j]) cnt++;
        vpush(&h_prof, cnt);
      }
      for (int e = 0; e < p->ndelta_extra; e++) {
        double ovde;
        int64_t ie = crossing_scan(dist.v, npart_sel, p->delta_extra[e], 0.0,
                                   munit, p->ncut, &ovde, NULL);
        vpush(&h_mext, (ovde > p->delta_extra[e]) ? -1 : ie - 1);
      }
    }
    /* claims, main:2148-2166 (particles die even if the halo is dropped) */
    for (int64_t k = 0; k < masse; k++) {
      int64_t q = sel.v[perm[k]];
      alive[q] = 0;
      if (keep) vpush(&m_idx, q);
    }
    if (keep) vpush(&m_off, m_idx.n);
  }

  res->status = status;
  if (status == PSOD_ORACLE_OK) {
    res->nhalo = h_id.n;
    res->nmember = m_idx.n;
    res->halo_id = h_id.v;
    res->halo_mass = h_mass.v;
    res->halo_rank = h_rank.v;
    res->halo_cidx = h_cidx.v;
    res->halo_center = h_c.v;
    res->halo_rdelta = h_r.v;
    res->halo_mass2 = h_m2.v;
    res->halo_mextra = h_mext.v;
    res->halo_profile = h_prof.v;
    res->member_offset = m_off.v;
    res->member_index = m_idx.v;
  } else {
    /* the whole zone's output is lost (main:1684-1692, 2082-2089) */
    free(h_id.v); free(h_mass.v); free(h_rank.v); free(h_cidx.v);
    free(h_c.v); free(h_r.v); free(h_m2.v); free(h_mext.v); free(h_prof.v);
    free(m_off.v); free(m_idx.v);
    res->member_offset = (int64_t *)calloc(1, sizeof(int64_t));
  }
  free(edges);
  free(perm);
  free(sel.v);
  free(sel2.v);
  free(dist.v);
  free(alive);
  free(first);
  free(num);
  free(isort_ngp);
  free(cell_of);
  free(pg);
  return status;
}

int psod_oracle_spherover(const psod_oracle_params *p, int64_t n,
                          const float *pos, const int64_t *ids,
                          const int64_t *isort, int64_t npart_new, int mode,
                          psod_oracle_result *res) {
  return spherover_impl(p, n, pos, ids, isort, npart_new, mode, res, NULL);
}

int psod_oracle_audit_spherover(const psod_oracle_params *p, int64_t n,
                                const float *pos, const int64_t *ids,
                                const int64_t *isort, int64_t npart_new,
                                int mode, psod_oracle_result *res,
                                psod_oracle_audit *au) {
  return spherover_impl(p, n, pos, ids, isort, npart_new, mode, res, au);
}

int psod_oracle_run(const psod_oracle_params *p, int64_t n, const float *pos,
                    const int64_t *ids, int mode, psod_oracle_result *res) {
  memset(res, 0, sizeof(*res));
  zone_t z;
  int st = zone_setup(p, &z);
  if (st) {
    res->status = st;
    res->fail_rank = -1;
    return st;
  }
  const int64_t nc = z.nxcic;
  double *grid = (double *)malloc(sizeof(double) * (size_t)(nc * nc * nc));
  double *rho = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  int64_t *isort = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
  int64_t npart_new = 0;
  st = psod_oracle_cic(p, n, pos, mode, grid);
  if (!st) st = psod_oracle_cicm1(p, n, pos, grid, rho);
  free(grid);
  if (!st) st = psod_oracle_tri_cic(n, rho, mode, isort, &npart_new);
  free(rho);
  if (!st)
    st = psod_oracle_spherover(p, n, pos, ids, isort, npart_new, mode, res);
  else {
    res->status = st;
    res->fail_rank = -1;
  }
  free(isort);
  return st;
}

void psod_oracle_free(psod_oracle_result *res) {
  free(res->halo_id);
  free(res->halo_mass);
  free(res->halo_rank);
  free(res->halo_cidx);
  free(res->halo_center);
  free(res->halo_rdelta);
  free(res->halo_mass2);
  free(res->halo_mextra);
  free(res->halo_profile);
  free(res->member_offset);
  free(res->member_index);
  memset(res, 0, sizeof(*res));
}
