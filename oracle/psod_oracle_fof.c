/*
 * psod_oracle_fof.c -- CPU oracle for the friends-of-friends halo finder of
 * pFoF (test infrastructure only: tests/ and bench.py's cpu_baseline leg use
 * it as the checker; nothing in the product links it).
 *
 * Single-threaded restatement, for one MPI rank on the periodic unit box, of
 *   fofpara      Pfof/trunk/pfof_snap/src/modfofpara.f90:31-296
 *                (grid of 2*nres cells a side, the per-particle neighbour
 *                scan with nsign cells per axis, the in-place queue `lamas`
 *                whose front gives each local group its seed and label)
 *   init         modfofpara.f90:478-556 (cell stacks in particle order)
 *   mergehaloes  Pfof/trunk/common/src/modfofmpi.f90:37-91, with
 *   initmerging  modfofmpi.f90:98-173  (face lists, particle order)
 *   findbridge   modfofmpi.f90:183-317 (FP32 minimum-image pair test)
 *   setcommonhaloid modfofmpi.f90:323-649 (labels merged to the smallest)
 *                with one rank every face list is paired with the opposite
 *                face list of the same rank, so the bridges are the pairs
 *                that meet across the periodic boundary
 *   gatherhaloes Pfof/trunk/common/src/modhalo.f90:36-246 (one rank: the
 *                particles stay in their order)
 *   heapsort     Pfof/trunk/common/src/modsortinterf.f90:650-681 and its
 *                construction/entasser/echanger helpers (max-heap on the
 *                structure id; the member order inside a halo is heap order)
 *   selecthaloes sod/modhalo.f90:253-376 (halos in ascending id, mass >= Mmin)
 *   computecom   sod/modhalo.f90:381-441 (FP64 running sums, periodic
 *                unwrap against the running mean)
 *   computeradius sod/modhalo.f90:445-488
 *
 * Parity status: pinned by known-answer boxes (tests/test_fof_oracle.py)
 * only; pFoF ships no golden outputs for this path.
 */
#include "psod_oracle_fof.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* positions equal to 1.0 are moved to 0.0 as the scan reaches them
   (modfofpara.f90:162-164) */
static float wrap_one(float x) { return fabsf(x - 1.0f) < 1.e-8f ? 0.0f : x; }

/* FP32 squared distance as the reference evaluates it: products rounded,
   summed left to right (modfofpara.f90:234-238; the Makefile builds with
   -ffp-contract=off, so no product is fused into a sum) */
static float d2_direct(const float *a, const float *b) {
  const float dx = fabsf(a[0] - b[0]), dy = fabsf(a[1] - b[1]), dz = fabsf(a[2] - b[2]);
  return dx * dx + dy * dy + dz * dz;
}

/* findbridge's periodic form (modfofmpi.f90:226-233) */
static float d2_bridge(const float *a, const float *b) {
  float dx = fabsf(a[0] - b[0]), dy = fabsf(a[1] - b[1]), dz = fabsf(a[2] - b[2]);
  dx = fminf(dx, 1.0f - dx);
  dy = fminf(dy, 1.0f - dy);
  dz = fminf(dz, 1.0f - dz);
  return dx * dx + dy * dy + dz * dz;
}

/* (label, particle) pairs in ascending order */
static int cmp_pair(const void *a, const void *b) {
  const int64_t *x = (const int64_t *)a, *y = (const int64_t *)b;
  if (x[0] != y[0]) return x[0] < y[0] ? -1 : 1;
  return x[1] < y[1] ? -1 : (x[1] > y[1]);
}

/* -------------------------------------------------------------------------
 * heapsort on the structure id, the other arrays moved along
 * (modsortinterf.f90:650-681; entasser is the sift-down of a max-heap)
 * ------------------------------------------------------------------------- */
typedef struct {
  int64_t *ref;
  float *x, *v;
  int64_t *id;
  int64_t *idx; /* input index, carried for the caller */
} heap_t;

static void heap_swap(heap_t *h, int64_t i, int64_t j) { /* 1-based */
  int64_t t;
  float f;
  t = h->ref[i - 1]; h->ref[i - 1] = h->ref[j - 1]; h->ref[j - 1] = t;
  t = h->id[i - 1]; h->id[i - 1] = h->id[j - 1]; h->id[j - 1] = t;
  t = h->idx[i - 1]; h->idx[i - 1] = h->idx[j - 1]; h->idx[j - 1] = t;
  for (int a = 0; a < 3; a++) {
    f = h->x[3 * (i - 1) + a]; h->x[3 * (i - 1) + a] = h->x[3 * (j - 1) + a]; h->x[3 * (j - 1) + a] = f;
    f = h->v[3 * (i - 1) + a]; h->v[3 * (i - 1) + a] = h->v[3 * (j - 1) + a]; h->v[3 * (j - 1) + a] = f;
  }
}

static void heap_sift(heap_t *h, int64_t size, int64_t i) {
  for (;;) {
    const int64_t l = 2 * i, r = 2 * i + 1;
    int64_t m = (l <= size && h->ref[l - 1] > h->ref[i - 1]) ? l : i;
    if (r <= size && h->ref[r - 1] > h->ref[m - 1]) m = r;
    if (m == i) return;
    heap_swap(h, i, m);
    i = m;
  }
}

static void heapsort_ref(heap_t *h, int64_t n) {
  int64_t size = n;
  for (int64_t i = n / 2; i >= 1; i--) heap_sift(h, size, i);
  for (int64_t i = n; i >= 2; i--) {
    heap_swap(h, 1, i);
    size--;
    heap_sift(h, size, 1);
  }
}

/* -------------------------------------------------------------------------
 * label merging: every bridge joins the labels of its two particles and
 * each merged set takes its smallest label, the fixed point of
 * setcommonhaloid's passes
 * ------------------------------------------------------------------------- */
static int64_t uf_find(int64_t *par, int64_t a) {
  while (par[a] != a) {
    par[a] = par[par[a]];
    a = par[a];
  }
  return a;
}

int psod_oracle_fof(const psod_oracle_fof_params *p, int64_t n, const float *pos_in, const float *vel_in,
                    const int64_t *id, psod_oracle_fof_result *res) {
  memset(res, 0, sizeof(*res));
  if (!p || n < 1 || n >= 2147483647 || !pos_in || !id || p->nres < 1 || !(p->percolation > 0.0f) || p->mmin < 1)
    return res->status = PSOD_ORACLE_FOF_ERR_ARG;
  const int refine_fof = 2;
  /* modfofpara.f90:101-117: percolation_length * refine_fof must stay
     below 1 */
  if (p->percolation * (float)refine_fof >= 1.0f) return res->status = PSOD_ORACLE_FOF_ERR_ARG;
  const int64_t res_fof = refine_fof * p->nres; /* one rank: dims(1) = 1 */
  if (res_fof > 2097151) return res->status = PSOD_ORACLE_FOF_ERR_ARG;
  const int64_t ngrid = res_fof * res_fof * res_fof;
  const float size = (float)p->nres, size_fof = (float)refine_fof * size;
  const int nsign = p->percolation * (float)refine_fof >= 0.5f ? 3 : 2;
  const float xmin = 0.0f, xmax = 1.0f;
  const float r = p->percolation;
  const float rT = r / size;
  const float r2 = rT * rT;

  float *pos = (float *)malloc(sizeof(float) * 3 * (size_t)n);
  int32_t *adfirst = (int32_t *)calloc((size_t)ngrid, sizeof(int32_t));
  int32_t *adlast = (int32_t *)calloc((size_t)ngrid, sizeof(int32_t));
  int32_t *npcase = (int32_t *)calloc((size_t)ngrid, sizeof(int32_t));
  int32_t *pile = (int32_t *)calloc((size_t)n + 1, sizeof(int32_t));
  int32_t *lamas = (int32_t *)malloc(sizeof(int32_t) * ((size_t)n + 2));
  int32_t *indl = (int32_t *)malloc(sizeof(int32_t) * ((size_t)n + 1));
  int64_t *structure = (int64_t *)malloc(sizeof(int64_t) * ((size_t)n + 1));
  unsigned char *border = (unsigned char *)calloc((size_t)n + 1, 1);
  if (!pos || !adfirst || !adlast || !npcase || !pile || !lamas || !indl || !structure || !border) {
    free(pos); free(adfirst); free(adlast); free(npcase); free(pile); free(lamas); free(indl);
    free(structure); free(border);
    return res->status = PSOD_ORACLE_FOF_ERR_ARG;
  }
  memcpy(pos, pos_in, sizeof(float) * 3 * (size_t)n);
#define POS(i, a) pos[3 * ((i) - 1) + (a)]

  /* init (modfofpara.f90:478-556): one stack per cell, particle order */
  for (int64_t ip = 1; ip <= n; ip++) {
    const float xx = (POS(ip, 0) - xmin) * size_fof, yy = (POS(ip, 1) - xmin) * size_fof,
                zz = (POS(ip, 2) - xmin) * size_fof;
    int64_t ix = (int64_t)xx, iy = (int64_t)yy, iz = (int64_t)zz;
    if (ix == res_fof) ix--;
    if (iy == res_fof) iy--;
    if (iz == res_fof) iz--;
    const int64_t ic = 1 + ix + iy * res_fof + iz * res_fof * res_fof;
    npcase[ic - 1]++;
    if (adfirst[ic - 1] == 0) {
      adfirst[ic - 1] = (int32_t)ip;
      adlast[ic - 1] = (int32_t)ip;
    } else {
      pile[adlast[ic - 1]] = (int32_t)ip;
      adlast[ic - 1] = (int32_t)ip;
    }
  }
  free(adlast);

  for (int64_t i = 1; i <= n; i++) lamas[i] = indl[i] = (int32_t)i;
  int64_t namas = id[0];
  int64_t ipermut = 2;
  int64_t nflag[6] = {0, 0, 0, 0, 0, 0};
  int64_t ngroups = 0;
  int signx[3] = {0, 0, 1}, signy[3] = {0, 0, 1}, signz[3] = {0, 0, 1};

  /* the local scan (modfofpara.f90:158-288) */
  for (int64_t i = 1; i <= n; i++) {
    const int64_t ipart = lamas[i];
    for (int a = 0; a < 3; a++) POS(ipart, a) = wrap_one(POS(ipart, a));
    unsigned char b = 0;
    if (fabsf(POS(ipart, 0) - xmin) <= rT) { b += 4; nflag[0]++; }
    if (fabsf(POS(ipart, 0) - xmax) <= rT) { b += 8; nflag[1]++; }
    if (fabsf(POS(ipart, 1) - xmin) <= rT) { b += 1; nflag[2]++; }
    if (fabsf(POS(ipart, 1) - xmax) <= rT) { b += 2; nflag[3]++; }
    if (fabsf(POS(ipart, 2) - xmin) <= rT) { b += 16; nflag[4]++; }
    if (fabsf(POS(ipart, 2) - xmax) <= rT) { b += 32; nflag[5]++; }
    border[ipart] = b;
    const float xx = POS(ipart, 0), yy = POS(ipart, 1), zz = POS(ipart, 2);
    const float fx = (xx - xmin) * size_fof, fy = (yy - xmin) * size_fof, fz = (zz - xmin) * size_fof;
    const int64_t ix = (int64_t)fx, iy = (int64_t)fy, iz = (int64_t)fz;
    signx[1] = signy[1] = signz[1] = -1;
    if (nsign == 2) {
      if (fx - (float)ix > 0.5f) signx[1] = 1;
      if (fy - (float)iy > 0.5f) signy[1] = 1;
      if (fz - (float)iz > 0.5f) signz[1] = 1;
    }
    structure[ipart] = namas;
    for (int i1 = 0; i1 < nsign; i1++) {
      const int64_t j1 = ix + signx[i1];
      if (j1 >= res_fof || j1 < 0) continue;
      for (int i2 = 0; i2 < nsign; i2++) {
        const int64_t j2 = iy + signy[i2];
        if (j2 >= res_fof || j2 < 0) continue;
        for (int i3 = 0; i3 < nsign; i3++) {
          const int64_t j3 = iz + signz[i3];
          if (j3 >= res_fof || j3 < 0) continue;
          const int64_t index = j1 + j2 * res_fof + j3 * res_fof * res_fof; /* 0-based */
          int64_t ic = 0;
          if (npcase[index] >= 1) {
            int64_t ipile = adfirst[index], ipilepr = adfirst[index];
            const int64_t cnt = npcase[index];
            for (int64_t ind = 1; ind <= cnt; ind++) {
              if (ipart != ipile) {
                if (d2_direct(&POS(ipart, 0), &POS(ipile, 0)) <= r2) {
                  /* the linked particle takes the queue's front slot */
                  const int32_t sttmp = lamas[ipermut];
                  lamas[ipermut] = (int32_t)ipile;
                  lamas[indl[ipile]] = sttmp;
                  indl[sttmp] = indl[ipile];
                  indl[ipile] = (int32_t)ipermut;
                  ipermut++;
                  if (ipile == adfirst[index]) {
                    adfirst[index] = pile[ipile];
                    ipilepr = pile[ipile];
                  } else {
                    pile[ipilepr] = pile[ipile];
                  }
                  ic++;
                } else {
                  ipilepr = ipile;
                }
              } else {
                if (ipile == adfirst[index]) {
                  adfirst[index] = pile[ipile];
                  ipilepr = pile[ipile];
                } else {
                  pile[ipilepr] = pile[ipile];
                }
                ic++;
              }
              ipile = pile[ipile];
            }
          }
          npcase[index] -= ic;
        }
      }
    }
    if (ipermut == i + 1) {
      /* the group is complete; the queue's front starts the next one */
      ipermut++;
      ngroups++;
      if (i < n) namas = id[lamas[i + 1] - 1];
    }
  }
  free(adfirst);
  free(npcase);
  free(pile);
  free(lamas);
  free(indl);

  /* merging (modfofmpi.f90:37-173, 183-317, 323-649): face lists in
     particle order; bridges pair each lower-face list with the upper-face
     list of the same axis; labels merge to the smallest */
  int64_t *flist[6];
  int64_t fcnt[6] = {0, 0, 0, 0, 0, 0};
  for (int f = 0; f < 6; f++) flist[f] = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nflag[f] + 1));
  static const unsigned char bit[6] = {4, 8, 1, 2, 16, 32}; /* x lo/hi, y lo/hi, z lo/hi */
  for (int64_t i = 1; i <= n; i++)
    for (int f = 0; f < 6; f++)
      if (border[i] & bit[f]) flist[f][fcnt[f]++] = i;
  free(border);
  /* labels are particle IDs: merge them through the particles that carry
     them (the first particle of each label stands for it) */
  int64_t *par = (int64_t *)malloc(sizeof(int64_t) * ((size_t)n + 1));
  int64_t *rep = (int64_t *)malloc(sizeof(int64_t) * ((size_t)n + 1)); /* particle -> label representative */
  for (int64_t i = 1; i <= n; i++) par[i] = i;
  {
    /* representative of each label: the first particle holding it */
    int64_t *keys = (int64_t *)malloc(sizeof(int64_t) * (size_t)n * 2);
    for (int64_t i = 1; i <= n; i++) {
      keys[2 * (i - 1)] = structure[i];
      keys[2 * (i - 1) + 1] = i;
    }
    qsort(keys, (size_t)n, 2 * sizeof(int64_t), cmp_pair);
    int64_t first = 0;
    for (int64_t k = 0; k < n; k++) {
      if (k == 0 || keys[2 * k] != keys[2 * (k - 1)]) first = keys[2 * k + 1];
      rep[keys[2 * k + 1]] = first;
    }
    free(keys);
  }
  int64_t nbridge = 0;
  for (int axis = 0; axis < 3; axis++) {
    const int64_t *lo = flist[2 * axis], *hi = flist[2 * axis + 1];
    for (int64_t a = 0; a < fcnt[2 * axis]; a++)
      for (int64_t b = 0; b < fcnt[2 * axis + 1]; b++) {
        if (d2_bridge(&POS(lo[a], 0), &POS(hi[b], 0)) <= r2) {
          nbridge++;
          int64_t ra = uf_find(par, rep[lo[a]]), rb = uf_find(par, rep[hi[b]]);
          if (ra != rb) {
            /* keep the representative with the smaller label on top */
            if (structure[rb] < structure[ra]) {
              int64_t t = ra;
              ra = rb;
              rb = t;
            }
            par[rb] = ra;
          }
        }
      }
  }
  for (int f = 0; f < 6; f++) free(flist[f]);
  for (int64_t i = 1; i <= n; i++) structure[i] = structure[uf_find(par, rep[i])];
  free(par);
  free(rep);

  /* gatherhaloes (one rank: particle order), then heapsort on the label */
  heap_t h;
  h.ref = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
  h.x = (float *)malloc(sizeof(float) * 3 * (size_t)n);
  h.v = (float *)malloc(sizeof(float) * 3 * (size_t)n);
  h.id = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
  h.idx = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
  for (int64_t i = 0; i < n; i++) {
    h.ref[i] = structure[i + 1];
    h.id[i] = id[i];
    h.idx[i] = i;
    for (int a = 0; a < 3; a++) {
      h.x[3 * i + a] = pos[3 * i + a];
      h.v[3 * i + a] = vel_in ? vel_in[3 * i + a] : 0.0f;
    }
  }
  res->structure = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
  for (int64_t i = 0; i < n; i++) res->structure[i] = structure[i + 1];
  free(structure);
  free(pos);
  heapsort_ref(&h, n);

  /* selecthaloes (sod/modhalo.f90:253-376): runs of one label, ascending */
  int64_t nh = 0, nm = 0;
  for (int64_t s = 0; s < n;) {
    int64_t e = s;
    while (e < n && h.ref[e] == h.ref[s]) e++;
    if (e - s >= p->mmin) {
      nh++;
      nm += e - s;
    }
    s = e;
  }
  res->nhalo = nh;
  res->nmember = nm;
  res->ngroups_local = ngroups;
  res->nbridges = nbridge;
  res->halo_id = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nh + 1));
  res->halo_mass = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nh + 1));
  res->halo_com = (double *)malloc(sizeof(double) * 3 * (size_t)(nh + 1));
  res->halo_vel = (double *)malloc(sizeof(double) * 3 * (size_t)(nh + 1));
  res->halo_radius = (double *)malloc(sizeof(double) * (size_t)(nh + 1));
  res->member_offset = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nh + 1));
  res->member_index = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nm + 1));
  int64_t hh = 0, mm = 0;
  res->member_offset[0] = 0;
  for (int64_t s = 0; s < n;) {
    int64_t e = s;
    while (e < n && h.ref[e] == h.ref[s]) e++;
    if (e - s >= p->mmin) {
      res->halo_id[hh] = h.ref[s];
      res->halo_mass[hh] = e - s;
      for (int64_t k = s; k < e; k++) res->member_index[mm++] = h.idx[k];
      /* computecom (sod/modhalo.f90:381-441) */
      double cp[3], cv[3];
      int64_t halom = 1;
      for (int a = 0; a < 3; a++) {
        cp[a] = (double)h.x[3 * s + a];
        cv[a] = (double)h.v[3 * s + a];
      }
      for (int64_t k = s + 1; k < e; k++) {
        for (int a = 0; a < 3; a++) {
          const double delta = cp[a] / (double)halom - (double)h.x[3 * k + a];
          if (fabs(delta) > 0.5) {
            if (delta > 0.0) cp[a] = cp[a] + 1.0;
            if (delta < 0.0) cp[a] = cp[a] - 1.0;
          }
        }
        halom++;
        for (int a = 0; a < 3; a++) {
          cp[a] = cp[a] + (double)h.x[3 * k + a];
          cv[a] = cv[a] + (double)h.v[3 * k + a];
        }
      }
      const double mass = (double)(e - s);
      for (int a = 0; a < 3; a++) {
        cp[a] = cp[a] / mass;
        cv[a] = cv[a] / mass;
        if (cp[a] > 1.0) cp[a] = cp[a] - 1.0;
        if (cp[a] < 0.0) cp[a] = cp[a] + 1.0;
        res->halo_com[3 * hh + a] = cp[a];
        res->halo_vel[3 * hh + a] = cv[a];
      }
      /* computeradius (sod/modhalo.f90:445-488) */
      double rmax2 = 0.0;
      for (int64_t k = s; k < e; k++) {
        double dl[3];
        for (int a = 0; a < 3; a++) {
          dl[a] = (double)h.x[3 * k + a] - cp[a];
          if (fabs(dl[a]) > 0.5) dl[a] = 1.0 - fabs(dl[a]);
        }
        const double d2 = dl[0] * dl[0] + dl[1] * dl[1] + dl[2] * dl[2];
        if (d2 > rmax2) rmax2 = d2;
      }
      res->halo_radius[hh] = sqrt(rmax2);
      hh++;
      res->member_offset[hh] = mm;
    }
    s = e;
  }
  free(h.ref);
  free(h.x);
  free(h.v);
  free(h.id);
  free(h.idx);
  return res->status = PSOD_ORACLE_FOF_OK;
#undef POS
}

void psod_oracle_fof_free(psod_oracle_fof_result *res) {
  if (!res) return;
  free(res->halo_id);
  free(res->halo_mass);
  free(res->halo_com);
  free(res->halo_vel);
  free(res->halo_radius);
  free(res->member_offset);
  free(res->member_index);
  free(res->structure);
  memset(res, 0, sizeof(*res));
}
