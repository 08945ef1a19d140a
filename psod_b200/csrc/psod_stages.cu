// psod_stages.cu -- cell-sorted cube, CIC density and seed order.
//
//  stage_cellsort  the linked list of spherover (main:1564-1604) as a
//                  counting sort of the particles into nx^3 SOD cells.
//                  Each particle becomes one 16-byte float4 record, so every
//                  later gather is a coalesced stream of whole cells.
//  stage_cic       cic (main:1077-1265) on the 2nx-per-side periodic grid,
//                  deposited as int64 fixed point (integer atomics are
//                  associative, so the grid is the same on every run).
//  stage_cicm1     cicm1 (main:1268-1390): 8-node gather per particle in the
//                  reference's term order, FP64 without contraction.
//  stage_tri_cic   tri_cic (main:998-1037): 1/rho < 0.01 compaction and a
//                  stable radix sort of the seeds, ties by input index.
#include <algorithm>
#include <cmath>

#include "psod_internal.cuh"

namespace psod {

namespace {

constexpr double FIX_ONE = 1099511627776.0;  // 2^40

// ---------------------------------------------------------------------------
// cell sort
// ---------------------------------------------------------------------------
// Slab partition.  The particles arrive in random order, so a direct
// counting sort into nx^3 cells spreads its atomics and its record writes
// over the whole cube.  A first pass groups them by slab (a run of z-planes
// of cells, at most SLAB_MAX slabs) with coalesced writes: each CTA orders a
// tile of SLAB_TILE particles by slab in shared memory and writes one run
// per slab.  The counting sort then reads the records slab after slab, so at
// any moment its atomics and record writes fall into the few slabs that the
// running CTAs hold, which stay in L2.
constexpr int SLAB_MAX = 512;
constexpr int SLAB_TILE = 4096;
constexpr int SLAB_THREADS = 256;
constexpr int SLAB_PER = SLAB_TILE / SLAB_THREADS;

__device__ __forceinline__ bool in_unit_box(float x, float y, float z) {
  return x >= 0.f && x <= 1.f && y >= 0.f && y <= 1.f && z >= 0.f && z <= 1.f;
}

// slab of a position: its z cell scaled to the slab count (slabs are runs of
// whole z-planes, so runs of cell indices)
__device__ __forceinline__ unsigned slab_of(float z, float nxf, double xs, int nx, int nslab) {
  const int k = sod_cell_axis(to_grid(z, nxf), xs, nx);
  return (unsigned)(((long long)k * nslab) / nx);
}

__global__ void __launch_bounds__(SLAB_THREADS) k_slab_count(const float *pos, long long n, float nxf, double xs,
                                                             int nx, int nslab, unsigned *hist, int *bad) {
  __shared__ unsigned h[SLAB_MAX];
  for (int k = threadIdx.x; k < nslab; k += SLAB_THREADS) h[k] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * SLAB_TILE;
  int badl = 0;
  for (int u = 0; u < SLAB_PER; u++) {
    const long long i = base + (long long)u * SLAB_THREADS + threadIdx.x;
    if (i >= n) break;
    const float x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    if (!in_unit_box(x, y, z)) badl = 1;
    atomicAdd(&h[slab_of(z, nxf, xs, nx, nslab)], 1u);
  }
  if (badl) atomicOr(bad, 1);
  __syncthreads();
  for (int k = threadIdx.x; k < nslab; k += SLAB_THREADS)
    if (h[k]) atomicAdd(&hist[k], h[k]);
}

// exclusive scan of the slab counts into the write cursors (one CTA)
__global__ void k_slab_scan(const unsigned *hist, int nslab, unsigned *cursor) {
  __shared__ unsigned s[SLAB_MAX];
  for (int k = threadIdx.x; k < SLAB_MAX; k += blockDim.x) s[k] = k < nslab ? hist[k] : 0u;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned run = 0;
    for (int k = 0; k < nslab; k++) {
      const unsigned v = s[k];
      cursor[k] = run;
      run += v;
    }
  }
}

// records (x, y, z, input index) grouped by slab; the order inside a slab
// carries no meaning
__global__ void __launch_bounds__(SLAB_THREADS) k_slab_scatter(const float *pos, long long n, float nxf, double xs,
                                                               int nx, int nslab, unsigned *cursor, float4 *rec) {
  __shared__ unsigned cnt[SLAB_MAX], start[SLAB_MAX], gbase[SLAB_MAX];
  extern __shared__ __align__(16) unsigned char slab_smem[];
  float4 *stage = reinterpret_cast<float4 *>(slab_smem);                                // SLAB_TILE records
  unsigned short *sdig = reinterpret_cast<unsigned short *>(stage + SLAB_TILE);          // their slabs
  for (int k = threadIdx.x; k < nslab; k += SLAB_THREADS) cnt[k] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * SLAB_TILE;
  const int m = (int)min((long long)SLAB_TILE, n - base);
  unsigned d[SLAB_PER], r[SLAB_PER];
#pragma unroll
  for (int u = 0; u < SLAB_PER; u++) {
    const int j = u * SLAB_THREADS + threadIdx.x;
    if (j < m) {
      d[u] = slab_of(pos[3 * (base + j) + 2], nxf, xs, nx, nslab);
      r[u] = atomicAdd(&cnt[d[u]], 1u);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned run = 0;
    for (int k = 0; k < nslab; k++) {
      start[k] = run;
      run += cnt[k];
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < nslab; k += SLAB_THREADS)
    if (cnt[k]) gbase[k] = atomicAdd(&cursor[k], cnt[k]);
#pragma unroll
  for (int u = 0; u < SLAB_PER; u++) {
    const int j = u * SLAB_THREADS + threadIdx.x;
    if (j < m) {
      const long long i = base + j;
      const unsigned at = start[d[u]] + r[u];
      stage[at] = make_float4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], __uint_as_float((unsigned)i));
      sdig[at] = (unsigned short)d[u];
    }
  }
  __syncthreads();
  // consecutive threads write consecutive records of each slab's run
  for (int j = threadIdx.x; j < m; j += SLAB_THREADS) {
    const unsigned k = sdig[j];
    rec[gbase[k] + (j - start[k])] = stage[j];
  }
}

__global__ void k_cell_count(const float4 *rec, long long n, float nxf, double3 xs, int nx, unsigned *cell,
                             unsigned *count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned c = 0xffffffffu;
  if (i < n) {
    const float4 v = rec[i];
    const int ci = sod_cell_axis(to_grid(v.x, nxf), xs.x, nx);
    const int cj = sod_cell_axis(to_grid(v.y, nxf), xs.y, nx);
    const int ck = sod_cell_axis(to_grid(v.z, nxf), xs.z, nx);
    c = (unsigned)ci + (unsigned)nx * ((unsigned)cj + (unsigned)nx * (unsigned)ck);
    cell[i] = c;
  }
  // one atomic per distinct cell in the warp
  const unsigned peers = __match_any_sync(0xffffffffu, c);
  if (c != 0xffffffffu && __ffs(peers) - 1 == (int)(threadIdx.x & 31)) atomicAdd(&count[c], __popc(peers));
}

// Cells holding at least SUB_MIN particles are ordered inside by a 4x4x4
// sub-cell key (Morton order), so that consecutive records of a dense cell lie
// close together.  Records inside a cell carry no order of their own (every
// later result is ordered by input index), so this changes no output; it lets
// the refinement hand a warp 32 nearby candidates.
constexpr unsigned SUB_MIN = 64;
constexpr unsigned SUB_N = 64;
constexpr unsigned BIG_FLAG = 0x80000000u;

__device__ __forceinline__ unsigned sub_axis(float xg, double xs) {
  const double d = dsub((double)xg, xs);
  const int s = (int)(dsub(d, floor(d)) * 4.0);
  return (unsigned)min(max(s, 0), 3);
}

__device__ __forceinline__ unsigned sub_key(const float4 &p, float nxf, double3 xs) {
  const unsigned a = sub_axis(to_grid(p.x, nxf), xs.x), b = sub_axis(to_grid(p.y, nxf), xs.y),
                 c = sub_axis(to_grid(p.z, nxf), xs.z);
  return (a & 1u) | ((b & 1u) << 1) | ((c & 1u) << 2) | ((a >> 1) << 3) | ((b >> 1) << 4) | ((c >> 1) << 5);
}

// count[c] becomes BIG_FLAG | table index for cells of SUB_MIN or more
// particles, else the cell's first slot start[c] (the fill cursor of the
// scatter, so that one atomic gives the slot; start < n < 2^31 keeps the
// flag bit clear).  With assign false it only counts them.
__global__ void k_mark_big(unsigned *count, unsigned long long ncell, unsigned *nbig, bool assign,
                           unsigned *bigcell, const unsigned *start) {
  const unsigned long long c = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool big = c < ncell && count[c] >= SUB_MIN;
  const unsigned m = __ballot_sync(0xffffffffu, big);
  const int lane = threadIdx.x & 31;
  unsigned base = 0;
  if (lane == 0 && m) base = atomicAdd(nbig, (unsigned)__popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (!assign || c >= ncell) return;
  if (big) {
    const unsigned idx = base + __popc(m & ((1u << lane) - 1u));
    bigcell[idx] = (unsigned)c;
    count[c] = BIG_FLAG | idx;
  } else {
    count[c] = start[c];
  }
}

__global__ void k_sub_count(const float4 *rec, long long n, const unsigned *cell, const unsigned *count, float nxf,
                            double3 xs, unsigned *tab) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned v = count[cell[i]];
  if (v & BIG_FLAG) atomicAdd(&tab[(unsigned long long)(v & ~BIG_FLAG) * SUB_N + sub_key(rec[i], nxf, xs)], 1u);
}

// one warp per dense cell: sub-cell counts -> absolute start slots
__global__ void k_sub_scan(unsigned *tab, const unsigned *bigcell, unsigned nbig, const unsigned *start) {
  const unsigned b = (unsigned)(((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (b >= nbig) return;
  unsigned *t = tab + (unsigned long long)b * SUB_N;
  const unsigned a0 = t[2 * lane], a1 = t[2 * lane + 1];
  unsigned x = a0 + a1;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  const unsigned excl = start[bigcell[b]] + x - (a0 + a1);
  t[2 * lane] = excl;
  t[2 * lane + 1] = excl + a0;
}

__global__ void k_cell_scatter(const float4 *rec, long long n, const unsigned *cell, unsigned *fill, unsigned *tab,
                               float nxf, double3 xs, float4 *cube, unsigned *inv) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned c = i < n ? cell[i] : 0xffffffffu;
  const unsigned v = i < n ? fill[c] : 0u;  // the flag bit never changes under the atomics below
  const bool big = (v & BIG_FLAG) != 0;
  const float4 r = i < n ? rec[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  const unsigned long long key =
      i >= n ? ~0ull
      : big  ? (1ull << 63) | ((unsigned long long)(v & ~BIG_FLAG) * SUB_N + sub_key(r, nxf, xs))
             : (unsigned long long)c;
  const unsigned peers = __match_any_sync(0xffffffffu, key);
  const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
  unsigned base = 0;
  if (i < n && lane == leader)
    base = big ? atomicAdd(&tab[key & ~(1ull << 63)], __popc(peers)) : atomicAdd(&fill[c], __popc(peers));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (i >= n) return;
  const unsigned slot = base + __popc(peers & ((1u << lane) - 1u));
  cube[slot] = r;
  inv[__float_as_uint(r.w)] = slot;
}

// Dense sub-cells are then ordered by a finer Morton key inside the
// sub-cell: 4, 8 or 16 bins per axis for sub-cells of at least 32, 128 or
// 1024 records, so a bin holds about one record and 64 consecutive records
// of a dense cell span a box a few bins wide.  This is what lets the
// refinement's group boxes stay small in halo cores (tens of thousands of
// particles per cell), where the 4x4x4 order alone leaves a 64-record group
// spread over a whole sub-cell.  Like the sub-cell order it changes no
// output.
constexpr unsigned FINE_MIN = 32, FINE_BINS_MAX = 4096;

__device__ __forceinline__ unsigned fine_axis(float xg, double xs, int bits) {
  const double d = dsub((double)xg, xs);
  const int q = (int)(dsub(d, floor(d)) * (double)(4 << bits));
  return (unsigned)q & ((1u << bits) - 1u);
}

__device__ __forceinline__ unsigned fine_key(const float4 &p, float nxf, double3 xs, int bits) {
  const unsigned a = fine_axis(to_grid(p.x, nxf), xs.x, bits), b = fine_axis(to_grid(p.y, nxf), xs.y, bits),
                 c = fine_axis(to_grid(p.z, nxf), xs.z, bits);
  unsigned k = 0;
  for (int j = 0; j < bits; j++)
    k |= (((a >> j) & 1u) << (3 * j)) | (((b >> j) & 1u) << (3 * j + 1)) | (((c >> j) & 1u) << (3 * j + 2));
  return k;
}

// one CTA per dense cell, its 64 sub-cells in turn: a counting sort of each
// sub-cell of FINE_MIN or more records by its fine key, through tmp (the
// same slots of a spare record array), then back into the cube with inv
// updated.  tab holds the sub-cells' end slots (the scatter's cursors).
__global__ void __launch_bounds__(256) k_sub_fine(float4 *cube, unsigned *inv, float4 *tmp, const unsigned *tab,
                                                  const unsigned *bigcell, const unsigned *start, float nxf,
                                                  double3 xs) {
  __shared__ unsigned hist[FINE_BINS_MAX];
  __shared__ unsigned wtot[8];
  const unsigned b = blockIdx.x;
  const unsigned *t = tab + (unsigned long long)b * SUB_N;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  unsigned a = start[bigcell[b]];
  for (unsigned s = 0; s < SUB_N; s++) {
    const unsigned e = t[s], m = e - a;
    if (m >= FINE_MIN) {
      const int bits = m >= 1024u ? 4 : (m >= 128u ? 3 : 2);
      const unsigned nb = 1u << (3 * bits), per = (nb + 255u) / 256u;  // nb <= 4096: per <= 16
      for (unsigned i = tid; i < nb; i += 256u) hist[i] = 0u;
      __syncthreads();
      for (unsigned i = a + tid; i < e; i += 256u) atomicAdd(&hist[fine_key(cube[i], nxf, xs, bits)], 1u);
      __syncthreads();
      // exclusive scan: thread tid owns bins [tid*per, tid*per + per)
      const unsigned lo = min(nb, (unsigned)tid * per), hi = min(nb, lo + per);
      unsigned own = 0;
      for (unsigned i = lo; i < hi; i++) own += hist[i];
      unsigned x = own;
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) wtot[wid] = x;
      __syncthreads();
      unsigned wbase = 0;
      for (int q = 0; q < wid; q++) wbase += wtot[q];
      unsigned run = wbase + x - own;
      for (unsigned i = lo; i < hi; i++) {
        const unsigned h = hist[i];
        hist[i] = run;
        run += h;
      }
      __syncthreads();
      for (unsigned i = a + tid; i < e; i += 256u) {
        const float4 v = cube[i];
        tmp[a + atomicAdd(&hist[fine_key(v, nxf, xs, bits)], 1u)] = v;
      }
      __syncthreads();
      for (unsigned i = a + tid; i < e; i += 256u) {
        const float4 v = tmp[i];
        cube[i] = v;
        inv[__float_as_uint(v.w)] = i;
      }
      __syncthreads();
    }
    a = e;
  }
}

__global__ void k_set_range(unsigned *a, unsigned long long lo, unsigned long long hi, unsigned v) {
  unsigned long long i = lo + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < hi) a[i] = v;
}

// ---------------------------------------------------------------------------
// CIC along one axis (main:1154-1190): returns the two node indices and the
// weights ddx (upper node) and dex (lower node).
// ---------------------------------------------------------------------------
struct CicConst {
  double xxmin[3], xxmax[3];  // zone with buffer per axis, box units
  double dx, kc;
  double inv_dx;  // 1/dx when it is exact (dx a power of two), else 0
  int nc;
  int zone_test;  // 1: particles outside the zone with buffer are skipped (main:1138-1146)
};

// CIC along one axis (main:1154-1190): the two node indices and the weights
// ddx (upper node) and dex (lower node).  (x - xxmin)/dx is formed as a
// product when 1/dx is exact, which gives the same double.
__device__ __forceinline__ void cic_axis(float xf, const CicConst &k, int a, int &i0, int &i1, double &dd, double &de) {
  const double diff = dsub((double)xf, k.xxmin[a]);
  double d = k.inv_dx != 0.0 ? dmul(diff, k.inv_dx) : ddiv(diff, k.dx);
  int ix = (int)d;  // Fortran int(): truncation
  if (d < 0.0) ix = ix - 1;
  d = dsub(d, (double)ix);
  const double e = dsub(1.0, d);
  int ixp1 = ix + 1;
  const int nc = k.nc;
  if (ixp1 < 0) ixp1 += nc;
  if (ix < 0) ix += nc;
  if (ixp1 >= nc) ixp1 -= nc;
  if (ix >= nc) ix -= nc;
  i0 = ix;
  i1 = ixp1;
  dd = d;
  de = e;
}

__device__ __forceinline__ bool in_zone_periodic(double x, double lo, double hi) {
  return (x >= lo && x <= hi) || (x >= dadd(lo, 1.0) && x <= dadd(hi, 1.0)) ||
         (x >= dsub(lo, 1.0) && x <= dsub(hi, 1.0));
}

// the particle selection of cic and cicm1 (main:1138-1146, 1309-1317)
__device__ __forceinline__ bool in_cic_zone(const float4 &p, const CicConst &k) {
  return in_zone_periodic(p.x, k.xxmin[0], k.xxmax[0]) && in_zone_periodic(p.y, k.xxmin[1], k.xxmax[1]) &&
         in_zone_periodic(p.z, k.xxmin[2], k.xxmax[2]);
}

// deposit: 8 int64 atomics per particle, weights quantised to 2^-40
__global__ void k_cic_deposit(const float4 *cube, long long n, CicConst k, unsigned long long *grid) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = cube[i];
  if (!in_cic_zone(p, k)) return;
  int ix, ixp, iy, iyp, iz, izp;
  double ddx, dex, ddy, dey, ddz, dez;
  cic_axis(p.x, k, 0, ix, ixp, ddx, dex);
  cic_axis(p.y, k, 1, iy, iyp, ddy, dey);
  cic_axis(p.z, k, 2, iz, izp, ddz, dez);
  const long long nc = k.nc;
  const int cx[2] = {ix, ixp}, cy[2] = {iy, iyp}, cz[2] = {iz, izp};
  const double wx[2] = {dex, ddx}, wy[2] = {dey, ddy}, wz[2] = {dez, ddz};
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const int a = c & 1, b = (c >> 1) & 1, e = c >> 2;
    double w = dmul(dmul(wx[a], wy[b]), wz[e]);
    unsigned long long q = (unsigned long long)__double2ll_rn(dmul(w, FIX_ONE));
    long long node = (long long)cx[a] + nc * ((long long)cy[b] + nc * (long long)cz[e]);
    atomicAdd(&grid[node], q);
  }
}

// interpolation: rho in the reference's term order (main:1368-1383)
__global__ void k_cic_interp(const float4 *cube, long long n, CicConst k, const unsigned long long *grid,
                             double *rho) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = cube[i];
  unsigned idx = __float_as_uint(p.w) & PSOD_IDX_MASK;
  if (!in_cic_zone(p, k)) {
    rho[idx] = 0.0;
    return;
  }
  int ix, ixp, iy, iyp, iz, izp;
  double ddx, dex, ddy, dey, ddz, dez;
  cic_axis(p.x, k, 0, ix, ixp, ddx, dex);
  cic_axis(p.y, k, 1, iy, iyp, ddy, dey);
  cic_axis(p.z, k, 2, iz, izp, ddz, dez);
  const long long nc = k.nc;
  const int cx[2] = {ix, ixp}, cy[2] = {iy, iyp}, cz[2] = {iz, izp};
  const double wx[2] = {dex, ddx}, wy[2] = {dey, ddy}, wz[2] = {dez, ddz};
  double r = 0.0;
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const int a = c & 1, b = (c >> 1) & 1, e = c >> 2;
    long long node = (long long)cx[a] + nc * ((long long)cy[b] + nc * (long long)cz[e]);
    double g = dmul((double)(long long)grid[node], k.kc);
    r = dadd(r, dmul(dmul(dmul(g, wx[a]), wy[b]), wz[e]));
  }
  rho[idx] = r;
}

// Tile-fused CIC: one CTA owns CT^3 SOD cells.  It deposits the particles
// of those cells and of a one-cell halo into a shared-memory window of
// fixed-point nodes, then interpolates rho for its own particles.  Every
// node the own particles read receives all its contributions inside the
// window, so the integer node sums, and therefore rho, equal the global
// grid's exactly.  Needs each particle's CIC cell to be one of the two fine
// cells of its SOD cell (true when nx is a power of two); a particle that
// breaks this sets *bad and the caller falls back to the global grid.
constexpr int CT = 8;                 // SOD cells per tile side
constexpr int CW = 2 * (CT + 2) + 1;  // window nodes per side
constexpr int CW3 = CW * CW * CW;
constexpr unsigned DEP_BATCH = 4;    // record loads in flight per thread in the deposit

constexpr int CRNG = 2 * (CT + 2) * (CT + 2);  // record ranges of a tile plus halo (two where x wraps)

// exclusive prefix of s_len[0..n) into s_pre[0..n], n <= 32 * 8, by warp 0
__device__ __forceinline__ void range_prefix(const unsigned *s_len, unsigned *s_pre, int n) {
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x, per = (n + 31) / 32, lo = lane * per;
  unsigned t = 0;
  for (int i = lo; i < min(n, lo + per); i++) t += s_len[i];
  unsigned x = t;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  unsigned run = x - t;
  for (int i = lo; i < min(n, lo + per); i++) {
    s_pre[i] = run;
    run += s_len[i];
  }
  if (lane == 31) s_pre[n] = x;
}

// ZONE: particles outside the zone with buffer are skipped (zone contexts;
// the test costs registers, so one-zone contexts run without it)
template <bool ZONE>
__global__ void __launch_bounds__(256) k_cic_tile(const float4 *cube, const unsigned *cs, int nx, double3 xs, CicConst k,
                                                  double *rho, int *bad, unsigned quirk_pos) {
  extern __shared__ __align__(16) unsigned long long win[];
  __shared__ unsigned s_rb[CRNG], s_len[CRNG], s_pre[CRNG + 1];
  const int ntile = nx / CT;
  const int tx = blockIdx.x % ntile, ty = (blockIdx.x / ntile) % ntile, tz = blockIdx.x / (ntile * ntile);
  const int x0 = tx * CT, y0 = ty * CT, z0 = tz * CT;
  const int nc = k.nc;  // 2*nx fine cells
  const float nxf = (float)nx;
  for (int i = threadIdx.x; i < CW3; i += blockDim.x) win[i] = 0ull;
  auto widx = [&](int f, int o) {  // fine index -> window offset (periodic)
    int d = f - o;
    if (d < 0) d += nc;
    if (d >= nc) d -= nc;
    return d;
  };
  const int ox = 2 * (x0 - 1), oy = 2 * (y0 - 1), oz = 2 * (z0 - 1);
  // record ranges of the rows of the tile plus halo; the particles are then
  // dealt to all threads of the CTA evenly, whatever their spread over rows
  for (int row = threadIdx.x; row < (CT + 2) * (CT + 2); row += blockDim.x) {
    const int yy = (y0 - 1 + row % (CT + 2) + nx) % nx, zz = (z0 - 1 + row / (CT + 2) + nx) % nx;
    const unsigned long long base = (unsigned long long)nx * ((unsigned)yy + (unsigned long long)nx * (unsigned)zz);
    const int xa = x0 - 1, xb = x0 + CT;  // inclusive, may wrap
    int pa[2] = {0, 0}, pb[2] = {-1, -1};
    if (xa < 0) { pa[0] = xa + nx; pb[0] = nx - 1; pa[1] = 0; pb[1] = xb; }
    else if (xb >= nx) { pa[0] = xa; pb[0] = nx - 1; pa[1] = 0; pb[1] = xb - nx; }
    else { pa[0] = xa; pb[0] = xb; }
    for (int q = 0; q < 2; q++) {
      unsigned rb = 0, len = 0;
      if (pb[q] >= pa[q]) {
        rb = cs[base + (unsigned)pa[q]];
        len = cs[base + (unsigned)pb[q] + 1] - rb;
        // the quirk particle (the cube's last record, at the end of its
        // listed cell's run) is deposited below from its own cell
        if (len && rb + len - 1u == quirk_pos) len--;
      }
      s_rb[2 * row + q] = rb;
      s_len[2 * row + q] = len;
    }
  }
  __syncthreads();
  range_prefix(s_len, s_pre, CRNG);
  __syncthreads();
  {
    // Each thread deposits one contiguous share of the tile's particles
    // (all threads busy, whatever the tile's count).  Dense cells are
    // sub-cell ordered, so consecutive particles mostly share a fine cell
    // and its 8 nodes: their fixed-point weights are summed in registers and
    // written with one atomic per node when the fine cell changes (integer
    // sums, so the grid is the same).  Records are loaded DEP_BATCH at a
    // time before any is used.
    const unsigned total = s_pre[CRNG];
    const unsigned per = (total + blockDim.x - 1) / blockDim.x;
    const unsigned f0 = min(total, threadIdx.x * per), f1 = min(total, f0 + per);
    int r = 0;  // last range with s_pre[r] <= f0
    {
      int hi = CRNG;
      while (hi - r > 1) {
        const int mid = (r + hi) >> 1;
        if (s_pre[mid] <= f0) r = mid;
        else hi = mid;
      }
    }
    unsigned long long acc[8];
    int kx = -1, ky = -1, kz = -1;  // fine cell of the accumulated run
    int ncx[2], ncy[2], ncz[2];     // its nodes' window offsets
    auto flush = [&]() {
      if (kx < 0) return;
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const int a = c & 1, bb = (c >> 1) & 1, ee = c >> 2;
        if (ncx[a] < CW && ncy[bb] < CW && ncz[ee] < CW && acc[c])
          atomicAdd(&win[ncx[a] + CW * (ncy[bb] + CW * ncz[ee])], acc[c]);
      }
      kx = -1;
    };
    for (unsigned fb = f0; fb < f1; fb += DEP_BATCH) {
      float4 vb[DEP_BATCH];
#pragma unroll
      for (unsigned u = 0; u < DEP_BATCH; u++) {
        const unsigned f = fb + u;
        if (f < f1) {
          while (s_pre[r + 1] <= f) r++;
          vb[u] = cube[s_rb[r] + (f - s_pre[r])];
        }
      }
#pragma unroll
      for (unsigned u = 0; u < DEP_BATCH; u++) {
        if (fb + u >= f1) break;
        const float4 v = vb[u];
        int ix, ixp, iy, iyp, iz, izp;
        double ddx, dex, ddy, dey, ddz, dez;
        cic_axis(v.x, k, 0, ix, ixp, ddx, dex);
        cic_axis(v.y, k, 1, iy, iyp, ddy, dey);
        cic_axis(v.z, k, 2, iz, izp, ddz, dez);
        if (ZONE && !in_cic_zone(v, k)) continue;
        const int sx = sod_cell_axis(to_grid(v.x, nxf), xs.x, nx), sy = sod_cell_axis(to_grid(v.y, nxf), xs.y, nx),
                  sz = sod_cell_axis(to_grid(v.z, nxf), xs.z, nx);
        if ((ix >> 1) != sx || (iy >> 1) != sy || (iz >> 1) != sz) {
          atomicOr(bad, 1);
          continue;
        }
        if (ix != kx || iy != ky || iz != kz) {
          flush();
          kx = ix;
          ky = iy;
          kz = iz;
          ncx[0] = widx(ix, ox);
          ncx[1] = widx(ixp, ox);
          ncy[0] = widx(iy, oy);
          ncy[1] = widx(iyp, oy);
          ncz[0] = widx(iz, oz);
          ncz[1] = widx(izp, oz);
#pragma unroll
          for (int c = 0; c < 8; c++) acc[c] = 0ull;
        }
        const double wx[2] = {dex, ddx}, wy[2] = {dey, ddy}, wz[2] = {dez, ddz};
#pragma unroll
        for (int c = 0; c < 8; c++) {
          const int a = c & 1, bb = (c >> 1) & 1, ee = c >> 2;
          const double wgt = dmul(dmul(wx[a], wy[bb]), wz[ee]);
          acc[c] += (unsigned long long)__double2ll_rn(dmul(wgt, FIX_ONE));
        }
      }
    }
    flush();
  }
  // The run scan files a single particle of the last cell under the
  // previous cell's run (the linked-list quirk), which may lie in another
  // tile.  Its CIC weights belong to its own cell: every tile whose cells
  // with halo hold that cell deposits it, and the tile owning the cell
  // interpolates it.
  auto cell_rel = [&](int c, int c0) {  // periodic offset of cell c from c0 - 1
    int d = c - (c0 - 1);
    if (d < 0) d += nx;
    if (d >= nx) d -= nx;
    return d;
  };
  float4 vq = make_float4(0.f, 0.f, 0.f, 0.f);
  int qx = 0, qy = 0, qz = 0;
  const bool has_q = quirk_pos != 0xffffffffu;
  if (has_q) {
    vq = cube[quirk_pos];
    qx = cell_rel(sod_cell_axis(to_grid(vq.x, nxf), xs.x, nx), x0);
    qy = cell_rel(sod_cell_axis(to_grid(vq.y, nxf), xs.y, nx), y0);
    qz = cell_rel(sod_cell_axis(to_grid(vq.z, nxf), xs.z, nx), z0);
  }
  if (threadIdx.x == 0 && has_q && qx <= CT + 1 && qy <= CT + 1 && qz <= CT + 1 &&
      !(ZONE && !in_cic_zone(vq, k))) {
    int ix, ixp, iy, iyp, iz, izp;
    double ddx, dex, ddy, dey, ddz, dez;
    cic_axis(vq.x, k, 0, ix, ixp, ddx, dex);
    cic_axis(vq.y, k, 1, iy, iyp, ddy, dey);
    cic_axis(vq.z, k, 2, iz, izp, ddz, dez);
    const int cx[2] = {widx(ix, ox), widx(ixp, ox)}, cy[2] = {widx(iy, oy), widx(iyp, oy)},
              cz[2] = {widx(iz, oz), widx(izp, oz)};
    const double wx[2] = {dex, ddx}, wy[2] = {dey, ddy}, wz[2] = {dez, ddz};
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int a = c & 1, bb = (c >> 1) & 1, ee = c >> 2;
      if (cx[a] < CW && cy[bb] < CW && cz[ee] < CW) {
        const double wgt = dmul(dmul(wx[a], wy[bb]), wz[ee]);
        atomicAdd(&win[cx[a] + CW * (cy[bb] + CW * cz[ee])], (unsigned long long)__double2ll_rn(dmul(wgt, FIX_ONE)));
      }
    }
  }
  __syncthreads();
  // own particles: rho in the reference's term order (main:1368-1383)
  for (int row = threadIdx.x; row < CT * CT; row += blockDim.x) {
    const int yy = y0 + row % CT, zz = z0 + row / CT;
    const unsigned long long base = (unsigned long long)nx * ((unsigned)yy + (unsigned long long)nx * (unsigned)zz);
    const unsigned rb = cs[base + (unsigned)x0];
    unsigned len = cs[base + (unsigned)(x0 + CT - 1) + 1] - rb;
    if (len && rb + len - 1u == quirk_pos) len--;  // interpolated below, by its own cell's tile
    s_rb[row] = rb;
    s_len[row] = len;
  }
  __syncthreads();
  range_prefix(s_len, s_pre, CT * CT);
  __syncthreads();
  const unsigned total = s_pre[CT * CT];
  auto interp = [&](const float4 v) {
    const unsigned idx = __float_as_uint(v.w) & PSOD_IDX_MASK;
    if (ZONE && !in_cic_zone(v, k)) {  // not selected by cicm1: rho stays 0
      rho[idx] = 0.0;
      return;
    }
    int ix, ixp, iy, iyp, iz, izp;
    double ddx, dex, ddy, dey, ddz, dez;
    cic_axis(v.x, k, 0, ix, ixp, ddx, dex);
    cic_axis(v.y, k, 1, iy, iyp, ddy, dey);
    cic_axis(v.z, k, 2, iz, izp, ddz, dez);
    const int cx[2] = {widx(ix, ox), widx(ixp, ox)}, cy[2] = {widx(iy, oy), widx(iyp, oy)},
              cz[2] = {widx(iz, oz), widx(izp, oz)};
    const double wx[2] = {dex, ddx}, wy[2] = {dey, ddy}, wz[2] = {dez, ddz};
    double rr = 0.0;
    bool ok = true;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int a = c & 1, bb = (c >> 1) & 1, ee = c >> 2;
      if (cx[a] >= CW || cy[bb] >= CW || cz[ee] >= CW) {
        ok = false;
        continue;
      }
      const double gval = dmul((double)(long long)win[cx[a] + CW * (cy[bb] + CW * cz[ee])], k.kc);
      rr = dadd(rr, dmul(dmul(dmul(gval, wx[a]), wy[bb]), wz[ee]));
    }
    if (!ok) atomicOr(bad, 1);
    rho[idx] = rr;
  };
  // two records per thread and step, both loaded before either is used
  int r = 0;
  for (unsigned fa = threadIdx.x; fa < total; fa += 2 * blockDim.x) {
    const unsigned fb = fa + blockDim.x;
    while (s_pre[r + 1] <= fa) r++;
    const float4 va = cube[s_rb[r] + (fa - s_pre[r])];
    float4 vb = va;
    if (fb < total) {
      while (s_pre[r + 1] <= fb) r++;
      vb = cube[s_rb[r] + (fb - s_pre[r])];
    }
    interp(va);
    if (fb < total) interp(vb);
  }
  // the quirk particle, by the tile that owns its cell
  if (threadIdx.x == 0 && has_q && qx >= 1 && qx <= CT && qy >= 1 && qy <= CT && qz >= 1 && qz <= CT) interp(vq);
}

__global__ void k_grid_to_double(const unsigned long long *grid, long long nnode, double kc, double *out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nnode) out[i] = dmul((double)(long long)grid[i], kc);
}

// ---------------------------------------------------------------------------
// seeds
// ---------------------------------------------------------------------------
// Seed flags (1/rho < 0.01) and the smallest key of the others.  Fixed
// grid, each thread over a strided range; one atomic per CTA (a per-warp
// atomic on the single minimum serialises tens of millions of updates).
__global__ void __launch_bounds__(256) k_seed_flags(const double *rho, long long n, unsigned *flag,
                                                    unsigned long long *minbits) {
  __shared__ unsigned long long s_min[8];
  unsigned long long mb = ~0ull;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double pd = ddiv(1.0, rho[i]);  // main:1022
    unsigned f = 0;
    if (pd < 0.01) {
      f = 1;  // main:1029: 1/rho < 1/100
    } else {
      const unsigned long long b = dbits(pd);
      mb = b < mb ? b : mb;
    }
    flag[i] = f;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_down_sync(0xffffffffu, mb, o);
    mb = t < mb ? t : mb;
  }
  if ((threadIdx.x & 31) == 0) s_min[threadIdx.x >> 5] = mb;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x >> 5); q++) mb = s_min[q] < mb ? s_min[q] : mb;
    if (mb != ~0ull) atomicMin(minbits, mb);
  }
}

__global__ void k_seed_extra_idx(const double *rho, long long n, unsigned long long minbits, unsigned *minidx) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double pd = ddiv(1.0, rho[i]);
  if (!(pd < 0.01) && dbits(pd) == minbits) atomicMin(minidx, (unsigned)i);
}

__global__ void k_seed_compact(const double *rho, long long n, const unsigned *flag, const unsigned *pos,
                               unsigned long long *keys, unsigned *vals) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flag[i]) return;
  unsigned o = pos[i];
  keys[o] = dbits(ddiv(1.0, rho[i]));
  vals[o] = (unsigned)i;
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// ---------------------------------------------------------------------------
int stage_cellsort(psod_ctx *c, const float *dpos) {
  const long long n = c->n;
  const int nx = c->nx;
  c->ncell = (unsigned long long)nx * nx * nx;
  int st;
  unsigned *cell = nullptr, *count = nullptr, *slabs = nullptr;
  float4 *rec = nullptr;
  int *bad = nullptr;
  if ((st = scratch(c, SLOT_PART_U32, (size_t)n, &cell))) return st;
  if ((st = scratch(c, SLOT_SLAB_REC, (size_t)n, &rec))) return st;
  if ((st = scratch(c, SLOT_SLABS, 2 * SLAB_MAX, &slabs))) return st;
  if ((st = scratch(c, SLOT_CELL_U32, (size_t)c->ncell + 1, &count))) return st;
  if ((st = scratch(c, SLOT_LOAD_FLAGS, 2, &bad))) return st;
  if ((st = ensure(c, &c->d_cell_start, &c->cs_cap, (size_t)c->ncell + 1))) return st;
  if ((st = ensure(c, &c->d_cube, &c->cube_cap, (size_t)n))) return st;
  if ((st = ensure(c, &c->d_inv, &c->inv_cap, (size_t)n))) return st;
  PSOD_CUDA(c, cudaMemsetAsync(count, 0, sizeof(unsigned) * (c->ncell + 1), c->stream));
  PSOD_CUDA(c, cudaMemsetAsync(bad, 0, 2 * sizeof(int), c->stream));
  // xxmin*scale per axis (main:1565); slabs follow the z axis
  const double3 xs = make_double3(c->xxmin[0] * c->scale, c->xxmin[1] * c->scale, c->xxmin[2] * c->scale);
  // records grouped by slab first (see k_slab_scatter)
  const int nslab = std::min(nx, SLAB_MAX);
  PSOD_CUDA(c, cudaMemsetAsync(slabs, 0, sizeof(unsigned) * SLAB_MAX, c->stream));
  const unsigned ntile = nblk(n, SLAB_TILE);
  k_slab_count<<<ntile, SLAB_THREADS, 0, c->stream>>>(dpos, n, (float)nx, xs.z, nx, nslab, slabs, bad);
  k_slab_scan<<<1, 32, 0, c->stream>>>(slabs, nslab, slabs + SLAB_MAX);
  const int slab_smem = SLAB_TILE * (int)(sizeof(float4) + sizeof(unsigned short));
  PSOD_CUDA(c, cudaFuncSetAttribute(k_slab_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, slab_smem));
  k_slab_scatter<<<ntile, SLAB_THREADS, slab_smem, c->stream>>>(dpos, n, (float)nx, xs.z, nx, nslab, slabs + SLAB_MAX,
                                                                rec);
  k_cell_count<<<nblk(n, 256), 256, 0, c->stream>>>(rec, n, (float)nx, xs, nx, cell, count);
  if ((st = scan_u32(c, count, c->d_cell_start, (long long)c->ncell, true))) return st;
  unsigned *nbig = reinterpret_cast<unsigned *>(bad + 1);
  const long long ncell = (long long)c->ncell;
  k_mark_big<<<nblk(ncell, 256), 256, 0, c->stream>>>(count, c->ncell, nbig, false, nullptr, nullptr);
  int hflags[2] = {0, 0};
  PSOD_CUDA(c, cudaMemcpyAsync(hflags, bad, sizeof(hflags), cudaMemcpyDeviceToHost, c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  const int hbad = hflags[0];
  const unsigned hnbig = (unsigned)hflags[1];
  unsigned *tab = nullptr, *bigcell = nullptr;
  if (!hbad) {
    if ((st = scratch(c, SLOT_BIG_TAB, (size_t)hnbig * SUB_N + 1, &tab))) return st;
    if ((st = scratch(c, SLOT_BIG_CELL, (size_t)hnbig + 1, &bigcell))) return st;
    PSOD_CUDA(c, cudaMemsetAsync(nbig, 0, sizeof(unsigned), c->stream));
    PSOD_CUDA(c, cudaMemsetAsync(tab, 0, sizeof(unsigned) * ((size_t)hnbig * SUB_N + 1), c->stream));
    k_mark_big<<<nblk(ncell, 256), 256, 0, c->stream>>>(count, c->ncell, nbig, true, bigcell, c->d_cell_start);
    if (hnbig) {
      k_sub_count<<<nblk(n, 256), 256, 0, c->stream>>>(rec, n, cell, count, (float)nx, xs, tab);
      k_sub_scan<<<nblk((long long)hnbig * 32, 256), 256, 0, c->stream>>>(tab, bigcell, hnbig, c->d_cell_start);
    }
    k_cell_scatter<<<nblk(n, 256), 256, 0, c->stream>>>(rec, n, cell, count, tab, (float)nx, xs, c->d_cube,
                                                        c->d_inv);
    // rec is free once the scatter has read it
    if (hnbig)
      k_sub_fine<<<hnbig, 256, 0, c->stream>>>(c->d_cube, c->d_inv, rec, tab, bigcell, c->d_cell_start, (float)nx, xs);
    PSOD_CUDA(c, cudaGetLastError());
    PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  if (hbad) return set_err(c, PSOD_ERR_ARG, "particle positions must lie in [0,1] (box units)");

  // The reference's run scan (main:1591-1604) files a final cell holding a
  // single particle under the previous run.  Reproduce that by extending the
  // previous cell's range over it.
  c->has_quirk = 0;
  c->quirk_pos = 0xffffffffu;
  if (n >= 2) {
    float4 last2[2];
    PSOD_CUDA(c, cudaMemcpyAsync(last2, c->d_cube + (n - 2), sizeof(last2), cudaMemcpyDeviceToHost, c->stream));
    PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
    auto host_cell = [&](const float4 &p) {
      const float v[3] = {p.x, p.y, p.z};
      unsigned idx[3];
      for (int a = 0; a < 3; a++) {
        float xg = v[a] * (float)nx;  // exact product rounded once, as on the device
        int i = (int)std::floor((double)xg - (a == 0 ? xs.x : a == 1 ? xs.y : xs.z));
        if (i < 0) i += nx;
        if (i >= nx) i -= nx;
        idx[a] = (unsigned)i;
      }
      return idx[0] + (unsigned)nx * (idx[1] + (unsigned)nx * idx[2]);
    };
    unsigned ca = host_cell(last2[0]), cl = host_cell(last2[1]);
    if (ca != cl) {
      c->has_quirk = 1;
      c->quirk_pos = (unsigned)(n - 1);
      c->quirk_listed = ca;
      c->quirk_phys = cl;
      unsigned long long lo = (unsigned long long)ca + 1, hi = (unsigned long long)cl + 1;
      k_set_range<<<nblk((long long)(hi - lo), 256), 256, 0, c->stream>>>(c->d_cell_start, lo, hi, (unsigned)n);
    }
  }
  PSOD_CUDA(c, cudaGetLastError());
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  return PSOD_OK;
}

static CicConst make_cic_const(const psod_ctx *c) {
  CicConst k;
  k.nc = 2 * c->nx;                                 // main:667
  k.dx = 1.0 / (double)k.nc;                        // main:1126
  k.inv_dx = ((k.nc & (k.nc - 1)) == 0) ? (double)k.nc : 0.0;
  for (int a = 0; a < 3; a++) {
    k.xxmin[a] = c->xxmin[a];                       // main:665
    k.xxmax[a] = c->xxmax[a];                       // zone + buffer upper edge
  }
  // one zone covers the box: every particle is selected
  k.zone_test = c->nxcpu > 1 ? 1 : 0;
  const double vol = (k.dx * k.dx) * k.dx;          // main:1263
  k.kc = ((double)c->mpf / FIX_ONE) / vol;
  return k;
}

int stage_cic(psod_ctx *c, double *grid_out) {
  CicConst k = make_cic_const(c);
  const long long nnode = (long long)k.nc * k.nc * k.nc;
  int st;
  if (!c->d_rho || c->rho_cap < c->n) {
    if ((st = dalloc(c, &c->d_rho, (size_t)c->n))) return st;
    c->rho_cap = c->n;
  }
  // fused tile path (no global grid) when the box tiles evenly
  bool tiled = false;
  if (c->nx % CT == 0 && c->nx >= 2 * (CT + 2)) {
    int *bad = nullptr;
    if ((st = scratch(c, SLOT_CIC_FLAG, 1, &bad))) return st;
    PSOD_CUDA(c, cudaMemsetAsync(bad, 0, sizeof(int), c->stream));
    const int smem = CW3 * (int)sizeof(unsigned long long);
    PSOD_CUDA(c, cudaFuncSetAttribute(k_cic_tile<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    PSOD_CUDA(c, cudaFuncSetAttribute(k_cic_tile<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const long long ntiles = (long long)(c->nx / CT) * (c->nx / CT) * (c->nx / CT);
    const double3 xs = make_double3(c->xxmin[0] * c->scale, c->xxmin[1] * c->scale, c->xxmin[2] * c->scale);
    const unsigned qpos = c->has_quirk ? c->quirk_pos : 0xffffffffu;
    if (k.zone_test)
      k_cic_tile<true><<<(unsigned)ntiles, 256, smem, c->stream>>>(c->d_cube, c->d_cell_start, c->nx, xs, k, c->d_rho,
                                                                   bad, qpos);
    else
      k_cic_tile<false><<<(unsigned)ntiles, 256, smem, c->stream>>>(c->d_cube, c->d_cell_start, c->nx, xs, k, c->d_rho,
                                                                    bad, qpos);
    int hbad = 0;
    PSOD_CUDA(c, cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
    tiled = (hbad == 0);
  }
  if (!tiled || grid_out) {
    if ((st = dalloc(c, &c->d_grid, (size_t)nnode))) return st;
    PSOD_CUDA(c, cudaMemsetAsync(c->d_grid, 0, sizeof(unsigned long long) * nnode, c->stream));
    k_cic_deposit<<<nblk(c->n, 256), 256, 0, c->stream>>>(c->d_cube, c->n, k, c->d_grid);
    if (!tiled) k_cic_interp<<<nblk(c->n, 256), 256, 0, c->stream>>>(c->d_cube, c->n, k, c->d_grid, c->d_rho);
  }
  c->cic_tiled = tiled;
  PSOD_CUDA(c, cudaGetLastError());
  if (grid_out) {
    double *tmp = nullptr;
    if (is_device_ptr(grid_out)) {
      tmp = grid_out;
    } else if ((st = dalloc(c, &tmp, (size_t)nnode))) {
      return st;
    }
    k_grid_to_double<<<nblk(nnode, 256), 256, 0, c->stream>>>(c->d_grid, nnode, k.kc, tmp);
    if (tmp != grid_out) {
      st = copy_out(c, grid_out, tmp, sizeof(double) * nnode);
      dfree(&tmp);
      if (st) return st;
    }
  }
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  dfree(&c->d_grid);
  c->cic_done = true;
  c->rho_done = true;
  return PSOD_OK;
}

int stage_cicm1(psod_ctx *c, double *rho_out) {
  if (!c->rho_done) return set_err(c, PSOD_ERR_STATE, "psod_cicm1 needs psod_cic first");
  if (rho_out) return copy_out(c, rho_out, c->d_rho, sizeof(double) * c->n);
  return PSOD_OK;
}

int stage_tri_cic(psod_ctx *c, int64_t *isort_out) {
  if (!c->rho_done) return set_err(c, PSOD_ERR_STATE, "psod_tri_cic needs psod_cic first");
  const long long n = c->n;
  int st;
  unsigned *flag = nullptr, *posn = nullptr, *minidx = nullptr;
  unsigned long long *minbits = nullptr, *keys = nullptr;
  if ((st = scratch(c, SLOT_PART_U32, (size_t)n, &flag))) return st;
  if ((st = scratch(c, SLOT_PART_U64, (size_t)n + 1, &posn))) return st;
  if ((st = scratch(c, SLOT_TRI_MIN, 2, &minbits))) return st;
  minidx = reinterpret_cast<unsigned *>(minbits + 1);
  PSOD_CUDA(c, cudaMemsetAsync(minbits, 0xff, sizeof(unsigned long long), c->stream));
  PSOD_CUDA(c, cudaMemsetAsync(minidx, 0xff, sizeof(unsigned), c->stream));
  {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(nblk(n, 256), (long long)sms * 8));
    k_seed_flags<<<grid, 256, 0, c->stream>>>(c->d_rho, n, flag, minbits);
  }
  if ((st = scan_u32(c, flag, posn, n, true))) return st;
  unsigned nd = 0;
  unsigned long long hmin = 0;
  PSOD_CUDA(c, cudaMemcpyAsync(&nd, posn + n, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
  PSOD_CUDA(c, cudaMemcpyAsync(&hmin, minbits, sizeof(hmin), cudaMemcpyDeviceToHost, c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  const bool has_extra = hmin != ~0ull;
  if (has_extra) k_seed_extra_idx<<<nblk(n, 256), 256, 0, c->stream>>>(c->d_rho, n, hmin, minidx);
  const long long nseed = (long long)nd + (has_extra ? 1 : 0);
  if ((st = scratch(c, SLOT_TRI_KEYS, (size_t)nd + 1, &keys))) return st;
  if ((st = scratch(c, SLOT_SEED_IDX, (size_t)nseed + 1, &c->d_seed_idx))) return st;
  k_seed_compact<<<nblk(n, 256), 256, 0, c->stream>>>(c->d_rho, n, flag, posn, keys, c->d_seed_idx);
  // seeds arrive in input order; a stable sort on 1/rho leaves ties in
  // input order
  if ((st = radix_sort_u64(c, keys, c->d_seed_idx, (long long)nd, 64))) return st;
  if (has_extra)
    PSOD_CUDA(c, cudaMemcpyAsync(c->d_seed_idx + nd, minidx, sizeof(unsigned), cudaMemcpyDeviceToDevice, c->stream));
  PSOD_CUDA(c, cudaGetLastError());
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  c->nseed_dense = nd;
  c->npart_new = nseed;  // main:1032 (clamped to n when every particle is dense)
  if (isort_out && nseed > 0) {
    std::vector<unsigned> h((size_t)nseed);
    PSOD_CUDA(c, cudaMemcpy(h.data(), c->d_seed_idx, sizeof(unsigned) * nseed, cudaMemcpyDeviceToHost));
    if (is_device_ptr(isort_out)) {
      std::vector<int64_t> hh(h.begin(), h.end());
      PSOD_CUDA(c, cudaMemcpy(isort_out, hh.data(), sizeof(int64_t) * nseed, cudaMemcpyHostToDevice));
    } else {
      for (long long i = 0; i < nseed; i++) isort_out[i] = (int64_t)h[(size_t)i];
    }
  }
  c->seeds_done = true;
  return PSOD_OK;
}

}  // namespace psod
