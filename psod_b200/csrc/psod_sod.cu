// psod_sod.cu -- spherover (main:1396-2201) on the GPU.
//
// Seeds are processed in the reference's order semantics but many at a time.
// Seed k depends on seed j < k only through particles that j claims inside
// its preselect cube (+-ncut cells) and that k reads inside +-max(ncut,2)
// cells.  Per scheduler round, a seed is ready when no unresolved seed of
// lower rank lies within ncut + max(ncut,2) cells (checked on a coarse
// block grid, which is conservative).  Ready seeds therefore touch disjoint
// particles and give exactly the sequential result.
//
// One CTA processes one ready seed (work stealing over the ready list):
//   1. count alive particles of the +-ncut cube (nsel / Mmin tests, main:1681, 1759)
//   2. centre refinement over the +-1 cells (main:1799-1909): per candidate
//      the sum of 1/sqrt(d2+eps2) over alive particles within one cell,
//      accumulated in int64 fixed point (order independent); argmax with
//      ties to the first candidate in the reference's scan order
//   3. radial selection instead of a full sort (main:2030-2100): 4096-bucket
//      histograms over the FP64 bit pattern of d2 locate the bucket that can
//      hold the crossing; only that bucket is sorted.  A bucket can be skipped
//      exactly: the reference's overdensity i/(cvol*r^3), evaluated with
//      correctly rounded FP64 operations, is monotone in i and in d2.
//   4. profile counts (main:2103-2115) and claims (main:2148-2166).
#include <algorithm>
#include <cmath>

#include "psod_internal.cuh"

namespace psod {

namespace {

constexpr int TPB = 256;          // threads per seed CTA
constexpr int NWARP = TPB / 32;
constexpr int NB = 4096;          // histogram buckets per level
constexpr int MAXLEV = 4;         // histogram levels kept in shared memory
constexpr int CAP = 2048;         // elements sorted in shared memory
constexpr unsigned long long L1_BASE = 128896ull;  // (1023-16) << 7
constexpr int L1_SHIFT = 45;

enum { ERR_NONE = 0 };

struct SodBufs {
  float4 *cube;
  const unsigned *cs;        // cell_start
  const long long *ids;
  const unsigned *seed_idx;  // rank -> input index
  const unsigned *inv;       // input index -> cube position
  const double *edge_fac;    // [nbins]
  unsigned char *processed;  // per rank
  const unsigned *ready;
  const unsigned *nready;
  unsigned *work;            // work-stealing counter
  unsigned long long *err;   // (rank << 8) | code, atomicMin
  // halo records by slot
  unsigned long long *nhalo;
  unsigned long long *pool_used;
  unsigned *h_rank;
  long long *h_id, *h_mass, *h_mass2, *h_mextra, *h_profile;
  float *h_center;
  double *h_rdelta;
  unsigned long long *h_pool;  // pool offset
  unsigned long long *pool_key;  // d2 bits
  unsigned *pool_idx;            // input index
  unsigned long long *touched;
  unsigned long long *nprocessed;
};

struct Level {
  unsigned long long lo, hi;  // bit range of the level
  unsigned long long cum;     // elements below lo
  int shift;                  // bucket = (bits - lo) >> shift (levels >= 1)
  int next;                   // next bucket to examine
};

struct Smem {
  unsigned hist[MAXLEV][NB];
  unsigned long long skey[CAP];
  unsigned sidx[CAP];
  unsigned pref[NB];
  Level lev[MAXLEV];
  double edges[PSOD_MAX_BINS];
  unsigned phist[PSOD_MAX_BINS + 1];
  unsigned long long red_u64[NWARP];
  unsigned long long red_u64b[NWARP];
  unsigned red_u32[NWARP];
  int red_i[NWARP];
  long long red_i64[NWARP];
  // per-seed scalars
  unsigned na;
  unsigned cube_records;
  unsigned long long best_sq;
  unsigned long long best_key;
  unsigned best_pos;
  unsigned nsorted;
  unsigned long long pool_base;
  unsigned claim_cnt;
  // last radial_search hit: sorted-buffer index and bucket lower bound
  int res_k;
  unsigned long long res_lo;
};

__device__ __forceinline__ int wrapi(int a, int nx) {
  if (a >= nx) a -= nx;
  if (a < 0) a += nx;
  return a;
}

// Visit every particle record filed under the cells of the cube of
// half-width R around (ic,jc,kc): warp per row of cells, lanes stride along
// the row's contiguous run of records.
template <typename F>
__device__ __forceinline__ void for_cube(const SodConst &K, const SodBufs &B, int ic, int jc, int kc, int R, F f) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int side = 2 * R + 1;
  const int nrow = side * side;
  const unsigned nx = (unsigned)K.nx;
  for (int row = w; row < nrow; row += NWARP) {
    const int dj = row % side - R, dk = row / side - R;
    const unsigned jj = (unsigned)wrapi(jc + dj, K.nx), kk = (unsigned)wrapi(kc + dk, K.nx);
    const unsigned long long base = (unsigned long long)nx * (jj + (unsigned long long)nx * kk);
    int x0 = ic - R, x1 = ic + R;
    int pa[2], pb[2], np = 0;
    if (x0 < 0) {
      pa[0] = x0 + K.nx; pb[0] = K.nx - 1; pa[1] = 0; pb[1] = x1; np = 2;
    } else if (x1 >= K.nx) {
      pa[0] = x0; pb[0] = K.nx - 1; pa[1] = 0; pb[1] = x1 - K.nx; np = 2;
    } else {
      pa[0] = x0; pb[0] = x1; np = 1;
    }
    for (int q = 0; q < np; q++) {
      const unsigned b = B.cs[base + (unsigned)pa[q]];
      const unsigned e = B.cs[base + (unsigned)pb[q] + 1];
      for (unsigned p = b + lane; p < e; p += 32) f(p, B.cube[p]);
    }
  }
}

__device__ __forceinline__ unsigned block_sum_u32(Smem &S, unsigned v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) S.red_u32[threadIdx.x >> 5] = v;
  __syncthreads();
  unsigned s = 0;
#pragma unroll
  for (int q = 0; q < NWARP; q++) s += S.red_u32[q];
  return s;
}

__device__ __forceinline__ int block_min_i(Smem &S, int v) {
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_down_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) S.red_i[threadIdx.x >> 5] = v;
  __syncthreads();
  int s = S.red_i[0];
#pragma unroll
  for (int q = 1; q < NWARP; q++) s = min(s, S.red_i[q]);
  return s;
}

__device__ __forceinline__ int block_max_i(Smem &S, int v) {
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_down_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) S.red_i[threadIdx.x >> 5] = v;
  __syncthreads();
  int s = S.red_i[0];
#pragma unroll
  for (int q = 1; q < NWARP; q++) s = max(s, S.red_i[q]);
  return s;
}

// lexicographic (a, b) maximum over the block
__device__ __forceinline__ void block_max_pair(Smem &S, unsigned long long &a, unsigned long long &b) {
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long ta = __shfl_down_sync(0xffffffffu, a, o);
    unsigned long long tb = __shfl_down_sync(0xffffffffu, b, o);
    if (ta > a || (ta == a && tb > b)) { a = ta; b = tb; }
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    S.red_u64[threadIdx.x >> 5] = a;
    S.red_u64b[threadIdx.x >> 5] = b;
  }
  __syncthreads();
  a = S.red_u64[0];
  b = S.red_u64b[0];
#pragma unroll
  for (int q = 1; q < NWARP; q++) {
    unsigned long long ta = S.red_u64[q], tb = S.red_u64b[q];
    if (ta > a || (ta == a && tb > b)) { a = ta; b = tb; }
  }
}

// block exclusive scan over S.hist[l] into S.pref (NB = 16 per thread)
__device__ void hist_prefix(Smem &S, int l) {
  const int t = threadIdx.x;
  unsigned v[NB / TPB];
  unsigned s = 0;
#pragma unroll
  for (int k = 0; k < NB / TPB; k++) {
    v[k] = S.hist[l][t * (NB / TPB) + k];
    s += v[k];
  }
  // warp inclusive scan
  const int lane = t & 31, w = t >> 5;
  unsigned inc = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned x = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += x;
  }
  __syncthreads();
  if (lane == 31) S.red_u32[w] = inc;
  __syncthreads();
  unsigned woff = 0;
  for (int q = 0; q < w; q++) woff += S.red_u32[q];
  unsigned off = woff + inc - s;
#pragma unroll
  for (int k = 0; k < NB / TPB; k++) {
    S.pref[t * (NB / TPB) + k] = off;
    off += v[k];
  }
  __syncthreads();
}

// bucket of bit pattern x at level l (x must lie in the level's range)
__device__ __forceinline__ int bucket_of(const Level &L, int l, unsigned long long x) {
  if (l == 0) {
    long long b = (long long)(x >> L1_SHIFT) - (long long)L1_BASE;
    return (int)(b < 0 ? 0 : (b > NB - 1 ? NB - 1 : b));
  }
  return (int)((x - L.lo) >> L.shift);
}

__device__ __forceinline__ void bucket_range(const Level &L, int l, int b, unsigned long long &lo,
                                             unsigned long long &hi) {
  if (l == 0) {
    lo = (b == 0) ? 0ull : ((unsigned long long)b + L1_BASE) << L1_SHIFT;
    hi = (b == NB - 1) ? 0x7fefffffffffffffull : ((((unsigned long long)b + 1 + L1_BASE) << L1_SHIFT) - 1);
    return;
  }
  lo = L.lo + ((unsigned long long)b << L.shift);
  unsigned long long h = lo + ((1ull << L.shift) - 1);
  hi = h < L.hi ? h : L.hi;
}

// overdensity of the reference's loop at 1-based position i and squared
// distance d2 (main:2048-2051): amass = i*munit is exact
__device__ __forceinline__ double overdens(const SodConst &K, long long i, double d2) {
  double r = dsqrt(d2);
  double vol = dmul(K.cvol, dmul(dmul(r, r), r));
  return ddiv(dmul((double)i, K.munit), vol);
}

// reference loop condition at position i >= 2 (main:2046)
__device__ __forceinline__ bool keeps_going(const SodConst &K, long long i, double d2, long long na, double delta) {
  if (i < 10) return true;
  double r = dsqrt(d2);
  double vol = dmul(K.cvol, dmul(dmul(r, r), r));
  double ovd = ddiv(dmul((double)i, K.munit), vol);
  return ovd > delta && i < na && r < (double)K.ncut;
}

// fill S.hist[l] with the bucket counts of alive records whose d2 bits lie
// in [lo, hi]
__device__ void build_hist(const SodConst &K, const SodBufs &B, Smem &S, int l, int ic, int jc, int kc, double xc,
                           double yc, double zc) {
  for (int k = threadIdx.x; k < NB; k += TPB) S.hist[l][k] = 0;
  __syncthreads();
  const Level L = S.lev[l];
  for_cube(K, B, ic, jc, kc, K.ncut, [&](unsigned p, float4 v) {
    if (__float_as_uint(v.w) & PSOD_DEAD_BIT) return;
    double d2 = min_image_d2((double)to_grid(v.x, K.nxf), (double)to_grid(v.y, K.nxf), (double)to_grid(v.z, K.nxf),
                             xc, yc, zc, K.tx);
    unsigned long long x = dbits(d2);
    if (l > 0 && (x < L.lo || x > L.hi)) return;
    atomicAdd(&S.hist[l][bucket_of(L, l, x)], 1u);
  });
  __syncthreads();
}

// load alive records with d2 bits in [lo, hi] into S.skey/S.sidx, sort them
// by (bits, input index); returns the count
__device__ unsigned extract_sorted(const SodConst &K, const SodBufs &B, Smem &S, int ic, int jc, int kc, double xc,
                                   double yc, double zc, unsigned long long lo, unsigned long long hi) {
  if (threadIdx.x == 0) S.nsorted = 0;
  __syncthreads();
  for_cube(K, B, ic, jc, kc, K.ncut, [&](unsigned p, float4 v) {
    unsigned wv = __float_as_uint(v.w);
    if (wv & PSOD_DEAD_BIT) return;
    double d2 = min_image_d2((double)to_grid(v.x, K.nxf), (double)to_grid(v.y, K.nxf), (double)to_grid(v.z, K.nxf),
                             xc, yc, zc, K.tx);
    unsigned long long x = dbits(d2);
    if (x < lo || x > hi) return;
    unsigned s = atomicAdd(&S.nsorted, 1u);
    if (s < CAP) {
      S.skey[s] = x;
      S.sidx[s] = wv & PSOD_IDX_MASK;
    }
  });
  __syncthreads();
  const unsigned n = min(S.nsorted, (unsigned)CAP);
  unsigned m = 1;
  while (m < n) m <<= 1;
  for (unsigned k = n + threadIdx.x; k < m; k += TPB) {
    S.skey[k] = ~0ull;
    S.sidx[k] = 0xffffffffu;
  }
  __syncthreads();
  // bitonic sort of m (power of two) pairs
  for (unsigned size = 2; size <= m; size <<= 1) {
    for (unsigned stride = size >> 1; stride > 0; stride >>= 1) {
      for (unsigned k = threadIdx.x; k < m / 2; k += TPB) {
        unsigned a = 2 * k - (k & (stride - 1));
        unsigned bb = a + stride;
        bool up = ((a & size) == 0);
        unsigned long long ka = S.skey[a], kb = S.skey[bb];
        unsigned ia = S.sidx[a], ib = S.sidx[bb];
        bool gt = (ka > kb) || (ka == kb && ia > ib);
        if (gt == up) {
          S.skey[a] = kb; S.skey[bb] = ka;
          S.sidx[a] = ib; S.sidx[bb] = ia;
        }
      }
      __syncthreads();
    }
  }
  return n;
}

// Search over the sorted d2 sequence of the cube.
//  mode 0 (forward): first 1-based position i >= 10 where the reference's
//                    loop stops for threshold delta.
//  mode 1 (backward): last position i in [2, imax] with overdensity > delta.
// Returns 0 if not found, else the position; *d2_out its squared distance.
// Returns -1 on an unresolvable bucket (more than CAP exact-equal keys).
__device__ long long radial_search(const SodConst &K, const SodBufs &B, Smem &S, int ic, int jc, int kc, double xc,
                                   double yc, double zc, long long na, double delta, int mode, long long imax,
                                   double *d2_out) {
  // level 0 histogram is built by the caller
  int l = 0;
  if (threadIdx.x == 0) {
    S.lev[0].cum = 0;
    S.lev[0].next = (mode == 0) ? 0 : NB - 1;
  }
  __syncthreads();
  while (true) {
    hist_prefix(S, l);
    const Level L = S.lev[l];
    // find the first (forward) / last (backward) bucket that may hold a hit
    int cand = (mode == 0) ? 0x7fffffff : -1;
    for (int k = 0; k < NB / TPB; k++) {
      int b = threadIdx.x * (NB / TPB) + k;
      if (mode == 0 ? (b < L.next) : (b > L.next)) continue;
      unsigned nb = S.hist[l][b];
      if (nb == 0) continue;
      unsigned long long lo, hi;
      bucket_range(L, l, b, lo, hi);
      long long c0 = (long long)L.cum + S.pref[b];
      long long ilo = c0 + 1, ihi = c0 + nb;
      bool maybe;
      if (mode == 0) {
        if (ihi < 10) {
          maybe = false;
        } else {
          long long i0 = ilo < 10 ? 10 : ilo;
          double hd = bitsd(hi);
          bool sure_go = overdens(K, i0, hd) > delta && ihi < na && dsqrt(hd) < (double)K.ncut;
          maybe = !sure_go;
        }
      } else {
        long long i1 = ihi < imax ? ihi : imax;
        long long i0 = ilo < 2 ? 2 : ilo;
        if (i1 < i0) {
          maybe = false;
        } else {
          double ld = bitsd(lo);
          maybe = overdens(K, i1, ld) > delta;  // upper bound of the bucket
        }
      }
      if (maybe) {
        if (mode == 0) cand = min(cand, b);
        else cand = max(cand, b);
      }
    }
    cand = (mode == 0) ? block_min_i(S, cand) : block_max_i(S, cand);
    if (mode == 0 ? (cand == 0x7fffffff) : (cand < 0)) {
      if (l == 0) return 0;
      l--;
      continue;
    }
    if (threadIdx.x == 0) S.lev[l].next = (mode == 0) ? cand + 1 : cand - 1;
    __syncthreads();
    unsigned nb = S.hist[l][cand];
    unsigned long long lo, hi;
    bucket_range(L, l, cand, lo, hi);
    const long long c0 = (long long)L.cum + S.pref[cand];
    if (nb <= CAP) {
      unsigned n = extract_sorted(K, B, S, ic, jc, kc, xc, yc, zc, lo, hi);
      long long hit;
      if (mode == 0) {
        int best = 0x7fffffff;
        for (unsigned k = threadIdx.x; k < n; k += TPB) {
          long long i = c0 + 1 + k;
          if (!keeps_going(K, i, bitsd(S.skey[k]), na, delta)) best = min(best, (int)k);
        }
        best = block_min_i(S, best);
        hit = (best == 0x7fffffff) ? -1 : best;
      } else {
        int best = -1;
        for (unsigned k = threadIdx.x; k < n; k += TPB) {
          long long i = c0 + 1 + k;
          if (i >= 2 && i <= imax && overdens(K, i, bitsd(S.skey[k])) > delta) best = max(best, (int)k);
        }
        best = block_max_i(S, best);
        hit = best;
      }
      if (hit >= 0) {
        *d2_out = bitsd(S.skey[hit]);
        if (threadIdx.x == 0) {
          S.res_k = (int)hit;
          S.res_lo = lo;
        }
        __syncthreads();
        return c0 + 1 + hit;
      }
      continue;  // no hit in this bucket: next candidate at this level
    }
    // descend
    if (l + 1 >= MAXLEV || hi == lo) return -1;
    if (threadIdx.x == 0) {
      Level &C = S.lev[l + 1];
      C.lo = lo;
      C.hi = hi;
      C.cum = (unsigned long long)c0;
      unsigned long long span = hi - lo;
      int bl = 64 - __clzll((long long)span);
      C.shift = bl > 12 ? bl - 12 : 0;
      C.next = (mode == 0) ? 0 : NB - 1;
    }
    __syncthreads();
    l++;
    build_hist(K, B, S, l, ic, jc, kc, xc, yc, zc);
  }
}

// the pos-th (1-based) element of the sorted sequence when it is the last
// element below `below_lo`: the maximum (bits, index) under that bound
__device__ void max_below(const SodConst &K, const SodBufs &B, Smem &S, int ic, int jc, int kc, double xc, double yc,
                          double zc, unsigned long long below_lo, unsigned long long &kout, unsigned &iout) {
  unsigned long long a = 0, b = 0;
  for_cube(K, B, ic, jc, kc, K.ncut, [&](unsigned p, float4 v) {
    unsigned wv = __float_as_uint(v.w);
    if (wv & PSOD_DEAD_BIT) return;
    double d2 = min_image_d2((double)to_grid(v.x, K.nxf), (double)to_grid(v.y, K.nxf), (double)to_grid(v.z, K.nxf),
                             xc, yc, zc, K.tx);
    unsigned long long x = dbits(d2);
    if (x >= below_lo) return;
    unsigned long long ix = wv & PSOD_IDX_MASK;
    if (x > a || (x == a && ix > b)) { a = x; b = ix; }
  });
  block_max_pair(S, a, b);
  kout = a;
  iout = (unsigned)b;
}

__device__ void record_error(const SodBufs &B, unsigned rank, unsigned code) {
  atomicMin(B.err, ((unsigned long long)rank << 8) | code);
}

__device__ void process_seed(const SodConst &K, const SodBufs &B, Smem &S, unsigned rank) {
  const unsigned sidx = B.seed_idx[rank];
  const unsigned sp = B.inv[sidx];
  const float4 sv = B.cube[sp];
  if (__float_as_uint(sv.w) & PSOD_DEAD_BIT) return;  // claimed (main:1628)
  // seed position and cell (main:1631-1654)
  const double xs0 = (double)to_grid(sv.x, K.nxf), ys0 = (double)to_grid(sv.y, K.nxf),
               zs0 = (double)to_grid(sv.z, K.nxf);
  const int ic = sod_cell_axis(to_grid(sv.x, K.nxf), K.xs, K.nx);
  const int jc = sod_cell_axis(to_grid(sv.y, K.nxf), K.xs, K.nx);
  const int kc = sod_cell_axis(to_grid(sv.z, K.nxf), K.xs, K.nx);

  // 1. preselect count (main:1657-1716)
  unsigned cnt = 0, recs = 0;
  for_cube(K, B, ic, jc, kc, K.ncut, [&](unsigned p, float4 v) {
    recs++;
    if (!(__float_as_uint(v.w) & PSOD_DEAD_BIT)) cnt++;
  });
  const unsigned na = block_sum_u32(S, cnt);
  const unsigned nrec = block_sum_u32(S, recs);
  if (threadIdx.x == 0) atomicAdd(B.touched, (unsigned long long)nrec);
  if ((long long)na > K.nsel) {
    if (threadIdx.x == 0) record_error(B, rank, PSOD_ERR_NSEL);
    return;
  }
  if (!(dmul((double)na, K.munit) >= K.mmin)) return;  // main:1759
  if (threadIdx.x == 0) atomicAdd(B.nprocessed, 1ull);

  // 2. centre refinement (main:1799-1909).  Warp per candidate; lanes stride
  // over the candidate's 27 neighbour cells, keeping those filed within +-2
  // cells of the seed (the x_sel2 set, main:1720-1755).
  {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned long long my_sq = 0, my_key = ~0ull;
    unsigned my_pos = 0xffffffffu;
    bool have = false;
    // enumerate candidate rows: 9 rows of 3 cells around the seed cell
    for (int row = 0; row < 9; row++) {
      const int dj = row % 3 - 1, dk = row / 3 - 1;
      const unsigned jj = (unsigned)wrapi(jc + dj, K.nx), kk = (unsigned)wrapi(kc + dk, K.nx);
      const unsigned long long rbase = (unsigned long long)K.nx * (jj + (unsigned long long)K.nx * kk);
      for (int di = -1; di <= 1; di++) {
        const unsigned ii = (unsigned)wrapi(ic + di, K.nx);
        const unsigned cb = B.cs[rbase + ii], ce = B.cs[rbase + ii + 1];
        // warps take candidates of this cell round-robin
        for (unsigned cp = cb + w; cp < ce; cp += NWARP) {
          const float4 cv = B.cube[cp];
          const unsigned cw = __float_as_uint(cv.w);
          if (cw & PSOD_DEAD_BIT) continue;
          const float cxg = to_grid(cv.x, K.nxf), cyg = to_grid(cv.y, K.nxf), czg = to_grid(cv.z, K.nxf);
          const double cx = cxg, cy = cyg, cz = czg;
          const int pcx = sod_cell_axis(cxg, K.xs, K.nx), pcy = sod_cell_axis(cyg, K.xs, K.nx),
                    pcz = sod_cell_axis(czg, K.xs, K.nx);
          unsigned long long sq = 0;
          for (int nrow = 0; nrow < 9; nrow++) {
            const int ny = wrapi(pcy + nrow % 3 - 1, K.nx), nz = wrapi(pcz + nrow / 3 - 1, K.nx);
            if (abs(pdiff(ny, jc, K.nx)) > 2 || abs(pdiff(nz, kc, K.nx)) > 2) continue;
            const unsigned long long nbase = (unsigned long long)K.nx * ((unsigned)ny + (unsigned long long)K.nx * (unsigned)nz);
            for (int ndi = -1; ndi <= 1; ndi++) {
              const int nxc = wrapi(pcx + ndi, K.nx);
              if (abs(pdiff(nxc, ic, K.nx)) > 2) continue;
              const unsigned nb = B.cs[nbase + (unsigned)nxc], ne = B.cs[nbase + (unsigned)nxc + 1];
              for (unsigned q = nb + lane; q < ne; q += 32) {
                const float4 nv = B.cube[q];
                if (__float_as_uint(nv.w) & PSOD_DEAD_BIT) continue;
                double d2 = min_image_d2((double)to_grid(nv.x, K.nxf), (double)to_grid(nv.y, K.nxf),
                                         (double)to_grid(nv.z, K.nxf), cx, cy, cz, K.tx);
                if (d2 <= K.rmin2) {
                  double t = ddiv(1.0, dsqrt(dadd(d2, K.eps2)));  // main:1854-1855
                  sq += (unsigned long long)__double2ll_rn(dmul(t, 1099511627776.0));
                }
              }
            }
          }
          // the particle the run scan files under another cell
          if (K.has_quirk && lane == 0) {
            const int ax = (int)(K.quirk_listed % K.nx), ay = (int)((K.quirk_listed / K.nx) % K.nx),
                      az = (int)(K.quirk_listed / ((unsigned)K.nx * K.nx));
            const bool listed_in_sel2 = abs(pdiff(ax, ic, K.nx)) <= 2 && abs(pdiff(ay, jc, K.nx)) <= 2 &&
                                        abs(pdiff(az, kc, K.nx)) <= 2;
            const bool seen = abs(pdiff(ax, pcx, K.nx)) <= 1 && abs(pdiff(ay, pcy, K.nx)) <= 1 &&
                              abs(pdiff(az, pcz, K.nx)) <= 1;
            if (listed_in_sel2 && !seen) {
              const float4 qv = B.cube[K.quirk_pos];
              if (!(__float_as_uint(qv.w) & PSOD_DEAD_BIT)) {
                double d2 = min_image_d2((double)to_grid(qv.x, K.nxf), (double)to_grid(qv.y, K.nxf),
                                         (double)to_grid(qv.z, K.nxf), cx, cy, cz, K.tx);
                if (d2 <= K.rmin2) {
                  double t = ddiv(1.0, dsqrt(dadd(d2, K.eps2)));
                  sq += (unsigned long long)__double2ll_rn(dmul(t, 1099511627776.0));
                }
              }
            }
          }
          for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
          if (lane == 0) {
            // scan-order key: listed cell offset (x outer, z inner), then index
            int lx = di, ly = dj, lz = dk;
            if (K.has_quirk && cp == K.quirk_pos) {
              lx = pdiff((int)(K.quirk_listed % K.nx), ic, K.nx);
              ly = pdiff((int)((K.quirk_listed / K.nx) % K.nx), jc, K.nx);
              lz = pdiff((int)(K.quirk_listed / ((unsigned)K.nx * K.nx)), kc, K.nx);
            }
            const unsigned o = (unsigned)(((lx + 1) * 3 + (ly + 1)) * 3 + (lz + 1));
            const unsigned long long key = ((unsigned long long)o << 32) | (cw & PSOD_IDX_MASK);
            if (!have || sq > my_sq || (sq == my_sq && key < my_key)) {
              have = true;
              my_sq = sq;
              my_key = key;
              my_pos = cp;
            }
          }
        }
      }
    }
    // block argmax: larger sum wins; equal sums go to the smaller key.
    // Encode as (sq, ~key) and take the lexicographic maximum.
    unsigned long long a = have ? my_sq : 0ull, b = have ? ~my_key : 0ull;
    unsigned long long pa = a, pb = b;
    if (threadIdx.x == 0) S.best_pos = sp;  // no candidate: the seed stays the centre
    block_max_pair(S, a, b);
    if (have && a > 0 && pa == a && pb == b) S.best_pos = my_pos;
    __syncthreads();
  }
  const unsigned cpos = S.best_pos;
  const float4 cvv = B.cube[cpos];
  const double xc = (double)to_grid(cvv.x, K.nxf), yc = (double)to_grid(cvv.y, K.nxf),
               zc = (double)to_grid(cvv.z, K.nxf);
  const unsigned cidx = __float_as_uint(cvv.w) & PSOD_IDX_MASK;
  (void)xs0; (void)ys0; (void)zs0;

  // 3. crossing (main:2040-2100)
  if (threadIdx.x == 0) {
    S.lev[0].lo = 0;
    S.lev[0].hi = 0x7fefffffffffffffull;
    S.lev[0].shift = L1_SHIFT;
  }
  __syncthreads();
  build_hist(K, B, S, 0, ic, jc, kc, xc, yc, zc);
  double d2stop = 0;
  long long istop = radial_search(K, B, S, ic, jc, kc, xc, yc, zc, (long long)na, K.delta, 0, 0, &d2stop);
  if (istop <= 0) {
    if (threadIdx.x == 0) record_error(B, rank, PSOD_ERR_STATE);
    return;
  }
  if (overdens(K, istop, d2stop) > K.delta) {  // main:2072
    if (threadIdx.x == 0) record_error(B, rank, PSOD_ERR_SELRADIUS);
    return;
  }
  const long long masse = istop - 1;
  // the masse-th element closes the member set (main:2090-2100, 2148)
  unsigned long long thr_key;
  unsigned thr_idx;
  {
    const int hk = S.res_k;
    const unsigned long long blo = S.res_lo;
    __syncthreads();
    if (hk > 0) {
      thr_key = S.skey[hk - 1];
      thr_idx = S.sidx[hk - 1];
    } else {
      max_below(K, B, S, ic, jc, kc, xc, yc, zc, blo, thr_key, thr_idx);
    }
  }
  const double rayon = dsqrt(bitsd(thr_key));

  // seuil2 capture (main:2062-2069): last step i in [2, istop] above seuil2
  long long masse2 = 0;
  {
    double dd;
    long long i2 = radial_search(K, B, S, ic, jc, kc, xc, yc, zc, (long long)na, K.delta2, 1, istop, &dd);
    if (i2 > 0) masse2 = i2;
  }
  // extra thresholds: the same stop rule, -1 when not crossed
  long long mext[PSOD_MAX_EXTRA_DELTA];
  for (int e = 0; e < K.ndx; e++) {
    double dd;
    long long ie = radial_search(K, B, S, ic, jc, kc, xc, yc, zc, (long long)na, K.dx_extra[e], 0, 0, &dd);
    mext[e] = (ie <= 0 || overdens(K, ie, dd) > K.dx_extra[e]) ? -1 : ie - 1;
  }

  // keep test (main:2118-2120)
  const double amass = dmul((double)masse, K.munit);
  const bool keep = amass >= K.mmin && xc <= K.zmax && xc > K.zmin && yc <= K.zmax && yc > K.zmin &&
                    zc <= K.zmax && zc > K.zmin;

  // 4a. profile (main:2103-2115): cumulative counts below each edge
  if (keep) {
    for (int j = threadIdx.x; j < K.nbins; j += TPB) S.edges[j] = dmul(rayon, B.edge_fac[j]);
    for (int j = threadIdx.x; j <= K.nbins; j += TPB) S.phist[j] = 0;
    __syncthreads();
    const double emax = S.edges[K.nbins - 1];
    for_cube(K, B, ic, jc, kc, K.ncut, [&](unsigned p, float4 v) {
      if (__float_as_uint(v.w) & PSOD_DEAD_BIT) return;
      double d2 = min_image_d2((double)to_grid(v.x, K.nxf), (double)to_grid(v.y, K.nxf),
                               (double)to_grid(v.z, K.nxf), xc, yc, zc, K.tx);
      double r = dsqrt(d2);
      if (!(r < emax)) return;
      int lo = 0, hi = K.nbins - 1;  // first edge with r < edge
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (r < S.edges[mid]) hi = mid;
        else lo = mid + 1;
      }
      atomicAdd(&S.phist[lo], 1u);
    });
    __syncthreads();
    if (threadIdx.x == 0) {
      S.pool_base = atomicAdd(B.pool_used, (unsigned long long)masse);
      S.claim_cnt = 0;
    }
    __syncthreads();
  } else {
    if (threadIdx.x == 0) S.claim_cnt = 0;
    __syncthreads();
  }

  // 4b. claims (main:2148-2166): the masse nearest die, kept or not
  const unsigned long long pool_base = S.pool_base;
  for_cube(K, B, ic, jc, kc, K.ncut, [&](unsigned p, float4 v) {
    const unsigned wv = __float_as_uint(v.w);
    if (wv & PSOD_DEAD_BIT) return;
    double d2 = min_image_d2((double)to_grid(v.x, K.nxf), (double)to_grid(v.y, K.nxf), (double)to_grid(v.z, K.nxf),
                             xc, yc, zc, K.tx);
    const unsigned long long x = dbits(d2);
    const unsigned ix = wv & PSOD_IDX_MASK;
    if (x < thr_key || (x == thr_key && ix <= thr_idx)) {
      B.cube[p].w = __uint_as_float(wv | PSOD_DEAD_BIT);
      const unsigned slot = atomicAdd(&S.claim_cnt, 1u);
      if (keep && slot < (unsigned)masse) {
        B.pool_key[pool_base + slot] = x;
        B.pool_idx[pool_base + slot] = ix;
      }
    }
  });
  __syncthreads();
  if (S.claim_cnt != (unsigned)masse) {
    if (threadIdx.x == 0) record_error(B, rank, PSOD_ERR_STATE);
    return;
  }
  if (!keep) return;

  // 5. halo record
  __shared__ unsigned long long s_slot;
  if (threadIdx.x == 0) {
    const unsigned long long slot = atomicAdd(B.nhalo, 1ull);
    s_slot = slot;
    B.h_rank[slot] = rank;
    B.h_id[slot] = B.ids[cidx];
    B.h_mass[slot] = masse;
    B.h_mass2[slot] = masse2;
    B.h_rdelta[slot] = rayon;
    B.h_center[3 * slot + 0] = __double2float_rn(ddiv(xc, K.scale));
    B.h_center[3 * slot + 1] = __double2float_rn(ddiv(yc, K.scale));
    B.h_center[3 * slot + 2] = __double2float_rn(ddiv(zc, K.scale));
    B.h_pool[slot] = pool_base;
    for (int e = 0; e < K.ndx; e++) B.h_mextra[slot * K.ndx + e] = mext[e];
  }
  __syncthreads();
  {
    const unsigned long long slot = s_slot;
    unsigned run = 0;
    // cumulative profile (serial over <= 128 bins)
    if (threadIdx.x == 0) {
      for (int j = 0; j < K.nbins; j++) {
        run += S.phist[j];
        B.h_profile[slot * K.nbins + j] = run;
      }
    }
  }
}

__global__ void __launch_bounds__(TPB) k_sod_seeds(SodConst K, SodBufs B) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem &S = *reinterpret_cast<Smem *>(smem_raw);
  __shared__ unsigned s_item;
  while (true) {
    if (threadIdx.x == 0) s_item = atomicAdd(B.work, 1u);
    __syncthreads();
    const unsigned item = s_item;
    __syncthreads();
    if (item >= *B.nready) break;
    const unsigned rank = B.ready[item];
    process_seed(K, B, S, rank);
    __syncthreads();
    if (threadIdx.x == 0) B.processed[rank] = 1;
  }
}


// ---------------------------------------------------------------------------
// scheduler
// ---------------------------------------------------------------------------
__global__ void k_seed_blocks(const unsigned *seed_idx, const unsigned *inv, const float4 *cube, long long nseed,
                              SodConst K, int bs, int nb, unsigned *block_of, unsigned *rank) {
  long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nseed) return;
  const float4 v = cube[inv[seed_idx[r]]];
  const int ci = sod_cell_axis(to_grid(v.x, K.nxf), K.xs, K.nx) / bs;
  const int cj = sod_cell_axis(to_grid(v.y, K.nxf), K.xs, K.nx) / bs;
  const int ck = sod_cell_axis(to_grid(v.z, K.nxf), K.xs, K.nx) / bs;
  block_of[r] = (unsigned)ci + (unsigned)nb * ((unsigned)cj + (unsigned)nb * (unsigned)ck);
  rank[r] = (unsigned)r;
}

__global__ void k_count_u32(const unsigned *keys, long long n, unsigned *count) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(&count[keys[i]], 1u);
}

// advance each block's cursor past resolved seeds; head = lowest unresolved rank
__global__ void k_heads(long long nblocks, const unsigned *bbegin, unsigned *cursor, const unsigned *blist,
                        const unsigned char *processed, const unsigned *seed_idx, const unsigned *inv,
                        const float4 *cube, unsigned *head, unsigned *gmin) {
  long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblocks) return;
  unsigned cur = cursor[b];
  const unsigned end = bbegin[b + 1];
  unsigned h = PSOD_INF_RANK;
  while (cur < end) {
    const unsigned r = blist[cur];
    if (processed[r] || (__float_as_uint(cube[inv[seed_idx[r]]].w) & PSOD_DEAD_BIT)) {
      cur++;
      continue;
    }
    h = r;
    break;
  }
  cursor[b] = cur;
  head[b] = h;
  if (h != PSOD_INF_RANK) atomicMin(gmin, h);
}

// periodic sliding minimum of radius rb along one axis of the nb^3 grid
__global__ void k_minfilter(const unsigned *in, unsigned *out, int nb, int axis, int rb) {
  long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nbl = (long long)nb * nb * nb;
  if (b >= nbl) return;
  int c[3] = {(int)(b % nb), (int)((b / nb) % nb), (int)(b / ((long long)nb * nb))};
  const int full = (2 * rb + 1 >= nb);
  const int lo = full ? 0 : -rb, hi = full ? nb - 1 : rb;
  unsigned m = PSOD_INF_RANK;
  const int c0 = c[axis];
  for (int d = lo; d <= hi; d++) {
    int v = full ? d : c0 + d;
    if (v < 0) v += nb;
    if (v >= nb) v -= nb;
    c[axis] = v;
    unsigned x = in[(long long)c[0] + (long long)nb * ((long long)c[1] + (long long)nb * c[2])];
    m = x < m ? x : m;
  }
  out[b] = m;
}

__global__ void k_ready(long long nblocks, const unsigned *head, const unsigned *filt, unsigned quirk_rank,
                        const unsigned *gmin, unsigned *ready, unsigned *nready) {
  long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblocks) return;
  const unsigned h = head[b];
  if (h == PSOD_INF_RANK || h != filt[b]) return;
  // the particle filed under another cell waits until it is the global minimum
  if (h == quirk_rank && h != *gmin) return;
  ready[atomicAdd(nready, 1u)] = h;
}

__global__ void k_find_rank(const unsigned *seed_idx, long long nseed, unsigned idx, unsigned *out) {
  long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < nseed && seed_idx[r] == idx) *out = (unsigned)r;
}

// ---------------------------------------------------------------------------
// output assembly
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_gather(const T *src, const unsigned *order, long long n, int width, T *dst) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * width) return;
  long long h = i / width, k = i % width;
  dst[i] = src[(long long)order[h] * width + k];
}

__global__ void k_mass_u32(const long long *mass, long long n, unsigned *out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (unsigned)mass[i];
}

__global__ void k_widen(const unsigned *in, long long n, long long *out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (long long)in[i];
}

constexpr int MS_CHUNK = 4096;

__device__ __forceinline__ bool pair_less(unsigned long long ka, unsigned ia, unsigned long long kb, unsigned ib) {
  return ka < kb || (ka == kb && ia < ib);
}

// sort each halo's members by (d2 bits, input index) and write the input
// indices at the halo's output offset; one CTA per halo
__global__ void __launch_bounds__(256) k_member_sort(const unsigned *order, long long nh, const unsigned long long *h_pool,
                                                     const long long *h_mass_sorted, const unsigned *moff,
                                                     unsigned long long *pkey, unsigned *pidx,
                                                     unsigned long long *tkey, unsigned *tidx, unsigned *m_index) {
  __shared__ unsigned long long sk[MS_CHUNK];
  __shared__ unsigned si[MS_CHUNK];
  for (long long h = blockIdx.x; h < nh; h += gridDim.x) {
    const unsigned slot = order[h];
    const unsigned long long base = h_pool[slot];
    const unsigned m = (unsigned)h_mass_sorted[h];
    unsigned long long *ka = pkey + base, *kb = tkey + base;
    unsigned *ia = pidx + base, *ib = tidx + base;
    // 1. sort chunks in shared memory
    for (unsigned c0 = 0; c0 < m; c0 += MS_CHUNK) {
      const unsigned n = min((unsigned)MS_CHUNK, m - c0);
      unsigned p2 = 1;
      while (p2 < n) p2 <<= 1;
      for (unsigned k = threadIdx.x; k < p2; k += blockDim.x) {
        sk[k] = k < n ? ka[c0 + k] : ~0ull;
        si[k] = k < n ? ia[c0 + k] : 0xffffffffu;
      }
      __syncthreads();
      for (unsigned size = 2; size <= p2; size <<= 1) {
        for (unsigned stride = size >> 1; stride > 0; stride >>= 1) {
          for (unsigned k = threadIdx.x; k < p2 / 2; k += blockDim.x) {
            unsigned a = 2 * k - (k & (stride - 1));
            unsigned bb = a + stride;
            bool up = ((a & size) == 0);
            bool gt = pair_less(sk[bb], si[bb], sk[a], si[a]);
            if (gt == up) {
              unsigned long long t = sk[a]; sk[a] = sk[bb]; sk[bb] = t;
              unsigned ti = si[a]; si[a] = si[bb]; si[bb] = ti;
            }
          }
          __syncthreads();
        }
      }
      for (unsigned k = threadIdx.x; k < n; k += blockDim.x) {
        ka[c0 + k] = sk[k];
        ia[c0 + k] = si[k];
      }
      __syncthreads();
    }
    // 2. merge runs pairwise through global memory
    for (unsigned w = MS_CHUNK; w < m; w <<= 1) {
      for (unsigned k = threadIdx.x; k < m; k += blockDim.x) {
        const unsigned run = k / (2 * w);
        const unsigned s0 = run * 2 * w;
        const unsigned amid = min(s0 + w, m), aend = min(s0 + 2 * w, m);
        const unsigned long long key = ka[k];
        const unsigned ix = ia[k];
        unsigned pos;
        if (k < amid) {
          // count of the other run strictly below
          unsigned lo = amid, hi = aend;
          while (lo < hi) {
            unsigned mid = (lo + hi) >> 1;
            if (pair_less(ka[mid], ia[mid], key, ix)) lo = mid + 1;
            else hi = mid;
          }
          pos = s0 + (k - s0) + (lo - amid);
        } else {
          unsigned lo = s0, hi = amid;
          while (lo < hi) {
            unsigned mid = (lo + hi) >> 1;
            if (pair_less(ka[mid], ia[mid], key, ix)) lo = mid + 1;
            else hi = mid;
          }
          pos = s0 + (k - amid) + (lo - s0);
        }
        kb[pos] = key;
        ib[pos] = ix;
      }
      __syncthreads();
      unsigned long long *tk = ka; ka = kb; kb = tk;
      unsigned *ti = ia; ia = ib; ib = ti;
    }
    const unsigned o = moff[h];
    for (unsigned k = threadIdx.x; k < m; k += blockDim.x) m_index[o + k] = ia[k];
    __syncthreads();
  }
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

SodConst make_sod_const(const psod_ctx *c) {
  SodConst K{};
  K.nx = c->nx;
  K.ncut = c->ncut;
  K.nxf = (float)c->nx;
  K.scale = c->scale;
  K.xs = c->xxmin * c->scale;                 // main:1565
  K.tx = (double)c->nx;                       // main:1517
  K.delta = c->p.delta;
  K.delta2 = c->p.delta2;
  K.cvol = 2.0 / 3.0 * 6.283185307179586;     // main:1424, 2049
  K.munit = (double)c->munit;
  K.mmin = (double)c->p.nmin;                 // main:698
  K.nsel = c->nsel;
  K.zmin = 0.0 * c->scale;                    // main:420, 691
  K.zmax = 1.0 * c->scale;                    // main:421, 692
  const double rmin = c->scale / c->nx;       // main:1526
  K.rmin2 = rmin * rmin;
  const double eps = c->scale / c->nx / 64.0; // main:1527
  K.eps2 = eps * eps;
  K.nbins = c->p.nbins;
  K.ndx = c->p.ndelta_extra;
  for (int e = 0; e < K.ndx; e++) K.dx_extra[e] = c->p.delta_extra[e];
  K.quirk_pos = c->quirk_pos;
  K.quirk_listed = c->quirk_listed;
  K.quirk_phys = c->quirk_phys;
  K.has_quirk = c->has_quirk;
  return K;
}

namespace {
struct DevBuf {
  std::vector<void *> ptrs;
  ~DevBuf() {
    for (void *p : ptrs) cudaFree(p);
  }
  template <typename T>
  T *get(psod_ctx *c, size_t n, int *st) {
    T *p = nullptr;
    if (*st) return nullptr;
    *st = dalloc(c, &p, n);
    if (!*st) ptrs.push_back(p);
    return p;
  }
};
}  // namespace

int stage_spherover(psod_ctx *c, psod_run_stats *out_stats) {
  if (!c->seeds_done) return set_err(c, PSOD_ERR_STATE, "psod_spherover needs psod_tri_cic first");
  psod_run_stats st{};
  st.fail_rank = -1;
  st.npart_new = c->npart_new;
  cudaEvent_t e0, e1, k0, k1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventCreate(&k0);
  cudaEventCreate(&k1);
  cudaEventRecord(e0, c->stream);
  int rc = PSOD_OK;
  DevBuf tmp;
  const SodConst K = make_sod_const(c);
  const long long n = c->n;
  const long long nseed = c->npart_new;
  long long kernels = 0;

  // reset alive flags: every call starts from the loaded cube
  PSOD_CUDA(c, cudaMemcpyAsync(c->d_cube, c->d_cube_orig, sizeof(float4) * n, cudaMemcpyDeviceToDevice, c->stream));

  // block grid of the scheduler
  int bs = 1;
  for (int cand : {4, 2}) {
    if (c->nx % cand == 0) {
      bs = cand;
      break;
    }
  }
  const int nb = c->nx / bs;
  const long long nblocks = (long long)nb * nb * nb;
  const int rdep = c->ncut + std::max(c->ncut, 2);
  const int rb = (rdep + bs - 1) / bs;

  unsigned *block_of = tmp.get<unsigned>(c, (size_t)nseed + 1, &rc);
  unsigned *blist = tmp.get<unsigned>(c, (size_t)nseed + 1, &rc);
  unsigned *bbegin = tmp.get<unsigned>(c, (size_t)nblocks + 1, &rc);
  unsigned *cursor = tmp.get<unsigned>(c, (size_t)nblocks + 1, &rc);
  unsigned *head = tmp.get<unsigned>(c, (size_t)nblocks, &rc);
  unsigned *filt_a = tmp.get<unsigned>(c, (size_t)nblocks, &rc);
  unsigned *filt_b = tmp.get<unsigned>(c, (size_t)nblocks, &rc);
  unsigned *ready = tmp.get<unsigned>(c, (size_t)nblocks + 1, &rc);
  unsigned *ctrs = tmp.get<unsigned>(c, 4, &rc);  // nready, work, gmin, quirk_rank
  unsigned char *processed = tmp.get<unsigned char>(c, (size_t)nseed + 1, &rc);
  unsigned long long *u64s = tmp.get<unsigned long long>(c, 6, &rc);  // err, nhalo, pool_used, touched, nprocessed
  double *edge_fac = tmp.get<double>(c, (size_t)c->p.nbins, &rc);
  // halo records by slot: at most one halo per Mmin particles
  const long long hcap = std::max<long long>(1, n / std::max(1, c->p.nmin) + 1);
  unsigned *h_rank = tmp.get<unsigned>(c, (size_t)hcap, &rc);
  long long *h_id = tmp.get<long long>(c, (size_t)hcap, &rc);
  long long *h_mass = tmp.get<long long>(c, (size_t)hcap, &rc);
  long long *h_mass2 = tmp.get<long long>(c, (size_t)hcap, &rc);
  long long *h_mextra = tmp.get<long long>(c, (size_t)hcap * std::max(1, c->p.ndelta_extra), &rc);
  long long *h_profile = tmp.get<long long>(c, (size_t)hcap * c->p.nbins, &rc);
  float *h_center = tmp.get<float>(c, (size_t)hcap * 3, &rc);
  double *h_rdelta = tmp.get<double>(c, (size_t)hcap, &rc);
  unsigned long long *h_pool = tmp.get<unsigned long long>(c, (size_t)hcap, &rc);
  unsigned long long *pool_key = tmp.get<unsigned long long>(c, (size_t)n, &rc);
  unsigned *pool_idx = tmp.get<unsigned>(c, (size_t)n, &rc);
  if (rc) return rc;

  PSOD_CUDA(c, cudaMemcpyAsync(edge_fac, c->edge_fac.data(), sizeof(double) * c->p.nbins, cudaMemcpyHostToDevice,
                               c->stream));
  PSOD_CUDA(c, cudaMemsetAsync(processed, 0, (size_t)nseed + 1, c->stream));
  PSOD_CUDA(c, cudaMemsetAsync(u64s, 0, sizeof(unsigned long long) * 6, c->stream));
  PSOD_CUDA(c, cudaMemsetAsync(u64s, 0xff, sizeof(unsigned long long), c->stream));  // err = none
  PSOD_CUDA(c, cudaMemsetAsync(ctrs, 0xff, sizeof(unsigned) * 4, c->stream));

  // seeds bucketed by scheduler block, in rank order within a block
  if (nseed > 0) {
    k_seed_blocks<<<nblk(nseed, 256), 256, 0, c->stream>>>(c->d_seed_idx, c->d_inv, c->d_cube, nseed, K, bs, nb,
                                                           block_of, blist);
    kernels++;
    unsigned *counts = tmp.get<unsigned>(c, (size_t)nblocks + 1, &rc);
    if (rc) return rc;
    PSOD_CUDA(c, cudaMemsetAsync(counts, 0, sizeof(unsigned) * (nblocks + 1), c->stream));
    k_count_u32<<<nblk(nseed, 256), 256, 0, c->stream>>>(block_of, nseed, counts);
    kernels++;
    if ((rc = scan_u32(c, counts, bbegin, nblocks, true))) return rc;
    if ((rc = radix_sort_u32(c, block_of, blist, nseed, 32))) return rc;
    PSOD_CUDA(c, cudaMemcpyAsync(cursor, bbegin, sizeof(unsigned) * nblocks, cudaMemcpyDeviceToDevice, c->stream));
    if (c->has_quirk) {
      unsigned qidx = 0;
      float4 qv;
      PSOD_CUDA(c, cudaMemcpyAsync(&qv, c->d_cube_orig + c->quirk_pos, sizeof(qv), cudaMemcpyDeviceToHost, c->stream));
      PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
      memcpy(&qidx, &qv.w, 4);
      qidx &= PSOD_IDX_MASK;
      k_find_rank<<<nblk(nseed, 256), 256, 0, c->stream>>>(c->d_seed_idx, nseed, qidx, ctrs + 3);
      kernels++;
    }
  }

  unsigned quirk_rank = PSOD_INF_RANK;
  PSOD_CUDA(c, cudaMemcpyAsync(&quirk_rank, ctrs + 3, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));

  const size_t smem = sizeof(Smem);
  PSOD_CUDA(c, cudaFuncSetAttribute(k_sod_seeds, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev_sms = 148;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->device);
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sod_seeds, TPB, smem);
  if (per_sm < 1) per_sm = 1;
  const unsigned seed_grid = (unsigned)(dev_sms * per_sm);

  float sod_ms = 0.f;
  long long rounds = 0, sod_launches = 0;
  while (nseed > 0) {
    PSOD_CUDA(c, cudaMemsetAsync(ctrs, 0, sizeof(unsigned) * 2, c->stream));            // nready, work
    PSOD_CUDA(c, cudaMemsetAsync(ctrs + 2, 0xff, sizeof(unsigned), c->stream));         // gmin
    k_heads<<<nblk(nblocks, 256), 256, 0, c->stream>>>(nblocks, bbegin, cursor, blist, processed, c->d_seed_idx,
                                                       c->d_inv, c->d_cube, head, ctrs + 2);
    k_minfilter<<<nblk(nblocks, 256), 256, 0, c->stream>>>(head, filt_a, nb, 0, rb);
    k_minfilter<<<nblk(nblocks, 256), 256, 0, c->stream>>>(filt_a, filt_b, nb, 1, rb);
    k_minfilter<<<nblk(nblocks, 256), 256, 0, c->stream>>>(filt_b, filt_a, nb, 2, rb);
    k_ready<<<nblk(nblocks, 256), 256, 0, c->stream>>>(nblocks, head, filt_a, quirk_rank, ctrs + 2, ready, ctrs);
    kernels += 5;
    unsigned nready = 0;
    PSOD_CUDA(c, cudaMemcpyAsync(&nready, ctrs, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
    if (nready == 0) break;
    SodBufs B;
    B.cube = c->d_cube;
    B.cs = c->d_cell_start;
    B.ids = c->d_ids;
    B.seed_idx = c->d_seed_idx;
    B.inv = c->d_inv;
    B.edge_fac = edge_fac;
    B.processed = processed;
    B.ready = ready;
    B.nready = ctrs;
    B.work = ctrs + 1;
    B.err = u64s;
    B.nhalo = u64s + 1;
    B.pool_used = u64s + 2;
    B.touched = u64s + 3;
    B.nprocessed = u64s + 4;
    B.h_rank = h_rank;
    B.h_id = h_id;
    B.h_mass = h_mass;
    B.h_mass2 = h_mass2;
    B.h_mextra = h_mextra;
    B.h_profile = h_profile;
    B.h_center = h_center;
    B.h_rdelta = h_rdelta;
    B.h_pool = h_pool;
    B.pool_key = pool_key;
    B.pool_idx = pool_idx;
    const unsigned grid = std::min<unsigned>(seed_grid, nready);
    cudaEventRecord(k0, c->stream);
    k_sod_seeds<<<grid, TPB, smem, c->stream>>>(K, B);
    cudaEventRecord(k1, c->stream);
    PSOD_CUDA(c, cudaGetLastError());
    PSOD_CUDA(c, cudaEventSynchronize(k1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, k0, k1);
    sod_ms += ms;
    rounds++;
    sod_launches++;
    kernels++;
  }
  unsigned long long hv[6];
  PSOD_CUDA(c, cudaMemcpyAsync(hv, u64s, sizeof(hv), cudaMemcpyDeviceToHost, c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  st.rounds = rounds;
  st.touched = (int64_t)hv[3];
  st.nprocessed = (int64_t)hv[4];
  st.ms_sod_kernel = sod_ms;
  st.sod_launches = sod_launches;
  c->nhalo = 0;
  c->nmember = 0;
  c->sod_done = false;
  if (hv[0] != ~0ull) {
    const int code = (int)(hv[0] & 0xff);
    st.fail_rank = (int64_t)(hv[0] >> 8);
    cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(k0); cudaEventDestroy(k1);
    st.kernel_launches = kernels;
    c->last_stats = st;
    if (out_stats) *out_stats = st;
    c->sod_done = true;  // zone output lost: empty table
    if (code == PSOD_ERR_NSEL)
      return set_err(c, PSOD_ERR_NSEL, "preselection exceeded nsel at seed rank " + std::to_string(st.fail_rank) +
                                           " (zone output lost; increase -nse)");
    if (code == PSOD_ERR_SELRADIUS)
      return set_err(c, PSOD_ERR_SELRADIUS, "overdensity above delta at the selection edge, seed rank " +
                                                std::to_string(st.fail_rank) + " (zone output lost; increase -sel)");
    return set_err(c, PSOD_ERR_STATE, "internal consistency check failed at seed rank " + std::to_string(st.fail_rank));
  }
  const long long nh = (long long)hv[1];
  // order halos by seed rank (the reference's output order)
  unsigned *order = tmp.get<unsigned>(c, (size_t)nh + 1, &rc);
  unsigned *rkeys = tmp.get<unsigned>(c, (size_t)nh + 1, &rc);
  unsigned *mass32 = tmp.get<unsigned>(c, (size_t)nh + 1, &rc);
  unsigned *moff = tmp.get<unsigned>(c, (size_t)nh + 1, &rc);
  unsigned long long *tkey = tmp.get<unsigned long long>(c, (size_t)std::max<unsigned long long>(hv[2], 1), &rc);
  unsigned *tidx = tmp.get<unsigned>(c, (size_t)std::max<unsigned long long>(hv[2], 1), &rc);
  if (rc) return rc;
  if (nh > 0) {
    std::vector<unsigned> iota((size_t)nh);
    for (long long i = 0; i < nh; i++) iota[(size_t)i] = (unsigned)i;
    PSOD_CUDA(c, cudaMemcpyAsync(order, iota.data(), sizeof(unsigned) * nh, cudaMemcpyHostToDevice, c->stream));
    PSOD_CUDA(c, cudaMemcpyAsync(rkeys, h_rank, sizeof(unsigned) * nh, cudaMemcpyDeviceToDevice, c->stream));
    PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
    if ((rc = radix_sort_u32(c, rkeys, order, nh, 32))) return rc;
  }
  const int ne = std::max(1, c->p.ndelta_extra);
  if ((rc = dalloc(c, &c->d_h_id, (size_t)nh))) return rc;
  if ((rc = dalloc(c, &c->d_h_mass, (size_t)nh))) return rc;
  if ((rc = dalloc(c, &c->d_h_rank, (size_t)nh))) return rc;
  if ((rc = dalloc(c, &c->d_h_mass2, (size_t)nh))) return rc;
  if ((rc = dalloc(c, &c->d_h_mextra, (size_t)nh * ne))) return rc;
  if ((rc = dalloc(c, &c->d_h_profile, (size_t)nh * c->p.nbins))) return rc;
  if ((rc = dalloc(c, &c->d_h_center, (size_t)nh * 3))) return rc;
  if ((rc = dalloc(c, &c->d_h_rdelta, (size_t)nh))) return rc;
  if ((rc = dalloc(c, &c->d_m_offset, (size_t)nh + 1))) return rc;
  if ((rc = dalloc(c, &c->d_m_index, (size_t)std::max<unsigned long long>(hv[2], 1)))) return rc;
  if (nh > 0) {
    const unsigned g1 = nblk(nh, 256);
    k_gather<long long><<<g1, 256, 0, c->stream>>>(h_id, order, nh, 1, c->d_h_id);
    k_gather<long long><<<g1, 256, 0, c->stream>>>(h_mass, order, nh, 1, c->d_h_mass);
    k_gather<long long><<<g1, 256, 0, c->stream>>>(h_mass2, order, nh, 1, c->d_h_mass2);
    k_gather<double><<<g1, 256, 0, c->stream>>>(h_rdelta, order, nh, 1, c->d_h_rdelta);
    k_gather<float><<<nblk(nh * 3, 256), 256, 0, c->stream>>>(h_center, order, nh, 3, c->d_h_center);
    if (c->p.ndelta_extra > 0)
      k_gather<long long><<<nblk(nh * ne, 256), 256, 0, c->stream>>>(h_mextra, order, nh, ne, c->d_h_mextra);
    k_gather<long long><<<nblk(nh * c->p.nbins, 256), 256, 0, c->stream>>>(h_profile, order, nh, c->p.nbins,
                                                                           c->d_h_profile);
    k_widen<<<g1, 256, 0, c->stream>>>(rkeys, nh, c->d_h_rank);
    k_mass_u32<<<g1, 256, 0, c->stream>>>(c->d_h_mass, nh, mass32);
    if ((rc = scan_u32(c, mass32, moff, nh, true))) return rc;
    k_widen<<<nblk(nh + 1, 256), 256, 0, c->stream>>>(moff, nh + 1, c->d_m_offset);
    k_member_sort<<<std::min<long long>(nh, 4 * dev_sms), 256, 0, c->stream>>>(
        order, nh, h_pool, c->d_h_mass, moff, pool_key, pool_idx, tkey, tidx, c->d_m_index);
    kernels += 11;
  } else {
    PSOD_CUDA(c, cudaMemsetAsync(c->d_m_offset, 0, sizeof(long long), c->stream));
  }
  PSOD_CUDA(c, cudaGetLastError());
  cudaEventRecord(e1, c->stream);
  PSOD_CUDA(c, cudaEventSynchronize(e1));
  float tot = 0.f;
  cudaEventElapsedTime(&tot, e0, e1);
  st.ms_total = tot;
  st.nhalo = nh;
  st.nmember = (int64_t)hv[2];
  st.kernel_launches = kernels;
  c->nhalo = nh;
  c->nmember = (long long)hv[2];
  c->sod_done = true;
  c->last_stats = st;
  if (out_stats) *out_stats = st;
  cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(k0); cudaEventDestroy(k1);
  return PSOD_OK;
}

}  // namespace psod
