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
#include <cstdio>
#include <cstdlib>

#include "psod_internal.cuh"

namespace psod {

namespace {

constexpr int TPB = 256;          // threads per seed CTA
constexpr unsigned RN_CHUNK = 2048;  // neighbour records per refinement work item
constexpr int NWARP = TPB / 32;
constexpr unsigned SEL_SPLIT_MAX = 4;  // select: contenders summed by the whole CTA
constexpr int NB = 4096;          // histogram buckets per level
constexpr int MAXLEV = 4;         // histogram levels kept in shared memory
constexpr int CAP = 2048;         // elements sorted in shared memory
constexpr unsigned long long POOL_SORTED = 1ull << 63;
constexpr double BALL0 = 1.5;      // first crossing ball of the batched mode (cells)
constexpr unsigned long long L1_BASE = 128896ull;  // (1023-16) << 7
constexpr int L1_SHIFT = 45;

enum { ERR_NONE = 0 };

// Seeds with fewer refinement candidates than this are neither bounded nor
// pruned: their pair work is small and the bound pass would cost as much as
// it saves.

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
  unsigned long long *err;   // (rank << 8) | code, atomicMin
  // halo records by slot
  unsigned long long *nhalo;
  unsigned long long *pool_used;
  unsigned *h_rank;
  long long *h_id, *h_mass, *h_mass2, *h_mextra;
  unsigned *h_profile;         // cumulative counts (widened on output)
  float *h_center;
  double *h_rdelta;
  unsigned long long *h_pool;  // pool offset; top bit: members already in (d2, index) order
  unsigned long long *pool_key;  // d2 bits
  unsigned *pool_idx;            // input index
  unsigned long long *touched;
  unsigned long long *nprocessed;
  // per ready slot (this round)
  unsigned *st_active;  // 1: refine and cross
  unsigned *st_na;      // alive particles in the preselect cube
  unsigned *st_coff;    // candidate slice offset
  unsigned *st_cn;      // candidate count
  unsigned *st_centre;  // cube position of the refined centre
  // candidates of this round
  unsigned *cand_pos;
  unsigned *cand_slot;  // owning ready slot
  double *cand_s;       // approximate refinement sum
  unsigned *cand_used;  // allocator
  unsigned *work;       // [4] work-stealing counters: prep, refine, select, cross
  unsigned *nbig;       // seeds of this round with bound_min candidates or more
  unsigned bound_min;   // seeds with this many candidates or more get the bound pass
  unsigned *maxcand;    // largest candidate count of a seed this round (or null)
  unsigned max_cand;    // seeds with more candidates wait (device tail loop), else ~0u
  unsigned *deferred;   // set when a seed waited for that reason
  unsigned *alive_cnt;  // alive records per cell (batched modes)
  unsigned long long *pairs;       // candidate-neighbour records visited
  unsigned long long *touch;       // records of the balls out to each stop
  unsigned long long *kept_members; // members of the kept halos written
  unsigned long long *pair_slots;  // lane slots spent on pair tests
  unsigned long long *ncand_total; // candidates over all rounds
  // refinement work: per (ready slot, candidate cell) counts, offsets into
  // cand_pos, 256-candidate chunks and their exclusive prefix
  unsigned *cell_cnt, *cell_off, *cell_chunks, *chunk_pref;
  unsigned *cell_nch;              // neighbour chunks per candidate cell
  unsigned nitems_cells;           // 27 * nready
  unsigned long long cand_cap;     // candidate buffer entries
  unsigned cap_ready;              // seeds processed per round at most
  int mode;
  // learned radius bracket
  const double *rho;               // input order
  unsigned long long *st_sbest;    // fixed-point refinement sum of the centre
  float *st_feat;                  // [slot][16] raw features
  float *st_rb0;                   // first ball radius (cells) when learn_use
  int learn_use, learn_collect;
  // FoF features (learn_fof): per input particle its halo rank or group
  // size (top bit), per FoF halo its mass, centre, radius and shape
  int learn_fof;
  const unsigned *fof_code;
  const long long *fof_mass;
  const double *fof_com, *fof_rad;
  const float4 *fof_feat;
  float *learn_x, *learn_t;        // collected samples
  unsigned long long *learn_n, learn_cap;
  unsigned long long *bracket_hits, *bracket_seeds, *cross_balls, *cross_records;
  // refinement bounds: 64-candidate groups per (slot, candidate cell) and
  // their prefix; per candidate an upper bound U of its sum; per slot the
  // best lower bound of the maximum sum (float bits)
  unsigned *cell_groups, *group_pref;
  float *cand_u;  // per candidate position (as cand_s), bounded seeds only
  unsigned *s_lmax;
  unsigned *work_bound;
  int bound_on;
  // per bounded seed the group with the largest upper bound (~0u: none),
  // whose sums run first; pair-pass phase: 0 all items (no bounds), 1 the
  // top groups, 2 the surviving candidates
  unsigned *s_top, *work_top;
  // phase-1 items: per seed the top group's candidate cell, first item
  // offset within the cell, item count, and the prefix sum of the counts
  unsigned *top_ci, *top_rem0, *top_n, *top_pref;
  int ref_phase;
  // phase 2 runs over the surviving candidates only: per candidate cell
  // their count and item count, the items' prefix sum, and the candidate
  // positions (cell by cell, at the cell's candidate offset)
  unsigned *cnt2, *chunks2, *chunk_pref2, *cand_list;
  unsigned long long *cand_pruned;
  unsigned *st_big;  // 1: the crossing needs the CTA path (null: CTA for all)
  // scheduler: one bit per seed in block-list order, set once the seed is
  // processed or claimed; list position of each rank and of each cube slot
  // (~0 for particles that are not seeds)
  unsigned *resolved, *bidx_of_rank, *bidx_of_cube;
  // crossing buffer: the entries (d2 bits, input index, cube slot) of large
  // balls, bucketed by their level-0 histogram bucket, one slice per seed;
  // xused allocates the slices of a round
  unsigned long long *xkey;
  unsigned *xidx, *xpos;
  unsigned long long *xused, xcap;
};

__device__ __forceinline__ void mark_resolved(const SodBufs &B, unsigned bi) {
  if (bi != 0xffffffffu) atomicOr(&B.resolved[bi >> 5], 1u << (bi & 31));
}

// Bitonic stages of a block-wide sort: thread k of a stage compares the
// pair (a, a + stride), a = 2k - (k mod stride), for k = threadIdx.x + j *
// blockDim.x.  For strides of at most 16 the pairs of warp w lie in its own
// 64-element blocks (a in [64w + 2j*blockDim.x, +64)), so consecutive stages
// with such strides need only a warp barrier; a stage with a wider stride
// (or the end of the sort) needs the block barrier.
__device__ __forceinline__ void bitonic_stage_sync(unsigned size, unsigned stride, unsigned m) {
  const unsigned next = stride > 1 ? (stride >> 1) : ((size << 1) <= m ? size : 0u);
  if (next != 0u && next <= 16u) __syncwarp();
  else __syncthreads();
}

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
  unsigned long long xbase;  // the seed's slice of the crossing buffer (bucketed ball)
  unsigned claim_cnt;
  // last radial_search hit: sorted-buffer index and bucket lower bound
  int res_k;
  unsigned long long res_lo;
  // select: the contenders of a seed that has few
  unsigned nsel;
  unsigned sel[SEL_SPLIT_MAX];
};

__device__ __forceinline__ int wrapi(int a, int nx) {
  if (a >= nx) a -= nx;
  if (a < 0) a += nx;
  return a;
}

// Visit every particle record filed under the cells of the cube of
// half-width R around (ic,jc,kc): warp per row of cells, lanes stride along
// the row's contiguous run of records.
// The records [b, e) of one run, lanes on consecutive records, each lane in
// increasing order.  Four loads per lane are issued before the first record
// is used: a CTA that walks a large region alone is bound by the loads it
// keeps in flight.
template <typename F>
__device__ __forceinline__ void run_records(const SodBufs &B, unsigned b, unsigned e, F &f) {
  unsigned p = b + (threadIdx.x & 31u);
  for (; p + 96u < e; p += 128u) {
    const float4 v0 = B.cube[p], v1 = B.cube[p + 32u], v2 = B.cube[p + 64u], v3 = B.cube[p + 96u];
    f(p, v0);
    f(p + 32u, v1);
    f(p + 64u, v2);
    f(p + 96u, v3);
  }
  for (; p < e; p += 32u) f(p, B.cube[p]);
}

template <typename F>
__device__ __forceinline__ void for_cube(const SodConst &K, const SodBufs &B, int ic, int jc, int kc, int R, F f) {
  const int w = threadIdx.x >> 5;
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
    for (int q = 0; q < np; q++) run_records(B, B.cs[base + (unsigned)pa[q]], B.cs[base + (unsigned)pb[q] + 1], f);
  }
}

// The part of a seed's preselect cube the crossing search visits: the whole
// cube (rb2 < 0), or only the cube cells that intersect the ball of radius
// rb around the centre.  Inside such a ball every alive particle of the cube
// is visited, so ranks of particles with d2 <= rb2 are exact.
struct Region {
  int ic, jc, kc;     // seed cell: the cube centre
  double xc, yc, zc;  // refined centre, grid units
  double rb2;         // ball radius squared; < 0 means the whole cube
  double rb;
};

// distance from ball-centre offset t0 (cells, relative to the seed cell
// centre) to the cell at offset t, minus half a cell, periodic, >= 0
__device__ __forceinline__ double cell_gap(double t0, int t, double nxd) {
  double d = fabs((double)t - t0);
  d = fmin(d, nxd - d);
  return fmax(d - 0.5, 0.0);
}

template <typename F>
__device__ __forceinline__ void for_region(const SodConst &K, const SodBufs &B, const Region &G, F f) {
  if (G.rb2 < 0.0) {
    for_cube(K, B, G.ic, G.jc, G.kc, K.ncut, f);
    return;
  }
  const int w = threadIdx.x >> 5;
  const int R = K.ncut, side = 2 * R + 1, nrow = side * side;
  const unsigned nx = (unsigned)K.nx;
  const double nxd = (double)K.nx;
  // ball centre relative to the seed cell centre (cell i spans [i+xs, i+xs+1))
  auto rel = [&](double x, int i, int a) {
    double d = x - ((double)i + K.xs[a] + 0.5);
    d = d - nxd * floor(d / nxd + 0.5);
    return d;
  };
  const double tx = rel(G.xc, G.ic, 0), ty = rel(G.yc, G.jc, 1), tz = rel(G.zc, G.kc, 2);
  const double rm = G.rb + 1e-3;  // margin for rounding at cell edges
  const double rm2 = rm * rm;
  for (int row = w; row < nrow; row += NWARP) {
    const int dj = row % side - R, dk = row / side - R;
    const double gy = cell_gap(ty, dj, nxd), gz = cell_gap(tz, dk, nxd);
    const double rem = rm2 - gy * gy - gz * gz;
    if (rem < 0.0) continue;
    const double wx = sqrt(rem);
    int t0 = (int)ceil(tx - 0.5 - wx), t1 = (int)floor(tx + 0.5 + wx);
    t0 = max(t0, -R);
    t1 = min(t1, R);
    if (t0 > t1) continue;
    const unsigned jj = (unsigned)wrapi(G.jc + dj, K.nx), kk = (unsigned)wrapi(G.kc + dk, K.nx);
    const unsigned long long base = (unsigned long long)nx * (jj + (unsigned long long)nx * kk);
    const int x0 = G.ic + t0, x1 = G.ic + t1;
    int pa[2], pb[2], np;
    if (x0 < 0) {
      pa[0] = x0 + K.nx; pb[0] = K.nx - 1; pa[1] = 0; pb[1] = x1; np = 2;
      if (x1 < 0) { pa[0] = x0 + K.nx; pb[0] = x1 + K.nx; np = 1; }
    } else if (x1 >= K.nx) {
      pa[0] = x0; pb[0] = K.nx - 1; pa[1] = 0; pb[1] = x1 - K.nx; np = 2;
      if (x0 >= K.nx) { pa[0] = x0 - K.nx; pb[0] = x1 - K.nx; np = 1; }
    } else {
      pa[0] = x0; pb[0] = x1; np = 1;
    }
    for (int q = 0; q < np; q++) run_records(B, B.cs[base + (unsigned)pa[q]], B.cs[base + (unsigned)pb[q] + 1], f);
  }
}

// Records filed under the region's cells (alive or not), from the cell
// offsets alone (no record loads).  For the ball out to the stopping
// particle this is the algorithmic read volume of the crossing search.
__device__ __forceinline__ unsigned region_records(const SodConst &K, const SodBufs &B, const Region &G) {
  const int R = K.ncut, side = 2 * R + 1, nrow = side * side;
  const unsigned nx = (unsigned)K.nx;
  const double nxd = (double)K.nx;
  auto rel = [&](double x, int i, int a) {
    double d = x - ((double)i + K.xs[a] + 0.5);
    d = d - nxd * floor(d / nxd + 0.5);
    return d;
  };
  const double tx = rel(G.xc, G.ic, 0), ty = rel(G.yc, G.jc, 1), tz = rel(G.zc, G.kc, 2);
  const double rm2 = G.rb * G.rb;
  unsigned sum = 0;
  for (int row = threadIdx.x; row < nrow; row += TPB) {
    const int dj = row % side - R, dk = row / side - R;
    const double gy = cell_gap(ty, dj, nxd), gz = cell_gap(tz, dk, nxd);
    // each operation rounded on its own (no contraction): the count is
    // restated exactly by the oracle
    const double rem = __dsub_rn(__dsub_rn(rm2, __dmul_rn(gy, gy)), __dmul_rn(gz, gz));
    if (rem < 0.0) continue;
    const double wx = sqrt(rem);
    const int t0 = max((int)ceil(tx - 0.5 - wx), -R), t1 = min((int)floor(tx + 0.5 + wx), R);
    if (t0 > t1) continue;
    const unsigned jj = (unsigned)wrapi(G.jc + dj, K.nx), kk = (unsigned)wrapi(G.kc + dk, K.nx);
    const unsigned long long base = (unsigned long long)nx * (jj + (unsigned long long)nx * kk);
    for (int t = t0; t <= t1; t++) {
      const unsigned c = (unsigned)wrapi(G.ic + t, K.nx);
      sum += B.cs[base + c + 1] - B.cs[base + c];
    }
  }
  return sum;
}

// d2 of a record to the region's centre if it is alive and inside the
// region's ball (always inside for the whole cube); else returns false
__device__ __forceinline__ bool region_d2(const SodConst &K, const Region &G, float4 v, double &d2) {
  if (__float_as_uint(v.w) & PSOD_DEAD_BIT) return false;
  d2 = min_image_d2((double)to_grid(v.x, K.nxf), (double)to_grid(v.y, K.nxf), (double)to_grid(v.z, K.nxf), G.xc,
                    G.yc, G.zc, K.tx);
  return G.rb2 < 0.0 || d2 <= G.rb2;
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
__device__ __forceinline__ void hist_prefix(Smem &S, int l) {
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

// Entry sources of the crossing searches: (d2 bits, input index, cube slot)
// of the alive records of a region, computed from the records as they are
// walked, or a contiguous slice of the seed's bucketed crossing buffer
// (written once per ball by scatter_ball).
struct RegionSrc {
  const Region &g;
  template <typename F>
  __device__ __forceinline__ void each(const SodConst &K, const SodBufs &B, F &&f) const {
    for_region(K, B, g, [&](unsigned p, float4 v) {
      double d2;
      if (!region_d2(K, g, v, d2)) return;
      f(dbits(d2), __float_as_uint(v.w) & PSOD_IDX_MASK, p);
    });
  }
};

struct BufSrc {
  unsigned long long lo, hi;  // entries [lo, hi) of the crossing buffer
  template <typename F>
  __device__ __forceinline__ void each(const SodConst &K, const SodBufs &B, F &&f) const {
    for (unsigned long long e = lo + threadIdx.x; e < hi; e += TPB) f(B.xkey[e], B.xidx[e], B.xpos[e]);
  }
};

// fill S.hist[l] with the bucket counts of the source's entries whose d2
// bits lie in the level's range (level 0: all)
template <class Src>
__device__ __forceinline__ void build_hist(const SodConst &K, const SodBufs &B, Smem &S, int l, const Src &src) {
  for (int k = threadIdx.x; k < NB; k += TPB) S.hist[l][k] = 0;
  __syncthreads();
  const Level L = S.lev[l];
  src.each(K, B, [&](unsigned long long x, unsigned, unsigned) {
    if (l > 0 && (x < L.lo || x > L.hi)) return;
    atomicAdd(&S.hist[l][bucket_of(L, l, x)], 1u);
  });
  __syncthreads();
}

// level-0 histogram of a ball's alive records (one region walk); returns
// the ball's entry count and adds it to the ball-record statistic
__device__ __forceinline__ unsigned ball_hist0(const SodConst &K, const SodBufs &B, Smem &S, const Region &G) {
  if (threadIdx.x == 0) {
    S.lev[0].lo = 0;
    S.lev[0].hi = 0x7fefffffffffffffull;
    S.lev[0].shift = L1_SHIFT;
  }
  for (int k = threadIdx.x; k < NB; k += TPB) S.hist[0][k] = 0;
  __syncthreads();
  unsigned inball = 0;
  RegionSrc{G}.each(K, B, [&](unsigned long long x, unsigned, unsigned) {
    inball++;
    atomicAdd(&S.hist[0][bucket_of(S.lev[0], 0, x)], 1u);
  });
  __syncthreads();
  const unsigned tot = block_sum_u32(S, inball);
  if (threadIdx.x == 0) atomicAdd(B.cross_records, (unsigned long long)tot);
  return tot;
}

// load the source's entries with d2 bits in [lo, hi] into S.skey/S.sidx and
// sort them by (bits, input index); returns the count
template <class Src>
__device__ __forceinline__ unsigned extract_sorted(const SodConst &K, const SodBufs &B, Smem &S, const Src &src,
                                   unsigned long long lo, unsigned long long hi) {
  if (threadIdx.x == 0) S.nsorted = 0;
  __syncthreads();
  src.each(K, B, [&](unsigned long long x, unsigned ix, unsigned) {
    if (x < lo || x > hi) return;
    unsigned s = atomicAdd(&S.nsorted, 1u);
    if (s < CAP) {
      S.skey[s] = x;
      S.sidx[s] = ix;
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
      bitonic_stage_sync(size, stride, m);
    }
  }
  return n;
}

// Small balls.  When a seed's ball holds at most CAP alive records, one pass
// loads them all (d2 bits, input index, cube position) and one bitonic sort
// orders them by (d2 bits, index).  The crossing searches, the profile and
// the claims then read the sorted list instead of visiting the cells again.
// The positions live in the deepest histogram level, which this path never
// uses.
__device__ __forceinline__ unsigned *small_pos(Smem &S) { return S.hist[MAXLEV - 1]; }

// every alive record of region G, sorted; returns the count, or CAP + 1 when
// the region holds more than CAP (the list is then unusable)
__device__ __forceinline__ unsigned load_ball_sorted(const SodConst &K, const SodBufs &B, Smem &S, const Region &G) {
  unsigned *spos = small_pos(S);
  if (threadIdx.x == 0) S.nsorted = 0;
  __syncthreads();
  for_region(K, B, G, [&](unsigned p, float4 v) {
    double d2;
    if (!region_d2(K, G, v, d2)) return;
    const unsigned s = atomicAdd(&S.nsorted, 1u);
    if (s < CAP) {
      S.skey[s] = dbits(d2);
      S.sidx[s] = __float_as_uint(v.w) & PSOD_IDX_MASK;
      spos[s] = p;
    }
  });
  __syncthreads();
  const unsigned n = S.nsorted;
  if (threadIdx.x == 0) atomicAdd(B.cross_records, (unsigned long long)n);
  __syncthreads();
  if (n > CAP) return CAP + 1;
  unsigned m = 1;
  while (m < n) m <<= 1;
  for (unsigned k = n + threadIdx.x; k < m; k += TPB) {
    S.skey[k] = ~0ull;
    S.sidx[k] = 0xffffffffu;
  }
  __syncthreads();
  for (unsigned size = 2; size <= m; size <<= 1) {
    for (unsigned stride = size >> 1; stride > 0; stride >>= 1) {
      for (unsigned k = threadIdx.x; k < m / 2; k += TPB) {
        const unsigned a = 2 * k - (k & (stride - 1)), bb = a + stride;
        const bool up = ((a & size) == 0);
        const unsigned long long ka = S.skey[a], kb = S.skey[bb];
        const unsigned ia = S.sidx[a], ib = S.sidx[bb];
        const bool gt = (ka > kb) || (ka == kb && ia > ib);
        if (gt == up) {
          S.skey[a] = kb;
          S.skey[bb] = ka;
          S.sidx[a] = ib;
          S.sidx[bb] = ia;
          const unsigned pa = spos[a];
          spos[a] = spos[bb];
          spos[bb] = pa;
        }
      }
      bitonic_stage_sync(size, stride, m);
    }
  }
  return n;
}

// forward crossing search over the sorted list [0, n): the first 1-based
// position i >= 10 where the reference's loop stops (main:2046); 0 if none
__device__ __forceinline__ long long sorted_stop(const SodConst &K, Smem &S, unsigned n, long long na, double delta) {
  int best = 0x7fffffff;
  for (unsigned k = 9 + threadIdx.x; k < n; k += TPB)
    if (!keeps_going(K, (long long)k + 1, bitsd(S.skey[k]), na, delta)) best = min(best, (int)k);
  best = block_min_i(S, best);
  return best == 0x7fffffff ? 0 : (long long)best + 1;
}

// Search over the sorted d2 sequence of the ball.
//  mode 0 (forward): first 1-based position i >= 10 where the reference's
//                    loop stops for threshold delta.
//  mode 1 (backward): last position i in [2, imax] with overdensity > delta.
// The level-0 histogram of the ball is in S.hist[0] (built by the caller).
// BUF: the ball's entries are bucketed in the crossing buffer from S.xbase
// (level-0 bucket order), so descents and extractions read the slice of the
// level-0 bucket under examination; otherwise they walk the region G.
// Returns 0 if not found, else the position; *d2_out its squared distance.
// Returns -1 on an unresolvable bucket (more than CAP exact-equal keys).
template <bool BUF>
__device__ __forceinline__ long long radial_search(const SodConst &K, const SodBufs &B, Smem &S, const Region &G, long long na,
                                   double delta, int mode, long long imax, double *d2_out) {
  int l = 0;
  unsigned long long b0lo = 0, b0hi = 0;  // buffer slice of the level-0 bucket being resolved
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
    if (BUF && l == 0) {
      b0lo = S.xbase + S.pref[cand];
      b0hi = b0lo + nb;
    }
    if (nb <= CAP) {
      unsigned n;
      if constexpr (BUF) n = extract_sorted(K, B, S, BufSrc{b0lo, b0hi}, lo, hi);
      else n = extract_sorted(K, B, S, RegionSrc{G}, lo, hi);
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
    if constexpr (BUF) build_hist(K, B, S, l, BufSrc{b0lo, b0hi});
    else build_hist(K, B, S, l, RegionSrc{G});
  }
}

// the pos-th (1-based) element of the sorted sequence when it is the last
// element below `below_lo`: the maximum (bits, index) under that bound
template <class Src>
__device__ __forceinline__ void max_below(const SodConst &K, const SodBufs &B, Smem &S, const Src &src,
                          unsigned long long below_lo, unsigned long long &kout, unsigned &iout) {
  unsigned long long a = 0, b = 0;
  src.each(K, B, [&](unsigned long long x, unsigned ixu, unsigned) {
    if (x >= below_lo) return;
    const unsigned long long ix = ixu;
    if (x > a || (x == a && ix > b)) { a = x; b = ix; }
  });
  block_max_pair(S, a, b);
  kout = a;
  iout = (unsigned)b;
}

__device__ __forceinline__ void record_error(const SodBufs &B, unsigned rank, unsigned code) {
  atomicMin(B.err, ((unsigned long long)rank << 8) | code);
}

struct SeedGeo {
  unsigned sp;  // cube position of the seed
  int ic, jc, kc;
};

__device__ __forceinline__ SeedGeo seed_geo(const SodConst &K, const SodBufs &B, unsigned rank) {
  SeedGeo g;
  g.sp = B.inv[B.seed_idx[rank]];
  const float4 v = B.cube[g.sp];
  g.ic = sod_cell_axis(to_grid(v.x, K.nxf), K.xs[0], K.nx);
  g.jc = sod_cell_axis(to_grid(v.y, K.nxf), K.xs[1], K.nx);
  g.kc = sod_cell_axis(to_grid(v.z, K.nxf), K.xs[2], K.nx);
  return g;
}

// CTA-level work stealing over the round's ready list
__device__ __forceinline__ unsigned next_item(unsigned *ctr) {
  __shared__ unsigned s_item;
  __syncthreads();
  if (threadIdx.x == 0) s_item = atomicAdd(ctr, 1u);
  __syncthreads();
  return s_item;
}

// records filed under the cube's cells (alive or not): one run per row
__device__ __forceinline__ unsigned cube_records(const SodConst &K, const SodBufs &B, Smem &S, int ic, int jc, int kc) {
  const int R = K.ncut, side = 2 * R + 1;
  unsigned sum = 0;
  for (int row = threadIdx.x; row < side * side; row += TPB) {
    const int dj = row % side - R, dk = row / side - R;
    const unsigned jj = (unsigned)wrapi(jc + dj, K.nx), kk = (unsigned)wrapi(kc + dk, K.nx);
    const unsigned long long base = (unsigned long long)K.nx * (jj + (unsigned long long)K.nx * kk);
    const int x0 = ic - R, x1 = ic + R;
    if (x0 < 0) {
      sum += B.cs[base + K.nx] - B.cs[base + (unsigned)(x0 + K.nx)];
      sum += B.cs[base + (unsigned)x1 + 1] - B.cs[base];
    } else if (x1 >= K.nx) {
      sum += B.cs[base + K.nx] - B.cs[base + (unsigned)x0];
      sum += B.cs[base + (unsigned)(x1 - K.nx) + 1] - B.cs[base];
    } else {
      sum += B.cs[base + (unsigned)x1 + 1] - B.cs[base + (unsigned)x0];
    }
  }
  return block_sum_u32(S, sum);
}

__device__ __forceinline__ int zig(int a) { return (a & 1) ? -((a + 1) >> 1) : (a >> 1); }

// alive particles of the cube from the per-cell counts, rows nearest the
// seed first; stops once `need` is reached (returns the running sum)
__device__ __forceinline__ unsigned alive_rows(const SodConst &K, const SodBufs &B, Smem &S, int ic, int jc, int kc, unsigned need) {
  const int R = K.ncut, side = 2 * R + 1, nrow = side * side;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned total = 0;
  for (int r0 = 0; r0 < nrow; r0 += NWARP) {
    const int row = r0 + w;
    unsigned part = 0;
    if (row < nrow) {
      const int dj = zig(row % side), dk = zig(row / side);
      const unsigned jj = (unsigned)wrapi(jc + dj, K.nx), kk = (unsigned)wrapi(kc + dk, K.nx);
      const unsigned long long base = (unsigned long long)K.nx * (jj + (unsigned long long)K.nx * kk);
      for (int t = lane; t < side; t += 32) part += B.alive_cnt[base + (unsigned)wrapi(ic - R + t, K.nx)];
    }
    total += block_sum_u32(S, part);
    if (total >= need) break;
  }
  return total;
}

// ---------------------------------------------------------------------------
// phase 1: preselect count (main:1657-1716) and the candidate list of the
// +-1 cells (main:1807-1826)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void prep_seed(const SodConst &K, const SodBufs &B, Smem &S, unsigned slot, unsigned rank) {
  if (threadIdx.x == 0) {
    B.st_active[slot] = 0;
    B.st_cn[slot] = 0;
    B.processed[rank] = 1;
    mark_resolved(B, B.bidx_of_rank[rank]);
  }
  // no refinement work unless this seed turns out active
  if (threadIdx.x < 27) {
    B.cell_cnt[slot * 27 + threadIdx.x] = 0;
    B.cell_chunks[slot * 27 + threadIdx.x] = 0;
    B.cell_groups[slot * 27 + threadIdx.x] = 0;
  }
  const SeedGeo g = seed_geo(K, B, rank);
  if (__float_as_uint(B.cube[g.sp].w) & PSOD_DEAD_BIT) return;  // claimed (main:1628)
  unsigned na = 0;
  if (B.mode == PSOD_MODE_PLAIN) {
    // the reference's preselect: every record of the cube
    unsigned cnt = 0, recs = 0;
    for_cube(K, B, g.ic, g.jc, g.kc, K.ncut, [&](unsigned p, float4 v) {
      recs++;
      if (!(__float_as_uint(v.w) & PSOD_DEAD_BIT)) cnt++;
    });
    na = block_sum_u32(S, cnt);
    const unsigned nrec = block_sum_u32(S, recs);
    if (threadIdx.x == 0) atomicAdd(B.touched, (unsigned long long)nrec);
    if ((long long)na > K.nsel) {
      if (threadIdx.x == 0) record_error(B, rank, PSOD_ERR_NSEL);
      return;
    }
    if (!(dmul((double)na, K.munit) >= K.mmin)) return;  // main:1759
  } else {
    // same tests from the per-cell alive counts: nsel against the cube's
    // record count (exact alive count only when that bound exceeds nsel),
    // Mmin by summing rows nearest the seed first until it is reached
    if (K.n_total > K.nsel) {
      const unsigned recs = cube_records(K, B, S, g.ic, g.jc, g.kc);
      if ((long long)recs > K.nsel) {
        const unsigned exact = alive_rows(K, B, S, g.ic, g.jc, g.kc, ~0u);
        if ((long long)exact > K.nsel) {
          if (threadIdx.x == 0) record_error(B, rank, PSOD_ERR_NSEL);
          return;
        }
      }
    }
    const unsigned need = K.mmin_count;
    const unsigned got = alive_rows(K, B, S, g.ic, g.jc, g.kc, need);
    if (got < need) return;  // main:1759
  }
  // candidates: alive records filed under the 27 cells around the seed cell,
  // grouped by cell in the reference's scan order (x outer, z inner)
  __shared__ unsigned s_cnt[27], s_coff[27], s_base;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int o = w; o < 27; o += NWARP) {
    const int di = o / 9 - 1, dj = (o / 3) % 3 - 1, dk = o % 3 - 1;
    const unsigned cell = (unsigned)wrapi(g.ic + di, K.nx) +
                          (unsigned)K.nx * ((unsigned)wrapi(g.jc + dj, K.nx) + (unsigned)K.nx * (unsigned)wrapi(g.kc + dk, K.nx));
    const unsigned b = B.cs[cell], e = B.cs[cell + 1];
    unsigned c = 0;
    for (unsigned p = b + lane; p < e; p += 32) c += !(__float_as_uint(B.cube[p].w) & PSOD_DEAD_BIT);
    for (int sh = 16; sh > 0; sh >>= 1) c += __shfl_down_sync(0xffffffffu, c, sh);
    if (lane == 0) s_cnt[o] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned tot = 0;
    for (int o = 0; o < 27; o++) {
      s_coff[o] = tot;
      tot += s_cnt[o];
    }
    const bool too_many = tot > B.max_cand;
    s_base = too_many ? 0u : atomicAdd(B.cand_used, tot);
    if (B.maxcand) atomicMax(B.maxcand, tot);
    if (too_many || (unsigned long long)s_base + tot > B.cand_cap) {
      // candidate buffer full this round, or more candidates than the
      // device tail loop takes: the seed waits for the next round
      s_base = 0xffffffffu;
      B.processed[rank] = 0;
      {
        const unsigned bi = B.bidx_of_rank[rank];
        atomicAnd(&B.resolved[bi >> 5], ~(1u << (bi & 31)));
      }
      if (too_many) atomicOr(B.deferred, 1u);
      else if (tot > B.cand_cap) record_error(B, rank, PSOD_ERR_STATE);
    } else {
      B.st_na[slot] = na;  // 0 when unknown (batched modes)
      B.st_coff[slot] = s_base;
      B.st_cn[slot] = tot;
      B.st_active[slot] = 1;
      if (tot >= B.bound_min) atomicAdd(B.nbig, 1u);
      B.st_centre[slot] = g.sp;  // no candidate: the seed stays the centre
      atomicAdd(B.nprocessed, 1ull);
    }
  }
  __syncthreads();
  if (s_base == 0xffffffffu) return;
  if (threadIdx.x < 27) {
    const int o = threadIdx.x;
    const int ci = wrapi(g.ic + o / 9 - 1, K.nx), cj = wrapi(g.jc + (o / 3) % 3 - 1, K.nx),
              ck = wrapi(g.kc + o % 3 - 1, K.nx);
    // records of the 3x3x3 cells around this candidate cell
    unsigned nbr = 0;
    for (int r = 0; r < 9; r++) {
      const unsigned yy = (unsigned)wrapi(cj + r % 3 - 1, K.nx), zz = (unsigned)wrapi(ck + r / 3 - 1, K.nx);
      const unsigned long long base = (unsigned long long)K.nx * (yy + (unsigned long long)K.nx * zz);
      const int x0 = ci - 1, x1 = ci + 1;
      if (x0 < 0) {
        nbr += B.cs[base + K.nx] - B.cs[base + (unsigned)(x0 + K.nx)] + B.cs[base + (unsigned)x1 + 1] - B.cs[base];
      } else if (x1 >= K.nx) {
        nbr += B.cs[base + K.nx] - B.cs[base + (unsigned)x0] + B.cs[base + (unsigned)(x1 - K.nx) + 1] - B.cs[base];
      } else {
        nbr += B.cs[base + (unsigned)x1 + 1] - B.cs[base + (unsigned)x0];
      }
    }
    const unsigned nch = max(1u, (nbr + RN_CHUNK - 1) / RN_CHUNK);
    B.cell_cnt[slot * 27 + o] = s_cnt[o];
    B.cell_off[slot * 27 + o] = s_base + s_coff[o];
    B.cell_nch[slot * 27 + o] = nch;
    B.cell_chunks[slot * 27 + o] = ((s_cnt[o] + 63u) / 64u) * nch;
    B.cell_groups[slot * 27 + o] = (s_cnt[o] + 63u) / 64u;
  }
  for (int o = w; o < 27; o += NWARP) {
    const int di = o / 9 - 1, dj = (o / 3) % 3 - 1, dk = o % 3 - 1;
    const unsigned cell = (unsigned)wrapi(g.ic + di, K.nx) +
                          (unsigned)K.nx * ((unsigned)wrapi(g.jc + dj, K.nx) + (unsigned)K.nx * (unsigned)wrapi(g.kc + dk, K.nx));
    const unsigned b = B.cs[cell], e = B.cs[cell + 1];
    unsigned q = s_base + s_coff[o];
    for (unsigned p0 = b; p0 < e; p0 += 32) {
      const unsigned p = p0 + lane;
      const bool alive = p < e && !(__float_as_uint(B.cube[p].w) & PSOD_DEAD_BIT);
      const unsigned m = __ballot_sync(0xffffffffu, alive);
      if (alive) {
        const unsigned at = q + __popc(m & ((1u << lane) - 1u));
        B.cand_pos[at] = p;
        B.cand_slot[at] = slot;
        // refinement partial sums accumulate here; the foreign-filed
        // particle always goes to the exact pass
        B.cand_s[at] = (K.has_quirk && p == K.quirk_pos) ? __longlong_as_double(0x7ff0000000000000ll) : 0.0;
      }
      q += __popc(m);
    }
  }
}

__global__ void __launch_bounds__(TPB) k_prep(SodConst K, SodBufs B) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem &S = *reinterpret_cast<Smem *>(smem_raw);
  while (true) {
    const unsigned item = next_item(&B.work[0]);
    if (item >= min(*B.nready, B.cap_ready)) break;
    prep_seed(K, B, S, item, B.ready[item]);
  }
}

// ---------------------------------------------------------------------------
// phase 2: approximate refinement sums, one warp per candidate over the whole
// GPU.  Distances in FP32 with a relative error below 1e-6; pairs whose FP32
// d2 lies within 1e-5 of the inclusion edge are decided in exact FP64; the
// sum is accumulated in FP64.  |S_approx - S| <= REF_TOL * S.
// ---------------------------------------------------------------------------
constexpr double REF_TOL = 1e-5;

// FP32 minimum-image |a - b| with one rounding on the small branch
__device__ __forceinline__ float mi_dx(float a, float b, float nxf) {
  const float hi = fmaxf(a, b), lo = fminf(a, b);
  const float d1 = __fsub_rn(hi, lo);
  const float d2 = __fadd_rn(__fsub_rn(nxf, hi), lo);
  return fminf(d1, d2);
}

// does candidate cell (x,y,z) lie within +-2 cells of the seed (x_sel2)?
__device__ __forceinline__ bool in_sel2(const SodConst &K, int x, int y, int z, int ic, int jc, int kc) {
  return abs(pdiff(x, ic, K.nx)) <= 2 && abs(pdiff(y, jc, K.nx)) <= 2 && abs(pdiff(z, kc, K.nx)) <= 2;
}

// Refinement sum of one candidate, warp-cooperative.  exact: canonical
// int64 fixed-point sum of FP64 terms (main:1840-1859); else the FP64 sum of
// FP32 terms.  Result valid in lane 0.
// The alive records of the 3x3x3 cells around cell (cx, cy, cz) that lie
// within +-2 cells of the seed cell (ic, jc, kc), as one list: lane l < 27
// holds cell l's record range (begin, exclusive prefix of the lengths);
// `at` maps a list position to its cube slot.  One warp; all lanes call.
struct NbrList {
  unsigned beg, pre, total;  // this lane's cell (lanes < 27), the list length
  __device__ __forceinline__ unsigned at(unsigned t) const {
    // the last cell whose prefix is <= t (cells 0..26 held by lanes 0..26):
    // five halvings cover 27 cells; every lane takes all five steps, so
    // every shuffle has the whole warp
    int lo = 0, hi = 26;
#pragma unroll
    for (int step = 0; step < 5; step++) {
      const int mid = (lo + hi + 1) >> 1;
      const unsigned pm = __shfl_sync(0xffffffffu, pre, mid);
      if (lo < hi) {
        if (pm <= t) lo = mid;
        else hi = mid - 1;
      }
    }
    return __shfl_sync(0xffffffffu, beg, lo) + (t - __shfl_sync(0xffffffffu, pre, lo));
  }
};

__device__ __forceinline__ NbrList nbr_list(const SodConst &K, const SodBufs &B, int cx, int cy, int cz, int ic,
                                            int jc, int kc) {
  const int lane = threadIdx.x & 31;
  unsigned beg = 0, len = 0;
  if (lane < 27) {
    const int xx = wrapi(cx + lane % 3 - 1, K.nx), yy = wrapi(cy + (lane / 3) % 3 - 1, K.nx),
              zz = wrapi(cz + lane / 9 - 1, K.nx);
    if (abs(pdiff(xx, ic, K.nx)) <= 2 && abs(pdiff(yy, jc, K.nx)) <= 2 && abs(pdiff(zz, kc, K.nx)) <= 2) {
      const unsigned long long c = (unsigned long long)xx + (unsigned long long)K.nx * ((unsigned)yy + (unsigned long long)K.nx * (unsigned)zz);
      beg = B.cs[c];
      len = B.cs[c + 1] - beg;
    }
  }
  unsigned inc = len;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  NbrList L;
  L.beg = beg;
  L.pre = inc - len;
  L.total = __shfl_sync(0xffffffffu, inc, 26);
  return L;
}

// Refinement sum of one candidate, warp-cooperative.  exact: canonical
// int64 fixed-point sum of FP64 terms (main:1840-1859); else the FP64 sum of
// FP32 terms.  Result valid in lane 0.  The 27 neighbour cells are walked
// as one list, 32 records a step.
template <bool EXACT>
__device__ __forceinline__ void refine_sum(const SodConst &K, const SodBufs &B, unsigned cp, int ic, int jc, int kc,
                           unsigned long long &sq_out, double &sf_out, unsigned *visits = nullptr,
                           unsigned part = 0, unsigned nparts = 1) {
  const int lane = threadIdx.x & 31;
  const float4 cv = B.cube[cp];
  const float cxg = to_grid(cv.x, K.nxf), cyg = to_grid(cv.y, K.nxf), czg = to_grid(cv.z, K.nxf);
  const double cx = cxg, cy = cyg, cz = czg;
  const int pcx = sod_cell_axis(cxg, K.xs[0], K.nx), pcy = sod_cell_axis(cyg, K.xs[1], K.nx),
            pcz = sod_cell_axis(czg, K.xs[2], K.nx);
  const float e2f = (float)K.eps2;
  unsigned long long sq = 0;
  double sf = 0.0;
  const NbrList L = nbr_list(K, B, pcx, pcy, pcz, ic, jc, kc);
  if (visits && lane == 0) *visits += L.total;
  // warp `part` of `nparts` takes every nparts-th step of 32 records
  for (unsigned t0 = 32 * part; t0 < L.total; t0 += 32 * nparts) {
    const unsigned t = t0 + (unsigned)lane;
    const unsigned q = L.at(t < L.total ? t : L.total - 1);
    if (t >= L.total) continue;
    const float4 nv = B.cube[q];
    if (__float_as_uint(nv.w) & PSOD_DEAD_BIT) continue;
    const float nxg = to_grid(nv.x, K.nxf), nyg = to_grid(nv.y, K.nxf), nzg = to_grid(nv.z, K.nxf);
    if (EXACT) {
      const double d2 = min_image_d2((double)nxg, (double)nyg, (double)nzg, cx, cy, cz, K.tx);
      if (d2 <= K.rmin2) {
        const double tt = ddiv(1.0, dsqrt(dadd(d2, K.eps2)));
        sq += (unsigned long long)__double2ll_rn(dmul(tt, 1099511627776.0));
      }
    } else {
      const float dx = mi_dx(nxg, cxg, K.nxf), dy = mi_dx(nyg, cyg, K.nxf), dz = mi_dx(nzg, czg, K.nxf);
      const float d2f = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
      bool in = d2f <= 0.99999f;
      if (!in && d2f <= 1.00001f) {
        const double d2 = min_image_d2((double)nxg, (double)nyg, (double)nzg, cx, cy, cz, K.tx);
        in = d2 <= K.rmin2;
      }
      if (in) sf += (double)rsqrtf(__fadd_rn(d2f, e2f));
    }
  }
  // the particle the run scan files under another cell
  if (K.has_quirk && lane == 0 && part == 0) {
    const int ax = (int)(K.quirk_listed % K.nx), ay = (int)((K.quirk_listed / K.nx) % K.nx),
              az = (int)(K.quirk_listed / ((unsigned)K.nx * K.nx));
    const bool listed_in_sel2 = in_sel2(K, ax, ay, az, ic, jc, kc);
    const bool seen = abs(pdiff(ax, pcx, K.nx)) <= 1 && abs(pdiff(ay, pcy, K.nx)) <= 1 &&
                      abs(pdiff(az, pcz, K.nx)) <= 1;
    if (listed_in_sel2 && !seen) {
      const float4 qv = B.cube[K.quirk_pos];
      if (!(__float_as_uint(qv.w) & PSOD_DEAD_BIT)) {
        const double d2 = min_image_d2((double)to_grid(qv.x, K.nxf), (double)to_grid(qv.y, K.nxf),
                                       (double)to_grid(qv.z, K.nxf), cx, cy, cz, K.tx);
        if (d2 <= K.rmin2) {
          const double tt = ddiv(1.0, dsqrt(dadd(d2, K.eps2)));
          if (EXACT) sq += (unsigned long long)__double2ll_rn(dmul(tt, 1099511627776.0));
          else sf += tt;
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    sq += __shfl_down_sync(0xffffffffu, sq, o);
    sf += __shfl_down_sync(0xffffffffu, sf, o);
  }
  sq_out = sq;
  sf_out = sf;
}

// Approximate refinement sums (fast path).  For a pair at FP32 offset
// (dx,dy,dz) the term is rsqrt(d2e) with d2e = dx^2+dy^2+dz^2+eps^2 formed by
// three FFMAs.  Each difference of two grid coordinates rounds at most once,
// and d2e adds three roundings of positive quantities, so d2e is within
// 3.6e-7 relative and the term, after rsqrtf, within 5e-7.  A pair is
// counted when d2e <= 1 + eps^2; near that edge d2e is within 3.6e-7 of the
// exact value, so the FP32 decision is the exact one whenever |d2e - (1 +
// eps^2)| >= EDGE_MARGIN (5.5 times that bound).  The lane tracks how close
// its pairs came to the edge and a tile with a pair within EDGE_MARGIN of it
// is redone with the exact FP64 inclusion test.  Terms are summed in two FP32
// partials of at most 16 positive terms (relative error below 1e-6) and the
// partials in FP64, so |S_approx - S| <= 2e-6 S < REF_TOL S.
// (REF_TOL bounds the gap that sends a candidate to the exact pass.)
constexpr float EDGE_MARGIN = 2e-6f;

// reciprocal square root of a normal positive float (d2e >= eps^2 here), one
// MUFU operation, relative error below 2^-22.9 (PTX rsqrt.approx)
__device__ __forceinline__ float rsqrt_pos(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// A warp's staged records, one array per coordinate (grid units), so that
// one 16-byte shared load gives one coordinate of four consecutive records.
struct __align__(16) RecTile {
  float x[64], y[64], z[64];
};

template <bool WRAPFREE>
__device__ __forceinline__ void pair_fast(float rx, float ry, float rz, float cx, float cy, float cz, float e2f,
                                          float limf, float nxf, float &acc, float &edge) {
  float dx, dy, dz;
  if (WRAPFREE) {
    dx = __fsub_rn(rx, cx);
    dy = __fsub_rn(ry, cy);
    dz = __fsub_rn(rz, cz);
  } else {
    dx = mi_dx(rx, cx, nxf);
    dy = mi_dx(ry, cy, nxf);
    dz = mi_dx(rz, cz, nxf);
  }
  const float d2e = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmaf_rn(dz, dz, e2f)));
  // e has the sign of d2e - limf (a rounded difference never changes sign)
  const float e = __fsub_rn(d2e, limf);
  edge = fminf(edge, fabsf(e));
  const float t = rsqrt_pos(d2e);
  asm("{\n\t.reg .pred p;\n\tsetp.le.f32 p, %1, 0f00000000;\n\t@p add.rn.f32 %0, %0, %2;\n\t}" : "+f"(acc) : "f"(e), "f"(t));
}

// a tile whose lane met a pair near the inclusion edge: the same FP32 terms,
// with the inclusion decided by the FP64 minimum-image distance
template <bool WRAPFREE>
__device__ __noinline__ double tile_terms_edge(const RecTile &tile, unsigned nt, float cx, float cy, float cz,
                                               float e2f, float nxf, double tx, double rmin2) {
  double sum = 0.0;
  for (unsigned j = 0; j < nt; j++) {
    const float rx = tile.x[j], ry = tile.y[j], rz = tile.z[j];
    float dx, dy, dz;
    if (WRAPFREE) {
      dx = __fsub_rn(rx, cx);
      dy = __fsub_rn(ry, cy);
      dz = __fsub_rn(rz, cz);
    } else {
      dx = mi_dx(rx, cx, nxf);
      dy = mi_dx(ry, cy, nxf);
      dz = mi_dx(rz, cz, nxf);
    }
    const float d2e = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmaf_rn(dz, dz, e2f)));
    if (min_image_d2((double)rx, (double)ry, (double)rz, (double)cx, (double)cy, (double)cz, tx) <= rmin2)
      sum += (double)rsqrt_pos(d2e);
  }
  return sum;
}

// sum of the terms of nt staged records; the tile is padded with far
// records up to a multiple of 8
template <bool WRAPFREE>
__device__ __forceinline__ double tile_terms(const RecTile &tile, unsigned nt, float cx, float cy, float cz,
                                             const SodConst &K) {
  const float e2f = (float)K.eps2, limf = (float)(1.0 + K.eps2);
  float p0 = 0.f, p1 = 0.f, edge = 1.f;
  for (unsigned j = 0; j < nt; j += 8) {
#pragma unroll
    for (int u = 0; u < 8; u += 2) {
      pair_fast<WRAPFREE>(tile.x[j + u], tile.y[j + u], tile.z[j + u], cx, cy, cz, e2f, limf, K.nxf, p0, edge);
      pair_fast<WRAPFREE>(tile.x[j + u + 1], tile.y[j + u + 1], tile.z[j + u + 1], cx, cy, cz, e2f, limf, K.nxf, p1,
                          edge);
    }
  }
  if (edge < EDGE_MARGIN) return tile_terms_edge<WRAPFREE>(tile, nt, cx, cy, cz, e2f, K.nxf, K.tx, K.rmin2);
  return (double)p0 + (double)p1;
}

// Packed FP32 pairs (the f32x2 operations of sm_100): two floats in one
// 64-bit register pair, both halves rounded exactly as the scalar operation.
__device__ __forceinline__ unsigned long long f2_pack(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2_unpack(unsigned long long r, float &lo, float &hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(r));
}
__device__ __forceinline__ unsigned long long f2_add(unsigned long long a, unsigned long long b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ unsigned long long f2_fma(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
// 1.0f where x <= 0, else 0.0f
__device__ __forceinline__ float le0(float x) {
  float m;
  asm("set.le.f32.f32 %0, %1, 0f00000000;" : "=f"(m) : "f"(x));
  return m;
}

// One candidate against records (j, j+1) held packed in (px, py, pz): the
// same operations as pair_fast on each half.  The accumulator's low half
// sums the even records and its high half the odd ones, as tile_terms does;
// t * 1.0 + acc rounds as acc + t, and t * 0.0 + acc is acc.
__device__ __forceinline__ void pair_packed(unsigned long long px, unsigned long long py, unsigned long long pz,
                                            unsigned long long ncx, unsigned long long ncy, unsigned long long ncz,
                                            unsigned long long e2, unsigned long long nlim, unsigned long long &acc,
                                            float &edge) {
  const unsigned long long dx = f2_add(px, ncx), dy = f2_add(py, ncy), dz = f2_add(pz, ncz);
  const unsigned long long d2e = f2_fma(dx, dx, f2_fma(dy, dy, f2_fma(dz, dz, e2)));
  const unsigned long long e = f2_add(d2e, nlim);
  float d0, d1, e0, e1;
  f2_unpack(d2e, d0, d1);
  f2_unpack(e, e0, e1);
  edge = fminf(edge, fminf(fabsf(e0), fabsf(e1)));
  acc = f2_fma(f2_pack(rsqrt_pos(d0), rsqrt_pos(d1)), f2_pack(le0(e0), le0(e1)), acc);
}

// the same for two candidates per lane: each staged record serves both.
// Wrap-free tiles use the packed form: four records a step, one 16-byte
// load per coordinate, two packed records per operation.
template <bool WRAPFREE>
__device__ __forceinline__ void tile_terms2(const RecTile &tile, unsigned nt, float ax, float ay, float az, float bx,
                                            float by, float bz, const SodConst &K, double &sa, double &sb) {
  const float e2f = (float)K.eps2, limf = (float)(1.0 + K.eps2);
  float ea = 1.f, eb = 1.f;
  double ra, rb;
  if (WRAPFREE) {
    const unsigned long long nax = f2_pack(-ax, -ax), nay = f2_pack(-ay, -ay), naz = f2_pack(-az, -az);
    const unsigned long long nbx = f2_pack(-bx, -bx), nby = f2_pack(-by, -by), nbz = f2_pack(-bz, -bz);
    const unsigned long long e2 = f2_pack(e2f, e2f), nlim = f2_pack(-limf, -limf);
    unsigned long long acca = f2_pack(0.f, 0.f), accb = f2_pack(0.f, 0.f);
    const ulonglong2 *tx = reinterpret_cast<const ulonglong2 *>(tile.x);
    const ulonglong2 *ty = reinterpret_cast<const ulonglong2 *>(tile.y);
    const ulonglong2 *tz = reinterpret_cast<const ulonglong2 *>(tile.z);
    for (unsigned j = 0; j < nt; j += 8) {
#pragma unroll
      for (unsigned u = 0; u < 8; u += 4) {
        const ulonglong2 X = tx[(j + u) >> 2], Y = ty[(j + u) >> 2], Z = tz[(j + u) >> 2];
        pair_packed(X.x, Y.x, Z.x, nax, nay, naz, e2, nlim, acca, ea);
        pair_packed(X.x, Y.x, Z.x, nbx, nby, nbz, e2, nlim, accb, eb);
        pair_packed(X.y, Y.y, Z.y, nax, nay, naz, e2, nlim, acca, ea);
        pair_packed(X.y, Y.y, Z.y, nbx, nby, nbz, e2, nlim, accb, eb);
      }
    }
    float a0, a1, b0, b1;
    f2_unpack(acca, a0, a1);
    f2_unpack(accb, b0, b1);
    ra = (double)a0 + (double)a1;
    rb = (double)b0 + (double)b1;
  } else {
    float a0 = 0.f, a1 = 0.f, b0 = 0.f, b1 = 0.f;
    for (unsigned j = 0; j < nt; j += 8) {
#pragma unroll
      for (int u = 0; u < 8; u += 2) {
        const float x0 = tile.x[j + u], y0 = tile.y[j + u], z0 = tile.z[j + u];
        const float x1 = tile.x[j + u + 1], y1 = tile.y[j + u + 1], z1 = tile.z[j + u + 1];
        pair_fast<false>(x0, y0, z0, ax, ay, az, e2f, limf, K.nxf, a0, ea);
        pair_fast<false>(x0, y0, z0, bx, by, bz, e2f, limf, K.nxf, b0, eb);
        pair_fast<false>(x1, y1, z1, ax, ay, az, e2f, limf, K.nxf, a1, ea);
        pair_fast<false>(x1, y1, z1, bx, by, bz, e2f, limf, K.nxf, b1, eb);
      }
    }
    ra = (double)a0 + (double)a1;
    rb = (double)b0 + (double)b1;
  }
  sa += ea < EDGE_MARGIN ? tile_terms_edge<WRAPFREE>(tile, nt, ax, ay, az, e2f, K.nxf, K.tx, K.rmin2) : ra;
  sb += eb < EDGE_MARGIN ? tile_terms_edge<WRAPFREE>(tile, nt, bx, by, bz, e2f, K.nxf, K.tx, K.rmin2) : rb;
}

// Work item: up to 64 candidates of one candidate cell (two per lane) against
// one chunk of RN_CHUNK records of the cell's 3x3x3 neighbourhood.  Records
// pass through a warp-private shared slice, 32 at a time, and every lane
// reads each one by broadcast; warps never wait on one another.  Partial
// sums of a candidate's neighbour chunks are added into cand_s.
//
// BOUND: the same items, giving each candidate c an upper bound U(c) of its
// sum.  Records nearer than sqrt(NEAR2) cells to the group's box are staged
// in tiles and summed exactly for every candidate (the pair pass's own
// loop); each farther record within reach adds k(d to the group's box),
// which no candidate's term exceeds, to every candidate of the group.  U is
// inflated by 1e-3, far above the FP32 error of the sums.  The second pair
// pass keeps only candidates whose bound reaches the seed's lower bound;
// the others cannot hold the argmax and their sums stay 0, below the select
// threshold.
//
// The near field is where a box bound is loose (a record inside the box
// counts 1/eps = 64 against a true term of a few), so it is summed exactly;
// the far field varies little across a compact group.  With the fine order
// of dense cells (a 64-candidate group spans ~0.1-0.3 cells in halo cores)
// a CPU model of NFW halos of 3e5-1e6 particles (c = 4-12) measured the
// near sums at 8-10 % of the unpruned pair work and the survivors at 2-15 %,
// against 37-61 % survivors with box bounds on sub-groups of 4.
constexpr unsigned ITEM_GRAB = 1;  // refinement items claimed per counter update
constexpr float NEAR2 = 0.09f;

template <bool BOUND>
__global__ void __launch_bounds__(256, 3) k_refine_warp(SodConst K, SodBufs B) {
  __shared__ RecTile s_tile[8];
  __shared__ unsigned s_rb[8][18], s_rp[8][19];
  __shared__ int s_nr[8], s_wf[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const bool phase1 = !BOUND && B.ref_phase == 1;
  const unsigned nready = min(*B.nready, B.cap_ready);
  const bool phase2 = !BOUND && B.ref_phase == 2;
  const unsigned *cpref = phase2 ? B.chunk_pref2 : B.chunk_pref;
  const unsigned nitems = phase1 ? B.top_pref[nready] : cpref[B.nitems_cells];
  // pair, slot and staged-record counts: per item in 32 bits, per warp in
  // shared memory (keeps 64-bit totals out of the registers)
  // (pair pass: also items taken)
  __shared__ unsigned long long s_count[8][4];
  if (lane < 4) s_count[w][lane] = 0;
  // items are claimed ITEM_GRAB at a time (one counter update per group of
  // consecutive items)
  unsigned grab = 0, grab_left = 0;
  while (true) {
    unsigned item = 0, ci = 0, rem = 0;
    if (lane == 0) {
      if (grab_left == 0) {
        grab = atomicAdd(BOUND ? B.work_bound : (B.ref_phase == 1 ? B.work_top : &B.work[1]), ITEM_GRAB);
        grab_left = ITEM_GRAB;
      }
      item = grab++;
      grab_left--;
      if (item < nitems && phase1) {
        unsigned lo = 0, hi = nready;  // last seed with top_pref <= item
        while (hi - lo > 1) {
          const unsigned mid = (lo + hi) >> 1;
          if (B.top_pref[mid] <= item) lo = mid;
          else hi = mid;
        }
        ci = B.top_ci[lo];
        rem = B.top_rem0[lo] + (item - B.top_pref[lo]);
      } else if (item < nitems) {
        unsigned lo = 0, hi = B.nitems_cells;  // last ci with cpref[ci] <= item
        while (hi - lo > 1) {
          const unsigned mid = (lo + hi) >> 1;
          if (cpref[mid] <= item) lo = mid;
          else hi = mid;
        }
        ci = lo;
        rem = item - cpref[lo];
      }
    }
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= nitems) break;
    ci = __shfl_sync(0xffffffffu, ci, 0);
    rem = __shfl_sync(0xffffffffu, rem, 0);
    const unsigned nch = B.cell_nch[ci];
    const unsigned chunk = rem / nch, nchunk = rem % nch;
    const unsigned slot = ci / 27, o = ci % 27;
    const bool bounded = B.bound_on && B.st_cn[slot] >= B.bound_min;
    if (BOUND && !bounded) continue;
    if (!BOUND && lane == 0) s_count[w][3]++;
    const SeedGeo g = seed_geo(K, B, B.ready[slot]);
    const int di = (int)(o / 9) - 1, dj = (int)((o / 3) % 3) - 1, dk = (int)(o % 3) - 1;
    const int cxc = wrapi(g.ic + di, K.nx), cyc = wrapi(g.jc + dj, K.nx), czc = wrapi(g.kc + dk, K.nx);
    const unsigned cnt = phase2 ? B.cnt2[ci] : B.cell_cnt[ci];
    // candidates k0 = 64*chunk + lane and k1 = k0 + 32 of the cell (phase 2:
    // of its surviving candidates); items of at most 32 candidates run one
    // per lane
    const unsigned k0 = chunk * 64u + (unsigned)lane, k1 = k0 + 32u;
    const bool two = cnt > chunk * 64u + 32u;
    const bool have = k0 < cnt, have1 = k1 < cnt;
    const unsigned coff = B.cell_off[ci];
    const unsigned q = phase2 ? (have ? B.cand_list[coff + k0] : 0u) : coff + k0;
    const unsigned q1 = phase2 ? (have1 ? B.cand_list[coff + k1] : 0u) : coff + k1;
    const unsigned cp = have ? B.cand_pos[q] : 0u, cp1 = have1 ? B.cand_pos[q1] : 0u;
    const bool quirk = have && K.has_quirk && cp == K.quirk_pos;
    const bool quirk1 = have1 && K.has_quirk && cp1 == K.quirk_pos;
    float cx = 0.f, cy = 0.f, cz = 0.f, bx = 1e18f, by = 1e18f, bz = 1e18f;
    if (have) {
      const float4 cv = B.cube[cp];
      cx = to_grid(cv.x, K.nxf);
      cy = to_grid(cv.y, K.nxf);
      cz = to_grid(cv.z, K.nxf);
    }
    if (have1) {
      const float4 cv = B.cube[cp1];
      bx = to_grid(cv.x, K.nxf);
      by = to_grid(cv.y, K.nxf);
      bz = to_grid(cv.z, K.nxf);
    }
    {
      // record runs of the 3x3x3 cells around the candidate cell: 9 rows of a
      // 3-cell x-run each (two runs when it wraps), lane r < 9 on row r; a
      // warp scan of the run counts and lengths places them in row order
      int np = 0;
      unsigned b0 = 0, l0 = 0, b1 = 0, l1 = 0;
      if (lane < 9) {
        const unsigned yy = (unsigned)wrapi(cyc + lane % 3 - 1, K.nx), zz = (unsigned)wrapi(czc + lane / 3 - 1, K.nx);
        const unsigned long long base = (unsigned long long)K.nx * (yy + (unsigned long long)K.nx * zz);
        const int x0 = cxc - 1, x1 = cxc + 1;
        int pa0, pb0, pa1 = 0, pb1 = -1;
        if (x0 < 0) { pa0 = x0 + K.nx; pb0 = K.nx - 1; pa1 = 0; pb1 = x1; np = 2; }
        else if (x1 >= K.nx) { pa0 = x0; pb0 = K.nx - 1; pa1 = 0; pb1 = x1 - K.nx; np = 2; }
        else { pa0 = x0; pb0 = x1; np = 1; }
        b0 = B.cs[base + (unsigned)pa0];
        l0 = B.cs[base + (unsigned)pb0 + 1] - b0;
        if (np == 2) {
          b1 = B.cs[base + (unsigned)pa1];
          l1 = B.cs[base + (unsigned)pb1 + 1] - b1;
        }
      }
      unsigned pc = (unsigned)np, len = l0 + l1;
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned tp = __shfl_up_sync(0xffffffffu, pc, o), tl = __shfl_up_sync(0xffffffffu, len, o);
        if (lane >= o) {
          pc += tp;
          len += tl;
        }
      }
      if (lane < 9) {
        const unsigned pf = pc - (unsigned)np, lf = len - (l0 + l1);
        s_rb[w][pf] = b0;
        s_rp[w][pf] = lf;
        if (np == 2) {
          s_rb[w][pf + 1] = b1;
          s_rp[w][pf + 1] = lf + l0;
        }
      }
      if (lane == 8) {
        s_rp[w][pc] = len;
        s_nr[w] = (int)pc;
      }
      if (lane == 0) {
        // the 3-cell coordinate window of each axis stays clear of the box edge
        auto clear = [&](int c, int a) {
          double s0 = (double)(c - 1) + K.xs[a];
          s0 -= K.tx * floor(s0 / K.tx);
          return s0 >= 1.0 && s0 + 3.0 <= K.tx - 1.0;
        };
        s_wf[w] = clear(cxc, 0) && clear(cyc, 1) && clear(czc, 2);
      }
    }
    __syncwarp();
    const int nr = s_nr[w];
    const unsigned total = s_rp[w][nr];
    const bool wf = s_wf[w];
    const bool active = have && !quirk, active1 = have1 && !quirk1;
    // bounding box of the item's candidates: records farther than 1 from it
    // in every direction meet no candidate (wrap-free items only)
    float lox = active ? cx : 3e38f, hix = active ? cx : -3e38f, loy = active ? cy : 3e38f,
          hiy = active ? cy : -3e38f, loz = active ? cz : 3e38f, hiz = active ? cz : -3e38f;
    if (active1) {
      lox = fminf(lox, bx);
      hix = fmaxf(hix, bx);
      loy = fminf(loy, by);
      hiy = fmaxf(hiy, by);
      loz = fminf(loz, bz);
      hiz = fmaxf(hiz, bz);
    }
    for (int o = 16; o > 0; o >>= 1) {
      lox = fminf(lox, __shfl_xor_sync(0xffffffffu, lox, o));
      hix = fmaxf(hix, __shfl_xor_sync(0xffffffffu, hix, o));
      loy = fminf(loy, __shfl_xor_sync(0xffffffffu, loy, o));
      hiy = fmaxf(hiy, __shfl_xor_sync(0xffffffffu, hiy, o));
      loz = fminf(loz, __shfl_xor_sync(0xffffffffu, loz, o));
      hiz = fmaxf(hiz, __shfl_xor_sync(0xffffffffu, hiz, o));
    }
    const bool any_active = lox <= hix;
    const unsigned r0 = nchunk * RN_CHUNK, r1 = any_active ? min(total, r0 + RN_CHUNK) : r0;
    const unsigned lt = (1u << lane) - 1u;
    double sum = 0.0, sum1 = 0.0;
    unsigned visits = 0, slots = 0, loaded = 0;
    // tile of 32 kept records: the pair tests of every candidate lane
    float uf = 0.f;  // BOUND: this lane's far records
    const float e2b = (float)K.eps2;
    auto consume = [&](unsigned nt) {
      // pad to a multiple of 8 with records far from every candidate
      if ((unsigned)lane < ((8u - (nt & 7u)) & 7u)) {
        s_tile[w].x[nt + lane] = 1e18f;
        s_tile[w].y[nt + lane] = 1e18f;
        s_tile[w].z[nt + lane] = 1e18f;
      }
      __syncwarp();
      if (two) {
        if (active || active1) {
          if (wf) tile_terms2<true>(s_tile[w], nt, cx, cy, cz, bx, by, bz, K, sum, sum1);
          else tile_terms2<false>(s_tile[w], nt, cx, cy, cz, bx, by, bz, K, sum, sum1);
        }
      } else if (active) {
        sum += wf ? tile_terms<true>(s_tile[w], nt, cx, cy, cz, K) : tile_terms<false>(s_tile[w], nt, cx, cy, cz, K);
      }
      if (lane == 0) {
        visits += min(64u, cnt - chunk * 64u) * nt;
        slots += (two ? 64u : 32u) * ((nt + 7u) & ~7u);
      }
      __syncwarp();
    };
    // Stage the chunk's records run by run, lanes on consecutive records of
    // one run.  Only alive records within reach of the candidates' box are
    // kept (warp-wide compaction into a 64-entry buffer); each full tile of
    // 32 is consumed at once and the overflow moves to the front, so no
    // record is loaded twice.
    unsigned fill = 0;
    int r = 0;
    while (r + 1 < nr && s_rp[w][r + 1] <= r0) r++;
    // (items near the periodic edge have no box filter: their bound is
    // infinite and they are not staged by the bound pass)
    for (unsigned pos = (BOUND && !wf) ? r1 : r0; pos < r1; r++) {
      const unsigned run_end = min(s_rp[w][r + 1], r1);
      const unsigned base = s_rb[w][r] - s_rp[w][r];  // cube slot = base + record number
      // SD steps of 32 records per pass: each lane issues its SD loads
      // before the first is used.  Both passes run best with one (measured
      // at 1024^3: with its exact near-field tiles the bound pass needs the
      // registers more than the loads in flight; four took it from 325 to
      // 603 ms through spills).
      constexpr int SD = 1;
      for (unsigned xs0 = pos; xs0 < run_end; xs0 += 32u * SD) {
        float4 vs[SD];
#pragma unroll
        for (int u = 0; u < SD; u++) {
          const unsigned x = xs0 + 32u * (unsigned)u + (unsigned)lane;
          vs[u] = x < run_end ? B.cube[base + x] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < SD; u++) {
          const unsigned x0 = xs0 + 32u * (unsigned)u;
          if (x0 >= run_end) break;  // warp-uniform
          const unsigned x = x0 + (unsigned)lane;
          bool keep = false;
          float4 rec = make_float4(0.f, 0.f, 0.f, 0.f);
          if (x < run_end) {
            const float4 v = vs[u];
            rec = make_float4(to_grid(v.x, K.nxf), to_grid(v.y, K.nxf), to_grid(v.z, K.nxf), 0.f);
            keep = !(__float_as_uint(v.w) & PSOD_DEAD_BIT);
            if (wf) {
              const float ex = fmaxf(fmaxf(lox - rec.x, rec.x - hix), 0.f), ey = fmaxf(fmaxf(loy - rec.y, rec.y - hiy), 0.f),
                          ez = fmaxf(fmaxf(loz - rec.z, rec.z - hiz), 0.f);
              const float db2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
              if (BOUND) {
                // far records add k(d to the group's box) to every
                // candidate here; near ones go to the tile for exact sums
                if (keep && db2 >= NEAR2 && db2 <= 1.0001f) uf += rsqrt_pos(db2 + e2b);
                keep = keep && db2 < NEAR2;
              } else {
                keep = keep && db2 <= 1.0001f;
              }
            }
          }
          const unsigned m = __ballot_sync(0xffffffffu, keep);
          if (keep) {  // fill < 32: index < 64
            const unsigned at = fill + __popc(m & lt);
            s_tile[w].x[at] = rec.x;
            s_tile[w].y[at] = rec.y;
            s_tile[w].z[at] = rec.z;
          }
          fill += (unsigned)__popc(m);
          if (!BOUND) loaded += min(32u, run_end - x0);
          if (fill >= 32u) {
            consume(32u);
            if ((unsigned)lane < fill - 32u) {
              s_tile[w].x[lane] = s_tile[w].x[32 + lane];
              s_tile[w].y[lane] = s_tile[w].y[32 + lane];
              s_tile[w].z[lane] = s_tile[w].z[32 + lane];
            }
            __syncwarp();
            fill -= 32u;
          }
        }
      }
      pos = run_end;
    }
    if (fill > 0) consume(fill);
    if (BOUND) {
      for (int sh = 16; sh > 0; sh >>= 1) uf += __shfl_xor_sync(0xffffffffu, uf, sh);
      // the particle the run scan files under another cell may add up to
      // 1/eps = 64 to any candidate's sum outside these runs; a candidate
      // that is the run scan's own quirk particle gets no bound (it always
      // stays in the exact pass), nor do items near the periodic edge
      const float extra = (K.has_quirk && nchunk == 0) ? 64.f : 0.f;
      const float inf = __int_as_float(0x7f800000);
      if (have) atomicAdd(&B.cand_u[q], (wf && !quirk) ? (float)((sum + (double)uf) * 1.001) + extra : inf);
      if (have1) atomicAdd(&B.cand_u[q1], (wf && !quirk1) ? (float)((sum1 + (double)uf) * 1.001) + extra : inf);
    }
    if (lane == 0) {
      s_count[w][0] += visits;
      s_count[w][1] += slots;
      s_count[w][2] += loaded;
    }
    if (BOUND) continue;
    if (nchunk == 0 && K.has_quirk && (active || active1)) {
      // the particle the run scan files under another cell: counted if that
      // cell is in x_sel2 but outside this candidate cell's 27 neighbours
      const int ax = (int)(K.quirk_listed % K.nx), ay = (int)((K.quirk_listed / K.nx) % K.nx),
                az = (int)(K.quirk_listed / ((unsigned)K.nx * K.nx));
      const bool listed_in_sel2 = in_sel2(K, ax, ay, az, g.ic, g.jc, g.kc);
      const bool seen = abs(pdiff(ax, cxc, K.nx)) <= 1 && abs(pdiff(ay, cyc, K.nx)) <= 1 && abs(pdiff(az, czc, K.nx)) <= 1;
      if (listed_in_sel2 && !seen) {
        const float4 qv = B.cube[K.quirk_pos];
        if (!(__float_as_uint(qv.w) & PSOD_DEAD_BIT)) {
          const double qx = to_grid(qv.x, K.nxf), qy = to_grid(qv.y, K.nxf), qz = to_grid(qv.z, K.nxf);
          if (active) {
            const double d2 = min_image_d2(qx, qy, qz, (double)cx, (double)cy, (double)cz, K.tx);
            if (d2 <= K.rmin2) sum += ddiv(1.0, dsqrt(dadd(d2, K.eps2)));
          }
          if (active1) {
            const double d2 = min_image_d2(qx, qy, qz, (double)bx, (double)by, (double)bz, K.tx);
            if (d2 <= K.rmin2) sum1 += ddiv(1.0, dsqrt(dadd(d2, K.eps2)));
          }
        }
      }
    }
    if (active && sum != 0.0) atomicAdd(&B.cand_s[q], sum);
    if (active1 && sum1 != 0.0) atomicAdd(&B.cand_s[q1], sum1);
  }
  if (lane == 0) {
    if (s_count[w][0]) atomicAdd(B.pairs, s_count[w][0]);
    if (s_count[w][1]) atomicAdd(B.pair_slots, s_count[w][1]);
    if (s_count[w][2]) atomicAdd(B.pair_slots + 1, s_count[w][2]);
    if (!BOUND && s_count[w][3]) atomicAdd(B.pair_slots + 6, s_count[w][3]);
  }
}

// ---------------------------------------------------------------------------
// phase 3: exact sums for the contenders and the argmax (main:1864-1875):
// largest sum wins, equal sums go to the first candidate in the reference's
// scan order (listed cell offset x-outer/z-inner, then input index)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void select_seed(const SodConst &K, const SodBufs &B, Smem &S, unsigned slot, unsigned rank) {
  if (!B.st_active[slot]) return;
  const unsigned off = B.st_coff[slot], n = B.st_cn[slot];
  if (n == 0) {
    if (threadIdx.x == 0) B.st_sbest[slot] = 0;
    return;
  }
  const SeedGeo g = seed_geo(K, B, rank);
  // max of the finite approximate sums (non-negative doubles order as their
  // bits); an infinite entry marks a candidate that always goes exact
  unsigned long long mb = 0, dummy = 0;
  for (unsigned k = threadIdx.x; k < n; k += TPB) {
    const unsigned long long b = dbits(B.cand_s[off + k]);
    if (b < 0x7ff0000000000000ull) mb = b > mb ? b : mb;
  }
  block_max_pair(S, mb, dummy);
  const double thr = dmul(bitsd(mb), 1.0 - 2.0 * REF_TOL);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned long long best_sq = 0, best_key = ~0ull;
  unsigned best_pos = 0xffffffffu;
  // Contenders (approximate sum within 2*REF_TOL of the maximum) get exact
  // sums.  Most seeds have one or two: then every warp of the CTA takes a
  // share of each contender's records (the int64 fixed-point sum is exact,
  // so the split leaves it unchanged); with more, a warp sums a contender.
  if (threadIdx.x == 0) S.nsel = 0;
  __syncthreads();
  for (unsigned k = threadIdx.x; k < n; k += TPB)
    if (B.cand_s[off + k] >= thr) {
      const unsigned j = atomicAdd(&S.nsel, 1u);
      if (j < SEL_SPLIT_MAX) S.sel[j] = k;
    }
  __syncthreads();
  const unsigned nsel = S.nsel;
  const bool split = nsel <= SEL_SPLIT_MAX;
  const unsigned nloop = split ? nsel : n;
  for (unsigned k = split ? 0u : (unsigned)w; k < nloop; k += split ? 1u : (unsigned)NWARP) {
    const unsigned ck = split ? S.sel[k] : k;
    if (!split && !(B.cand_s[off + ck] >= thr)) continue;  // cannot reach the maximum
    const unsigned cp = B.cand_pos[off + ck];
    unsigned long long sq;
    double sf;
    if (split) {
      refine_sum<true>(K, B, cp, g.ic, g.jc, g.kc, sq, sf, nullptr, (unsigned)w, NWARP);
      __syncthreads();
      if (lane == 0) S.red_u64[w] = sq;
      __syncthreads();
      sq = 0;
#pragma unroll
      for (int q = 0; q < NWARP; q++) sq += S.red_u64[q];
    } else {
      refine_sum<true>(K, B, cp, g.ic, g.jc, g.kc, sq, sf);
    }
    if (lane == 0 && (!split || w == 0)) {
      const float4 cv = B.cube[cp];
      const unsigned cw = __float_as_uint(cv.w);
      int lx, ly, lz;
      if (K.has_quirk && cp == K.quirk_pos) {
        lx = pdiff((int)(K.quirk_listed % K.nx), g.ic, K.nx);
        ly = pdiff((int)((K.quirk_listed / K.nx) % K.nx), g.jc, K.nx);
        lz = pdiff((int)(K.quirk_listed / ((unsigned)K.nx * K.nx)), g.kc, K.nx);
      } else {
        lx = pdiff(sod_cell_axis(to_grid(cv.x, K.nxf), K.xs[0], K.nx), g.ic, K.nx);
        ly = pdiff(sod_cell_axis(to_grid(cv.y, K.nxf), K.xs[1], K.nx), g.jc, K.nx);
        lz = pdiff(sod_cell_axis(to_grid(cv.z, K.nxf), K.xs[2], K.nx), g.kc, K.nx);
      }
      const unsigned o = (unsigned)(((lx + 1) * 3 + (ly + 1)) * 3 + (lz + 1));
      const unsigned long long key = ((unsigned long long)o << 32) | (cw & PSOD_IDX_MASK);
      if (sq > best_sq || (sq == best_sq && key < best_key)) {
        best_sq = sq;
        best_key = key;
        best_pos = cp;
      }
    }
  }
  unsigned long long a = best_sq, b = ~best_key;
  const unsigned long long pa = a, pb = b;
  block_max_pair(S, a, b);
  if (lane == 0 && best_pos != 0xffffffffu && pa == a && pb == b) B.st_centre[slot] = best_pos;
  if (threadIdx.x == 0) B.st_sbest[slot] = a;
}

// Learned-bracket features of a ready seed, once its centre is known:
//   0 log rho(seed)             1 log rho(centre)
//   2..6 log(1 + alive records) in the cubes of half-width 0..4 cells
//   7 log S(centre), the refinement sum   8 centre offset from the seed (cells)
//   9 log(1 + refinement candidates)
// In the learned mode only seeds with at least LEARN_MIN_CAND refinement
// candidates get features and a prediction: a halo whose stops lie beyond the
// first ball (1.5 cells, N above ~3000 at mean density one per cell) fills
// its 27 central cells with far more candidates.  The others are marked in
// column 15 and start at the batched mode's ball.  Collection for training
// covers every seed.
constexpr unsigned LEARN_MIN_CAND = 256;

// The FoF feature set (the configuration the task names for the learned
// seed), from the FoF group holding the seed particle:
//   0 log N_FoF      1..3 inertia axis ratios b/a, c/a, c/b
//   4 log rho(seed), the CIC peak overdensity
//   5..7 seed - FoF centre of mass (cells, minimum image)
//   8 R_FoF (cells)  9 RMS radius (cells)
// Targets: log(R_stop / R_FoF), the farthest threshold's stop over the FoF
// radius, and the centre offset |centre - seed| (cells); the first ball is
// exp(y0) * margin * R_FoF.  A seed outside the FoF halos (a group below
// Mmin) has no R_FoF: it gets no prediction and no sample.
__device__ __forceinline__ void fof_features(const SodConst &K, const SodBufs &B, unsigned slot, unsigned rank,
                                             float *f) {
  const unsigned i = B.seed_idx[rank];
  const unsigned code = B.fof_code[i];
  const SeedGeo g = seed_geo(K, B, rank);
  const float4 sv = B.cube[g.sp];
  for (int k = 0; k < 16; k++) f[k] = 0.f;
  f[4] = (float)log(fmax(B.rho[i], 1e-30));
  if (code & 0x80000000u) {
    f[0] = (float)log((double)max(code & 0x7fffffffu, 1u));
    f[1] = f[2] = f[3] = 1.f;
    f[15] = 1.f;
    return;
  }
  const float4 q = B.fof_feat[code];
  f[0] = (float)log((double)B.fof_mass[code]);
  f[1] = q.y;
  f[2] = q.z;
  f[3] = q.w;
  const double x[3] = {(double)sv.x, (double)sv.y, (double)sv.z};
  for (int a = 0; a < 3; a++) {
    double d = x[a] - B.fof_com[3ull * code + a];
    d -= floor(d + 0.5);  // minimum image in box units
    f[5 + a] = (float)(d * K.nxf);
  }
  f[8] = (float)(B.fof_rad[code] * K.nxf);
  f[9] = q.x * K.nxf;
  if (!(f[8] > 0.f)) f[15] = 1.f;
}

// the two training targets of a crossing sample; false: no sample
__device__ __forceinline__ bool learn_targets(const SodConst &K, const SodBufs &B, unsigned slot, double d2far,
                                              long long masse, unsigned seed_pos, unsigned centre_pos, float &t0,
                                              float &t1) {
  if (!B.learn_fof) {
    t0 = (float)(0.5 * log(fmax(d2far, 1e-12)));
    t1 = (float)log((double)masse);
    return true;
  }
  const float *f = B.st_feat + (size_t)slot * 16;
  if (f[15] != 0.f || !(f[8] > 0.f)) return false;
  const float4 a = B.cube[seed_pos], b = B.cube[centre_pos];
  const double d2 = min_image_d2((double)to_grid(a.x, K.nxf), (double)to_grid(a.y, K.nxf),
                                 (double)to_grid(a.z, K.nxf), (double)to_grid(b.x, K.nxf),
                                 (double)to_grid(b.y, K.nxf), (double)to_grid(b.z, K.nxf), K.tx);
  t0 = (float)(0.5 * log(fmax(d2far, 1e-12)) - log((double)f[8]));
  t1 = (float)sqrt(d2);
  return true;
}

// the learned first ball (cells) of a ready seed, 0 when none
__device__ __forceinline__ float learned_ball(const SodBufs &B, unsigned slot) {
  const float r = B.st_rb0[slot];
  return B.learn_fof ? r * B.st_feat[(size_t)slot * 16 + 8] : r;
}

__device__ __forceinline__ void seed_features(const SodConst &K, const SodBufs &B, Smem &S, unsigned slot, unsigned rank) {
  float *f = B.st_feat + (size_t)slot * 16;
  if (!B.st_active[slot] || (!B.learn_collect && B.st_cn[slot] < LEARN_MIN_CAND)) {
    if (threadIdx.x < 16) f[threadIdx.x] = threadIdx.x == 15 ? 1.f : 0.f;
    return;
  }
  if (B.learn_fof) {
    if (threadIdx.x == 0) fof_features(K, B, slot, rank, f);
    return;
  }
  const SeedGeo g = seed_geo(K, B, rank);
  unsigned s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0;
  if (B.alive_cnt) {
    for (int q = threadIdx.x; q < 729; q += TPB) {
      const int dx = q % 9 - 4, dy = (q / 9) % 9 - 4, dz = q / 81 - 4;
      const int d = max(abs(dx), max(abs(dy), abs(dz)));
      const unsigned cell = (unsigned)wrapi(g.ic + dx, K.nx) +
                            (unsigned)K.nx * ((unsigned)wrapi(g.jc + dy, K.nx) +
                                              (unsigned)K.nx * (unsigned)wrapi(g.kc + dz, K.nx));
      const unsigned v = B.alive_cnt[cell];
      s4 += v;
      if (d <= 3) s3 += v;
      if (d <= 2) s2 += v;
      if (d <= 1) s1 += v;
      if (d == 0) s0 += v;
    }
  }
  s0 = block_sum_u32(S, s0);
  s1 = block_sum_u32(S, s1);
  s2 = block_sum_u32(S, s2);
  s3 = block_sum_u32(S, s3);
  s4 = block_sum_u32(S, s4);
  if (threadIdx.x != 0) return;
  const float4 sv = B.cube[g.sp], cv = B.cube[B.st_centre[slot]];
  const unsigned ci = __float_as_uint(cv.w) & PSOD_IDX_MASK;
  const double d2 = min_image_d2((double)to_grid(sv.x, K.nxf), (double)to_grid(sv.y, K.nxf),
                                 (double)to_grid(sv.z, K.nxf), (double)to_grid(cv.x, K.nxf),
                                 (double)to_grid(cv.y, K.nxf), (double)to_grid(cv.z, K.nxf), K.tx);
  f[0] = (float)log(fmax(B.rho[B.seed_idx[rank]], 1e-30));
  f[1] = (float)log(fmax(B.rho[ci], 1e-30));
  f[2] = (float)log1p((double)s0);
  f[3] = (float)log1p((double)s1);
  f[4] = (float)log1p((double)s2);
  f[5] = (float)log1p((double)s3);
  f[6] = (float)log1p((double)s4);
  f[7] = (float)log(fmax((double)B.st_sbest[slot] * (1.0 / 1099511627776.0), 1e-30));
  f[8] = (float)sqrt(d2);
  f[9] = (float)log1p((double)B.st_cn[slot]);
  for (int k = PSOD_LEARN_FEATURES; k < 16; k++) f[k] = 0.f;
}

__global__ void __launch_bounds__(TPB) k_select(SodConst K, SodBufs B) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem &S = *reinterpret_cast<Smem *>(smem_raw);
  while (true) {
    const unsigned item = next_item(&B.work[2]);
    if (item >= min(*B.nready, B.cap_ready)) break;
    select_seed(K, B, S, item, B.ready[item]);
    if (B.learn_use || B.learn_collect) seed_features(K, B, S, item, B.ready[item]);
  }
}

// ---------------------------------------------------------------------------
// phase 4: crossing (main:2040-2100), profile (main:2103-2115), keep
// (main:2118-2141) and claims (main:2148-2166)
// ---------------------------------------------------------------------------
// exact alive count of the whole cube (the reference's npart_sel)
__device__ __forceinline__ unsigned count_alive_cube(const SodConst &K, const SodBufs &B, Smem &S, int ic, int jc, int kc) {
  unsigned cnt = 0;
  for_cube(K, B, ic, jc, kc, K.ncut, [&](unsigned p, float4 v) {
    if (!(__float_as_uint(v.w) & PSOD_DEAD_BIT)) cnt++;
  });
  return block_sum_u32(S, cnt);
}

// listed cell of a record for the alive-count bookkeeping
__device__ __forceinline__ unsigned listed_cell(const SodConst &K, unsigned p, float4 v) {
  if (K.has_quirk && p == K.quirk_pos) return K.quirk_listed;
  const unsigned i = (unsigned)sod_cell_axis(to_grid(v.x, K.nxf), K.xs[0], K.nx);
  const unsigned j = (unsigned)sod_cell_axis(to_grid(v.y, K.nxf), K.xs[1], K.nx);
  const unsigned k = (unsigned)sod_cell_axis(to_grid(v.z, K.nxf), K.xs[2], K.nx);
  return i + (unsigned)K.nx * (j + (unsigned)K.nx * k);
}

// Forward crossing search for threshold delta over a region that grows from
// rb0 (cells) until the stop is proven inside it, walking the region for
// every histogram level.  The plain mode starts from the whole cube.
// Returns the stop position; G is left at the region used.
__device__ __forceinline__ long long bracketed_stop(const SodConst &K, const SodBufs &B, Smem &S, Region &G, double rb0,
                                    unsigned &na, bool &na_known, double delta, double *d2stop) {
  double rb = rb0;
  while (true) {
    const bool full = !(rb > 0.0) || rb >= (double)K.ncut;
    G.rb = full ? -1.0 : rb;
    G.rb2 = full ? -1.0 : rb * rb;
    if (full && !na_known) {
      na = count_alive_cube(K, B, S, G.ic, G.jc, G.kc);
      na_known = true;
    }
    ball_hist0(K, B, S, G);
    if (threadIdx.x == 0) atomicAdd(B.cross_balls, 1ull);
    // inside a partial ball the cube's count is not reached: i < npart_sel holds
    const long long na_eff = full ? (long long)na : 0x7fffffffffffffffll;
    const long long i = radial_search<false>(K, B, S, G, na_eff, delta, 0, 0, d2stop);
    if (i != 0 || full) return i;
    rb *= 2.0;
  }
}

// Does some level-0 bucket of the ball (S.hist[0]) possibly hold the stop for
// threshold delta?  (the forward test of radial_search at level 0)
__device__ __forceinline__ bool stop_may_lie_inside(const SodConst &K, Smem &S, long long na, double delta) {
  hist_prefix(S, 0);
  const Level L = S.lev[0];
  int any = 0;
  for (int k = 0; k < NB / TPB; k++) {
    const int b = threadIdx.x * (NB / TPB) + k;
    const unsigned nb = S.hist[0][b];
    if (nb == 0) continue;
    unsigned long long lo, hi;
    bucket_range(L, 0, b, lo, hi);
    const long long ilo = (long long)S.pref[b] + 1, ihi = (long long)S.pref[b] + nb;
    if (ihi < 10) continue;
    const long long i0 = ilo < 10 ? 10 : ilo;
    const double hd = bitsd(hi);
    if (!(overdens(K, i0, hd) > delta && ihi < na && dsqrt(hd) < (double)K.ncut)) any = 1;
  }
  return block_max_i(S, any) > 0;
}

// Bucketed ball: grow the ball (one histogram walk per size) until every
// threshold's stop may lie inside it, then scatter its entries into a slice
// of the crossing buffer in level-0 bucket order (one more walk).  Returns
// the entry count, or -1 when the buffer has no room this round (the caller
// then walks the region for every search).
__device__ __forceinline__ long long bucket_ball(const SodConst &K, const SodBufs &B, Smem &S, Region &G, double rb0, unsigned &na,
                                 bool &na_known) {
  double rb = rb0;
  unsigned nball = 0;
  while (true) {
    const bool full = !(rb > 0.0) || rb >= (double)K.ncut;
    G.rb = full ? -1.0 : rb;
    G.rb2 = full ? -1.0 : rb * rb;
    if (full && !na_known) {
      na = count_alive_cube(K, B, S, G.ic, G.jc, G.kc);
      na_known = true;
    }
    nball = ball_hist0(K, B, S, G);
    if (threadIdx.x == 0) atomicAdd(B.cross_balls, 1ull);
    if (full) break;
    bool inside = stop_may_lie_inside(K, S, 0x7fffffffffffffffll, K.delta);
    for (int e = 0; e < K.ndx && inside; e++) inside = stop_may_lie_inside(K, S, 0x7fffffffffffffffll, K.dx_extra[e]);
    if (inside) break;
    rb *= 2.0;
  }
  if (threadIdx.x == 0) {
    const unsigned long long at = atomicAdd(B.xused, (unsigned long long)nball);
    S.xbase = (at + nball <= B.xcap) ? at : ~0ull;
  }
  __syncthreads();
  if (S.xbase == ~0ull) return -1;
  // cursors: the level-0 bucket starts
  hist_prefix(S, 0);
  unsigned *cur = S.hist[1];
  for (int k = threadIdx.x; k < NB; k += TPB) cur[k] = S.pref[k];
  __syncthreads();
  const unsigned long long base = S.xbase;
  RegionSrc{G}.each(K, B, [&](unsigned long long x, unsigned ix, unsigned p) {
    const unsigned slot = atomicAdd(&cur[bucket_of(S.lev[0], 0, x)], 1u);
    B.xkey[base + slot] = x;
    B.xidx[base + slot] = ix;
    B.xpos[base + slot] = p;
  });
  __syncthreads();
  return (long long)nball;
}

__device__ __forceinline__ void cross_seed(const SodConst &K, const SodBufs &B, Smem &S, unsigned slot, unsigned rank) {
  if (!B.st_active[slot]) return;
  const SeedGeo g = seed_geo(K, B, rank);
  unsigned na = B.st_na[slot];
  bool na_known = (B.mode == PSOD_MODE_PLAIN);
  const unsigned cpos = B.st_centre[slot];
  const float4 cvv = B.cube[cpos];
  Region G;
  G.ic = g.ic;
  G.jc = g.jc;
  G.kc = g.kc;
  G.xc = (double)to_grid(cvv.x, K.nxf);
  G.yc = (double)to_grid(cvv.y, K.nxf);
  G.zc = (double)to_grid(cvv.z, K.nxf);
  const double xc = G.xc, yc = G.yc, zc = G.zc;
  const unsigned cidx = __float_as_uint(cvv.w) & PSOD_IDX_MASK;
  double rb0 = (B.mode == PSOD_MODE_PLAIN) ? -1.0 : BALL0;
  if (B.learn_use) {
    // The learned radius only enlarges the first ball (up to the whole cube
    // at ncut).  A smaller ball saves records but not time: a pass costs
    // mostly its fixed walk and sort, and a miss adds a pass.  Starting at
    // or above BALL0, the doubling never needs more passes than from BALL0.
    const float r = learned_ball(B, slot);
    if (r > 0.f) rb0 = fmin(fmax((double)r, BALL0), (double)K.ncut);
  }

  // 3. crossing (main:2040-2100), in one of three forms:
  //  SMALL  the ball holds at most CAP alive records: sorted whole in shared
  //         memory; every later step reads the sorted list;
  //  BUF    a larger ball bucketed into the crossing buffer (bucket_ball):
  //         searches, profile and claims read bucket slices;
  //  REGION the buffer is full: every search level walks the region.
  enum { SMALL, BUF, REGION };
  int form = REGION;
  double d2stop = 0;
  long long istop = 0;
  unsigned nball = 0;
  {
    double rb = rb0;
    while (true) {
      const bool full = !(rb > 0.0) || rb >= (double)K.ncut;
      G.rb = full ? -1.0 : rb;
      G.rb2 = full ? -1.0 : rb * rb;
      if (full && !na_known) {
        na = count_alive_cube(K, B, S, G.ic, G.jc, G.kc);
        na_known = true;
      }
      const unsigned n = load_ball_sorted(K, B, S, G);
      if (threadIdx.x == 0) atomicAdd(B.cross_balls, 1ull);
      if (n > CAP) break;
      const long long i = sorted_stop(K, S, n, full ? (long long)na : 0x7fffffffffffffffll, K.delta);
      if (i != 0 || full) {
        istop = i;
        if (i > 0) d2stop = bitsd(S.skey[i - 1]);
        form = SMALL;
        nball = n;
        break;
      }
      rb *= 2.0;
    }
    if (form != SMALL) {
      // the ball that overflowed CAP is where the large forms start
      double rb = G.rb2 < 0.0 ? -1.0 : G.rb;
      while (true) {
        const long long nb = bucket_ball(K, B, S, G, rb, na, na_known);
        if (nb < 0) {
          form = REGION;
          istop = bracketed_stop(K, B, S, G, G.rb2 < 0.0 ? -1.0 : G.rb, na, na_known, K.delta, &d2stop);
          break;
        }
        form = BUF;
        nball = (unsigned)nb;
        const long long na_eff = G.rb2 < 0.0 ? (long long)na : 0x7fffffffffffffffll;
        istop = radial_search<true>(K, B, S, G, na_eff, K.delta, 0, 0, &d2stop);
        if (istop != 0 || G.rb2 < 0.0) break;
        rb = 2.0 * G.rb;  // no stop in this ball after all: a larger one
      }
    }
  }
  if (istop <= 0) {
    if (threadIdx.x == 0) record_error(B, rank, PSOD_ERR_STATE);
    return;
  }
  if (overdens(K, istop, d2stop) > K.delta) {  // main:2072
    if (threadIdx.x == 0) record_error(B, rank, PSOD_ERR_SELRADIUS);
    return;
  }
  const long long masse = istop - 1;
  const BufSrc ball_buf{S.xbase, S.xbase + nball};  // BUF: the whole ball
  {
    // algorithmic read volume: records of the cube cells that meet the ball
    // out to the stopping particle
    Region Gt = G;
    Gt.rb = dsqrt(d2stop);
    Gt.rb2 = d2stop;
    const unsigned nt = block_sum_u32(S, region_records(K, B, Gt));
    if (threadIdx.x == 0) atomicAdd(B.touch, (unsigned long long)nt);
  }
  // the masse-th element closes the member set (main:2090-2100, 2148)
  unsigned long long thr_key;
  unsigned thr_idx;
  if (form == SMALL) {
    thr_key = S.skey[masse - 1];
    thr_idx = S.sidx[masse - 1];
  } else {
    const int hk = S.res_k;
    const unsigned long long blo = S.res_lo;
    __syncthreads();
    if (hk > 0) {
      thr_key = S.skey[hk - 1];
      thr_idx = S.sidx[hk - 1];
    } else if (form == BUF) {
      max_below(K, B, S, ball_buf, blo, thr_key, thr_idx);
    } else {
      max_below(K, B, S, RegionSrc{G}, blo, thr_key, thr_idx);
    }
  }
  const double rayon = dsqrt(bitsd(thr_key));

  // seuil2 capture (main:2062-2069): last step i in [2, istop] above seuil2;
  // every such step lies inside the region that held the stop
  long long masse2 = 0;
  if (form == SMALL) {
    int best = -1;
    for (unsigned k = 1 + threadIdx.x; k < (unsigned)istop; k += TPB)
      if (overdens(K, (long long)k + 1, bitsd(S.skey[k])) > K.delta2) best = max(best, (int)k);
    best = block_max_i(S, best);
    if (best >= 0) masse2 = best + 1;
  } else {
    double dd;
    const long long na_eff = G.rb2 < 0.0 ? (long long)na : 0x7fffffffffffffffll;
    const long long i2 = form == BUF ? radial_search<true>(K, B, S, G, na_eff, K.delta2, 1, istop, &dd)
                                     : radial_search<false>(K, B, S, G, na_eff, K.delta2, 1, istop, &dd);
    if (i2 > 0) masse2 = i2;
  }
  // extra thresholds: the same stop rule, -1 when not crossed
  long long mext[PSOD_MAX_EXTRA_DELTA];
  double d2far = d2stop;  // farthest stop over the thresholds
  bool list_ok = form == SMALL;  // the sorted list still holds the ball
  bool buf_ok = form == BUF;     // S.hist[0] still describes the bucketed ball
  for (int e = 0; e < K.ndx; e++) {
    double dd = 0.0;
    long long ie = 0;
    const long long na_eff = G.rb2 < 0.0 ? (long long)na : 0x7fffffffffffffffll;
    if (list_ok) {
      ie = sorted_stop(K, S, nball, na_eff, K.dx_extra[e]);
      if (ie > 0) dd = bitsd(S.skey[ie - 1]);
    } else if (buf_ok) {
      ie = radial_search<true>(K, B, S, G, na_eff, K.dx_extra[e], 0, 0, &dd);
    }
    if ((!list_ok && !buf_ok) || (ie == 0 && G.rb2 >= 0.0)) {
      // the stop lies outside this ball (or nothing is cached): the region
      // search takes over from this ball's size; it rebuilds S.hist[0] and
      // the sort buffer for another ball
      list_ok = false;
      buf_ok = false;
      Region Ge = G;
      const double rbe = G.rb2 < 0.0 ? -1.0 : G.rb;
      ie = bracketed_stop(K, B, S, Ge, rbe, na, na_known, K.dx_extra[e], &dd);
    }
    mext[e] = (ie <= 0 || overdens(K, ie, dd) > K.dx_extra[e]) ? -1 : ie - 1;
    if (ie > 0) d2far = fmax(d2far, dd);
  }
  const bool small = form == SMALL && list_ok;
  // bracket bookkeeping: did the first ball hold every stop; samples for
  // training the bracket (this seed's features, log stop radius, log N)
  if (threadIdx.x == 0 && rb0 > 0.0) {
    atomicAdd(B.bracket_seeds, 1ull);
    if (d2far <= rb0 * rb0) atomicAdd(B.bracket_hits, 1ull);
  }
  if (threadIdx.x == 0 && B.learn_collect) {
    float t0, t1;
    if (learn_targets(K, B, slot, d2far, masse, g.sp, cpos, t0, t1)) {
      const unsigned long long q = atomicAdd(B.learn_n, 1ull);
      if (q < B.learn_cap) {
        for (int k = 0; k < PSOD_LEARN_FEATURES; k++) B.learn_x[q * PSOD_LEARN_FEATURES + k] = B.st_feat[slot * 16 + k];
        B.learn_t[2 * q] = t0;
        B.learn_t[2 * q + 1] = t1;
      }
    }
  }

  // keep test (main:2118-2120)
  const double amass = dmul((double)masse, K.munit);
  const bool keep = amass >= K.mmin && xc <= K.zmax[0] && xc > K.zmin[0] && yc <= K.zmax[1] &&
                    yc > K.zmin[1] && zc <= K.zmax[2] && zc > K.zmin[2];

  // 4a. profile (main:2103-2115): cumulative counts below each edge; the
  // region must hold every particle closer than the last edge
  if (keep) {
    for (int j = threadIdx.x; j < K.nbins; j += TPB) S.edges[j] = dmul(rayon, B.edge_fac[j]);
    for (int j = threadIdx.x; j <= K.nbins; j += TPB) S.phist[j] = 0;
    __syncthreads();
    const double emax = S.edges[K.nbins - 1];
    const bool ball_holds = G.rb2 < 0.0 || emax * (1.0 + 1e-9) < G.rb;
    auto bin_entry = [&](unsigned long long x) {
      const double r = dsqrt(bitsd(x));
      if (!(r < emax)) return;
      int lo = 0, hi = K.nbins - 1;  // first edge with r < edge
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (r < S.edges[mid]) hi = mid;
        else lo = mid + 1;
      }
      atomicAdd(&S.phist[lo], 1u);
    };
    if (small && ball_holds) {
      // every particle closer than the last edge is in the sorted list:
      // cumulative counts by binary search, one bin per thread
      for (int j = threadIdx.x; j < K.nbins; j += TPB) {
        unsigned lo = 0, hi = nball;  // first k with r_k >= edge
        while (lo < hi) {
          const unsigned mid = (lo + hi) >> 1;
          if (dsqrt(bitsd(S.skey[mid])) < S.edges[j]) lo = mid + 1;
          else hi = mid;
        }
        S.pref[j] = lo;
      }
      __syncthreads();
      for (int j = threadIdx.x; j < K.nbins; j += TPB) S.phist[j] = S.pref[j] - (j > 0 ? S.pref[j - 1] : 0u);
      __syncthreads();
    } else if (form == BUF && ball_holds) {
      ball_buf.each(K, B, [&](unsigned long long x, unsigned, unsigned) { bin_entry(x); });
      __syncthreads();
    } else {
      Region Gp = G;
      if (Gp.rb2 >= 0.0 && !ball_holds) {
        const double r = emax * 1.01 + 0.01;
        if (r >= (double)K.ncut) {
          Gp.rb = -1.0;
          Gp.rb2 = -1.0;
        } else {
          Gp.rb = r;
          Gp.rb2 = r * r;
        }
      }
      RegionSrc{Gp}.each(K, B, [&](unsigned long long x, unsigned, unsigned) { bin_entry(x); });
      __syncthreads();
    }
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
  auto claim = [&](unsigned long long x, unsigned ix, unsigned p) {
    if (!(x < thr_key || (x == thr_key && ix <= thr_idx))) return;
    const float4 v = B.cube[p];
    B.cube[p].w = __uint_as_float(__float_as_uint(v.w) | PSOD_DEAD_BIT);
    mark_resolved(B, B.bidx_of_cube[p]);
    if (B.alive_cnt) atomicSub(&B.alive_cnt[listed_cell(K, p, v)], 1u);
    const unsigned slot2 = atomicAdd(&S.claim_cnt, 1u);
    if (keep && slot2 < (unsigned)masse) {
      B.pool_key[pool_base + slot2] = x;
      B.pool_idx[pool_base + slot2] = ix;
    }
  };
  if (small) {
    // the first masse entries of the sorted list
    const unsigned *spos = small_pos(S);
    for (unsigned k = threadIdx.x; k < (unsigned)masse; k += TPB) {
      const unsigned p = spos[k];
      const float4 v = B.cube[p];
      B.cube[p].w = __uint_as_float(__float_as_uint(v.w) | PSOD_DEAD_BIT);
      mark_resolved(B, B.bidx_of_cube[p]);
      if (B.alive_cnt) atomicSub(&B.alive_cnt[listed_cell(K, p, v)], 1u);
      if (keep) {
        B.pool_key[pool_base + k] = S.skey[k];
        B.pool_idx[pool_base + k] = S.sidx[k];
      }
    }
    if (threadIdx.x == 0) S.claim_cnt = (unsigned)masse;
  } else if (form == BUF) {
    ball_buf.each(K, B, claim);
  } else {
    RegionSrc{G}.each(K, B, claim);
  }
  __syncthreads();
  if (S.claim_cnt != (unsigned)masse) {
    if (threadIdx.x == 0) record_error(B, rank, PSOD_ERR_STATE);
    return;
  }
  if (!keep) return;

  // 5. halo record
  if (threadIdx.x == 0) {
    atomicAdd(B.kept_members, (unsigned long long)masse);
    const unsigned long long hs = atomicAdd(B.nhalo, 1ull);
    B.h_rank[hs] = rank;
    B.h_id[hs] = B.ids[cidx];
    B.h_mass[hs] = masse;
    B.h_mass2[hs] = masse2;
    B.h_rdelta[hs] = rayon;
    B.h_center[3 * hs + 0] = __double2float_rn(ddiv(xc, K.scale));
    B.h_center[3 * hs + 1] = __double2float_rn(ddiv(yc, K.scale));
    B.h_center[3 * hs + 2] = __double2float_rn(ddiv(zc, K.scale));
    B.h_pool[hs] = pool_base | (small ? POOL_SORTED : 0ull);
    for (int e = 0; e < K.ndx; e++) B.h_mextra[hs * K.ndx + e] = mext[e];
    unsigned run = 0;
    for (int j = 0; j < K.nbins; j++) {
      run += S.phist[j];
      B.h_profile[hs * K.nbins + j] = run;
    }
  }
}

// ---------------------------------------------------------------------------
// Crossing search of small balls, one warp per seed.  Most seeds are small
// halos whose first ball holds a few hundred records; for them the CTA path's
// block barriers cost more than the work.  A warp loads the ball (alive
// records of the cells that meet it, d2 <= rb^2) into its own slice of
// shared memory, sorts it by (d2 bits, index) with warp-synchronous bitonic
// stages and runs the same searches as the CTA small path.  Everything is
// decided before the first write: a ball of more than WCAP records, a ball
// that reaches the whole cube, a threshold whose stop lies outside the ball
// or a profile that needs a wider region marks the seed for the CTA kernel
// (st_big), which then processes it from scratch in the same round.
// ---------------------------------------------------------------------------
constexpr int WCAP = 512;  // records per warp slice
struct WSlice {
  unsigned long long key[WCAP];
  unsigned idx[WCAP];
  unsigned pos[WCAP];
};

__device__ __forceinline__ int warp_min_i(int v) {
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ int warp_max_i(int v) {
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ unsigned warp_sum_u(unsigned v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// the bounded window of cube rows (dj, dk) that can meet a ball of radius rm
// around (ty, tz) (cell offsets relative to the seed cell centre)
__device__ __forceinline__ void ball_rows(const SodConst &K, double ty, double tz, double rm, int &jlo, int &jhi,
                                          int &klo, int &khi) {
  const int R = K.ncut;
  jlo = max(-R, (int)floor(ty - rm - 0.5));
  jhi = min(R, (int)ceil(ty + rm + 0.5));
  klo = max(-R, (int)floor(tz - rm - 0.5));
  khi = min(R, (int)ceil(tz + rm + 0.5));
}

// x-ranges of cube row (dj, dk) meeting the ball (the row rule of
// for_region); returns the number of cell-start ranges (0..2)
__device__ __forceinline__ int ball_row_ranges(const SodConst &K, const SodBufs &B, const Region &G, double tx,
                                               double ty, double tz, double rm2, int dj, int dk, unsigned rb_[2],
                                               unsigned re_[2]) {
  const int R = K.ncut;
  const double nxd = (double)K.nx;
  const double gy = cell_gap(ty, dj, nxd), gz = cell_gap(tz, dk, nxd);
  const double rem = __dsub_rn(__dsub_rn(rm2, __dmul_rn(gy, gy)), __dmul_rn(gz, gz));  // as region_records
  if (rem < 0.0) return 0;
  const double wx = sqrt(rem);
  int t0 = (int)ceil(tx - 0.5 - wx), t1 = (int)floor(tx + 0.5 + wx);
  t0 = max(t0, -R);
  t1 = min(t1, R);
  if (t0 > t1) return 0;
  const unsigned nx = (unsigned)K.nx;
  const unsigned jj = (unsigned)wrapi(G.jc + dj, K.nx), kk = (unsigned)wrapi(G.kc + dk, K.nx);
  const unsigned long long base = (unsigned long long)nx * (jj + (unsigned long long)nx * kk);
  const int x0 = G.ic + t0, x1 = G.ic + t1;
  int pa[2], pb[2], np;
  if (x0 < 0) {
    pa[0] = x0 + K.nx; pb[0] = K.nx - 1; pa[1] = 0; pb[1] = x1; np = 2;
    if (x1 < 0) { pa[0] = x0 + K.nx; pb[0] = x1 + K.nx; np = 1; }
  } else if (x1 >= K.nx) {
    pa[0] = x0; pb[0] = K.nx - 1; pa[1] = 0; pb[1] = x1 - K.nx; np = 2;
    if (x0 >= K.nx) { pa[0] = x0 - K.nx; pb[0] = x1 - K.nx; np = 1; }
  } else {
    pa[0] = x0; pb[0] = x1; np = 1;
  }
  for (int q = 0; q < np; q++) {
    rb_[q] = B.cs[base + (unsigned)pa[q]];
    re_[q] = B.cs[base + (unsigned)pb[q] + 1];
  }
  return np;
}

// load the ball's alive records into the slice, sorted; returns the count
// (above WCAP: overflow, slice unusable)
__device__ __forceinline__ unsigned warp_load_ball(const SodConst &K, const SodBufs &B, WSlice &W, const Region &G) {
  const int lane = threadIdx.x & 31;
  const double nxd = (double)K.nx;
  auto rel = [&](double x, int i, int a) {
    double d = x - ((double)i + K.xs[a] + 0.5);
    d = d - nxd * floor(d / nxd + 0.5);
    return d;
  };
  const double tx = rel(G.xc, G.ic, 0), ty = rel(G.yc, G.jc, 1), tz = rel(G.zc, G.kc, 2);
  const double rm = G.rb + 1e-3, rm2 = rm * rm;
  int jlo, jhi, klo, khi;
  ball_rows(K, ty, tz, rm, jlo, jhi, klo, khi);
  unsigned n = 0;
  for (int dk = klo; dk <= khi; dk++)
    for (int dj = jlo; dj <= jhi; dj++) {
      unsigned rb_[2], re_[2];
      const int np = ball_row_ranges(K, B, G, tx, ty, tz, rm2, dj, dk, rb_, re_);
      for (int q = 0; q < np; q++)
        for (unsigned p0 = rb_[q]; p0 < re_[q]; p0 += 32u) {
          const unsigned p = p0 + (unsigned)lane;
          double d2 = 0.0;
          float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
          bool in = false;
          if (p < re_[q]) {
            v = B.cube[p];
            in = region_d2(K, G, v, d2);
          }
          const unsigned m = __ballot_sync(0xffffffffu, in);
          const unsigned at = n + __popc(m & ((1u << lane) - 1u));
          if (in && at < WCAP) {
            W.key[at] = dbits(d2);
            W.idx[at] = __float_as_uint(v.w) & PSOD_IDX_MASK;
            W.pos[at] = p;
          }
          n += __popc(m);
        }
    }
  if (n > WCAP) return n;
  unsigned m2 = 32;
  while (m2 < n) m2 <<= 1;
  for (unsigned k = n + lane; k < m2; k += 32) {
    W.key[k] = ~0ull;
    W.idx[k] = 0xffffffffu;
  }
  __syncwarp();
  for (unsigned size = 2; size <= m2; size <<= 1)
    for (unsigned stride = size >> 1; stride > 0; stride >>= 1) {
      for (unsigned k = lane; k < m2 / 2; k += 32) {
        const unsigned a = 2 * k - (k & (stride - 1)), bb = a + stride;
        const bool up = ((a & size) == 0);
        const unsigned long long ka = W.key[a], kb = W.key[bb];
        const unsigned ia = W.idx[a], ib = W.idx[bb];
        const bool gt = (ka > kb) || (ka == kb && ia > ib);
        if (gt == up) {
          W.key[a] = kb;
          W.key[bb] = ka;
          W.idx[a] = ib;
          W.idx[bb] = ia;
          const unsigned pa = W.pos[a];
          W.pos[a] = W.pos[bb];
          W.pos[bb] = pa;
        }
      }
      __syncwarp();
    }
  return n;
}

// first 1-based i >= 10 of the sorted slice where the loop stops (partial
// ball: i < npart_sel always holds); 0 if none
__device__ __forceinline__ long long warp_stop(const SodConst &K, const WSlice &W, unsigned n, double delta) {
  const int lane = threadIdx.x & 31;
  int best = 0x7fffffff;
  for (unsigned k = 9 + lane; k < n; k += 32)
    if (!keeps_going(K, (long long)k + 1, bitsd(W.key[k]), 0x7fffffffffffffffll, delta)) {
      best = (int)k;
      break;
    }
  best = warp_min_i(best);
  return best == 0x7fffffff ? 0 : (long long)best + 1;
}

// records of the cube cells meeting the ball of radius rb (the touch count)
__device__ __forceinline__ unsigned warp_ball_records(const SodConst &K, const SodBufs &B, const Region &G) {
  const int lane = threadIdx.x & 31;
  const double nxd = (double)K.nx;
  auto rel = [&](double x, int i, int a) {
    double d = x - ((double)i + K.xs[a] + 0.5);
    d = d - nxd * floor(d / nxd + 0.5);
    return d;
  };
  const double tx = rel(G.xc, G.ic, 0), ty = rel(G.yc, G.jc, 1), tz = rel(G.zc, G.kc, 2);
  const double rm2 = G.rb * G.rb;
  int jlo, jhi, klo, khi;
  ball_rows(K, ty, tz, G.rb, jlo, jhi, klo, khi);
  const int ny = jhi - jlo + 1, nrow = ny * (khi - klo + 1);
  unsigned sum = 0;
  for (int row = lane; row < nrow; row += 32) {
    const int dj = jlo + row % ny, dk = klo + row / ny;
    unsigned rb_[2], re_[2];
    const int np = ball_row_ranges(K, B, G, tx, ty, tz, rm2, dj, dk, rb_, re_);
    for (int q = 0; q < np; q++) sum += re_[q] - rb_[q];
  }
  return warp_sum_u(sum);
}

__global__ void __launch_bounds__(256) k_cross_warp(SodConst K, SodBufs B) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  WSlice &W = reinterpret_cast<WSlice *>(smem_raw)[w];
  const unsigned slot = (unsigned)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (slot >= min(*B.nready, B.cap_ready) || !B.st_active[slot]) return;
  if (lane == 0) B.st_big[slot] = 0;
  const unsigned rank = B.ready[slot];
  const SeedGeo g = seed_geo(K, B, rank);
  const unsigned cpos = B.st_centre[slot];
  const float4 cvv = B.cube[cpos];
  Region G;
  G.ic = g.ic;
  G.jc = g.jc;
  G.kc = g.kc;
  G.xc = (double)to_grid(cvv.x, K.nxf);
  G.yc = (double)to_grid(cvv.y, K.nxf);
  G.zc = (double)to_grid(cvv.z, K.nxf);
  const double xc = G.xc, yc = G.yc, zc = G.zc;
  const unsigned cidx = __float_as_uint(cvv.w) & PSOD_IDX_MASK;
  double rb0 = BALL0;
  if (B.learn_use) {
    const float r = learned_ball(B, slot);
    if (r > 0.f) rb0 = fmin(fmax((double)r, BALL0), (double)K.ncut);
  }
  auto to_cta = [&]() {
    if (lane == 0) B.st_big[slot] = 1;
  };
  // 3. crossing (main:2040-2100) in growing partial balls
  unsigned passes = 0;
  unsigned long long records = 0;
  unsigned n = 0;
  long long istop = 0;
  double rb = rb0;
  while (true) {
    if (rb >= (double)K.ncut) {
      to_cta();
      return;
    }
    G.rb = rb;
    G.rb2 = rb * rb;
    n = warp_load_ball(K, B, W, G);
    passes++;
    records += n;
    if (n > WCAP) {
      to_cta();
      return;
    }
    istop = warp_stop(K, W, n, K.delta);
    if (istop != 0) break;
    rb *= 2.0;
  }
  const double d2stop = bitsd(W.key[istop - 1]);
  if (overdens(K, istop, d2stop) > K.delta) {  // main:2072
    if (lane == 0) record_error(B, rank, PSOD_ERR_SELRADIUS);
    return;
  }
  const long long masse = istop - 1;
  const unsigned long long thr_key = W.key[masse - 1];
  (void)thr_key;
  const double rayon = dsqrt(bitsd(W.key[masse - 1]));
  // seuil2 capture (main:2062-2069)
  long long masse2 = 0;
  {
    int best = -1;
    for (unsigned k = 1 + lane; k < (unsigned)istop; k += 32)
      if (overdens(K, (long long)k + 1, bitsd(W.key[k])) > K.delta2) best = max(best, (int)k);
    best = warp_max_i(best);
    if (best >= 0) masse2 = best + 1;
  }
  // extra thresholds: their stops must lie in this ball too
  long long mext[PSOD_MAX_EXTRA_DELTA];
  double d2far = d2stop;
  for (int e = 0; e < K.ndx; e++) {
    const long long ie = warp_stop(K, W, n, K.dx_extra[e]);
    if (ie == 0) {
      to_cta();
      return;
    }
    const double dd = bitsd(W.key[ie - 1]);
    mext[e] = overdens(K, ie, dd) > K.dx_extra[e] ? -1 : ie - 1;
    d2far = fmax(d2far, dd);
  }
  // keep test (main:2118-2120)
  const double amass = dmul((double)masse, K.munit);
  const bool keep = amass >= K.mmin && xc <= K.zmax[0] && xc > K.zmin[0] && yc <= K.zmax[1] &&
                    yc > K.zmin[1] && zc <= K.zmax[2] && zc > K.zmin[2];
  if (keep) {
    const double emax = dmul(rayon, B.edge_fac[K.nbins - 1]);
    if (!(emax * (1.0 + 1e-9) < G.rb)) {
      to_cta();
      return;
    }
  }
  // ---- committed: counters, bookkeeping, profile, claims, halo record ----
  {
    Region Gt = G;
    Gt.rb = dsqrt(d2stop);
    Gt.rb2 = d2stop;
    const unsigned nt = warp_ball_records(K, B, Gt);
    if (lane == 0) {
      atomicAdd(B.touch, (unsigned long long)nt);
      atomicAdd(B.cross_balls, (unsigned long long)passes);
      atomicAdd(B.cross_records, records);
      atomicAdd(B.bracket_seeds, 1ull);
      if (d2far <= rb0 * rb0) atomicAdd(B.bracket_hits, 1ull);
    }
  }
  if (lane == 0 && B.learn_collect) {
    float t0, t1;
    if (learn_targets(K, B, slot, d2far, masse, g.sp, cpos, t0, t1)) {
      const unsigned long long q = atomicAdd(B.learn_n, 1ull);
      if (q < B.learn_cap) {
        for (int k = 0; k < PSOD_LEARN_FEATURES; k++) B.learn_x[q * PSOD_LEARN_FEATURES + k] = B.st_feat[slot * 16 + k];
        B.learn_t[2 * q] = t0;
        B.learn_t[2 * q + 1] = t1;
      }
    }
  }
  unsigned long long pool_base = 0;
  unsigned long long hs = 0;
  if (lane == 0) {
    if (keep) {
      pool_base = atomicAdd(B.pool_used, (unsigned long long)masse);
      hs = atomicAdd(B.nhalo, 1ull);
      atomicAdd(B.kept_members, (unsigned long long)masse);
    }
  }
  pool_base = __shfl_sync(0xffffffffu, pool_base, 0);
  hs = __shfl_sync(0xffffffffu, hs, 0);
  // 4a. profile (main:2103-2115): cumulative counts below each edge
  if (keep) {
    for (int j = lane; j < K.nbins; j += 32) {
      const double edge = dmul(rayon, B.edge_fac[j]);
      unsigned lo = 0, hi = n;
      while (lo < hi) {
        const unsigned mid = (lo + hi) >> 1;
        if (dsqrt(bitsd(W.key[mid])) < edge) lo = mid + 1;
        else hi = mid;
      }
      B.h_profile[hs * K.nbins + j] = lo;
    }
  }
  // 4b. claims (main:2148-2166): the masse nearest die, kept or not
  for (unsigned k = lane; k < (unsigned)masse; k += 32) {
    const unsigned p = W.pos[k];
    const float4 v = B.cube[p];
    B.cube[p].w = __uint_as_float(__float_as_uint(v.w) | PSOD_DEAD_BIT);
    mark_resolved(B, B.bidx_of_cube[p]);
    if (B.alive_cnt) atomicSub(&B.alive_cnt[listed_cell(K, p, v)], 1u);
    if (keep) {
      B.pool_key[pool_base + k] = W.key[k];
      B.pool_idx[pool_base + k] = W.idx[k];
    }
  }
  // 5. halo record
  if (keep && lane == 0) {
    B.h_rank[hs] = rank;
    B.h_id[hs] = B.ids[cidx];
    B.h_mass[hs] = masse;
    B.h_mass2[hs] = masse2;
    B.h_rdelta[hs] = rayon;
    B.h_center[3 * hs + 0] = __double2float_rn(ddiv(xc, K.scale));
    B.h_center[3 * hs + 1] = __double2float_rn(ddiv(yc, K.scale));
    B.h_center[3 * hs + 2] = __double2float_rn(ddiv(zc, K.scale));
    B.h_pool[hs] = pool_base | POOL_SORTED;
    for (int e = 0; e < K.ndx; e++) B.h_mextra[hs * K.ndx + e] = mext[e];
  }
}

__global__ void __launch_bounds__(TPB) k_cross(SodConst K, SodBufs B) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem &S = *reinterpret_cast<Smem *>(smem_raw);
  while (true) {
    const unsigned item = next_item(&B.work[3]);
    if (item >= min(*B.nready, B.cap_ready)) break;
    if (B.st_big && !B.st_big[item]) continue;  // done by the warp pass
    cross_seed(K, B, S, item, B.ready[item]);
  }
}

// Lower bound of each ready seed's best refinement sum: the seed is one of
// its own candidates, so its sum (FP32 terms, relative error below 2e-6),
// deflated by 1e-3, is at most the maximum.  Warp per seed.
__global__ void k_seed_lower(SodConst K, SodBufs B) {
  const unsigned slot = (unsigned)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (slot >= min(*B.nready, B.cap_ready) || !B.st_active[slot] || B.st_cn[slot] < B.bound_min) return;
  const SeedGeo g = seed_geo(K, B, B.ready[slot]);
  unsigned long long sq = 0;
  double sf = 0.0;
  refine_sum<false>(K, B, g.sp, g.ic, g.jc, g.kc, sq, sf);
  if ((threadIdx.x & 31) == 0) atomicMax(&B.s_lmax[slot], __float_as_uint((float)(sf * 0.999)));
}

// The group holding the candidate with the largest finite upper bound, per
// bounded seed (warp per seed).  Its candidates are the likeliest to hold
// the maximum, so their sums, computed before all others, give a lower bound
// close to it.  Also the group's item range for the phase-1 pass.
__global__ void k_top_group(SodConst K, SodBufs B) {
  const unsigned slot = (unsigned)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (slot >= min(*B.nready, B.cap_ready)) return;
  float bu = -1.f;
  unsigned best = 0xffffffffu;
  if (B.bound_on && B.st_cn[slot] >= B.bound_min) {
    for (unsigned ci = slot * 27u; ci < slot * 27u + 27u; ci++) {
      const unsigned cnt = B.cell_cnt[ci], off = B.cell_off[ci], gp = B.group_pref[ci];
      for (unsigned k = (unsigned)lane; k < cnt; k += 32u) {
        const float u = B.cand_u[off + k];
        if (u <= 3e38f && u > bu) {  // an infinite bound (item near the periodic edge) says nothing
          bu = u;
          best = gp + k / 64u;
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const float ou = __shfl_xor_sync(0xffffffffu, bu, o);
    const unsigned og = __shfl_xor_sync(0xffffffffu, best, o);
    if (ou > bu || (ou == bu && og < best)) {
      bu = ou;
      best = og;
    }
  }
  if (lane != 0) return;
  B.s_top[slot] = best;
  unsigned n = 0;
  if (best != 0xffffffffu) {
    unsigned ci = slot * 27u;  // the candidate cell holding the group: last ci with group_pref[ci] <= best
    while (ci + 1 < slot * 27u + 27u && B.group_pref[ci + 1] <= best) ci++;
    n = B.cell_nch[ci];
    B.top_ci[slot] = ci;
    B.top_rem0[slot] = (best - B.group_pref[ci]) * n;
  }
  B.top_n[slot] = n;
}

// Lower bound from the top group's sums (warp per seed): every candidate's
// sum is at most the maximum, and the approximate sums are within 2e-6 of
// the exact ones, so max * (1 - 1e-5) is a lower bound of the maximum.
// Candidates that always go to the exact pass (infinite entries) are skipped.
__global__ void k_top_lower(SodConst K, SodBufs B) {
  const unsigned slot = (unsigned)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (slot >= min(*B.nready, B.cap_ready)) return;
  const unsigned top = B.s_top[slot];
  if (top == 0xffffffffu) return;
  unsigned ci = slot * 27u;  // the candidate cell holding the group: last ci with group_pref[ci] <= top
  while (ci + 1 < slot * 27u + 27u && B.group_pref[ci + 1] <= top) ci++;
  const unsigned chunk = top - B.group_pref[ci], cnt = B.cell_cnt[ci];
  double m = 0.0;
  for (unsigned k = chunk * 64u + (unsigned)lane; k < min(cnt, chunk * 64u + 64u); k += 32u) {
    const double v = B.cand_s[B.cell_off[ci] + k];
    if (v < 1e300 && v > m) m = v;
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0 && m > 0.0) atomicMax(&B.s_lmax[slot], __float_as_uint((float)(m * (1.0 - 1e-5))));
}

// The candidates the second pair pass must still sum (warp per candidate
// cell, stable): all of an unbounded seed's; of a bounded seed's, those
// outside the top group whose own bound reaches the seed's lower
// bound.  Their positions go to cand_list at the cell's candidate offset;
// the cell's phase-2 item count follows from their number.
__global__ void k_survivors(SodConst K, SodBufs B) {
  const unsigned ci = (unsigned)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (ci >= B.nitems_cells) return;
  const unsigned slot = ci / 27u, cnt = B.cell_cnt[ci], off = B.cell_off[ci], gp = B.group_pref[ci];
  const bool bounded = B.bound_on && B.st_cn[slot] >= B.bound_min;
  const float lmax = __uint_as_float(B.s_lmax[slot]);
  const unsigned top = B.s_top[slot];
  unsigned n2 = 0, gone = 0;
  for (unsigned k0 = 0; k0 < cnt; k0 += 32u) {
    const unsigned k = k0 + (unsigned)lane;
    bool keep = k < cnt;
    if (keep && bounded) {
      const unsigned grp = gp + k / 64u;
      keep = grp != top && B.cand_u[off + k] >= lmax;
      gone += (!keep && grp != top) ? 1u : 0u;
    }
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (keep) B.cand_list[off + n2 + __popc(m & ((1u << lane) - 1u))] = off + k;
    n2 += (unsigned)__popc(m);
  }
  for (int o = 16; o > 0; o >>= 1) gone += __shfl_xor_sync(0xffffffffu, gone, o);
  if (lane == 0) {
    B.cnt2[ci] = n2;
    B.chunks2[ci] = (n2 + 63u) / 64u * B.cell_nch[ci];
    if (gone) atomicAdd(B.cand_pruned, (unsigned long long)gone);
  }
}

// zero the per-candidate bounds of this round (candidate count on the device)
__global__ void k_zero_bounds(const unsigned *used, unsigned long long cap, float *u) {
  const unsigned n = (unsigned)min((unsigned long long)*used, cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) u[i] = 0.f;
}

__global__ void k_clear_dead(float4 *cube, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    float *w = &cube[i].w;
    *w = __uint_as_float(__float_as_uint(*w) & PSOD_IDX_MASK);
  }
}

__global__ void k_init_alive(const unsigned *cs, unsigned long long ncell, unsigned *alive) {
  unsigned long long c = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncell) alive[c] = cs[c + 1] - cs[c];
}

// ---------------------------------------------------------------------------
// scheduler
// ---------------------------------------------------------------------------
__global__ void k_seed_blocks(const unsigned *seed_idx, const unsigned *inv, const float4 *cube, long long nseed,
                              SodConst K, int bs, int nb, unsigned *block_of, unsigned *rank) {
  long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nseed) return;
  const float4 v = cube[inv[seed_idx[r]]];
  const int ci = sod_cell_axis(to_grid(v.x, K.nxf), K.xs[0], K.nx) / bs;
  const int cj = sod_cell_axis(to_grid(v.y, K.nxf), K.xs[1], K.nx) / bs;
  const int ck = sod_cell_axis(to_grid(v.z, K.nxf), K.xs[2], K.nx) / bs;
  block_of[r] = (unsigned)ci + (unsigned)nb * ((unsigned)cj + (unsigned)nb * (unsigned)ck);
  rank[r] = (unsigned)r;
}

__global__ void k_count_u32(const unsigned *keys, long long n, unsigned *count) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(&count[keys[i]], 1u);
}

// cube position of each seed in block order (saves an indirection per test)
__global__ void k_seed_pos(const unsigned *blist, long long nseed, const unsigned *seed_idx, const unsigned *inv,
                           unsigned *bpos) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nseed) bpos[i] = inv[seed_idx[blist[i]]];
}

__global__ void k_init_active(long long nblocks, const unsigned *bbegin, unsigned *head, unsigned *active,
                              unsigned *nactive) {
  long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblocks) return;
  head[b] = PSOD_INF_RANK;
  if (bbegin[b + 1] > bbegin[b]) active[atomicAdd(nactive, 1u)] = (unsigned)b;
}

// first index in [cur, end) whose resolved bit is clear, or end
__device__ __forceinline__ unsigned first_unresolved(const unsigned *res, unsigned cur, unsigned end) {
  while (cur < end) {
    const unsigned sh = cur & 31u;
    const unsigned zero = ~(res[cur >> 5] >> sh) & (0xffffffffu >> sh);
    if (zero) return min(end, cur + (unsigned)(__ffs(zero) - 1));
    cur = (cur | 31u) + 1u;
  }
  return end;
}

// One lane per active block: the head is the block's first unresolved
// (neither processed nor claimed) seed at or after its cursor, found in the
// resolved bitmap (32 seeds a word).  Blocks that still hold seeds go to
// next_active.
__global__ void k_heads(const unsigned *active, unsigned nactive, const unsigned *bbegin, unsigned *cursor,
                        const unsigned *blist, const unsigned *resolved, unsigned *head, unsigned *gmin,
                        unsigned *next_active, unsigned *n_next) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool have = i < nactive;
  unsigned b = 0, cur = 0, h = PSOD_INF_RANK;
  if (have) {
    b = active[i];
    const unsigned end = bbegin[b + 1];
    cur = first_unresolved(resolved, cursor[b], end);
    if (cur < end) h = blist[cur];
  }
  const bool live = have && h != PSOD_INF_RANK;
  const unsigned lm = __ballot_sync(0xffffffffu, live);
  unsigned base = 0;
  if (lane == 0 && lm) base = atomicAdd(n_next, (unsigned)__popc(lm));
  base = __shfl_sync(0xffffffffu, base, 0);
  unsigned hmin = live ? h : PSOD_INF_RANK;
  for (int o = 16; o > 0; o >>= 1) hmin = min(hmin, __shfl_xor_sync(0xffffffffu, hmin, o));
  if (gmin && lane == 0 && hmin != PSOD_INF_RANK) atomicMin(gmin, hmin);
  if (!have) return;
  cursor[b] = cur;
  head[b] = h;
  if (live) next_active[base + __popc(lm & ((1u << lane) - 1u))] = b;
}

// list positions of the seeds: by rank and by cube slot
__global__ void k_seed_index(const unsigned *blist, const unsigned *bpos, long long nseed, unsigned *bidx_of_rank,
                             unsigned *bidx_of_cube) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nseed) return;
  bidx_of_rank[blist[i]] = (unsigned)i;
  bidx_of_cube[bpos[i]] = (unsigned)i;
}

// periodic sliding minimum of radius rb along one axis of the nb^3 grid
__global__ void k_minfilter(const unsigned *in, unsigned *out, int nb, int axis, int rb) {
  const unsigned nbl = (unsigned)nb * nb * nb;
  const unsigned b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbl) return;
  int c[3] = {(int)(b % (unsigned)nb), (int)((b / (unsigned)nb) % (unsigned)nb), (int)(b / ((unsigned)nb * nb))};
  const int full = (2 * rb + 1 >= nb);
  const int lo = full ? 0 : -rb, hi = full ? nb - 1 : rb;
  unsigned m = PSOD_INF_RANK;
  const int c0 = c[axis];
  for (int d = lo; d <= hi; d++) {
    int v = full ? d : c0 + d;
    if (v < 0) v += nb;
    if (v >= nb) v -= nb;
    c[axis] = v;
    const unsigned x = in[(unsigned)c[0] + (unsigned)nb * ((unsigned)c[1] + (unsigned)nb * (unsigned)c[2])];
    m = x < m ? x : m;
  }
  out[b] = m;
}

__global__ void k_ready(const unsigned *active, const unsigned *nactive, const unsigned *head, const unsigned *filt,
                        unsigned quirk_rank, const unsigned *gmin, unsigned *ready, unsigned *nready, unsigned cap) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *nactive) return;
  const unsigned b = active[i];
  const unsigned h = head[b];
  if (h == PSOD_INF_RANK || h != filt[b]) return;
  // the particle filed under another cell waits until it is the global minimum
  if (h == quirk_rank && h != *gmin) return;
  // seeds past the cap stay unprocessed and are ready again next round
  const unsigned at = atomicAdd(nready, 1u);
  if (at < cap) ready[at] = h;
}

// seeds among [0, nseed) whose resolved bit is clear
__global__ void k_count_unresolved(const unsigned *resolved, long long nseed, unsigned long long *out) {
  const long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (w * 32 >= nseed) return;
  unsigned open = ~resolved[w];
  const long long left = nseed - w * 32;
  if (left < 32) open &= (1u << left) - 1u;
  if (open) atomicAdd(out, (unsigned long long)__popc(open));
}

// Per-round counters back to their start values in one launch: nready, the
// four work counters, the bound/top-group pass counters, the candidate and
// crossing-buffer allocators, the next active count, the bounded-seed count
// and the global minimum head.
__global__ void k_round_reset(unsigned *ctrs, unsigned long long *xused) {
  const int t = threadIdx.x;
  if (t < 5) ctrs[t] = 0;                   // nready, work[4]
  if (t == 5) ctrs[5] = 0xffffffffu;        // gmin
  if (t == 7) ctrs[7] = 0;                  // cand_used
  if (t >= 9 && t <= 13) ctrs[t] = 0;       // next active count, bound / top work, nbig, max candidates
  if (t == 0) *xused = 0ull;
}

// Readiness of an active block's head by a direct look at the heads of its
// window (Chebyshev radius rb blocks, periodic; the whole axis when the
// window covers it): ready when no head there is lower.  The same set as the
// separable min filter + k_ready, for rounds with few active blocks.  One
// warp per block: the lanes read the window's heads side by side.
__device__ __forceinline__ void ready_test_warp(unsigned b, const unsigned *head, int nb, int rb, unsigned quirk_rank,
                                                unsigned gmin, unsigned *ready, unsigned *nready, unsigned cap) {
  const int lane = threadIdx.x & 31;
  const unsigned h = head[b];
  if (h == PSOD_INF_RANK) return;
  const int bx = (int)(b % (unsigned)nb), by = (int)((b / (unsigned)nb) % (unsigned)nb),
            bz = (int)(b / ((unsigned)nb * nb));
  const bool full = 2 * rb + 1 >= nb;
  const int side = full ? nb : 2 * rb + 1, lo = full ? 0 : -rb;
  const int nwin = side * side * side;
  bool lower = false;
  for (int e = lane; e < nwin; e += 32) {
    const int dx = e % side + lo, dy = (e / side) % side + lo, dz = e / (side * side) + lo;
    int x = full ? dx : bx + dx, y = full ? dy : by + dy, z = full ? dz : bz + dz;
    if (x < 0) x += nb;
    if (x >= nb) x -= nb;
    if (y < 0) y += nb;
    if (y >= nb) y -= nb;
    if (z < 0) z += nb;
    if (z >= nb) z -= nb;
    lower |= head[(unsigned)x + (unsigned)nb * ((unsigned)y + (unsigned)nb * (unsigned)z)] < h;
  }
  if (__any_sync(0xffffffffu, lower)) return;
  // the particle filed under another cell waits until it is the global minimum
  if (h == quirk_rank && h != gmin) return;
  if (lane == 0) {
    const unsigned at = atomicAdd(nready, 1u);
    if (at < cap) ready[at] = h;
  }
}

__global__ void k_ready_direct(const unsigned *active, const unsigned *nactive, const unsigned *head, int nb, int rb,
                               unsigned quirk_rank, const unsigned *gmin, unsigned *ready, unsigned *nready,
                               unsigned cap) {
  const unsigned wi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (wi >= *nactive) return;
  ready_test_warp(active[wi], head, nb, rb, quirk_rank, *gmin, ready, nready, cap);
}

// ---------------------------------------------------------------------------
// Device tail loop.  Late rounds hold few, small seeds; run as separate
// launches with a host read per round they cost more in launch and
// synchronisation latency than in work.  One cooperative launch (all CTAs
// resident) runs round after round on the device: the heads of the active
// blocks, their readiness (the direct window test, or the separable min
// filter when many blocks are active) and every ready seed's preselect,
// refinement (FP32 approximate sums, a warp per candidate, then the exact
// sums of the contenders and the argmax, as k_select does) and crossing by
// one CTA, with a grid-wide barrier between the steps.  A seed with more
// than max_cand candidates waits; the launch ends after its round and the
// host runs the next rounds with the batched kernels.  The learned first
// ball is not used here (the crossing starts from BALL0; the halo table does
// not depend on it).  Every barrier wait is bounded: a wait that runs out
// records PSOD_ERR_TIMEOUT and every CTA leaves at its next barrier.
// ---------------------------------------------------------------------------
// Approximate refinement sums of the candidates of one candidate cell (o of
// the 27 around the seed) by one warp (the device tail loop): 32 candidates
// a pass, the alive records of the cell's 3x3x3 neighbourhood staged 32 at
// a time in the warp's tile and summed by tile_terms, i.e. the same FP32
// terms and partial sums as k_refine_warp and the same error bound.
__device__ __forceinline__ void tail_refine_cell(const SodConst &K, const SodBufs &B, unsigned slot, int o,
                                                 const SeedGeo &g, RecTile &T) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  auto clear = [&](int c, int a) {  // the 3-cell coordinate window stays clear of the box edge
    double s0 = (double)(c - 1) + K.xs[a];
    s0 -= K.tx * floor(s0 / K.tx);
    return s0 >= 1.0 && s0 + 3.0 <= K.tx - 1.0;
  };
  {
    const unsigned ci = slot * 27u + (unsigned)o;
    const unsigned cnt = B.cell_cnt[ci];
    if (cnt == 0) return;
    const unsigned coff = B.cell_off[ci];
    const int cxc = wrapi(g.ic + o / 9 - 1, K.nx), cyc = wrapi(g.jc + (o / 3) % 3 - 1, K.nx),
              czc = wrapi(g.kc + o % 3 - 1, K.nx);
    const bool wf = clear(cxc, 0) && clear(cyc, 1) && clear(czc, 2);
    const NbrList L = nbr_list(K, B, cxc, cyc, czc, g.ic, g.jc, g.kc);
    for (unsigned c0 = 0; c0 < cnt; c0 += 32) {
      const unsigned k = c0 + (unsigned)lane;
      const bool have = k < cnt;
      const unsigned cp = have ? B.cand_pos[coff + k] : 0u;
      const bool active = have && !(K.has_quirk && cp == K.quirk_pos);  // that one goes exact
      float cx = 1e18f, cy = 1e18f, cz = 1e18f;
      if (active) {
        const float4 cv = B.cube[cp];
        cx = to_grid(cv.x, K.nxf);
        cy = to_grid(cv.y, K.nxf);
        cz = to_grid(cv.z, K.nxf);
      }
      double sum = 0.0;
      unsigned fill = 0;
      for (unsigned t0 = 0; t0 < L.total; t0 += 32) {
        const unsigned t = t0 + (unsigned)lane;
        const unsigned q = L.at(t < L.total ? t : L.total - 1);
        bool keep = false;
        float rx = 0.f, ry = 0.f, rz = 0.f;
        if (t < L.total) {
          const float4 v = B.cube[q];
          keep = !(__float_as_uint(v.w) & PSOD_DEAD_BIT);
          rx = to_grid(v.x, K.nxf);
          ry = to_grid(v.y, K.nxf);
          rz = to_grid(v.z, K.nxf);
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {  // fill < 32: index < 64
          const unsigned at = fill + __popc(m & lt);
          T.x[at] = rx;
          T.y[at] = ry;
          T.z[at] = rz;
        }
        fill += (unsigned)__popc(m);
        __syncwarp();
        if (fill >= 32u) {
          if (active) sum += wf ? tile_terms<true>(T, 32u, cx, cy, cz, K) : tile_terms<false>(T, 32u, cx, cy, cz, K);
          __syncwarp();
          if ((unsigned)lane < fill - 32u) {
            T.x[lane] = T.x[32 + lane];
            T.y[lane] = T.y[32 + lane];
            T.z[lane] = T.z[32 + lane];
          }
          __syncwarp();
          fill -= 32u;
        }
      }
      if (fill > 0) {
        // pad to a multiple of 8 with records far from every candidate
        if ((unsigned)lane < ((8u - (fill & 7u)) & 7u)) {
          T.x[fill + lane] = 1e18f;
          T.y[fill + lane] = 1e18f;
          T.z[fill + lane] = 1e18f;
        }
        __syncwarp();
        if (active) sum += wf ? tile_terms<true>(T, fill, cx, cy, cz, K) : tile_terms<false>(T, fill, cx, cy, cz, K);
        __syncwarp();
      }
      if (active && K.has_quirk) {
        // the particle the run scan files under another cell: counted if
        // that cell is in x_sel2 but outside this candidate cell's 27
        // neighbours (as k_refine_warp does)
        const int ax = (int)(K.quirk_listed % K.nx), ay = (int)((K.quirk_listed / K.nx) % K.nx),
                  az = (int)(K.quirk_listed / ((unsigned)K.nx * K.nx));
        const bool listed_in_sel2 = in_sel2(K, ax, ay, az, g.ic, g.jc, g.kc);
        const bool seen = abs(pdiff(ax, cxc, K.nx)) <= 1 && abs(pdiff(ay, cyc, K.nx)) <= 1 && abs(pdiff(az, czc, K.nx)) <= 1;
        if (listed_in_sel2 && !seen) {
          const float4 qv = B.cube[K.quirk_pos];
          if (!(__float_as_uint(qv.w) & PSOD_DEAD_BIT)) {
            const double d2 = min_image_d2((double)to_grid(qv.x, K.nxf), (double)to_grid(qv.y, K.nxf),
                                           (double)to_grid(qv.z, K.nxf), (double)cx, (double)cy, (double)cz, K.tx);
            if (d2 <= K.rmin2) sum += ddiv(1.0, dsqrt(dadd(d2, K.eps2)));
          }
        }
      }
      if (active) B.cand_s[coff + k] = sum;
    }
  }
}

enum : unsigned { TAIL_RUNNING = 0, TAIL_DONE = 1, TAIL_DEFERRED = 2, TAIL_STALLED = 3, TAIL_TIMEOUT = 4 };

struct TailState {
  unsigned nact[2];       // active-block count of list act[p]
  unsigned nready[2];     // per round parity
  unsigned work[2];       // work counters of the seed steps: preselect,
  unsigned work_r[2];     // refinement (candidate cells), select, crossing
  unsigned work_s[2];
  unsigned work_c[2];
  unsigned cand_used[2];
  unsigned gmin[2];
  unsigned deferred;
  unsigned status;
  unsigned rounds;        // rounds completed by the launch
  unsigned parity;        // parity of the next round (its live list is act[parity])
  unsigned bar_count, bar_gen;
  unsigned long long xused[2];
  // time spent by the launch in each step (ns, block 0's clock, each step
  // up to the barrier that ends it)
  unsigned long long t_heads, t_ready, t_seeds;
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

constexpr unsigned long long BARRIER_POLLS = 1ull << 24;  // about 2-4 s of polling

// Grid-wide barrier of the cooperative launch (generation counting).  The
// fences make every write before the barrier visible to every read after
// it.  Returns false when the wait ran out or another CTA's did.
__device__ bool grid_barrier(TailState *ts) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile unsigned *gen = &ts->bar_gen;
    volatile unsigned *status = &ts->status;
    const unsigned g0 = *gen;
    __threadfence();
    if (atomicAdd(&ts->bar_count, 1u) == gridDim.x - 1) {
      ts->bar_count = 0;
      __threadfence();
      atomicAdd(&ts->bar_gen, 1u);
    } else {
      unsigned long long polls = 0;
      while (*gen == g0) {
        if (*status == TAIL_TIMEOUT || ++polls > BARRIER_POLLS) {
          ok = 0;
          break;
        }
        __nanosleep(128);
      }
      if (!ok) atomicExch(&ts->status, TAIL_TIMEOUT);
    }
    __threadfence();
    if (*status == TAIL_TIMEOUT) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// value written by another CTA before the last barrier
__device__ __forceinline__ unsigned ld_shared_state(const unsigned *p) { return *(volatile const unsigned *)p; }

__global__ void __launch_bounds__(TPB) k_tail_rounds(SodConst K, SodBufs B, TailState *ts, unsigned *act0,
                                                    unsigned *act1, const unsigned *bbegin, unsigned *cursor,
                                                    const unsigned *blist, unsigned *head, int nb, int rb,
                                                    unsigned quirk_rank, unsigned *ready) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem &S = *reinterpret_cast<Smem *>(smem_raw);
  __shared__ unsigned s_cnt, s_next, s_nready;
  __shared__ RecTile t_tiles[NWARP];
  const unsigned gtid = blockIdx.x * blockDim.x + threadIdx.x, gthreads = gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  // the round parity: every CTA flips its own copy once per round
  unsigned q = ts->parity;
  while (true) {
    // this round's active count was written (heads of the previous round,
    // or the host) before the last barrier
    if (threadIdx.x == 0) s_cnt = ld_shared_state(&ts->nact[q]);
    __syncthreads();
    const unsigned cnt = s_cnt;
    const bool timer = blockIdx.x == 0 && threadIdx.x == 0;
    unsigned long long tk = timer ? global_ns() : 0ull;
    unsigned *cur = q ? act1 : act0, *nxt = q ? act0 : act1;
    // heads (k_heads): warp-uniform strides over the active list
    for (unsigned base = gtid - (unsigned)lane; base < cnt; base += gthreads) {
      const unsigned i = base + (unsigned)lane;
      const bool have = i < cnt;
      unsigned b = 0, h = PSOD_INF_RANK, cu = 0;
      if (have) {
        b = cur[i];
        const unsigned end = bbegin[b + 1];
        cu = first_unresolved(B.resolved, cursor[b], end);
        if (cu < end) h = blist[cu];
      }
      const bool live = have && h != PSOD_INF_RANK;
      const unsigned lm = __ballot_sync(0xffffffffu, live);
      unsigned at = 0;
      if (lane == 0 && lm) at = atomicAdd(&ts->nact[q ^ 1u], (unsigned)__popc(lm));
      at = __shfl_sync(0xffffffffu, at, 0);
      unsigned hmin = live ? h : PSOD_INF_RANK;
      for (int o = 16; o > 0; o >>= 1) hmin = min(hmin, __shfl_xor_sync(0xffffffffu, hmin, o));
      if (lane == 0 && hmin != PSOD_INF_RANK) atomicMin(&ts->gmin[q], hmin);
      if (have) {
        cursor[b] = cu;
        head[b] = h;
        if (live) nxt[at + __popc(lm & ((1u << lane) - 1u))] = b;
      }
    }
    if (!grid_barrier(ts)) return;
    if (timer) {
      const unsigned long long now = global_ns();
      ts->t_heads += now - tk;
      tk = now;
    }
    // the next round's counters (parity q^1) are free now: reset them
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ts->nact[q] = 0;
      ts->gmin[q ^ 1u] = PSOD_INF_RANK;
      ts->nready[q ^ 1u] = 0;
      ts->work[q ^ 1u] = 0;
      ts->work_r[q ^ 1u] = 0;
      ts->work_s[q ^ 1u] = 0;
      ts->work_c[q ^ 1u] = 0;
      ts->cand_used[q ^ 1u] = 0;
      ts->xused[q ^ 1u] = 0;
    }
    if (threadIdx.x == 0) s_next = ld_shared_state(&ts->nact[q ^ 1u]);
    __syncthreads();
    const unsigned next = s_next;
    const unsigned gmin = ld_shared_state(&ts->gmin[q]);
    // readiness: the direct window test (the launch is used only while few
    // blocks are active), a warp per active block
    for (unsigned wi = gtid >> 5; wi < next; wi += gthreads >> 5)
      ready_test_warp(nxt[wi], head, nb, rb, quirk_rank, gmin, ready, &ts->nready[q], B.cap_ready);
    if (!grid_barrier(ts)) return;
    if (timer) {
      const unsigned long long now = global_ns();
      ts->t_ready += now - tk;
      tk = now;
    }
    if (threadIdx.x == 0) s_nready = ld_shared_state(&ts->nready[q]);
    __syncthreads();
    const unsigned nready = min(s_nready, B.cap_ready);
    if (nready == 0) {
      // the lowest-ranked unresolved seed is always ready: an empty round
      // with active blocks left is a scheduler fault
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        ts->status = next > 0 ? TAIL_STALLED : TAIL_DONE;
        ts->parity = q ^ 1u;
      }
      return;
    }
    // the round's seeds, a CTA each
    SodBufs Br = B;
    Br.nready = &ts->nready[q];
    Br.cand_used = &ts->cand_used[q];
    Br.xused = &ts->xused[q];
    Br.deferred = &ts->deferred;
    Br.maxcand = nullptr;
    Br.learn_use = 0;
    // preselect: a CTA per seed
    while (true) {
      const unsigned item = next_item(&ts->work[q]);
      if (item >= nready) break;
      prep_seed(K, Br, S, item, B.ready[item]);
    }
    if (!grid_barrier(ts)) return;
    // refinement: a warp per (seed, candidate cell) over the whole grid
    {
      const int w = threadIdx.x >> 5;
      while (true) {
        unsigned it = 0;
        if (lane == 0) it = atomicAdd(&ts->work_r[q], 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= nready * 27u) break;
        const unsigned slot = it / 27u;
        if (!Br.st_active[slot]) continue;
        tail_refine_cell(K, Br, slot, (int)(it % 27u), seed_geo(K, Br, B.ready[slot]), t_tiles[w]);
      }
    }
    if (!grid_barrier(ts)) return;
    // exact sums of the contenders and the argmax: a CTA per seed
    while (true) {
      const unsigned item = next_item(&ts->work_s[q]);
      if (item >= nready) break;
      select_seed(K, Br, S, item, B.ready[item]);
      if (Br.learn_collect) seed_features(K, Br, S, item, B.ready[item]);
    }
    if (!grid_barrier(ts)) return;
    // crossing, profile and claims: a CTA per seed
    while (true) {
      const unsigned item = next_item(&ts->work_c[q]);
      if (item >= nready) break;
      cross_seed(K, Br, S, item, B.ready[item]);
    }
    if (!grid_barrier(ts)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ts->rounds++;
      ts->parity = q ^ 1u;
      ts->t_seeds += global_ns() - tk;
    }
    if (threadIdx.x == 0) s_nready = ld_shared_state(&ts->deferred);
    __syncthreads();
    if (s_nready) {
      if (blockIdx.x == 0 && threadIdx.x == 0) ts->status = TAIL_DEFERRED;
      return;
    }
    q ^= 1u;
  }
}

__global__ void k_tail_init(TailState *ts, unsigned n_active) {
  ts->nact[0] = n_active;
  ts->nact[1] = 0;
  ts->nready[0] = ts->nready[1] = 0;
  ts->work[0] = ts->work[1] = 0;
  ts->work_r[0] = ts->work_r[1] = 0;
  ts->work_s[0] = ts->work_s[1] = 0;
  ts->work_c[0] = ts->work_c[1] = 0;
  ts->cand_used[0] = ts->cand_used[1] = 0;
  ts->gmin[0] = ts->gmin[1] = PSOD_INF_RANK;
  ts->xused[0] = ts->xused[1] = 0;
  ts->deferred = 0;
  ts->status = TAIL_RUNNING;
  ts->rounds = 0;
  ts->parity = 0;
  ts->bar_count = 0;
  ts->bar_gen = 0;
  ts->t_heads = ts->t_ready = ts->t_seeds = 0;
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

__global__ void k_gather_widen(const unsigned *src, const unsigned *order, long long n, int width, long long *dst) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * width) return;
  long long h = i / width, k = i % width;
  dst[i] = (long long)src[(long long)order[h] * width + k];
}

__global__ void k_mass_u32(const long long *mass, long long n, unsigned *out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (unsigned)mass[i];
}

__global__ void k_widen(const unsigned *in, long long n, long long *out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (long long)in[i];
}

constexpr int MS_CHUNK = 2048;

__device__ __forceinline__ bool pair_less(unsigned long long ka, unsigned ia, unsigned long long kb, unsigned ib) {
  return ka < kb || (ka == kb && ia < ib);
}

// Members leave in (d2 bits, input index) order, written as input indices at
// the halo's output offset.  Halos claimed from a sorted list are copied;
// the others hold members in claim order.  Those of at most MS_CHUNK members
// are sorted by one CTA each in shared memory (k_member_sort); the larger
// ones, a few thousand halos holding most of the members, are sorted
// together by one device-wide radix sort on (halo, top 32 bits of d2)
// (k_big_keys), after which the rare runs of equal truncated keys are put
// in full-key order (k_big_ties) and scattered to the output (k_big_out).
__global__ void __launch_bounds__(256) k_member_sort(const unsigned *order, long long nh, const unsigned long long *h_pool,
                                                     const long long *h_mass_sorted, const unsigned *moff,
                                                     const unsigned long long *pkey, const unsigned *pidx,
                                                     unsigned *m_index) {
  __shared__ unsigned long long sk[MS_CHUNK];
  __shared__ unsigned si[MS_CHUNK];
  for (long long h = blockIdx.x; h < nh; h += gridDim.x) {
    const unsigned slot = order[h];
    const unsigned long long base = h_pool[slot] & ~POOL_SORTED;
    const unsigned m = (unsigned)h_mass_sorted[h];
    const unsigned o = moff[h];
    if (h_pool[slot] & POOL_SORTED) {
      // claimed from a sorted list: already in (d2, index) order
      for (unsigned k = threadIdx.x; k < m; k += blockDim.x) m_index[o + k] = pidx[base + k];
      continue;
    }
    if (m > (unsigned)MS_CHUNK) continue;  // the device-wide pass
    unsigned p2 = 1;
    while (p2 < m) p2 <<= 1;
    for (unsigned k = threadIdx.x; k < p2; k += blockDim.x) {
      sk[k] = k < m ? pkey[base + k] : ~0ull;
      si[k] = k < m ? pidx[base + k] : 0xffffffffu;
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
        bitonic_stage_sync(size, stride, p2);
      }
    }
    for (unsigned k = threadIdx.x; k < m; k += blockDim.x) m_index[o + k] = si[k];
    __syncthreads();
  }
}

// big[h] = 1 for a halo (output order) claimed unsorted with more than
// MS_CHUNK members, msz[h] its member count there (0 otherwise); both are
// scanned in place afterwards
__global__ void k_big_flags(const unsigned *order, long long nh, const unsigned long long *h_pool,
                            const long long *h_mass_sorted, unsigned *big, unsigned *msz) {
  const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= nh) return;
  const unsigned m = (unsigned)h_mass_sorted[h];
  const bool b = !(h_pool[order[h]] & POOL_SORTED) && m > (unsigned)MS_CHUNK;
  big[h] = b ? 1u : 0u;
  msz[h] = b ? m : 0u;
}

// the large halos as segments s = 0 .. nbig-1 in output order: their halo,
// start in the concatenated key array (seg_start[nbig] = total) and pool base
__global__ void k_big_list(const unsigned *order, long long nh, const unsigned long long *h_pool,
                           const unsigned *big_scan, const unsigned *msz_scan, unsigned *seg_h, unsigned *seg_start,
                           unsigned *seg_base) {
  const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= nh) return;
  if (h == 0) seg_start[big_scan[nh]] = msz_scan[nh];
  if (big_scan[h + 1] == big_scan[h]) return;
  const unsigned s = big_scan[h];
  seg_h[s] = (unsigned)h;
  seg_start[s] = msz_scan[h];
  seg_base[s] = (unsigned)(h_pool[order[h]] & ~POOL_SORTED);
}

// key j of the concatenated segments: (segment << 32) | d2 bits >> 31 (the
// top 32 bits below the sign, monotone in d2 >= 0); value = pool position
__global__ void k_big_keys(const unsigned *seg_start, unsigned nbig, const unsigned *seg_base,
                           const unsigned long long *pool_key, unsigned ntot, unsigned long long *key,
                           unsigned *val) {
  const unsigned j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ntot) return;
  unsigned lo = 0, hi = nbig;  // seg_start[lo] <= j < seg_start[hi]
  while (hi - lo > 1) {
    const unsigned mid = (lo + hi) >> 1;
    if (seg_start[mid] <= j) lo = mid;
    else hi = mid;
  }
  const unsigned p = seg_base[lo] + (j - seg_start[lo]);
  key[j] = ((unsigned long long)lo << 32) | (unsigned)(pool_key[p] >> 31);
  val[j] = p;
}

// after the radix sort: each run of equal keys (same segment, d2 equal in
// its top 32 bits) is put in (full d2 bits, input index) order by the thread
// at its start; runs are short (pairs of members within 2^-21 in d2)
__global__ void k_big_ties(const unsigned long long *key, unsigned *val, unsigned ntot,
                           const unsigned long long *pool_key, const unsigned *pool_idx) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i + 1 >= ntot) return;
  const unsigned long long k = key[i];
  if (key[i + 1] != k || (i > 0 && key[i - 1] == k)) return;
  unsigned e = i + 2;
  while (e < ntot && key[e] == k) e++;
  for (unsigned a = i + 1; a < e; a++) {
    const unsigned v = val[a];
    const unsigned long long fk = pool_key[v];
    const unsigned fi = pool_idx[v];
    unsigned b = a;
    while (b > i && pair_less(fk, fi, pool_key[val[b - 1]], pool_idx[val[b - 1]])) {
      val[b] = val[b - 1];
      b--;
    }
    val[b] = v;
  }
}

__global__ void k_big_out(const unsigned long long *key, const unsigned *val, unsigned ntot, const unsigned *seg_h,
                          const unsigned *seg_start, const unsigned *moff, const unsigned *pool_idx,
                          unsigned *m_index) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ntot) return;
  const unsigned s = (unsigned)(key[i] >> 32);
  m_index[moff[seg_h[s]] + (i - seg_start[s])] = pool_idx[val[i]];
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

SodConst make_sod_const(const psod_ctx *c) {
  SodConst K{};
  K.nx = c->nx;
  K.ncut = c->ncut;
  K.nxf = (float)c->nx;
  K.scale = c->scale;
  for (int a = 0; a < 3; a++) K.xs[a] = c->xxmin[a] * c->scale;  // main:1565
  K.tx = (double)c->nx;                       // main:1517
  K.delta = c->p.delta;
  K.delta2 = c->p.delta2;
  K.cvol = 2.0 / 3.0 * 6.283185307179586;     // main:1424, 2049
  K.munit = (double)c->munit;
  K.mmin = (double)c->p.nmin;                 // main:698
  K.nsel = c->nsel;
  K.n_total = c->n;
  // smallest alive count with count*munit >= Mmin (main:1759)
  {
    const double mu = (double)c->munit;
    long long m = (long long)std::ceil((double)c->p.nmin / mu) - 2;
    if (m < 0) m = 0;
    while ((double)m * mu < (double)c->p.nmin) m++;
    K.mmin_count = (unsigned)m;
  }
  for (int a = 0; a < 3; a++) {
    K.zmin[a] = c->zone_lo[a] * c->scale;     // main:420, 691
    K.zmax[a] = c->zone_hi[a] * c->scale;     // main:421, 692
  }
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

// scratch slots of the SOD stage (kept by the context between calls)
enum {
  SC_BLOCK_OF = 16, SC_BLIST, SC_BBEGIN, SC_CURSOR, SC_HEAD, SC_FILT_A, SC_FILT_B, SC_READY, SC_CTRS,
  SC_PROCESSED, SC_U64, SC_EDGES, SC_HRANK, SC_HID, SC_HMASS, SC_HMASS2, SC_HMEXTRA, SC_HPROF, SC_HCENTER,
  SC_HRDELTA, SC_HPOOL, SC_COUNTS, SC_ST_ACTIVE, SC_ST_NA, SC_ST_COFF, SC_ST_CN,
  SC_ST_CENTRE, SC_CAND_POS, SC_CAND_SLOT, SC_CAND_S, SC_ORDER, SC_RKEYS, SC_MASS32, SC_MOFF, SC_TKEY, SC_TIDX,
  SC_CELLCNT, SC_CELLOFF, SC_CELLCHUNK, SC_CHUNKPREF, SC_ACT_A, SC_ACT_B, SC_BPOS, SC_CELLNCH, SC_FEAT, SC_RB0,
  SC_SBEST, SC_CELLGROUPS, SC_GROUPPREF, SC_CANDU, SC_CANDLIST, SC_CNT2, SC_LMAX, SC_BIG, SC_RESOLVED, SC_BIDXRANK,
  SC_BIDXCUBE, SC_TOPG, SC_XKEY, SC_XIDX, SC_XPOS, SC_TAIL, SC_BIGSEG
};
static_assert((int)SC_BIGSEG < (int)SLOT_CELL_U32, "SOD scratch slots overlap the shared ones");

// Rounds go to the device tail loop once the last host round had no seed
// for the bound pass, no seed with more than tail_max_cand candidates, at
// most tail_max_ready ready seeds (psod_tuning) and few enough active blocks
// for the direct readiness test; after a launch that ended on a larger
// seed, the host runs at least TAIL_REST rounds before the next launch.
constexpr int TAIL_REST = 8;

struct PhaseTimer {
  cudaEvent_t a, b;
  float total = 0.f, last = 0.f;
  PhaseTimer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
  }
  ~PhaseTimer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
  void start(cudaStream_t s) { cudaEventRecord(a, s); }
  void stop(cudaStream_t s) { cudaEventRecord(b, s); }
  void collect() {
    float ms = 0.f;
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    last = ms;
    total += ms;
  }
};

int stage_spherover(psod_ctx *c, psod_run_stats *out_stats) {
  if (!c->seeds_done) return set_err(c, PSOD_ERR_STATE, "psod_spherover needs psod_tri_cic first");
  {
    const int wst = wait_ids(c);  // the halo records read the particle IDs
    if (wst) return wst;
  }
  psod_run_stats st{};
  st.fail_rank = -1;
  st.npart_new = c->npart_new;
  PhaseTimer t_all, t_sched, t_prep, t_ref, t_sel, t_cross, t_setup, t_out, t_learn, t_bound, t_tail;
  t_all.start(c->stream);
  int rc = PSOD_OK;
  const SodConst K = make_sod_const(c);
  const long long n = c->n;
  const long long nseed = c->npart_new;
  long long kernels = 0;

  // reset alive flags: every call starts from the loaded cube
  k_clear_dead<<<nblk(n, 256), 256, 0, c->stream>>>(c->d_cube, n);
  kernels++;

  // block grid of the scheduler
  // block side: the largest power of two dividing nx and at most half the
  // dependency radius, so the window spans 2-4 blocks each way
  const int rdep = c->ncut + std::max(c->ncut, 2);
  int bs = 1;
  for (int cand = 16; cand >= 2; cand >>= 1) {
    if (c->nx % cand == 0 && cand <= std::max(1, rdep / 2)) {
      bs = cand;
      break;
    }
  }
  const int nb = c->nx / bs;
  const long long nblocks = (long long)nb * nb * nb;
  const int rb = (rdep + bs - 1) / bs;
  const long long hcap = std::max<long long>(1, n / std::max(1, c->p.nmin) + 1);
  // refinement candidates held per round (seeds that do not fit wait a round)
  const long long cand_cap = std::min<long long>(n, 128ll << 20);
  const int ne = std::max(1, c->p.ndelta_extra);

  unsigned *block_of, *blist, *bbegin, *cursor, *head, *filt_a, *filt_b, *ready, *ctrs, *counts;
  unsigned char *processed;
  unsigned long long *u64s, *h_pool, *pool_key;
  double *edge_fac, *h_rdelta, *cand_s;
  unsigned *h_rank, *pool_idx, *st_active, *st_na, *st_coff, *st_cn, *st_centre, *cand_pos, *cand_slot;
  long long *h_id, *h_mass, *h_mass2, *h_mextra;
  unsigned *h_profile;
  float *h_center;
  if ((rc = scratch(c, SC_BLOCK_OF, (size_t)nseed + 1, &block_of)) || (rc = scratch(c, SC_BLIST, (size_t)nseed + 1, &blist)) ||
      (rc = scratch(c, SC_BBEGIN, (size_t)nblocks + 1, &bbegin)) || (rc = scratch(c, SC_CURSOR, (size_t)nblocks + 1, &cursor)) ||
      (rc = scratch(c, SC_HEAD, (size_t)nblocks, &head)) || (rc = scratch(c, SC_FILT_A, (size_t)nblocks, &filt_a)) ||
      (rc = scratch(c, SC_FILT_B, (size_t)nblocks, &filt_b)) || (rc = scratch(c, SC_READY, (size_t)nblocks + 1, &ready)) ||
      (rc = scratch(c, SC_CTRS, 16, &ctrs)) || (rc = scratch(c, SC_COUNTS, (size_t)nblocks + 1, &counts)) ||
      (rc = scratch(c, SC_PROCESSED, (size_t)nseed + 1, &processed)) || (rc = scratch(c, SC_U64, 32, &u64s)) ||
      (rc = scratch(c, SC_EDGES, (size_t)c->p.nbins, &edge_fac)) || (rc = scratch(c, SC_HRANK, (size_t)hcap, &h_rank)) ||
      (rc = scratch(c, SC_HID, (size_t)hcap, &h_id)) || (rc = scratch(c, SC_HMASS, (size_t)hcap, &h_mass)) ||
      (rc = scratch(c, SC_HMASS2, (size_t)hcap, &h_mass2)) || (rc = scratch(c, SC_HMEXTRA, (size_t)hcap * ne, &h_mextra)) ||
      (rc = scratch(c, SC_HPROF, (size_t)hcap * c->p.nbins, &h_profile)) || (rc = scratch(c, SC_HCENTER, (size_t)hcap * 3, &h_center)) ||
      (rc = scratch(c, SC_HRDELTA, (size_t)hcap, &h_rdelta)) || (rc = scratch(c, SC_HPOOL, (size_t)hcap, &h_pool)) ||
      (rc = scratch(c, SLOT_PART_U64, (size_t)n, &pool_key)) || (rc = scratch(c, SLOT_PART_U32, (size_t)n, &pool_idx)) ||
      (rc = scratch(c, SC_ST_ACTIVE, (size_t)nblocks + 1, &st_active)) || (rc = scratch(c, SC_ST_NA, (size_t)nblocks + 1, &st_na)) ||
      (rc = scratch(c, SC_ST_COFF, (size_t)nblocks + 1, &st_coff)) || (rc = scratch(c, SC_ST_CN, (size_t)nblocks + 1, &st_cn)) ||
      (rc = scratch(c, SC_ST_CENTRE, (size_t)nblocks + 1, &st_centre)) || (rc = scratch(c, SC_CAND_POS, (size_t)cand_cap, &cand_pos)) ||
      (rc = scratch(c, SC_CAND_SLOT, (size_t)cand_cap, &cand_slot)) || (rc = scratch(c, SC_CAND_S, (size_t)cand_cap, &cand_s)))
    return rc;
  // seeds per round at most (bounds the per-round buffers)
  const unsigned cap_ready = (unsigned)std::min<long long>(nblocks + 1, 1ll << 20);
  unsigned *act_a, *act_b, *bpos;
  if ((rc = scratch(c, SC_ACT_A, (size_t)nblocks + 1, &act_a)) || (rc = scratch(c, SC_ACT_B, (size_t)nblocks + 1, &act_b)) ||
      (rc = scratch(c, SC_BPOS, (size_t)nseed + 1, &bpos)))
    return rc;
  unsigned *cell_cnt, *cell_off, *cell_chunks, *chunk_pref;
  if ((rc = scratch(c, SC_CELLCNT, (size_t)cap_ready * 27, &cell_cnt)) ||
      (rc = scratch(c, SC_CELLOFF, (size_t)cap_ready * 27, &cell_off)) ||
      (rc = scratch(c, SC_CELLCHUNK, (size_t)cap_ready * 27, &cell_chunks)) ||
      (rc = scratch(c, SC_CHUNKPREF, (size_t)cap_ready * 27 + 1, &chunk_pref)))
    return rc;
  unsigned *cell_nch;
  if ((rc = scratch(c, SC_CELLNCH, (size_t)cap_ready * 27, &cell_nch))) return rc;
  // refinement bound groups (64 candidates) and the per-candidate bounds
  unsigned *cell_groups, *group_pref, *s_lmax, *cand_list, *cnt2;
  float *cand_u;
  if ((rc = scratch(c, SC_CELLGROUPS, (size_t)cap_ready * 27, &cell_groups)) ||
      (rc = scratch(c, SC_GROUPPREF, (size_t)cap_ready * 27 + 1, &group_pref)) ||
      (rc = scratch(c, SC_CANDU, (size_t)cand_cap, &cand_u)) || (rc = scratch(c, SC_CANDLIST, (size_t)cand_cap, &cand_list)) ||
      (rc = scratch(c, SC_CNT2, (size_t)cap_ready * 27 * 3 + 1, &cnt2)) ||
      (rc = scratch(c, SC_LMAX, (size_t)cap_ready, &s_lmax)))
    return rc;
  unsigned *s_top;
  if ((rc = scratch(c, SC_TOPG, (size_t)cap_ready * 5 + 1, &s_top))) return rc;
  unsigned *st_big;
  if ((rc = scratch(c, SC_BIG, (size_t)cap_ready, &st_big))) return rc;
  unsigned *resolved, *bidx_of_rank, *bidx_of_cube;
  if ((rc = scratch(c, SC_RESOLVED, (size_t)nseed / 32 + 2, &resolved)) ||
      (rc = scratch(c, SC_BIDXRANK, (size_t)nseed + 1, &bidx_of_rank)) ||
      (rc = scratch(c, SC_BIDXCUBE, (size_t)n, &bidx_of_cube)))
    return rc;
  // crossing buffer of the bucketed balls, shared by the seeds of a round
  const long long xcap = std::min<long long>(n, 256ll << 20);
  unsigned long long *xkey;
  unsigned *xidx, *xpos;
  if ((rc = scratch(c, SC_XKEY, (size_t)xcap, &xkey)) || (rc = scratch(c, SC_XIDX, (size_t)xcap, &xidx)) ||
      (rc = scratch(c, SC_XPOS, (size_t)xcap, &xpos)))
    return rc;
  float *st_feat, *st_rb0;
  unsigned long long *st_sbest;
  if ((rc = scratch(c, SC_FEAT, (size_t)cap_ready * 16, &st_feat)) || (rc = scratch(c, SC_RB0, (size_t)cap_ready, &st_rb0)) ||
      (rc = scratch(c, SC_SBEST, (size_t)cap_ready, &st_sbest)))
    return rc;
  // ctrs: 0 nready, 1..4 work counters, 5 gmin, 6 quirk rank, 7 cand_used,
  // 8/9 active-block counts, 10/11 bound and top-group pass work, 12 nbig
  unsigned *nready_d = ctrs, *work = ctrs + 1, *gmin = ctrs + 5, *qrank_d = ctrs + 6, *cand_used = ctrs + 7;

  PSOD_CUDA(c, cudaMemcpyAsync(edge_fac, c->edge_fac.data(), sizeof(double) * c->p.nbins, cudaMemcpyHostToDevice,
                               c->stream));
  PSOD_CUDA(c, cudaMemsetAsync(processed, 0, (size_t)nseed + 1, c->stream));
  PSOD_CUDA(c, cudaMemsetAsync(u64s, 0, sizeof(unsigned long long) * 32, c->stream));
  PSOD_CUDA(c, cudaMemsetAsync(u64s, 0xff, sizeof(unsigned long long), c->stream));  // err = none
  PSOD_CUDA(c, cudaMemsetAsync(ctrs, 0xff, sizeof(unsigned) * 16, c->stream));

  // seeds bucketed by scheduler block, in rank order within a block
  t_setup.start(c->stream);
  if (nseed > 0) {
    k_seed_blocks<<<nblk(nseed, 256), 256, 0, c->stream>>>(c->d_seed_idx, c->d_inv, c->d_cube, nseed, K, bs, nb,
                                                           block_of, blist);
    PSOD_CUDA(c, cudaMemsetAsync(counts, 0, sizeof(unsigned) * (nblocks + 1), c->stream));
    k_count_u32<<<nblk(nseed, 256), 256, 0, c->stream>>>(block_of, nseed, counts);
    kernels += 2;
    if ((rc = scan_u32(c, counts, bbegin, nblocks, true))) return rc;
    if ((rc = radix_sort_u32(c, block_of, blist, nseed, 32))) return rc;
    PSOD_CUDA(c, cudaMemcpyAsync(cursor, bbegin, sizeof(unsigned) * nblocks, cudaMemcpyDeviceToDevice, c->stream));
    k_seed_pos<<<nblk(nseed, 256), 256, 0, c->stream>>>(blist, nseed, c->d_seed_idx, c->d_inv, bpos);
    PSOD_CUDA(c, cudaMemsetAsync(resolved, 0, sizeof(unsigned) * ((size_t)nseed / 32 + 2), c->stream));
    PSOD_CUDA(c, cudaMemsetAsync(bidx_of_cube, 0xff, sizeof(unsigned) * (size_t)n, c->stream));
    k_seed_index<<<nblk(nseed, 256), 256, 0, c->stream>>>(blist, bpos, nseed, bidx_of_rank, bidx_of_cube);
    kernels += 2;
    if (c->has_quirk) {
      float4 qv;
      PSOD_CUDA(c, cudaMemcpyAsync(&qv, c->d_cube + c->quirk_pos, sizeof(qv), cudaMemcpyDeviceToHost, c->stream));
      PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
      unsigned qidx;
      memcpy(&qidx, &qv.w, 4);
      qidx &= PSOD_IDX_MASK;
      k_find_rank<<<nblk(nseed, 256), 256, 0, c->stream>>>(c->d_seed_idx, nseed, qidx, qrank_d);
      kernels++;
    }
  }
  unsigned quirk_rank = PSOD_INF_RANK;
  PSOD_CUDA(c, cudaMemcpyAsync(&quirk_rank, qrank_d, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
  t_setup.stop(c->stream);
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  t_setup.collect();

  const size_t smem = sizeof(Smem);
  PSOD_CUDA(c, cudaFuncSetAttribute(k_prep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  PSOD_CUDA(c, cudaFuncSetAttribute(k_select, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  PSOD_CUDA(c, cudaFuncSetAttribute(k_cross, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev_sms = 148;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->device);
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cross, TPB, smem);
  if (per_sm < 1) per_sm = 1;
  const unsigned seed_grid = (unsigned)(dev_sms * per_sm);
  int per_sm_ref = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_ref, k_refine_warp<false>, 256, 0);
  const unsigned ref_grid = (unsigned)(dev_sms * std::max(1, per_sm_ref));

  SodBufs B;
  B.cube = c->d_cube;
  B.cs = c->d_cell_start;
  B.ids = c->d_ids;
  B.seed_idx = c->d_seed_idx;
  B.inv = c->d_inv;
  B.edge_fac = edge_fac;
  B.processed = processed;
  B.ready = ready;
  B.nready = nready_d;
  B.cap_ready = cap_ready;
  B.cand_cap = (unsigned long long)cand_cap;
  B.cell_cnt = cell_cnt;
  B.cell_off = cell_off;
  B.cell_chunks = cell_chunks;
  B.chunk_pref = chunk_pref;
  B.cell_nch = cell_nch;
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
  B.st_active = st_active;
  B.st_na = st_na;
  B.st_coff = st_coff;
  B.st_cn = st_cn;
  B.st_centre = st_centre;
  B.cand_pos = cand_pos;
  B.cand_slot = cand_slot;
  B.cand_s = cand_s;
  B.cand_used = cand_used;
  B.work = work;
  B.nbig = ctrs + 12;
  B.bound_min = (unsigned)c->tune.bound_min_cand;
  B.maxcand = ctrs + 13;
  B.max_cand = ~0u;
  B.deferred = ctrs + 14;
  B.alive_cnt = nullptr;
  B.pairs = u64s + 5;
  B.touch = u64s + 7;
  B.kept_members = u64s + 18;
  B.pair_slots = u64s + 8;
  B.ncand_total = u64s + 6;
  B.mode = c->p.mode;
  B.rho = c->d_rho;
  B.st_sbest = st_sbest;
  B.st_feat = st_feat;
  B.st_rb0 = st_rb0;
  B.bracket_hits = u64s + 10;
  B.bracket_seeds = u64s + 11;
  B.cross_balls = u64s + 12;
  B.cross_records = u64s + 13;
  B.cell_groups = cell_groups;
  B.group_pref = group_pref;
  B.cand_u = cand_u;
  B.s_lmax = s_lmax;
  B.cand_list = cand_list;
  B.cnt2 = cnt2;
  B.chunks2 = cnt2 + (size_t)cap_ready * 27;
  B.chunk_pref2 = cnt2 + (size_t)cap_ready * 54;
  B.cand_pruned = u64s + 15;
  B.work_bound = ctrs + 10;
  B.work_top = ctrs + 11;
  B.s_top = s_top;
  B.top_ci = s_top + cap_ready;
  B.top_rem0 = s_top + 2 * (size_t)cap_ready;
  B.top_n = s_top + 3 * (size_t)cap_ready;
  B.top_pref = s_top + 4 * (size_t)cap_ready;
  B.ref_phase = 0;
  B.bound_on = 1;
  // small balls take the warp-per-seed crossing; the CTA kernel the rest
  B.st_big = (c->p.mode != PSOD_MODE_PLAIN) ? st_big : nullptr;
  B.resolved = resolved;
  B.bidx_of_rank = bidx_of_rank;
  B.bidx_of_cube = bidx_of_cube;
  B.xkey = xkey;
  B.xidx = xidx;
  B.xpos = xpos;
  B.xused = u64s + 17;
  B.xcap = (unsigned long long)xcap;
  const size_t wsmem = 8 * sizeof(WSlice);
  PSOD_CUDA(c, cudaFuncSetAttribute(k_cross_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsmem));
  // the learned bracket needs the per-cell alive counts of the batched modes
  B.learn_use = (c->p.mode == PSOD_MODE_LEARNED && learn_ready(c)) ? 1 : 0;
  B.learn_collect = (c->p.mode != PSOD_MODE_PLAIN && learn_collecting(c)) ? 1 : 0;
  B.learn_fof = 0;
  B.fof_code = nullptr;
  B.fof_mass = nullptr;
  B.fof_com = B.fof_rad = nullptr;
  B.fof_feat = nullptr;
  if ((B.learn_use || B.learn_collect) && c->learn_features == PSOD_LEARN_FEATURES_FOF) {
    if (!c->fof_done || c->fof_n != c->n)
      return set_err(c, PSOD_ERR_STATE, "learned FoF features: call psod_fof on the loaded particles first");
    B.learn_fof = 1;
    B.fof_code = static_cast<const unsigned *>(c->scratch[SLOT_F_CODE].first);
    B.fof_mass = static_cast<const long long *>(c->scratch[SLOT_F_MASS].first);
    B.fof_com = static_cast<const double *>(c->scratch[SLOT_F_COM].first);
    B.fof_rad = static_cast<const double *>(c->scratch[SLOT_F_RAD].first);
    B.fof_feat = static_cast<const float4 *>(c->scratch[SLOT_F_FEAT].first);
  }
  B.learn_x = B.learn_t = nullptr;
  B.learn_n = nullptr;
  B.learn_cap = 0;
  if (B.learn_collect) learn_sample_buffers(c, &B.learn_x, &B.learn_t, &B.learn_n, &B.learn_cap);
  if (c->p.mode != PSOD_MODE_PLAIN) {
    unsigned *alive_cnt;
    if ((rc = scratch(c, SLOT_CELL_U32, (size_t)c->ncell, &alive_cnt))) return rc;
    k_init_alive<<<nblk((long long)c->ncell, 256), 256, 0, c->stream>>>(c->d_cell_start, c->ncell, alive_cnt);
    kernels++;
    B.alive_cnt = alive_cnt;
  }

  long long rounds = 0, seed_launches = 0;
  // ctrs[8]: active-block count of the current list, ctrs[9]: of the next
  unsigned n_active = 0;
  if (nseed > 0) {
    PSOD_CUDA(c, cudaMemsetAsync(ctrs + 8, 0, sizeof(unsigned) * 2, c->stream));
    k_init_active<<<nblk(nblocks, 256), 256, 0, c->stream>>>(nblocks, bbegin, head, act_a, ctrs + 8);
    kernels++;
    PSOD_CUDA(c, cudaMemcpyAsync(&n_active, ctrs + 8, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  // Each round launches the counter reset, the heads, the readiness test and
  // the preselect back to back; the host then reads the round's counters
  // (its only synchronisation per round) and launches the refinement,
  // select and crossing kernels sized by them, the bound pipeline only when
  // some seed has bound_min_cand candidates.  Phase timers of the refinement
  // onwards are read one round later, when their events have completed.
  const long long window = (long long)std::min(2 * rb + 1, nb);
  const long long direct_cost_per_block = window * window * window, filter_cost = 3 * nblocks * window;
  bool pending = false, pend_learn = false, pend_bound = false;
  // device tail loop: one CTA per seed slot resident on every SM
  int tail_grid = 0, rest = 0;
  long long tail_rounds = 0;
  TailState *tail = nullptr;
  {
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device);
    int per_sm_tail = 0;
    if (coop && (rc = scratch(c, SC_TAIL, 1, &tail)) == PSOD_OK &&
        cudaFuncSetAttribute(k_tail_rounds, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_tail, k_tail_rounds, TPB, smem) == cudaSuccess &&
        per_sm_tail > 0)
      tail_grid = dev_sms * per_sm_tail;
    if (rc) return rc;
    cudaGetLastError();
  }
  auto collect_pending = [&]() {
    if (!pending) return;
    t_ref.collect();
    t_sel.collect();
    t_cross.collect();
    if (pend_learn) t_learn.collect();
    if (pend_bound) t_bound.collect();
    pending = false;
  };
  while (nseed > 0 && n_active > 0) {
    t_sched.start(c->stream);
    k_round_reset<<<1, 32, 0, c->stream>>>(ctrs, u64s + 17);
    k_heads<<<nblk((long long)n_active, 256), 256, 0, c->stream>>>(
        act_a, n_active, bbegin, cursor, blist, resolved, head,
        quirk_rank != PSOD_INF_RANK ? gmin : nullptr, act_b, ctrs + 9);
    if ((long long)n_active * direct_cost_per_block <= filter_cost) {
      k_ready_direct<<<nblk((long long)n_active * 32, 256), 256, 0, c->stream>>>(act_b, ctrs + 9, head, nb, rb,
                                                                                  quirk_rank, gmin, ready, nready_d,
                                                                                  cap_ready);
      kernels += 3;
    } else {
      k_minfilter<<<nblk(nblocks, 256), 256, 0, c->stream>>>(head, filt_a, nb, 0, rb);
      k_minfilter<<<nblk(nblocks, 256), 256, 0, c->stream>>>(filt_a, filt_b, nb, 1, rb);
      k_minfilter<<<nblk(nblocks, 256), 256, 0, c->stream>>>(filt_b, filt_a, nb, 2, rb);
      k_ready<<<nblk(n_active, 256), 256, 0, c->stream>>>(act_b, ctrs + 9, head, filt_a, quirk_rank, gmin, ready,
                                                           nready_d, cap_ready);
      kernels += 6;
    }
    t_sched.stop(c->stream);
    // preselect over a persistent grid: the ready count is read on the device
    t_prep.start(c->stream);
    k_prep<<<seed_grid, TPB, smem, c->stream>>>(K, B);
    t_prep.stop(c->stream);
    kernels++;
    unsigned hc[14];
    PSOD_CUDA(c, cudaMemcpyAsync(hc, ctrs, sizeof(hc), cudaMemcpyDeviceToHost, c->stream));
    PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
    t_sched.collect();
    t_prep.collect();
    collect_pending();
    unsigned nready = hc[0];
    n_active = hc[9];
    const unsigned nbig = hc[12], maxcand = hc[13];
    std::swap(act_a, act_b);
    if (nready == 0) {
      // the lowest-ranked unresolved seed is always ready, so an empty
      // round with unresolved seeds left is a scheduler fault
      if (n_active > 0) return set_err(c, PSOD_ERR_STATE, "scheduler stalled with unresolved seeds");
      break;
    }
    nready = std::min(nready, cap_ready);
    const unsigned g = std::min<unsigned>(seed_grid, nready);
    B.bound_on = nbig > 0 ? 1 : 0;
    t_ref.start(c->stream);
    B.nitems_cells = 27u * nready;
    if ((rc = scan_u32(c, cell_chunks, chunk_pref, (long long)B.nitems_cells, true))) return rc;
    if (B.bound_on) {
      if ((rc = scan_u32(c, cell_groups, group_pref, (long long)B.nitems_cells, true))) return rc;
      t_bound.start(c->stream);
      k_zero_bounds<<<ref_grid, 256, 0, c->stream>>>(cand_used, (unsigned long long)cand_cap, cand_u);
      PSOD_CUDA(c, cudaMemsetAsync(s_lmax, 0, sizeof(unsigned) * nready, c->stream));
      k_seed_lower<<<nblk((long long)nready * 32, 256), 256, 0, c->stream>>>(K, B);
      k_refine_warp<true><<<ref_grid, 256, 0, c->stream>>>(K, B);
      k_top_group<<<nblk((long long)nready * 32, 256), 256, 0, c->stream>>>(K, B);
      if ((rc = scan_u32(c, B.top_n, B.top_pref, (long long)nready, true))) return rc;
      t_bound.stop(c->stream);
      // the top groups' sums first, then the lower bound they give, then
      // the surviving candidates of every cell
      SodBufs Bt = B;
      Bt.ref_phase = 1;
      k_refine_warp<false><<<ref_grid, 256, 0, c->stream>>>(K, Bt);
      k_top_lower<<<nblk((long long)nready * 32, 256), 256, 0, c->stream>>>(K, B);
      k_survivors<<<nblk((long long)B.nitems_cells * 32, 256), 256, 0, c->stream>>>(K, B);
      if ((rc = scan_u32(c, B.chunks2, B.chunk_pref2, (long long)B.nitems_cells, true))) return rc;
      kernels += 7;
    }
    SodBufs Bp = B;
    Bp.ref_phase = B.bound_on ? 2 : 0;
    k_refine_warp<false><<<ref_grid, 256, 0, c->stream>>>(K, Bp);
    t_ref.stop(c->stream);
    t_sel.start(c->stream);
    k_select<<<g, TPB, smem, c->stream>>>(K, B);
    t_sel.stop(c->stream);
    if (B.learn_use) {
      // features were written by k_select; one inference launch per round
      t_learn.start(c->stream);
      if ((rc = learn_predict(c, st_feat, nready, st_rb0))) return rc;
      kernels++;
      t_learn.stop(c->stream);
    }
    t_cross.start(c->stream);
    // The warp pass pays off when a round has many seeds; in the sparse tail
    // a round lasts as long as its slowest seed, and a CTA handles one seed
    // with eight warps.
    SodBufs Bc = B;
    if (!(B.st_big && nready >= (unsigned)c->tune.warp_cross_min_ready)) Bc.st_big = nullptr;
    if (Bc.st_big) {
      k_cross_warp<<<nblk((long long)nready * 32, 256), 256, wsmem, c->stream>>>(K, Bc);
      kernels++;
    }
    k_cross<<<g, TPB, smem, c->stream>>>(K, Bc);
    t_cross.stop(c->stream);
    PSOD_CUDA(c, cudaGetLastError());
    pending = true;
    pend_learn = B.learn_use;
    pend_bound = B.bound_on;
#ifdef PSOD_TRACE_ROUNDS
    {
      // diagnostic build only (-DPSOD_TRACE_ROUNDS): one line per round on
      // stderr with the ready seeds, active blocks, candidates and phase times
      collect_pending();
      unsigned cu = 0;
      unsigned long long tv[21];
      cudaMemcpyAsync(&cu, cand_used, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream);
      cudaMemcpyAsync(tv, u64s, sizeof(tv), cudaMemcpyDeviceToHost, c->stream);
      cudaStreamSynchronize(c->stream);
      fprintf(stderr,
              "psod round %lld ready %u active %u cand %u nbig %u sched %.3f prep %.3f refine %.3f select %.3f cross %.3f "
              "pairs %llu slots %llu staged %llu bound %.3f items %llu pruned_cand %llu touch %llu kept %llu\n",
              rounds, nready, n_active, cu, nbig, t_sched.last, t_prep.last, t_ref.last, t_sel.last, t_cross.last,
              tv[5], tv[8], tv[9], B.bound_on ? t_bound.last : 0.0, tv[14], tv[15], tv[7], tv[18]);
    }
#endif
    rounds++;
    seed_launches += 4;
    kernels += 4;
    rest++;
    if (tail_grid > 0 && nbig == 0 && maxcand <= (unsigned)c->tune.tail_max_cand &&
        nready <= (unsigned)c->tune.tail_max_ready && rest >= TAIL_REST &&
        n_active > 0 && (long long)n_active * direct_cost_per_block <= filter_cost) {
      // the following rounds on the device, until a larger seed or the end
      k_tail_init<<<1, 1, 0, c->stream>>>(tail, n_active);
      SodBufs Bt = B;
      Bt.max_cand = (unsigned)c->tune.tail_max_cand;
      Bt.st_big = nullptr;
      Bt.touch = u64s + 19;  // the tail's crossings counted apart from k_cross
      Bt.kept_members = u64s + 20;
      void *args[] = {(void *)&K,     (void *)&Bt,   (void *)&tail, (void *)&act_a,      (void *)&act_b,
                      (void *)&bbegin, (void *)&cursor, (void *)&blist, (void *)&head, (void *)&nb,
                      (void *)&rb,    (void *)&quirk_rank, (void *)&ready};
      t_tail.start(c->stream);
      PSOD_CUDA(c, cudaLaunchCooperativeKernel((const void *)k_tail_rounds, dim3(tail_grid), dim3(TPB), args, smem,
                                               c->stream));
      t_tail.stop(c->stream);
      kernels += 2;
      TailState ts;
      PSOD_CUDA(c, cudaMemcpyAsync(&ts, tail, sizeof(ts), cudaMemcpyDeviceToHost, c->stream));
      PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
      t_tail.collect();
      collect_pending();
      rounds += ts.rounds;
      tail_rounds += ts.rounds;
#ifdef PSOD_TRACE_ROUNDS
      fprintf(stderr, "psod tail launch rounds %u status %u heads %.3f ready %.3f seeds %.3f ms total %.3f ms grid %d\n",
              ts.rounds, ts.status, ts.t_heads * 1e-6, ts.t_ready * 1e-6, ts.t_seeds * 1e-6, t_tail.last, tail_grid);
#endif
      if (ts.status == TAIL_TIMEOUT)
        return set_err(c, PSOD_ERR_TIMEOUT, "device tail loop: a grid barrier wait ran out");
      if (ts.status == TAIL_STALLED) return set_err(c, PSOD_ERR_STATE, "scheduler stalled with unresolved seeds");
      if (ts.status != TAIL_DONE && ts.status != TAIL_DEFERRED)
        return set_err(c, PSOD_ERR_STATE, "device tail loop ended in an unknown state");
      // the live list and its count for the host's next round
      if (ts.parity) std::swap(act_a, act_b);
      n_active = ts.status == TAIL_DONE ? 0u : ts.nact[ts.parity];
      rest = 0;
    }
  }
  collect_pending();
  // every seed must end processed or claimed; u64s[16] counts those that did not
  if (nseed > 0) {
    k_count_unresolved<<<nblk(nseed / 32 + 1, 256), 256, 0, c->stream>>>(resolved, nseed, u64s + 16);
    kernels++;
  }
  unsigned long long hv[21];
  PSOD_CUDA(c, cudaMemcpyAsync(hv, u64s, sizeof(hv), cudaMemcpyDeviceToHost, c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  st.rounds = rounds;
  st.touched = (int64_t)hv[3];
  st.nprocessed = (int64_t)hv[4];
  st.ms_sched = t_sched.total;
  st.ms_prep = t_prep.total;
  st.ms_refine = t_ref.total;
  st.ms_select = t_sel.total;
  st.ms_cross = t_cross.total;
  st.ms_sod_kernel = t_prep.total + t_ref.total + t_sel.total + t_cross.total;
  st.sod_launches = seed_launches;
  st.ncandidates = (int64_t)hv[6];
  st.refine_pairs = (int64_t)hv[5];
  st.cross_touch = (int64_t)(hv[7] + hv[19]);
  st.tail_touch = (int64_t)hv[19];
  st.cross_members = (int64_t)hv[18];
  st.tail_members = (int64_t)hv[20];
  st.refine_slots = (int64_t)hv[8];
  st.ms_learn = t_learn.total;
  st.bracket_hits = (int64_t)hv[10];
  st.bracket_seeds = (int64_t)hv[11];
  st.cross_balls = (int64_t)hv[12];
  st.cross_records = (int64_t)hv[13];
  st.ms_refine_bound = t_bound.total;
  st.refine_items = (int64_t)hv[14];
  st.refine_pruned = (int64_t)hv[15];
  st.ms_tail = t_tail.total;
  st.tail_rounds = tail_rounds;
  c->nhalo = 0;
  c->nmember = 0;
  c->sod_done = false;
  if (hv[0] == ~0ull && hv[16] != 0) {
    st.kernel_launches = kernels;
    c->last_stats = st;
    if (out_stats) *out_stats = st;
    return set_err(c, PSOD_ERR_STATE, std::to_string(hv[16]) + " seeds left unresolved by the scheduler");
  }
  if (hv[0] != ~0ull) {
    const int code = (int)(hv[0] & 0xff);
    st.fail_rank = (int64_t)(hv[0] >> 8);
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
  t_out.start(c->stream);
  const long long nh = (long long)hv[1];
  const unsigned long long npool = std::max<unsigned long long>(hv[2], 1);
  unsigned *order, *rkeys, *mass32, *moff, *tidx;
  unsigned long long *tkey;
  if ((rc = scratch(c, SC_ORDER, (size_t)nh + 1, &order)) || (rc = scratch(c, SC_RKEYS, (size_t)nh + 1, &rkeys)) ||
      (rc = scratch(c, SC_MASS32, (size_t)nh + 1, &mass32)) || (rc = scratch(c, SC_MOFF, (size_t)nh + 1, &moff)) ||
      (rc = scratch(c, SC_TKEY, (size_t)npool, &tkey)) || (rc = scratch(c, SC_TIDX, (size_t)npool, &tidx)))
    return rc;
  if (nh > 0) {
    std::vector<unsigned> iota((size_t)nh);
    for (long long i = 0; i < nh; i++) iota[(size_t)i] = (unsigned)i;
    PSOD_CUDA(c, cudaMemcpyAsync(order, iota.data(), sizeof(unsigned) * nh, cudaMemcpyHostToDevice, c->stream));
    PSOD_CUDA(c, cudaMemcpyAsync(rkeys, h_rank, sizeof(unsigned) * nh, cudaMemcpyDeviceToDevice, c->stream));
    PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
    if ((rc = radix_sort_u32(c, rkeys, order, nh, 32))) return rc;
  }
  if ((rc = scratch(c, SLOT_H_ID, (size_t)nh, &c->d_h_id)) || (rc = scratch(c, SLOT_H_MASS, (size_t)nh, &c->d_h_mass)) ||
      (rc = scratch(c, SLOT_H_RANK, (size_t)nh, &c->d_h_rank)) ||
      (rc = scratch(c, SLOT_H_MASS2, (size_t)nh, &c->d_h_mass2)) ||
      (rc = scratch(c, SLOT_H_MEXTRA, (size_t)nh * ne, &c->d_h_mextra)) ||
      (rc = scratch(c, SLOT_H_PROFILE, (size_t)nh * c->p.nbins, &c->d_h_profile)) ||
      (rc = scratch(c, SLOT_H_CENTER, (size_t)nh * 3, &c->d_h_center)) ||
      (rc = scratch(c, SLOT_H_RDELTA, (size_t)nh, &c->d_h_rdelta)) ||
      (rc = scratch(c, SLOT_M_OFFSET, (size_t)nh + 1, &c->d_m_offset)) ||
      (rc = scratch(c, SLOT_M_INDEX, (size_t)npool, &c->d_m_index)))
    return rc;
  if (nh > 0) {
    const unsigned g1 = nblk(nh, 256);
    k_gather<long long><<<g1, 256, 0, c->stream>>>(h_id, order, nh, 1, c->d_h_id);
    k_gather<long long><<<g1, 256, 0, c->stream>>>(h_mass, order, nh, 1, c->d_h_mass);
    k_gather<long long><<<g1, 256, 0, c->stream>>>(h_mass2, order, nh, 1, c->d_h_mass2);
    k_gather<double><<<g1, 256, 0, c->stream>>>(h_rdelta, order, nh, 1, c->d_h_rdelta);
    k_gather<float><<<nblk(nh * 3, 256), 256, 0, c->stream>>>(h_center, order, nh, 3, c->d_h_center);
    if (c->p.ndelta_extra > 0)
      k_gather<long long><<<nblk(nh * ne, 256), 256, 0, c->stream>>>(h_mextra, order, nh, ne, c->d_h_mextra);
    k_gather_widen<<<nblk(nh * c->p.nbins, 256), 256, 0, c->stream>>>(h_profile, order, nh, c->p.nbins,
                                                                      c->d_h_profile);
    k_widen<<<g1, 256, 0, c->stream>>>(rkeys, nh, c->d_h_rank);
    k_mass_u32<<<g1, 256, 0, c->stream>>>(c->d_h_mass, nh, mass32);
    if ((rc = scan_u32(c, mass32, moff, nh, true))) return rc;
    k_widen<<<nblk(nh + 1, 256), 256, 0, c->stream>>>(moff, nh + 1, c->d_m_offset);
    k_member_sort<<<std::min<long long>(nh, 4 * dev_sms), 256, 0, c->stream>>>(
        order, nh, h_pool, c->d_h_mass, moff, pool_key, pool_idx, c->d_m_index);
    kernels += 11;
    // the large halos claimed unsorted: one device-wide sort
    unsigned *bsc;
    if ((rc = scratch(c, SC_BIGSEG, 5 * ((size_t)nh + 2), &bsc))) return rc;
    unsigned *big_scan = bsc, *msz_scan = bsc + (nh + 2), *seg_h = bsc + 2 * (nh + 2),
             *seg_start = bsc + 3 * (nh + 2), *seg_base = bsc + 4 * (nh + 2);
    k_big_flags<<<g1, 256, 0, c->stream>>>(order, nh, h_pool, c->d_h_mass, big_scan, msz_scan);
    kernels++;
    if ((rc = scan_u32(c, big_scan, big_scan, nh, true)) || (rc = scan_u32(c, msz_scan, msz_scan, nh, true)))
      return rc;
    k_big_list<<<g1, 256, 0, c->stream>>>(order, nh, h_pool, big_scan, msz_scan, seg_h, seg_start, seg_base);
    kernels++;
    unsigned tot[2] = {0, 0};
    PSOD_CUDA(c, cudaMemcpyAsync(&tot[0], big_scan + nh, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    PSOD_CUDA(c, cudaMemcpyAsync(&tot[1], msz_scan + nh, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
    const unsigned nbig = tot[0], ntot = tot[1];
    if (nbig > 0) {
      k_big_keys<<<nblk(ntot, 256), 256, 0, c->stream>>>(seg_start, nbig, seg_base, pool_key, ntot, tkey, tidx);
      kernels++;
      if ((rc = radix_sort_u64(c, tkey, tidx, ntot, 64))) return rc;
      k_big_ties<<<nblk(ntot, 256), 256, 0, c->stream>>>(tkey, tidx, ntot, pool_key, pool_idx);
      k_big_out<<<nblk(ntot, 256), 256, 0, c->stream>>>(tkey, tidx, ntot, seg_h, seg_start, moff, pool_idx,
                                                        c->d_m_index);
      kernels += 2;
    }
  } else {
    PSOD_CUDA(c, cudaMemsetAsync(c->d_m_offset, 0, sizeof(long long), c->stream));
  }
  PSOD_CUDA(c, cudaGetLastError());
  t_out.stop(c->stream);
  t_all.stop(c->stream);
  t_out.collect();
  t_all.collect();
  st.ms_total = t_all.total;
  st.ms_setup = t_setup.total;
  st.ms_output = t_out.total;
  st.nhalo = nh;
  st.nmember = (int64_t)hv[2];
  st.kernel_launches = kernels;
  c->nhalo = nh;
  c->nmember = (long long)hv[2];
  c->sod_done = true;
  c->last_stats = st;
  if (out_stats) *out_stats = st;
  return PSOD_OK;
}

}  // namespace psod
