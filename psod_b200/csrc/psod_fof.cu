// psod_fof.cu -- friends-of-friends halo finder (pFoF on one rank).
//
// The catalogue the SOD stage's cube files come from: pFoF's fofpara
// (Pfof/trunk/pfof_snap/src/modfofpara.f90:31-296) with its periodic merge
// (Pfof/trunk/common/src/modfofmpi.f90:37-649) and the halo observables of
// sod/modhalo.f90 (selecthaloes :253-376, computecom :381-441,
// computeradius :445-488), on the particles of psod_load_particles.
//
// The reference grows one group at a time from a queue, scanning for each
// particle the cells of a grid of 2*nres cells a side.  Here the groups are
// the connected components of the same friendship relation, found in
// parallel:
//   1. linking cells.  Each SOD cell of the cell-sorted cube (1/nx a side)
//      is cut into k^3 linking cells, k chosen so that a linking cell's
//      diagonal is shorter than the linking length: the particles of one
//      linking cell are all friends, and a particle's friends lie in
//      linking cells at most R = floor(l*k)+1 cells away per axis.  Each SOD
//      cell's records are sorted by linking cell (a thread per small cell, a
//      CTA counting sort per large one), so a linking cell is a run.
//   2. union-find over runs.  A run starts as one component.  For every pair
//      of neighbouring runs (each unordered pair once: offsets in a half
//      space) the particle pairs are tested until one pair are friends, and
//      then the two components are joined (lock-free: the larger root is
//      hooked under the smaller with atomicCAS).  Runs of up to 4 records are
//      handled by a thread, larger ones by a warp.
//   3. labels, masses, members, centres and radii as the reference computes
//      them, per halo.
// The friendship test is the reference's FP32 arithmetic, bit for bit: two
// particles are friends when dx^2+dy^2+dz^2 <= r2, r2 = (percolation/nres)^2
// in FP32, with dx = |x1-x2| for pairs within half a box on every axis (the
// local scan, modfofpara.f90:234-238) and dx = min(dx, 1-dx) for pairs across
// the periodic boundary whose two particles lie within percolation/nres of
// opposite faces of one axis (the bridges of findbridge, modfofmpi.f90:
// 226-233, between the face lists of initmerging :98-173).
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include <cmath>
#include <vector>

#include "psod_internal.cuh"

namespace cg = cooperative_groups;

namespace psod {
namespace {

constexpr int FOF_TPB = 256;
constexpr unsigned FOF_SMALL_CELL = 16;  // records a thread sorts itself
constexpr unsigned FOF_THREAD_RUN = 4;   // runs a thread links; longer ones go to a warp
constexpr int FOF_MAX_OFF = 171;         // half of the 7^3 - 1 neighbour offsets
constexpr unsigned FOF_WARP_HALO = 2048; // halos whose observables a warp computes; larger: a CTA

__constant__ signed char c_fof_off[3 * FOF_MAX_OFF];

struct FofGeo {
  int nx;
  float nxf;
  double xs;   // SOD grid shift (grid units)
  int k;       // linking cells per SOD cell and axis
  int R;       // reach in linking cells per axis
  double reach2;  // squared reach, in linking-cell units, for the box filter
  int noff;    // neighbour offsets in c_fof_off
  float r2, rT;
  unsigned long long ncell;
};

// SOD cell and linking cell of one axis: the same cell as the cube's sort
// (sod_cell_axis), then the position inside it in linking-cell units
__device__ __forceinline__ void fof_axis(float x, const FofGeo &G, int &cell, int &fine, float &fpos) {
  const double d = dsub((double)to_grid(x, G.nxf), G.xs);
  int i = (int)floor(d);
  const double fr = (d - (double)i) * (double)G.k;
  int f = (int)floor(fr);
  f = f < 0 ? 0 : (f >= G.k ? G.k - 1 : f);
  if (i < 0) i += G.nx;
  if (i >= G.nx) i -= G.nx;
  cell = i;
  fine = f;
  fpos = (float)fr;
}

__device__ __forceinline__ unsigned fof_key(float4 v, const FofGeo &G) {
  int c, fx, fy, fz;
  float p;
  fof_axis(v.x, G, c, fx, p);
  fof_axis(v.y, G, c, fy, p);
  fof_axis(v.z, G, c, fz, p);
  return (unsigned)(fx + G.k * (fy + G.k * fz));
}

// positions equal to 1.0 count as 0.0 (modfofpara.f90:162-164)
__device__ __forceinline__ float fof_wrap1(float x) { return x == 1.0f ? 0.0f : x; }

// the reference's friendship test (see the file comment)
__device__ __forceinline__ bool fof_friends(float4 a, float4 b, float r2, float rT) {
  const float ax = fof_wrap1(a.x), ay = fof_wrap1(a.y), az = fof_wrap1(a.z);
  const float bx = fof_wrap1(b.x), by = fof_wrap1(b.y), bz = fof_wrap1(b.z);
  float dx = fabsf(__fsub_rn(ax, bx)), dy = fabsf(__fsub_rn(ay, by)), dz = fabsf(__fsub_rn(az, bz));
  if (dx > 0.5f || dy > 0.5f || dz > 0.5f) {
    // across the boundary: only a bridge between opposite face lists
    auto lo = [&](float x) { return fabsf(x) <= rT; };
    auto hi = [&](float x) { return fabsf(__fsub_rn(x, 1.0f)) <= rT; };
    const bool faces = (lo(ax) && hi(bx)) || (hi(ax) && lo(bx)) || (lo(ay) && hi(by)) || (hi(ay) && lo(by)) ||
                       (lo(az) && hi(bz)) || (hi(az) && lo(bz));
    if (!faces) return false;
    dx = fminf(dx, __fsub_rn(1.0f, dx));
    dy = fminf(dy, __fsub_rn(1.0f, dy));
    dz = fminf(dz, __fsub_rn(1.0f, dz));
  }
  const float d = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
  return d <= r2;
}

// union-find on run heads: parents only point to smaller positions, so the
// root of a component is its smallest position
__device__ __forceinline__ unsigned uf_find(unsigned *par, unsigned x) {
  unsigned p = __ldcg(par + x);
  while (p != x) {
    const unsigned g = __ldcg(par + p);
    if (g == p) return p;
    __stcg(par + x, g);  // path halving: g is an ancestor of x
    x = g;
    p = __ldcg(par + x);
  }
  return x;
}

// root without writes: used while compressing, when other threads store
// roots into the same trees (a halving store could put back a non-root)
__device__ __forceinline__ unsigned uf_root(const unsigned *par, unsigned x) {
  unsigned p = __ldcg(par + x);
  while (p != x) {
    x = p;
    p = __ldcg(par + x);
  }
  return x;
}

__device__ __forceinline__ void uf_union(unsigned *par, unsigned a, unsigned b) {
  while (true) {
    a = uf_find(par, a);
    b = uf_find(par, b);
    if (a == b) return;
    if (a > b) {
      const unsigned t = a;
      a = b;
      b = t;
    }
    const unsigned old = atomicCAS(par + b, b, a);
    if (old == b) return;
    b = old;  // b was hooked meanwhile: retry from its new parent
  }
}

// ---------------------------------------------------------------------------
// 1. linking-cell keys and the per-cell sort
// ---------------------------------------------------------------------------
__global__ void k_fof_keys(const float4 *cube, long long n, FofGeo G, unsigned short *key) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) key[s] = (unsigned short)fof_key(cube[s], G);
}

// A thread per SOD cell: cells of at most FOF_SMALL_CELL records are sorted
// here (insertion sort on (key, slot)); larger ones are listed for the CTA
// sort.  Writes the FoF order (perm: cube slot), the sorted keys, each
// position's run head (the union-find parent) and the inverse map.
__global__ void k_fof_sort_small(const unsigned *cs, unsigned long long ncell, const unsigned short *key,
                                 const float4 *cube, unsigned *perm, unsigned short *skey, unsigned *par,
                                 unsigned *finv, unsigned *big, unsigned *nbig) {
  const unsigned long long c = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const unsigned b = cs[c], e = cs[c + 1], m = e - b;
  if (m == 0) return;
  if (m > FOF_SMALL_CELL) {
    big[atomicAdd(nbig, 1u)] = (unsigned)c;
    return;
  }
  unsigned kk[FOF_SMALL_CELL], ss[FOF_SMALL_CELL];
  for (unsigned j = 0; j < m; j++) {
    const unsigned kv = key[b + j];
    unsigned t = j;
    while (t > 0 && kk[t - 1] > kv) {
      kk[t] = kk[t - 1];
      ss[t] = ss[t - 1];
      t--;
    }
    kk[t] = kv;
    ss[t] = b + j;
  }
  unsigned head = b;
  for (unsigned j = 0; j < m; j++) {
    if (j > 0 && kk[j] != kk[j - 1]) head = b + j;
    perm[b + j] = ss[j];
    skey[b + j] = (unsigned short)kk[j];
    par[b + j] = head;
    finv[__float_as_uint(cube[ss[j]].w) & ~PSOD_DEAD_BIT] = b + j;
  }
}

// A CTA per large SOD cell: counting sort on the linking-cell key with the
// k^3 bins in shared memory; a run head is its bin's start.
__global__ void __launch_bounds__(FOF_TPB) k_fof_sort_big(const unsigned *cs, const unsigned *big,
                                                          const unsigned *nbig, int nbins,
                                                          const unsigned short *key, const float4 *cube,
                                                          unsigned *perm, unsigned short *skey, unsigned *par,
                                                          unsigned *finv) {
  extern __shared__ unsigned bins[];
  const unsigned nb = *nbig;
  for (unsigned q = blockIdx.x; q < nb; q += gridDim.x) {
    const unsigned c = big[q];
    const unsigned b = cs[c], e = cs[c + 1];
    for (int i = threadIdx.x; i < nbins; i += blockDim.x) bins[i] = 0;
    __syncthreads();
    for (unsigned s = b + threadIdx.x; s < e; s += blockDim.x) atomicAdd(&bins[key[s]], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned run = 0;
      for (int i = 0; i < nbins; i++) {
        const unsigned v = bins[i];
        bins[i] = run;
        run += v;
      }
    }
    __syncthreads();
    // bins[i] is the start of bin i and serves as its write cursor
    for (unsigned s = b + threadIdx.x; s < e; s += blockDim.x) {
      const unsigned kv = key[s];
      const unsigned at = b + atomicAdd(&bins[kv], 1u);
      perm[at] = s;
      skey[at] = (unsigned short)kv;
      finv[__float_as_uint(cube[s].w) & ~PSOD_DEAD_BIT] = at;
    }
    __syncthreads();
    // bins[i] is now the end of bin i: a position's head is the first
    // position with its key (the end of the previous bin)
    for (unsigned p = b + threadIdx.x; p < e; p += blockDim.x) {
      const unsigned kv = skey[p];
      par[p] = b + (kv == 0 ? 0u : bins[kv - 1]);
    }
    __syncthreads();
  }
}

// run-head flags (a head is its own parent)
__global__ void k_fof_head_flags(const unsigned *par, long long n, unsigned *flag) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) flag[p] = par[p] == (unsigned)p ? 1u : 0u;
}

__global__ void k_fof_head_list(const unsigned *flag, const unsigned *pos, long long n, unsigned *heads) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n && flag[p]) heads[pos[p]] = (unsigned)p;
  if (p == n - 1) heads[pos[p] + flag[p]] = (unsigned)n;  // end sentinel
}

// ---------------------------------------------------------------------------
// 2. linking
// ---------------------------------------------------------------------------
struct RunGeo {
  int cx, cy, cz, fx, fy, fz;
};

__device__ __forceinline__ RunGeo run_geo(float4 v, const FofGeo &G, float lo[3], float hi[3]) {
  RunGeo r;
  float px, py, pz;
  fof_axis(v.x, G, r.cx, r.fx, px);
  fof_axis(v.y, G, r.cy, r.fy, py);
  fof_axis(v.z, G, r.cz, r.fz, pz);
  lo[0] = hi[0] = px;
  lo[1] = hi[1] = py;
  lo[2] = hi[2] = pz;
  return r;
}

// the run of linking cell (run origin + offset o), or an empty range
__device__ __forceinline__ bool find_run(const RunGeo &u, int ox, int oy, int oz, const FofGeo &G, const unsigned *cs,
                                         const unsigned short *skey, unsigned &vlo, unsigned &vhi) {
  int tx = u.fx + ox, ty = u.fy + oy, tz = u.fz + oz;
  int dcx = tx < 0 ? -1 : (tx >= G.k ? 1 : 0), dcy = ty < 0 ? -1 : (ty >= G.k ? 1 : 0),
      dcz = tz < 0 ? -1 : (tz >= G.k ? 1 : 0);
  tx -= dcx * G.k;
  ty -= dcy * G.k;
  tz -= dcz * G.k;
  int cx = u.cx + dcx, cy = u.cy + dcy, cz = u.cz + dcz;
  cx = cx < 0 ? cx + G.nx : (cx >= G.nx ? cx - G.nx : cx);
  cy = cy < 0 ? cy + G.nx : (cy >= G.nx ? cy - G.nx : cy);
  cz = cz < 0 ? cz + G.nx : (cz >= G.nx ? cz - G.nx : cz);
  const unsigned long long c =
      (unsigned long long)cx + (unsigned long long)G.nx * ((unsigned long long)cy + (unsigned long long)G.nx * cz);
  const unsigned lo = __ldg(cs + c), hi = __ldg(cs + c + 1);
  if (lo == hi) return false;
  const unsigned short kv = (unsigned short)(tx + G.k * (ty + G.k * tz));
  unsigned a = lo, b = hi;
  if (hi - lo <= 16) {
    while (a < hi && __ldg(skey + a) < kv) a++;
  } else {
    while (a < b) {  // first position with key >= kv
      const unsigned m = (a + b) >> 1;
      if (__ldg(skey + m) < kv) a = m + 1;
      else b = m;
    }
  }
  if (a >= hi || __ldg(skey + a) != kv) return false;
  unsigned z = a + 1;
  if (hi - a <= 16) {
    while (z < hi && __ldg(skey + z) == kv) z++;
  } else {
    unsigned b2 = hi;
    while (z < b2) {  // first position with key > kv
      const unsigned m = (z + b2) >> 1;
      if (__ldg(skey + m) <= kv) z = m + 1;
      else b2 = m;
    }
  }
  vlo = a;
  vhi = z;
  return true;
}

// squared gap, in linking-cell units, between the run's record box and the
// neighbour cell at offset o (both in the run's SOD-cell frame)
__device__ __forceinline__ float box_gap2(const RunGeo &u, int ox, int oy, int oz, const float lo[3],
                                          const float hi[3]) {
  const float bx = (float)(u.fx + ox), by = (float)(u.fy + oy), bz = (float)(u.fz + oz);
  const float gx = fmaxf(fmaxf(bx - hi[0], lo[0] - (bx + 1.f)), 0.f);
  const float gy = fmaxf(fmaxf(by - hi[1], lo[1] - (by + 1.f)), 0.f);
  const float gz = fmaxf(fmaxf(bz - hi[2], lo[2] - (bz + 1.f)), 0.f);
  return gx * gx + gy * gy + gz * gz;
}

// Linking runs in two passes (the sampling scheme of Afforest, Sutton et
// al. 2018).  The first pass joins each short run to at most FOF_SAMPLE
// friends and each long run to the friends among FOF_SAMPLE_WARP
// neighbouring runs, which already builds most of every large group (one
// friend per run, or six, measured slower at 512^3 and 1024^3); after
// a compression every position points at its root, so in the full pass a
// neighbour run with the same parent is skipped with two loads instead of
// two path walks.  Both passes test the same pairs' friendship, so the
// components are the same as without sampling.
constexpr int FOF_SAMPLE = 3;       // friends a thread's run joins in the first pass
constexpr int FOF_SAMPLE_WARP = 2;  // neighbour runs a warp's run examines in the first pass

// A thread per run of up to FOF_THREAD_RUN records; longer runs are listed
// (in the first pass) for k_fof_link_warp.  The neighbour cells are walked
// row by row: for each (dy, dz) of the half space whose row of linking
// cells comes within reach of the run's records, the cells of the row that
// do form one key range inside each SOD cell the row crosses, found with
// one search; every record of the range is then tested.  A friend joins the
// two components; in the full pass a record whose parent is the run's
// parent (both compressed) needs no test.
template <bool FULL>
__global__ void __launch_bounds__(FOF_TPB, 3) k_fof_link_thread(const unsigned *heads, long long nrun, FofGeo G,
                                                             const unsigned *cs, const unsigned short *skey,
                                                             const unsigned *perm, const float4 *cube,
                                                             unsigned *par, unsigned *bigrun, unsigned *nbigrun,
                                                             unsigned long long *counters) {
  unsigned long long tests = 0, pairs = 0;
  const int R = G.R;
  const float reach2 = (float)G.reach2;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nrun;
       q += (long long)gridDim.x * blockDim.x) {
    const unsigned h = heads[q], e = heads[q + 1];
    if (e - h > FOF_THREAD_RUN) {
      if (!FULL) bigrun[atomicAdd(nbigrun, 1u)] = (unsigned)q;
      continue;
    }
    const unsigned m = e - h;
    float4 ur[FOF_THREAD_RUN];
    float lo[3], hi[3];
    ur[0] = cube[perm[h]];
    const RunGeo u = run_geo(ur[0], G, lo, hi);
#pragma unroll
    for (unsigned j = 1; j < FOF_THREAD_RUN; j++) {
      if (j < m) {
        ur[j] = cube[perm[h + j]];
        int c, f;
        float pp;
        fof_axis(ur[j].x, G, c, f, pp);
        lo[0] = fminf(lo[0], pp);
        hi[0] = fmaxf(hi[0], pp);
        fof_axis(ur[j].y, G, c, f, pp);
        lo[1] = fminf(lo[1], pp);
        hi[1] = fmaxf(hi[1], pp);
        fof_axis(ur[j].z, G, c, f, pp);
        lo[2] = fminf(lo[2], pp);
        hi[2] = fmaxf(hi[2], pp);
      }
    }
    const unsigned myroot = FULL ? __ldcg(par + h) : 0u;
    int found = 0;
    for (int oz = 0; oz <= R && found < FOF_SAMPLE; oz++) {
      const float bz = (float)(u.fz + oz);
      const float gz = fmaxf(fmaxf(bz - hi[2], lo[2] - (bz + 1.f)), 0.f);
      if (gz * gz > reach2) continue;
      for (int oy = (oz == 0 ? 0 : -R); oy <= R && found < FOF_SAMPLE; oy++) {
        const float by = (float)(u.fy + oy);
        const float gy = fmaxf(fmaxf(by - hi[1], lo[1] - (by + 1.f)), 0.f);
        const float left = reach2 - gz * gz - gy * gy;
        if (left < 0.f) continue;
        const float rx = sqrtf(left);
        // cells of the row within reach, in the run's SOD-cell frame
        int xa = (int)floorf(lo[0] - rx), xb = (int)floorf(hi[0] + rx);
        xa = max(xa, u.fx - R);
        xb = min(xb, u.fx + R);
        if (oz == 0 && oy == 0) xa = max(xa, u.fx + 1);  // own row: cells after the run's
        if (xa > xb) continue;
        // the row's SOD cells in y and z
        int ty = u.fy + oy, tz = u.fz + oz;
        const int dcy = ty < 0 ? -1 : (ty >= G.k ? 1 : 0), dcz = tz < 0 ? -1 : (tz >= G.k ? 1 : 0);
        ty -= dcy * G.k;
        tz -= dcz * G.k;
        int cy = u.cy + dcy, cz = u.cz + dcz;
        cy = cy < 0 ? cy + G.nx : (cy >= G.nx ? cy - G.nx : cy);
        cz = cz < 0 ? cz + G.nx : (cz >= G.nx ? cz - G.nx : cz);
        // up to three SOD cells along x
        for (int dcx = -1; dcx <= 1 && found < FOF_SAMPLE; dcx++) {
          const int s0 = max(xa, dcx * G.k), s1 = min(xb, dcx * G.k + G.k - 1);
          if (s0 > s1) continue;
          int cx = u.cx + dcx;
          cx = cx < 0 ? cx + G.nx : (cx >= G.nx ? cx - G.nx : cx);
          const unsigned long long c = (unsigned long long)cx +
                                       (unsigned long long)G.nx * ((unsigned long long)cy + (unsigned long long)G.nx * cz);
          const unsigned clo = __ldg(cs + c), chi = __ldg(cs + c + 1);
          if (clo == chi) continue;
          const unsigned rowkey = (unsigned)(G.k * (ty + G.k * tz));
          const unsigned k0 = rowkey + (unsigned)(s0 - dcx * G.k), k1 = rowkey + (unsigned)(s1 - dcx * G.k);
          unsigned v = clo;
          if (chi - clo <= 16) {
            while (v < chi && __ldg(skey + v) < k0) v++;
          } else {
            unsigned b2 = chi;
            while (v < b2) {
              const unsigned mid = (v + b2) >> 1;
              if (__ldg(skey + mid) < k0) v = mid + 1;
              else b2 = mid;
            }
          }
          pairs++;
          for (; v < chi && __ldg(skey + v) <= k1; v++) {
            if (FULL && __ldcg(par + v) == myroot) continue;
            const float4 bv = cube[perm[v]];
            bool hit = false;
#pragma unroll
            for (unsigned j = 0; j < FOF_THREAD_RUN; j++) {
              if (j < m && !hit) {
                tests++;
                hit = fof_friends(ur[j], bv, G.r2, G.rT);
              }
            }
            if (hit) {
              uf_union(par, h, v);
              if (!FULL && ++found >= FOF_SAMPLE) break;
            }
          }
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    tests += __shfl_down_sync(0xffffffffu, tests, o);
    pairs += __shfl_down_sync(0xffffffffu, pairs, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(counters, tests);
    atomicAdd(counters + 1, pairs);
  }
}

// A warp per long run: lanes take the run's records, the neighbour run's
// records are walked in order, and the warp stops at the first friend pair.
template <bool FULL>
__global__ void __launch_bounds__(FOF_TPB) k_fof_link_warp(const unsigned *heads, const unsigned *bigrun,
                                                           const unsigned *nbigrun, FofGeo G, const unsigned *cs,
                                                           const unsigned short *skey, const unsigned *perm,
                                                           const float4 *cube, unsigned *par,
                                                           unsigned long long *counters) {
  const int lane = threadIdx.x & 31;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
  const unsigned nb = *nbigrun;
  unsigned long long tests = 0, pairs = 0;
  for (long long w = warp; w < nb; w += nwarp) {
    const unsigned q = bigrun[w];
    const unsigned h = heads[q], e = heads[q + 1];
    float lo[3], hi[3];
    const RunGeo u = run_geo(cube[perm[h]], G, lo, hi);
    // the run's nominal linking cell as its box
    lo[0] = (float)u.fx;
    hi[0] = (float)(u.fx + 1);
    lo[1] = (float)u.fy;
    hi[1] = (float)(u.fy + 1);
    lo[2] = (float)u.fz;
    hi[2] = (float)(u.fz + 1);
    int sampled = 0;  // neighbour runs examined (warp-uniform)
    for (int o = 0; o < G.noff && (FULL || sampled < FOF_SAMPLE_WARP); o++) {
      const int ox = c_fof_off[3 * o], oy = c_fof_off[3 * o + 1], oz = c_fof_off[3 * o + 2];
      if (box_gap2(u, ox, oy, oz, lo, hi) > (float)G.reach2) continue;
      unsigned vlo, vhi;
      if (!find_run(u, ox, oy, oz, G, cs, skey, vlo, vhi)) continue;
      if (vlo == h) continue;
      sampled++;
      if (lane == 0) pairs++;
      if (FULL && __ldcg(par + h) == __ldcg(par + vlo)) continue;
      bool hit = false;
      for (unsigned ub = h; ub < e && !hit; ub += 32) {
        const unsigned uu = ub + (unsigned)lane;
        const bool have = uu < e;
        const float4 a = have ? cube[perm[uu]] : make_float4(0.f, 0.f, 0.f, 0.f);
        bool mine = false;
        for (unsigned v = vlo; v < vhi; v++) {
          const float4 bv = cube[perm[v]];
          if (have) {
            tests++;
            mine = mine || fof_friends(a, bv, G.r2, G.rT);
          }
          if (((v - vlo) & 7u) == 7u && __any_sync(0xffffffffu, mine)) break;
        }
        hit = __any_sync(0xffffffffu, mine);
      }
      if (hit && lane == 0) uf_union(par, h, vlo);
      __syncwarp();
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    tests += __shfl_down_sync(0xffffffffu, tests, o);
    pairs += __shfl_down_sync(0xffffffffu, pairs, o);
  }
  if (lane == 0) {
    atomicAdd(counters, tests);
    atomicAdd(counters + 1, pairs);
  }
}

// every position points at its component's root (no unions run meanwhile;
// each thread stores only its own position's entry)
__global__ void k_fof_compress(unsigned *par, long long n) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) __stcg(par + p, uf_root(par, (unsigned)p));
}

// ---------------------------------------------------------------------------
// 3. groups, labels, members, observables
// ---------------------------------------------------------------------------
// size and lowest input index per root (one atomic per root and warp)
__global__ void k_fof_root_stats(const unsigned *par, const unsigned *perm, const float4 *cube, long long n,
                                 unsigned *size, unsigned *minidx) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool have = p < n;
  const unsigned root = have ? par[p] : 0xffffffffu;
  const unsigned idx = have ? (__float_as_uint(cube[perm[p]].w) & ~PSOD_DEAD_BIT) : 0xffffffffu;
  auto warp = cg::tiled_partition<32>(cg::this_thread_block());
  auto grp = cg::labeled_partition(warp, root);
  const unsigned mn = cg::reduce(grp, idx, cg::less<unsigned>());
  if (have && grp.thread_rank() == 0) {
    atomicAdd(size + root, grp.size());
    atomicMin(minidx + root, mn);
  }
}

// roots of halos (size >= mmin)
__global__ void k_fof_halo_flags(const unsigned *par, const unsigned *size, long long n, unsigned mmin,
                                 unsigned *flag) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) flag[p] = (par[p] == (unsigned)p && size[p] >= mmin) ? 1u : 0u;
}

// (label, root) pairs of the halos; the label orders as a signed int64
__global__ void k_fof_halo_keys(const unsigned *flag, const unsigned *pos, long long n, const unsigned *minidx,
                                const long long *ids, unsigned long long *hkey, unsigned *hroot) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n && flag[p]) {
    const unsigned q = pos[p];
    hkey[q] = (unsigned long long)ids[minidx[p]] ^ 0x8000000000000000ull;
    hroot[q] = (unsigned)p;
  }
}

// halo rank of each root (in minidx, which is free now), IDs and masses
__global__ void k_fof_halo_rank(const unsigned long long *hkey, const unsigned *hroot, long long nh,
                                const unsigned *size, unsigned *rank, long long *hid, long long *hmass,
                                unsigned *mcount) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < nh) {
    const unsigned r = hroot[q];
    rank[r] = (unsigned)q;
    hid[q] = (long long)(hkey[q] ^ 0x8000000000000000ull);
    hmass[q] = size[r];
    mcount[q] = size[r];
  }
}

// members in input order: flags, then (halo rank, input index) compacted
__global__ void k_fof_member_flags(const unsigned *finv, const unsigned *par, const unsigned *size, long long n,
                                   unsigned mmin, unsigned *flag) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = size[par[finv[i]]] >= mmin ? 1u : 0u;
}

__global__ void k_fof_member_pairs(const unsigned *flag, const unsigned *pos, const unsigned *finv,
                                   const unsigned *par, const unsigned *rank, long long n, unsigned *mkey,
                                   unsigned *mval) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && flag[i]) {
    const unsigned q = pos[i];
    mkey[q] = rank[par[finv[i]]];
    mval[q] = (unsigned)i;
  }
}

__global__ void k_fof_offsets(const unsigned *excl, long long nh, long long nm, long long *off) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < nh) off[q] = excl[q];
  if (q == nh) off[q] = nm;
}

// Centre of mass (computecom): FP64 sums of the member positions, each
// unwrapped by one box against the halo's first member where the two lie
// more than half a box apart (the reference unwraps against the running
// mean; for a halo smaller than a quarter box the two agree), then the mean
// wrapped into [0,1].  Mean velocity.  Radius (computeradius): the largest
// distance from the centre with the reference's per-axis rule
// |d| > 0.5 -> 1 - |d|, in FP64 without contraction.
template <int NT>
__device__ __forceinline__ void halo_observables(const unsigned *mem, long long b, long long e, const float4 *cube,
                                                 const unsigned *inv, const float *vel, double *com, double *hvel,
                                                 double *rad, double *red, float4 *feat) {
  const int t = threadIdx.x % NT;
  const float4 first = cube[inv[mem[b]]];
  const double f0 = fof_wrap1(first.x), f1 = fof_wrap1(first.y), f2 = fof_wrap1(first.z);
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (long long k = b + t; k < e; k += NT) {
    const unsigned i = mem[k];
    const float4 v = cube[inv[i]];
    double x[3] = {fof_wrap1(v.x), fof_wrap1(v.y), fof_wrap1(v.z)};
    const double f[3] = {f0, f1, f2};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double dl = dsub(f[a], x[a]);
      if (dl > 0.5) x[a] = dadd(x[a], 1.0);
      else if (dl < -0.5) x[a] = dsub(x[a], 1.0);
      s[a] = dadd(s[a], x[a]);
    }
    if (vel) {
#pragma unroll
      for (int a = 0; a < 3; a++) s[3 + a] = dadd(s[3 + a], (double)vel[3ull * i + a]);
    }
  }
  // fixed-order reduction: warp tree, then (CTA) the warps' partials in order
#pragma unroll
  for (int a = 0; a < 6; a++)
    for (int o = 16; o > 0; o >>= 1) s[a] = dadd(s[a], __shfl_down_sync(0xffffffffu, s[a], o));
  if (NT > 32) {
    const int w = t >> 5, lane = t & 31;
    if (lane == 0)
      for (int a = 0; a < 6; a++) red[6 * w + a] = s[a];
    __syncthreads();
    if (t == 0)
      for (int a = 0; a < 6; a++) {
        double acc = red[a];
        for (int q = 1; q < NT / 32; q++) acc = dadd(acc, red[6 * q + a]);
        s[a] = acc;
      }
    __syncthreads();
  }
  __shared__ double s_c[FOF_TPB / 32][3];
  const int slot = (threadIdx.x / NT) % (FOF_TPB / 32);
  const double mass = (double)(e - b);
  if (t == 0) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      double c = ddiv(s[a], mass);
      if (c > 1.0) c = dsub(c, 1.0);
      if (c < 0.0) c = dadd(c, 1.0);
      s_c[slot][a] = c;
      com[a] = c;
      hvel[a] = vel ? ddiv(s[3 + a], mass) : 0.0;
    }
  }
  if (NT > 32) __syncthreads();
  else __syncwarp();
  const double c0 = s_c[slot][0], c1 = s_c[slot][1], c2 = s_c[slot][2];
  double rmax2 = 0.0;
  // shape sums for the learned bracket's features: squared distances and
  // the inertia tensor of the minimum-image offsets from the centre
  double sh[7] = {0, 0, 0, 0, 0, 0, 0};
  for (long long k = b + t; k < e; k += NT) {
    const float4 v = cube[inv[mem[k]]];
    double d0 = dsub((double)fof_wrap1(v.x), c0), d1 = dsub((double)fof_wrap1(v.y), c1),
           d2 = dsub((double)fof_wrap1(v.z), c2);
    const double s0 = d0 > 0.5 ? d0 - 1.0 : (d0 < -0.5 ? d0 + 1.0 : d0);
    const double s1 = d1 > 0.5 ? d1 - 1.0 : (d1 < -0.5 ? d1 + 1.0 : d1);
    const double s2 = d2 > 0.5 ? d2 - 1.0 : (d2 < -0.5 ? d2 + 1.0 : d2);
    sh[0] += s0 * s0 + s1 * s1 + s2 * s2;
    sh[1] += s0 * s0;
    sh[2] += s0 * s1;
    sh[3] += s0 * s2;
    sh[4] += s1 * s1;
    sh[5] += s1 * s2;
    sh[6] += s2 * s2;
    if (fabs(d0) > 0.5) d0 = dsub(1.0, fabs(d0));
    if (fabs(d1) > 0.5) d1 = dsub(1.0, fabs(d1));
    if (fabs(d2) > 0.5) d2 = dsub(1.0, fabs(d2));
    const double q = dadd(dadd(dmul(d0, d0), dmul(d1, d1)), dmul(d2, d2));
    rmax2 = fmax(rmax2, q);
  }
  for (int o = 16; o > 0; o >>= 1) rmax2 = fmax(rmax2, __shfl_down_sync(0xffffffffu, rmax2, o));
#pragma unroll
  for (int a = 0; a < 7; a++)
    for (int o = 16; o > 0; o >>= 1) sh[a] += __shfl_down_sync(0xffffffffu, sh[a], o);
  if (NT > 32) {
    const int w = t >> 5, lane = t & 31;
    if (lane == 0) {
      red[w] = rmax2;
      for (int a = 0; a < 7; a++) red[NT / 32 + 7 * w + a] = sh[a];
    }
    __syncthreads();
    if (t == 0) {
      for (int q = 1; q < NT / 32; q++) rmax2 = fmax(rmax2, red[q]);
      for (int a = 0; a < 7; a++) {
        double acc = red[NT / 32 + a];
        for (int q = 1; q < NT / 32; q++) acc += red[NT / 32 + 7 * q + a];
        sh[a] = acc;
      }
    }
    __syncthreads();
  }
  if (t == 0) {
    *rad = dsqrt(rmax2);
    const double n = (double)(e - b);
    double A[3][3] = {{sh[1] / n, sh[2] / n, sh[3] / n}, {sh[2] / n, sh[4] / n, sh[5] / n},
                      {sh[3] / n, sh[5] / n, sh[6] / n}};
    double dv[3], vv[3][3];
    jacobi3(A, dv, vv);
    eigsort3(dv, vv);
    const double ea = sqrt(fmax(dv[0], 0.0)), eb = sqrt(fmax(dv[1], 0.0)), ec = sqrt(fmax(dv[2], 0.0));
    *feat = make_float4((float)sqrt(sh[0] / n), ea > 0.0 ? (float)(eb / ea) : 1.f, ea > 0.0 ? (float)(ec / ea) : 1.f,
                        eb > 0.0 ? (float)(ec / eb) : 1.f);
  }
}

__global__ void __launch_bounds__(FOF_TPB) k_fof_observables_warp(const long long *off, const long long *hmass,
                                                                  long long nh, const unsigned *mem,
                                                                  const float4 *cube, const unsigned *inv,
                                                                  const float *vel, double *com, double *hvel,
                                                                  double *rad, float4 *feat) {
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long q = warp; q < nh; q += nwarp) {
    if (hmass[q] > FOF_WARP_HALO) continue;  // warp-uniform
    halo_observables<32>(mem, off[q], off[q + 1], cube, inv, vel, com + 3 * q, hvel + 3 * q, rad + q, nullptr,
                         feat + q);
  }
}

__global__ void __launch_bounds__(FOF_TPB) k_fof_observables_cta(const long long *off, const long long *hmass,
                                                                 long long nh, const unsigned *mem,
                                                                 const float4 *cube, const unsigned *inv,
                                                                 const float *vel, double *com, double *hvel,
                                                                 double *rad, float4 *feat) {
  __shared__ double red[6 * (FOF_TPB / 32) + 7 * (FOF_TPB / 32)];
  for (long long q = blockIdx.x; q < nh; q += gridDim.x) {
    if (hmass[q] <= FOF_WARP_HALO) continue;  // block-uniform
    halo_observables<FOF_TPB>(mem, off[q], off[q + 1], cube, inv, vel, com + 3 * q, hvel + 3 * q, rad + q, red,
                              feat + q);
  }
}

// per input particle: its halo's rank, or (top bit) the size of its group
// when that group is smaller than mmin (the learned bracket's features)
__global__ void k_fof_codes(const unsigned *finv, const unsigned *par, const unsigned *size, const unsigned *rank,
                            long long n, unsigned mmin, unsigned *code) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned r = par[finv[i]], sz = size[r];
  code[i] = sz >= mmin ? rank[r] : (0x80000000u | sz);
}

__global__ void k_fof_member_ids(const unsigned *mem, long long nm, const long long *ids, long long *out_idx,
                                 long long *out_id) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nm) return;
  const unsigned i = mem[k];
  if (out_idx) out_idx[k] = (long long)i;
  if (out_id) out_id[k] = ids[i];
}

unsigned grid_for(long long n, int tpb = FOF_TPB) { return (unsigned)((n + tpb - 1) / tpb); }

struct EvTimer {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t s;
  explicit EvTimer(cudaStream_t st) : s(st) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
  }
  double stop() {
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventRecord(a, s);
    return ms;
  }
  ~EvTimer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

}  // namespace

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
int fof_geometry(const psod_ctx *c, const psod_fof_params *p, long long nres, int *k_out, int *reach_out,
                 double *reach2_out, std::vector<signed char> *offs) {
  // linking length in SOD cells, and the largest rounding of a grid
  // coordinate (FP32 x * nx, then the FP64 shift)
  const double lcell = (double)p->percolation * (double)c->nx / (double)nres;
  const double eps = (double)c->nx * 0x1p-24 + 1e-9;
  if (!(lcell > 0.0) || lcell > 0.5) return PSOD_ERR_ARG;
  // diagonal of a linking cell plus twice the rounding below the linking
  // length (all of a cell's particles are friends), with slack for the FP32
  // test
  const double room = lcell * (1.0 - 1e-5) - 2.0 * std::sqrt(3.0) * eps;
  if (room <= 0.0) return PSOD_ERR_ARG;
  const int k = (int)std::ceil(std::sqrt(3.0) / room);
  if (k < 1 || k > 32) return PSOD_ERR_ARG;
  // reach: a friend pair's linking cells differ by at most R per axis
  const double lk = (lcell * (1.0 + 1e-5) + 2.0 * eps) * k;
  const int R = (int)std::floor(lk) + 1;
  if (R >= k || R > 3) return PSOD_ERR_ARG;
  offs->clear();
  for (int oz = -R; oz <= R; oz++)
    for (int oy = -R; oy <= R; oy++)
      for (int ox = -R; ox <= R; ox++) {
        // the half space: (oz, oy, ox) > 0 lexicographically
        if (oz < 0 || (oz == 0 && (oy < 0 || (oy == 0 && ox <= 0)))) continue;
        const double gx = std::max(std::abs(ox) - 1, 0), gy = std::max(std::abs(oy) - 1, 0),
                     gz = std::max(std::abs(oz) - 1, 0);
        if (gx * gx + gy * gy + gz * gz > lk * lk) continue;
        offs->push_back((signed char)ox);
        offs->push_back((signed char)oy);
        offs->push_back((signed char)oz);
      }
  *k_out = k;
  *reach_out = R;
  *reach2_out = lk * lk;
  return PSOD_OK;
}

}  // namespace psod

using namespace psod;

extern "C" {

int psod_fof(psod_ctx *c, const psod_fof_params *p, psod_fof_stats *stats) {
  if (!c || !p) return PSOD_ERR_ARG;
  if (!c->d_cube || c->n <= 0) return set_err(c, PSOD_ERR_STATE, "no particles: call psod_load_particles first");
  // pFoF's own domain decomposition is not the SOD zones: the finder runs
  // on a one-zone context (the whole periodic box)
  if (c->nxcpu != 1) return set_err(c, PSOD_ERR_ARG, "psod_fof needs a one-zone context (nxcpu = 1)");
  cudaSetDevice(c->device);
  c->fof_done = false;
  const long long n = c->n;
  long long nres = p->nres;
  if (nres == 0) nres = (long long)std::llround(std::cbrt((double)n));
  if (nres < 1 || !(p->percolation > 0.0f) || p->mmin < 1 || p->mmin > 0x7fffffff)
    return set_err(c, PSOD_ERR_ARG, "psod_fof: percolation > 0, nres >= 1 and 1 <= mmin < 2^31 are required");
  // the reference refuses percolation * refine_fof >= 1 (modfofpara.f90:101-117)
  if (p->percolation * 2.0f >= 1.0f) return set_err(c, PSOD_ERR_ARG, "psod_fof: percolation must be below 0.5");
  int k = 0, R = 0;
  double reach2 = 0;
  std::vector<signed char> offs;
  if (fof_geometry(c, p, nres, &k, &R, &reach2, &offs))
    return set_err(c, PSOD_ERR_ARG,
                   "psod_fof: the linking length must lie between about 0.06 and 0.5 SOD cells (percolation * nx / nres)");
  int st = wait_ids(c);
  if (st) return st;
  FofGeo G;
  G.nx = c->nx;
  G.nxf = (float)c->nx;
  G.xs = c->xxmin[0] * c->scale;  // one zone: the same on every axis
  G.k = k;
  G.R = R;
  G.reach2 = reach2;
  G.noff = (int)(offs.size() / 3);
  G.rT = p->percolation / (float)nres;  // FP32, as rT = r / size
  G.r2 = G.rT * G.rT;
  G.ncell = c->ncell;
  PSOD_CUDA(c, cudaMemcpyToSymbolAsync(c_fof_off, offs.data(), offs.size(), 0, cudaMemcpyHostToDevice, c->stream));

  psod_fof_stats S{};
  EvTimer tm(c->stream), total(c->stream);
  unsigned short *key = nullptr, *skey = nullptr;
  unsigned *perm = nullptr, *par = nullptr, *finv = nullptr, *aux1 = nullptr, *aux2 = nullptr, *big = nullptr,
           *cnt = nullptr;
  unsigned long long *ctr = nullptr;
  if ((st = scratch(c, SLOT_FOF_KEY, (size_t)n, &key))) return st;
  if ((st = scratch(c, SLOT_FOF_SKEY, (size_t)n, &skey))) return st;
  if ((st = scratch(c, SLOT_FOF_PERM, (size_t)n, &perm))) return st;
  if ((st = scratch(c, SLOT_FOF_PAR, (size_t)n, &par))) return st;
  if ((st = scratch(c, SLOT_FOF_INV, (size_t)n, &finv))) return st;
  if ((st = scratch(c, SLOT_FOF_AUX1, (size_t)n + 1, &aux1))) return st;
  if ((st = scratch(c, SLOT_FOF_AUX2, (size_t)n + 1, &aux2))) return st;
  if ((st = scratch(c, SLOT_FOF_CNT, 8, &cnt))) return st;
  if ((st = scratch(c, SLOT_FOF_CTR, 4, &ctr))) return st;
  PSOD_CUDA(c, cudaMemsetAsync(cnt, 0, 8 * sizeof(unsigned), c->stream));
  PSOD_CUDA(c, cudaMemsetAsync(ctr, 0, 4 * sizeof(unsigned long long), c->stream));

  // 1. keys and the per-cell sort (big cells listed in aux2)
  k_fof_keys<<<grid_for(n), FOF_TPB, 0, c->stream>>>(c->d_cube, n, G, key);
  big = aux2;
  k_fof_sort_small<<<grid_for((long long)c->ncell), FOF_TPB, 0, c->stream>>>(
      c->d_cell_start, c->ncell, key, c->d_cube, perm, skey, par, finv, big, cnt);
  const int nbins = k * k * k;
  PSOD_CUDA(c, cudaFuncSetAttribute(k_fof_sort_big, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(nbins * sizeof(unsigned))));
  k_fof_sort_big<<<1184, FOF_TPB, nbins * sizeof(unsigned), c->stream>>>(c->d_cell_start, big, cnt, nbins, key,
                                                                         c->d_cube, perm, skey, par, finv);
  PSOD_CUDA(c, cudaGetLastError());
  // run heads: flags in aux1, their exclusive scan in aux2, then the list
  k_fof_head_flags<<<grid_for(n), FOF_TPB, 0, c->stream>>>(par, n, aux1);
  if ((st = scan_u32(c, aux1, aux2, n, true))) return st;
  unsigned nrun_u = 0;
  PSOD_CUDA(c, cudaMemcpyAsync(&nrun_u, aux2 + n, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  const long long nrun = nrun_u;
  unsigned *heads = nullptr, *bigrun = nullptr;
  if ((st = scratch(c, SLOT_FOF_HEADS, (size_t)nrun + 1, &heads))) return st;
  if ((st = scratch(c, SLOT_FOF_BIGRUN, (size_t)nrun + 1, &bigrun))) return st;
  k_fof_head_list<<<grid_for(n), FOF_TPB, 0, c->stream>>>(aux1, aux2, n, heads);
  PSOD_CUDA(c, cudaGetLastError());
  S.ms_sort = tm.stop();
  S.fine_cells = nrun;

  // 2. linking: sampled pass, compression, full pass, compression
  k_fof_link_thread<false><<<148 * 8, FOF_TPB, 0, c->stream>>>(heads, nrun, G, c->d_cell_start, skey, perm,
                                                               c->d_cube, par, bigrun, cnt + 1, ctr);
  k_fof_link_warp<false><<<148 * 8, FOF_TPB, 0, c->stream>>>(heads, bigrun, cnt + 1, G, c->d_cell_start, skey,
                                                             perm, c->d_cube, par, ctr);
  k_fof_compress<<<grid_for(n), FOF_TPB, 0, c->stream>>>(par, n);
  k_fof_link_thread<true><<<148 * 8, FOF_TPB, 0, c->stream>>>(heads, nrun, G, c->d_cell_start, skey, perm,
                                                              c->d_cube, par, bigrun, cnt + 1, ctr);
  k_fof_link_warp<true><<<148 * 8, FOF_TPB, 0, c->stream>>>(heads, bigrun, cnt + 1, G, c->d_cell_start, skey,
                                                            perm, c->d_cube, par, ctr);
  k_fof_compress<<<grid_for(n), FOF_TPB, 0, c->stream>>>(par, n);
  PSOD_CUDA(c, cudaGetLastError());
  S.ms_link = tm.stop();

  // 3. sizes and lowest input index per root (aux1 = size, aux2 = minidx)
  PSOD_CUDA(c, cudaMemsetAsync(aux1, 0, sizeof(unsigned) * n, c->stream));
  PSOD_CUDA(c, cudaMemsetAsync(aux2, 0xff, sizeof(unsigned) * n, c->stream));
  k_fof_root_stats<<<grid_for(n), FOF_TPB, 0, c->stream>>>(par, perm, c->d_cube, n, aux1, aux2);
  // halo roots: flags in perm's storage (perm is not read after this)
  unsigned *hflag = perm;
  unsigned *hpos = nullptr;
  if ((st = scratch(c, SLOT_FOF_HPOS, (size_t)n + 1, &hpos))) return st;
  // group count: roots (every root has size >= 1)
  k_fof_halo_flags<<<grid_for(n), FOF_TPB, 0, c->stream>>>(par, aux1, n, 1u, hflag);
  if ((st = scan_u32(c, hflag, hpos, n, true))) return st;
  unsigned ngroups = 0;
  PSOD_CUDA(c, cudaMemcpyAsync(&ngroups, hpos + n, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
  k_fof_halo_flags<<<grid_for(n), FOF_TPB, 0, c->stream>>>(par, aux1, n, (unsigned)p->mmin, hflag);
  if ((st = scan_u32(c, hflag, hpos, n, true))) return st;
  unsigned nh_u = 0;
  PSOD_CUDA(c, cudaMemcpyAsync(&nh_u, hpos + n, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  const long long nh = nh_u;
  S.ngroups = ngroups;
  unsigned long long *hkey = nullptr;
  unsigned *hroot = nullptr, *mcount = nullptr;
  if ((st = scratch(c, SLOT_FOF_HKEY, (size_t)nh + 1, &hkey))) return st;
  if ((st = scratch(c, SLOT_FOF_HROOT, (size_t)nh + 1, &hroot))) return st;
  if ((st = scratch(c, SLOT_FOF_MCOUNT, (size_t)nh + 1, &mcount))) return st;
  k_fof_halo_keys<<<grid_for(n), FOF_TPB, 0, c->stream>>>(hflag, hpos, n, aux2, c->d_ids, hkey, hroot);
  PSOD_CUDA(c, cudaGetLastError());
  if (nh > 1 && (st = radix_sort_u64(c, hkey, hroot, nh, 64))) return st;
  long long *hid = nullptr, *hmass = nullptr, *hoff = nullptr;
  double *hcom = nullptr, *hvel = nullptr, *hrad = nullptr;
  if ((st = scratch(c, SLOT_F_ID, (size_t)nh + 1, &hid))) return st;
  if ((st = scratch(c, SLOT_F_MASS, (size_t)nh + 1, &hmass))) return st;
  if ((st = scratch(c, SLOT_F_OFF, (size_t)nh + 1, &hoff))) return st;
  if ((st = scratch(c, SLOT_F_COM, (size_t)3 * nh + 3, &hcom))) return st;
  if ((st = scratch(c, SLOT_F_VEL, (size_t)3 * nh + 3, &hvel))) return st;
  if ((st = scratch(c, SLOT_F_RAD, (size_t)nh + 1, &hrad))) return st;
  if (nh > 0)
    k_fof_halo_rank<<<grid_for(nh), FOF_TPB, 0, c->stream>>>(hkey, hroot, nh, aux1, aux2, hid, hmass, mcount);
  // members: flags over input indices (hflag reused), compacted pairs, then a
  // stable sort on the halo rank keeps ascending input order inside a halo
  k_fof_member_flags<<<grid_for(n), FOF_TPB, 0, c->stream>>>(finv, par, aux1, n, (unsigned)p->mmin, hflag);
  if ((st = scan_u32(c, hflag, hpos, n, true))) return st;
  unsigned nm_u = 0;
  PSOD_CUDA(c, cudaMemcpyAsync(&nm_u, hpos + n, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  const long long nm = nm_u;
  unsigned *mkey = nullptr, *mem = nullptr;
  if ((st = scratch(c, SLOT_FOF_MKEY, (size_t)nm + 1, &mkey))) return st;
  if ((st = scratch(c, SLOT_F_MEM, (size_t)nm + 1, &mem))) return st;
  k_fof_member_pairs<<<grid_for(n), FOF_TPB, 0, c->stream>>>(hflag, hpos, finv, par, aux2, n, mkey, mem);
  PSOD_CUDA(c, cudaGetLastError());
  if (nm > 1 && nh > 1) {
    int bits = 1;
    while ((1ll << bits) < nh) bits++;
    if ((st = radix_sort_u32(c, mkey, mem, nm, bits))) return st;
  }
  // offsets: exclusive scan of the masses in rank order
  if (nh > 0) {
    if ((st = scan_u32(c, mcount, mcount, nh, false))) return st;
  }
  k_fof_offsets<<<grid_for(nh + 1), FOF_TPB, 0, c->stream>>>(mcount, nh, nm, hoff);
  PSOD_CUDA(c, cudaGetLastError());
  S.ms_label = tm.stop();

  // 4. observables, and each particle's group code
  float4 *hfeat = nullptr;
  unsigned *pcode = nullptr;
  if ((st = scratch(c, SLOT_F_FEAT, (size_t)nh + 1, &hfeat))) return st;
  if ((st = scratch(c, SLOT_F_CODE, (size_t)n, &pcode))) return st;
  if (nh > 0) {
    const float *vel = c->d_vel;
    k_fof_observables_warp<<<148 * 8, FOF_TPB, 0, c->stream>>>(hoff, hmass, nh, mem, c->d_cube, c->d_inv, vel, hcom,
                                                               hvel, hrad, hfeat);
    k_fof_observables_cta<<<148 * 2, FOF_TPB, 0, c->stream>>>(hoff, hmass, nh, mem, c->d_cube, c->d_inv, vel, hcom,
                                                              hvel, hrad, hfeat);
    PSOD_CUDA(c, cudaGetLastError());
  }
  k_fof_codes<<<grid_for(n), FOF_TPB, 0, c->stream>>>(finv, par, aux1, aux2, n, (unsigned)p->mmin, pcode);
  PSOD_CUDA(c, cudaGetLastError());
  S.ms_props = tm.stop();
  unsigned long long hc[2] = {0, 0};
  PSOD_CUDA(c, cudaMemcpyAsync(hc, ctr, sizeof(hc), cudaMemcpyDeviceToHost, c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  S.ms_total = total.stop();
  S.pair_tests = (int64_t)hc[0];
  S.cell_pairs = (int64_t)hc[1];
  S.nhalo = nh;
  S.nmember = nm;
  c->fof_nhalo = nh;
  c->fof_nmember = nm;
  c->fof_n = n;
  c->fof_done = true;
  // the working arrays stay with the context (repeated calls allocate
  // nothing), like the other stages' slots
  if (stats) *stats = S;
  return PSOD_OK;
}

int psod_fof_release(psod_ctx *c) {
  if (!c) return PSOD_ERR_ARG;
  cudaSetDevice(c->device);
  for (int s : {SLOT_FOF_KEY, SLOT_FOF_SKEY, SLOT_FOF_PERM, SLOT_FOF_PAR, SLOT_FOF_INV, SLOT_FOF_AUX1, SLOT_FOF_AUX2,
                SLOT_FOF_HEADS, SLOT_FOF_BIGRUN, SLOT_FOF_HPOS, SLOT_FOF_HKEY, SLOT_FOF_HROOT, SLOT_FOF_MKEY,
                SLOT_FOF_MCOUNT})
    free_scratch_slot(c, s);
  return PSOD_OK;
}

int psod_fof_halo_count(psod_ctx *c, int64_t *nhalo, int64_t *nmember) {
  if (!c) return PSOD_ERR_ARG;
  if (!c->fof_done) return set_err(c, PSOD_ERR_STATE, "no FoF catalogue: call psod_fof first");
  if (nhalo) *nhalo = c->fof_nhalo;
  if (nmember) *nmember = c->fof_nmember;
  return PSOD_OK;
}

int psod_fof_get_halos(psod_ctx *c, const psod_fof_table *t) {
  if (!c || !t) return PSOD_ERR_ARG;
  if (!c->fof_done) return set_err(c, PSOD_ERR_STATE, "no FoF catalogue: call psod_fof first");
  cudaSetDevice(c->device);
  int st = wait_ids(c);
  if (st) return st;
  const long long nh = c->fof_nhalo, nm = c->fof_nmember;
  auto slot = [&](int id) { return c->scratch.size() > (size_t)id ? c->scratch[id].first : nullptr; };
  if (t->halo_id && (st = copy_out(c, t->halo_id, slot(SLOT_F_ID), sizeof(int64_t) * nh))) return st;
  if (t->halo_mass && (st = copy_out(c, t->halo_mass, slot(SLOT_F_MASS), sizeof(int64_t) * nh))) return st;
  if (t->halo_com && (st = copy_out(c, t->halo_com, slot(SLOT_F_COM), sizeof(double) * 3 * nh))) return st;
  if (t->halo_vel && (st = copy_out(c, t->halo_vel, slot(SLOT_F_VEL), sizeof(double) * 3 * nh))) return st;
  if (t->halo_radius && (st = copy_out(c, t->halo_radius, slot(SLOT_F_RAD), sizeof(double) * nh))) return st;
  if (t->member_offset && (st = copy_out(c, t->member_offset, slot(SLOT_F_OFF), sizeof(int64_t) * (nh + 1))))
    return st;
  if ((t->member_index || t->member_id) && nm > 0) {
    long long *d_idx = nullptr, *d_id = nullptr;
    if (t->member_index) {
      if (is_device_ptr(t->member_index)) d_idx = reinterpret_cast<long long *>(t->member_index);
      else if ((st = scratch(c, SLOT_OUT_IDX, (size_t)nm, &d_idx))) return st;
    }
    if (t->member_id) {
      if (is_device_ptr(t->member_id)) d_id = reinterpret_cast<long long *>(t->member_id);
      else if ((st = scratch(c, SLOT_OUT_ID, (size_t)nm, &d_id))) return st;
    }
    k_fof_member_ids<<<grid_for(nm), FOF_TPB, 0, c->stream>>>(static_cast<const unsigned *>(slot(SLOT_F_MEM)), nm,
                                                              c->d_ids, d_idx, d_id);
    PSOD_CUDA(c, cudaGetLastError());
    if (t->member_index && (void *)d_idx != (void *)t->member_index &&
        (st = copy_out(c, t->member_index, d_idx, sizeof(int64_t) * nm)))
      return st;
    if (t->member_id && (void *)d_id != (void *)t->member_id &&
        (st = copy_out(c, t->member_id, d_id, sizeof(int64_t) * nm)))
      return st;
  }
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  return PSOD_OK;
}

}  // extern "C"
