// psod_internal.cuh -- shared definitions of the B200 SOD engine.
//
// Data layout in HBM (one context = one zone of the reference's 1-rank run):
//   cube4[n]        float4, particles sorted by SOD cell (the reference's
//                   linked list, main:1564-1604): x, y, z in box units and
//                   w = input index | DEAD_BIT (bit 31 set once claimed).
//   cell_start[nc+1] uint32 offsets of each cell's run in cube4, nc = nx^3,
//                   cell index = i + nx*(j + nx*k).
//   ids[n], vel[3n] input order.
//   rho[n]          double, input order (cicm1 output).
//   seeds           ranks 0..npart_new-1 -> cube4 position.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/psod.h"

#define PSOD_DEAD_BIT 0x80000000u
#define PSOD_IDX_MASK 0x7fffffffu
#define PSOD_INF_RANK 0xffffffffu
#define PSOD_MAX_BINS 128
#define PSOD_STATIC_MAX_NX 64  // zone limit of psod_cic_rho_static

namespace psod {

// ---------------------------------------------------------------------------
// exact FP64 building blocks: explicit round-to-nearest intrinsics so that no
// multiply-add is ever contracted (the reference is built at -O0)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dsqrt(double a) { return __dsqrt_rn(a); }

// posf = posf*scale stored back to real(4) (main:690).  The double product
// of a float and a float-exact nx is exact, so one correctly rounded float
// multiply gives the same value.
__device__ __forceinline__ float to_grid(float x, float nxf) { return __fmul_rn(x, nxf); }

// SOD cell along one axis (main:1565-1576): floor(x_g - xxmin*scale), wrapped
// once into [0, nx).
__device__ __forceinline__ int sod_cell_axis(float xg, double xs, int nx) {
  double d = dsub((double)xg, xs);
  int i = (int)floor(d);
  if (i < 0) i += nx;
  if (i >= nx) i -= nx;
  return i;
}

// minimum-image squared distance (main:2014-2020 and 1844-1850):
// dx = |xx-xc|; dx = min(dx, nx-dx); d2 = (dx*dx + dy*dy) + dz*dz.
__device__ __forceinline__ double min_image_d2(double xx, double yy, double zz, double xc, double yc,
                                               double zc, double tx) {
  double dx = fabs(dsub(xx, xc));
  double t = dsub(tx, dx);
  dx = dx < t ? dx : t;
  double dy = fabs(dsub(yy, yc));
  t = dsub(tx, dy);
  dy = dy < t ? dy : t;
  double dz = fabs(dsub(zz, zc));
  t = dsub(tx, dz);
  dz = dz < t ? dz : t;
  return dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
}

__device__ __forceinline__ unsigned long long dbits(double d) {
  return (unsigned long long)__double_as_longlong(d);
}
__device__ __forceinline__ double bitsd(unsigned long long b) {
  return __longlong_as_double((long long)b);
}

// periodic signed offset a-b in (-nx/2, nx/2]
__device__ __forceinline__ int pdiff(int a, int b, int nx) {
  int d = a - b;
  if (d > nx / 2) d -= nx;
  if (d <= -((nx + 1) / 2)) d += nx;
  return d;
}

// ---------------------------------------------------------------------------
// parameters shared by the SOD kernels (passed by value)
// ---------------------------------------------------------------------------
struct SodConst {
  int nx;
  int ncut;
  float nxf;
  double xs[3];     // xxmin*scale per axis (grid units)
  double tx;        // taillex = nx (main:1517)
  double scale;     // nx
  double delta;     // seuil
  double delta2;    // seuil2
  double cvol;      // 2/3*twopi (main:2049)
  double munit;     // per-particle mass after main:685
  double mmin;      // Mmin
  long long nsel;
  long long n_total;    // records in the zone
  unsigned mmin_count;  // smallest alive count reaching Mmin
  double zmin[3], zmax[3]; // utile zone per axis in grid units (main:691-696)
  double eps2;      // (scale/nx/2**6)**2 (main:1527)
  double rmin2;     // (scale/nx)**2 (main:1526)
  int nbins;
  int ndx;
  double dx_extra[PSOD_MAX_EXTRA_DELTA];
  // the one particle the reference's run scan files under the previous cell
  // (main:1596-1599): cube position, listed cell, own cell
  unsigned quirk_pos;
  unsigned quirk_listed;
  unsigned quirk_phys;
  int has_quirk;
};

}  // namespace psod

namespace psod {
struct LearnState;
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
struct psod_ctx {
  psod_params p;  // resolved parameters
  int nx = 0, nxbuffer = 0, ncut = 0;
  long long nsel = 0;
  double xxmin[3] = {0, 0, 0};  // zone-with-buffer lower edge per axis, box units
  double xxmax[3] = {0, 0, 0};  // its upper edge
  double zone_lo[3] = {0, 0, 0}, zone_hi[3] = {0, 0, 0};  // utile zone, box units
  int nxcpu = 1;
  double scale = 0;
  float mpf = 0, munit = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // host IDs and velocities are copied on a side stream (they are first
  // read by spherover); ev_ids marks that copy's end
  cudaStream_t side_stream = nullptr;
  cudaEvent_t ev_pos = nullptr, ev_ids = nullptr;
  bool ids_pending = false;
  std::string err;

  // particles
  long long n = 0, npart_total = 0;
  float *d_pos = nullptr;   // input order, 3n (box units)
  float *d_vel = nullptr;   // input order, 3n (optional)
  long long *d_ids = nullptr;
  long long ids_cap = 0, cube_cap = 0, cs_cap = 0, inv_cap = 0;
  float4 *d_cube = nullptr;       // sorted
  unsigned *d_cell_start = nullptr;
  unsigned *d_inv = nullptr;  // input index -> cube position
  unsigned long long ncell = 0;
  unsigned quirk_pos = 0xffffffffu, quirk_listed = 0, quirk_phys = 0;
  int has_quirk = 0;

  // cic
  double *d_rho = nullptr;  // input order
  long long rho_cap = 0;
  bool cic_done = false, rho_done = false, cic_tiled = false;
  unsigned long long *d_grid = nullptr;  // fixed-point grid (tests only)

  // seeds
  long long npart_new = 0, nseed_dense = 0;
  unsigned *d_seed_idx = nullptr;  // rank -> input index
  bool seeds_done = false;

  // halos
  bool sod_done = false;
  long long nhalo = 0, nmember = 0;
  long long *d_h_id = nullptr, *d_h_mass = nullptr, *d_h_rank = nullptr, *d_h_mass2 = nullptr;
  long long *d_h_mextra = nullptr, *d_h_profile = nullptr;
  float *d_h_center = nullptr;
  double *d_h_rdelta = nullptr;
  long long *d_m_offset = nullptr;
  unsigned *d_m_index = nullptr;
  psod_run_stats last_stats{};

  std::vector<double> edge_fac;  // profile edge factors (host libm)

  // device scratch kept across calls (grown on demand, freed at destroy)
  std::vector<std::pair<void *, size_t>> scratch;

  // learned radius bracket (model, optimiser state, collected samples)
  psod::LearnState *learn = nullptr;

  // scheduling thresholds of psod_spherover (psod_set_tuning / psod_autotune);
  // none of them changes a result
  psod_tuning tune{2048, 4096, 256, 1024};

  // friends-of-friends catalogue (psod_fof; arrays in the SLOT_F_* slots)
  bool fof_done = false;
  long long fof_nhalo = 0, fof_nmember = 0;
  long long fof_n = 0;  // particles the catalogue was built on
  int learn_features = 0;  // PSOD_LEARN_FEATURES_SEED or _FOF

  // halo properties (psod_halo_properties; arrays in the SLOT_PO_* slots)
  bool props_done = false;
  long long props_nhalo = 0;
  struct {
    void *npart, *vir, *f32, *cos;
  } props_out{};
};

namespace psod {

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
int set_err(psod_ctx *c, int code, const std::string &msg);
int cuda_check(psod_ctx *c, cudaError_t e, const char *what);
#define PSOD_STR2(x) #x
#define PSOD_STR(x) PSOD_STR2(x)
#define PSOD_CUDA(ctx, call)                                                                          \
  do {                                                                                                \
    cudaError_t _e = (call);                                                                          \
    if (_e != cudaSuccess) return psod::cuda_check(ctx, _e, #call " (" __FILE__ ":" PSOD_STR(__LINE__) ")"); \
  } while (0)

template <typename T>
int dalloc(psod_ctx *c, T **p, size_t count) {
  if (*p) {
    cudaFree(*p);
    *p = nullptr;
  }
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_err(c, PSOD_ERR_NOMEM,
                   std::string("device allocation of ") + std::to_string(count * sizeof(T)) + " bytes failed");
  }
  return PSOD_OK;
}
// (re)allocate *p to hold count elements unless its capacity suffices
template <typename T>
int ensure(psod_ctx *c, T **p, long long *cap, size_t count) {
  if (*p && *cap >= (long long)count) return PSOD_OK;
  int st = dalloc(c, p, count);
  *cap = st ? 0 : (long long)count;
  return st;
}

template <typename T>
void dfree(T **p) {
  if (*p) cudaFree(*p);
  *p = nullptr;
}

// scratch slot `id` of at least `count` elements, kept by the context
template <typename T>
int scratch(psod_ctx *c, int id, size_t count, T **out) {
  if (c->scratch.size() <= (size_t)id) c->scratch.resize(id + 1, {nullptr, 0});
  auto &e = c->scratch[id];
  const size_t bytes = (count ? count : 1) * sizeof(T);
  if (e.second < bytes) {
    if (e.first) cudaFree(e.first);
    e.first = nullptr;
    e.second = 0;
    if (cudaMalloc(&e.first, bytes) != cudaSuccess) {
      cudaGetLastError();
      *out = nullptr;
      return set_err(c, PSOD_ERR_NOMEM, "device scratch allocation of " + std::to_string(bytes) + " bytes failed");
    }
    e.second = bytes;
  }
  *out = (T *)e.first;
  return PSOD_OK;
}
void free_scratch(psod_ctx *c);
void free_scratch_slot(psod_ctx *c, int id);

// Scratch slots.  Device buffers beyond the particle arrays live in numbered
// slots that only grow and are kept until the context is destroyed, so that
// repeated steps allocate nothing.  Stages that never hold a slot at the same
// time share it.  Slots 8-15 are the scan levels; 16-79 belong to the SOD
// stage.
enum : int {
  SLOT_CIC_FLAG = 2,    // CIC: out-of-tile flag
  SLOT_BIG_TAB = 3,     // cell sort: sub-cell slot tables of dense cells
  SLOT_BIG_CELL = 4,    // cell sort: the dense cells
  SLOT_LOAD_FLAGS = 5,  // cell sort: bad-position flag, dense-cell count
  SLOT_PART_U32 = 6,    // n u32: cell ids (load), seed flags (tri_cic), member pool indices (SOD)
  SLOT_PART_U64 = 7,    // n u64: seed prefix sums (tri_cic), member pool keys (SOD)
  SLOT_CELL_U32 = 80,   // ncell+1 u32: cell counts (load), alive counts per cell (SOD)
  SLOT_SORT_KEYS = 81,  // radix sort: key ping-pong buffer
  SLOT_SORT_VALS = 82,  // radix sort: value ping-pong buffer
  SLOT_SORT_HIST = 83,  // radix sort: per-tile digit counts
  SLOT_SORT_RNG = 84,   // radix sort: key range
  SLOT_TRI_KEYS = 85,   // tri_cic: seed sort keys
  SLOT_TRI_MIN = 86,    // tri_cic: densest-non-seed key and index
  SLOT_HOST_POS = 87,   // load: device copy of host positions
  SLOT_VEL = 88,        // load: velocities
  SLOT_SEED_IDX = 89,   // tri_cic: seed order (persistent)
  SLOT_OUT_IDX = 90,    // psod_get_halos: member indices staged for a host copy
  SLOT_OUT_ID = 91,     // psod_get_halos: member IDs staged for a host copy
  SLOT_H_ID = 92,       // halo table (persistent until the next SOD call)
  SLOT_H_MASS,
  SLOT_H_RANK,
  SLOT_H_MASS2,
  SLOT_H_MEXTRA,
  SLOT_H_PROFILE,
  SLOT_H_CENTER,
  SLOT_H_RDELTA,
  SLOT_M_OFFSET,
  SLOT_M_INDEX,
  SLOT_LEARN_X,         // learned bracket: raw feature rows of an API call
  SLOT_LEARN_Y,         // learned bracket: outputs / raw targets of an API call
  SLOT_LEARN_XB,        // learned bracket: standardised bf16 inputs
  SLOT_LEARN_TS,        // learned bracket: standardised targets
  SLOT_LEARN_PERM,      // learned bracket: batch order
  SLOT_SLAB_REC,        // load: particle records grouped by slab (n float4)
  SLOT_SLABS,           // load: slab counts and write cursors
  SLOT_FOF_KEY,         // fof: linking-cell keys in cube order
  SLOT_FOF_SKEY,        // fof: keys in FoF order
  SLOT_FOF_PERM,        // fof: FoF order -> cube slot; later halo-root flags
  SLOT_FOF_PAR,         // fof: union-find parents
  SLOT_FOF_INV,         // fof: input index -> FoF position
  SLOT_FOF_AUX1,        // fof: head flags, then component sizes
  SLOT_FOF_AUX2,        // fof: large cells and head scan, then lowest index / halo rank
  SLOT_FOF_HEADS,       // fof: run heads (+ end)
  SLOT_FOF_BIGRUN,      // fof: runs linked by a warp
  SLOT_FOF_HPOS,        // fof: flag scans
  SLOT_FOF_HKEY,        // fof: halo labels (sort keys)
  SLOT_FOF_HROOT,       // fof: halo roots
  SLOT_FOF_MKEY,        // fof: member halo ranks
  SLOT_FOF_MCOUNT,      // fof: halo masses, then their exclusive scan
  SLOT_FOF_CNT,         // fof: list counters
  SLOT_FOF_CTR,         // fof: test counters
  SLOT_F_ID,            // fof catalogue (kept until the next psod_fof)
  SLOT_F_MASS,
  SLOT_F_OFF,
  SLOT_F_COM,
  SLOT_F_VEL,
  SLOT_F_RAD,
  SLOT_F_MEM,
  SLOT_F_FEAT,          // fof: per halo RMS radius and inertia axis ratios (float4)
  SLOT_F_CODE,          // fof: per input particle, its halo rank or (top bit) group size
  SLOT_PR_POS,          // props: member positions after the periodic shifts
  SLOT_PR_EPI,          // props: per-member potential sums
  SLOT_PR_WORK,         // props: per-halo sums
  SLOT_PR_CNT,          // props: potential items per halo, then their scan
  SLOT_PR_PREF,         // props: the scan as int64
  SLOT_PR_IHALO,        // props: halo of each potential item
  SLOT_PO_NPART,        // props outputs (kept until the next call)
  SLOT_PO_VIR,
  SLOT_PO_F32,
  SLOT_PO_COS
};

// Eigen decomposition of a symmetric 3x3 matrix by the cyclic Jacobi
// method with thresholds (Rutishauser's, as published in Numerical Recipes'
// jacobi; haloanalyzer's diag, modfunctions.f90:840-933, follows it): d gets
// the eigenvalues, v the eigenvectors as columns.  eigsort3 orders them by
// descending eigenvalue, a later equal value moving first (eigsrt :812-837).
__device__ inline void jacobi3(double a[3][3], double d[3], double v[3][3]) {
  double bb[3], z[3];
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) v[i][j] = 0.0;
    v[i][i] = 1.0;
    bb[i] = d[i] = a[i][i];
    z[i] = 0.0;
  }
  for (int sweep = 1; sweep <= 50; sweep++) {
    double sm = 0.0;
    for (int p = 0; p < 2; p++)
      for (int q = p + 1; q < 3; q++) sm += fabs(a[p][q]);
    if (sm == 0.0) return;
    const double tresh = sweep < 4 ? (double)0.2f * sm / 9.0 : 0.0;
    for (int p = 0; p < 2; p++)
      for (int q = p + 1; q < 3; q++) {
        double g = 100.0 * fabs(a[p][q]);
        if (sweep > 4 && fabs(d[p]) + g == fabs(d[p]) && fabs(d[q]) + g == fabs(d[q])) {
          a[p][q] = 0.0;
        } else if (fabs(a[p][q]) > tresh) {
          double hh = d[q] - d[p], t;
          if (fabs(hh) + g == fabs(hh)) {
            t = a[p][q] / hh;
          } else {
            const double theta = 0.5 * hh / a[p][q];
            t = 1.0 / (fabs(theta) + sqrt(1.0 + theta * theta));
            if (theta < 0.0) t = -t;
          }
          const double c = 1.0 / sqrt(1 + t * t), s = t * c, tau = s / (1.0 + c);
          hh = t * a[p][q];
          z[p] -= hh;
          z[q] += hh;
          d[p] -= hh;
          d[q] += hh;
          a[p][q] = 0.0;
          for (int j = 0; j < p; j++) {
            g = a[j][p];
            hh = a[j][q];
            a[j][p] = g - s * (hh + g * tau);
            a[j][q] = hh + s * (g - hh * tau);
          }
          for (int j = p + 1; j < q; j++) {
            g = a[p][j];
            hh = a[j][q];
            a[p][j] = g - s * (hh + g * tau);
            a[j][q] = hh + s * (g - hh * tau);
          }
          for (int j = q + 1; j < 3; j++) {
            g = a[p][j];
            hh = a[q][j];
            a[p][j] = g - s * (hh + g * tau);
            a[q][j] = hh + s * (g - hh * tau);
          }
          for (int j = 0; j < 3; j++) {
            g = v[j][p];
            hh = v[j][q];
            v[j][p] = g - s * (hh + g * tau);
            v[j][q] = hh + s * (g - hh * tau);
          }
        }
      }
    for (int p = 0; p < 3; p++) {
      bb[p] += z[p];
      d[p] = bb[p];
      z[p] = 0.0;
    }
  }
}

__device__ inline void eigsort3(double d[3], double v[3][3]) {
  for (int i = 0; i < 2; i++) {
    int k = i;
    double p = d[i];
    for (int j = i + 1; j < 3; j++)
      if (d[j] >= p) {
        k = j;
        p = d[j];
      }
    if (k != i) {
      d[k] = d[i];
      d[i] = p;
      for (int j = 0; j < 3; j++) {
        const double t = v[j][i];
        v[j][i] = v[j][k];
        v[j][k] = t;
      }
    }
  }
}


// learned radius bracket (psod_learn.cu)
void learn_free(psod_ctx *c);
bool learn_ready(const psod_ctx *c);
bool learn_collecting(const psod_ctx *c);
void learn_sample_buffers(const psod_ctx *c, float **x, float **t, unsigned long long **count,
                          unsigned long long *cap);
int learn_predict(psod_ctx *c, const float *feat, unsigned n, float *rb0);

bool is_device_ptr(const void *p);
// make the context's stream wait for a pending side-stream copy of the IDs
int wait_ids(psod_ctx *c);
int copy_out(psod_ctx *c, void *dst, const void *dsrc, size_t bytes);
int copy_in(psod_ctx *c, void *ddst, const void *src, size_t bytes);

// device-wide exclusive scan of uint32 (values and total must fit 32 bits);
// out may alias in; out[n] receives the total when with_total.
int scan_u32(psod_ctx *c, const unsigned *in, unsigned *out, long long n, bool with_total);

// stable LSD radix sort of (key, value) pairs on bits [0, end_bit); keys and
// vals hold the input and receive the output.
int radix_sort_u64(psod_ctx *c, unsigned long long *keys, unsigned *vals, long long n, int end_bit);
int radix_sort_u32(psod_ctx *c, unsigned *keys, unsigned *vals, long long n, int end_bit);

SodConst make_sod_const(const psod_ctx *c);

int stage_cellsort(psod_ctx *c, const float *dpos);
int stage_cic(psod_ctx *c, double *grid_out);
int stage_cicm1(psod_ctx *c, double *rho_out);
int stage_tri_cic(psod_ctx *c, int64_t *isort_out);
int stage_spherover(psod_ctx *c, psod_run_stats *st);

}  // namespace psod
