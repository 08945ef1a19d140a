// psod_static.cu -- CIC density without any device allocation.
//
// psod_cic_rho_static() computes the same per-particle density as
// psod_cic + psod_cicm1 (fixed-point nodes, the reference's interpolation
// order), for zones of at most PSOD_STATIC_MAX_NX cells per side, using a
// node grid that lives in a file-scope __device__ array instead of memory
// the library allocates.  It exists for host codes that cannot let a library
// allocate device memory: drivers that size all of the GPU's memory
// themselves (for instance several MPI ranks sharing a GPU under fixed
// per-rank budgets, or a host whose own pool allocator owns the device) and
// forbid libraries from calling cudaMalloc.
//
// The array (PSOD_STATIC_MAX_NX = 64: (2*64)^3 int64 nodes, 16 MiB) is held
// on every device that loads the library until the process exits.  Host code
// cannot use the array's name as a device address, so the first call on each
// device looks the address up with cudaGetSymbolAddress (that device current)
// and keeps it; make that first call before any stream capture.  Every call
// clears the nodes before depositing.  All calls share the array: calls
// whose work overlaps on the GPU (two streams, or two host threads) race and
// give wrong densities; serialise them.
#include <cuda_runtime.h>

#include <mutex>

#include "psod_internal.cuh"

#define PSOD_STATIC_GRID_NODES (2 * PSOD_STATIC_MAX_NX) * (2 * PSOD_STATIC_MAX_NX) * (2 * PSOD_STATIC_MAX_NX)

// the scratch: fixed-point CIC nodes, cleared by every call
static __device__ __align__(256) unsigned long long g_static_nodes[PSOD_STATIC_GRID_NODES];

namespace {

using psod::dadd;
using psod::ddiv;
using psod::dmul;
using psod::dsub;

constexpr double kFixOne = 1099511627776.0;  // 2^40 per unit weight
constexpr int kMaxDevices = 64;

// device address of g_static_nodes, per device (set up on first use)
unsigned long long *g_node_ptr[kMaxDevices] = {nullptr};
std::mutex g_setup_mutex;

struct StaticCic {
  double xxmin, xxmax, dx, kc;
  int nc;
};

// one axis of the CIC stencil (main:1154-1190)
__device__ __forceinline__ void static_cic_axis(float xf, double xxmin, double dx, int nc, int &i0, int &i1,
                                                double &dd, double &de) {
  double d = ddiv(dsub((double)xf, xxmin), dx);
  int ix = (int)d;
  if (d < 0.0) ix = ix - 1;
  d = dsub(d, (double)ix);
  const double e = dsub(1.0, d);
  int ixp1 = ix + 1;
  if (ixp1 < 0) ixp1 += nc;
  if (ix < 0) ix += nc;
  if (ixp1 >= nc) ixp1 -= nc;
  if (ix >= nc) ix -= nc;
  i0 = ix;
  i1 = ixp1;
  dd = d;
  de = e;
}

__global__ void k_static_clear(unsigned long long *nodes, long long nnode, int *bad) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nnode; i += (long long)gridDim.x * blockDim.x)
    nodes[i] = 0ull;
  if (bad && blockIdx.x == 0 && threadIdx.x == 0) *bad = 0;
}

// positions outside [0,1] are skipped: they would index outside the grid
__device__ __forceinline__ bool in_box(float x, float y, float z) {
  return x >= 0.f && x <= 1.f && y >= 0.f && y <= 1.f && z >= 0.f && z <= 1.f;
}

__global__ void k_static_deposit(const float *pos, long long n, StaticCic k, unsigned long long *nodes, int *bad) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
  if (!in_box(x, y, z)) {
    if (bad) atomicOr(bad, 1);
    return;
  }
  int ix, ixp, iy, iyp, iz, izp;
  double ddx, dex, ddy, dey, ddz, dez;
  static_cic_axis(x, k.xxmin, k.dx, k.nc, ix, ixp, ddx, dex);
  static_cic_axis(y, k.xxmin, k.dx, k.nc, iy, iyp, ddy, dey);
  static_cic_axis(z, k.xxmin, k.dx, k.nc, iz, izp, ddz, dez);
  const long long nc = k.nc;
  const int cx[2] = {ix, ixp}, cy[2] = {iy, iyp}, cz[2] = {iz, izp};
  const double wx[2] = {dex, ddx}, wy[2] = {dey, ddy}, wz[2] = {dez, ddz};
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const int a = c & 1, b = (c >> 1) & 1, e = c >> 2;
    const double w = dmul(dmul(wx[a], wy[b]), wz[e]);
    const long long node = (long long)cx[a] + nc * ((long long)cy[b] + nc * (long long)cz[e]);
    atomicAdd(&nodes[node], (unsigned long long)__double2ll_rn(dmul(w, kFixOne)));
  }
}

__global__ void k_static_interp(const float *pos, long long n, StaticCic k, const unsigned long long *nodes,
                                double *rho) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
  if (!in_box(x, y, z)) {
    rho[i] = 0.0;
    return;
  }
  int ix, ixp, iy, iyp, iz, izp;
  double ddx, dex, ddy, dey, ddz, dez;
  static_cic_axis(x, k.xxmin, k.dx, k.nc, ix, ixp, ddx, dex);
  static_cic_axis(y, k.xxmin, k.dx, k.nc, iy, iyp, ddy, dey);
  static_cic_axis(z, k.xxmin, k.dx, k.nc, iz, izp, ddz, dez);
  const long long nc = k.nc;
  const int cx[2] = {ix, ixp}, cy[2] = {iy, iyp}, cz[2] = {iz, izp};
  const double wx[2] = {dex, ddx}, wy[2] = {dey, ddy}, wz[2] = {dez, ddz};
  double r = 0.0;
#pragma unroll
  for (int c = 0; c < 8; c++) {  // main:1368-1383 term order
    const int a = c & 1, b = (c >> 1) & 1, e = c >> 2;
    const long long node = (long long)cx[a] + nc * ((long long)cy[b] + nc * (long long)cz[e]);
    const double g = dmul((double)(long long)nodes[node], k.kc);
    r = dadd(r, dmul(dmul(dmul(g, wx[a]), wy[b]), wz[e]));
  }
  rho[i] = r;
}

// the node grid's device address on the current device
int static_nodes(unsigned long long **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return PSOD_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_node_ptr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_static_nodes) != cudaSuccess || !p) {
      cudaGetLastError();
      return PSOD_ERR_CUDA;
    }
    g_node_ptr[dev] = (unsigned long long *)p;
  }
  *out = g_node_ptr[dev];
  return PSOD_OK;
}

bool on_device(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" int psod_cic_rho_static(int64_t n, const float *pos, int32_t nx, int64_t npart_total, int32_t nxbuffer,
                                   double *rho, int *bad_flag, void *stream) {
  if (n < 1 || !pos || !rho) return PSOD_ERR_ARG;
  if (nx < 1 || nx > PSOD_STATIC_MAX_NX) return PSOD_ERR_ARG;  // node grid bound
  if (npart_total < 1) npart_total = n;
  const int nxb = nxbuffer == 0 ? nx / 2 : nxbuffer;  // main:380-381
  if (nxb < 0 || nxb >= nx) return PSOD_ERR_ARG;  // keeps every node index below 2*nx
  if (!on_device(pos) || !on_device(rho) || (bad_flag && !on_device(bad_flag))) return PSOD_ERR_ARG;
  unsigned long long *nodes = nullptr;
  int st = static_nodes(&nodes);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  StaticCic k;
  k.nc = 2 * nx;                                       // main:667
  k.dx = 1.0 / (double)k.nc;                           // main:1126
  k.xxmin = (0.0 - (double)nxb / (double)nx) / 1.0;    // main:401, 665
  k.xxmax = (0.0 + 1.0 + (double)nxb / (double)nx) / 1.0;
  const float mpf = (float)(1.0 / (double)npart_total);  // main:662
  k.kc = ((double)mpf / kFixOne) / ((k.dx * k.dx) * k.dx);
  const long long nnode = (long long)k.nc * k.nc * k.nc;
  const unsigned g = (unsigned)((n + 255) / 256);
  k_static_clear<<<256, 256, 0, s>>>(nodes, nnode, bad_flag);
  k_static_deposit<<<g, 256, 0, s>>>(pos, n, k, nodes, bad_flag);
  k_static_interp<<<g, 256, 0, s>>>(pos, n, k, nodes, rho);
  if (cudaGetLastError() != cudaSuccess) return PSOD_ERR_CUDA;
  return PSOD_OK;
}
