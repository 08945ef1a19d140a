// psod_capi.cu -- the extern "C" boundary of libpsod.so (include/psod.h).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "psod_internal.cuh"

namespace psod {

int set_err(psod_ctx *c, int code, const std::string &msg) {
  if (c) c->err = msg;
  return code;
}

int cuda_check(psod_ctx *c, cudaError_t e, const char *what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();
  return set_err(c, PSOD_ERR_CUDA, m);
}

void free_scratch(psod_ctx *c) {
  for (auto &e : c->scratch)
    if (e.first) cudaFree(e.first);
  c->scratch.clear();
}

void free_scratch_slot(psod_ctx *c, int id) {
  if ((size_t)id < c->scratch.size() && c->scratch[id].first) {
    cudaFree(c->scratch[id].first);
    c->scratch[id] = {nullptr, 0};
  }
}

bool is_device_ptr(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int copy_out(psod_ctx *c, void *dst, const void *dsrc, size_t bytes) {
  if (bytes == 0) return PSOD_OK;
  PSOD_CUDA(c, cudaMemcpyAsync(dst, dsrc, bytes, cudaMemcpyDefault, c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  return PSOD_OK;
}

int wait_ids(psod_ctx *c) {
  if (c->ids_pending) {
    PSOD_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_ids, 0));
    c->ids_pending = false;
  }
  return PSOD_OK;
}

int copy_in(psod_ctx *c, void *ddst, const void *src, size_t bytes) {
  if (bytes == 0) return PSOD_OK;
  PSOD_CUDA(c, cudaMemcpyAsync(ddst, src, bytes, cudaMemcpyDefault, c->stream));
  return PSOD_OK;
}

}  // namespace psod

using namespace psod;

static void free_all(psod_ctx *c) {
  dfree(&c->d_ids);
  dfree(&c->d_cube);
  dfree(&c->d_cell_start);
  dfree(&c->d_inv);
  dfree(&c->d_rho);
  dfree(&c->d_grid);
  // the remaining arrays live in scratch slots
  c->d_pos = nullptr;
  c->d_vel = nullptr;
  c->d_seed_idx = nullptr;
  c->d_h_id = c->d_h_mass = c->d_h_rank = c->d_h_mass2 = c->d_h_mextra = c->d_h_profile = nullptr;
  c->d_h_center = nullptr;
  c->d_h_rdelta = nullptr;
  c->d_m_offset = nullptr;
  c->d_m_index = nullptr;
  free_scratch(c);
  learn_free(c);
}

extern "C" {

int psod_abi_version(void) { return PSOD_ABI_VERSION; }

const char *psod_status_string(int s) {
  switch (s) {
    case PSOD_OK: return "ok";
    case PSOD_ERR_NSEL: return "preselection exceeded nsel (zone output lost)";
    case PSOD_ERR_SELRADIUS: return "overdensity above delta at the selection radius (zone output lost)";
    case PSOD_ERR_TIMEOUT: return "bounded device wait ran out";
    case PSOD_ERR_CUDA: return "CUDA error";
    case PSOD_ERR_ARG: return "invalid argument";
    case PSOD_ERR_STATE: return "call out of order or internal check failed";
    case PSOD_ERR_NOMEM: return "device allocation failed";
    case PSOD_ERR_IO: return "output file could not be written";
    default: return "unknown status";
  }
}

void psod_params_default(psod_params *p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->nx = 0;
  p->nmin = 100;        // main:112
  p->delta = 200.0;     // main:110
  p->delta2 = 800.0;    // main:110
  p->ncut = 4;          // main:114
  p->nsel = 4000000;    // main:114
  p->nxbuffer = 0;      // main:114 (0 -> nx/2 at main:380-381)
  p->npu = 0;
  p->nbins = 60;        // main:1414
  p->rbin_lo = 0.01;    // main:2105
  p->rbin_hi = 1.0;     // main:2105
  p->ndelta_extra = 0;
  p->mode = PSOD_MODE_PLAIN;
  p->device = 0;
  p->nxcpu = 1;  // one zone: the one-rank run
  p->nzone = 0;
}

int psod_ctx_create(const psod_params *pin, psod_ctx **out) {
  if (!pin || !out) return PSOD_ERR_ARG;
  *out = nullptr;
  psod_ctx *c = new psod_ctx();
  c->p = *pin;
  psod_params &p = c->p;
  // -npu (main:211-219): derive ncut, nxbuffer and nsel from a halo-size bound
  if (p.npu > 0) {
    p.ncut = (int)std::ceil(std::pow(p.npu * 2.0 / p.delta, 1.0 / 3.0) / 2.0);
    p.nxbuffer = 4 * p.ncut;
    p.nsel = (int64_t)std::ceil(std::pow(2.0 * p.ncut + 1.0, 3) * p.delta * 4.0);
  }
  std::string why;
  if (p.nx < 5) why = "nx must be >= 5";
  else if (p.ncut < 1 || 2 * p.ncut + 1 > p.nx) why = "ncut must satisfy 1 <= ncut and 2*ncut+1 <= nx";
  else if (p.nmin < 10) why = "nmin must be >= 10 (the crossing loop always takes 10 steps, main:2046)";
  else if (p.nbins < 1 || p.nbins > PSOD_MAX_BINS) why = "nbins must be in [1, 128]";
  else if (p.nsel < 1) why = "nsel must be positive";
  else if (!(p.rbin_lo > 0.0) || !(p.rbin_hi > 0.0)) why = "profile edge factors must be positive";
  else if (p.ndelta_extra < 0 || p.ndelta_extra > PSOD_MAX_EXTRA_DELTA) why = "at most 4 extra thresholds";
  else if (!(p.delta > 0.0)) why = "delta must be positive";
  if (p.nxcpu == 0) p.nxcpu = 1;
  if (why.empty() && (p.nxcpu < 1 || p.nx % p.nxcpu != 0)) why = "nxcpu must be >= 1 and divide nx";
  if (why.empty() && (p.nzone < 0 || (long long)p.nzone >= (long long)p.nxcpu * p.nxcpu * p.nxcpu))
    why = "nzone must lie in [0, nxcpu^3)";
  const int nxzone = why.empty() ? p.nx / p.nxcpu : 1;          // main:349
  int nxbuffer = p.nxbuffer == 0 ? nxzone / 2 : p.nxbuffer;     // main:380-381
  if (why.empty() && nxbuffer < p.ncut) why = "nxbuffer must be >= ncut (main:386)";
  if (p.nxcpu == 1) {
    // the reference allows nxbuffer == nx (main:392); its CIC array is then
    // padded past the periodic grid, which this engine does not keep
    if (why.empty() && nxbuffer >= p.nx) why = "nxbuffer must be < nx";
  } else {
    if (why.empty() && nxbuffer > nxzone) why = "nxbuffer must be <= nxzone (main:392)";
    // the linked-list walks (main:1657-1675) wrap cell indices modulo nx
    // and then skip those outside the local grid: unless the local grid
    // spans the box or leaves max(ncut, 2) cells outside, a wrapped index
    // lands on the far side of the local grid
    const int local = nxzone + 2 * nxbuffer, reach = std::max(p.ncut, 2);
    if (why.empty() && local < p.nx && local > p.nx - reach)
      why = "the zone with its buffer must span the box or leave max(ncut, 2) cells outside";
  }
  if (!why.empty()) {
    delete c;
    return PSOD_ERR_ARG;
  }
  c->nx = p.nx;
  c->nxbuffer = nxbuffer;
  c->ncut = p.ncut;
  c->nsel = p.nsel;
  // zone indices (main:344-346) and the zone with its buffer (main:401-406)
  // and without (main:420-425), box units
  c->nxcpu = p.nxcpu;
  const int ncpu = p.nxcpu;
  const int izone[3] = {p.nzone / (ncpu * ncpu), (p.nzone / ncpu) % ncpu, p.nzone % ncpu};
  const double q = (double)nxbuffer / (double)nxzone;
  for (int a = 0; a < 3; a++) {
    c->xxmin[a] = ((double)izone[a] - q) / (double)ncpu;
    c->xxmax[a] = ((double)izone[a] + 1.0 + q) / (double)ncpu;
    c->zone_lo[a] = (double)izone[a] / (double)ncpu;
    c->zone_hi[a] = ((double)izone[a] + 1.0) / (double)ncpu;
  }
  c->scale = (double)p.nx;  // main:689
  // profile edge factors with the host libm, as the reference evaluates
  // exp(log(lo) + (j-1)*(log(hi)-log(lo))/(nbins-1)) (main:2105)
  c->edge_fac.resize(p.nbins);
  for (int j = 0; j < p.nbins; j++) {
    const double denom = (double)p.nbins - 1.0;
    c->edge_fac[j] = denom > 0.0 ? std::exp(std::log(p.rbin_lo) + ((double)j * (std::log(p.rbin_hi) - std::log(p.rbin_lo))) / denom)
                                 : p.rbin_hi;
  }
  c->device = p.device;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev <= p.device) {
    cudaGetLastError();
    delete c;
    return PSOD_ERR_CUDA;
  }
  if (cudaSetDevice(p.device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return PSOD_ERR_CUDA;
  }
  c->own_stream = true;
  *out = c;
  return PSOD_OK;
}

int psod_ctx_destroy(psod_ctx *c) {
  if (!c) return PSOD_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->side_stream) cudaStreamSynchronize(c->side_stream);
  free_all(c);
  if (c->side_stream) cudaStreamDestroy(c->side_stream);
  if (c->ev_pos) cudaEventDestroy(c->ev_pos);
  if (c->ev_ids) cudaEventDestroy(c->ev_ids);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return PSOD_OK;
}

int psod_set_stream(psod_ctx *c, void *stream) {
  if (!c) return PSOD_ERR_ARG;
  cudaSetDevice(c->device);
  // a pending ID copy is ordered before the new stream's work
  if (c->ids_pending) {
    if (cudaStreamWaitEvent((cudaStream_t)stream, c->ev_ids, 0) != cudaSuccess)
      return cuda_check(c, cudaGetLastError(), "cudaStreamWaitEvent");
    c->ids_pending = false;
  }
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  c->stream = (cudaStream_t)stream;
  c->own_stream = false;
  return PSOD_OK;
}

int psod_load_particles(psod_ctx *c, int64_t n, const float *pos, const float *vel, const int64_t *id,
                        int64_t npart_total) {
  if (!c) return PSOD_ERR_ARG;
  if (n < 1 || !pos || !id) return set_err(c, PSOD_ERR_ARG, "need n >= 1, pos and id");
  if (n >= (int64_t)PSOD_DEAD_BIT) return set_err(c, PSOD_ERR_ARG, "n must be below 2^31");
  if (npart_total < 1) npart_total = n;
  if (cudaSetDevice(c->device) != cudaSuccess) return cuda_check(c, cudaGetLastError(), "cudaSetDevice");
  c->n = n;
  c->npart_total = npart_total;
  c->mpf = (float)(1.0 / (double)npart_total);                // main:662
  c->munit = (float)((double)c->mpf * (double)npart_total);   // main:685
  c->cic_done = c->rho_done = c->seeds_done = c->sod_done = false;
  int st;
  // positions are only read by the cell sort: a device buffer is used in
  // place, a host buffer goes through a temporary device copy
  const float *dpos = pos;
  if (!is_device_ptr(pos)) {
    if ((st = scratch(c, SLOT_HOST_POS, (size_t)n * 3, &c->d_pos))) return st;
    if ((st = copy_in(c, c->d_pos, pos, sizeof(float) * 3 * n))) return st;
    dpos = c->d_pos;
  }
  if (!c->d_ids || c->ids_cap < n) {
    if ((st = wait_ids(c))) return st;  // the old buffer may still be a copy's target
    if ((st = dalloc(c, &c->d_ids, (size_t)n))) return st;
    c->ids_cap = n;
  }
  if (vel) {
    if ((st = wait_ids(c))) return st;
    if ((st = scratch(c, SLOT_VEL, (size_t)n * 3, &c->d_vel))) return st;
  } else {
    c->d_vel = nullptr;
  }
  // IDs and velocities are first read by spherover (halo records): host
  // arrays go over on a side stream after the positions, so their copy
  // overlaps the cell sort, the CIC and the seed order.  The side stream
  // first waits for the context's stream, which may still read the previous
  // IDs; spherover and psod_get_halos wait for the copy.
  const bool side = !is_device_ptr(id) || (vel && !is_device_ptr(vel));
  if (side) {
    if (!c->side_stream) {
      PSOD_CUDA(c, cudaStreamCreateWithFlags(&c->side_stream, cudaStreamNonBlocking));
      PSOD_CUDA(c, cudaEventCreateWithFlags(&c->ev_pos, cudaEventDisableTiming));
      PSOD_CUDA(c, cudaEventCreateWithFlags(&c->ev_ids, cudaEventDisableTiming));
    }
    if ((st = wait_ids(c))) return st;
    PSOD_CUDA(c, cudaEventRecord(c->ev_pos, c->stream));
    PSOD_CUDA(c, cudaStreamWaitEvent(c->side_stream, c->ev_pos, 0));
    PSOD_CUDA(c, cudaMemcpyAsync(c->d_ids, id, sizeof(int64_t) * n, cudaMemcpyDefault, c->side_stream));
    if (vel) PSOD_CUDA(c, cudaMemcpyAsync(c->d_vel, vel, sizeof(float) * 3 * n, cudaMemcpyDefault, c->side_stream));
    PSOD_CUDA(c, cudaEventRecord(c->ev_ids, c->side_stream));
    c->ids_pending = true;
  } else {
    if ((st = copy_in(c, c->d_ids, id, sizeof(int64_t) * n))) return st;
    if (vel && (st = copy_in(c, c->d_vel, vel, sizeof(float) * 3 * n))) return st;
  }
  return stage_cellsort(c, dpos);
}

int psod_cic(psod_ctx *c, double *grid_out) {
  if (!c) return PSOD_ERR_ARG;
  if (c->n == 0) return set_err(c, PSOD_ERR_STATE, "psod_cic needs psod_load_particles first");
  cudaSetDevice(c->device);
  return stage_cic(c, grid_out);
}

int psod_cicm1(psod_ctx *c, double *rho_out) {
  if (!c) return PSOD_ERR_ARG;
  cudaSetDevice(c->device);
  return stage_cicm1(c, rho_out);
}

int psod_tri_cic(psod_ctx *c, int64_t *isort_out, int64_t *npart_new_out) {
  if (!c) return PSOD_ERR_ARG;
  cudaSetDevice(c->device);
  int st = stage_tri_cic(c, isort_out);
  if (!st && npart_new_out) *npart_new_out = c->npart_new;
  return st;
}

int psod_spherover(psod_ctx *c, psod_run_stats *stats) {
  if (!c) return PSOD_ERR_ARG;
  cudaSetDevice(c->device);
  return stage_spherover(c, stats);
}

int psod_run(psod_ctx *c, psod_run_stats *stats) {
  int st;
  if ((st = psod_cic(c, nullptr))) return st;
  if ((st = psod_cicm1(c, nullptr))) return st;
  if ((st = psod_tri_cic(c, nullptr, nullptr))) return st;
  return psod_spherover(c, stats);
}

int psod_halo_count(psod_ctx *c, int64_t *nhalo, int64_t *nmember) {
  if (!c) return PSOD_ERR_ARG;
  if (!c->sod_done) return set_err(c, PSOD_ERR_STATE, "no halo table: call psod_spherover first");
  if (nhalo) *nhalo = c->nhalo;
  if (nmember) *nmember = c->nmember;
  return PSOD_OK;
}

namespace {
__global__ void k_member_ids(const unsigned *midx, long long n, const long long *ids, long long *out_idx,
                             long long *out_id) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned k = midx[i];
  if (out_idx) out_idx[i] = (long long)k;
  if (out_id) out_id[i] = ids[k];
}
}  // namespace

int psod_get_halos(psod_ctx *c, const psod_halo_table *t) {
  if (!c || !t) return PSOD_ERR_ARG;
  if (!c->sod_done) return set_err(c, PSOD_ERR_STATE, "no halo table: call psod_spherover first");
  cudaSetDevice(c->device);
  int wst = wait_ids(c);
  if (wst) return wst;
  const long long nh = c->nhalo, nm = c->nmember;
  int st;
  if (t->halo_id && (st = copy_out(c, t->halo_id, c->d_h_id, sizeof(int64_t) * nh))) return st;
  if (t->halo_mass && (st = copy_out(c, t->halo_mass, c->d_h_mass, sizeof(int64_t) * nh))) return st;
  if (t->halo_rank && (st = copy_out(c, t->halo_rank, c->d_h_rank, sizeof(int64_t) * nh))) return st;
  if (t->halo_center && (st = copy_out(c, t->halo_center, c->d_h_center, sizeof(float) * 3 * nh))) return st;
  if (t->halo_rdelta && (st = copy_out(c, t->halo_rdelta, c->d_h_rdelta, sizeof(double) * nh))) return st;
  if (t->halo_mass2 && (st = copy_out(c, t->halo_mass2, c->d_h_mass2, sizeof(int64_t) * nh))) return st;
  if (t->halo_mextra && c->p.ndelta_extra > 0 &&
      (st = copy_out(c, t->halo_mextra, c->d_h_mextra, sizeof(int64_t) * nh * c->p.ndelta_extra)))
    return st;
  if (t->halo_profile && (st = copy_out(c, t->halo_profile, c->d_h_profile, sizeof(int64_t) * nh * c->p.nbins)))
    return st;
  if (t->member_offset && (st = copy_out(c, t->member_offset, c->d_m_offset, sizeof(int64_t) * (nh + 1))))
    return st;
  if ((t->member_index || t->member_id) && nm > 0) {
    // device destinations are written in place; host ones are staged
    long long *d_idx = nullptr, *d_id = nullptr;
    if (t->member_index) {
      if (is_device_ptr(t->member_index)) d_idx = reinterpret_cast<long long *>(t->member_index);
      else if ((st = scratch(c, SLOT_OUT_IDX, (size_t)nm, &d_idx))) return st;
    }
    if (t->member_id) {
      if (is_device_ptr(t->member_id)) d_id = reinterpret_cast<long long *>(t->member_id);
      else if ((st = scratch(c, SLOT_OUT_ID, (size_t)nm, &d_id))) return st;
    }
    k_member_ids<<<(unsigned)((nm + 255) / 256), 256, 0, c->stream>>>(c->d_m_index, nm, c->d_ids, d_idx, d_id);
    st = PSOD_OK;
    if (t->member_index && (void *)d_idx != (void *)t->member_index)
      st = copy_out(c, t->member_index, d_idx, sizeof(int64_t) * nm);
    if (!st && t->member_id && (void *)d_id != (void *)t->member_id)
      st = copy_out(c, t->member_id, d_id, sizeof(int64_t) * nm);
    if (st) return st;
    PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  return PSOD_OK;
}

int psod_learn_set_features(psod_ctx *c, int32_t set) {
  if (!c) return PSOD_ERR_ARG;
  if (set != PSOD_LEARN_FEATURES_SEED && set != PSOD_LEARN_FEATURES_FOF)
    return set_err(c, PSOD_ERR_ARG, "psod_learn_set_features: PSOD_LEARN_FEATURES_SEED or PSOD_LEARN_FEATURES_FOF");
  c->learn_features = set;
  return PSOD_OK;
}

int psod_get_tuning(psod_ctx *c, psod_tuning *t) {
  if (!c || !t) return PSOD_ERR_ARG;
  *t = c->tune;
  return PSOD_OK;
}

int psod_set_tuning(psod_ctx *c, const psod_tuning *t) {
  if (!c || !t) return PSOD_ERR_ARG;
  if (t->warp_cross_min_ready < 1 || t->bound_min_cand < 256 || t->tail_max_ready < 0 || t->tail_max_cand < 1 ||
      t->tail_max_cand > t->bound_min_cand)
    return set_err(c, PSOD_ERR_ARG,
                   "psod_set_tuning: warp_cross_min_ready >= 1, bound_min_cand >= 256, tail_max_ready >= 0, "
                   "1 <= tail_max_cand <= bound_min_cand");
  c->tune = *t;
  return PSOD_OK;
}

int psod_autotune(psod_ctx *c, psod_tuning *chosen, double *ms_best, int32_t *runs) {
  if (!c) return PSOD_ERR_ARG;
  if (!c->seeds_done) return set_err(c, PSOD_ERR_STATE, "psod_autotune: call psod_tri_cic first");
  int nrun = 0;
  auto time_run = [&](double *ms) {
    psod_run_stats st{};
    const int s = psod_spherover(c, &st);
    nrun++;
    *ms = st.ms_total;
    return s;
  };
  double best_ms = 0.0;
  int st = time_run(&best_ms);
  if (st) return st;
  psod_tuning best = c->tune;
  // candidates per threshold; 1 << 30 turns the warp pass off
  const int32_t warp_c[] = {512, 1024, 2048, 4096, 1 << 30};
  const int32_t bound_c[] = {2048, 4096, 8192};
  const int32_t tail_c[] = {0, 128, 256, 512, 1024};
  const int32_t tcand_c[] = {256, 1024, 2048};
  auto sweep = [&](int32_t psod_tuning::*field, const int32_t *vals, int nv) -> int {
    for (int k = 0; k < nv; k++) {
      psod_tuning t = best;
      t.*field = vals[k];
      if (t.*field == best.*field || t.tail_max_cand > t.bound_min_cand) continue;
      c->tune = t;
      double ms = 0.0;
      const int s = time_run(&ms);
      if (s) {
        c->tune = best;
        return s;
      }
      if (ms < best_ms * 0.995) {
        best_ms = ms;
        best = t;
      }
    }
    c->tune = best;
    return PSOD_OK;
  };
  if ((st = sweep(&psod_tuning::warp_cross_min_ready, warp_c, 5))) return st;
  if ((st = sweep(&psod_tuning::bound_min_cand, bound_c, 3))) return st;
  if ((st = sweep(&psod_tuning::tail_max_ready, tail_c, 5))) return st;
  if ((st = sweep(&psod_tuning::tail_max_cand, tcand_c, 3))) return st;
  // the table of the last run came from the last candidate tried: run once
  // more with the chosen thresholds so that every counter matches them
  double last = 0.0;
  if ((st = time_run(&last))) return st;
  if (chosen) *chosen = best;
  if (ms_best) *ms_best = best_ms;
  if (runs) *runs = nrun;
  return PSOD_OK;
}

const char *psod_last_error(const psod_ctx *c) { return c ? c->err.c_str() : "null context"; }

}  // extern "C"
