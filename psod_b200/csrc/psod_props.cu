// psod_props.cu -- halo properties (haloanalyzer's halo_properties) on the GPU.
//
// haloanalyzer_new/src/modfunctions.f90 halo_properties (:47-808) reads
// each halo's particles from the halo finder's files and computes, in
// simulation units converted to physical ones: virial mass, radius and
// velocity from the particle count; centre of mass and mean velocity;
// R_max, V_max and the position / velocity dispersions; kinetic and
// potential energy and the position of the most bound particle; density,
// integrated-density and circular-velocity profiles in 100 log bins of
// radius and 30 log bins of R/R178, the circular-velocity maximum and the
// interpolated R178/M178; angular momentum and the two spin parameters; the
// inertia tensor's eigenvalues (Jacobi, sorted) and minor axis, and the
// cosine between that axis and the angular momentum.  Here the halos are a
// context's SOD table (psod_get_halos) or FoF catalogue (psod_fof_get_halos),
// members in the table's order, and the work is:
//   k_props_moments   a CTA per halo: the periodic unwrap, the centre, every
//                     sum over the members (fixed-order reductions), the
//                     unwrapped member positions staged in member order;
//   k_props_potential (halo, 256-member chunk) items over all CTAs: each
//                     member's potential sum against the halo's members,
//                     read through shared-memory tiles;
//   k_props_finish    a CTA per halo: total potential and its most bound
//                     member, the two radial histograms, the R178
//                     interpolation, the eigen solve and every output.
// The arithmetic follows the Fortran statement by statement in its
// precisions (real(4) positions shifted in real(4), real(8) sums); this
// file is built with --fmad=false, so no product is fused into a sum.  The
// sums run in another order than the sequential reference, so FP64 values
// can differ in their last bits before the real(4) outputs are rounded.
#include <cmath>

#include "psod_internal.cuh"

namespace psod {
namespace {

constexpr int PR_TPB = 256;
constexpr int NB1 = PSOD_PROPS_NBIN1, NB2 = PSOD_PROPS_NBIN2;
constexpr double MSUN = 1.98892e33, MPC = 3.08568e24;
constexpr double MIN_R = 1.0, DELTA_LR = 0.1, MIN_R178 = 1e-2, DELTA_LR178 = 0.2;

struct PropsConst {
  double unit_l, unit_d, unit_t, aexp, h0, hz, delta_vir;
  double pi, g, f43, third, sqrt2, mass_part, delta_x2, lmin_r, lmin_r178;
  int periodic, center_on_mass;
  long long threshold, tcalc;
};

// per-halo values handed from one kernel to the next
struct HaloWork {
  double comx[3], comv[3];
  double rmax, dispx, vmax, dispv, ekin;
  double ang[3];
  double inert[6];  // xx, xy, xz, yy, yz, zz
  double epot, epot_max;
  double cpot[3];
  long long np, m;  // members, members in the potential sum
};

__device__ __forceinline__ double p2(double x) { return x * x; }
__device__ __forceinline__ double p3(double x) { return x * x * x; }
__device__ __forceinline__ double p5(double x) {
  const double t = x * x;
  return (t * t) * x;
}

// fixed-order block reductions (every thread gets the result)
__device__ double block_sum_d(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = red[0];
    for (int q = 1; q < PR_TPB / 32; q++) s += red[q];
    red[PR_TPB / 32] = s;
  }
  __syncthreads();
  const double r = red[PR_TPB / 32];
  __syncthreads();
  return r;
}

__device__ double block_max_d(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = red[0];
    for (int q = 1; q < PR_TPB / 32; q++) s = fmax(s, red[q]);
    red[PR_TPB / 32] = s;
  }
  __syncthreads();
  const double r = red[PR_TPB / 32];
  __syncthreads();
  return r;
}

__device__ float block_max_f(float v, float *red) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    float s = red[0];
    for (int q = 1; q < PR_TPB / 32; q++) s = fmaxf(s, red[q]);
    red[PR_TPB / 32] = s;
  }
  __syncthreads();
  const float r = red[PR_TPB / 32];
  __syncthreads();
  return r;
}

// ---------------------------------------------------------------------------
// moments
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(PR_TPB) k_props_moments(PropsConst K, long long nh, const long long *off,
                                                          const unsigned *mem, const float4 *cube,
                                                          const unsigned *inv, const float *vel, float *hpos,
                                                          HaloWork *W) {
  __shared__ double red[PR_TPB / 32 + 1];
  __shared__ float redf[PR_TPB / 32 + 1];
  for (long long h = blockIdx.x; h < nh; h += gridDim.x) {
    const long long b = off[h], e = off[h + 1], np = e - b;
    // periodic unwrap (:181-190): per axis, when the halo spans more than
    // half a box, positions above 0.5 move down by one box (real(4))
    bool s1[3] = {false, false, false};
    if (K.periodic) {
      float mx[3] = {-3e38f, -3e38f, -3e38f}, mnn[3] = {-3e38f, -3e38f, -3e38f};  // mnn holds -min
      for (long long k = b + threadIdx.x; k < e; k += PR_TPB) {
        const float4 v = cube[inv[mem[k]]];
        const float x[3] = {v.x, v.y, v.z};
        for (int a = 0; a < 3; a++) {
          mx[a] = fmaxf(mx[a], x[a]);
          mnn[a] = fmaxf(mnn[a], -x[a]);
        }
      }
      for (int a = 0; a < 3; a++) {
        const float hi = block_max_f(mx[a], redf), lo = -block_max_f(mnn[a], redf);
        s1[a] = __fsub_rn(hi, lo) > 0.5f;
      }
    }
    // centre of mass and mean velocity
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (long long k = b + threadIdx.x; k < e; k += PR_TPB) {
      const unsigned i = mem[k];
      const float4 v = cube[inv[i]];
      float x[3] = {v.x, v.y, v.z};
      for (int a = 0; a < 3; a++) {
        if (s1[a] && x[a] > 0.5f) x[a] = __fsub_rn(x[a], 1.0f);
        s[a] += (double)x[a];
        s[3 + a] += vel ? (double)vel[3ull * i + a] : 0.0;
      }
    }
    double comx[3], comv[3];
    const double npf = (double)(float)np;
    for (int a = 0; a < 3; a++) {
      comx[a] = block_sum_d(s[a], red) / npf;
      comv[a] = block_sum_d(s[3 + a], red) / npf;
    }
    bool s2[3] = {false, false, false};
    if (K.periodic)
      for (int a = 0; a < 3; a++)
        if (comx[a] < 0.0) {
          comx[a] = comx[a] + 1.0;
          s2[a] = true;
        }
    // every sum over the members, with the positions as the reference holds
    // them after both shifts; the staged copy serves the later passes
    double rmax = 0.0, dispx = 0.0, vmax = 0.0, dispv = 0.0, ang[3] = {0, 0, 0}, in[6] = {0, 0, 0, 0, 0, 0};
    for (long long k = b + threadIdx.x; k < e; k += PR_TPB) {
      const unsigned i = mem[k];
      const float4 v = cube[inv[i]];
      float x[3] = {v.x, v.y, v.z};
      for (int a = 0; a < 3; a++) {
        if (s1[a] && x[a] > 0.5f) x[a] = __fsub_rn(x[a], 1.0f);
        if (s2[a]) x[a] = __fadd_rn(x[a], 1.0f);
        hpos[3 * k + a] = x[a];
      }
      const double q[3] = {(double)x[0] - comx[0], (double)x[1] - comx[1], (double)x[2] - comx[2]};
      const double vv[3] = {vel ? (double)vel[3ull * i] - comv[0] : -comv[0],
                            vel ? (double)vel[3ull * i + 1] - comv[1] : -comv[1],
                            vel ? (double)vel[3ull * i + 2] - comv[2] : -comv[2]};
      const double r2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
      rmax = fmax(rmax, sqrt(r2));
      dispx += r2;
      const double u0 = vv[0] + (q[0] * K.hz), u1 = vv[1] + (q[1] * K.hz), u2 = vv[2] + (q[2] * K.hz);
      const double u2s = u0 * u0 + u1 * u1 + u2 * u2;
      vmax = fmax(vmax, sqrt(u2s));
      dispv += u2s;
      ang[0] = ang[0] + K.mass_part * q[1] * vv[2] - K.mass_part * q[2] * vv[1];
      ang[1] = ang[1] + K.mass_part * q[2] * vv[0] - K.mass_part * q[0] * vv[2];
      ang[2] = ang[2] + K.mass_part * q[0] * vv[1] - K.mass_part * q[1] * vv[0];
      in[0] += q[0] * q[0];
      in[1] += q[0] * q[1];
      in[2] += q[0] * q[2];
      in[3] += q[1] * q[1];
      in[4] += q[1] * q[2];
      in[5] += q[2] * q[2];
    }
    const double t_rmax = block_max_d(rmax, red), t_vmax = block_max_d(vmax, red);
    const double t_dispx = block_sum_d(dispx, red), t_dispv = block_sum_d(dispv, red);
    double t_ang[3], t_in[6];
    for (int a = 0; a < 3; a++) t_ang[a] = block_sum_d(ang[a], red);
    for (int a = 0; a < 6; a++) t_in[a] = block_sum_d(in[a], red);
    if (threadIdx.x == 0) {
      HaloWork &w = W[h];
      for (int a = 0; a < 3; a++) {
        w.comx[a] = comx[a];
        w.comv[a] = comv[a];
        w.ang[a] = t_ang[a];
      }
      for (int a = 0; a < 6; a++) w.inert[a] = t_in[a];
      w.rmax = t_rmax;
      w.vmax = t_vmax;
      w.dispx = t_dispx;
      w.dispv = t_dispv;
      w.ekin = t_dispv;  // the kinetic sum has the same terms (:343-347)
      w.np = np;
      w.m = np < K.threshold ? np : K.tcalc;
    }
  }
}

// ---------------------------------------------------------------------------
// potential: member i of the halo's potential list (every member, or the
// sample of K.tcalc members of a halo of at least K.threshold) against all
// the others; the pair term is real(4) up to the smoothing term (:369-371)
// ---------------------------------------------------------------------------
__device__ __forceinline__ long long pot_member(long long k, long long np, long long m) {
  return m == np ? k : (k * np) / m;
}

__global__ void __launch_bounds__(PR_TPB) k_props_potential(PropsConst K, const long long *ipref, long long nitem,
                                                            const unsigned *ihalo, const long long *off,
                                                            const HaloWork *W, const float *hpos, double *epi) {
  __shared__ float tx[PR_TPB], ty[PR_TPB], tz[PR_TPB];
  const double mp2 = K.mass_part * K.mass_part;
  for (long long it = blockIdx.x; it < nitem; it += gridDim.x) {
    const unsigned h = ihalo[it];
    const long long chunk = it - ipref[h];
    const long long b = off[h], np = W[h].np, m = W[h].m;
    const long long ii = chunk * PR_TPB + threadIdx.x;
    const bool have = ii < m;
    float xi = 0.f, yi = 0.f, zi = 0.f;
    if (have) {
      const long long k = b + pot_member(ii, np, m);
      xi = hpos[3 * k];
      yi = hpos[3 * k + 1];
      zi = hpos[3 * k + 2];
    }
    double ei = 0.0;
    for (long long j0 = 0; j0 < m; j0 += PR_TPB) {
      const long long jj = j0 + threadIdx.x;
      __syncthreads();
      if (jj < m) {
        const long long k = b + pot_member(jj, np, m);
        tx[threadIdx.x] = hpos[3 * k];
        ty[threadIdx.x] = hpos[3 * k + 1];
        tz[threadIdx.x] = hpos[3 * k + 2];
      }
      __syncthreads();
      const int nt = (int)min((long long)PR_TPB, m - j0);
      if (have)
        for (int t = 0; t < nt; t++) {
          if (j0 + t == ii) continue;
          const float ax = xi - tx[t], ay = yi - ty[t], az = zi - tz[t];
          const float s3 = ax * ax + ay * ay + az * az;
          ei = ei + mp2 / sqrt((double)s3 + K.delta_x2);
        }
    }
    if (have) epi[b + ii] = ei;
  }
}

// ---------------------------------------------------------------------------
// finish
// ---------------------------------------------------------------------------
// the bin of log r in [lmin + (j-1) dl, lmin + j dl), j = 1..nb, with the
// reference's per-bin comparisons; 0 below the first edge, -1 beyond
__device__ __forceinline__ int log_bin(double lr, double lmin, double dl, int nb) {
  if (lr < lmin) return 0;
  int j = (int)floor((lr - lmin) / dl) + 1;
  if (j < 1) j = 1;
  if (j > nb + 1) j = nb + 1;
  // settle on the reference's edges (the quotient can be one off)
  while (j > 1 && lr < lmin + (j - 1) * dl) j--;
  while (j <= nb && !(lr < lmin + j * dl)) j++;
  if (j > nb) return -1;
  return (lmin + (j - 1) * dl <= lr && lr < lmin + j * dl) ? j : -1;
}

struct PropsOut {
  long long *npart;
  double *mvir, *rvir, *rvircom, *vvir;
  float *com, *comv, *rmax, *vmax, *dispx, *dispv, *ekin, *epot, *lambda, *lambda_prime, *eig_val, *eig_vec;
  double *cos_alpha;
  float *center_pot, *circ, *delta_vals, *dens, *dens_int, *vcirc, *dens178, *dens_int178;
};

__global__ void __launch_bounds__(PR_TPB) k_props_finish(PropsConst K, long long nh, const long long *off,
                                                         HaloWork *W, const float *hpos, const double *epi,
                                                         PropsOut o) {
  __shared__ double red[PR_TPB / 32 + 1];
  __shared__ unsigned long long s_arg;
  __shared__ unsigned hist1[NB1 + 1], hist2[NB2 + 1];
  __shared__ double s_r178;
  for (long long h = blockIdx.x; h < nh; h += gridDim.x) {
    HaloWork &w = W[h];
    const long long b = off[h], np = w.np, m = w.m;
    // total potential (member order in fixed-order pieces) and the first
    // member of largest potential sum (strict >, :383-386)
    double es = 0.0, emx = -1.0;
    long long earg = 0x7fffffffffffffffll;
    for (long long k = threadIdx.x; k < m; k += PR_TPB) {
      const double v = epi[b + k];
      es += v;
      if (v > emx) {
        emx = v;
        earg = k;
      }
    }
    const double epot_sum = block_sum_d(es, red);
    const double emax = block_max_d(emx, red);
    if (threadIdx.x == 0) s_arg = ~0ull;
    __syncthreads();
    if (emx == emax && emax > 0.0) atomicMin(&s_arg, (unsigned long long)earg);
    __syncthreads();
    double cpot[3] = {0, 0, 0};
    if (s_arg != ~0ull) {
      const long long k = b + pot_member((long long)s_arg, np, m);
      for (int a = 0; a < 3; a++) cpot[a] = (double)hpos[3 * k + a];
    }
    const double *cen = K.center_on_mass ? w.comx : cpot;
    const double M_vir = (double)np * K.mass_part * K.unit_d * p3(K.unit_l);
    const double R_vir = pow(3 * M_vir / (4 * K.pi * K.delta_vir * K.unit_d), K.third);
    const double V_vir = sqrt(K.g * M_vir / R_vir);
    const double h100 = K.h0 / 100.0;
    const double Rho_m = K.unit_d;
    // first histogram (:440-455)
    for (int j = threadIdx.x; j <= NB1; j += PR_TPB) hist1[j] = 0;
    for (int j = threadIdx.x; j <= NB2; j += PR_TPB) hist2[j] = 0;
    __syncthreads();
    for (long long k = b + threadIdx.x; k < b + np; k += PR_TPB) {
      const double dx = (double)hpos[3 * k] - cen[0], dy = (double)hpos[3 * k + 1] - cen[1],
                   dz = (double)hpos[3 * k + 2] - cen[2];
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      r = r * K.unit_l / (MPC / 1e3);
      const int j = log_bin(log(r), K.lmin_r, DELTA_LR, NB1);
      if (j >= 0) atomicAdd(&hist1[j], 1u);  // bin 0: inside the first edge
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double dint[NB1];
      double V_circ_max = 0.0, M_circ_max = 0.0, R_circ_max = 0.0, Rho_circ_max = 0.0;
      long long cum = hist1[0];
      for (int j = 1; j <= NB1; j++) {
        double d = (double)hist1[j] * K.mass_part * K.unit_d * p3(K.unit_l) / MSUN * h100;
        d = d / (K.f43 * K.pi * (p3(exp(K.lmin_r + j * DELTA_LR)) - p3(exp(K.lmin_r + (j - 1) * DELTA_LR))));
        d = d * MSUN / h100 / p3(MPC / 1e3);
        d = d / Rho_m;
        cum += hist1[j];
        double di = (double)cum * K.mass_part * K.unit_d * p3(K.unit_l);
        const double R_tmp = exp(K.lmin_r + j * DELTA_LR) * (MPC / 1e3);
        const double vc = sqrt(K.g * di / R_tmp);
        if (vc > V_circ_max) {
          V_circ_max = vc;
          M_circ_max = di / MSUN * h100;
          R_circ_max = R_tmp / (MPC / 1e3) * h100;
          Rho_circ_max = di / (K.f43 * K.pi * p3(R_tmp));
          Rho_circ_max = Rho_circ_max / Rho_m;
        }
        di = di / (K.f43 * K.pi * p3(R_tmp));
        di = di / Rho_m;
        dint[j - 1] = di;
        o.vcirc[NB1 * h + j - 1] = (float)(vc / 1e5);
        o.dens[NB1 * h + j - 1] = (float)d;
        o.dens_int[NB1 * h + j - 1] = (float)di;
      }
      // R178 interpolation (:567-602), Fortran's 1-based j
      int j = 1;
      bool never = true;
      const double Dm = K.delta_vir;
      while ((dint[j - 1] > Dm && j < NB1) || (never && j < NB1) || (j < 10 && j < NB1)) {
        if (never && dint[j - 1] > Dm) never = false;
        j++;
      }
      double R_tmp = (K.lmin_r + j * DELTA_LR) * (log(Dm) - log(dint[j - 2])) / (log(dint[j - 1]) - log(dint[j - 2])) +
                     (K.lmin_r + (j - 1) * DELTA_LR) * (log(Dm) - log(dint[j - 1])) /
                         (log(dint[j - 2]) - log(dint[j - 1]));
      R_tmp = exp(R_tmp) * (MPC / 1e3);
      const double R178 = R_tmp / (MPC / 1e3);
      double M178 = (K.f43 * K.pi * p3(R_tmp)) * Dm * Rho_m;
      M178 = M178 / MSUN * h100;
      s_r178 = R178;
      o.circ[4 * h + 0] = (float)M_circ_max;
      o.circ[4 * h + 1] = (float)R_circ_max;
      o.circ[4 * h + 2] = (float)(V_circ_max / 1e5);
      o.circ[4 * h + 3] = (float)Rho_circ_max;
      o.delta_vals[2 * h + 0] = (float)M178;
      o.delta_vals[2 * h + 1] = (float)(R178 * K.h0 / 100.0);
    }
    __syncthreads();
    const double R178 = s_r178;
    for (long long k = b + threadIdx.x; k < b + np; k += PR_TPB) {
      const double dx = (double)hpos[3 * k] - cen[0], dy = (double)hpos[3 * k + 1] - cen[1],
                   dz = (double)hpos[3 * k + 2] - cen[2];
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      r = r * K.unit_l / (MPC / 1e3);
      r = r / R178;
      const int j = log_bin(log(r), K.lmin_r178, DELTA_LR178, NB2);
      if (j >= 0) atomicAdd(&hist2[j], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      long long cum = hist2[0];
      for (int j = 1; j <= NB2; j++) {
        double d = (double)hist2[j] * K.mass_part * K.unit_d * p3(K.unit_l) / MSUN * h100;
        d = d / p3(R178) /
            (K.f43 * K.pi * (p3(exp(K.lmin_r178 + j * DELTA_LR178)) - p3(exp(K.lmin_r178 + (j - 1) * DELTA_LR178))));
        d = d * MSUN / h100 / p3(MPC / 1e3);
        d = d / Rho_m;
        cum += hist2[j];
        double di = (double)cum * K.mass_part * K.unit_d * p3(K.unit_l);
        const double Rt = exp(K.lmin_r178 + j * DELTA_LR178) * R178 * (MPC / 1e3);
        di = di / (K.f43 * K.pi * p3(Rt));
        di = di / Rho_m;
        o.dens178[NB2 * h + j - 1] = (float)d;
        o.dens_int178[NB2 * h + j - 1] = (float)di;
      }
      // scalar outputs (:280-300, 312-313, 327-331, 350-354, 400-438, 672-720)
      const double conv = K.h0 / 100.0 / K.aexp;
      o.npart[h] = np;
      o.mvir[h] = M_vir / MSUN * K.h0 / 100.0;
      o.rvir[h] = R_vir / (MPC / 1e3) * K.h0 / 100.0;
      o.rvircom[h] = R_vir / (MPC / 1e3) * K.h0 / 100.0 / K.aexp;
      o.vvir[h] = V_vir / 1e5;
      for (int a = 0; a < 3; a++) {
        o.com[3 * h + a] = (float)(w.comx[a] * K.unit_l / MPC * conv);
        o.comv[3 * h + a] = (float)(w.comv[a] * K.unit_l / K.unit_t / 1e5);
        o.center_pot[3 * h + a] = (float)(cpot[a] * K.unit_l / MPC * conv);
      }
      const double npf = (double)(float)np;
      o.rmax[h] = (float)(w.rmax * K.unit_l / MPC / (R_vir / MPC));
      o.dispx[h] = (float)(sqrt(w.dispx / npf) * K.unit_l / MPC / (R_vir / MPC));
      o.vmax[h] = (float)(w.vmax * K.unit_l / K.unit_t / 1e5 / (V_vir / 1e5));
      o.dispv[h] = (float)(sqrt(w.dispv / npf) * K.unit_l / K.unit_t / 1e5 / (V_vir / 1e5));
      double Ekin = 0.5 * K.mass_part * w.ekin;
      Ekin = Ekin * K.unit_d * p3(K.unit_l) * p2(K.unit_l) * (1.0 / p2(K.unit_t));
      const double scale = p2(K.unit_d * p3(K.unit_l)) * (1.0 / K.unit_l);
      double Epot;
      if (np < K.threshold) {
        Epot = -0.5 * K.g * epot_sum * scale;
      } else {
        const double n = (double)np, t = (double)K.tcalc;
        Epot = -((n * n - n) / (t * t - t) * 0.5 * K.g * epot_sum * scale);
      }
      const double Etot = Ekin + Epot;
      const double ev = 0.5 * M_vir / MSUN * p2(V_vir / 1e5);
      o.epot[h] = (float)(Epot / (MSUN * 1e10) / ev);
      o.ekin[h] = (float)(Ekin / (MSUN * 1e10) / ev);
      double ang[3];
      for (int a = 0; a < 3; a++) ang[a] = w.ang[a] * K.unit_d * p5(K.unit_l) / K.unit_t;
      for (int a = 0; a < 3; a++) {
        o.lambda[3 * h + a] = (float)(ang[a] * sqrt(fabs(Etot)) / (K.g * pow(M_vir, 2.5)));
        o.lambda_prime[3 * h + a] = (float)(ang[a] / (K.sqrt2 * M_vir * R_vir * V_vir));
      }
      double A[3][3] = {{w.inert[0] / npf, w.inert[1] / npf, w.inert[2] / npf},
                        {w.inert[1] / npf, w.inert[3] / npf, w.inert[4] / npf},
                        {w.inert[2] / npf, w.inert[4] / npf, w.inert[5] / npf}};
      double d[3], v[3][3];
      jacobi3(A, d, v);
      eigsort3(d, v);
      for (int a = 0; a < 3; a++) {
        o.eig_val[3 * h + a] = (float)(sqrt(d[a]) * K.unit_l / MPC / (R_vir / MPC));
        o.eig_vec[3 * h + a] = (float)v[a][2];
      }
      o.cos_alpha[h] = (v[0][2] * ang[0] + v[1][2] * ang[1] + v[2][2] * ang[2]) /
                       sqrt((v[0][2] * v[0][2] + v[1][2] * v[1][2] + v[2][2] * v[2][2]) *
                            (ang[0] * ang[0] + ang[1] * ang[1] + ang[2] * ang[2]));
    }
    __syncthreads();
  }
}

// potential work items: ceil(m / PR_TPB) per halo
__global__ void k_props_items(const HaloWork *W, long long nh, unsigned *cnt) {
  const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (h < nh) cnt[h] = (unsigned)((W[h].m + PR_TPB - 1) / PR_TPB);
}

__global__ void k_props_item_halo(const unsigned *pref, long long nh, unsigned *ihalo) {
  const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= nh) return;
  for (unsigned q = pref[h]; q < pref[h + 1]; q++) ihalo[q] = (unsigned)h;
}

__global__ void k_props_pref64(const unsigned *pref, long long nh, long long *out) {
  const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (h <= nh) out[h] = pref[h];
}

unsigned grid_of(long long n, int tpb = PR_TPB) { return (unsigned)((n + tpb - 1) / tpb); }

}  // namespace
}  // namespace psod

using namespace psod;

extern "C" {

int psod_halo_properties(psod_ctx *c, const psod_props_params *p, psod_props_stats *stats) {
  if (!c || !p) return PSOD_ERR_ARG;
  cudaSetDevice(c->device);
  c->props_done = false;
  const long long *off = nullptr;
  const unsigned *mem = nullptr;
  long long nh = 0;
  if (p->source == PSOD_PROPS_FROM_SOD) {
    if (!c->sod_done) return set_err(c, PSOD_ERR_STATE, "psod_halo_properties: no halo table (call psod_spherover)");
    off = c->d_m_offset;
    mem = c->d_m_index;
    nh = c->nhalo;
  } else if (p->source == PSOD_PROPS_FROM_FOF) {
    if (!c->fof_done) return set_err(c, PSOD_ERR_STATE, "psod_halo_properties: no FoF catalogue (call psod_fof)");
    off = static_cast<const long long *>(c->scratch[SLOT_F_OFF].first);
    mem = static_cast<const unsigned *>(c->scratch[SLOT_F_MEM].first);
    nh = c->fof_nhalo;
  } else {
    return set_err(c, PSOD_ERR_ARG, "psod_halo_properties: source must be PSOD_PROPS_FROM_SOD or PSOD_PROPS_FROM_FOF");
  }
  if (!(p->unit_l > 0) || !(p->unit_d > 0) || !(p->unit_t > 0) || !(p->aexp > 0) || !(p->h0 > 0) ||
      !(p->delta_vir > 0) || p->levelmin < 0 || p->levelmin > 30 || p->epot_threshold < 20)
    return set_err(c, PSOD_ERR_ARG, "psod_halo_properties: units, aexp, h0, delta_vir must be > 0, 0 <= levelmin <= 30, "
                                    "epot_threshold >= 20");
  PropsConst K;
  K.unit_l = p->unit_l;
  K.unit_d = p->unit_d;
  K.unit_t = p->unit_t;
  K.aexp = p->aexp;
  K.h0 = p->h0;
  K.hz = p->hz;
  K.delta_vir = p->delta_vir;
  K.pi = (double)3.14159265359879f;  // real(8) :: PI=3.14159265359879 (a default-real literal)
  K.g = (double)6.6731E-08f;         // real(8) :: G=6.6731E-08
  K.f43 = (double)(4.0f / 3.0f);
  K.third = (double)(1.0f / 3.0f);
  K.sqrt2 = (double)sqrtf(2.0f);
  K.mass_part = 1.0 / std::pow(std::pow(2.0, (double)p->levelmin), 3.0);
  {
    const float dxf = (1.0f / (float)std::pow(2.0, (double)p->levelmin)) * (1.0f / 64.0f);
    K.delta_x2 = (double)dxf * (double)dxf;
  }
  K.lmin_r = std::log(MIN_R);
  K.lmin_r178 = std::log(MIN_R178);
  K.periodic = p->periodic != 0;
  K.center_on_mass = p->center_on_mass != 0;
  K.threshold = p->epot_threshold;
  K.tcalc = (long long)((float)p->epot_threshold / 10.0f);
  int st = wait_ids(c);
  if (st) return st;
  long long nm = 0;
  if (nh > 0) PSOD_CUDA(c, cudaMemcpyAsync(&nm, off + nh, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, c->stream);
  float *hpos = nullptr;
  double *epi = nullptr;
  HaloWork *W = nullptr;
  unsigned *cnt = nullptr, *ihalo = nullptr;
  long long *ipref = nullptr;
  if ((st = scratch(c, SLOT_PR_POS, (size_t)3 * nm + 3, &hpos))) return st;
  if ((st = scratch(c, SLOT_PR_EPI, (size_t)nm + 1, &epi))) return st;
  if ((st = scratch(c, SLOT_PR_WORK, (size_t)nh + 1, &W))) return st;
  if ((st = scratch(c, SLOT_PR_CNT, (size_t)nh + 1, &cnt))) return st;
  if ((st = scratch(c, SLOT_PR_PREF, (size_t)nh + 1, &ipref))) return st;
  // outputs
  PropsOut o;
  auto out = [&](int slot, size_t count, auto **ptr) { return scratch(c, slot, count, ptr); };
  if ((st = out(SLOT_PO_NPART, nh + 1, &o.npart)) || (st = out(SLOT_PO_VIR, 4 * nh + 4, &o.mvir))) return st;
  o.rvir = o.mvir + nh;
  o.rvircom = o.mvir + 2 * nh;
  o.vvir = o.mvir + 3 * nh;
  float *f = nullptr;
  // float outputs in one slot: 3+3+1+1+1+1+1+1+3+3+3+3+3+4+2 + 3*NB1 + 2*NB2 per halo
  const size_t per = 3 + 3 + 1 + 1 + 1 + 1 + 1 + 1 + 3 + 3 + 3 + 3 + 3 + 4 + 2 + 3 * NB1 + 2 * NB2;
  if ((st = out(SLOT_PO_F32, per * nh + 1, &f))) return st;
  if ((st = out(SLOT_PO_COS, nh + 1, &o.cos_alpha))) return st;
  {
    float *q = f;
    auto take = [&](float **dst, size_t k) {
      *dst = q;
      q += k * nh;
    };
    take(&o.com, 3);
    take(&o.comv, 3);
    take(&o.rmax, 1);
    take(&o.vmax, 1);
    take(&o.dispx, 1);
    take(&o.dispv, 1);
    take(&o.ekin, 1);
    take(&o.epot, 1);
    take(&o.lambda, 3);
    take(&o.lambda_prime, 3);
    take(&o.eig_val, 3);
    take(&o.eig_vec, 3);
    take(&o.center_pot, 3);
    take(&o.circ, 4);
    take(&o.delta_vals, 2);
    take(&o.dens, NB1);
    take(&o.dens_int, NB1);
    take(&o.vcirc, NB1);
    take(&o.dens178, NB2);
    take(&o.dens_int178, NB2);
  }
  c->props_out = {o.npart, o.mvir, o.com, o.cos_alpha};
  psod_props_stats S{};
  if (nh > 0) {
    k_props_moments<<<148 * 4, PR_TPB, 0, c->stream>>>(K, nh, off, mem, c->d_cube, c->d_inv, c->d_vel, hpos, W);
    k_props_items<<<grid_of(nh), PR_TPB, 0, c->stream>>>(W, nh, cnt);
    if ((st = scan_u32(c, cnt, cnt, nh, true))) return st;
    unsigned nitem_u = 0;
    PSOD_CUDA(c, cudaMemcpyAsync(&nitem_u, cnt + nh, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
    const long long nitem = nitem_u;
    if ((st = scratch(c, SLOT_PR_IHALO, (size_t)nitem + 1, &ihalo))) return st;
    k_props_item_halo<<<grid_of(nh), PR_TPB, 0, c->stream>>>(cnt, nh, ihalo);
    k_props_pref64<<<grid_of(nh + 1), PR_TPB, 0, c->stream>>>(cnt, nh, ipref);
    k_props_potential<<<148 * 8, PR_TPB, 0, c->stream>>>(K, ipref, nitem, ihalo, off, W, hpos, epi);
    k_props_finish<<<148 * 4, PR_TPB, 0, c->stream>>>(K, nh, off, W, hpos, epi, o);
    PSOD_CUDA(c, cudaGetLastError());
    S.potential_items = nitem;
  }
  cudaEventRecord(e1, c->stream);
  PSOD_CUDA(c, cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  S.nhalo = nh;
  S.nmember = nm;
  S.ms_total = ms;
  c->props_nhalo = nh;
  c->props_done = true;
  if (stats) *stats = S;
  return PSOD_OK;
}

int psod_props_get(psod_ctx *c, const psod_props_table *t) {
  if (!c || !t) return PSOD_ERR_ARG;
  if (!c->props_done) return set_err(c, PSOD_ERR_STATE, "no halo properties: call psod_halo_properties first");
  cudaSetDevice(c->device);
  const long long nh = c->props_nhalo;
  const long long *npart = static_cast<const long long *>(c->props_out.npart);
  const double *vir = static_cast<const double *>(c->props_out.vir);
  const float *f = static_cast<const float *>(c->props_out.f32);
  const double *cosa = static_cast<const double *>(c->props_out.cos);
  int st;
  struct F {
    float *dst;
    size_t k;
  };
  const F fl[] = {{t->com, 3},         {t->comv, 3},    {t->rmax, 1},     {t->vmax, 1},         {t->dispx, 1},
                  {t->dispv, 1},       {t->ekin, 1},    {t->epot, 1},     {t->lambda, 3},       {t->lambda_prime, 3},
                  {t->eig_val, 3},     {t->eig_vec, 3}, {t->center_pot, 3}, {t->circ, 4},       {t->delta_vals, 2},
                  {t->dens, (size_t)NB1}, {t->dens_int, (size_t)NB1}, {t->vcirc, (size_t)NB1},
                  {t->dens178, (size_t)NB2}, {t->dens_int178, (size_t)NB2}};
  if (t->npart && (st = copy_out(c, t->npart, npart, sizeof(int64_t) * nh))) return st;
  double *const vd[4] = {t->mvir, t->rvir, t->rvircom, t->vvir};
  for (int k = 0; k < 4; k++)
    if (vd[k] && (st = copy_out(c, vd[k], vir + k * nh, sizeof(double) * nh))) return st;
  const float *q = f;
  for (const F &x : fl) {
    if (x.dst && (st = copy_out(c, x.dst, q, sizeof(float) * x.k * nh))) return st;
    q += x.k * nh;
  }
  if (t->cos_alpha && (st = copy_out(c, t->cos_alpha, cosa, sizeof(double) * nh))) return st;
  PSOD_CUDA(c, cudaStreamSynchronize(c->stream));
  return PSOD_OK;
}

}  // extern "C"
