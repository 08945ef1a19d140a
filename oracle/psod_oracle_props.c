/*
 * psod_oracle_props.c -- CPU oracle for haloanalyzer's halo_properties
 * (test infrastructure only: tests/ and bench.py's cpu_baseline leg use it
 * as the checker; nothing in the product links it).
 *
 * A single-threaded restatement of haloanalyzer_new/src/modfunctions.f90
 * halo_properties (:47-808) for one halo at a time, at a fixed redshift
 * (do_lightcone false) and without the volume estimate (compute_volume is
 * false there), in the statement order and precision of the Fortran:
 * positions and velocities are real(4) and are shifted in place in real(4)
 * (periodic unwrap :181-190, :198-207), the centre and every sum are
 * real(8), and the module's constants keep the values their default-real
 * literals give them (PI = 3.14159265359879 and G = 6.6731E-08 are single
 * literals stored in real(8), modvariables.f90:262-263; 4./3., 1./3.,
 * sqrt(2.) are single values promoted in the expressions).  The Makefile
 * builds it with -ffp-contract=off, like the reference's -O2 x86-64 build.
 *
 * Two departures, both shared with the GPU path:
 *   - halos of at least epot_threshold members: the reference draws
 *     threshold/10 members with random_number for the potential energy
 *     (:364-399); that draw has no reproducible target, so both paths use
 *     the members at positions floor(k*np/(threshold/10)), k = 0, 1, ...;
 *   - the eigen solver is the cyclic Jacobi method with thresholds
 *     (Rutishauser's, as published in Numerical Recipes' jacobi), which the
 *     reference's diag (:840-933) follows; eigsrt (:812-837) sorts the
 *     eigenvalues in descending order.
 */
#include "psod_oracle_props.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NB1 PSOD_ORACLE_PROPS_NBIN1
#define NB2 PSOD_ORACLE_PROPS_NBIN2

static const double MSUN = 1.98892e33, MPC = 3.08568e24;
/* real(8) variables initialised from default-real literals */
static double pi_(void) { return (double)3.14159265359879f; }
static double g_(void) { return (double)6.6731E-08f; }
static double four3(void) { return (double)(4.0f / 3.0f); }
static double third(void) { return (double)(1.0f / 3.0f); }
static double sqrt2f(void) { return (double)sqrtf(2.0f); }

static const double MIN_R = 1.0, DELTA_LR = 0.1, MIN_R178 = 1e-2, DELTA_LR178 = 0.2;

/* integer powers as gfortran evaluates x**n for small constant n */
static double p2(double x) { return x * x; }
static double p3(double x) { return x * x * x; }
static double p5(double x) {
  const double t = x * x;
  return (t * t) * x;
}

/* cyclic Jacobi rotations on a symmetric 3x3 matrix (row-major a[i][j]
   with i < j above the diagonal); d gets the eigenvalues, v the
   eigenvectors as columns */
static void jacobi3(double a[3][3], double d[3], double v[3][3]) {
  double b[3], z[3];
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) v[i][j] = 0.0;
    v[i][i] = 1.0;
    b[i] = d[i] = a[i][i];
    z[i] = 0.0;
  }
  for (int sweep = 1; sweep <= 50; sweep++) {
    double sm = 0.0;
    for (int p = 0; p < 2; p++)
      for (int q = p + 1; q < 3; q++) sm += fabs(a[p][q]);
    if (sm == 0.0) return;
    const double tresh = sweep < 4 ? (double)0.2f * sm / 9.0 : 0.0;  /* 0.2 is a default-real literal */
    for (int p = 0; p < 2; p++)
      for (int q = p + 1; q < 3; q++) {
        double g = 100.0 * fabs(a[p][q]);
        if (sweep > 4 && fabs(d[p]) + g == fabs(d[p]) && fabs(d[q]) + g == fabs(d[q])) {
          a[p][q] = 0.0;
        } else if (fabs(a[p][q]) > tresh) {
          double h = d[q] - d[p], t;
          if (fabs(h) + g == fabs(h)) {
            t = a[p][q] / h;
          } else {
            const double theta = 0.5 * h / a[p][q];
            t = 1.0 / (fabs(theta) + sqrt(1.0 + theta * theta));
            if (theta < 0.0) t = -t;
          }
          const double c = 1.0 / sqrt(1 + t * t), s = t * c, tau = s / (1.0 + c);
          h = t * a[p][q];
          z[p] -= h;
          z[q] += h;
          d[p] -= h;
          d[q] += h;
          a[p][q] = 0.0;
          for (int j = 0; j < p; j++) {
            g = a[j][p];
            h = a[j][q];
            a[j][p] = g - s * (h + g * tau);
            a[j][q] = h + s * (g - h * tau);
          }
          for (int j = p + 1; j < q; j++) {
            g = a[p][j];
            h = a[j][q];
            a[p][j] = g - s * (h + g * tau);
            a[j][q] = h + s * (g - h * tau);
          }
          for (int j = q + 1; j < 3; j++) {
            g = a[p][j];
            h = a[q][j];
            a[p][j] = g - s * (h + g * tau);
            a[q][j] = h + s * (g - h * tau);
          }
          for (int j = 0; j < 3; j++) {
            g = v[j][p];
            h = v[j][q];
            v[j][p] = g - s * (h + g * tau);
            v[j][q] = h + s * (g - h * tau);
          }
        }
      }
    for (int p = 0; p < 3; p++) {
      b[p] += z[p];
      d[p] = b[p];
      z[p] = 0.0;
    }
  }
}

/* descending eigenvalues, a later equal value moving first (eigsrt's .ge.) */
static void eigsort3(double d[3], double v[3][3]) {
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

static void one_halo(const psod_oracle_props_params *P, int64_t np, float *pos, const float *vel, int64_t h,
                     const psod_oracle_props_out *o) {
  const double PI = pi_(), G = g_(), F43 = four3();
  const double h100 = P->h0 / 100.0, conv = P->h0 / 100.0 / P->aexp;
  const double unit_l = P->unit_l, unit_d = P->unit_d, unit_t = P->unit_t, Hz = P->hz;
  const double Rho_m = unit_d;
  const double mass_part = 1.0 / pow(pow(2.0, (double)P->levelmin), 3.0);
  const double Delta_matter = P->delta_vir;
  const double lmin_r = log(MIN_R), lmin_r178 = log(MIN_R178);
#define X(i, a) pos[3 * (i) + (a)]
#define V(i, a) vel[3 * (i) + (a)]
  /* periodic unwrap (:181-190) */
  if (P->periodic)
    for (int j = 0; j < 3; j++) {
      float mx = X(0, j), mn = X(0, j);
      for (int64_t i = 1; i < np; i++) {
        if (X(i, j) > mx) mx = X(i, j);
        if (X(i, j) < mn) mn = X(i, j);
      }
      if (mx - mn > 0.5f)
        for (int64_t i = 0; i < np; i++)
          if (X(i, j) > 0.5f) X(i, j) = X(i, j) - 1.0f;
    }
  double comx[3] = {0, 0, 0}, comv[3] = {0, 0, 0};
  for (int64_t i = 0; i < np; i++)
    for (int a = 0; a < 3; a++) {
      comx[a] = comx[a] + (double)X(i, a);
      comv[a] = comv[a] + (double)V(i, a);
    }
  for (int a = 0; a < 3; a++) {
    comx[a] = comx[a] / (double)(float)np;
    comv[a] = comv[a] / (double)(float)np;
  }
  if (P->periodic)
    for (int j = 0; j < 3; j++)
      if (comx[j] < 0.0) {
        comx[j] = comx[j] + 1.0;
        for (int64_t i = 0; i < np; i++) X(i, j) = X(i, j) + 1.0f;
      }
  const double M_vir = (double)np * mass_part * unit_d * p3(unit_l);
  const double R_vir = pow(3 * M_vir / (4 * PI * Delta_matter * Rho_m), third());
  const double V_vir = sqrt(G * M_vir / R_vir);
  o->npart[h] = np;
  o->mvir[h] = M_vir / MSUN * P->h0 / 100.0;
  o->rvir[h] = R_vir / (MPC / 1e3) * P->h0 / 100.0;
  o->rvircom[h] = R_vir / (MPC / 1e3) * P->h0 / 100.0 / P->aexp;
  o->vvir[h] = V_vir / 1e5;
  for (int a = 0; a < 3; a++) {
    o->com[3 * h + a] = (float)(comx[a] * unit_l / MPC * conv);
    o->comv[3 * h + a] = (float)(comv[a] * unit_l / unit_t / 1e5);
  }
  /* R_max, DispX (:295-313) */
  double R_max = 0.0, DispX = 0.0;
  for (int64_t i = 0; i < np; i++) {
    const double dx = (double)X(i, 0) - comx[0], dy = (double)X(i, 1) - comx[1], dz = (double)X(i, 2) - comx[2];
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    if (r > R_max) R_max = r;
  }
  for (int64_t i = 0; i < np; i++) {
    const double dx = (double)X(i, 0) - comx[0], dy = (double)X(i, 1) - comx[1], dz = (double)X(i, 2) - comx[2];
    DispX = DispX + dx * dx + dy * dy + dz * dz;
  }
  DispX = sqrt(DispX / (double)(float)np);
  o->rmax[h] = (float)(R_max * unit_l / MPC / (R_vir / MPC));
  o->dispx[h] = (float)(DispX * unit_l / MPC / (R_vir / MPC));
  /* V_max, DispV, Ekin (:315-354) */
  double V_max = 0.0, DispV = 0.0, Ekin = 0.0;
  for (int64_t i = 0; i < np; i++) {
    const double ux = ((double)V(i, 0) - comv[0]) + (((double)X(i, 0) - comx[0]) * Hz);
    const double uy = ((double)V(i, 1) - comv[1]) + (((double)X(i, 1) - comx[1]) * Hz);
    const double uz = ((double)V(i, 2) - comv[2]) + (((double)X(i, 2) - comx[2]) * Hz);
    const double v = sqrt(ux * ux + uy * uy + uz * uz);
    if (v > V_max) V_max = v;
  }
  for (int64_t i = 0; i < np; i++) {
    const double ux = ((double)V(i, 0) - comv[0]) + (((double)X(i, 0) - comx[0]) * Hz);
    const double uy = ((double)V(i, 1) - comv[1]) + (((double)X(i, 1) - comx[1]) * Hz);
    const double uz = ((double)V(i, 2) - comv[2]) + (((double)X(i, 2) - comx[2]) * Hz);
    DispV = DispV + ux * ux + uy * uy + uz * uz;
  }
  DispV = sqrt(DispV / (double)(float)np);
  o->vmax[h] = (float)(V_max * unit_l / unit_t / 1e5 / (V_vir / 1e5));
  o->dispv[h] = (float)(DispV * unit_l / unit_t / 1e5 / (V_vir / 1e5));
  for (int64_t i = 0; i < np; i++) {
    const double ux = ((double)V(i, 0) - comv[0]) + (((double)X(i, 0) - comx[0]) * Hz);
    const double uy = ((double)V(i, 1) - comv[1]) + (((double)X(i, 1) - comx[1]) * Hz);
    const double uz = ((double)V(i, 2) - comv[2]) + (((double)X(i, 2) - comx[2]) * Hz);
    Ekin = Ekin + ux * ux + uy * uy + uz * uz;
  }
  Ekin = 0.5 * mass_part * Ekin;
  Ekin = Ekin * unit_d * p3(unit_l) * p2(unit_l) * (1.0 / p2(unit_t));
  /* potential energy (:356-420) */
  const double Delta_X = (double)((1.0f / (float)pow(2.0, (double)P->levelmin)) * (1.0f / 64.0f));
  const double dx2 = Delta_X * Delta_X, mp2 = mass_part * mass_part;
  const int64_t threshold = P->epot_threshold, tcalc = (int64_t)((float)threshold / 10.0f);
  double Epot = 0.0, Epot_max = 0.0, center_pot[3] = {0, 0, 0};
  {
    const int64_t m = np < threshold ? np : tcalc;
    int64_t *sel = (int64_t *)malloc(sizeof(int64_t) * (size_t)(m > 0 ? m : 1));
    for (int64_t k = 0; k < m; k++) sel[k] = np < threshold ? k : (k * np) / tcalc;
    for (int64_t ii = 0; ii < m; ii++) {
      const int64_t i = sel[ii];
      double Ei = 0.0;
      for (int64_t jj = 0; jj < m; jj++) {
        if (jj == ii) continue;
        const int64_t j = sel[jj];
        const float ax = X(i, 0) - X(j, 0), ay = X(i, 1) - X(j, 1), az = X(i, 2) - X(j, 2);
        const float s3 = ax * ax + ay * ay + az * az; /* real(4) up to the Delta_X term */
        Ei = Ei + mp2 / sqrt((double)s3 + dx2);
      }
      Epot = Epot + Ei;
      if (Ei > Epot_max) {
        Epot_max = Ei;
        for (int a = 0; a < 3; a++) center_pot[a] = (double)X(i, a);
      }
    }
    free(sel);
    const double scale = p2(unit_d * p3(unit_l)) * (1.0 / unit_l);
    if (np < threshold) {
      Epot = -0.5 * G * Epot * scale;
    } else {
      const double n = (double)np, t = (double)tcalc;
      Epot = -((n * n - n) / (t * t - t) * 0.5 * G * Epot * scale);
    }
  }
  const double Etot = Ekin + Epot;
  const double ev = 0.5 * M_vir / MSUN * p2(V_vir / 1e5);
  o->epot[h] = (float)(Epot / (MSUN * 1e10) / ev);
  o->ekin[h] = (float)(Ekin / (MSUN * 1e10) / ev);
  for (int a = 0; a < 3; a++) o->center_pot[3 * h + a] = (float)(center_pot[a] * unit_l / MPC * conv);
  /* radial profiles (:440-565) */
  int64_t dn[NB1], dn178[NB2];
  memset(dn, 0, sizeof(dn));
  memset(dn178, 0, sizeof(dn178));
  const double *cen = P->center_on_mass ? comx : center_pot;
  int64_t inner = 0;
  for (int64_t i = 0; i < np; i++) {
    const double dx = (double)X(i, 0) - cen[0], dy = (double)X(i, 1) - cen[1], dz = (double)X(i, 2) - cen[2];
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    r = r * unit_l / (MPC / 1e3);
    const double lr = log(r);
    if (lr < lmin_r) {
      inner++;
    } else {
      for (int j = 1; j <= NB1; j++)
        if (lmin_r + (j - 1) * DELTA_LR <= lr && lr < lmin_r + j * DELTA_LR) dn[j - 1]++;
    }
  }
  double dens[NB1], dint[NB1], vc[NB1];
  double V_circ_max = 0.0, M_circ_max = 0.0, R_circ_max = 0.0, Rho_circ_max = 0.0, Diff = 1e10, M178 = 0.0,
         R178 = 0.0;
  int64_t cum = inner;
  for (int j = 1; j <= NB1; j++) {
    double d = (double)dn[j - 1] * mass_part * unit_d * p3(unit_l) / MSUN * h100;
    d = d / (F43 * PI * (p3(exp(lmin_r + j * DELTA_LR)) - p3(exp(lmin_r + (j - 1) * DELTA_LR))));
    d = d * MSUN / h100 / p3(MPC / 1e3);
    d = d / Rho_m;
    dens[j - 1] = d;
    cum += dn[j - 1];
    double di = (double)cum * mass_part * unit_d * p3(unit_l);
    const double R_tmp = exp(lmin_r + j * DELTA_LR) * (MPC / 1e3);
    vc[j - 1] = sqrt(G * di / R_tmp);
    if (vc[j - 1] > V_circ_max) {
      V_circ_max = vc[j - 1];
      M_circ_max = di / MSUN * h100;
      R_circ_max = R_tmp / (MPC / 1e3) * h100;
      Rho_circ_max = di / (F43 * PI * p3(R_tmp));
      Rho_circ_max = Rho_circ_max / Rho_m;
    }
    di = di / (F43 * PI * p3(R_tmp));
    di = di / Rho_m;
    dint[j - 1] = di;
    if (fabs(di - Delta_matter) < Diff) {
      R178 = R_tmp / (MPC / 1e3);
      M178 = (F43 * PI * p3(R_tmp)) * di * Rho_m;
      M178 = M178 / MSUN * h100;
      Diff = fabs(di - Delta_matter);
    }
  }
  /* R178 interpolation (:567-602); Fortran's 1-based j kept */
  {
    const int jstart = 10;
    int j = 1;
    int never = 1;
#define DI(k) dint[(k) - 1]
    while ((DI(j) > Delta_matter && j < NB1) || (never && j < NB1) || (j < jstart && j < NB1)) {
      if (never && DI(j) > Delta_matter) never = 0;
      j++;
    }
    double R_tmp = (lmin_r + j * DELTA_LR) * (log(Delta_matter) - log(DI(j - 1))) / (log(DI(j)) - log(DI(j - 1))) +
                   (lmin_r + (j - 1) * DELTA_LR) * (log(Delta_matter) - log(DI(j))) / (log(DI(j - 1)) - log(DI(j)));
#undef DI
    R_tmp = exp(R_tmp) * (MPC / 1e3);
    R178 = R_tmp / (MPC / 1e3);
    M178 = (F43 * PI * p3(R_tmp)) * Delta_matter * Rho_m;
    M178 = M178 / MSUN * h100;
  }
  for (int j = 0; j < NB1; j++) {
    o->vcirc[NB1 * h + j] = (float)(vc[j] / 1e5);
    o->dens[NB1 * h + j] = (float)dens[j];
    o->dens_int[NB1 * h + j] = (float)dint[j];
  }
  o->circ[4 * h + 0] = (float)M_circ_max;
  o->circ[4 * h + 1] = (float)R_circ_max;
  o->circ[4 * h + 2] = (float)(V_circ_max / 1e5);
  o->circ[4 * h + 3] = (float)Rho_circ_max;
  o->delta_vals[2 * h + 0] = (float)M178;
  o->delta_vals[2 * h + 1] = (float)(R178 * P->h0 / 100.0);
  inner = 0;
  for (int64_t i = 0; i < np; i++) {
    const double dx = (double)X(i, 0) - cen[0], dy = (double)X(i, 1) - cen[1], dz = (double)X(i, 2) - cen[2];
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    r = r * unit_l / (MPC / 1e3);
    r = r / R178;
    const double lr = log(r);
    if (lr < lmin_r178) {
      inner++;
    } else {
      for (int j = 1; j <= NB2; j++)
        if (lmin_r178 + (j - 1) * DELTA_LR178 <= lr && lr < lmin_r178 + j * DELTA_LR178) dn178[j - 1]++;
    }
  }
  cum = inner;
  for (int j = 1; j <= NB2; j++) {
    double d = (double)dn178[j - 1] * mass_part * unit_d * p3(unit_l) / MSUN * h100;
    d = d / p3(R178) /
        (F43 * PI * (p3(exp(lmin_r178 + j * DELTA_LR178)) - p3(exp(lmin_r178 + (j - 1) * DELTA_LR178))));
    d = d * MSUN / h100 / p3(MPC / 1e3);
    d = d / Rho_m;
    cum += dn178[j - 1];
    double di = (double)cum * mass_part * unit_d * p3(unit_l);
    const double R_tmp = exp(lmin_r178 + j * DELTA_LR178) * R178 * (MPC / 1e3);
    di = di / (F43 * PI * p3(R_tmp));
    di = di / Rho_m;
    o->dens178[NB2 * h + j - 1] = (float)d;
    o->dens_int178[NB2 * h + j - 1] = (float)di;
  }
  /* angular momentum, spin (:672-690) */
  double ang[3] = {0, 0, 0};
  for (int64_t i = 0; i < np; i++) {
    const double px = (double)X(i, 0) - comx[0], py = (double)X(i, 1) - comx[1], pz = (double)X(i, 2) - comx[2];
    const double vx = (double)V(i, 0) - comv[0], vy = (double)V(i, 1) - comv[1], vz = (double)V(i, 2) - comv[2];
    ang[0] = ang[0] + mass_part * py * vz - mass_part * pz * vy;
    ang[1] = ang[1] + mass_part * pz * vx - mass_part * px * vz;
    ang[2] = ang[2] + mass_part * px * vy - mass_part * py * vx;
  }
  for (int a = 0; a < 3; a++) ang[a] = ang[a] * unit_d * p5(unit_l) / unit_t;
  for (int a = 0; a < 3; a++) {
    o->lambda[3 * h + a] = (float)(ang[a] * sqrt(fabs(Etot)) / (G * pow(M_vir, 2.5)));
    o->lambda_prime[3 * h + a] = (float)(ang[a] / (sqrt2f() * M_vir * R_vir * V_vir));
  }
  /* inertia tensor (:692-705) */
  double I[3][3];
  memset(I, 0, sizeof(I));
  for (int64_t i = 0; i < np; i++) {
    const double q[3] = {(double)X(i, 0) - comx[0], (double)X(i, 1) - comx[1], (double)X(i, 2) - comx[2]};
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) I[a][b] = I[a][b] + q[a] * q[b];
  }
  double A[3][3], d[3], v[3][3];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) A[a][b] = I[a][b] / (double)(float)np;
  jacobi3(A, d, v);
  eigsort3(d, v);
  for (int a = 0; a < 3; a++) {
    o->eig_val[3 * h + a] = (float)(sqrt(d[a]) * unit_l / MPC / (R_vir / MPC));
    o->eig_vec[3 * h + a] = (float)v[a][2];
  }
  o->cos_alpha[h] = ((v[0][2] * ang[0] + v[1][2] * ang[1] + v[2][2] * ang[2]) /
                            sqrt((v[0][2] * v[0][2] + v[1][2] * v[1][2] + v[2][2] * v[2][2]) *
                                 (ang[0] * ang[0] + ang[1] * ang[1] + ang[2] * ang[2])));
#undef X
#undef V
}

int psod_oracle_halo_properties(const psod_oracle_props_params *p, int64_t nhalo, const int64_t *offset,
                                const int64_t *member, const float *pos, const float *vel,
                                const psod_oracle_props_out *out) {
  if (!p || nhalo < 0 || !offset || !member || !pos || !out) return 5;
  for (int64_t h = 0; h < nhalo; h++) {
    const int64_t b = offset[h], e = offset[h + 1], np = e - b;
    if (np < 1) return 5;
    float *x = (float *)malloc(sizeof(float) * 3 * (size_t)np);
    float *v = (float *)malloc(sizeof(float) * 3 * (size_t)np);
    for (int64_t k = 0; k < np; k++)
      for (int a = 0; a < 3; a++) {
        x[3 * k + a] = pos[3 * member[b + k] + a];
        v[3 * k + a] = vel ? vel[3 * member[b + k] + a] : 0.0f;
      }
    one_halo(p, np, x, v, h, out);
    free(x);
    free(v);
  }
  return 0;
}
