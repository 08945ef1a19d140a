/*
 * psod_oracle_props.h -- CPU oracle for haloanalyzer's halo_properties
 * (haloanalyzer_new/src/modfunctions.f90:47-808, with diag :840-933 and
 * eigsrt :812-837), for halos at a fixed redshift (no lightcone) and without
 * the volume estimate (compute_volume is false there).
 *
 * TEST INFRASTRUCTURE ONLY: tests/ and bench.py's cpu_baseline leg use it
 * as the checker; nothing in the product links it.
 */
#ifndef PSOD_ORACLE_PROPS_H
#define PSOD_ORACLE_PROPS_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSOD_ORACLE_PROPS_NBIN1 100 /* modvariables.f90:301 */
#define PSOD_ORACLE_PROPS_NBIN2 30

typedef struct psod_oracle_props_params {
  double unit_l, unit_d, unit_t; /* simu_info units (cgs) */
  double aexp, h0;               /* expansion factor; H0 in km/s/Mpc */
  double hz;                     /* a^2 H(a)/H0, as interpolated from the cosmology table */
  double delta_vir;              /* simu_info%delta_vir (Delta_matter) */
  int32_t levelmin;              /* simu_info%levelmin */
  int32_t center_on_mass;        /* do_center_mass */
  int32_t periodic;              /* do_periodic_boundary */
  int32_t epot_threshold;        /* 30000: above it the potential uses threshold/10 members */
} psod_oracle_props_params;

/* every array is per halo, float32 as haloanalyzer stores it, except npart
   and the four virial values (stored as real(8) there) */
typedef struct psod_oracle_props_out {
  int64_t *npart;
  double *mvir, *rvir, *rvircom, *vvir;
  float *com, *comv;                  /* [3] */
  float *rmax, *vmax, *dispx, *dispv;
  float *ekin, *epot;
  float *lambda, *lambda_prime;       /* [3] */
  float *eig_val, *eig_vec;           /* [3] */
  double *cos_alpha;                  /* stored without the real(4) conversion */
  float *center_pot;                  /* [3] */
  float *circ;                        /* [4] */
  float *delta_vals;                  /* [2] */
  float *dens, *dens_int, *vcirc;     /* [NBIN1] */
  float *dens178, *dens_int178;       /* [NBIN2] */
} psod_oracle_props_out;

/* Halo h is members member[offset[h] .. offset[h+1]) (input indices into
   pos/vel, 3 floats each; vel may be NULL for zeros), in the order the
   halo file lists them.  out's arrays are the caller's. */
int psod_oracle_halo_properties(const psod_oracle_props_params *p, int64_t nhalo, const int64_t *offset,
                                const int64_t *member, const float *pos, const float *vel,
                                const psod_oracle_props_out *out);

#ifdef __cplusplus
}
#endif
#endif
