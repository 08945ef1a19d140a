/*
 * psod_oracle_fof.h -- CPU oracle for pFoF's friends-of-friends halo finder
 * on one MPI rank (Pfof/trunk/pfof_snap/src/modfofpara.f90 fofpara, the
 * periodic merge of Pfof/trunk/common/src/modfofmpi.f90, and the halo
 * observables of sod/modhalo.f90).
 *
 * TEST INFRASTRUCTURE ONLY: tests/ and bench.py's cpu_baseline leg use it
 * as the checker; nothing in the product links it.
 */
#ifndef PSOD_ORACLE_FOF_H
#define PSOD_ORACLE_FOF_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { PSOD_ORACLE_FOF_OK = 0, PSOD_ORACLE_FOF_ERR_ARG = 5 };

typedef struct psod_oracle_fof_params {
  float percolation; /* param%percolation_length: linking length in mean spacings */
  int64_t nres;      /* particles per side of the simulation (nres) */
  int64_t mmin;      /* param%Mmin: smallest halo kept */
} psod_oracle_fof_params;

typedef struct psod_oracle_fof_result {
  int32_t status;
  int64_t ngroups_local; /* groups of the local scan, singletons included */
  int64_t nbridges;      /* pairs linked across the periodic boundary */
  int64_t nhalo, nmember;
  int64_t *halo_id;       /* [nhalo] label (a particle ID), ascending */
  int64_t *halo_mass;     /* [nhalo] particle count */
  double *halo_com;       /* [3*nhalo] centre of mass, box units in [0,1] */
  double *halo_vel;       /* [3*nhalo] mean velocity */
  double *halo_radius;    /* [nhalo] largest member distance from the centre */
  int64_t *member_offset; /* [nhalo+1] */
  int64_t *member_index;  /* [nmember] input indices, heap order inside a halo */
  int64_t *structure;     /* [n] final label of every particle */
} psod_oracle_fof_result;

/* pos: 3n floats in [0,1]; vel: 3n floats or NULL (zeros); id: n IDs */
int psod_oracle_fof(const psod_oracle_fof_params *p, int64_t n, const float *pos, const float *vel,
                    const int64_t *id, psod_oracle_fof_result *res);
void psod_oracle_fof_free(psod_oracle_fof_result *res);

#ifdef __cplusplus
}
#endif
#endif
