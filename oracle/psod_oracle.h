/*
 * psod_oracle.h -- CPU oracle for the SOD stage of Psod.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this
 * code; only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg use it, and only as the checker.
 *
 * It restates, single-threaded and in plain C, the 1-rank path of
 * sod/sod_profile_rdfof_parallel_hdf5.f90:
 *   cic        main:1077-1265   (FP64 CIC deposit on the 2nx periodic grid)
 *   cicm1      main:1268-1390   (FP64 CIC interpolation back to particles)
 *   tri_cic    main:998-1037    (1/rho seed order + npart_new)
 *   quick_sort main:2477-2571   (Brainerd/Miller quicksort, its tie order)
 *   spherover  main:1396-2201   (linked list, preselect, centre refinement,
 *                                distance sort, Delta crossing, profile,
 *                                keep/claim)
 * with the driver glue of main:183-757 for one MPI rank and one zone.
 *
 * Parity status: UNPINNED.  The reference ships no golden vectors or tests
 * for this path and cannot be compiled here (Fortran + MPI + HDF5 are
 * absent); the oracle is checked against analytic known-answer cases.
 *
 * Two arithmetic modes:
 *   PSOD_ORACLE_REFERENCE  the reference's own arithmetic: FP64 CIC summed
 *                          in file order, quicksort tie orders everywhere,
 *                          FP64 refinement sums in x_sel2 order.
 *   PSOD_ORACLE_CANONICAL  the order-independent arithmetic the GPU uses:
 *                          int64 fixed-point CIC nodes, int64 fixed-point
 *                          refinement sums, ties broken by original index.
 * Both share every other step.  They agree except on near-ties (relative
 * gaps of ~1e-12 in rho or in the refinement sum) and exact key ties.
 */
#ifndef PSOD_ORACLE_H
#define PSOD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  PSOD_ORACLE_REFERENCE = 0,
  PSOD_ORACLE_CANONICAL = 1
};

/* status codes (same values as include/psod.h) */
enum {
  PSOD_ORACLE_OK = 0,
  PSOD_ORACLE_ERR_NSEL = 1,      /* main:1681-1693 */
  PSOD_ORACLE_ERR_SELRADIUS = 2, /* main:2072-2089 */
  PSOD_ORACLE_ERR_ARG = 5
};

#define PSOD_ORACLE_MAX_EXTRA_DELTA 4

typedef struct psod_oracle_params {
  int32_t nx;        /* -nx : grid cells per side (CIC uses 2*nx) */
  int32_t nmin;      /* -min: Mmin */
  double delta;      /* -del: seuil */
  double delta2;     /* -dl2: seuil2 (mass2 capture) */
  int32_t ncut;      /* -sel: preselect half-width in cells */
  int64_t nsel;      /* -nse: max preselected particles */
  int32_t nxbuffer;  /* -nxb: buffer cells (0 -> nx/2, main:380-381) */
  int32_t nbins;     /* profile bins (reference: 60, main:1414) */
  double rbin_lo;    /* profile inner edge factor (reference: 0.01) */
  double rbin_hi;    /* profile outer edge factor (reference: 1.0) */
  int32_t ndelta_extra;                          /* extra thresholds */
  double delta_extra[PSOD_ORACLE_MAX_EXTRA_DELTA];
  int64_t npart_total; /* nparttotal (mpf = 1/npart_total) */
  int32_t nxcpu;     /* zones per axis (nxcpu^3 zones, main:340-342); 0 or 1: one zone */
  int32_t nzone;     /* the zone analysed, z fastest (main:344-346) */
} psod_oracle_params;

typedef struct psod_oracle_result {
  int32_t status;
  int64_t fail_rank;      /* 0-based seed rank (ipart-1) that failed, or -1 */
  int64_t npart_new;      /* tri_cic count (includes the first rho<=100) */
  int64_t nprocessed;     /* seeds that passed Mtotsel >= Mmin */
  int64_t cross_touch;    /* records stored in the preselect-cube cells that
                             meet each crossing seed's ball out to its
                             stopping particle, summed (the algorithmic reads
                             of the crossing search) */
  int64_t nhalo;
  int64_t nmember;
  int64_t *halo_id;       /* iamas */
  int64_t *halo_mass;     /* masse = N_Delta */
  int64_t *halo_rank;     /* seed rank of the halo */
  int64_t *halo_cidx;     /* input index of the refined centre particle */
  float *halo_center;     /* 3*nhalo, xc/scale in box units, float */
  double *halo_rdelta;    /* R_Delta in grid units */
  int64_t *halo_mass2;    /* masse2 for seuil2 (0 if never above) */
  int64_t *halo_mextra;   /* ndelta_extra*nhalo, -1 if not crossed */
  int64_t *halo_profile;  /* nbins*nhalo cumulative counts */
  int64_t *member_offset; /* nhalo+1 */
  int64_t *member_index;  /* nmember input indices, ascending distance */
} psod_oracle_result;

/* Reference quick_sort (main:2477-2571) on 0-based arrays: sorts list in
 * place and writes the permutation (0-based original positions) to order. */
void psod_oracle_quick_sort(double *list, int64_t *order, int64_t n);

/* CIC grid on the (2nx)^3 periodic nodes (main:1077-1265), x fastest.
 * grid must hold (2nx)^3 doubles.  mode selects FP64 file-order sums or
 * int64 fixed point. */
int psod_oracle_cic(const psod_oracle_params *p, int64_t n, const float *pos,
                    int mode, double *grid);

/* Per-particle density (main:1268-1390) from a grid made by
 * psod_oracle_cic with the same mode. */
int psod_oracle_cicm1(const psod_oracle_params *p, int64_t n,
                      const float *pos, const double *grid, double *rho);

/* Seed order (main:998-1037): isort[n] (0-based) and npart_new. */
int psod_oracle_tri_cic(int64_t n, const double *rho, int mode,
                        int64_t *isort, int64_t *npart_new);

/* Full 1-rank SOD stage: cic, cicm1, tri_cic, spherover.  Fills res;
 * free it with psod_oracle_free.  Returns res->status. */
int psod_oracle_run(const psod_oracle_params *p, int64_t n, const float *pos,
                    const int64_t *ids, int mode, psod_oracle_result *res);

/* spherover alone, given the seed order (isort, npart_new). */
int psod_oracle_spherover(const psod_oracle_params *p, int64_t n,
                          const float *pos, const int64_t *ids,
                          const int64_t *isort, int64_t npart_new, int mode,
                          psod_oracle_result *res);

/* Arithmetic audit of one spherover run: how often the reference's FP64
 * arithmetic and the canonical fixed-point arithmetic would decide a step
 * differently on the same inputs. */
typedef struct psod_oracle_audit {
  int64_t refine_seeds;     /* seeds that ran the centre refinement */
  int64_t refine_flips;     /* seeds whose FP64-sum argmax (main:1851-1875)
                               and fixed-point-sum argmax differ */
  int64_t refine_near;      /* seeds whose two largest fixed-point sums are
                               within 1e-9 relative */
  int64_t dist_tie_cut;     /* crossings whose N_Delta-th and next sorted
                               distances are exactly equal */
  int64_t dist_tie_cut_nmax; /* the largest N_Delta among those: below 10
                               whenever the loop's monotonicity holds */
  int64_t dist_tie_members; /* crossings with an exact distance tie among
                               the members */
} psod_oracle_audit;

/* spherover (as psod_oracle_spherover, same outputs for the given mode)
 * with both arithmetics of the centre refinement evaluated side by side and
 * the audit counters filled. */
int psod_oracle_audit_spherover(const psod_oracle_params *p, int64_t n,
                                const float *pos, const int64_t *ids,
                                const int64_t *isort, int64_t npart_new,
                                int mode, psod_oracle_result *res,
                                psod_oracle_audit *au);

void psod_oracle_free(psod_oracle_result *res);

/* Fixed-point scale of the canonical CIC and refinement sums. */
#define PSOD_FIX_SHIFT 40

#ifdef __cplusplus
}
#endif
#endif
