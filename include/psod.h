/*
 * psod.h -- C-ABI of the B200 SOD engine (libpsod.so).
 *
 * Drop-in for the hot path of the reference's SOD stage,
 * sod/sod_profile_rdfof_parallel_hdf5.f90 ("main").  The reference calls
 * four external Fortran subroutines with implicit interfaces, passing the
 * particle arrays through module globals (modvar posf/idf/mpf, modcic
 * cube/rho, main:1-24):
 *
 *   call cic(...)        main:673-674   ->  psod_cic
 *   call cicm1(...)      main:679       ->  psod_cicm1
 *   call tri_cic(...)    main:713       ->  psod_tri_cic
 *   call spherover(...)  main:740-744   ->  psod_spherover (+ psod_get_halos)
 *
 * Here the module globals become a context that owns device copies of the
 * particles (psod_load_particles).  Conventions:
 *   - plain pointers and sizes; no torch or CUDA types in any signature;
 *   - array pointers may be host (pageable or pinned) or device memory; the
 *     library detects which and copies as needed;
 *   - indices are 0-based (the reference's are 1-based);
 *   - every entry point returns a psod_status; psod_last_error() gives the
 *     message of the last failure on that context;
 *   - one context per thread; contexts are independent.
 * The library has no CPU fallback: without a usable CUDA device every
 * compute entry point returns PSOD_ERR_CUDA.
 */
#ifndef PSOD_H
#define PSOD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSOD_ABI_VERSION 4
#define PSOD_MAX_EXTRA_DELTA 4

typedef enum psod_status {
  PSOD_OK = 0,
  PSOD_ERR_NSEL = 1,      /* preselection exceeded nsel (main:1681-1693):
                             the whole zone's output is lost */
  PSOD_ERR_SELRADIUS = 2, /* overdensity still above delta at the selection
                             edge (main:2072-2089): zone output lost */
  PSOD_ERR_TIMEOUT = 3,   /* a bounded device wait ran out */
  PSOD_ERR_CUDA = 4,      /* CUDA runtime error or no device */
  PSOD_ERR_ARG = 5,       /* invalid argument or parameter */
  PSOD_ERR_STATE = 6,     /* entry point called out of order */
  PSOD_ERR_NOMEM = 7,     /* device allocation failed */
  PSOD_ERR_IO = 8         /* an output file could not be written */
} psod_status;

typedef enum psod_mode {
  PSOD_MODE_PLAIN = 0,   /* one launch per round, full-cube gather */
  PSOD_MODE_BATCHED = 1, /* per-cell alive counts, growing-ball crossing
                            (warp per small ball, CTA per large one) */
  PSOD_MODE_LEARNED = 2  /* batched + learned first ball of the crossing
                            search (psod_learn_*); batched without a model */
} psod_mode;

#define PSOD_LEARN_FEATURES 10     /* network inputs per seed */
#define PSOD_LEARN_PARAMS 5768     /* weights and biases (padded layout) */
#define PSOD_LEARN_MODEL_FLOATS 5804 /* 36 scales + PSOD_LEARN_PARAMS */

/* Parameters: the reference's CLI flags (read_params, main:767-906) and the
 * hard-coded constants of spherover.  psod_params_default() fills the
 * reference defaults (main:110-114, 1414, 1459, 1525-1530, 1558-1559). */
typedef struct psod_params {
  int32_t nx;          /* -nx : grid cells per side; CIC uses 2*nx */
  int32_t nmin;        /* -min: minimum halo particle count Mmin (100) */
  double delta;        /* -del: overdensity threshold seuil (200) */
  double delta2;       /* -dl2: second threshold seuil2 (800) */
  int32_t ncut;        /* -sel: preselect half-width in cells (4) */
  int64_t nsel;        /* -nse: preselected-particle capacity (4000000) */
  int32_t nxbuffer;    /* -nxb: buffer cells; 0 means nx/2 (main:380-381) */
  int64_t npu;         /* -npu: halo-size upper bound; >0 derives ncut,
                          nxbuffer and nsel as main:211-219 does */
  int32_t nbins;       /* profile bins (60, main:1414) */
  double rbin_lo;      /* inner profile edge as a fraction of R_delta (0.01) */
  double rbin_hi;      /* outer profile edge as a fraction of R_delta (1.0) */
  int32_t ndelta_extra;                     /* extra thresholds, <= 4 */
  double delta_extra[PSOD_MAX_EXTRA_DELTA]; /* N and R for each, same rule */
  int32_t mode;        /* psod_mode */
  int32_t device;      /* CUDA device ordinal */
  /* Zone decomposition (main:321-441): the box is cut into nxcpu^3 zones
   * and this context analyses zone nzone (0-based, z fastest: nzone =
   * iz + nxcpu*(iy + nxcpu*ix), main:344-346) with its buffer of nxbuffer
   * cells (0 means nxzone/2, nxzone = nx/nxcpu).  The caller loads the
   * zone's particles with their buffer (main:573-600, or
   * psod_read_cube_zone); halos are kept only when their centre lies in
   * the zone (main:2118-2120).  nxcpu = 1 (default) is the one-rank box.
   * nx must be a multiple of nxcpu, and for nxcpu > 1 the zone with its
   * buffer must either span at least the box (nxzone + 2*nxbuffer >= nx)
   * or leave max(ncut, 2) cells outside it: between the two the
   * reference's linked-list walk would wrap into the far side of its local
   * grid, which is refused.  0 (left unset) reads as 1. */
  int32_t nxcpu;
  int32_t nzone;
} psod_params;

/* Halo table.  The caller provides the arrays it wants (NULL = skip), sized
 * from psod_halo_count(); host or device memory.  Halos are in the
 * reference's order (seed processing order); members of halo h are
 * member_*[member_offset[h] .. member_offset[h+1]) in ascending distance
 * from the centre, as the reference writes them (main:2306-2315). */
typedef struct psod_halo_table {
  int64_t *halo_id;       /* [nhalo]  ID of the centre particle (iamas) */
  int64_t *halo_mass;     /* [nhalo]  N_delta (particle count) */
  int64_t *halo_rank;     /* [nhalo]  seed rank in density order */
  float *halo_center;     /* [3*nhalo] centre, box units (xc/scale) */
  double *halo_rdelta;    /* [nhalo]  R_delta in grid cells */
  int64_t *halo_mass2;    /* [nhalo]  last step above delta2, 0 if none */
  int64_t *halo_mextra;   /* [nhalo*ndelta_extra] N for extra thresholds,
                             -1 when not crossed inside the selection */
  int64_t *halo_profile;  /* [nhalo*nbins] cumulative counts below each
                             log-spaced edge */
  int64_t *member_offset; /* [nhalo+1] */
  int64_t *member_index;  /* [nmember] 0-based input particle index */
  int64_t *member_id;     /* [nmember] particle IDs */
} psod_halo_table;

/* Counters of the last psod_spherover call. */
typedef struct psod_run_stats {
  int64_t npart_new;     /* seeds examined (tri_cic's npart_new) */
  int64_t nprocessed;    /* seeds that passed Mtotsel >= Mmin */
  int64_t nhalo;         /* kept halos */
  int64_t nmember;       /* members of kept halos */
  int64_t rounds;        /* scheduler rounds */
  int64_t fail_rank;     /* failing seed rank, -1 if none */
  int64_t touched;       /* particle records read by the SOD kernels */
  double ms_total;       /* device time of psod_spherover */
  double ms_sod_kernel;  /* device time of the per-seed phase kernels */
  int64_t sod_launches;  /* per-seed kernel launches */
  int64_t kernel_launches; /* all kernels launched by psod_spherover */
  double ms_sched;       /* scheduler kernels */
  double ms_prep;        /* preselect count + candidate lists */
  double ms_refine;      /* approximate centre-refinement sums */
  double ms_select;      /* exact contender sums + argmax */
  double ms_cross;       /* crossing, profile, claims */
  int64_t ncandidates;   /* refinement candidates */
  int64_t refine_pairs;  /* candidate-neighbour pairs tested */
  int64_t cross_touch;   /* records of the cube cells meeting each ball out to
                            its stopping particle (algorithmic reads) */
  int64_t refine_slots;  /* lane slots spent on refinement pair tests */
  double ms_setup;       /* seed bucketing before the first round */
  double ms_output;      /* halo table ordering and member sort */
  double ms_learn;       /* bracket features and network inference */
  int64_t bracket_hits;  /* seeds whose first crossing ball held every stop */
  int64_t bracket_seeds; /* seeds that ran the crossing search (batched modes) */
  int64_t cross_balls;   /* ball passes of the crossing search */
  int64_t cross_records; /* alive records inside those balls, summed */
  double ms_refine_bound; /* refinement bound pass (part of ms_refine) */
  int64_t refine_items;   /* refinement work items summed (64 candidates x one record chunk) */
  int64_t refine_pruned;  /* refinement candidates not summed: their bound is below the best lower bound */
  double ms_tail;         /* device tail loop (late rounds run by one cooperative launch) */
  int64_t tail_rounds;    /* rounds run by the device tail loop (part of rounds) */
  int64_t tail_touch;     /* part of cross_touch from the tail loop's crossings */
  int64_t cross_members;  /* members of kept halos written by the crossing kernels (k_cross, k_cross_warp) */
  int64_t tail_members;   /* members of kept halos written by the tail loop */
} psod_run_stats;

typedef struct psod_ctx psod_ctx;

void psod_params_default(psod_params *p);

/* Create a context on p->device.  Validates the parameters the way the
 * reference driver does (main:386-397): nxbuffer >= ncut; and nxbuffer < nx
 * (the reference also allows nxbuffer == nx, where its CIC array is padded
 * past the periodic grid; that case is refused here). */
int psod_ctx_create(const psod_params *p, psod_ctx **out);
int psod_ctx_destroy(psod_ctx *ctx);

/* Optional: run on the caller's stream (a cudaStream_t passed as void*).
 * Default: a stream owned by the context. */
int psod_set_stream(psod_ctx *ctx, void *stream);

/* Load n particles: pos is xyz-interleaved float32 in box units [0,1]
 * (posf(3,n), modvar main:9), id int64 (idf, main:8), vel optional
 * (velf; copied for the member table only).  npart_total is the
 * simulation's particle count (nparttotal, main:302-310); mpf = 1/that.
 * Builds the cell-sorted cube (the linked list of main:1564-1604).
 * Device arrays are read on the context's stream: data written on another
 * stream must be complete first (synchronise, or run the context on the
 * producer's stream with psod_set_stream). */
int psod_load_particles(psod_ctx *ctx, int64_t n, const float *pos,
                        const float *vel, const int64_t *id,
                        int64_t npart_total);

/* cic (main:1077-1265): CIC density on the (2nx)^3 periodic grid,
 * accumulated in int64 fixed point (2^-40 per unit weight) so the grid is
 * the same on every run.  grid_out (optional, (2nx)^3 doubles, x fastest)
 * receives the grid in units of the mean density. */
int psod_cic(psod_ctx *ctx, double *grid_out);

/* cicm1 (main:1268-1390): per-particle density.  rho_out (optional, n
 * doubles) in input order. */
int psod_cicm1(psod_ctx *ctx, double *rho_out);

/* tri_cic (main:998-1037): seeds in ascending 1/rho, ties by input index.
 * isort_out (optional, npart_new entries, 0-based input indices);
 * *npart_new_out gets the reference's npart_new. */
int psod_tri_cic(psod_ctx *ctx, int64_t *isort_out, int64_t *npart_new_out);

/* spherover compute (main:1396-2201).  Returns PSOD_ERR_NSEL or
 * PSOD_ERR_SELRADIUS with the reference's zone-abort meaning (no halos).
 * stats optional. */
int psod_spherover(psod_ctx *ctx, psod_run_stats *stats);

int psod_halo_count(psod_ctx *ctx, int64_t *nhalo, int64_t *nmember);
int psod_get_halos(psod_ctx *ctx, const psod_halo_table *t);

/* Convenience: cic, cicm1, tri_cic and spherover in one call. */
int psod_run(psod_ctx *ctx, psod_run_stats *stats);

/* The reference's binary halo files, written by spherover when it is built
 * without HDF5 (main:2230-2259): Fortran unformatted sequential records
 * (int32 byte length, payload, int32 byte length), from a halo table that
 * psod_get_halos filled into HOST memory.  Host-only: no context, no device.
 *   psod_write_masst ("sod_<snap>_masst_<zone>", main:2234-2239): record
 *     namas (int32); per halo one record: ID (int64), N_delta (int32),
 *     centre x, y, z (float32, box units).  Reads halo_id, halo_mass,
 *     halo_center.
 *   psod_write_strct ("sod_<snap>_strct_<zone>", main:2246-2256): record
 *     namas (int32); per halo the records N_delta (int32), member positions
 *     (3 float32 each, box units), velocities (3 float32 each; zeros when
 *     vel is NULL), IDs (int64), then potential (float32) and force (3
 *     float32) when pot / force are given, members in ascending distance.
 *     Reads halo_mass, member_offset, member_index; pos/vel/id/pot/force
 *     are the zone's particle arrays (n entries, input order, as loaded).
 * Returns PSOD_ERR_ARG for missing arrays, inconsistent offsets, member
 * indices outside [0, n) or records of 2^31 bytes or more, PSOD_ERR_IO
 * when the file cannot be written. */
int psod_write_masst(const char *path, const psod_halo_table *t, int64_t nhalo);
int psod_write_strct(const char *path, const psod_halo_table *t, int64_t nhalo, int64_t n, const float *pos,
                     const float *vel, const int64_t *id, const float *pot, const float *force);

/* The reference's binary particle reader (main:455-534), host-only: the
 * zone's particles from the FoF step's cube files "<root>_cube_NNNNN", each
 * Fortran unformatted sequential records of nloc (int32), the writer's rank
 * (int32), the cube bounds (6 float32), positions (3*nloc float32, box
 * units), velocities (3*nloc float32) and IDs (nloc int64; int32 when
 * id_bytes = 4, a build without LONGINT).  ncpu = nxcpu^3 cubes; zone nzone
 * (0-based, x-major) reads the 27 cubes around it in the reference's order
 * (x outer, z inner, periodic) and keeps, in file order, the particles
 * within the zone plus nxbuffer cells (0 means half the zone, main:380-381)
 * by the reference's FP64 distance test (main:471-479).  With fewer than 3
 * cubes a side the reference lists some cubes twice and loads their
 * particles twice; each distinct cube is read once here.  Call with
 * pos == NULL to get *npart, then with arrays of at least *npart entries
 * (capacity); vel may be NULL.  Returns PSOD_ERR_IO for a missing or
 * malformed file, PSOD_ERR_ARG for bad arguments or a short capacity. */
int psod_read_cube_zone(const char *root, int32_t ncpu, int32_t nzone, int32_t nx, int32_t nxbuffer, int32_t id_bytes,
                        int64_t capacity, int64_t *npart, float *pos, float *vel, int64_t *id);

/* The driver's selection of one zone's particles with their buffer
 * (main:573-600, the FP64 test of main:578-584): keep[i] = 1 when particle
 * i (pos: xyz-interleaved float32, box units) lies in zone nzone of
 * nxcpu^3 (the numbering of psod_params) or within nxbuffer cells of it
 * (0 means nxzone/2), periodically; *nkeep gets their count.  Host code,
 * no device.  The selected particles, in input order, are what a zone
 * context (psod_params.nxcpu > 1) is loaded with. */
int psod_select_zone(int32_t nx, int32_t nxcpu, int32_t nzone, int32_t nxbuffer, const float *pos, int64_t n,
                     uint8_t *keep, int64_t *nkeep);

/* CIC density (cic + cicm1, the same fixed-point arithmetic) for a zone of
 * at most 64 cells per side, without any device allocation.  This entry
 * point has no counterpart in the reference.  It is for host codes that
 * cannot let a library allocate device memory: drivers that size all of the
 * GPU's memory themselves (several MPI ranks sharing one GPU under fixed
 * per-rank budgets, or a host whose own pool allocator owns the device) and
 * forbid libraries from calling cudaMalloc.  The node grid is a file-scope
 * device array of (2*64)^3 int64 (16 MiB) that every device loading the
 * library holds until exit.
 *   pos      device, xyz-interleaved float32 box units [0,1], n particles
 *   rho      device, n doubles, input order (as psod_cicm1)
 *   bad_flag device int or NULL: set to 1 when a position lies outside
 *            [0,1] (that particle is skipped and gets rho = 0), else 0
 *   stream   cudaStream_t as void* (NULL: legacy default stream)
 * Work is enqueued on the stream and not waited for.  Returns PSOD_ERR_ARG
 * for nx > 64, nxbuffer >= nx or host pointers.  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress, with that
 * device current); make that first call before any stream capture.  Every
 * call clears the array before depositing.  All calls share the array, so
 * calls that overlap on the GPU race and give wrong densities: serialise
 * them. */
int psod_cic_rho_static(int64_t n, const float *pos, int32_t nx, int64_t npart_total, int32_t nxbuffer,
                        double *rho, int *bad_flag, void *stream);

/* ---- Learned radius bracket (no counterpart in the reference) ----------
 * The crossing search of psod_spherover grows a ball around each centre
 * until the Delta stop lies inside it (1.5 cells, doubling, in the batched
 * mode).  In PSOD_MODE_LEARNED a small network predicts the first ball from
 * ten seed-local features; a miss falls back to the growing search, so the
 * halo table is identical with or without a model.  The network (10 -> 64 ->
 * 64 -> 2, ReLU, bf16 tensor-core GEMMs with FP32 accumulation, Adam) is
 * trained on the GPU on samples the engine itself produces:
 *   psod_learn_collect(ctx, cap)   record (features, targets) of every seed
 *                                  that crosses in later psod_spherover
 *                                  calls (batched or learned mode); cap 0
 *                                  stops recording.  Restarts the count.
 *   psod_learn_samples             count and copies of the samples (x: 10
 *                                  floats, t: log stop radius in cells and
 *                                  log N_delta per sample; NULL skips)
 *   psod_learn_train               scales from the samples, then Adam
 *   psod_learn_get/set_model       the model as PSOD_LEARN_MODEL_FLOATS floats:
 *                                  mu_x[16], sigma_x[16], mu_y[2], sigma_y[2],
 *                                  W1[64][16], b1[64], W2[64][64], b2[64],
 *                                  W3[8][64], b3[8] (rows/columns beyond the
 *                                  real sizes are zero)
 *   psod_learn_forward             outputs (original units) for raw features
 *   psod_learn_gradient            gradient of 0.5*mean|y_std - t_std|^2 over
 *                                  all PSOD_LEARN_PARAMS parameters
 *   psod_learn_set_margin          first ball = exp(y0) * margin (default 1.1) */
typedef struct psod_train_params {
  int32_t epochs;  /* passes over the samples (20) */
  int32_t batch;   /* samples per step, a multiple of 64 (4096) */
  float lr;        /* Adam step (1e-3) */
  float beta1;     /* 0: 0.9 */
  float beta2;     /* 0: 0.999 */
  float eps;       /* 0: 1e-8 */
  uint64_t seed;   /* weight initialisation and batch order */
} psod_train_params;

/* Feature sets of the learned bracket (both: PSOD_LEARN_FEATURES inputs):
 *   PSOD_LEARN_FEATURES_SEED (default): seed-local quantities (log rho of
 *     the seed and the centre, log alive records in cubes of half-width
 *     0..4 cells, log refinement sum, centre offset, log candidates);
 *     targets log stop radius (cells) and log N_delta; first ball
 *     exp(y0) * margin.
 *   PSOD_LEARN_FEATURES_FOF: from the FoF group of the seed particle, as
 *     the learned-seed configuration of the task names them: log N_FoF, the
 *     three inertia axis ratios (b/a, c/a, c/b), log rho(seed) (the CIC peak
 *     overdensity), seed - FoF centre of mass (3, cells), R_FoF and the RMS
 *     radius (cells); targets log(R_stop / R_FoF) and the centre offset
 *     |centre - seed| (cells); first ball exp(y0) * margin * R_FoF.  Needs
 *     psod_fof on the loaded particles before psod_spherover (else
 *     PSOD_ERR_STATE); seeds outside the FoF halos get no prediction.
 * A model is tied to the set it was trained with; the halo table never
 * depends on either. */
#define PSOD_LEARN_FEATURES_SEED 0
#define PSOD_LEARN_FEATURES_FOF 1
int psod_learn_set_features(psod_ctx *ctx, int32_t set);

int psod_learn_collect(psod_ctx *ctx, int64_t capacity);
int psod_learn_samples(psod_ctx *ctx, int64_t *n, float *x_out, float *t_out);
int psod_learn_train(psod_ctx *ctx, const psod_train_params *tp, float *loss_per_epoch);
int psod_learn_get_model(psod_ctx *ctx, float *model, int64_t nfloats);
int psod_learn_set_model(psod_ctx *ctx, const float *model, int64_t nfloats);
int psod_learn_set_margin(psod_ctx *ctx, float margin);
int psod_learn_forward(psod_ctx *ctx, int64_t n, const float *x, float *y);
int psod_learn_gradient(psod_ctx *ctx, int64_t n, const float *x, const float *t, float *grad, float *loss);

/* ---- Scheduling thresholds and their autotuner ---------------------------
 * psod_spherover's size classes and round handling depend on four
 * thresholds.  None of them changes the halo table (each only chooses which
 * kernel or pass does a piece of work); they change its speed.  Defaults
 * are the values measured best on the 1024^3 workload: 2048, 4096, 256,
 * 1024.  No counterpart in the reference. */
typedef struct psod_tuning {
  int32_t warp_cross_min_ready; /* rounds with at least this many ready seeds cross small balls a warp per seed */
  int32_t bound_min_cand;       /* seeds with at least this many candidates get the refinement bound pass */
  int32_t tail_max_ready;       /* the device tail loop takes rounds of at most this many ready seeds (0: never) */
  int32_t tail_max_cand;        /* ... whose seeds have at most this many candidates (<= bound_min_cand) */
} psod_tuning;

int psod_get_tuning(psod_ctx *ctx, psod_tuning *t);
/* PSOD_ERR_ARG unless warp_cross_min_ready >= 1, 256 <= bound_min_cand,
 * tail_max_ready >= 0 and 1 <= tail_max_cand <= bound_min_cand. */
int psod_set_tuning(psod_ctx *ctx, const psod_tuning *t);
/* Picks the thresholds by timing psod_spherover on the loaded particles
 * (after psod_tri_cic): starting from the current values, one threshold at a
 * time over a few candidates each (coordinate descent, a change kept when it
 * is at least 0.5 % faster), about a dozen spherover runs.  Leaves the best
 * thresholds set and the halo table of its last run (the same table as any
 * run).  chosen / ms_best / runs may be NULL. */
int psod_autotune(psod_ctx *ctx, psod_tuning *chosen, double *ms_best, int32_t *runs);

/* ---- Friends-of-friends (pFoF on one rank) -----------------------------
 * The halo finder that writes the catalogue and cube files the SOD stage
 * reads: pFoF's fofpara (Pfof/trunk/pfof_snap/src/modfofpara.f90:31-296)
 * with the periodic merge of Pfof/trunk/common/src/modfofmpi.f90 (:37-649),
 * then selecthaloes, computecom and computeradius (sod/modhalo.f90:253-376,
 * 381-441, 445-488), on the particles of psod_load_particles (the periodic
 * unit box).  psod_fof replaces that sequence for one MPI rank.
 *
 * Two particles are friends when their squared distance, evaluated in FP32
 * as the reference evaluates it, is <= r2 = (percolation / nres)^2 (FP32):
 * |x1 - x2| per axis for pairs within half a box on every axis (the local
 * scan, modfofpara.f90:234-238); min(d, 1 - d) per axis for pairs across the
 * periodic boundary whose particles lie within percolation / nres of
 * opposite faces of one axis (the bridges, modfofmpi.f90:226-233).
 * Positions equal to 1.0 count as 0.0.  A halo is a connected group of at
 * least mmin particles.
 *
 * Labels and order: a halo's ID is the ID of its member with the lowest
 * input index, and halos come in ascending ID; members in ascending input
 * index.  The reference labels a group with the ID of the particle its
 * sequential scan started the group from (the front of its in-place queue),
 * merged across the boundary to the smallest such label, and keeps members
 * in heap order; that label follows from the scan order and has no
 * parallel counterpart.  Member sets, masses, centres and radii are the
 * reference's.
 *
 * Centre of mass: FP64 mean of the member positions, each unwrapped by one
 * box against the halo's first member where they lie more than half a box
 * apart (the reference unwraps against the running mean: the same for
 * halos smaller than a quarter box), wrapped into [0,1].  Mean velocity
 * (zeros when no velocities were loaded).  Radius: the largest member
 * distance from the centre, per axis |d| > 0.5 -> 1 - |d| (computeradius).
 *
 * The linking length percolation * nx / nres must lie between about 0.06
 * and 0.5 SOD cells (PSOD_ERR_ARG otherwise); percolation < 0.5 as the
 * reference requires (modfofpara.f90:101-117). */
typedef struct psod_fof_params {
  float percolation; /* param%percolation_length, in mean inter-particle spacings (0.2) */
  int32_t reserved;  /* 0 */
  int64_t nres;      /* particles per side (nres); 0: cube root of the loaded count, rounded */
  int64_t mmin;      /* param%Mmin: smallest halo kept */
} psod_fof_params;

typedef struct psod_fof_stats {
  int64_t nhalo;      /* groups of at least mmin particles */
  int64_t nmember;    /* their particles */
  int64_t ngroups;    /* all groups, single particles included */
  int64_t fine_cells; /* non-empty linking cells */
  int64_t pair_tests; /* particle pairs tested */
  int64_t cell_pairs; /* neighbour look-ups (linking-cell rows or cells) */
  double ms_total;    /* device time of psod_fof */
  double ms_sort;     /* linking-cell sort */
  double ms_link;     /* union-find over the linking cells */
  double ms_label;    /* groups, labels, member lists */
  double ms_props;    /* centres, velocities, radii */
} psod_fof_stats;

typedef struct psod_fof_table {
  int64_t *halo_id;       /* [nhalo] ID of the lowest-index member, ascending */
  int64_t *halo_mass;     /* [nhalo] particle count */
  double *halo_com;       /* [3*nhalo] centre of mass, box units */
  double *halo_vel;       /* [3*nhalo] mean velocity */
  double *halo_radius;    /* [nhalo] largest member distance from the centre, box units */
  int64_t *member_offset; /* [nhalo+1] */
  int64_t *member_index;  /* [nmember] input indices, ascending inside a halo */
  int64_t *member_id;     /* [nmember] particle IDs */
} psod_fof_table;

int psod_fof(psod_ctx *ctx, const psod_fof_params *p, psod_fof_stats *stats);
/* Frees psod_fof's working arrays (about 26 bytes per particle); the
 * catalogue and the per-particle group codes the learned features read stay.
 * The next psod_fof allocates them again. */
int psod_fof_release(psod_ctx *ctx);
int psod_fof_halo_count(psod_ctx *ctx, int64_t *nhalo, int64_t *nmember);
int psod_fof_get_halos(psod_ctx *ctx, const psod_fof_table *t);

/* ---- Halo properties (haloanalyzer's halo_properties) -------------------
 * haloanalyzer_new/src/modfunctions.f90:47-808 for every halo of the last
 * SOD table (psod_spherover) or FoF catalogue (psod_fof) of the context,
 * members in the table's order, at a fixed redshift (no lightcone) and
 * without the volume estimate (which the reference leaves off): virial mass,
 * radius and velocity from the particle count, centre of mass and mean
 * velocity, R_max, V_max, the position and velocity dispersions, kinetic
 * and potential energy and the most bound member, the density,
 * integrated-density and circular-velocity profiles in 100 log bins of
 * radius (1 kpc, dlnR 0.1) and 30 of R/R178 (0.01, dlnR 0.2) around the
 * potential minimum (or the centre of mass), the circular-velocity maximum,
 * the interpolated R178/M178, the angular momentum's two spin parameters,
 * the inertia tensor's sorted eigenvalues (cyclic Jacobi) and minor axis,
 * and the cosine between that axis and the angular momentum.  Values are
 * the reference's, in its units and precision: real(4) where it stores
 * real(4) (the float arrays below), real(8) for the four virial values and
 * cos_alpha.  The halo's particles are the loaded positions (box units)
 * and velocities (zeros when none were loaded), in the units of the
 * simulation (unit_l / unit_t per velocity unit).
 * One departure: for a halo of at least epot_threshold particles the
 * reference estimates the potential from epot_threshold/10 members drawn
 * with random_number; here the members at positions floor(k*n/m), k = 0 ..
 * m-1 (m = epot_threshold/10), form the sample. */
#define PSOD_PROPS_NBIN1 100
#define PSOD_PROPS_NBIN2 30
#define PSOD_PROPS_FROM_SOD 0
#define PSOD_PROPS_FROM_FOF 1

typedef struct psod_props_params {
  double unit_l, unit_d, unit_t; /* simu_info%unit_l/_d/_t (cgs) */
  double aexp;                   /* simu_info%aexp */
  double h0;                     /* simu_info%h0 (km/s/Mpc) */
  double hz;                     /* a^2 H(a)/H0 as the reference interpolates it (modanalyzeengines.f90:305-313) */
  double delta_vir;              /* simu_info%delta_vir (Delta_matter) */
  int32_t levelmin;              /* simu_info%levelmin: mass_part = 2^-3 levelmin, smoothing 2^-levelmin / 64 */
  int32_t center_on_mass;        /* do_center_mass: profiles around the centre of mass (1) or the most bound member (0) */
  int32_t periodic;              /* do_periodic_boundary */
  int32_t source;                /* PSOD_PROPS_FROM_SOD or PSOD_PROPS_FROM_FOF */
  int32_t epot_threshold;        /* 30000 (modfunctions.f90:336) */
  int32_t reserved;              /* 0 */
} psod_props_params;

typedef struct psod_props_stats {
  int64_t nhalo, nmember;
  int64_t potential_items; /* (halo, 256-member) work items of the potential pass */
  double ms_total;         /* device time of psod_halo_properties */
} psod_props_stats;

/* per halo; [k] marks k values per halo, halo-major */
typedef struct psod_props_table {
  int64_t *npart;
  double *mvir, *rvir, *rvircom, *vvir;    /* Msun/h, kpc/h physical, kpc/h comoving, km/s */
  float *com, *comv;                       /* [3] Mpc/h comoving, km/s */
  float *rmax, *vmax, *dispx, *dispv;      /* over R_vir or V_vir */
  float *ekin, *epot;                      /* over M_vir V_vir^2 / 2 */
  float *lambda, *lambda_prime;            /* [3] */
  float *eig_val, *eig_vec;                /* [3] a, b, c over R_vir; minor axis */
  double *cos_alpha;
  float *center_pot;                       /* [3] Mpc/h comoving */
  float *circ;                             /* [4] M_circ_max, R_circ_max, V_circ_max, Rho_circ_max */
  float *delta_vals;                       /* [2] M178 (Msun/h), R178 (kpc/h physical) */
  float *dens, *dens_int, *vcirc;          /* [PSOD_PROPS_NBIN1] */
  float *dens178, *dens_int178;            /* [PSOD_PROPS_NBIN2] */
} psod_props_table;

int psod_halo_properties(psod_ctx *ctx, const psod_props_params *p, psod_props_stats *stats);
int psod_props_get(psod_ctx *ctx, const psod_props_table *t);

const char *psod_last_error(const psod_ctx *ctx);
const char *psod_status_string(int status);
int psod_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PSOD_H */
