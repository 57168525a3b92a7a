/*
 * a5g — B200-native (sm_100a) device path for a5_streamer's per-timestep work.
 *
 * C ABI: plain pointers and sizes, no C++ or torch types. One context holds
 * one run (a quadtree of boxes and their cell/face data) resident in device
 * memory. Every call returns an a5g_status; a5g_last_error() gives the text.
 *
 * The reference drives this path from Fortran through Afivo's procedure-
 * pointer "plugin" API (afivo/src/m_aX_t.f90:207-268 for the box-loop and
 * ghost-cell callback interfaces, afivo/src/m_aX_mg.f90:20-85 for the
 * multigrid operator table). Device code cannot call host procedure
 * pointers, so each callback the streamer drivers plug in becomes a named
 * entry point below; boundary-condition callbacks become enums.
 *
 * Data conventions (same as the reference):
 *  - box ids are 1-based (0 = no box, negative = physical boundary) and index
 *    device slots directly; slot 0 is unused;
 *  - cell variable iv of box id is a slot of (box_size+2)^2 doubles holding
 *    that box's (nc+2)^2 values i-fastest (nc = box_size on levels >= 1,
 *    smaller on the coarse subtree levels <= 0);
 *  - face variables: fx(1:nc+1,1:nc) and fy(1:nc,1:nc+1) in slots of
 *    (box_size+1)*box_size doubles;
 *  - cell variables: 0 n_e, 1 n_i, 2 n_e old, 3 n_i old, 4 phi, 5 |E|,
 *    6 rhs, 7 photoionization, 8 eps (src/m_streamer.f90:17-27);
 *    face variables: 0 electron flux, 1 field (src/m_streamer.f90:31-33).
 */
#ifndef A5G_H
#define A5G_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum a5g_status {
  A5G_OK = 0,
  A5G_EINVAL = 1,      /* bad argument or unsupported configuration */
  A5G_ENOMEM = 2,      /* device allocation failed */
  A5G_ECUDA = 3,       /* CUDA runtime error */
  A5G_TIMEOUT = 4,     /* a bounded device wait gave up */
  A5G_ENONFINITE = 5,  /* a NaN/Inf was detected where a finite value is required */
  A5G_ESTATE = 6       /* call out of order (no tree, no table, ...) */
} a5g_status;

#define A5G_N_VAR_CELL 9
#define A5G_N_VAR_FACE 2

/* Parameters of one run. Mirrors the reference's configuration variables
 * that the device path reads (src/m_streamer.f90:145-228, 386-417). */
typedef struct a5g_params {
  int box_size;          /* cells per box edge; 8 is supported */
  int coord;             /* 0 Cartesian (x,y), 1 cylindrical (r,z) */
  int lvls_max;          /* finest allowed level */
  double dr_base;        /* cell size at level 1 (a$D_lvl_dr) */
  double domain_len_z;   /* domain length along the last axis (m) */
  double applied_fld;    /* background field (V/m); phi(top) = -len_z * fld */
  double epsilon_diel;   /* ST_epsilon_diel: permittivity below a quarter of the
                            domain (set_box_eps); 1 for none, > 0 */
  double dt_max;         /* ST_dt_max */
  int use_drt;           /* 1: dielectric-relaxation limit enters the dt minimum */
  int n_cycle_base;      /* base-level Gauss-Seidel cycles (8 Cartesian, 4 cyl) */
  double ref_init_time;  /* refine around the seeds while t < this */
  double crv_refine;     /* refine if dx*alpha > 1 and crv_phi > this */
  int n_seeds;           /* seed lines for the refinement criterion (<= 8) */
  double seed_r0[8][2];
  double seed_r1[8][2];
  double seed_width[8];
  /* Monte Carlo photoionization, cylindrical form only: set_photoionization
   * (src/streamer_cyl.f90:572-617) and PH_set_src_2d with a constant
   * absorption level (src/m_photons.f90:207-436). */
  int photoi_enabled;
  int photoi_num_photons; /* ST_photoi_num_photons */
  int photoi_team;        /* OpenMP team whose execution of the photon loops
                             is reproduced; see a5g_photoionization */
  int photoi_pad;
  double photoi_coeff;    /* photons per ionization (photoi_eta * quench factor) */
  double photoi_fac_dx;   /* table fraction that sets the absorption level (0.25e-3) */
  int rng_seed[4];        /* state of the master generator ST_rng */
  /* > 0: refine every box below this level and keep the rest instead of the
   * streamer's criterion (a uniformly refined mesh, as the multigrid
   * benchmark afivo/examples/multigrid/test_mg_benchmark_2d.f90:40-86
   * builds); 0: set_ref_flags */
  int uniform_lvl;
  int uniform_pad;
} a5g_params;

/* Box metadata for a5g_upload_tree: per id (0..max_id) 16 ints
 *   [0] in_use, [1] lvl, [2] ix0, [3] ix1, [4] unused, [5] parent,
 *   [6..9] children, [10..13] neighbors (lx, hx, ly, hy), [14] n_cell, [15] 0
 * and per id 4 doubles: r_min0, r_min1, unused, dr.
 * Level lists: for lvl = min_lvl..max_lvl, counts[3*k + {0,1,2}] = number of
 * ids / leaves / parents, and ids[] holds, level by level, the ids, then the
 * leaves, then the parents (the lists of lvl_t, afivo/src/m_aX_t.f90:165-169).
 */

typedef struct a5g_ctx a5g_ctx;

const char *a5g_last_error(void);
int a5g_version(void);

/* Context life cycle. Replaces a$D_init (afivo/src/m_aX_core.f90:47-116):
 * the device context owns all box storage. */
int a5g_create(const a5g_params *p, a5g_ctx **out);
int a5g_destroy(a5g_ctx *ctx);

/* Transport table: replaces LT_create/LT_set_col
 * (fosito/m_lookup_table.f90:46-72). rows_cols is n_rows x n_cols,
 * column-major (rows_cols(n_rows, n_cols)); columns mobility, diffusion,
 * alpha, eta (src/m_streamer.f90:37-41). */
int a5g_set_table(a5g_ctx *ctx, int n_rows, int n_cols, double x_min,
                  double inv_dx, const double *rows_cols);

/* Photon absorption table: replaces PH_tbl_t (src/m_photons.f90:9-12).
 * dist[i] is the absorption distance at cumulative fraction
 * x_min + i / inv_dx (i = 0..n_rows-1), frac_in_tbl the fraction of photons
 * inside the table's range. Also fixes the absorption level
 * get_lvl_length(dr_base, LT_get_col(tbl, photoi_fac_dx))
 * (src/m_photons.f90:142-155, 331-336). */
int a5g_set_photon_table(a5g_ctx *ctx, int n_rows, double x_min, double inv_dx,
                         const double *dist, double frac_in_tbl);
/* State of the master generator (4 int32, fosito/m_random.f90 RNG_t). */
int a5g_get_rng(a5g_ctx *ctx, int *state4);
int a5g_set_rng(a5g_ctx *ctx, const int *state4);

/* Topology upload after a$D_set_base / a$D_adjust_refinement
 * (afivo/src/m_aX_core.f90:134-217, 456-520). Cell and face data of ids
 * that stay in use are preserved on the device; storage grows as needed. */
int a5g_upload_tree(a5g_ctx *ctx, int max_id, int min_lvl, int max_lvl,
                    const int *meta16, const double *geom4,
                    const int *lvl_counts, const int *lvl_ids);

/* Host <-> device copies of one cell / face variable for ids 0..max_id,
 * slot layout as described above. */
int a5g_upload_cc(a5g_ctx *ctx, int iv, const double *host);
int a5g_download_cc(a5g_ctx *ctx, int iv, double *host);
int a5g_upload_fc(a5g_ctx *ctx, int dimf, int f, const double *host);
int a5g_download_fc(a5g_ctx *ctx, int dimf, int f, double *host);

/* Box-loop equivalents of the streamer callbacks and Afivo tree routines. */
/* a$D_tree_copy_cc, afivo/src/m_aX_utils.f90:432-453 */
int a5g_tree_copy_cc(a5g_ctx *ctx, int iv_from, int iv_to);
/* a$D_loop_boxes_arg(fluxes_koren), src/streamer_2d.f90:384-489 (with the
 * second ghost layer of afivo/src/m_aX_gc.f90:407-622) */
int a5g_fluxes_koren(a5g_ctx *ctx, double dt);
/* a$D_consistent_fluxes([f_elec]), afivo/src/m_aX_core.f90:818-930 */
int a5g_consistent_fluxes(a5g_ctx *ctx);
/* a$D_loop_box_arg(update_solution), src/streamer_2d.f90:499-542,
 * src/streamer_cyl.f90:531-570 */
int a5g_update_solution(a5g_ctx *ctx, double dt);
/* a$D_restrict_tree, afivo/src/m_aX_restrict.f90:54-142 */
int a5g_restrict_tree(a5g_ctx *ctx, int iv);
/* a$D_gc_tree(iv, a$D_gc_interp_lim | a$D_gc_interp, a$D_gc_neumann),
 * afivo/src/m_aX_gc.f90:28-330. rb_kind 0 = interp_lim, 1 = interp. */
int a5g_gc_tree(a5g_ctx *ctx, int iv, int rb_kind);
/* a$D_loop_box(average_dens), src/streamer_2d.f90:492-496 */
int a5g_average_dens(a5g_ctx *ctx);
/* compute_fld, src/streamer_2d.f90:307-343: space charge, one FAS FMG cycle
 * (afivo/src/m_aX_mg.f90:163-565), fld_from_pot and the |E| ghost fill. */
int a5g_compute_fld(a5g_ctx *ctx, int no_guess);
/* compute_fld in FP64 whatever the run's precision (a5g_set_precision). For
 * the solve that follows prolong_to_new_boxes (src/streamer_2d.f90:134-138)
 * in the mixed form: on new boxes the potential's correction is large and
 * smooth, and one FP32 correction pass evaluates its Laplacian with too few
 * digits (max |E| 1.7e-3 off on the 7 MV/m 8 mm case) where the FP64 FAS
 * solve is not. The a5s driver uses it after every regrid. */
int a5g_compute_fld_fp64(a5g_ctx *ctx, int no_guess);
/* mg$D_fas_fmg(tree, mg, set_residual, first_call) alone */
int a5g_fas_fmg(a5g_ctx *ctx, int set_residual, int first_call);
/* mg$D_fas_vcycle(tree, mg, max_lvl, set_residual) alone
 * (afivo/src/m_aX_mg.f90:208-254): one FAS V-cycle from level max_lvl
 * (min_lvl..max_lvl of the tree) down to the coarsest level and back, the
 * potential's ghost cells valid on input and output; set_residual != 0 also
 * stores rhs - A phi of levels min_lvl..max_lvl in the scratch variable
 * (i_fld, as the reference's i_tmp). */
int a5g_mg_fas_vcycle(a5g_ctx *ctx, int max_lvl, int set_residual);
/* fld_from_pot on all boxes + a$D_gc_tree(i_fld, a$D_gc_interp, neumann) */
int a5g_fld_from_pot(a5g_ctx *ctx);
/* a$D_tree_max_cc / a$D_tree_min_cc (afivo/src/m_aX_utils.f90:559-619):
 * max / min of cell variable iv over the interior cells of the leaves.
 * Synchronises. */
int a5g_tree_max_cc(a5g_ctx *ctx, int iv, double *out);
int a5g_tree_min_cc(a5g_ctx *ctx, int iv, double *out);
/* a$D_tree_sum_cc (afivo/src/m_aX_utils.f90:621-680): sum over the leaves
 * of lvl_dr^2 times the box sum (cylindrical: of 2 pi r times the value).
 * The reference forms it in an OpenMP reduction whose rounding depends on the
 * team; this call gives the value a team of `team` threads forms (static
 * chunks of each level's leaves, partial sums added in thread order; team 1
 * is the plain loop order). Synchronises. */
int a5g_tree_sum_cc(a5g_ctx *ctx, int iv, int team, double *out);
/* The reductions of get_max_dt (src/streamer_2d.f90:280-282):
 * out3 = {max |E|, min |E|, max n_e} over leaf interiors. */
int a5g_dt_reductions(a5g_ctx *ctx, double *out3);
/* get_max_dt, src/streamer_2d.f90:271-303 (cyl :281-314) */
int a5g_get_max_dt(a5g_ctx *ctx, double *dt);
/* set_ref_flags for every box on levels 1..max_lvl
 * (src/streamer_2d.f90:177-216, cyl :190-227); flags has max_id+1 ints,
 * ids not visited hold INT_MIN+1 (the reference's -huge). */
int a5g_ref_flags(a5g_ctx *ctx, double time, int *flags);
/* prolong_to_new_boxes, src/streamer_2d.f90:592-617: for each level
 * min_lvl..max_lvl in turn, n_new[k] ids taken from new_ids in order. */
int a5g_prolong_new(a5g_ctx *ctx, const int *n_new, const int *new_ids);
/* set_photoionization(tree, eta, num_photons[, dt])
 * (src/streamer_cyl.f90:572-593): photon production per leaf cell, then
 * PH_set_src_2d (src/m_photons.f90:207-436): photons created by stochastic
 * rounding, absorbed at a sampled distance in a random direction, counted
 * per cell at the absorption level, then ghost cells and prolongation.
 * has_dt = 0 is the call before the time loop (no dt argument).
 * The reference runs these loops in OpenMP regions whose outcome depends on
 * the team: every thread draws from its own generator seeded from the master
 * (PRNG_t), loops are split by the static schedule, and photons are
 * numbered in the order threads pass a critical section. This call
 * reproduces the execution with photoi_team threads that pass that section
 * in thread order and add the partial sums of a$D_tree_sum_cc in thread
 * order, an execution the reference takes with OMP_NUM_THREADS equal to
 * photoi_team. The master generator advances by 8 * photoi_team draws. */
int a5g_photoionization(a5g_ctx *ctx, double dt, int has_dt);
/* Photons created by the last photoionization call and its factor fac
 * (photons per unit production, src/m_photons.f90:250-256). Synchronises. */
int a5g_photon_stats(a5g_ctx *ctx, long long *n_created, double *fac);
/* Precision of the run's time steps. The reference computes in FP64
 * throughout (dp = kind(0d0)); A5G_MIXED is an addition of this library with
 * no counterpart there:
 *  - fluxes_koren, update_solution and their table lookups run in FP32;
 *  - every field solve is a defect correction: the residual of the space
 *    charge (n_i - n_e, which cancels) against the FP64 potential is formed
 *    in FP64, the correction equation is solved by an FP32 multigrid with
 *    the schedule below, and the correction is added to the FP64 potential;
 *  - densities, the potential, the field and the step-size reductions are
 *    stored and reduced in FP64.
 * With A5G_MIXED, a5g_step, the batched steps and a5g_compute_fld (except
 * with no_guess, which keeps the FP64 FMG from a zero potential) take the
 * mixed form. */
#define A5G_FP64 0
#define A5G_MIXED 1
/* Multigrid schedule of the FP32 correction solve (the FP64 path always
 * uses the reference's: FMG, 2 down, 2 up and n_cycle_base base cycles,
 * afivo/src/m_aX_mg.f90:163-254). */
typedef struct a5g_mg_schedule {
  int fmg;          /* 1: mg$D_fas_fmg; 0: one V-cycle over all levels */
  int n_cycle_down; /* red-black cycles per level on the way down, 1..8 */
  int n_cycle_up;   /* red-black cycles per level on the way up, 1..8 */
  int n_cycle_base; /* red-black cycles on the coarsest level, 1..64 */
  int n_corr;       /* defect-correction passes per field solve, 1..8 */
} a5g_mg_schedule;
/* sched NULL: the reference's schedule (1, 2, 2, n_cycle_base, 1). */
int a5g_set_precision(a5g_ctx *ctx, int precision, const a5g_mg_schedule *sched);
int a5g_get_precision(a5g_ctx *ctx, int *precision, a5g_mg_schedule *sched);
/* One full time step on the current mesh (src/streamer_2d.f90:93-128, one
 * iteration of the n loop): set_photoionization when enabled, save old
 * densities, two forward-Euler stages with a field solve after the first,
 * trapezoidal average, field solve. Without photoionization it is a single
 * device launch; with it, three (photon sources, absorption, step). */
int a5g_step(a5g_ctx *ctx, double dt);
/* The same step for several independent runs in one launch (one persistent
 * thread block per run). dts[k] is the step of run k. The launches go on the
 * first run's stream, ordered on the device after the work already queued on
 * every member's stream; work queued afterwards on any member's stream runs
 * after the batch (event waits, no host synchronisation). The device-driven
 * batch (a5g_batch_*) replays whole blocks of steps from CUDA graphs
 * instead. */
int a5g_step_batch(a5g_ctx **ctxs, int n, const double *dts);
/* Batched step that allocates no device memory. Same result as
 * a5g_step_batch; no counterpart in the reference (its Fortran host has no
 * device at all).
 *
 * Some callers cannot allocate device memory while they step: a host that
 * fixed its device-memory budget before the time loop, or one whose stepping
 * path must not block on the allocator (cudaMallocAsync may wait on the
 * memory pool). This entry point keeps the per-run descriptor table of the
 * launch in a fixed file-scope device array of A5G_STATIC_BATCH_MAX entries
 * (40 KiB), held by every GPU that loads the library until the process
 * exits, and calls no allocating routine. The caller still creates the
 * contexts (which own the inputs and outputs) beforehand.
 *  - n above A5G_STATIC_BATCH_MAX is rejected with A5G_EINVAL;
 *  - all contexts must belong to the current device;
 *  - the first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress) with that device current; make that first call
 *    before any stream capture;
 *  - every call shares the one array: calls that overlap on the GPU (on
 *    different streams) race; calls queued on one stream are ordered;
 *  - a mixed-precision member whose tree does not fit in shared memory keeps
 *    its FP32 multigrid arrays in device memory, which this call does not
 *    allocate: after each tree upload, step it once through a5g_step or
 *    a5g_step_batch, else this call returns A5G_ESTATE. */
#define A5G_STATIC_BATCH_MAX 1024
int a5g_step_batch_static(a5g_ctx **ctxs, int n, const double *dts);
/* Device-driven batch: one main-loop block (src/streamer_2d.f90:68-128:
 * get_max_dt, then num_steps_amr steps) for n runs in one launch per kernel.
 * Each run's step size, simulated time and active flag live on the device:
 * the block computes dt from the run's leaf reductions with the host's
 * arithmetic (a5g_get_max_dt), a run stays active until dt < 1e-14 or its
 * time exceeds its end time (the loop exits of :72-75), and only active runs
 * step. Since nothing of a block is decided on the host, the block is a
 * fixed launch sequence; with use_graph it is captured once in a CUDA graph
 * and replayed. The reference has no counterpart (it runs one tree per
 * process); it replaces a5g_get_max_dt + a5g_step per run.
 *  a5g_batch_begin: each run's current time and end time; also picks up
 *    changed precision and block settings;
 *  a5g_batch_block: one block; returns each run's dt of the block, its time
 *    after it, whether it stepped, and the block's device time (ms). The
 *    members' own streams are synchronised first (their regrids and uploads
 *    come before the block). */
/* Box-to-block mapping: a member set to n_cta > 1 blocks (a5g_set_ctas)
 * takes that many blocks of the batch's launches, as its own group with its
 * own grid barrier; when any member does, the block-dt and step launches are
 * single cooperative launches of all members' blocks (at most the blocks the
 * device holds at once). Results do not depend on the mapping. */
typedef struct a5g_batch a5g_batch;
int a5g_batch_create(a5g_ctx **ctxs, int n, a5g_batch **out);
int a5g_batch_destroy(a5g_batch *b);
int a5g_batch_begin(a5g_batch *b, const double *time, const double *t_end);
int a5g_batch_block(a5g_batch *b, int num_steps, int use_graph, double *dt, double *time,
                    int *active, float *gpu_ms);
/* a5g_batch_block in two halves: launch queues the block on the batch's own
 * stream and returns; finish waits for it and returns its results. Between
 * the two the host may work on other batches (e.g. regrid their runs). The
 * block is ordered on the device after the work queued on the members'
 * streams, and work queued on a member's stream after the launch runs after
 * the block. */
int a5g_batch_launch(a5g_batch *b, int num_steps, int use_graph);
int a5g_batch_finish(a5g_batch *b, double *dt, double *time, int *active, float *gpu_ms);
/* Internal boundaries of the field solve from a level set, the multigrid
 * operators mg$D_box_gsrb_lpllsf / mg$D_box_lpllsf / mg$D_box_corr_lpllsf
 * (afivo/src/m_aX_mg.f90:1073-1340) that Afivo's mg$D_auto_* apply to the
 * boxes where the level-set function changes sign (mg$D_set_box_tag,
 * :673-712): lsf and bval give per cell (ids 0..max_id, slot layout as
 * a5g_upload_cc, ghost cells included) the level-set function and the
 * potential on its zero contour. The solve then takes neighbours across the
 * contour at their distance with the boundary value. Restriction stays
 * mg$D_box_rstr_lpl (the reference's default). NULL, NULL removes the level
 * set. New boxes of a later topology hold 0 until set again; the mixed form
 * rejects level sets. */
int a5g_set_level_set(a5g_ctx *ctx, const double *lsf, const double *bval);
/* Grid mode: the run's phases on n_cta thread blocks instead of one. The
 * reference runs a box loop over the boxes of a level with OpenMP threads
 * (afivo/src/m_aX_utils.f90:58-185); one block per run keeps a small tree's
 * phases behind block barriers, which is the fast form for trees of a few
 * thousand cells, but uses one SM. With n_cta > 1 every operation of the run
 * (steps, field solves, reductions, flags, prolongation) is one cooperative
 * launch of n_cta co-resident blocks that share each phase's items, with a
 * grid barrier between phases; results are identical to one block. Each
 * barrier wait is bounded by wait_cycles SM clock cycles (< 0: the default,
 * A5G_DEFAULT_WAIT_CYCLES); a wait that runs out makes the launch return
 * early and the next synchronising call report A5G_TIMEOUT (0 makes every
 * wait run out at once: a way to exercise that path). n_cta is limited to the
 * blocks the device can hold at once (a5g_get_ctas reports it) and to
 * A5G_MAX_CTAS. The reference has no counterpart (it has no device). */
#define A5G_MAX_CTAS 256
#define A5G_DEFAULT_WAIT_CYCLES 4000000000LL
int a5g_set_ctas(a5g_ctx *ctx, int n_cta, long long wait_cycles);
int a5g_get_ctas(a5g_ctx *ctx, int *n_cta, int *max_cta);
/* Grid mode: multigrid levels are visited in order and the coarse ones hold
 * few cells, so a stretch of phases on levels of at most `cells` cells (from
 * the coarsest level up) runs on one block of the group while the others
 * wait at the barrier that ends it, instead of a grid barrier per phase.
 * 0 spreads every phase over the whole group. Results do not depend on it. */
#define A5G_DEFAULT_LOCAL_CELLS 8192
int a5g_set_grid_local(a5g_ctx *ctx, int cells);
/* Wait for all work queued on the context's stream. */
int a5g_sync(a5g_ctx *ctx);
/* Change the background field of a run (ST_applied_fld; the potential at
 * the top is -domain_len_z * applied_fld, src/m_streamer.f90:411) without
 * rebuilding it, for runs that vary it on a fixed mesh (finite-difference
 * checks of the adjoint, include/a5a.h). Takes effect at the next field
 * solve. */
int a5g_set_applied_field(a5g_ctx *ctx, double applied_fld);
/* The cudaStream_t (as void*) all work of this context is queued on, so a
 * caller can order its own work or timing events with it. */
int a5g_get_stream(a5g_ctx *ctx, void **stream);
/* Leaf cells of the uploaded tree (for throughput accounting). */
int a5g_n_leaf_cells(a5g_ctx *ctx, long long *n);

#ifdef __cplusplus
}
#endif
#endif
