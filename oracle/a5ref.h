/*
 * a5ref — CPU oracle for the a5_streamer per-timestep path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is a plain C++ restatement of the
 * reference's Fortran algorithm (Afivo tree, ghost cells, restriction,
 * prolongation, FAS multigrid, and the 2D/cylindrical streamer callbacks).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it, and only as the checker or the timed CPU baseline. The product
 * (a5_streamer_b200) never links or calls it.
 *
 * Parity status: the reference is Fortran 2008 and no Fortran compiler exists
 * in this build environment, and the reference ships no golden vectors. The
 * restatement is therefore pinned only by the reference's own known-answer
 * cases (manufactured Poisson solutions, lookup-table convergence), restated
 * in tests/. In that sense its parity with the reference binary is UNPINNED.
 *
 * All arithmetic is IEEE double, compiled with -ffp-contract=off so that no
 * fused multiply-add changes the rounding of any expression; operation order
 * follows the Fortran source expression by expression.
 */
#ifndef A5REF_H
#define A5REF_H

#ifdef __cplusplus
extern "C" {
#endif

#define A5REF_MAX_SEEDS 8
#define A5REF_MAX_TD_ROWS 4096

typedef struct a5ref_params {
  int dim;               /* 2 (3 not yet restated) */
  int coord;             /* 0 = Cartesian, 1 = cylindrical (r,z) */
  int box_size;          /* cells per box edge (ST_box_size) */
  int n_base[3];         /* base boxes per direction (4x4 in the 8 mm case) */
  double dr_base;        /* cell size at level 1 */
  int lvls_max;          /* finest allowed level */
  double domain_len_z;   /* length along the last axis, sets the applied voltage */
  double applied_fld;    /* ST_applied_fld (V/m); voltage = -len_z * fld */
  double epsilon_diel;   /* ST_epsilon_diel */
  double bg_dens;
  int n_seeds;
  double seed_r0[A5REF_MAX_SEEDS][3];
  double seed_r1[A5REF_MAX_SEEDS][3];
  double seed_dens[A5REF_MAX_SEEDS];
  double seed_width[A5REF_MAX_SEEDS];
  int seed_falloff[A5REF_MAX_SEEDS];
  double dt_max;
  int num_steps_amr;
  int use_drt;           /* 1: include dt_drt in the step-size minimum */
  int n_cycle_base;      /* 8 (Cartesian) / 4 (cylindrical) in the reference */
  double ref_init_time;  /* refine around the seed while t < this */
  double crv_refine;     /* refine if adx > 1 and crv_phi > this */
  /* transport table */
  int lkptbl_size;
  double lkptbl_max_fld;
  int td_n[4];                          /* number of input pairs per column */
  double td_x[4][A5REF_MAX_TD_ROWS];    /* input x (|E|) per column */
  double td_y[4][A5REF_MAX_TD_ROWS];    /* input y per column */
  int n_threads;         /* OpenMP threads; <= 0 keeps the runtime default */
  /* Photoionization, src/m_photons.f90 and src/streamer_cyl.f90:572-617
   * (cylindrical form: constant absorption level, PH_set_src_2d with
   * const_dx and use_cyl). */
  int photoi_enabled;
  int photoi_num_photons;  /* ST_photoi_num_photons */
  int photoi_team;         /* size of the OpenMP team whose execution of the
                              photon loops is reproduced (see below) */
  int photoi_tbl_kind;     /* 0: PH_get_tbl_air; 1: log-uniform absorption length */
  double photoi_coeff;     /* photons per ionization: eta * quench factor */
  double photoi_p_O2;      /* kind 0: O2 partial pressure (bar) */
  double photoi_len_lo;    /* kind 1: shortest absorption length (m) */
  double photoi_len_hi;    /* kind 1: longest absorption length (m) */
  double photoi_max_dist;  /* table range; the reference uses 2 * domain length */
  double photoi_fac_dx;    /* 0.25e-3 in the cylindrical driver */
  int rng_seed[4];         /* state of the master generator ST_rng */
  int uniform_lvl;         /* > 0: refine every box below this level, keep the
                              rest (a uniformly refined mesh) */
} a5ref_params;

/* The photon loops of PH_set_src_2d run in OpenMP regions whose outcome
 * depends on the team: each thread draws from its own generator seeded from
 * the master, loops are split by the static schedule, and photons are
 * numbered in the order threads pass a critical section. The oracle
 * reproduces the execution in which a team of photoi_team threads passes
 * that section thread by thread (thread 0 first), and combines the
 * reduction of a$D_tree_sum_cc in thread order. Both are executions the
 * reference can take with OMP_NUM_THREADS = photoi_team. */

typedef struct a5ref_sim a5ref_sim;

a5ref_sim *a5ref_create(const a5ref_params *p);
void a5ref_destroy(a5ref_sim *s);

/* Initial refinement loop: set_init_cond / compute_fld / adjust_refinement
 * until no box is added (src/streamer_2d.f90:58-63). Returns #iterations. */
int a5ref_init(a5ref_sim *s);
/* One pass of set_init_cond over all boxes (no refinement). */
void a5ref_set_init_cond(a5ref_sim *s);

/* get_max_dt (src/streamer_2d.f90:271-303). */
double a5ref_get_max_dt(a5ref_sim *s);
/* The three reductions get_max_dt uses: max |E|, min |E|, max n_e. */
void a5ref_dt_reductions(a5ref_sim *s, double out3[3]);
/* One full time step at fixed dt on a frozen mesh
 * (src/streamer_2d.f90:93-128, one iteration of the n loop). */
void a5ref_step(a5ref_sim *s, double dt);
/* Main-loop block: get_max_dt, num_steps_amr steps, adjust_refinement,
 * prolong_to_new_boxes + compute_fld if the mesh changed. Returns dt used. */
double a5ref_advance(a5ref_sim *s, int do_regrid);
/* Run the main loop until time > t_end or max_blocks blocks; returns blocks. */
int a5ref_run(a5ref_sim *s, double t_end, int max_blocks);
double a5ref_time(a5ref_sim *s);
void a5ref_set_time(a5ref_sim *s, double t);

/* Individual operations, for per-phase parity tests. */
void a5ref_op_copy_cc(a5ref_sim *s, int iv_from, int iv_to);
void a5ref_op_fluxes_koren(a5ref_sim *s, double dt);
void a5ref_op_consistent_fluxes(a5ref_sim *s);
void a5ref_op_update_solution(a5ref_sim *s, double dt);
void a5ref_op_restrict_tree(a5ref_sim *s, int iv);
/* rb_kind: 0 = interp_lim, 1 = interp; bc is Neumann */
void a5ref_op_gc_tree(a5ref_sim *s, int iv, int rb_kind);
void a5ref_op_average_dens(a5ref_sim *s);
void a5ref_op_compute_fld(a5ref_sim *s, int no_guess);
void a5ref_op_set_rhs(a5ref_sim *s);
void a5ref_op_fmg(a5ref_sim *s, int set_residual, int first_call);
void a5ref_op_fld_from_pot(a5ref_sim *s);
void a5ref_op_vcycle(a5ref_sim *s, int max_lvl, int set_residual);
/* Level-set boundaries of the field solves (lsf, bval per cell, export
 * layout; NULL removes them); box tags are reset. */
void a5ref_set_level_set(a5ref_sim *s, const double *lsf, const double *bval);
/* Photons created by the last photoionization call. */
long long a5ref_photons_created(a5ref_sim *s);
/* get_streamer_properties (src/streamer_cyl.f90:682-828): 39 values. */
void a5ref_streamer_properties(a5ref_sim *s, double *props39);
/* get_cc_axis (src/streamer_cyl.f90:905-956): 5 x n values (z, n_e, n_i,
 * axial field, axial electron flux); returns n. */
int a5ref_cc_axis(a5ref_sim *s, double *out, int cap);
/* The arrays of a$D_write_vtk (afivo/src/m_aX_io.f90:20-207) for the leaves
 * of levels 1..max_lvl: node coordinates (x, y per node), connectivity,
 * offsets, cell types, and per cell the n_iv variables ivs and the fx / fy
 * cell means of the n_if face variables ifs (variable-major). Outputs may be
 * NULL; returns the number of cells. */
int a5ref_vtk_arrays(a5ref_sim *s, int n_iv, const int *ivs, int n_if, const int *ifs,
                     double *coords, int *connects, int *offsets, int *types, double *vals);
double a5ref_tree_max_cc(a5ref_sim *s, int iv);
double a5ref_tree_min_cc(a5ref_sim *s, int iv);
double a5ref_tree_sum_cc(a5ref_sim *s, int iv, int team);
/* Per-box refinement flags from set_ref_flags (levels 1..max_lvl; boxes not
 * visited hold -huge). out has max_id+1 entries, index = box id. */
void a5ref_op_ref_flags(a5ref_sim *s, int *out);
/* adjust_refinement + prolong_to_new_boxes; returns n_add + n_rm. */
int a5ref_op_regrid(a5ref_sim *s, int *n_add, int *n_rm);

/* Tree export. Boxes are numbered 1..max_id as in the reference. */
int a5ref_max_id(a5ref_sim *s);
int a5ref_max_lvl(a5ref_sim *s);
int a5ref_min_lvl(a5ref_sim *s);
int a5ref_n_leaf_cells(a5ref_sim *s);
int a5ref_n_cells_all(a5ref_sim *s);
/* meta: per id (0..max_id) 16 ints: in_use, lvl, ix0, ix1, ix2, parent,
 * children[4] (2D: first 4 used), neighbors[4], n_cell, pad. */
void a5ref_export_meta(a5ref_sim *s, int *meta);
/* per id: r_min[3], dr */
void a5ref_export_geom(a5ref_sim *s, double *geom);
/* level lists: for each level min..max writes ids/leaves/parents counts
 * into counts[3*(nlev)] and the ids concatenated into ids (capacity cap). */
int a5ref_export_levels(a5ref_sim *s, int *counts, int *ids, int cap);
/* Cell data for variable iv: per id, (n_cell+2)^2 values laid out i-fastest
 * in a slot of (box_size+2)^2 doubles; unused ids are zero. */
void a5ref_export_cc(a5ref_sim *s, int iv, double *out);
void a5ref_import_cc(a5ref_sim *s, int iv, const double *in);
/* Face data fx/fy of face variable f: per id a slot of (nc+1)*nc doubles. */
void a5ref_export_fc(a5ref_sim *s, int dimf, int f, double *out);
void a5ref_import_fc(a5ref_sim *s, int dimf, int f, const double *in);
/* The tree of a run checkpoint (per-id records and level lists in the
 * layout of a5s_checkpoint_save); data follow with a5ref_import_cc/_fc. */
int a5ref_import_tree(a5ref_sim *s, int max_id, int min_lvl, int max_lvl, const int *rec_i,
                      const double *rec_d, int n_lists, const int *counts, const int *ids);
/* The built lookup table rows_cols (n_rows x 4, column-major) and x grid. */
void a5ref_export_table(a5ref_sim *s, double *rows_cols, double *x_min,
                        double *inv_dx, int *n_rows);
double a5ref_applied_voltage(a5ref_sim *s);

/* Known-answer multigrid case restating afivo/examples/multigrid/test_mg2_2d.f90
 * (two Gaussians, Dirichlet by the exact solution, curvature refinement).
 * Writes per-FMG-cycle max |residual| and max |error| and returns #cells. */
int a5ref_kat_mg2_2d(int n_fmg, double *res_out, double *err_out,
                     int *max_lvl_out);
/* Cylindrical variant restating afivo/examples/multigrid/test_mg_cyl.f90. */
int a5ref_kat_mg_cyl(int n_fmg, double *res_out, double *err_out,
                     int *max_lvl_out);
/* Cylindrical problem with a jump in eps restating
 * afivo/examples/multigrid/test_mg_cyl_diel.f90 (eps operators); returns the
 * number of boxes the multigrid treats as dielectric. */
int a5ref_kat_mg_cyl_diel(int n_fmg, double *res_out, double *err_out,
                          int *max_lvl_out);
/* Layered dielectric restating afivo/examples/multigrid/test_mg3_2d.f90
 * (eps 1 / 4, exact piecewise-linear potential); returns the leaf boxes. */
int a5ref_kat_mg3_2d(int n_fmg, double *res_out, double *err_out, int *max_lvl_out);
/* Level-set boundary restating afivo/examples/multigrid/test_mgb_2d.f90
 * (shape 0: its ellipse; 1: a plane with an exact piecewise-linear
 * solution); returns the boxes the multigrid treats with the level-set
 * operators. */
int a5ref_kat_mgb_2d(int shape, int n_fmg, double *res_out, double *err_out);
/* Lookup-table convergence test restating fosito/test/test_m_lookup_table.f90:
 * max error of LT_get_col on sin(x) for a table of n_rows over [0, x_max]. */
double a5ref_kat_lookup(int n_rows, int n_pairs, double x_max, int n_samples);
/* set_photoionization (src/streamer_cyl.f90:572-593): photon production
 * rate per leaf cell, then PH_set_src_2d. has_dt = 0 is the call without dt
 * before the time loop (:68-69). Needs photoi_enabled and coord = 1. */
void a5ref_op_photoionization(a5ref_sim *s, double dt, int has_dt);
/* State of the master generator (4 int32). */
void a5ref_rng_get(a5ref_sim *s, int *state4);
void a5ref_rng_set(a5ref_sim *s, const int *state4);
/* The photon absorption table: n_rows distances at the cumulative
 * fractions x = (i-1)/(n_rows-1); frac_in_tbl; the absorption level. */
int a5ref_photon_table(a5ref_sim *s, double *dist, int cap, double *frac_in_tbl,
                       int *pho_lvl);
/* Stand-alone photon table (kind 0: air with p_O2; kind 1: log-uniform
 * lengths [len_lo, len_hi]) over [0, max_dist]: returns n_rows (500). */
int a5ref_kat_photon_table(int kind, double p_O2, double len_lo, double len_hi,
                           double max_dist, double *dist, double *frac_in_tbl);
/* Known-answer case restating src/test_m_photons.f90: n photons absorbed
 * from the origin in 3D with a team of n_team generators seeded from a
 * default master; returns the mean absorption distance. */
double a5ref_kat_photon_dist(double p_O2, double max_dist, int n_photons, int n_team);
/* The first n outputs of RNG_t%int4 from the given state (mzran). */
void a5ref_kat_rng(const int *state4, int n, int *out);
/* Koren limiter (src/m_streamer.f90:339-362). */
double a5ref_koren_mlim(double a, double b);
/* Known-answer case restating afivo/examples/transport/test_drift_diff_2d.f90:
 * exact advection of sin^4(x-t) cos^4(y-t) on the periodic square with Koren
 * fluxes, the trapezoidal step and AMR (uniform_lvl > 0: uniform mesh of that
 * level; regrid 0: frozen mesh). out8: max and mean |error| at the end, sum
 * of phi at the start and end, steps, max level, leaf cells, end time.
 * Returns 0, or -1 if a physical-boundary routine was called. */
int a5ref_kat_drift_diff(int uniform_lvl, double end_time, int regrid, double *out8);

/* ---------------------------------------------------------------------------
 * The 3D octree form (src/streamer_3d.f90, afivo's m_a3_* routines) on
 * uniformly refined octrees: params with dim 3, uniform_lvl >= 1 (every box
 * below that level refined; the tree is coarsened to 2^3-cell boxes below
 * level 1), n_base[3] base boxes, epsilon_diel 1 and no photoionization;
 * a5ref3_create returns NULL for anything else. Refinement-boundary rules
 * never apply on such a tree. Layouts: cell variables in slots of
 * (box_size+2)^3 doubles per id (i fastest), faces in slots of
 * (box_size+1) box_size^2 per id and direction, meta 24 ints per id (in_use,
 * lvl, ix[3], parent, children[8], neighbors[6], n_cell), geometry 4 doubles
 * per id (r_min[3], dr). */
typedef struct a5ref3_sim a5ref3_sim;
a5ref3_sim *a5ref3_create(const a5ref_params *p);
void a5ref3_destroy(a5ref3_sim *s);
/* set_init_cond / compute_fld / refine until uniform_lvl is reached
 * (src/streamer_3d.f90:55-61); returns #iterations, -1 on failure. */
int a5ref3_init(a5ref3_sim *s);
void a5ref3_set_init_cond(a5ref3_sim *s);
void a5ref3_dt_reductions(a5ref3_sim *s, double out3[3]);
double a5ref3_get_max_dt(a5ref3_sim *s);
void a5ref3_step(a5ref3_sim *s, double dt);
double a5ref3_advance(a5ref3_sim *s);
double a5ref3_time(a5ref3_sim *s);
void a5ref3_set_time(a5ref3_sim *s, double t);
void a5ref3_op_copy_cc(a5ref3_sim *s, int iv_from, int iv_to);
void a5ref3_op_fluxes_koren(a5ref3_sim *s, double dt);
void a5ref3_op_update_solution(a5ref3_sim *s, double dt);
void a5ref3_op_restrict_tree(a5ref3_sim *s, int iv);
void a5ref3_op_gc_tree(a5ref3_sim *s, int iv);
void a5ref3_op_average_dens(a5ref3_sim *s);
void a5ref3_op_set_rhs(a5ref3_sim *s);
void a5ref3_op_compute_fld(a5ref3_sim *s, int no_guess);
void a5ref3_op_fmg(a5ref3_sim *s, int set_residual, int first_call);
void a5ref3_op_vcycle(a5ref3_sim *s, int max_lvl, int set_residual);
void a5ref3_op_fld_from_pot(a5ref3_sim *s);
double a5ref3_tree_max_cc(a5ref3_sim *s, int iv);
double a5ref3_tree_min_cc(a5ref3_sim *s, int iv);
double a5ref3_applied_voltage(a5ref3_sim *s);
int a5ref3_max_id(a5ref3_sim *s);
int a5ref3_max_lvl(a5ref3_sim *s);
int a5ref3_min_lvl(a5ref3_sim *s);
long long a5ref3_n_leaf_cells(a5ref3_sim *s);
void a5ref3_export_meta(a5ref3_sim *s, int *meta24);
void a5ref3_export_geom(a5ref3_sim *s, double *geom4);
int a5ref3_export_levels(a5ref3_sim *s, int *counts, int *ids, int cap);
void a5ref3_export_cc(a5ref3_sim *s, int iv, double *out);
void a5ref3_import_cc(a5ref3_sim *s, int iv, const double *in);
void a5ref3_export_fc(a5ref3_sim *s, int dimf, int f, double *out);
void a5ref3_import_fc(a5ref3_sim *s, int dimf, int f, const double *in);
void a5ref3_export_table(a5ref3_sim *s, double *rows_cols, double *x_min, double *inv_dx,
                         int *n_rows);
/* afivo/examples/multigrid/test_mg2_3d.f90 on a uniform octree of `level`:
 * max |residual| and max |error| after each of n_fmg FMG cycles. Returns the
 * finest level, < 0 on failure. */
int a5ref3_kat_mg(int level, int n_fmg, double *res, double *err);
/* afivo/examples/transport/test_drift_diff_3d.f90 on a uniform octree of
 * `level`: out8 as a5ref_kat_drift_diff. */
int a5ref3_kat_drift_diff(int level, double end_time, double *out8);

/* Differentiation check (a5ref_tl.inc). P(p): set_init_cond on every box,
 * compute_fld with no guess, n_steps time steps at the step sizes dts on the
 * current (fixed) mesh, then J = the softmax-weighted height of the leaf
 * cells next to the line x = x0 (weights dy exp((|E| - max |E|) / T)).
 * a5ref_program returns J; a5ref_tl_program also runs n_dir tangent-linear
 * directions in lockstep (per direction: the derivative of the table rows,
 * n_rows x 4 column-major, in dtbl, and of the applied voltage in dV) and
 * writes dJ[n_dir]. */
double a5ref_program(a5ref_sim *s, int n_steps, const double *dts, double x0, double T);
double a5ref_tl_program(a5ref_sim *s, int n_steps, const double *dts, double x0, double T,
                        int n_dir, const double *dtbl, const double *dV, double *dJ);
/* (y, dy, |E|) of each leaf cell next to x = x0; returns the count. */
int a5ref_head_profile(a5ref_sim *s, double x0, double *out3);
/* Replace the table rows (n_rows x 4, column-major) / the applied field. */
void a5ref_set_table_rows(a5ref_sim *s, const double *rows_cols);
void a5ref_set_applied_fld(a5ref_sim *s, double fld);

#ifdef __cplusplus
}
#endif
#endif
