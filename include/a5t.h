/*
 * a5t — host-side quadtree topology and a5s — streamer driver, C ABI.
 *
 * a5t replaces the tree routines of Afivo's core that the streamer drivers
 * call on the host between device steps (afivo/src/m_aX_core.f90):
 * a$D_init (:47-116), a$D_set_base (:134-217), a$D_adjust_refinement
 * (:456-520) with consistent_ref_flags (:624-726), add/remove_children
 * (:729-788), set_nbs / find_nb (:386-445), set_leaves_parents (:328-359).
 * The refinement callback of the reference (a$D_subr_ref) is replaced by a
 * flag array computed on the device (a5g_ref_flags).
 *
 * a5s replaces the driver program src/streamer_2d.f90 / streamer_cyl.f90:
 * initial conditions, the initial refinement loop, and the main loop of
 * time steps with a regrid every num_steps_amr steps. Box data live on the
 * device (include/a5g.h); the host keeps only the topology.
 */
#ifndef A5T_H
#define A5T_H

#include "a5g.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct a5t_tree a5t_tree;

/* a$D_init with coarsen_to = 2 (coarse subtree down to 2x2-cell boxes). */
int a5t_create(int box_size, int lvls_max, double dr_base, const double r_base[2],
               int coord, a5t_tree **out);
int a5t_destroy(a5t_tree *t);
/* a$D_set_base: n_boxes base boxes with 1-based indices ix_list[2*k..] and
 * neighbours nb_list[4*k..] (1-based box number, or negative for a physical
 * boundary; 0 entries are resolved from the other side). */
int a5t_set_base(a5t_tree *t, int n_boxes, const int *ix_list, const int *nb_list);
/* a$D_adjust_refinement with the given per-id user flags (length max_id+1,
 * values a5_rm_ref/kp_ref/do_ref or INT_MIN+1 for "not set"). */
int a5t_adjust_refinement(a5t_tree *t, const int *user_flags, int *n_add, int *n_rm);
int a5t_max_id(a5t_tree *t);
int a5t_min_lvl(a5t_tree *t);
int a5t_max_lvl(a5t_tree *t);
/* Export in the a5g_upload_tree format; returns the number of level-list ids
 * written (call once with NULL lvl_ids to size it). */
int a5t_export(a5t_tree *t, int *meta16, double *geom4, int *lvl_counts, int *lvl_ids);
int a5t_n_level_ids(a5t_tree *t);
/* Checks the invariants a topology upload relies on (A5G_EINVAL if one
 * fails): every box in use listed exactly once in its level's list, leaves
 * and parents boxes of their level, parents, children and neighbours in use
 * on the adjacent / same level. Host only; a5s_checkpoint_load applies it to
 * a checkpoint's tree before anything reaches the device. */
int a5t_check(a5t_tree *t);
/* Boxes added by the last adjust_refinement, per level min_lvl..max_lvl
 * (ref_info%lvls(lvl)%add). Returns the total. */
int a5t_new_boxes(a5t_tree *t, int *counts, int *ids);

/* Photon absorption table: PH_get_tbl_air (src/m_photons.f90:25-140),
 * 500 absorption distances at cumulative fractions (i-1)/499 over
 * [0, max_dist], and the fraction of photons inside that range.
 * kind 0: air, a = O2 partial pressure (bar), the absorption function
 * PH_absfunc_air; kind 1: absorption length log-uniform in [a, b] (m), the
 * same function with coefficients 1/b and 1/a. dist needs 500 entries;
 * n_rows receives the number of rows (500). */
int a5t_photon_table(int kind, double a, double b, double max_dist, double *dist,
                     double *frac_in_tbl, int *n_rows);

typedef struct a5s_config {
  a5g_params dev;
  int n_base[2];            /* base boxes per direction */
  double bg_dens;
  int n_seeds;
  double seed_dens[8];
  int seed_falloff[8];      /* src/m_geom.f90:8-11 */
  int num_steps_amr;
  int lkptbl_size;
  double lkptbl_max_fld;
  int td_n[4];              /* transport input pairs per column */
  const double *td_x[4];
  const double *td_y[4];
  /* photon table when dev.photoi_enabled (see a5t_photon_table); the
   * reference's range is 2 * domain length (src/m_streamer.f90:327-330) */
  int photoi_tbl_kind;
  double photoi_tbl_a, photoi_tbl_b;
  double photoi_max_dist;
} a5s_config;

typedef struct a5s_sim a5s_sim;

int a5s_create(const a5s_config *cfg, a5s_sim **out);
int a5s_destroy(a5s_sim *s);
/* Initial refinement loop (src/streamer_2d.f90:58-63). */
int a5s_init(a5s_sim *s, int *n_iter);
/* set_init_cond on every box of the current tree (src/streamer_2d.f90:218-248:
 * the seed densities, phi = 0, eps), without refinement. */
int a5s_set_init_cond(a5s_sim *s);
/* One main-loop block: get_max_dt, num_steps_amr steps, regrid. */
int a5s_advance(a5s_sim *s, int regrid, double *dt_used);
/* Main loop until time > t_end (or max_blocks blocks). */
int a5s_run(a5s_sim *s, double t_end, int max_blocks, int *n_blocks);
/* Main loop of n runs as device-driven batches until each run's
 * time > t_end[k]: per block, each run's get_max_dt and its num_steps_amr
 * steps run for all members of a batch in one launch per kernel (replayed
 * from a CUDA graph when use_graph), then the runs that stepped are
 * regridded on the host, n_threads at a time. With n_groups > 1 the members
 * are dealt to that many batches, each on its own stream, and a group's
 * regrids overlap the other groups' blocks on the device. Each run ends in
 * the state a5s_run(t_end[k]) gives it. gpu_ms: sum of the blocks' device
 * times (groups overlap); host_ms: wall time of the regrids; cell_updates:
 * leaf cells times steps over all members. Members share num_steps_amr and
 * the current device. */
int a5s_batch_run(a5s_sim **sims, int n, const double *t_end, int use_graph, int n_threads,
                  int n_groups, int max_blocks, int *n_blocks, double *gpu_ms, double *host_ms,
                  double *cell_updates);
int a5s_time(a5s_sim *s, double *t);
int a5s_ctx(a5s_sim *s, a5g_ctx **ctx);
int a5s_tree(a5s_sim *s, a5t_tree **tree);
/* The built transport table (rows_cols n_rows x 4, column-major). */
int a5s_table(a5s_sim *s, double *rows_cols, double *x_min, double *inv_dx, int *n_rows);

/* Checkpoint / resume of a run. The reference has no counterpart: it
 * persists only output snapshots (afivo/src/m_aX_io.f90:20-600), and a run
 * restarts from its initial conditions.
 * A checkpoint holds everything the run's next main-loop block depends on:
 * the simulated time, the photon generator's state, the tree (per-id
 * records and the level lists as a$D_adjust_refinement left them) and every
 * cell and face variable of ids 0..max_id, ghost cells included. A run
 * resumed from it continues exactly as the run that wrote it would have.
 * Run settings (precision and schedule, thread blocks per run, level-set
 * boundaries) are not part of it: set them on the resumed run again.
 *  a5s_checkpoint_size: bytes the next a5s_checkpoint_save writes;
 *  a5s_checkpoint_save: writes it into buf (cap bytes; A5G_EINVAL if too
 *    small); waits for the run's queued device work;
 *  a5s_checkpoint_load: replaces the run's state with the checkpoint's.
 *    The run must have been created from the same configuration (a
 *    fingerprint of the settings and the transport table is compared):
 *    A5G_EINVAL otherwise, or for a truncated or malformed buffer, and the
 *    run is left unchanged. */
int a5s_checkpoint_size(a5s_sim *s, size_t *bytes);
int a5s_checkpoint_save(a5s_sim *s, void *buf, size_t cap, size_t *written);
int a5s_checkpoint_load(a5s_sim *s, const void *buf, size_t len);

#ifdef __cplusplus
}
#endif
#endif
