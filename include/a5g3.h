/*
 * a5g3 -- the 3D octree form of the device path (src/streamer_3d.f90 with
 * afivo's m_a3_* routines) on sm_100a, for uniformly refined octrees.
 *
 * C ABI: plain pointers and sizes. One context holds one run: a uniformly
 * refined octree (every box below uniform_lvl refined, the base boxes
 * coarsened to 2^3-cell boxes on levels min_lvl..0 as a3_init with
 * coarsen_to = 2 does) and its cell and face data, resident in device
 * memory. Every call returns an a5g_status (include/a5g.h);
 * a5g3_last_error() gives the text.
 *
 * The reference builds the tree with a3_init / a3_set_base /
 * a3_adjust_refinement (afivo/src/m_aX_core.f90:47-217, 456-520) and runs
 * the streamer callbacks through a3_loop_box*, a3_gc_tree, a3_restrict_tree
 * and mg3_fas_fmg. Here the context builds the same tree (same ids, levels,
 * neighbours; a5g3_export_meta / a5g3_export_levels give it) and each
 * callback becomes an entry point. On a uniform octree no box has a
 * refinement boundary, so a3_gc_interp(_lim), mg3_sides_rb,
 * a3_gc2_prolong1 and a3_consistent_fluxes never apply.
 *
 * Layouts (the reference's, per id 0..max_id; id 0 unused):
 *  - cell variable iv: slot of (box_size+2)^3 doubles, (nc+2)^3 values
 *    i fastest then j then k (nc = box_size on levels >= 1, box_size/2,
 *    box_size/4 on levels 0, -1);
 *  - face variables fx(1:nc+1,1:nc,1:nc), fy(1:nc,1:nc+1,1:nc),
 *    fz(1:nc,1:nc,1:nc+1) in slots of (box_size+1)*box_size^2 doubles;
 *  - cell variables 0 n_e, 1 n_i, 2 n_e old, 3 n_i old, 4 phi, 5 |E|,
 *    6 rhs, 7 photoionization (unused), 8 eps; face variables 0 electron
 *    flux, 1 field (src/m_streamer.f90:17-33).
 */
#ifndef A5G3_H
#define A5G3_H

#include "a5g.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct a5g3_params {
  int box_size;        /* cells per box edge; 8 is supported */
  int n_base[3];       /* base boxes per direction (1 1 1 in the 3D example) */
  int uniform_lvl;     /* finest level; every box below it is refined (>= 1) */
  int n_cycle_base;    /* base-level Gauss-Seidel cycles (8, streamer_3d.f90:43) */
  int use_drt;         /* 1: the dielectric-relaxation limit enters get_max_dt */
  int pad;
  double dr_base;      /* cell size at level 1 */
  double domain_len_z; /* domain length; phi(top) = -len * applied_fld */
  double applied_fld;  /* background field (V/m) */
  double dt_max;       /* ST_dt_max */
} a5g3_params;

typedef struct a5g3_ctx a5g3_ctx;

const char *a5g3_last_error(void);

/* Build the uniform octree and allocate its storage on the current device.
 * Replaces init_tree + the initial refinement (src/streamer_3d.f90:146-175,
 * 55-61) for the uniform mesh. */
int a5g3_create(const a5g3_params *p, a5g3_ctx **out);
int a5g3_destroy(a5g3_ctx *ctx);

/* Tree: max_id, min_lvl, max_lvl, number of leaf cells. */
int a5g3_info(a5g3_ctx *ctx, int *max_id, int *min_lvl, int *max_lvl, long long *n_leaf_cells);
/* Per id 24 ints: in_use, lvl, ix[3], parent, children[8], neighbors[6]
 * (lx hx ly hy lz hz), n_cell, 0, 0, 0. */
int a5g3_export_meta(a5g3_ctx *ctx, int *meta24);
/* Per level min..max: counts[3 k + {0,1,2}] = #ids, #leaves, #parents; ids
 * holds the level's ids, leaves, parents in turn. *n_out: total length. */
int a5g3_export_levels(a5g3_ctx *ctx, int *counts, int *ids, int cap, int *n_out);

/* Transport table (LT_create / LT_set_col, fosito/m_lookup_table.f90:46-72):
 * n_rows x n_cols column-major; columns mobility, diffusion, alpha, eta. */
int a5g3_set_table(a5g3_ctx *ctx, int n_rows, int n_cols, double x_min, double inv_dx,
                   const double *rows_cols);

/* Initial conditions (set_init_cond and set_box_eps,
 * src/streamer_3d.f90:217-270) on every box: background density plus the
 * seeds (GM_dens_line, src/m_geom.f90:48-111; r0, r1: 3 per seed), n_i = n_e,
 * phi = 0, eps = 1 (epsilon_diel 1). The exponential of the fall-off shapes
 * is CUDA's exp, within 2 ulp of the reference's libm. */
int a5g3_set_init_cond(a5g3_ctx *ctx, double bg_dens, int n_seeds, const double *r0, const double *r1,
                       const double *dens, const double *width, const int *falloff);

int a5g3_upload_cc(a5g3_ctx *ctx, int iv, const double *host);
int a5g3_download_cc(a5g3_ctx *ctx, int iv, double *host);
int a5g3_upload_fc(a5g3_ctx *ctx, int dimf, int f, const double *host);
int a5g3_download_fc(a5g3_ctx *ctx, int dimf, int f, double *host);

/* The operations of the time step (src/streamer_3d.f90:96-128). */
int a5g3_tree_copy_cc(a5g3_ctx *ctx, int iv_from, int iv_to);  /* a3_tree_copy_cc */
int a5g3_fluxes_koren(a5g3_ctx *ctx, double dt);                /* :396-554, leaves */
int a5g3_update_solution(a5g3_ctx *ctx, double dt);             /* :566-615, leaves */
int a5g3_restrict_tree(a5g3_ctx *ctx, int iv);                  /* a3_restrict_tree */
int a5g3_gc_tree(a5g3_ctx *ctx, int iv);                        /* a3_gc_tree, Neumann sides */
int a5g3_average_dens(a5g3_ctx *ctx);                           /* :557-563 */
/* compute_fld (:309-345): rhs on the leaves, one FMG cycle (no_guess: from
 * phi = 0), fld_from_pot and the |E| ghost cells. */
int a5g3_compute_fld(a5g3_ctx *ctx, int no_guess);
/* mg3_fas_fmg / mg3_fas_vcycle (afivo/src/m_aX_mg.f90:164-255) on the
 * current rhs, with sides_bc_pot (:693-715) on the walls. */
int a5g3_fmg(a5g3_ctx *ctx, int set_residual, int first_call);
int a5g3_vcycle(a5g3_ctx *ctx, int max_lvl, int set_residual);
int a5g3_set_rhs(a5g3_ctx *ctx);
int a5g3_fld_from_pot(a5g3_ctx *ctx);                           /* :348-393 + gc */
/* a3_tree_max_cc / a3_tree_min_cc (afivo/src/m_aX_utils.f90:559-619) */
int a5g3_tree_max_cc(a5g3_ctx *ctx, int iv, double *out);
int a5g3_tree_min_cc(a5g3_ctx *ctx, int iv, double *out);
/* get_max_dt (src/streamer_3d.f90:274-305) and its three reductions. */
int a5g3_dt_reductions(a5g3_ctx *ctx, double *out3);
int a5g3_get_max_dt(a5g3_ctx *ctx, double *dt);
/* One time step at dt on the fixed mesh (:96-128): replayed from a CUDA
 * graph captured at the first call; dt is read from device memory, so one
 * graph serves every step. Asynchronous on the context's stream. */
int a5g3_step(a5g3_ctx *ctx, double dt);
/* Precision of the run's steps, as a5g_set_precision does in 2D: with
 * A5G_MIXED the fluxes, the update and their lookups run in FP32 (densities
 * scaled by 2^-40 inside the fluxes, accumulated in FP64), and every field
 * solve with a guess is a defect correction -- per pass the FP64 residual of
 * the leaves, an FP32 multigrid on the correction equation with homogeneous
 * wall values and the schedule sched (NULL: the reference's FMG, 2, 2,
 * n_cycle_base, one pass), and the FP64 accumulation of the potential. The
 * densities, potential, field and step-size reductions stay FP64. The first
 * call allocates 3 FP32 variables of the box capacity. A first solve (no
 * guess) stays FP64. */
int a5g3_set_precision(a5g3_ctx *ctx, int precision, const a5g_mg_schedule *sched);
int a5g3_get_precision(a5g3_ctx *ctx, int *precision, a5g_mg_schedule *sched);
int a5g3_sync(a5g3_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), for event timing. */
int a5g3_stream(a5g3_ctx *ctx, void **stream);

#ifdef __cplusplus
}
#endif

#endif /* A5G3_H */
