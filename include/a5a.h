/*
 * a5a — adjoint of the fixed-mesh streamer program on the device (sm_100a):
 * gradients of a streamer-head observable with respect to the transport
 * table and the applied voltage, for one run of include/a5g.h.
 *
 * The reference has no adjoint. The program it differentiates is the
 * reference's own time step, src/streamer_2d.f90:93-128, repeated on a mesh
 * that does not change:
 *   1. the run's state when a5a_create is called is the initial state (call
 *      it after set_init_cond, e.g. a5s_set_init_cond: seed densities and
 *      phi = 0);
 *   2. compute_fld with no guess (src/streamer_2d.f90:307-343, the first
 *      FAS FMG call of afivo/src/m_aX_mg.f90:163-202);
 *   3. n_steps full time steps at the step sizes dts[] (no regrid, no
 *      photoionization);
 *   4. J = head height: over the leaf cells next to the line x = x0, the
 *      mean of the cell heights y weighted by dy * exp((|E| - max |E|) / T).
 * The gradient is that of this discrete program: the adjoint of every linear
 * operation (copies, restriction, consistent fluxes, space charge, the whole
 * FAS multigrid with its ghost recipes, the field's faces and ghost cells,
 * the trapezoidal average) is its exact transpose, and the nonlinear ones
 * (fluxes_koren with its limiter, upwinding and clamp; update_solution's
 * source norm; the cell |E|; gc_interp_lim) have hand-written adjoint
 * kernels. States are stored every checkpoint_every steps on the first
 * forward pass; the reverse pass recomputes each interval from its stored
 * state.
 *
 * Supported runs: Cartesian, FP64, no dielectric, no level set, no
 * photoionization (others are rejected with A5G_EINVAL).
 */
#ifndef A5A_H
#define A5A_H

#include "a5g.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct a5a_ctx a5a_ctx;

typedef struct a5a_params {
  int n_steps;           /* time steps of the program (>= 1) */
  int checkpoint_every;  /* steps between stored states (>= 1) */
  double x0;             /* the line x = x0 of the head profile (m) */
  double temperature;    /* softmax temperature T of the observable (V/m, > 0) */
} a5a_params;

/* Bind an adjoint to a run whose current tree is the fixed mesh and whose
 * current state is the program's initial state (copied here). dts holds
 * n_steps step sizes. Allocates all device storage the gradient needs:
 * (n_steps / checkpoint_every + 2) stored states and checkpoint_every steps
 * of intermediate fields. The run must not be regridded while bound. */
int a5a_create(a5g_ctx *run, const a5a_params *p, const double *dts, a5a_ctx **out);
int a5a_destroy(a5a_ctx *a);

/* Run the program with the run's current table (a5g_set_table) and applied
 * field (a5g_set_applied_field); J is the observable. The run is left in the
 * program's end state. */
int a5a_forward(a5a_ctx *a, double *J);

/* Forward pass with stored states, then the reverse pass. Writes J,
 * dJ_dtable (n_rows x 4, column-major like a5g_set_table's rows_cols: the
 * derivative with respect to every table entry) and dJ_dV (with respect to
 * the applied voltage, -domain_len_z * applied_fld). The run is left in the
 * program's end state. */
int a5a_gradient(a5a_ctx *a, double *J, double *dJ_dtable, double *dJ_dV);

/* The transposed linear phases the reverse pass applies, built on the host
 * from a topology in a5g_upload_tree's format (no GPU needed). seg selects
 * one operation: 0 old-density copies, 1 consistent fluxes, 2 restriction of
 * n_e and n_i, 3 space charge, 4 FAS FMG with a guess, 5 FAS FMG without
 * (first call), 6 field faces, 7 field ghost cells, 8 trapezoidal average.
 * Entries index one vector: cell variable iv of box id, cell (i, j) at
 * (iv * capacity + id) * (nc0+2)^2 + i + (nc+2) j with nc0 = box_size
 * (include/a5g.h slot layout); face variable f of direction d at
 * C + (d * 2 + f) * capacity * (nc0+1) nc0 + slot offset, C = 9 capacity
 * (nc0+2)^2; the applied voltage last. A phase writes rows d with
 * new x[d] = self * x[d] + sum_t c_t x[s_t] (all reads before writes).
 * sizes: n_phase, n_rows, n_terms, vector length. Arrays may be null to
 * query sizes. */
int a5a_debug_tape(int max_id, int min_lvl, int max_lvl, const int *meta16, const double *geom4,
                   const int *lvl_counts, const int *lvl_ids, int capacity, int n_cycle_base,
                   int seg, long long *sizes, int *phase_row, unsigned *row_d, double *row_self,
                   int *row_term, unsigned *term_s, double *term_c);

#ifdef __cplusplus
}
#endif
#endif
