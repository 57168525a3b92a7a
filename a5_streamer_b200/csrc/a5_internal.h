// Internal helpers shared by the translation units of liba5g.so.
#ifndef A5_INTERNAL_H
#define A5_INTERNAL_H
#ifdef __cplusplus
extern "C" {
#endif
/* Record an error message for a5g_last_error() and return code. */
int a5g_internal_fail(int code, const char *msg);
/* Diagnostics: shared-memory doubles per multigrid variable, dynamic shared
 * memory per launch, capacity, levels, device limit, boxes, and for the mixed
 * form the floats per staged FP32 array and the dynamic shared memory. */
struct a5g_ctx;
int a5g_debug_info(struct a5g_ctx *ctx, long long *out8);
#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
#include <vector>
// Host copy of a run's topology as last uploaded (a5g_upload_tree): per id
// 0..max_id the 16 ints and 4 doubles of the upload format, and per level
// index (level - min_lvl) the ids, leaves and parents lists.
struct A5Topo {
  int max_id = 0, min_lvl = 0, max_lvl = 0;
  std::vector<int> meta16;
  std::vector<double> geom4;
  std::vector<std::vector<int>> ids, leaves, parents;
};
// Device storage and the settings of a run that other translation units
// (the adjoint) work on.
struct A5View {
  void *stream;            // cudaStream_t of the run
  double *cc, *fx, *fy;    // cell / face slots, layout of include/a5g.h
  int capacity;            // slots per variable
  int coord, n_cycle_base, precision, photoi_enabled, n_cta, has_lsf, has_table;
  double applied_fld, domain_len_z, epsilon_diel;
  int tbl_rows, tbl_cols;
  double tbl_xmin, tbl_inv_dx;
  const double *tbl_host;  // rows_cols as set (column-major)
  const A5Topo *topo;
};
extern "C" int a5g_internal_view(struct a5g_ctx *ctx, A5View *out);
#endif
#endif
