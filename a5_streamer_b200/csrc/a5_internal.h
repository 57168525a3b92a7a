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
#endif
