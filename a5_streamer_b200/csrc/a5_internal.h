// Internal helpers shared by the translation units of liba5g.so.
#ifndef A5_INTERNAL_H
#define A5_INTERNAL_H
#ifdef __cplusplus
extern "C" {
#endif
/* Record an error message for a5g_last_error() and return code. */
int a5g_internal_fail(int code, const char *msg);
#ifdef __cplusplus
}
#endif
#endif
