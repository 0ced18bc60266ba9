/* CPU oracle for the BRiDCT hot path: TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, float32 restatement of the reference's Shao-Johnson route, used by
 * tests/, __graft_entry__.smoke() and bench.py's CPU leg as the checker.  The
 * shipped library never links or calls it.
 */
#ifndef SJ_ORACLE_H
#define SJ_ORACLE_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Johnson-Frigo scale s(n,k) (src/plan.c:40-47). */
double oracle_sj_scale(int n, int k);
/* Scaled DCT-II core y[k] = C[k]/s(4n,k) (col_fN, src/generated/rect_generated.inc). */
void oracle_core_f(int n, const float *x, ptrdiff_t xs, float *y, ptrdiff_t ys);
/* Its transpose, the scaled DCT-III core (col_t*). */
void oracle_core_t(int n, const float *x, ptrdiff_t xs, float *y, ptrdiff_t ys);
/* Plan tables normalization[h*w] and correction[h*w] (src/plan.c:92-108). */
int oracle_plan_tables(int h, int w, float *norm, float *corr);
/* 2D transform of `batch` contiguous h*w arrays, mode 0/1/2 (src/generated/rect.c). */
int oracle_apply_batch(int h, int w, int mode, size_t batch, const float *x, float *y);

#ifdef __cplusplus
}
#endif
#endif
