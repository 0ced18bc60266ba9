/* BRiDCT plan API, served by the B200 (sm_100a) CUDA library libbridct_b200.so.
 *
 * Drop-in for the reference's public header (include/bridct.h:1-55 of the reference):
 * same modes, status codes, opaque plan type and the same six exported functions with the
 * same argument meaning, validation order and return codes.  The declarations must match
 * the reference's byte for byte in meaning for callers to relink without change, so this
 * header keeps its names and values.  B200 extensions live in bridct_b200.h.
 *
 * Pointers passed to bridct_plan_apply / bridct_apply may be host memory (pageable or
 * pinned) or CUDA device/managed memory; the call returns when the output is written.
 */
#ifndef BRIDCT_H
#define BRIDCT_H

#include <stddef.h>

#if defined(__GNUC__)
#define BRIDCT_API __attribute__((visibility("default")))
#else
#define BRIDCT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define BRIDCT_VERSION "0.2.0-dev.7"

/* Reference include/bridct.h:24-28. */
enum bridct_mode {
    BRIDCT_FORWARD = 0,     /* Q_h X Q_w^T, orthonormal DCT-II  */
    BRIDCT_INVERSE = 1,     /* Q_h^T X Q_w, orthonormal DCT-III */
    BRIDCT_ROUNDTRIP = 2    /* Q_h^T Q_h X Q_w^T Q_w            */
};

/* Reference include/bridct.h:30-36; codes below -4 are B200 additions. */
enum bridct_status {
    BRIDCT_OK = 0,
    BRIDCT_INVALID_ARGUMENT = -1,
    BRIDCT_WORKSPACE_TOO_SMALL = -2,
    BRIDCT_BAD_ALIGNMENT = -3,
    BRIDCT_OVERLAPPING_BUFFERS = -4,
    BRIDCT_DEVICE_ERROR = -5,   /* a CUDA call failed; see bridct_last_error() */
    BRIDCT_TIMEOUT = -6         /* a bounded device-side wait expired */
};

typedef struct bridct_plan bridct_plan;

/* Replaces reference src/plan.c:33-37: 1 iff 8 <= h,w <= 1024, both powers of two. */
BRIDCT_API int bridct_supported(int height, int width);
/* Replaces src/plan.c:59-115: NULL for unsupported shapes or when no CUDA device/memory. */
BRIDCT_API bridct_plan *bridct_plan_create(int height, int width);
/* Replaces src/plan.c:49-57: NULL-safe. */
BRIDCT_API void bridct_plan_destroy(bridct_plan *plan);
/* Replaces src/plan.c:117-124: "paper8-square" (square <= 256) or "blocked-extension";
 * NULL for a NULL plan.  Static string. */
BRIDCT_API const char *bridct_plan_route(const bridct_plan *plan);
/* Replaces src/plan.c:126-163: NULL/mode -> INVALID_ARGUMENT, then overlap check
 * (|in - out| < h*w*4 bytes) -> OVERLAPPING_BUFFERS; nothing is written on error. */
BRIDCT_API int bridct_plan_apply(bridct_plan *plan, enum bridct_mode mode,
                                 const float *input, float *output);

/* Replaces src/bridct.c:13-21: scratch floats for squares 8..256, else 0. */
BRIDCT_API size_t bridct_workspace_floats(int size);
/* Replaces src/bridct.c:30-75: validation order invalid -> too small -> 16-byte alignment
 * of workspace -> pairwise overlap; then the square transform. */
BRIDCT_API int bridct_apply(int size, enum bridct_mode mode,
                            const float *input, float *output,
                            float *workspace, size_t workspace_count);

#ifdef __cplusplus
}
#endif
#endif
