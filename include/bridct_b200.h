/* B200 extensions of the BRiDCT plan API (libbridct_b200.so).
 *
 * The reference has no counterpart for these entry points: it transforms one host array
 * per call (include/bridct.h:44-45).  They let callers keep data in HBM, batch thousands of
 * arrays per launch, choose the tensor-core precision forms, and run mixed-shape (ragged)
 * batches in one persistent launch.  All return the status codes of bridct.h.
 */
#ifndef BRIDCT_B200_H
#define BRIDCT_B200_H

#include "bridct.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Execution form of a transform. */
enum bridct_form {
    BRIDCT_FORM_SJ = 0,        /* FP32 Shao-Johnson CUDA-core kernels (the plan API's form); all shapes */
    BRIDCT_FORM_TC_BF16X3 = 1, /* tensor cores: 3-term bf16 split of X, 6 products, FP32 accumulation;
                                  all shapes (8x8 as one Kronecker GEMM, the rest as two row passes) */
    BRIDCT_FORM_TC_TF32X3 = 2, /* tensor cores: 2-term tf32 split of X and C, 3 products; all shapes */
    BRIDCT_FORM_TC_FP8 = 3     /* FP8 E4M3, per-tile scales (32x32, or the array's axis where
                                  shorter), + one FP32 refinement step; all shapes */
};

/* Thread-local description of the last failure in this thread ("" if none). */
BRIDCT_API const char *bridct_last_error(void);

/* GPU schedule of the plan: "sj-tile" (both passes in shared memory) or
 * "sj-two-pass" (column pass then row pass).  NULL for a NULL plan. */
BRIDCT_API const char *bridct_plan_gpu_route(const bridct_plan *plan);

/* `batch` contiguous h*w arrays; host (pageable or pinned) or device pointers.
 * Synchronous.  Host buffers are streamed through the plan's device staging in
 * chunks (H2D, kernel, D2H overlapped on two streams); the first host-pointer call
 * allocates that staging.  Overlap of the two batch ranges -> OVERLAPPING_BUFFERS. */
BRIDCT_API int bridct_plan_apply_batch(bridct_plan *plan, enum bridct_mode mode,
                                       const float *input, float *output, size_t batch);

/* Round trip of `batch` arrays as a FORWARD call followed by an INVERSE call, with the float32
 * spectrum materialized in the plan's device staging instead of the caller's memory: the result
 * is bitwise that of the two calls (the NumPy Plan's round trip, python/bridct_numpy.c:119-123
 * of the reference), but a host batch crosses PCIe once each way.  Host or device pointers;
 * synchronous.  No reference counterpart. */
BRIDCT_API int bridct_plan_roundtrip_batch(bridct_plan *plan, const float *input, float *output,
                                           size_t batch);

/* Device-resident batch: input/output are CUDA device (or managed) pointers to
 * batch*h*w floats, 16-byte aligned, on the plan's device.  Asynchronous on `stream` (a
 * cudaStream_t of that device; NULL is the CUDA default stream).  The launch runs on the plan's
 * device whatever device is current, and the caller's current device is left as it was.  No
 * allocation, no host synchronisation. */
BRIDCT_API int bridct_plan_apply_device(bridct_plan *plan, enum bridct_mode mode,
                                        const float *input, float *output, size_t batch,
                                        void *stream);

/* Device-resident strided batch (plain form): element (r, c) of array b is read at
 * input[b * input_array_stride + r * input_row_pitch + c] and written at the same place of output
 * with the output's pitch and stride (all in floats).  Sub-images, tensor slices and arrays side by
 * side in a wider image transform where they lie, with no copy.  Pitches and strides must be
 * multiples of 4 floats and the pointers 16-byte aligned (else BRIDCT_BAD_ALIGNMENT); a pitch below
 * the width or arrays that overlap -> BRIDCT_INVALID_ARGUMENT; input and output extents that
 * overlap -> BRIDCT_OVERLAPPING_BUFFERS.  Asynchronous on `stream`, on the plan's device, no
 * allocation.  The reference accepts contiguous arrays only (docs/API.md:17). */
BRIDCT_API int bridct_plan_apply_strided_device(bridct_plan *plan, enum bridct_mode mode,
                                                const float *input, size_t input_row_pitch,
                                                size_t input_array_stride, float *output,
                                                size_t output_row_pitch, size_t output_array_stride,
                                                size_t batch, void *stream);

/* As bridct_plan_apply_device, with an explicit execution form (precision forms run
 * on the tensor cores; see enum bridct_form for the shapes each form supports).  The
 * two-pass tensor-core forms and the FP8 form keep their intermediate in scratch
 * owned by the plan (allocated by the first call that needs it, so make that call before any
 * stream capture): calls on one plan must not run concurrently on different streams.  The
 * scratch holds one chunk of the batch and grows with the largest batch a plan has seen: up
 * to 1 GB for BF16x3/TF32x3, about 17 bytes per element of up to 256 MB of input for FP8. */
BRIDCT_API int bridct_plan_apply_form_device(bridct_plan *plan, enum bridct_mode mode,
                                             enum bridct_form form, const float *input,
                                             float *output, size_t batch, void *stream);

/* Bytes of scratch a form needs for `batch` arrays of the plan's shape when the caller supplies
 * it (0: the form needs none).  No reference counterpart. */
BRIDCT_API size_t bridct_plan_form_workspace_bytes(const bridct_plan *plan, enum bridct_form form,
                                                   size_t batch);

/* As bridct_plan_apply_form_device, with the intermediate in a caller-owned device workspace
 * (16-byte aligned, at least bridct_plan_form_workspace_bytes bytes; too small ->
 * BRIDCT_WORKSPACE_TOO_SMALL).  The plan's own scratch is not touched, so calls on one plan may
 * run on several streams at once, each with its own workspace; a caching allocator that orders
 * its blocks by stream (PyTorch's) can supply it.  No reference counterpart. */
BRIDCT_API int bridct_plan_apply_form_device_ws(bridct_plan *plan, enum bridct_mode mode,
                                                enum bridct_form form, const float *input,
                                                float *output, size_t batch, void *workspace,
                                                size_t workspace_bytes, void *stream);

/* Reads and clears the bounded-wait flag of a device: nonzero when a tensor-core kernel's
 * mbarrier wait expired (the kernel then skipped its remaining tiles and returned). */
BRIDCT_API int bridct_device_timeout_flag(int device);

/* ---- Block transform of an image in place-layout (codec step) ------------------------- */

/* Transforms every 8x8 block of a height x width float32 image where it lies (row pitches in
 * floats, multiples of 4; 16-byte aligned device pointers; output may equal input with the
 * same pitch).  quant: NULL, or 64 positive quantization steps in host memory (row-major 8x8):
 * FORWARD then writes rint(Y / Q), INVERSE multiplies its input by Q before the DCT-III, and
 * ROUNDTRIP quantizes and dequantizes between the two.  Asynchronous on `stream` (NULL = CUDA
 * default stream); allocates nothing.  The reference has no strided or in-image entry point
 * (docs/API.md:17 requires contiguous arrays): callers there copy each block out and back. */
BRIDCT_API int bridct_image_blocks8_device(int mode, const float *input, size_t input_pitch,
                                           float *output, size_t output_pitch, int height, int width,
                                           const float *quant, void *stream);

/* ---- Batching form: mixed shapes and directions in one persistent launch ---------------- */

/* One array of a ragged batch: shape, mode (enum bridct_mode) and offset, in floats, from the
 * batch base pointers (a multiple of 4, so every array is 16-byte aligned). */
typedef struct {
    int height, width, mode, reserved;
    size_t offset;
} bridct_ragged_item;

/* Work-unit geometry of a ragged batch (chosen per shape class by the autotuner). */
typedef struct {
    int tile_floats;   /* arrays up to this many floats run both passes in one unit (<= 16384) */
    int strip_floats;  /* floats per column-strip unit of a larger array (<= 16384)            */
    int row_floats;    /* floats per row-block unit of a larger array (<= 16384)               */
    int lookahead;     /* larger arrays whose strips are queued ahead of a row pass (1..64)   */
} bridct_ragged_tuning;

typedef struct bridct_ragged bridct_ragged;

/* Fills the library default: units of up to 16384 floats and a look-ahead of 32 arrays (the
 * fastest measured on a mixed batch of all 64 shapes, apart from look-ahead 64, which was 0.6%
 * faster). */
BRIDCT_API void bridct_ragged_default_tuning(bridct_ragged_tuning *tuning);
/* Validates the items (supported shapes and modes, aligned, non-overlapping) and builds the
 * device work queue; NULL on error (see bridct_last_error). */
BRIDCT_API bridct_ragged *bridct_ragged_create(const bridct_ragged_item *items, size_t count);
BRIDCT_API bridct_ragged *bridct_ragged_create_tuned(const bridct_ragged_item *items, size_t count,
                                                     const bridct_ragged_tuning *tuning);
BRIDCT_API void bridct_ragged_destroy(bridct_ragged *batch);
BRIDCT_API size_t bridct_ragged_units(const bridct_ragged *batch);
/* Runs the whole batch (device pointers, asynchronous on `stream`, capturable in a CUDA graph):
 * the arrays of classes scheduled BRIDCT_RAGGED_QUEUE in one persistent launch (a counter reset and
 * one kernel), and every other class as its own launch on side streams forked from `stream` and
 * joined back into it.  A new batch schedules every class on the queue. */
BRIDCT_API int bridct_ragged_apply_device(bridct_ragged *batch, const float *input, float *output,
                                          void *stream);

/* ---- Per-shape-class schedules of a ragged batch ----------------------------------------------
 * The batch's arrays fall into shape classes (height, width, mode), numbered largest first (by
 * elements).  Each class runs either in the shared persistent queue, or as its own launch of the
 * fixed-shape kernels of that shape over the class's offset table, with the tile shapes measured
 * best for that shape, or with the few-array geometry (one four-step line group per warp).  The
 * autotuner (bridct_b200.autotune) measures the choices per class.  No reference counterpart: the
 * reference picks a per-(h, w, mode) policy from a table (src/generated/rect_policy.inc,
 * src/plan.c:140-148). */
enum bridct_ragged_schedule {
    BRIDCT_RAGGED_QUEUE = 0,               /* units in the persistent kernel's queue           */
    BRIDCT_RAGGED_CLASS_LAUNCH = 1,        /* the class's own fixed-shape launch               */
    BRIDCT_RAGGED_CLASS_LAUNCH_SMALL = 2,  /* the same with the few-array geometry (two-pass)  */
    BRIDCT_RAGGED_MERGED = 3               /* two-pass classes only: one column-pass launch per
                                              (column length, mode) and one row-pass launch per
                                              (row length, mode) over all MERGED classes      */
};
BRIDCT_API size_t bridct_ragged_class_count(const bridct_ragged *batch);
/* Kernel launches of one bridct_ragged_apply_device call with the current schedule: the merged
 * passes, one or two per class with its own launches, and the persistent queue kernel when any
 * class is queued. */
BRIDCT_API size_t bridct_ragged_launch_count(const bridct_ragged *batch);
/* Shape, mode, array count and schedule of class `cls` (any output pointer may be NULL). */
BRIDCT_API int bridct_ragged_class_info(const bridct_ragged *batch, size_t cls, int *height, int *width,
                                        int *mode, size_t *arrays, int *schedule);
/* Sets every class's schedule (count = bridct_ragged_class_count) and the number of side streams
 * (1..8) that own launches spread over.  Rebuilds the queue: synchronizes the device and may
 * allocate, so call it outside stream capture and before capturing the batch's launches. */
BRIDCT_API int bridct_ragged_set_schedule(bridct_ragged *batch, const int *schedules, size_t count,
                                          int streams);
/* One class alone as its own launch (schedule CLASS_LAUNCH or CLASS_LAUNCH_SMALL), for measuring. */
BRIDCT_API int bridct_ragged_apply_class_device(bridct_ragged *batch, size_t cls, int schedule,
                                                const float *input, float *output, void *stream);
/* The same batch as one plain-form launch per array (the comparison baseline). */
BRIDCT_API int bridct_ragged_apply_loop_device(bridct_ragged *batch, const float *input,
                                               float *output, void *stream);
/* Reads and clears the batch's bounded-wait flag (nonzero: a dependency wait expired). */
BRIDCT_API int bridct_ragged_timeout_flag(bridct_ragged *batch);
/* Sets how many times (about 256 ns apart) a row block polls for its array's column strips
 * before it gives up, skips its rows and raises the batch's timeout flag; the default is
 * 2^22 (about a second).  0 makes every row block give up at once, which tests use to drive the
 * timeout path deterministically.  No reference counterpart. */
BRIDCT_API int bridct_ragged_set_wait_limit(bridct_ragged *batch, unsigned polls);

/* No counterpart in the reference.  The ragged batch for callers that cannot let a library
 * allocate device memory (a framework whose caching allocator owns the whole GPU, a loop that
 * cannot afford cudaMalloc's implicit synchronisation, a fixed device footprint): the items and
 * the input/output buffers are passed in, and the work queue, counters and tables live in one
 * static device array of about 0.9 MB that every GPU loading this library holds until exit.
 * Limits: at most 4096 arrays and 49152 work units per call (default unit geometry), else
 * BRIDCT_INVALID_ARGUMENT with a message.  A successful call allocates nothing.  The first call
 * on a device resolves that array's address and uploads the four-step tables into it.  Every
 * call shares the array and overwrites the previous call's queue; calls are serialized and
 * synchronous (they return after their kernel finished), because two calls overlapping on the
 * GPU would race on it.  Returns BRIDCT_TIMEOUT if a bounded dependency wait expired. */
BRIDCT_API int bridct_ragged_apply_noalloc(const bridct_ragged_item *items, size_t count,
                                           const float *input, float *output, void *stream);

/* Waits for all work queued on the plan's own stream. */
BRIDCT_API int bridct_plan_synchronize(bridct_plan *plan);

#ifdef __cplusplus
}
#endif
#endif
