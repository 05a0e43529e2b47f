/*
 * ffb200 — C ABI of the B200 flow-filter library (libffb200.so).
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and returns an
 * ff_status.  The C++ drop-in classes (include/flowfilter/gpu/*.h) and the Python
 * package sit on top of this ABI.  Each declaration names the reference interface
 * it replaces (file:line inside the reference project jadarve/optical-flow-filter).
 *
 * Conventions
 *   - images are row-major with an explicit row pitch in bytes; two-channel fields
 *     (flow, gradient) are interleaved float pairs (x, y) as in the reference;
 *   - uint8 images are read as v/255 (the reference's normalised texture reads);
 *   - `stream` is a cudaStream_t passed as void* (NULL = the legacy default stream);
 *   - device pointers must stay valid until the work queued on `stream` finishes;
 *   - functions ending in _async only enqueue work; the others block like the
 *     reference's stages, which synchronise the host at the end of compute()
 *     (src/gpu/pipeline.cu:72-82).
 *   - errors never exit the process (the reference calls exit(), src/gpu/error.cu:22);
 *     ff_last_error() returns a thread-local message for the last failure.
 */
#ifndef FFB200_H_
#define FFB200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef enum ff_status {
    FF_OK = 0,
    FF_ERR_INVALID_ARGUMENT = 1, /* reference: std::invalid_argument / bare std::exception on a bad value */
    FF_ERR_LOGIC = 2,            /* reference: std::logic_error (e.g. compute() on an unconfigured stage) */
    FF_ERR_OUT_OF_RANGE = 3,     /* level index out of bounds (flowfilter.cu:756-759) */
    FF_ERR_SHAPE = 4,            /* shapes do not match (src/gpu/image.cu:113-119) */
    FF_ERR_CUDA = 5,             /* a CUDA runtime call failed */
    FF_ERR_OUT_OF_MEMORY = 6,    /* device or host allocation failed */
    FF_ERR_UNSUPPORTED = 7       /* a valid request this build does not support */
} ff_status;

/* Host image view, ABI-identical to flowfilter::image_t (include/flowfilter/image.h:30-49). */
typedef struct ff_image {
    int height;
    int width;
    int depth;
    size_t pitch;     /* row pitch in bytes */
    size_t itemSize;  /* bytes per channel item: 1 (uint8) or 4 (float32) */
    void* data;
} ff_image;

typedef struct ff_filter ff_filter; /* opaque: a single-level, delta-level or pyramidal filter */

/* ------------------------------------------------------------ library */
const char* ff_last_error(void);
/* Opt-in log.  The reference prints to stdout and stderr (a "first load" line on the first
 * frame, flowfilter.cu:133; parameter errors); this library is silent unless a callback is
 * set.  FF_LOG_ERROR: the message of every failing call (also kept for ff_last_error);
 * FF_LOG_INFO: a batch (re)building its step graph.  The callback runs on the thread that
 * made the call, under no lock of the library; NULL switches the log off. */
typedef void (*ff_log_fn)(int level, const char* message, void* user);
enum { FF_LOG_ERROR = 0, FF_LOG_INFO = 1 };
ff_status ff_set_log_callback(ff_log_fn fn, void* user);
const char* ff_status_string(ff_status s);
/* Library version as an integer (major*10000 + minor*100 + patch). */
int ff_version(void);
/* Select the CUDA device used by filters created afterwards on this thread (the
 * reference pins device 0 in every Stage constructor, src/gpu/pipeline.cu:26). */
ff_status ff_set_device(int device);
/* Testing aid (fault injection on the host; no reference counterpart): the library's
 * device allocations succeed n more times, then the next one fails with
 * FF_ERR_OUT_OF_MEMORY before CUDA is called, as a failed cudaMalloc would (the reference
 * exits the process there, src/gpu/error.cu:22); the injection then switches itself off.
 * n < 0 switches it off.  Process-wide. */
ff_status ff_debug_fail_allocation_after(long long n);

/* ------------------------------------------------------------ device buffers
 * Replaces GPUImage allocate/upload/download/copyFrom/clear (src/gpu/image.cu:81-197). */
ff_status ff_malloc_pitch(void** dptr, size_t* pitch, size_t width_bytes, size_t height);
ff_status ff_free(void* dptr);
/* kind: 0 host->device, 1 device->host, 2 device->device (synchronous, 2D) */
ff_status ff_memcpy2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width_bytes,
                      size_t height, int kind);
ff_status ff_memset2d(void* dptr, size_t pitch, int value, size_t width_bytes, size_t height);

/* ------------------------------------------------------------ filters
 * FlowFilter(height, width, smoothIterations, maxflow, gamma) with an owned uint8
 * input image (src/gpu/flowfilter.cu:45-76); FlowFilter(h, w) is (h, w, 1, 1, 1). */
ff_status ff_filter_create(int height, int width, int smooth_iterations, float maxflow, float gamma,
                           ff_filter** out);
/* FlowFilter(GPUImage inputImage) over an external device image of item size 1 or 4
 * (src/gpu/flowfilter.cu:32-38, configure() :84-122): gamma 1 (unscaled), maxflow 1,
 * one smoothing iteration, border 3.  The image is read on every compute(). */
ff_status ff_filter_create_on_device_image(const void* image, size_t pitch, int item_size, int height,
                                           int width, ff_filter** out);
/* DeltaFlowFilter(GPUImage inputImage, GPUImage inputFlow) (src/gpu/flowfilter.cu:349-426):
 * a finer level that refines the external coarse flow field (height_c x width_c x 2 floats). */
ff_status ff_delta_filter_create(const void* image, size_t pitch, int item_size, int height, int width,
                                 const void* coarse_flow, size_t coarse_pitch, int height_c, int width_c,
                                 ff_filter** out);
/* PyramidalFlowFilter(height, width, levels) with an owned uint8 input (flowfilter.cu:631-682). */
ff_status ff_pyramidal_create(int height, int width, int levels, ff_filter** out);
ff_status ff_filter_destroy(ff_filter* f);

ff_status ff_filter_shape(const ff_filter* f, int* height, int* width, int* levels);
/* Kind of filter: 0 FlowFilter, 1 DeltaFlowFilter, 2 PyramidalFlowFilter. */
ff_status ff_filter_kind(const ff_filter* f, int* kind);
ff_status ff_filter_level_shape(const ff_filter* f, int level, int* height, int* width);

/* Parameters.  Level 0 is the finest level; single-level filters use level 0.
 * setGamma scales by 1/255^2 for uint8 inputs (flowfilter.cu:276-285, 559-568);
 * ff_filter_get_gamma returns the scaled value, as the reference's getGamma does. */
ff_status ff_filter_set_gamma(ff_filter* f, int level, float gamma);
ff_status ff_filter_get_gamma(const ff_filter* f, int level, float* gamma);
/* setMaxFlow: iterations = ceil(maxflow) (flowfilter.cu:293-296); pyramids halve the
 * value per level and give the top level maxflow/2^(L-1) (flowfilter.cu:849-866). */
ff_status ff_filter_set_max_flow(ff_filter* f, float maxflow);
ff_status ff_filter_get_max_flow(const ff_filter* f, float* maxflow);
ff_status ff_filter_set_smooth_iterations(ff_filter* f, int level, int iterations);
ff_status ff_filter_get_smooth_iterations(const ff_filter* f, int level, int* iterations);
/* Applies to every level (the reference's pyramid loop overruns, flowfilter.cu:873-875). */
ff_status ff_filter_set_propagation_border(ff_filter* f, int border);
ff_status ff_filter_get_propagation_border(const ff_filter* f, int* border);
ff_status ff_filter_get_propagation_iterations(const ff_filter* f, int level, int* iterations);

/* Kernel selection per level: 0 per-stage kernels, 1 the streaming fused per-level kernel
 * wherever it is instantiated, 2 automatic (default: the autotuned choice, else the
 * streaming kernel for levels of at least 200,000 pixels and the tile-fused kernel below),
 * 3 the tile-fused kernel wherever it fits in shared memory.  All modes give bit-identical
 * results. */
ff_status ff_filter_set_fused(ff_filter* f, int mode);

/* Replay the frame step from CUDA graphs (one per state buffer parity, captured on first
 * use and re-captured after any parameter change).  Off by default. */
ff_status ff_filter_set_graphs(ff_filter* f, int enabled);
/* Autotuner: on the current inputs, time each level's per-stage kernels, its streaming
 * fused kernel at several band heights and its tile-fused kernel at several tile shapes
 * (`repetitions` runs each); then, for pyramids, time whole frames over combinations of each
 * level's best choices (the levels share the GPU within a frame) from a snapshot of the state
 * that is restored afterwards, and keep the fastest combination, used while the mode is 2.
 * Needs one computed frame; results are unchanged because every candidate writes
 * bit-identical outputs.  Parameter changes reset it. */
ff_status ff_filter_autotune(ff_filter* f, int repetitions);
/* ff_filter_autotune with the device buffer `flush` overwritten before every timed frame of
 * the whole-frame stage (outside the timing), so that frames read their state from HBM as
 * in a measurement that flushes L2 between frames. */
ff_status ff_filter_autotune_flush(ff_filter* f, int repetitions, void* flush, size_t flush_bytes);
/* Read or set one level's kernel choice (path: -1 untuned, 0 per-stage, 1 streaming fused,
 * 2 tile-fused; band: rows of a streaming band or the tile-shape index, 0 automatic), e.g.
 * to reuse a saved autotuning result. */
ff_status ff_filter_get_level_tuning(const ff_filter* f, int level, int* path, int* band);
ff_status ff_filter_set_level_tuning(ff_filter* f, int level, int path, int band);
/* Human-readable summary of the tuned choice per level (NUL-terminated, truncated to len). */
ff_status ff_filter_tuning(const ff_filter* f, char* buf, size_t len);
/* Rows per warp band of the fused kernels (0 = chosen from the SM count). */
ff_status ff_filter_set_band(ff_filter* f, int rows);
/* Per-level kernel timing, in the spirit of Stage::elapsedTime (src/gpu/pipeline.cu:63-88)
 * but without host syncs: events are recorded around each level's kernels for the
 * next `max_frames` computes (0 disables; graphs are not used while recording).
 * ff_filter_level_kernel_ms waits for them and returns the summed milliseconds. */
ff_status ff_filter_set_profiling(ff_filter* f, int max_frames);
ff_status ff_filter_level_kernel_ms(ff_filter* f, int level, float* total_ms, int* frames);

/* Device time of one level's step in its current kernel configuration: the step is
 * captured as a CUDA graph and launched `reps` times on the filter's stream, each launch
 * bracketed by events; when `flush` is non-NULL, `flush_bytes` of it are overwritten
 * before every launch, outside the events (evicting the L2).  Re-running a step rewrites
 * bit-identical outputs; needs one computed frame.  *total_ms is the sum over launches. */
ff_status ff_filter_time_level(ff_filter* f, int level, int reps, void* flush, size_t flush_bytes, float* total_ms);

/* Stream used by the blocking calls (default: a non-blocking stream owned by the filter). */
ff_status ff_filter_set_stream(ff_filter* f, void* stream);

/* loadImage(image_t&) (flowfilter.cu:218-220, 728-731): synchronous host upload with
 * the caller's pitch; shape and item size must match (src/gpu/image.cu:96-120). */
ff_status ff_filter_load_image_host(ff_filter* f, const ff_image* image);
/* Enqueue a device-to-device copy of a frame into the filter's input buffer. */
ff_status ff_filter_load_image_device_async(ff_filter* f, const void* image, size_t pitch, void* stream);
/* Read the next frames directly from a caller-owned device image (no copy).  The
 * pointer must stay valid and unchanged until the compute that reads it completes. */
ff_status ff_filter_bind_image_device(ff_filter* f, const void* image, size_t pitch);

/* compute() (flowfilter.cu:125-153, 685-716): one frame; blocks until done and
 * records elapsedTime() in milliseconds. */
ff_status ff_filter_compute(ff_filter* f);
/* Enqueue one frame on `stream` without blocking (elapsed time not updated). */
ff_status ff_filter_compute_async(ff_filter* f, void* stream);
/* Phase API of FlowFilter / DeltaFlowFilter (flowfilter.cu:155-197, 460-503). */
/* Pipelined host processing (no reference counterpart; replaces the loadImage ->
 * compute -> downloadFlow loop of a host-fed caller): uploads `in` on a copy stream,
 * computes on `stream` (NULL = legacy default), downloads the smoothed level-0 flow into
 * `out` on a second copy stream, and returns without waiting, so the copies of one frame
 * overlap the computation of its neighbours.  `in` and `out` (pinned host memory for
 * overlap) must stay untouched until ff_filter_synchronize; results equal those of the
 * blocking loop.  Needs a filter that owns its input image. */
ff_status ff_filter_process_host_async(ff_filter* f, const ff_image* in, ff_image* out, void* stream);
ff_status ff_filter_synchronize(ff_filter* f);
ff_status ff_filter_compute_image_model(ff_filter* f);
ff_status ff_filter_compute_propagation(ff_filter* f);
ff_status ff_filter_compute_update(ff_filter* f);
ff_status ff_filter_elapsed_ms(const ff_filter* f, float* ms);
/* Checkpoint and resume (no counterpart in the reference, whose filter state lives only in
 * device buffers): the state of the latest frame as a host byte image of
 * ff_filter_state_bytes bytes.  It holds per level the smoothed flow, the old image, the
 * delta flow (delta levels) or the unsmoothed flow (top level), and whether the level has
 * seen a frame.  Importing it into a filter of the same kind and level sizes continues that
 * stream exactly; parameters (gamma, maxflow, ...) are not part of it.  Both calls wait for
 * the filter's queued work and must come between frames. */
ff_status ff_filter_state_bytes(const ff_filter* f, size_t* bytes);
ff_status ff_filter_export_state(ff_filter* f, void* host, size_t bytes);
ff_status ff_filter_import_state(ff_filter* f, const void* host, size_t bytes);

/* downloadFlow (flowfilter.cu:238-240, 734-741): level-0 smoothed flow, H x W x 2 floats. */
ff_status ff_filter_download_flow_host(ff_filter* f, ff_image* flow);
/* downloadImage (flowfilter.cu:242-244, 744-751): level-0 updated image (current a0). */
ff_status ff_filter_download_image_host(ff_filter* f, ff_image* image);
/* Device views of the current results, valid until the next compute on the filter.
 * which: 0 smoothed flow (downloadFlow), 1 getFlow() (unsmoothed for single-level
 * filters, flowfilter.cu:266-268; smoothed for delta and pyramidal filters,
 * :545-547, 718-725), 2 updated image. */
ff_status ff_filter_device_result(ff_filter* f, int which, void** dptr, size_t* pitch);
/* Copy any level's state to the host for inspection: which as above plus 3 = delta flow. */
ff_status ff_filter_level_state_host(ff_filter* f, int level, int which, void* dst, size_t dst_pitch);

/* ------------------------------------------------------------ stages
 * Stateless kernels over caller-owned device buffers (the stage classes of
 * src/gpu/{imagemodel,pyramid,propagation,update,flowsmoothing}.cu).  `ws` is a
 * caller-provided device workspace of at least the size the matching
 * *_workspace_size call returns (may be NULL when that size is 0). */

/* ImagePyramid level step (pyramid.cu:110-167, pyramid_k.cu:14-145): X pass then Y pass
 * of [1/4, 1/2, 1/4] at stride 2; uint8 results truncate (unsigned char)(255*s). */
ff_status ff_stage_pyramid_down(const void* in, size_t in_pitch, int item_size, int height, int width,
                                void* out, size_t out_pitch, void* stream);
/* ImageModel::compute (imagemodel.cu:93-113, imagemodel_k.cu:31-133): a0 (float) and
 * gradient (float pairs) from a uint8 or float image. */
ff_status ff_stage_image_model(const void* img, size_t img_pitch, int item_size, int height, int width,
                               float* a0, size_t a0_pitch, float* grad, size_t grad_pitch, void* stream);
/* FlowPropagator::compute (propagation.cu:80-134): `iterations` upwind sub-steps
 * (X then Y), dt = 1/iterations, pixels within `border` of the edge unchanged. */
size_t ff_stage_propagate_workspace_size(int height, int width);
ff_status ff_stage_propagate(const float* flow, size_t flow_pitch, int height, int width, int iterations,
                             int border, float* out, size_t out_pitch, void* ws, void* stream);
/* FlowPropagatorPayload::compute (propagation.cu:324-373): flow plus a scalar and a
 * vector payload advected with the flow's dominant velocity. */
size_t ff_stage_propagate_payload_workspace_size(int height, int width);
ff_status ff_stage_propagate_payload(const float* flow, size_t flow_pitch, const float* scalar,
                                     size_t scalar_pitch, const float* vector, size_t vector_pitch,
                                     int height, int width, int iterations, int border, float* out_flow,
                                     size_t out_flow_pitch, float* out_scalar, size_t out_scalar_pitch,
                                     float* out_vector, size_t out_vector_pitch, void* ws, void* stream);
/* FlowUpdate::compute (update.cu:97-116, update_k.cu:15-79). gamma is used as given. */
ff_status ff_stage_update(const float* a0, size_t a0_pitch, const float* grad, size_t grad_pitch,
                          const float* a0_old, size_t a0_old_pitch, const float* flow, size_t flow_pitch,
                          int height, int width, float gamma, float maxflow, float* out_flow,
                          size_t out_flow_pitch, float* out_image, size_t out_image_pitch, void* stream);
/* DeltaFlowUpdate::compute (update.cu:328-349, update_k.cu:82-173). */
ff_status ff_stage_delta_update(const float* a0, size_t a0_pitch, const float* grad, size_t grad_pitch,
                                const float* a0_old, size_t a0_old_pitch, const float* delta,
                                size_t delta_pitch, const float* coarse, size_t coarse_pitch, int height_c,
                                int width_c, int height, int width, float gamma, float maxflow,
                                float* out_flow, size_t out_flow_pitch, float* out_delta,
                                size_t out_delta_pitch, float* out_image, size_t out_image_pitch,
                                void* stream);
/* FlowSmoother::compute (flowsmoothing.cu:74-108): `iterations` x (5-tap box X, then Y). */
size_t ff_stage_smooth_workspace_size(int height, int width);
ff_status ff_stage_smooth(const float* flow, size_t flow_pitch, int height, int width, int iterations,
                          float* out, size_t out_pitch, void* ws, void* stream);
/* scalarProductF2_k (src/gpu/device/misc_k.cu:18-38): every float2 of a flow field times
 * `scalar` (FlowPropagator::setInvertInputFlow uses -1, propagation.cu:92-96). */
ff_status ff_stage_scale_flow(const float* flow, size_t flow_pitch, int height, int width, float scalar, float* out,
                              size_t out_pitch, void* stream);
/* ------------------------------------------------------------ batched streams
 * No counterpart in the reference: many independent PyramidalFlowFilter streams of
 * different sizes, levels and parameters advanced together.  Stream i's frame is read from
 * a packed uint8 device buffer at the offset ff_batch_frame_layout gives (rows of width
 * bytes, no padding); one step runs ff_batch_launches kernel launches (4 for up to 3 levels
 * per stream within the streaming kernel's iterations and smoothing passes: ingest with
 * pyramid, one streaming launch per phase, one tile launch), a
 * number that depends on neither the number of streams nor their parameters; every stream's
 * results equal those of the same stream filtered alone.  Each stream is an ff_filter owned by the batch (ff_batch_stream):
 * set its parameters and read its results with the ff_filter_* calls; do not destroy it. */
typedef struct ff_batch ff_batch;
ff_status ff_batch_create(int n, const int* heights, const int* widths, const int* levels, ff_batch** batch);
ff_status ff_batch_destroy(ff_batch* batch);
ff_status ff_batch_size(const ff_batch* batch, int* n);
ff_status ff_batch_stream(ff_batch* batch, int index, ff_filter** filter);
ff_status ff_batch_frame_layout(const ff_batch* batch, size_t* offsets, size_t* total_bytes);
ff_status ff_batch_launches(const ff_batch* batch, int* launches);
/* frames: 16-byte aligned device buffer of total_bytes; stream: cudaStream_t (NULL = legacy) */
ff_status ff_batch_step(ff_batch* batch, const void* frames, void* stream);
/* Kernel selection (optional; results do not depend on it): the levels that read the
 * previous frame's coarse flow or are top levels (phase A) run the tile-fused kernel below
 * min_pixels pixels (< 0: 200000), every other level the streaming level kernel covers runs
 * it, in bands of band rows (<= 0: the default rule).  Phase-B levels beyond the streaming
 * kernel (more than 4 iterations or smoothing passes) add a second tile launch. */
ff_status ff_batch_set_tuning(ff_batch* batch, long long min_pixels, int band);
/* Levels of height x width pixels run the streaming kernel in bands of band rows (band <= 0
 * removes the override): the per-size choice the batch autotuner makes.  Results do not
 * depend on it. */
ff_status ff_batch_set_level_band(ff_batch* batch, int height, int width, int band);

/* ------------------------------------------------------------ differentiable stages
 * No counterpart in the reference: the float-input filter's stages as forward and adjoint
 * kernels for training (flowfilter_b200.diff builds torch.autograd Functions on them).
 * dtype 0 = float32, 1 = float64; B images per call, dense [B][H][W] scalar and
 * [B][H][W][2] vector layouts; gamma and the 5 smoothing weights are device scalars of the
 * same dtype.  The float32 forward equals the stage kernels above (with weights 0.2, the
 * reference's box).  Backward calls ADD into their gradient outputs (zero them first) and
 * take the stage's forward inputs; the upwind, dominant-velocity and clamp branches follow
 * the forward (zero gradient through a clamped or sanitised value).  Stencil adjoints are
 * gathers (deterministic); the coarse-flow gradient of the delta update uses atomics. */
ff_status ff_diff_pyramid(int dtype, int B, int H, int W, const void* in, void* out, void* stream);
ff_status ff_diff_pyramid_bwd(int dtype, int B, int H, int W, const void* gout, void* gin, void* stream);
ff_status ff_diff_model(int dtype, int B, int H, int W, const void* img, void* a0, void* grad, void* stream);
/* gby, gbx: scratch of B*H*W elements each (overwritten) */
ff_status ff_diff_model_bwd(int dtype, int B, int H, int W, const void* ga0, const void* ggrad, void* gby, void* gbx,
                            void* gimg, void* stream);
/* one sub-step along axis (0 = X, 1 = Y); payload: also advect scalar s and vector v */
ff_status ff_diff_propagate(int dtype, int B, int H, int W, int axis, int payload, double dt, int border,
                            const void* f, const void* s, const void* v, void* fo, void* so, void* vo, void* stream);
ff_status ff_diff_propagate_bwd(int dtype, int B, int H, int W, int axis, int payload, double dt, int border,
                                const void* f, const void* s, const void* v, const void* gfo, const void* gso,
                                const void* gvo, void* gf, void* gs, void* gv, void* stream);
ff_status ff_diff_update(int dtype, int B, int H, int W, const void* a0, const void* grad, const void* old,
                         const void* fhat, const void* gamma, double maxflow, void* out, void* stream);
ff_status ff_diff_update_bwd(int dtype, int B, int H, int W, const void* a0, const void* grad, const void* old,
                             const void* fhat, const void* gamma, double maxflow, const void* gout, void* ga0,
                             void* ggrad, void* gold, void* gfhat, void* ggamma, void* stream);
ff_status ff_diff_delta_update(int dtype, int B, int H, int W, int Hc, int Wc, const void* a0, const void* grad,
                               const void* old, const void* dhat, const void* coarse, const void* gamma,
                               double maxflow, void* flow, void* delta, void* stream);
ff_status ff_diff_delta_update_bwd(int dtype, int B, int H, int W, int Hc, int Wc, const void* a0, const void* grad,
                                   const void* old, const void* dhat, const void* coarse, const void* gamma,
                                   double maxflow, const void* gflow, const void* gdelta, void* ga0, void* ggrad,
                                   void* gold, void* gdhat, void* gcoarse, void* ggamma, void* stream);
/* one weighted 5-tap pass along axis over a vector field (weights w5[0..4]) */
ff_status ff_diff_smooth(int dtype, int B, int H, int W, int axis, const void* w5, const void* in, void* out,
                         void* stream);
ff_status ff_diff_smooth_bwd(int dtype, int B, int H, int W, int axis, const void* w5, const void* in,
                             const void* gout, void* gin, void* gw5, void* stream);

/* Camera model and rotational image prediction (no scalar kernels of the filter use them).
 * ff_camera is the reference's perspectiveCamera (include/flowfilter/gpu/camera.h:18-23);
 * ff_camera_perspective is createPerspectiveCamera (src/gpu/camera.cu:15-31). */
typedef struct ff_camera {
    float alphaX, alphaY, centerX, centerY;
} ff_camera;
ff_status ff_camera_perspective(float focal, int height, int width, float sensor_height, float sensor_width,
                                ff_camera* cam);
/* rotationalOpticalFlow_k (src/gpu/device/rotation_k.cu:17-43): the image flow of a camera
 * rotating at (wx, wy, wz) rad/frame, into [height][width] float2 (device, flow_pitch). */
ff_status ff_rotational_flow(const ff_camera* cam, float wx, float wy, float wz, float* flow, size_t flow_pitch,
                             int height, int width, void* stream);
/* LaxWendroffPropagator::compute (src/gpu/propagation.cu:572-645): `iterations` times a Y
 * then an X Lax-Wendroff pass of an image [height][width][depth] float (depth 1 or 4) by the
 * flow [height][width] float2, dt = 1/iterations; iterations 0 (never set) runs one pass pair
 * with dt = 0, as the reference does.  All device buffers; rows 4-byte (depth 1) or 16-byte
 * (depth 4) aligned; `out` must not be `image`.  One launch covers up to
 * ff_lax_wendroff_max_fused() iterations; more need `workspace` (an image like `out`). */
int ff_lax_wendroff_max_fused(void);
ff_status ff_lax_wendroff(const float* flow, size_t flow_pitch, const float* image, size_t image_pitch, int depth,
                          int height, int width, int iterations, float* out, size_t out_pitch, float* workspace,
                          size_t workspace_pitch, void* stream);
/* RotationalFlowImagePredictor::compute (src/gpu/rotation.cu:72-88): the rotational flow
 * (written to `flow`) and the image propagated by it (`out`), in one launch up to
 * ff_lax_wendroff_max_fused() iterations.  Buffers as for ff_lax_wendroff. */
ff_status ff_rotational_predict(const ff_camera* cam, float wx, float wy, float wz, const float* image,
                                size_t image_pitch, int depth, int height, int width, int iterations, float* flow,
                                size_t flow_pitch, float* out, size_t out_pitch, float* workspace,
                                size_t workspace_pitch, void* stream);

/* FlowToColor::compute (src/gpu/display.cu:95-110, kernel src/gpu/device/display_k.cu:14-43):
 * colour-encodes a flow field [height][width] float2 (device, rows flow_pitch bytes apart,
 * 8-byte aligned) into RGBA [height][width] uchar4 (device, color_pitch).  Each component is
 * normalised to u = (f + maxflow) / (2 maxflow) and picks a column (x) and a row (y) of a
 * 256x256 RGBA colour wheel exactly as the reference's clamped, point-sampled texture read
 * does.  `wheel` is a dense device array of 256*256*4 bytes; NULL selects the library's
 * default wheel (ff_color_wheel_default), which the first such call on a device uploads,
 * synchronously (make it before any stream capture).  maxflow <= 0 is rejected as the
 * reference's setMaxFlow does (display.cu:129-137). */
ff_status ff_flow_to_color(const float* flow, size_t flow_pitch, int height, int width, float maxflow,
                           const unsigned char* wheel, unsigned char* color, size_t color_pitch, void* stream);
/* The library's default colour wheel into a host buffer of 256*256*4 bytes (rows of 256 RGBA
 * texels, row = y, column = x): the reference's embedded table (src/colorwheel.cpp,
 * COLOR_WHEEL_D, returned by getColorWheelRGBA, include/flowfilter/colorwheel.h:20-27), byte
 * for byte, so default colours are the reference's. */
ff_status ff_color_wheel_default(unsigned char* rgba);

/* One frame of the differentiable pyramidal filter, and its adjoint, as single calls that
 * launch every stage kernel (the schedule of PyramidalFlowFilter::compute on float input,
 * src/gpu/flowfilter.cu:685-716: pyramid, top level, then delta levels L-2 .. 0).  State per
 * level: smoothed flow [B][H][W][2], old image [B][H][W], delta flow [B][H][W][2] (3 pointers
 * per level, level 0 first; inputs and outputs must not overlap).  The forward writes the
 * new state and keeps every intermediate the adjoint needs in `tape`
 * (ff_diff_frame_tape_bytes); `fu_out` (optional) receives the top level's unsmoothed flow,
 * `y_out` (optional) a second copy of level 0's smoothed flow (an output of its own, so a
 * caller can route one gradient to the state and another to the frame's output).
 * The backward ADDS the gradients of the frame, gamma (L), weights (L x 5) and the input
 * state into its outputs; absent output gradients may be NULL; `grad_y` (optional) is the
 * gradient of y_out, image b at grad_y + b * grad_y_bstride elements (rows dense), summed
 * with the smoothed flow's; `scratch` is ff_diff_frame_scratch_bytes of device memory.
 * Sizes return 0 for a bad geometry. */
#define FF_DIFF_MAX_LEVELS 8
typedef struct ff_diff_geom {
    int batch, levels, border;
    int height[FF_DIFF_MAX_LEVELS], width[FF_DIFF_MAX_LEVELS];
    int iterations[FF_DIFF_MAX_LEVELS], smooth[FF_DIFF_MAX_LEVELS];
    double maxflow[FF_DIFF_MAX_LEVELS];
} ff_diff_geom;
size_t ff_diff_frame_tape_bytes(int dtype, const ff_diff_geom* geom);
size_t ff_diff_frame_scratch_bytes(int dtype, const ff_diff_geom* geom);
ff_status ff_diff_frame_forward(int dtype, const ff_diff_geom* geom, int first, const void* frame, const void* gamma,
                                const void* weights, const void* const* state_in, void* const* state_out,
                                void* fu_out, void* y_out, void* tape, void* stream);
/* The same frame forward without a tape, for inference: identical outputs, with the
 * intermediates in a reused `scratch` of ff_diff_frame_infer_bytes (a few fields per level
 * instead of every sub-step's).  No counterpart in the reference (no adjoint there). */
size_t ff_diff_frame_infer_bytes(int dtype, const ff_diff_geom* geom);
ff_status ff_diff_frame_infer(int dtype, const ff_diff_geom* geom, int first, const void* frame, const void* gamma,
                              const void* weights, const void* const* state_in, void* const* state_out, void* fu_out,
                              void* scratch, void* stream);
ff_status ff_diff_frame_backward(int dtype, const ff_diff_geom* geom, int first, const void* frame, const void* gamma,
                                 const void* weights, const void* const* state_in, const void* const* state_out,
                                 const void* tape, const void* const* grad_state_out, const void* grad_fu,
                                 const void* grad_y, long long grad_y_bstride, void* grad_frame, void* grad_gamma,
                                 void* grad_weights, void* const* grad_state_in, void* scratch, void* stream);

/* Mean endpoint error of flows (B, T, H, W, 2; dense) against truth over the frames
 * first..T-1: mean of sqrt(dx^2 + dy^2 + eps), written to the device scalar `loss`. truth has
 * the same pixel layout; element (b, t, y, x, c) lies at truth[b * truth_bstride + t *
 * truth_tstride + 2 (y W + x) + c] (truth_tstride 0: one truth frame for every t). `scratch`:
 * ff_diff_epe_scratch_bytes(dtype) bytes. Deterministic. ff_diff_epe_bwd writes the gradient
 * of every flow element for the upstream gradient *grad_loss (device scalar): d / |d| * g /
 * count for frames first.., zero before them and where |d| = 0. No counterpart in the
 * reference (the differentiable filter's training loss). */
size_t ff_diff_epe_scratch_bytes(int dtype);
ff_status ff_diff_epe(int dtype, int B, int T, int H, int W, int first, double eps, const void* flows,
                      const void* truth, long long truth_bstride, long long truth_tstride, void* loss, void* scratch,
                      void* stream);
ff_status ff_diff_epe_bwd(int dtype, int B, int T, int H, int W, int first, double eps, const void* flows,
                          const void* truth, long long truth_bstride, long long truth_tstride, const void* grad_loss,
                          void* grad_flows, void* stream);

/* ff_stage_smooth without a workspace and without any allocation. It has no counterpart
 * in the reference. The X-pass scratch is a 32 MiB static device array of the library, so
 * flows of up to 32 MiB of 512-byte-aligned float2 rows (2048x2048) are accepted; larger
 * ones fail with FF_ERR_INVALID_ARGUMENT. The array is device memory that every device
 * holds once the library's module is loaded there (at context creation under
 * CUDA_MODULE_LOADING=EAGER, else at the library's first launch on it), whether or not this
 * entry point is ever called, until the process exits or the device is reset. The scratch
 * needs no initial contents. It is one array per device: calls that overlap on one device
 * (two streams, or two threads) race on it; calls queued on one stream do not. Make each
 * device's first call, and the first after a cudaDeviceReset, outside stream capture: it
 * looks the array's address up once per device and context. For callers that may not
 * allocate: code running under a frame deadline, where cudaMalloc would synchronise the
 * device, and hosts whose memory belongs to their own allocator. */
ff_status ff_stage_smooth_noalloc(const float* flow, size_t flow_pitch, int height, int width, int iterations,
                                  float* out, size_t out_pitch, void* stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* FFB200_H_ */
