/*
 * CPU ORACLE for the flow-filter hot path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement of the reference's per-pixel kernels and per-frame
 * schedule, used by tests/ (as the checker), by __graft_entry__.smoke() and by the
 * CPU-baseline leg of bench.py.  The product never links or calls it.
 *
 * Buffers are dense row-major (no pitch): images H*W, two-channel fields H*W*2
 * interleaved (x, y).  Each function cites the reference code it restates.
 *
 * Floating-point contraction: the reference is compiled by nvcc with FMA
 * contraction on (its default).  Which multiply-add pairs fuse is fixed here by
 * explicit std::fma calls, selected by or_set_variant(), and pinned against
 * outputs of the reference library itself (tests/golden/ref_stages.npz).
 */
#ifndef FF_ORACLE_H_
#define FF_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* contraction / sampling variants (see oracle.cpp for the meaning of each key) */
enum or_variant_key {
    OR_V_MODEL_FMA = 0,     /* image model tap chains fused (1) or mul+add (0) */
    OR_V_PROP_FMA = 1,      /* propagation f - t*d fused (1) or not (0) */
    OR_V_UPD_NFMA = 2,      /* gamma + a^2 fused (1) or not (0) */
    OR_V_UPD_Q = 3,         /* q = g*f + a*Yt: 0 fma(g,f,a*Yt), 1 fma(a,Yt,g*f), 2 none */
    OR_V_UPD_OX = 4,        /* N00*qx + N01*qy: 0 fma(N00,qx,.), 1 fma(N01,qy,.), 2 none */
    OR_V_UPD_OY = 5,        /* N10*qx + N11*qy: 0 fma(N10,qx,.), 1 fma(N11,qy,.), 2 none */
    OR_V_SMOOTH_FMA = 6,    /* smoothing tap chain fused (1) or not (0) */
    OR_V_UPMAP = 7,         /* coarse index: 0 floor(u*Wc) in float */
    OR_V_ROT = 8,           /* rotational flow contraction bits, see or_rotational_flow */
    OR_V_LW = 9,            /* Lax-Wendroff contraction bits, see or_lax_wendroff */
    OR_V_COUNT = 10
};

void or_set_variant(int key, int value);
int or_get_variant(int key);
/* u8 -> float conversion of a normalised texture read, 256 entries (default v/255.f) */
void or_set_norm_table(const float* table256);
void or_get_norm_table(float* table256);
/* 0 or 1 = single-threaded, otherwise the number of host threads for the stage loops */
void or_set_threads(int n);

/* ---- rotational flow and Lax-Wendroff propagation (src/gpu/camera.cu:15-31,
 * src/gpu/device/rotation_k.cu:17-43, src/gpu/rotation.cu:72-88,
 * include/flowfilter/gpu/device/propagation_k.h:49-132, src/gpu/propagation.cu:572-645) ---- */
/* cam4 = {alphaX, alphaY, centerX, centerY} */
void or_camera_perspective(float focal, int H, int W, float sensorH, float sensorW, float* cam4);
void or_rotational_flow(const float* cam4, float wx, float wy, float wz, int H, int W, float* flow);
/* image [H][W][depth] (depth 1 or 4); iterations <= 0 runs one pass pair with dt = 0 */
void or_lax_wendroff(const float* flow, const float* image, int depth, int H, int W, int iterations, float* out);

/* ---- stages (reference: src/gpu/device/*.cu) ---- */
void or_pyramid_down_u8(const uint8_t* in, int H, int W, uint8_t* out);
void or_pyramid_down_f32(const float* in, int H, int W, float* out);
void or_image_model(const void* img, int item_size, int H, int W, float* a0, float* grad);
void or_propagate(const float* flow, int H, int W, int N, int border, float* out);
void or_propagate_payload(const float* flow, const float* scalar, const float* vector,
                          int H, int W, int N, int border,
                          float* oflow, float* oscalar, float* ovector);
void or_update(const float* a0, const float* grad, const float* a0old, const float* flow,
               int H, int W, float gamma, float maxflow, float* oflow, float* oimage);
void or_delta_update(const float* a0, const float* grad, const float* a0old, const float* delta,
                     const float* coarse, int Hc, int Wc, int H, int W, float gamma,
                     float maxflow, float* oflow, float* odelta, float* oimage);
void or_smooth(const float* flow, int H, int W, int S, float* out);
/* coarse index used by the delta update for output coordinate x of an axis of size W */
int or_upmap_index(int x, int W, int Wc);

/* ---- filters (reference: src/gpu/flowfilter.cu) ---- */
typedef struct or_filter or_filter;
/* FlowFilter(h, w, smoothIterations, maxflow, gamma) with uint8 input, flowfilter.cu:45-76 */
or_filter* or_flowfilter_create(int H, int W, int smooth, float maxflow, float gamma);
/* FlowFilter(GPUImage) on an input of item size 1 or 4: configure() defaults, flowfilter.cu:32-38 */
or_filter* or_flowfilter_create_on(int H, int W, int item_size);
/* PyramidalFlowFilter(h, w, levels), uint8 input, flowfilter.cu:631-682 */
or_filter* or_pyramidal_create(int H, int W, int levels);
void or_filter_destroy(or_filter* f);
int or_filter_levels(const or_filter* f);
int or_filter_set_gamma(or_filter* f, int level, float gamma);
float or_filter_get_gamma(const or_filter* f, int level);
int or_filter_set_max_flow(or_filter* f, float maxflow);
float or_filter_get_max_flow(const or_filter* f);
int or_filter_set_smooth_iterations(or_filter* f, int level, int n);
int or_filter_get_smooth_iterations(const or_filter* f, int level);
int or_filter_set_propagation_border(or_filter* f, int border);
int or_filter_get_propagation_iterations(const or_filter* f, int level);
void or_filter_load(or_filter* f, const void* img);
void or_filter_compute(or_filter* f);
/* downloadFlow(): smoothed flow of level 0 (flowfilter.cu:238-240, 734-741) */
void or_filter_download_flow(const or_filter* f, float* out);
/* getFlow(): unsmoothed for a single level (flowfilter.cu:266-268), smoothed for pyramids */
void or_filter_get_flow(const or_filter* f, float* out);
/* downloadImage(): level-0 updated image = current a0 (flowfilter.cu:242-244, 744-751) */
void or_filter_download_image(const or_filter* f, float* out);
/* per-level state, for white-box comparisons: which = 0 smoothed flow, 1 unsmoothed flow,
   2 updated image, 3 updated delta flow (delta levels only).  Returns element count. */
size_t or_filter_level_state(const or_filter* f, int level, int which, float* out);
void or_filter_level_shape(const or_filter* f, int level, int* H, int* W);

#ifdef __cplusplus
}
#endif
#endif
