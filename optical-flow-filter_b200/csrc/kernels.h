// Host-side launchers of the device kernels (stage_kernels.cu, level_kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace ffb {

// ---- per-stage kernels (stage_kernels.cu)
cudaError_t launch_pyramid_down(const void* in, size_t in_pitch, int item, int H, int W, void* out,
                                size_t out_pitch, cudaStream_t s);
// every float2 of an H x W field times k
cudaError_t launch_scale_flow(const float* in, size_t in_pitch, int H, int W, float k, float* out, size_t out_pitch,
                              cudaStream_t s);
// two pyramid steps (levels 1 and 2 of an H x W level 0) in one launch; needs a level 2
cudaError_t launch_pyramid_down2(const void* in, size_t in_pitch, int item, int H, int W, void* out1,
                                 size_t out1_pitch, void* out2, size_t out2_pitch, cudaStream_t s);
cudaError_t launch_image_model(const void* img, size_t pitch, int item, int H, int W, float* a0, size_t a0p,
                               float* grad, size_t gp, cudaStream_t s);
cudaError_t launch_propagate(const float* flow, size_t fp, int H, int W, int N, int border, float* out, size_t op,
                             float* tmp, size_t tp, cudaStream_t s);
cudaError_t launch_propagate_payload(const float* flow, size_t fp, const float* sc, size_t sp, const float* ve,
                                     size_t vp, int H, int W, int N, int border, float* of, size_t ofp, float* os,
                                     size_t osp, float* ov, size_t ovp, float* tf, size_t tfp, float* ts, size_t tsp,
                                     float* tv, size_t tvp, cudaStream_t s);
cudaError_t launch_update(const float* a0, size_t a0p, const float* grad, size_t gp, const float* old, size_t olp,
                          const float* flow, size_t fp, int H, int W, float gamma, float maxflow, float* of,
                          size_t ofp, float* oi, size_t oip, int first, cudaStream_t s);
cudaError_t launch_delta_update(const float* a0, size_t a0p, const float* grad, size_t gp, const float* old,
                                size_t olp, const float* delta, size_t dp, const float* coarse, size_t cp, int Hc,
                                int Wc, int H, int W, float gamma, float maxflow, float* of, size_t ofp, float* od,
                                size_t odp, float* oi, size_t oip, int first, cudaStream_t s);
cudaError_t launch_smooth(const float* flow, size_t fp, int H, int W, int S, float* out, size_t op, float* tmp,
                          size_t tp, cudaStream_t s);

// ---- fused per-level kernels (level_kernels.cu)
struct LevelArgs {
    int H, W;
    int item;            // input image item size (1 or 4)
    const void* img;     // level image
    size_t img_pitch;
    // state read (previous frame) and written (this frame)
    const float* fs_in;  size_t fs_in_pitch;   // smoothed flow (float2)
    const float* io_in;  size_t io_in_pitch;   // old image (float)
    const float* d_in;   size_t d_in_pitch;    // delta flow (float2), delta levels
    float* fs_out;       size_t fs_out_pitch;
    float* io_out;       size_t io_out_pitch;
    float* d_out;        size_t d_out_pitch;   // delta levels
    float* fu_out;       size_t fu_out_pitch;  // unsmoothed flow (float2), top levels; may be null
    // coarse flow (delta levels)
    const float* coarse; size_t coarse_pitch; int Hc, Wc;
    const int* coarse_rows;  // coarse row read by each row (upmap_index), H entries
    float gamma, maxflow;
    int border;
    int first;
    int band;            // rows per warp band (0: chosen from the SM count)
    // programmatic dependent launch (tile kernel): wait for the preceding kernel only before
    // the update (its stages before need nothing that kernel writes), and let the next
    // kernel's blocks start right after this kernel's own wait
    int pdl_late_wait;
    int pdl_early_trigger;
    // tile kernel of a two-level pyramid's top level: compute this level's image from the
    // finer image (the pyramid step) instead of reading it, and store the tile's pixels of
    // it to img (so every other reader still finds the level image); null otherwise
    const void* pyr_src; size_t pyr_src_pitch; int pyr_src_H, pyr_src_W;
};

// true if a fused kernel exists for this (delta, item, iterations, smoothing)
bool fused_available(bool delta, int item, int N, int S);
cudaError_t launch_fused_level(bool delta, int N, int S, const LevelArgs& a, cudaStream_t s);

// one level of a batched streaming launch (uint8 images): its arguments, its grid of
// nwx window columns x nby bands of `band` rows, and the first of its blocks
struct StreamJob {
    LevelArgs a;
    int nwx, nby, band;
    int first_block;
    int kind;  // stream_kind(delta, N, S): the instantiation the phase kernel runs
};
// the warp grid of a level of W x H pixels cut into bands of `band` rows; returns the
// blocks it takes
int fused_warp_grid(int N, int S, int W, int H, int band, int* nwx, int* nby);
// warps of the streaming kernel resident on the current device at once
int fused_resident_warps();
// one launch over jobs of any (delta, N, S) (level_mega.cu): StreamJob::kind selects each
// job's instantiation; smem = the largest stream_block_smem of the jobs
int stream_kind(bool delta, int N, int S);
int stream_block_smem(bool delta, int S);
cudaError_t launch_stream_mega(const StreamJob* jobs, int n, int blocks, int smem, cudaStream_t s);

// ---- tile-fused per-level kernels (tile_level.cu); cfg 0 = automatic tile shape
int tile_config_count();
bool tile_available(bool delta, int N, int S, int W, int H, int cfg);
void tile_shape(bool delta, int N, int S, int W, int H, int cfg, int* tw, int* th);
cudaError_t launch_tile_level(bool delta, int N, int S, const LevelArgs& a, int cfg, cudaStream_t s);

}  // namespace ffb
