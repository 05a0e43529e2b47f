// Host-side filter objects behind the C ABI (capi.cu).
//
// One Filter covers the reference's three composites (src/gpu/flowfilter.cu):
//   FlowFilter          one "top" level on an owned uint8 image or an external image
//   DeltaFlowFilter     one "delta" level refining an external coarse flow
//   PyramidalFlowFilter an owned uint8 input, an image pyramid, L-1 delta levels and a top
//
// Filter state lives in HBM in ping-pong pairs (read the previous frame's copy, write
// this frame's), so every level of a frame can be computed by one fused kernel that
// reads its neighbours' halo pixels without racing other tiles.
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <memory>
#include <vector>

#include "ffb200.h"
#include "kernels.h"

namespace ffb {

// error carrying an ff_status across the C++ layer
struct Error : std::runtime_error {
    ff_status status;
    Error(ff_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void check_cuda(cudaError_t e, const char* what);

// sends a message to the caller's log callback, if one is set (ff_set_log_callback)
void log_message(int level, const std::string& msg);

// Every device allocation of the library goes through these two.  For fault-injection
// tests, inject_allocation_failure(n) lets n more allocations succeed and fails the next
// one with cudaErrorMemoryAllocation before CUDA is called (then switches itself off);
// n < 0 switches it off.
cudaError_t device_malloc(void** p, size_t bytes);
cudaError_t device_malloc_pitch(void** p, size_t* pitch, size_t width_bytes, size_t height);
void inject_allocation_failure(long long n);

// pitched device buffer (owning)
struct Buf {
    void* p = nullptr;
    size_t pitch = 0;
    int h = 0, w = 0;   // pixels
    int bpp = 0;        // bytes per pixel
    void alloc(int h_, int w_, int bpp_);
    void release();
    void clear(cudaStream_t s);
    size_t row_bytes() const { return (size_t)w * bpp; }
};

enum class Kind { Single = 0, Delta = 1, Pyramidal = 2 };

// how one level step runs
enum Path { kPerStage = 0, kStream = 1, kTile = 2 };

struct Level {
    bool delta = false;
    int H = 0, W = 0;
    int item = 1;                // input image item size
    const void* img = nullptr;   // level image (device)
    size_t img_pitch = 0;
    bool img_owned = false;      // image buffer allocated here (aligned, padded pitch)
    Buf fs[2], io[2], d[2];      // ping-pong state: smoothed flow, old image, delta flow
    Buf fu;                      // unsmoothed updated flow (top levels)
    // coarse flow source for delta levels
    const void* coarse = nullptr;  // external coarse flow (standalone DeltaFlowFilter)
    size_t coarse_pitch = 0;
    int Hc = 0, Wc = 0;
    float gamma = 1.0f;          // value used by the update (already scaled for uint8 input)
    float maxflow = 1.0f;
    int iters = 1;               // propagation iterations = ceil(maxflow)
    int smooth = 1;
    int border = 3;
    bool first = true;
    int tuned_path = -1;         // autotuned: -1 not tuned, else a Path
    int tuned_band = 0;          // streaming kernel: band rows; tile kernel: tile shape (0 automatic)
    Buf coarse_rows;             // int per row: coarse row its update reads (delta levels)
    void build_coarse_rows();
    // scratch of the unfused path (allocated on first use)
    Buf a0, grad, fp, ip, dp, t1, t2, t3, fut;
    void alloc_state();
    void alloc_scratch();
    void release();
};

class Filter {
public:
    // own_input: allocate the level-0 input image (FlowFilter(h, w, ...), pyramids)
    Filter(Kind kind, int H, int W, int levels, int item, bool own_input);
    ~Filter();
    Filter(const Filter&) = delete;
    Filter& operator=(const Filter&) = delete;

    Kind kind() const { return kind_; }
    int height() const { return H_; }
    int width() const { return W_; }
    int levels() const { return L_; }
    int item() const { return item_; }
    Level& level(int l);
    const Level& level(int l) const;

    // parameters (reference setter rules)
    void set_gamma(int level, float g);
    float gamma(int level) const;
    void set_max_flow(float m);
    float max_flow() const;
    void set_smooth(int level, int n);
    int smooth(int level) const;
    void set_border(int b);
    int border() const;
    int iterations(int level) const;

    void set_stream(cudaStream_t s);
    cudaStream_t stream() const { return stream_; }

    // inputs
    void load_host(const ff_image& img);
    void load_device_async(const void* img, size_t pitch, cudaStream_t s);
    void bind_device(const void* img, size_t pitch);
    void set_external_image(const void* img, size_t pitch);
    void set_external_coarse(const void* flow, size_t pitch, int Hc, int Wc);

    // compute
    void compute();                       // blocking, records elapsed time
    // Pipelined host processing: upload `in` (host) on a copy stream, compute on s, and
    // download the smoothed level-0 flow into `out` (host) on a second copy stream, so
    // consecutive frames overlap.  Host buffers must stay valid until synchronize().
    void process_host_async(const ff_image& in, ff_image& out, cudaStream_t s);
    // block until every operation queued on the filter (pipelined copies included) is done
    void synchronize();
    void compute_async(cudaStream_t s);   // enqueue only
    void phase_model();
    void phase_propagation();
    void phase_update();
    float elapsed_ms() const { return elapsed_; }

    // results (current frame)
    void result(int which, void** p, size_t* pitch);
    void download_flow(ff_image& out);
    void download_image(ff_image& out);
    void level_state(int level, int which, void* dst, size_t dst_pitch);

    // 0: per-stage kernels only, 1: streaming fused kernel wherever instantiated,
    // 2: automatic (the autotuned choice, else the streaming kernel for levels of at least
    // kFusedMinPixels pixels and the tile kernel below), 3: tile-fused kernel wherever it fits
    void set_fused(int mode) {
        fused_mode_ = mode;
        drop_graphs();
    }
    static constexpr long kFusedMinPixels = 200000;
    // time every candidate kernel configuration of each level on the current inputs and
    // keep the fastest (re-running a level step rewrites bit-identical outputs)
    void autotune(int reps, void* flush = nullptr, size_t flush_bytes = 0);
    float time_level(int l, int reps, void* flush, size_t flush_bytes);
    std::string tuning() const;
    void set_level_tuning(int l, int path, int band) {
        Level& v = level(l);
        v.tuned_path = path;
        v.tuned_band = band;
        drop_graphs();
    }
    // replay each parity's frame from a captured CUDA graph
    void set_graphs(bool on);
    // record per-level kernel events for the next `frames` computes
    void set_profiling(int frames);
    void level_kernel_ms(int level, float* total, int* frames);
    void set_band(int rows) {
        band_ = rows;
        drop_graphs();
    }

    // ---- checkpoint and resume: the state of the latest frame (per level the smoothed flow,
    // the old image, the delta flow of delta levels or the unsmoothed flow of the top level,
    // and whether the level has seen a frame) as a host byte image; importing it into a
    // filter of the same kind and level sizes continues that stream exactly.  Parameters are
    // not part of the state.
    size_t state_bytes() const;
    void export_state(void* host, size_t bytes) const;
    void import_state(const void* host, size_t bytes);

    // ---- stepping by a Batch (batch.cu), which launches this filter's level steps itself
    // kernel arguments of level l for the next frame (state copy cur -> cur ^ 1)
    LevelArgs level_args(int l) const;
    bool any_first() const;
    int parity() const { return cur_; }
    // can level l run the streaming fused kernel (instantiated, aligned rows, coarse flow)?
    bool streaming_ok(int l) const { return fused_ok(l); }
    // block until everything queued on the filter so far has finished
    void wait_done() const;
    // changes whenever a parameter that shapes the level steps changes
    unsigned long long config_generation() const { return config_gen_; }
    // order stream s after this filter's own work queued since the last batch step
    void batch_begin(cudaStream_t s);
    // a batch finished this filter's frame on s: record it and advance the state parity
    void batch_end(cudaStream_t s);

private:
    void enqueue_frame(cudaStream_t s);
    void begin_on(cudaStream_t s);
    void end_on(cudaStream_t s);
    void drop_graphs();
    void release_runtime();
    void step_level(int l, cudaStream_t s);
    bool fused_ok(int l) const;
    bool tile_ok(int l, int cfg) const;
    int path_of(int l, int* param) const;
    void launch_fused(int l, int band, cudaStream_t s);
    void launch_tile(int l, int cfg, cudaStream_t s);
    void step_level_unfused(int l, cudaStream_t s);
    void model_unfused(int l, cudaStream_t s);
    void propagate_unfused(int l, cudaStream_t s);
    void update_unfused(int l, cudaStream_t s);
    void coarse_of(int l, const void** p, size_t* pitch, int* Hc, int* Wc) const;
    void check_image_shape(int h, int w, int depth, int item) const;

    Kind kind_;
    int H_, W_, L_, item_;
    Buf input_;                    // owned level-0 input (Single owned, Pyramidal)
    std::vector<Buf> pyr_;         // pyr_[l-1] = level l image
    std::vector<Level> lv_;
    int cur_ = 0;                  // index of the latest state copy
    cudaStream_t stream_ = nullptr;
    bool own_stream_ = false;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    float elapsed_ = 0.0f;
    int fused_mode_ = 2;
    int phase_ = 0;                // phase API progress: 0 none, 1 model, 2 propagated
    int band_ = 0;                 // rows per warp band of the fused kernels (0 = automatic)
    cudaStream_t side_ = nullptr;  // levels 0..L-3 run here, concurrent with the top chain
    cudaStream_t cap_ = nullptr;   // graph capture stream
    cudaEvent_t ev_fork_ = nullptr, ev_pyr_ = nullptr, ev_join_ = nullptr;
    cudaEvent_t done_ = nullptr;   // end of the last operation queued on the filter
    bool graphs_ = false;
    unsigned long long config_gen_ = 0;  // bumped by drop_graphs (every parameter change)
    unsigned long long ops_ = 0;         // bumped by end_on
    unsigned long long batch_seen_ = 0;  // ops_ after the last batch step
    cudaGraphExec_t graph_exec_[2] = {nullptr, nullptr};
    int prof_cap_ = 0, prof_count_ = 0;
    std::vector<cudaEvent_t> prof_ev_;
    // pipelined host processing: per state parity a staging input image and the events of
    // its upload, its compute and the download of its result
    struct HostPipe {
        Buf staging[2];
        cudaStream_t in = nullptr, out = nullptr;
        cudaEvent_t h2d[2] = {nullptr, nullptr}, computed[2] = {nullptr, nullptr}, d2h[2] = {nullptr, nullptr};
        cudaEvent_t last_d2h = nullptr;
        bool pending = false;  // downloads queued that later non-pipelined work must wait for
        ~HostPipe();
    };
    std::unique_ptr<HostPipe> pipe_;
    bool pipe_mode_ = false;  // level 0 reads the staging images (graphs captured that way)
    bool in_pipe_ = false;
    bool pdl_chain_ = false;  // set while enqueue_frame launches the top -> L-2 chain
    bool fuse_pyramid_ = false;  // set while enqueue_frame runs a frame whose top kernel makes level 1
    void leave_pipe_mode();
};

}  // namespace ffb
