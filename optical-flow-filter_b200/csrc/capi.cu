// extern "C" entry points of libffb200.so (declared in include/ffb200.h).
//
// Every entry point converts C++ exceptions into ff_status codes and stores the
// message for ff_last_error(); nothing here exits the process.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <vector>
#include <new>
#include <string>

#include "batch.h"
#include "ffb200.h"
#include "filter.h"
#include "kernels.h"

using ffb::Error;
using ffb::Filter;
using ffb::Kind;

struct ff_filter {
    Filter* impl;
    int device;
    bool borrowed = false;  // a stream of an ff_batch: owned and destroyed by the batch
};

struct ff_batch {
    ffb::Batch* impl;
    int device;
    std::vector<ff_filter> streams;
};

namespace {

thread_local std::string g_last_error;

// the opt-in log callback (ff_set_log_callback)
std::mutex g_log_mutex;
ff_log_fn g_log_fn = nullptr;
void* g_log_user = nullptr;

ff_status fail(ff_status s, const std::string& msg) {
    g_last_error = msg;
    ffb::log_message(FF_LOG_ERROR, std::string(ff_status_string(s)) + ": " + msg);
    return s;
}

template <typename F>
ff_status guard(F&& fn) {
    try {
        fn();
        return FF_OK;
    } catch (const Error& e) {
        return fail(e.status, e.what());
    } catch (const std::bad_alloc&) {
        return fail(FF_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(FF_ERR_LOGIC, e.what());
    } catch (...) {
        return fail(FF_ERR_LOGIC, "unknown error");
    }
}

Filter* get(ff_filter* f) {
    if (!f || !f->impl) throw Error(FF_ERR_INVALID_ARGUMENT, "null filter");
    ffb::check_cuda(cudaSetDevice(f->device), "cudaSetDevice");
    return f->impl;
}
const Filter* cget(const ff_filter* f) {
    if (!f || !f->impl) throw Error(FF_ERR_INVALID_ARGUMENT, "null filter");
    return f->impl;
}

template <typename T>
void need(T* p, const char* what) {
    if (!p) throw Error(FF_ERR_INVALID_ARGUMENT, std::string("null ") + what);
}

ff_filter* wrap(Filter* impl) {
    int dev = 0;
    cudaGetDevice(&dev);
    ff_filter* h = new ff_filter;
    h->impl = impl;
    h->device = dev;
    return h;
}

void check_stage_dims(int h, int w) {
    if (h <= 0 || w <= 0) throw Error(FF_ERR_INVALID_ARGUMENT, "stage shape must be positive");
}

}  // namespace

namespace ffb {
void log_message(int level, const std::string& msg) {
    ff_log_fn fn;
    void* user;
    {
        std::lock_guard<std::mutex> lock(g_log_mutex);
        fn = g_log_fn;
        user = g_log_user;
    }
    if (fn) fn(level, msg.c_str(), user);
}
}  // namespace ffb

// failure reporting for entry points defined in other files (diff_kernels.cu, display.cu,
// rotation.cu): the last error and the FF_LOG_ERROR message, as for the entry points here
ff_status ffb_fail(ff_status s, const std::string& msg) { return fail(s, msg); }

extern "C" {

const char* ff_last_error(void) { return g_last_error.c_str(); }

ff_status ff_set_log_callback(ff_log_fn fn, void* user) {
    std::lock_guard<std::mutex> lock(g_log_mutex);
    g_log_fn = fn;
    g_log_user = user;
    return FF_OK;
}

const char* ff_status_string(ff_status s) {
    switch (s) {
        case FF_OK: return "ok";
        case FF_ERR_INVALID_ARGUMENT: return "invalid argument";
        case FF_ERR_LOGIC: return "logic error";
        case FF_ERR_OUT_OF_RANGE: return "out of range";
        case FF_ERR_SHAPE: return "shape mismatch";
        case FF_ERR_CUDA: return "CUDA error";
        case FF_ERR_OUT_OF_MEMORY: return "out of memory";
        case FF_ERR_UNSUPPORTED: return "unsupported";
    }
    return "unknown status";
}

int ff_version(void) { return 10000; }

ff_status ff_set_device(int device) {
    return guard([&] { ffb::check_cuda(cudaSetDevice(device), "cudaSetDevice"); });
}

// ------------------------------------------------------------------ buffers
ff_status ff_malloc_pitch(void** dptr, size_t* pitch, size_t width_bytes, size_t height) {
    return guard([&] {
        need(dptr, "pointer");
        need(pitch, "pitch");
        ffb::check_cuda(ffb::device_malloc_pitch(dptr, pitch, width_bytes, height), "cudaMallocPitch");
    });
}

ff_status ff_debug_fail_allocation_after(long long n) {
    return guard([&] { ffb::inject_allocation_failure(n); });
}

ff_status ff_free(void* dptr) {
    return guard([&] { ffb::check_cuda(cudaFree(dptr), "cudaFree"); });
}

ff_status ff_memcpy2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width_bytes, size_t height,
                      int kind) {
    return guard([&] {
        need(dst, "destination");
        need(src, "source");
        cudaMemcpyKind k = kind == 0 ? cudaMemcpyHostToDevice
                           : kind == 1 ? cudaMemcpyDeviceToHost
                           : kind == 2 ? cudaMemcpyDeviceToDevice
                                       : cudaMemcpyDefault;
        if (kind < 0 || kind > 2) throw Error(FF_ERR_INVALID_ARGUMENT, "copy kind must be 0, 1 or 2");
        ffb::check_cuda(cudaMemcpy2D(dst, dpitch, src, spitch, width_bytes, height, k), "cudaMemcpy2D");
    });
}

ff_status ff_memset2d(void* dptr, size_t pitch, int value, size_t width_bytes, size_t height) {
    return guard([&] {
        need(dptr, "pointer");
        ffb::check_cuda(cudaMemset2D(dptr, pitch, value, width_bytes, height), "cudaMemset2D");
    });
}

// ------------------------------------------------------------------ filters
ff_status ff_filter_create(int height, int width, int smooth_iterations, float maxflow, float gamma,
                           ff_filter** out) {
    return guard([&] {
        need(out, "output handle");
        *out = nullptr;
        Filter* f = new Filter(Kind::Single, height, width, 1, 1, true);
        try {
            // FlowFilter(h, w, S, maxflow, gamma): setGamma, setMaxFlow, setSmoothIterations
            f->set_gamma(0, gamma);
            f->set_max_flow(maxflow);
            f->set_smooth(0, smooth_iterations);
        } catch (...) {
            delete f;
            throw;
        }
        *out = wrap(f);
    });
}

ff_status ff_filter_create_on_device_image(const void* image, size_t pitch, int item_size, int height, int width,
                                           ff_filter** out) {
    return guard([&] {
        need(out, "output handle");
        need(image, "image");
        *out = nullptr;
        Filter* f = new Filter(Kind::Single, height, width, 1, item_size, false);
        try {
            f->set_external_image(image, pitch);
        } catch (...) {
            delete f;
            throw;
        }
        *out = wrap(f);
    });
}

ff_status ff_delta_filter_create(const void* image, size_t pitch, int item_size, int height, int width,
                                 const void* coarse_flow, size_t coarse_pitch, int height_c, int width_c,
                                 ff_filter** out) {
    return guard([&] {
        need(out, "output handle");
        need(image, "image");
        need(coarse_flow, "coarse flow");
        *out = nullptr;
        Filter* f = new Filter(Kind::Delta, height, width, 1, item_size, false);
        try {
            f->set_external_image(image, pitch);
            f->set_external_coarse(coarse_flow, coarse_pitch, height_c, width_c);
        } catch (...) {
            delete f;
            throw;
        }
        *out = wrap(f);
    });
}

ff_status ff_pyramidal_create(int height, int width, int levels, ff_filter** out) {
    return guard([&] {
        need(out, "output handle");
        *out = nullptr;
        *out = wrap(new Filter(Kind::Pyramidal, height, width, levels, 1, true));
    });
}

ff_status ff_filter_destroy(ff_filter* f) {
    return guard([&] {
        if (!f) return;
        if (f->borrowed) throw Error(FF_ERR_LOGIC, "this filter is a stream of a batch; destroy the batch instead");
        cudaSetDevice(f->device);
        delete f->impl;
        delete f;
    });
}

ff_status ff_filter_shape(const ff_filter* f, int* height, int* width, int* levels) {
    return guard([&] {
        const Filter* F = cget(f);
        if (height) *height = F->height();
        if (width) *width = F->width();
        if (levels) *levels = F->levels();
    });
}

ff_status ff_filter_kind(const ff_filter* f, int* kind) {
    return guard([&] {
        need(kind, "kind");
        *kind = (int)cget(f)->kind();
    });
}

ff_status ff_filter_level_shape(const ff_filter* f, int level, int* height, int* width) {
    return guard([&] {
        const ffb::Level& v = cget(f)->level(level);
        if (height) *height = v.H;
        if (width) *width = v.W;
    });
}

ff_status ff_filter_set_gamma(ff_filter* f, int level, float gamma) {
    return guard([&] { get(f)->set_gamma(level, gamma); });
}
ff_status ff_filter_get_gamma(const ff_filter* f, int level, float* gamma) {
    return guard([&] {
        need(gamma, "gamma");
        *gamma = cget(f)->gamma(level);
    });
}
ff_status ff_filter_set_max_flow(ff_filter* f, float maxflow) {
    return guard([&] { get(f)->set_max_flow(maxflow); });
}
ff_status ff_filter_get_max_flow(const ff_filter* f, float* maxflow) {
    return guard([&] {
        need(maxflow, "maxflow");
        *maxflow = cget(f)->max_flow();
    });
}
ff_status ff_filter_set_smooth_iterations(ff_filter* f, int level, int iterations) {
    return guard([&] { get(f)->set_smooth(level, iterations); });
}
ff_status ff_filter_get_smooth_iterations(const ff_filter* f, int level, int* iterations) {
    return guard([&] {
        need(iterations, "iterations");
        *iterations = cget(f)->smooth(level);
    });
}
ff_status ff_filter_set_propagation_border(ff_filter* f, int border) {
    return guard([&] { get(f)->set_border(border); });
}
ff_status ff_filter_get_propagation_border(const ff_filter* f, int* border) {
    return guard([&] {
        need(border, "border");
        *border = cget(f)->border();
    });
}
ff_status ff_filter_get_propagation_iterations(const ff_filter* f, int level, int* iterations) {
    return guard([&] {
        need(iterations, "iterations");
        *iterations = cget(f)->iterations(level);
    });
}

ff_status ff_filter_set_fused(ff_filter* f, int enabled) {
    return guard([&] {
        if (enabled < 0 || enabled > 3) throw Error(FF_ERR_INVALID_ARGUMENT, "fused mode must be 0, 1, 2 or 3");
        get(f)->set_fused(enabled);
    });
}

ff_status ff_filter_set_graphs(ff_filter* f, int enabled) {
    return guard([&] { get(f)->set_graphs(enabled != 0); });
}

ff_status ff_filter_autotune(ff_filter* f, int repetitions) {
    return guard([&] { get(f)->autotune(repetitions); });
}

ff_status ff_filter_autotune_flush(ff_filter* f, int repetitions, void* flush, size_t flush_bytes) {
    return guard([&] { get(f)->autotune(repetitions, flush, flush_bytes); });
}

ff_status ff_filter_get_level_tuning(const ff_filter* f, int level, int* path, int* band) {
    return guard([&] {
        need(path, "path");
        need(band, "band");
        const ffb::Level& v = cget(f)->level(level);
        *path = v.tuned_path;
        *band = v.tuned_band;
    });
}

ff_status ff_filter_set_level_tuning(ff_filter* f, int level, int path, int band) {
    return guard([&] {
        if (path < -1 || path > 2) throw Error(FF_ERR_INVALID_ARGUMENT, "path must be -1, 0, 1 or 2");
        if (band < 0) throw Error(FF_ERR_INVALID_ARGUMENT, "band rows must be >= 0");
        if (path == 2 && band >= ffb::tile_config_count())
            throw Error(FF_ERR_INVALID_ARGUMENT, "tile shape index must be below " + std::to_string(ffb::tile_config_count()));
        get(f)->set_level_tuning(level, path, band);
    });
}

ff_status ff_filter_tuning(const ff_filter* f, char* buf, size_t len) {
    return guard([&] {
        need(buf, "buffer");
        const std::string t = cget(f)->tuning();
        if (len == 0) throw Error(FF_ERR_INVALID_ARGUMENT, "empty buffer");
        const size_t n = t.size() < len - 1 ? t.size() : len - 1;
        std::memcpy(buf, t.data(), n);
        buf[n] = 0;
    });
}

ff_status ff_filter_set_band(ff_filter* f, int rows) {
    return guard([&] {
        if (rows < 0) throw Error(FF_ERR_INVALID_ARGUMENT, "band rows must be >= 0");
        get(f)->set_band(rows);
    });
}

ff_status ff_filter_set_profiling(ff_filter* f, int max_frames) {
    return guard([&] { get(f)->set_profiling(max_frames); });
}

ff_status ff_filter_level_kernel_ms(ff_filter* f, int level, float* total_ms, int* frames) {
    return guard([&] {
        need(total_ms, "total");
        need(frames, "frames");
        get(f)->level_kernel_ms(level, total_ms, frames);
    });
}

ff_status ff_filter_time_level(ff_filter* f, int level, int reps, void* flush, size_t flush_bytes, float* total_ms) {
    return guard([&] {
        need(total_ms, "total");
        *total_ms = get(f)->time_level(level, reps, flush, flush_bytes);
    });
}

ff_status ff_filter_set_stream(ff_filter* f, void* stream) {
    return guard([&] { get(f)->set_stream((cudaStream_t)stream); });
}

ff_status ff_filter_load_image_host(ff_filter* f, const ff_image* image) {
    return guard([&] {
        need(image, "image");
        get(f)->load_host(*image);
    });
}

ff_status ff_filter_load_image_device_async(ff_filter* f, const void* image, size_t pitch, void* stream) {
    return guard([&] { get(f)->load_device_async(image, pitch, (cudaStream_t)stream); });
}

ff_status ff_filter_bind_image_device(ff_filter* f, const void* image, size_t pitch) {
    return guard([&] { get(f)->bind_device(image, pitch); });
}

ff_status ff_filter_compute(ff_filter* f) {
    return guard([&] { get(f)->compute(); });
}
ff_status ff_filter_compute_async(ff_filter* f, void* stream) {
    return guard([&] { get(f)->compute_async((cudaStream_t)stream); });
}
ff_status ff_filter_process_host_async(ff_filter* f, const ff_image* in, ff_image* out, void* stream) {
    return guard([&] {
        need(in, "input image");
        need(out, "flow buffer");
        get(f)->process_host_async(*in, *out, (cudaStream_t)stream);
    });
}
ff_status ff_filter_synchronize(ff_filter* f) {
    return guard([&] { get(f)->synchronize(); });
}
ff_status ff_filter_compute_image_model(ff_filter* f) {
    return guard([&] { get(f)->phase_model(); });
}
ff_status ff_filter_compute_propagation(ff_filter* f) {
    return guard([&] { get(f)->phase_propagation(); });
}
ff_status ff_filter_compute_update(ff_filter* f) {
    return guard([&] { get(f)->phase_update(); });
}
ff_status ff_filter_elapsed_ms(const ff_filter* f, float* ms) {
    return guard([&] {
        need(ms, "ms");
        *ms = cget(f)->elapsed_ms();
    });
}

ff_status ff_filter_state_bytes(const ff_filter* f, size_t* bytes) {
    return guard([&] {
        need(bytes, "bytes");
        *bytes = cget(f)->state_bytes();
    });
}

ff_status ff_filter_export_state(ff_filter* f, void* host, size_t bytes) {
    return guard([&] { get(f)->export_state(host, bytes); });
}

ff_status ff_filter_import_state(ff_filter* f, const void* host, size_t bytes) {
    return guard([&] { get(f)->import_state(host, bytes); });
}

ff_status ff_filter_download_flow_host(ff_filter* f, ff_image* flow) {
    return guard([&] {
        need(flow, "flow");
        get(f)->download_flow(*flow);
    });
}
ff_status ff_filter_download_image_host(ff_filter* f, ff_image* image) {
    return guard([&] {
        need(image, "image");
        get(f)->download_image(*image);
    });
}
ff_status ff_filter_device_result(ff_filter* f, int which, void** dptr, size_t* pitch) {
    return guard([&] {
        need(dptr, "pointer");
        need(pitch, "pitch");
        get(f)->result(which, dptr, pitch);
    });
}
ff_status ff_filter_level_state_host(ff_filter* f, int level, int which, void* dst, size_t dst_pitch) {
    return guard([&] { get(f)->level_state(level, which, dst, dst_pitch); });
}

// ------------------------------------------------------------------ stages
ff_status ff_stage_pyramid_down(const void* in, size_t in_pitch, int item_size, int height, int width, void* out,
                                size_t out_pitch, void* stream) {
    return guard([&] {
        need(in, "input");
        need(out, "output");
        check_stage_dims(height, width);
        if (item_size != 1 && item_size != 4) throw Error(FF_ERR_INVALID_ARGUMENT, "item size should be 1 or 4");
        ffb::check_cuda(ffb::launch_pyramid_down(in, in_pitch, item_size, height, width, out, out_pitch,
                                                 (cudaStream_t)stream),
                        "pyramid");
    });
}

ff_status ff_stage_image_model(const void* img, size_t img_pitch, int item_size, int height, int width, float* a0,
                               size_t a0_pitch, float* grad, size_t grad_pitch, void* stream) {
    return guard([&] {
        need(img, "image");
        need(a0, "a0");
        need(grad, "gradient");
        check_stage_dims(height, width);
        if (item_size != 1 && item_size != 4) throw Error(FF_ERR_INVALID_ARGUMENT, "item size should be 1 or 4");
        ffb::check_cuda(ffb::launch_image_model(img, img_pitch, item_size, height, width, a0, a0_pitch, grad,
                                                grad_pitch, (cudaStream_t)stream),
                        "image model");
    });
}

static size_t ws_pitch(int width, int bpp) { return (((size_t)width * bpp) + 511) / 512 * 512; }

size_t ff_stage_propagate_workspace_size(int height, int width) {
    if (height <= 0 || width <= 0) return 0;
    return ws_pitch(width, 8) * (size_t)height;
}

ff_status ff_stage_propagate(const float* flow, size_t flow_pitch, int height, int width, int iterations,
                             int border, float* out, size_t out_pitch, void* ws, void* stream) {
    return guard([&] {
        need(flow, "flow");
        need(out, "output");
        need(ws, "workspace");
        check_stage_dims(height, width);
        if (iterations <= 0) throw Error(FF_ERR_INVALID_ARGUMENT, "iterations should be greater than zero");
        if (border < 0) throw Error(FF_ERR_INVALID_ARGUMENT, "border should be greater or equal zero");
        ffb::check_cuda(ffb::launch_propagate(flow, flow_pitch, height, width, iterations, border, out, out_pitch,
                                              (float*)ws, ws_pitch(width, 8), (cudaStream_t)stream),
                        "propagate");
    });
}

size_t ff_stage_propagate_payload_workspace_size(int height, int width) {
    if (height <= 0 || width <= 0) return 0;
    return (2 * ws_pitch(width, 8) + ws_pitch(width, 4)) * (size_t)height;
}

ff_status ff_stage_propagate_payload(const float* flow, size_t flow_pitch, const float* scalar, size_t scalar_pitch,
                                     const float* vector, size_t vector_pitch, int height, int width, int iterations,
                                     int border, float* out_flow, size_t out_flow_pitch, float* out_scalar,
                                     size_t out_scalar_pitch, float* out_vector, size_t out_vector_pitch, void* ws,
                                     void* stream) {
    return guard([&] {
        need(flow, "flow");
        need(scalar, "scalar");
        need(vector, "vector");
        need(out_flow, "output flow");
        need(out_scalar, "output scalar");
        need(out_vector, "output vector");
        need(ws, "workspace");
        check_stage_dims(height, width);
        if (iterations <= 0) throw Error(FF_ERR_INVALID_ARGUMENT, "iterations should be greater than zero");
        if (border < 0) throw Error(FF_ERR_INVALID_ARGUMENT, "border should be greater or equal zero");
        const size_t p8 = ws_pitch(width, 8), p4 = ws_pitch(width, 4);
        char* base = (char*)ws;
        float* tf = (float*)base;
        float* tv = (float*)(base + p8 * height);
        float* ts = (float*)(base + 2 * p8 * height);
        ffb::check_cuda(ffb::launch_propagate_payload(flow, flow_pitch, scalar, scalar_pitch, vector, vector_pitch,
                                                      height, width, iterations, border, out_flow, out_flow_pitch,
                                                      out_scalar, out_scalar_pitch, out_vector, out_vector_pitch, tf,
                                                      p8, ts, p4, tv, p8, (cudaStream_t)stream),
                        "propagate payload");
    });
}

ff_status ff_stage_update(const float* a0, size_t a0_pitch, const float* grad, size_t grad_pitch,
                          const float* a0_old, size_t a0_old_pitch, const float* flow, size_t flow_pitch, int height,
                          int width, float gamma, float maxflow, float* out_flow, size_t out_flow_pitch,
                          float* out_image, size_t out_image_pitch, void* stream) {
    return guard([&] {
        need(a0, "a0");
        need(grad, "gradient");
        need(a0_old, "old image");
        need(flow, "flow");
        need(out_flow, "output flow");
        need(out_image, "output image");
        check_stage_dims(height, width);
        if (!(gamma > 0.0f)) throw Error(FF_ERR_INVALID_ARGUMENT, "gamma should be greater than zero");
        ffb::check_cuda(ffb::launch_update(a0, a0_pitch, grad, grad_pitch, a0_old, a0_old_pitch, flow, flow_pitch,
                                           height, width, gamma, maxflow, out_flow, out_flow_pitch, out_image,
                                           out_image_pitch, 0, (cudaStream_t)stream),
                        "update");
    });
}

ff_status ff_stage_delta_update(const float* a0, size_t a0_pitch, const float* grad, size_t grad_pitch,
                                const float* a0_old, size_t a0_old_pitch, const float* delta, size_t delta_pitch,
                                const float* coarse, size_t coarse_pitch, int height_c, int width_c, int height,
                                int width, float gamma, float maxflow, float* out_flow, size_t out_flow_pitch,
                                float* out_delta, size_t out_delta_pitch, float* out_image, size_t out_image_pitch,
                                void* stream) {
    return guard([&] {
        need(a0, "a0");
        need(grad, "gradient");
        need(a0_old, "old image");
        need(delta, "delta");
        need(coarse, "coarse flow");
        need(out_flow, "output flow");
        need(out_delta, "output delta");
        need(out_image, "output image");
        check_stage_dims(height, width);
        check_stage_dims(height_c, width_c);
        if (!(gamma > 0.0f)) throw Error(FF_ERR_INVALID_ARGUMENT, "gamma should be greater than zero");
        ffb::check_cuda(ffb::launch_delta_update(a0, a0_pitch, grad, grad_pitch, a0_old, a0_old_pitch, delta,
                                                 delta_pitch, coarse, coarse_pitch, height_c, width_c, height, width,
                                                 gamma, maxflow, out_flow, out_flow_pitch, out_delta, out_delta_pitch,
                                                 out_image, out_image_pitch, 0, (cudaStream_t)stream),
                        "delta update");
    });
}

size_t ff_stage_smooth_workspace_size(int height, int width) {
    if (height <= 0 || width <= 0) return 0;
    return ws_pitch(width, 8) * (size_t)height;
}

ff_status ff_stage_smooth(const float* flow, size_t flow_pitch, int height, int width, int iterations, float* out,
                          size_t out_pitch, void* ws, void* stream) {
    return guard([&] {
        need(flow, "flow");
        need(out, "output");
        need(ws, "workspace");
        check_stage_dims(height, width);
        if (iterations <= 0) throw Error(FF_ERR_INVALID_ARGUMENT, "iterations should be greater than zero");
        ffb::check_cuda(ffb::launch_smooth(flow, flow_pitch, height, width, iterations, out, out_pitch, (float*)ws,
                                           ws_pitch(width, 8), (cudaStream_t)stream),
                        "smooth");
    });
}

ff_status ff_stage_scale_flow(const float* flow, size_t flow_pitch, int height, int width, float scalar, float* out,
                              size_t out_pitch, void* stream) {
    return guard([&] {
        need(flow, "flow");
        need(out, "output");
        check_stage_dims(height, width);
        if ((uintptr_t)flow % 8 || (uintptr_t)out % 8 || flow_pitch % 8 || out_pitch % 8 ||
            flow_pitch < (size_t)width * 8 || out_pitch < (size_t)width * 8)
            throw Error(FF_ERR_INVALID_ARGUMENT, "flow fields need 8-byte aligned rows of width float2");
        ffb::check_cuda(ffb::launch_scale_flow(flow, flow_pitch, height, width, scalar, out, out_pitch,
                                               (cudaStream_t)stream),
                        "scale flow");
    });
}

}  // extern "C"

// ---- batched step over many streams (batch.h)
extern "C" {

ff_status ff_batch_create(int n, const int* heights, const int* widths, const int* levels, ff_batch** out) {
    return guard([&] {
        need(out, "output handle");
        *out = nullptr;
        int dev = 0;
        ffb::check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
        ff_batch* b = new ff_batch;
        try {
            b->impl = new ffb::Batch(n, heights, widths, levels);
        } catch (...) {
            delete b;
            throw;
        }
        b->device = dev;
        b->streams.resize(n);
        for (int i = 0; i < n; ++i) {
            b->streams[i].impl = &b->impl->stream(i);
            b->streams[i].device = dev;
            b->streams[i].borrowed = true;
        }
        *out = b;
    });
}

ff_status ff_batch_destroy(ff_batch* b) {
    return guard([&] {
        if (!b) return;
        cudaSetDevice(b->device);
        delete b->impl;
        delete b;
    });
}

ff_status ff_batch_size(const ff_batch* b, int* n) {
    return guard([&] {
        need(b, "batch");
        need(n, "count");
        *n = b->impl->size();
    });
}

ff_status ff_batch_stream(ff_batch* b, int i, ff_filter** f) {
    return guard([&] {
        need(b, "batch");
        need(f, "output handle");
        if (i < 0 || i >= b->impl->size())
            throw Error(FF_ERR_OUT_OF_RANGE, "batch stream index out of bounds: " + std::to_string(i));
        *f = &b->streams[i];
    });
}

ff_status ff_batch_frame_layout(const ff_batch* b, size_t* offsets, size_t* total) {
    return guard([&] {
        need(b, "batch");
        if (offsets)
            for (int i = 0; i < b->impl->size(); ++i) offsets[i] = b->impl->frame_offset(i);
        if (total) *total = b->impl->frame_bytes();
    });
}

ff_status ff_batch_launches(const ff_batch* b, int* launches) {
    return guard([&] {
        need(b, "batch");
        need(launches, "count");
        *launches = b->impl->launches_per_step();
    });
}

ff_status ff_batch_set_tuning(ff_batch* b, long long min_pixels, int band) {
    return guard([&] {
        need(b, "batch");
        b->impl->set_tuning((long)min_pixels, band);
    });
}

ff_status ff_batch_set_level_band(ff_batch* b, int height, int width, int band) {
    return guard([&] {
        need(b, "batch");
        if (height <= 0 || width <= 0) throw ffb::Error(FF_ERR_INVALID_ARGUMENT, "batch: level size must be positive");
        b->impl->set_level_band(height, width, band);
    });
}

ff_status ff_batch_step(ff_batch* b, const void* frames, void* stream) {
    return guard([&] {
        need(b, "batch");
        ffb::check_cuda(cudaSetDevice(b->device), "cudaSetDevice");
        b->impl->step(frames, (cudaStream_t)stream);
    });
}

}  // extern "C"

// ---- smoothing on a static device scratch (ff_stage_smooth_noalloc)
//
// The X pass of every smoothing iteration writes its float2 field into this module-scope
// array and the Y pass reads it back, so the entry point needs neither a caller workspace
// nor an allocation. The array needs no initial contents: every element a Y pass reads
// was written by the X pass just before it, on the same stream.
namespace {

constexpr size_t kStaticScratchBytes = size_t(32) << 20;  // a 2048x2048 float2 field
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_smooth_scratch[kStaticScratchBytes];

std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};

// Unique id of the current device's primary context (cuCtxGetId through the runtime's
// driver entry points, so the library does not link libcuda). A cudaDeviceReset makes a
// new context, in which the module and its array are loaded again, maybe elsewhere.
unsigned long long current_context_id() {
    static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
    static PFN_cuCtxGetId_v12000 get_id = nullptr;
    if (!get_current || !get_id) {
        void* a = nullptr;
        void* b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        ffb::check_cuda(cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa), "cuCtxGetCurrent");
        ffb::check_cuda(cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb), "cuCtxGetId");
        if (qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b)
            throw Error(FF_ERR_CUDA, "driver entry points cuCtxGetCurrent / cuCtxGetId not found");
        get_current = (PFN_cuCtxGetCurrent_v4000)a;
        get_id = (PFN_cuCtxGetId_v12000)b;
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        throw Error(FF_ERR_CUDA, "no current CUDA context");
    return id;
}

// Device address of g_smooth_scratch on the current device, looked up once per device and
// context (again after a cudaDeviceReset). The lookup may load this module onto the
// device, which is not allowed while a stream is being captured, so each device's first
// call belongs before any capture.
void* static_scratch() {
    int dev = 0;
    ffb::check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) throw Error(FF_ERR_UNSUPPORTED, "device ordinal above 63");
    ffb::check_cuda(cudaSetDevice(dev), "cudaSetDevice");  // initialises and binds the device's context
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev] || g_scratch_ctx[dev] != ctx) {
        void* p = nullptr;
        ffb::check_cuda(cudaGetSymbolAddress(&p, g_smooth_scratch), "cudaGetSymbolAddress(static scratch)");
        if (!p) throw Error(FF_ERR_CUDA, "cudaGetSymbolAddress returned a null scratch address");
        g_scratch_ptr[dev] = p;
        g_scratch_ctx[dev] = ctx;
    }
    return g_scratch_ptr[dev];
}

}  // namespace

extern "C" {

ff_status ff_stage_smooth_noalloc(const float* flow, size_t flow_pitch, int height, int width, int iterations,
                                  float* out, size_t out_pitch, void* stream) {
    return guard([&] {
        need(flow, "flow");
        need(out, "output");
        check_stage_dims(height, width);
        if (iterations <= 0) throw Error(FF_ERR_INVALID_ARGUMENT, "iterations should be greater than zero");
        const size_t bytes = ws_pitch(width, 8) * (size_t)height;
        if (bytes > kStaticScratchBytes)
            throw Error(FF_ERR_INVALID_ARGUMENT,
                        "ff_stage_smooth_noalloc: a " + std::to_string(height) + "x" + std::to_string(width) +
                            " flow needs " + std::to_string(bytes) + " bytes of scratch, above the static " +
                            std::to_string(kStaticScratchBytes) + " bytes (use ff_stage_smooth with a workspace)");
        float* tmp = (float*)static_scratch();
        ffb::check_cuda(ffb::launch_smooth(flow, flow_pitch, height, width, iterations, out, out_pitch, tmp,
                                           ws_pitch(width, 8), (cudaStream_t)stream),
                        "smooth (static scratch)");
    });
}

}  // extern "C"
