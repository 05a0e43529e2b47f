// Flow to colour: the reference's FlowToColor stage (src/gpu/display.cu:95-110, kernel
// src/gpu/device/display_k.cu:14-43).  Each pixel's flow is normalised to
// u = (f + m) / (2m) per component and looks up a 256x256 RGBA colour wheel as a
// normalised-coordinate, point-sampled, clamp-addressed texture would: column from the x
// component, row from the y component.  The texel index is computed here in integer
// arithmetic (one thread per pixel, plain loads; the 256 KB wheel stays in L1/L2).
//
// The wheel is an input.  With none given, the library's own wheel is used: the reference's
// 256x256 RGBA table (src/colorwheel.cpp, include/flowfilter/colorwheel.h:20-27), byte for
// byte, so default colours are the reference's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "ffb200.h"
#include "launch.cuh"

ff_status ffb_fail(ff_status s, const std::string& msg);  // capi.cu: last error + log
extern const unsigned char ffb_colorwheel_rgba[256 * 256 * 4];  // colorwheel_data.cpp (generated)

namespace ffb {
namespace {

constexpr int kWheel = 256;  // texels per side

// the default wheel, one copy per device that uses it (uploaded on first use)
__device__ __align__(16) uchar4 g_default_wheel[kWheel * kWheel];

// Texel chosen along one axis for flow component f: u = (f + m) / (2m) as the reference
// computes it (display_k.cu:34-35: float add, multiply by 2, IEEE division), then the
// texture unit's clamp and point sampling.  u * 256 is exact in float, and the unit's
// truncation of u to 21 fractional bits does not change floor(u * 256).
__device__ __forceinline__ int wheel_texel(float f, float m) {
    const float u = __fdiv_rn(__fadd_rn(f, m), __fmul_rn(2.0f, m));
    if (!(u > 0.0f)) return 0;  // also NaN
    if (!(u < 1.0f)) return kWheel - 1;
    return (int)__fmul_rn(u, (float)kWheel);
}

__global__ void flow_to_color_k(const float* __restrict__ flow, size_t flow_pitch, int H, int W, float maxflow,
                                const uchar4* __restrict__ wheel, uchar4* __restrict__ color, size_t color_pitch) {
    grid_dep_wait();
    grid_dep_launch();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const float2 f = reinterpret_cast<const float2*>(reinterpret_cast<const char*>(flow) + y * flow_pitch)[x];
    const uchar4* w = wheel ? wheel : g_default_wheel;
    const uchar4 c = __ldg(&w[wheel_texel(f.y, maxflow) * kWheel + wheel_texel(f.x, maxflow)]);
    reinterpret_cast<uchar4*>(reinterpret_cast<char*>(color) + y * color_pitch)[x] = c;
}

// ---- the default wheel (host): the reference's table (colorwheel_asset.py, colorwheel.z)
const std::vector<unsigned char>& default_wheel() {
    static const std::vector<unsigned char> w(ffb_colorwheel_rgba, ffb_colorwheel_rgba + kWheel * kWheel * 4);
    return w;
}

// upload the default wheel to the current device once
cudaError_t ensure_default_wheel() {
    static std::mutex mu;
    static std::vector<bool> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)done.size() <= dev) done.resize(dev + 1, false);
    if (done[dev]) return cudaSuccess;
    e = cudaMemcpyToSymbol(g_default_wheel, default_wheel().data(), default_wheel().size());
    if (e == cudaSuccess) done[dev] = true;
    return e;
}

}  // namespace
}  // namespace ffb

extern "C" {

ff_status ff_color_wheel_default(unsigned char* rgba) {
    if (!rgba) {
        return ffb_fail(FF_ERR_INVALID_ARGUMENT, "rgba must not be NULL");
    }
    const auto& w = ffb::default_wheel();
    std::copy(w.begin(), w.end(), rgba);
    return FF_OK;
}

ff_status ff_flow_to_color(const float* flow, size_t flow_pitch, int height, int width, float maxflow,
                           const unsigned char* wheel, unsigned char* color, size_t color_pitch, void* stream) {
    if (height < 1 || width < 1 || height > 65535 * 8) {
        return ffb_fail(FF_ERR_SHAPE, "flow_to_color: height must be in [1, 524280] and width positive");
    }
    if (!(maxflow > 0.0f)) {
        return ffb_fail(FF_ERR_INVALID_ARGUMENT, "flow_to_color: maxflow should be greater than 0.0");
    }
    if (!flow || !color || flow_pitch < (size_t)width * 8 || color_pitch < (size_t)width * 4 ||
        ((uintptr_t)flow | flow_pitch) % 8 || ((uintptr_t)color | color_pitch) % 4 || (uintptr_t)wheel % 4) {
        return ffb_fail(FF_ERR_INVALID_ARGUMENT, "flow_to_color: flow needs 8-byte aligned rows of width float2, color 4-byte aligned "
                           "rows of width RGBA, the wheel 4-byte alignment");
    }
    cudaError_t e = wheel ? cudaSuccess : ffb::ensure_default_wheel();
    if (e == cudaSuccess)
        e = ffb::launch_k(ffb::flow_to_color_k, dim3((width + 31) / 32, (height + 7) / 8), dim3(32, 8), 0,
                     (cudaStream_t)stream, flow, flow_pitch, height, width, maxflow,
                     reinterpret_cast<const uchar4*>(wheel), reinterpret_cast<uchar4*>(color), color_pitch);
    if (e != cudaSuccess) {
        return ffb_fail(FF_ERR_CUDA, std::string("flow_to_color: ") + cudaGetErrorString(e));
    }
    return FF_OK;
}

}  // extern "C"
