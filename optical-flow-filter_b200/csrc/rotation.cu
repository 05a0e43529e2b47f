// Rotational flow and Lax-Wendroff image propagation: the reference's
// RotationalFlowImagePredictor (src/gpu/rotation.cu:55-96; flow kernel
// src/gpu/device/rotation_k.cu:17-43; camera src/gpu/camera.cu:15-31) and
// LaxWendroffPropagator (src/gpu/propagation.cu:506-716; kernels
// include/flowfilter/gpu/device/propagation_k.h:49-132).
//
// The reference runs 2N launches (a Y pass then an X pass per iteration, each a full-image
// round trip through HBM or L2).  Here one CTA computes one 32 x 32 output tile: it loads the
// image over the tile plus a halo of P pixels (P = iterations in this launch) into shared
// memory with the flow, then runs all 2P passes there, each over a region one pixel smaller
// along its axis (clamped at the image edges as the reference's texture reads are), and
// writes only the tile.  More than kMaxFused iterations take several launches through a
// caller workspace.  The rotational flow is computed in the same kernel from the camera and
// the angular velocity (and written once), so the predictor is one launch.
//
// Arithmetic follows the reference operation for operation, with the contraction nvcc
// applies to it made explicit (pinned against the reference on a B200):
//   flow: c = w x p with p.z = 1 folded, c.x = fma(-wz, py, wy), c.y = fma(wz, px, -wx),
//         c.z = fma(wx, py, -(wy px)); flow = (fma(ax, c.x, (cx - x) c.z), fma(ay, c.y, (cy - y) c.z)).
//   depth 1: the update is evaluated in double (the source's 0.5, and the Y pass's 2.0, are
//         double literals) and rounded once: fma(R^2/2, d2, I - R/2 d0).
//   depth 4: float through the float4 operators: t1 = fma(-d0, R/2, I), I' = fma(d2, R^2/2, t1).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <string>

#include "ffb200.h"
#include "launch.cuh"

ff_status ffb_fail(ff_status s, const std::string& msg);  // capi.cu: last error + log

namespace ffb {
namespace {

constexpr int kMaxFused = 16;  // iterations per launch (halo = iterations)

struct LWArgs {
    const float* flow;  // input flow (ROT = false)
    size_t flow_pitch;
    float* flow_out;  // rotational flow written for the tile (ROT = true)
    size_t flow_out_pitch;
    float ax, ay, cx, cy, wx, wy, wz;
    const float* src;
    size_t src_pitch;
    float* dst;
    size_t dst_pitch;
    int H, W, passes, tile;
    float dt;
};

__device__ __forceinline__ float2 rotational_flow(const LWArgs& a, int x, int y) {
    const float px = __fdiv_rn(__fsub_rn((float)x, a.cx), a.ax);
    const float py = __fdiv_rn(__fsub_rn((float)y, a.cy), a.ay);
    const float c_x = __fmaf_rn(-a.wz, py, a.wy);
    const float c_y = __fmaf_rn(a.wz, px, -a.wx);
    const float c_z = __fmaf_rn(a.wx, py, -__fmul_rn(a.wy, px));
    return make_float2(__fmaf_rn(a.ax, c_x, __fmul_rn(__fsub_rn(a.cx, (float)x), c_z)),
                       __fmaf_rn(a.ay, c_y, __fmul_rn(__fsub_rn(a.cy, (float)y), c_z)));
}

// one Lax-Wendroff update along AXIS (0 = X, 1 = Y) of a depth-1 value
template <int AXIS>
__device__ __forceinline__ float lw1(float m, float i0, float p, float R) {
    const float d0 = __fsub_rn(p, m);
    float d2;
    if (AXIS == 0)
        d2 = __fadd_rn(__fsub_rn(m, __fmul_rn(2.0f, i0)), p);
    else
        d2 = __double2float_rn(__dadd_rn(__dsub_rn((double)m, __dmul_rn(2.0, (double)i0)), (double)p));
    const double h = __dmul_rn(0.5, (double)R);
    const double t1 = __dsub_rn((double)i0, __dmul_rn(h, (double)d0));
    return __double2float_rn(__fma_rn(__dmul_rn(h, (double)R), (double)d2, t1));
}

// the same for one channel of a depth-4 value (float4 operator arithmetic)
__device__ __forceinline__ float lw4(float m, float i0, float p, float b, float b2) {
    const float d0 = __fsub_rn(p, m);
    const float d2 = __fadd_rn(__fsub_rn(m, __fmul_rn(2.0f, i0)), p);
    return __fmaf_rn(d2, b2, __fmaf_rn(-d0, b, i0));
}

template <int D>
struct Pix {
    float v[D];
};

// One CTA: the tile [tx0, tx0 + T) x [ty0, ty0 + T) of the output after `passes` iterations.
// Shared memory: flow (float2) and two D-float buffers over the region
// [rx0, rx1) x [ry0, ry1) = the tile grown by `passes` and cut to the image.
template <int D, bool ROT>
__global__ void __launch_bounds__(256) lw_tile_k(LWArgs a) {
    grid_dep_wait();
    extern __shared__ __align__(16) unsigned char smem[];
    const int T = a.tile, P = a.passes, H = a.H, W = a.W;
    const int tx0 = blockIdx.x * T, ty0 = blockIdx.y * T;
    const int rx0 = max(tx0 - P, 0), ry0 = max(ty0 - P, 0);
    const int rx1 = min(tx0 + T + P, W), ry1 = min(ty0 + T + P, H);
    const int RW = rx1 - rx0, RH = ry1 - ry0;
    float2* fl = reinterpret_cast<float2*>(smem);
    Pix<D>* A = reinterpret_cast<Pix<D>*>(fl + (size_t)RW * RH);
    Pix<D>* B = A + (size_t)RW * RH;
    const int lx = threadIdx.x, ly = threadIdx.y;  // 32 x 8
    // load the image and the flow over the region
    for (int y = ry0 + ly; y < ry1; y += 8) {
        const float* srow = reinterpret_cast<const float*>(reinterpret_cast<const char*>(a.src) + y * a.src_pitch);
        for (int x = rx0 + lx; x < rx1; x += 32) {
            const int k = (y - ry0) * RW + (x - rx0);
            Pix<D> px;
            if constexpr (D == 4) {
                const float4 q = reinterpret_cast<const float4*>(srow)[x];
                px.v[0] = q.x;
                px.v[1] = q.y;
                px.v[2] = q.z;
                px.v[3] = q.w;
            } else {
                px.v[0] = srow[x];
            }
            A[k] = px;
            float2 f;
            if (ROT) {
                f = rotational_flow(a, x, y);
                if (x >= tx0 && x < tx0 + T && y >= ty0 && y < ty0 + T)
                    reinterpret_cast<float2*>(reinterpret_cast<char*>(a.flow_out) + y * a.flow_out_pitch)[x] = f;
            } else {
                f = reinterpret_cast<const float2*>(reinterpret_cast<const char*>(a.flow) + y * a.flow_pitch)[x];
            }
            fl[k] = f;
        }
    }
    grid_dep_launch();
    __syncthreads();
    // valid region of the current buffer; a pass keeps the rows (columns) whose neighbours
    // are valid, the image edges clamping to themselves
    int vx0 = rx0, vx1 = rx1, vy0 = ry0, vy1 = ry1;
    const float dt = a.dt;
    for (int it = 0; it < P; ++it) {
        // Y pass, A -> B
        vy0 = vy0 == 0 ? 0 : vy0 + 1;
        vy1 = vy1 == H ? H : vy1 - 1;
        for (int y = vy0 + ly; y < vy1; y += 8) {
            const int rm = (max(y - 1, 0) - ry0) * RW, r0 = (y - ry0) * RW, rp = (min(y + 1, H - 1) - ry0) * RW;
            for (int x = vx0 + lx; x < vx1; x += 32) {
                const int c = x - rx0;
                const float R = __fmul_rn(dt, fl[r0 + c].y);
                const Pix<D> m = A[rm + c], i0 = A[r0 + c], p = A[rp + c];
                Pix<D> o;
                if constexpr (D == 1) {
                    o.v[0] = lw1<1>(m.v[0], i0.v[0], p.v[0], R);
                } else {
                    const float b = __double2float_rn(__dmul_rn(0.5, (double)R));
                    const float b2 = __double2float_rn(__dmul_rn(__dmul_rn(0.5, (double)R), (double)R));
#pragma unroll
                    for (int ch = 0; ch < D; ++ch) o.v[ch] = lw4(m.v[ch], i0.v[ch], p.v[ch], b, b2);
                }
                B[r0 + c] = o;
            }
        }
        __syncthreads();
        // X pass, B -> A
        vx0 = vx0 == 0 ? 0 : vx0 + 1;
        vx1 = vx1 == W ? W : vx1 - 1;
        for (int y = vy0 + ly; y < vy1; y += 8) {
            const int r0 = (y - ry0) * RW;
            for (int x = vx0 + lx; x < vx1; x += 32) {
                const int cm = max(x - 1, 0) - rx0, c = x - rx0, cp = min(x + 1, W - 1) - rx0;
                const float R = __fmul_rn(dt, fl[r0 + c].x);
                const Pix<D> m = B[r0 + cm], i0 = B[r0 + c], p = B[r0 + cp];
                Pix<D> o;
                if constexpr (D == 1) {
                    o.v[0] = lw1<0>(m.v[0], i0.v[0], p.v[0], R);
                } else {
                    const float b = __double2float_rn(__dmul_rn(0.5, (double)R));
                    const float b2 = __double2float_rn(__dmul_rn(__dmul_rn(0.5, (double)R), (double)R));
#pragma unroll
                    for (int ch = 0; ch < D; ++ch) o.v[ch] = lw4(m.v[ch], i0.v[ch], p.v[ch], b, b2);
                }
                A[r0 + c] = o;
            }
        }
        __syncthreads();
    }
    // the tile
    const int ox1 = min(tx0 + T, W), oy1 = min(ty0 + T, H);
    for (int y = ty0 + ly; y < oy1; y += 8) {
        float* drow = reinterpret_cast<float*>(reinterpret_cast<char*>(a.dst) + y * a.dst_pitch);
        for (int x = tx0 + lx; x < ox1; x += 32) {
            const Pix<D> o = A[(y - ry0) * RW + (x - rx0)];
            if constexpr (D == 4)
                reinterpret_cast<float4*>(drow)[x] = make_float4(o.v[0], o.v[1], o.v[2], o.v[3]);
            else
                drow[x] = o.v[0];
        }
    }
}

__global__ void rotational_flow_k(LWArgs a) {
    grid_dep_wait();
    grid_dep_launch();
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.W || y >= a.H) return;
    reinterpret_cast<float2*>(reinterpret_cast<char*>(a.flow_out) + y * a.flow_out_pitch)[x] = rotational_flow(a, x, y);
}

// 32 x 32 tiles: a VGA image gives 300 CTAs, several resident per SM (each a few to 164 KB
// of shared memory), which hides the shared-memory and FP64 latency of the passes
int tile_of(int D, int passes) {
    (void)D;
    (void)passes;
    return 32;
}

size_t smem_of(int D, int tile, int passes) {
    const size_t r = (size_t)(tile + 2 * passes);
    return r * r * (8 + 2 * 4 * (size_t)D);
}

template <int D, bool ROT>
cudaError_t launch_lw(LWArgs a, cudaStream_t s) {
    const size_t smem = smem_of(D, a.tile, a.passes);
    // once per device: room for the largest launch (kMaxFused iterations); no static smem
    static std::atomic<unsigned long long> prepared{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(prepared.load() & bit)) {
        e = cudaFuncSetAttribute(lw_tile_k<D, ROT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem_of(D, tile_of(D, kMaxFused), kMaxFused));
        if (e != cudaSuccess) return e;
        prepared.fetch_or(bit);
    }
    const dim3 grid((a.W + a.tile - 1) / a.tile, (a.H + a.tile - 1) / a.tile);
    return launch_k(lw_tile_k<D, ROT>, grid, dim3(32, 8), smem, s, a);
}

// Full propagation: ceil(n / kMaxFused) launches ending in `out`; earlier ones alternate
// with the workspace.  rot: the first launch computes (and writes) the rotational flow.
cudaError_t propagate(LWArgs a, int depth, int iterations, bool rot, float* out, size_t out_pitch, float* ws,
                      size_t ws_pitch, cudaStream_t s) {
    const int n = std::max(iterations, 1);
    a.dt = iterations > 0 ? 1.0f / (float)iterations : 0.0f;  // setIterations, propagation.cu:647-656
    const int launches = (n + kMaxFused - 1) / kMaxFused;
    int done = 0;
    for (int i = 0; i < launches; ++i) {
        const int p = std::min(kMaxFused, n - done);
        const bool to_out = ((launches - 1 - i) % 2) == 0;
        a.dst = to_out ? out : ws;
        a.dst_pitch = to_out ? out_pitch : ws_pitch;
        a.passes = p;
        a.tile = tile_of(depth, p);
        const bool r = rot && i == 0;
        cudaError_t e;
        if (depth == 1)
            e = r ? launch_lw<1, true>(a, s) : launch_lw<1, false>(a, s);
        else
            e = r ? launch_lw<4, true>(a, s) : launch_lw<4, false>(a, s);
        if (e != cudaSuccess) return e;
        if (r) {  // later launches read the flow just written
            a.flow = a.flow_out;
            a.flow_pitch = a.flow_out_pitch;
        }
        a.src = a.dst;
        a.src_pitch = a.dst_pitch;
        done += p;
    }
    return cudaSuccess;
}

bool aligned(const void* p, size_t pitch, size_t row_bytes, size_t align) {
    return p && pitch >= row_bytes && (((uintptr_t)p | pitch) % align) == 0;
}

ff_status fail(ff_status st, const std::string& msg) { return ffb_fail(st, msg); }

ff_status check_common(int depth, int h, int w, int iterations, const float* image, size_t image_pitch, float* out,
                       size_t out_pitch, float* ws, size_t ws_pitch) {
    if (h < 1 || w < 1 || h > 65535 * 32) return fail(FF_ERR_SHAPE, "lax_wendroff: bad height or width");
    if (depth != 1 && depth != 4) return fail(FF_ERR_INVALID_ARGUMENT, "lax_wendroff: image depth should be 1 or 4");
    if (iterations < 0) return fail(FF_ERR_INVALID_ARGUMENT, "lax_wendroff: iterations less than zero");
    const size_t row = (size_t)w * depth * 4, al = depth == 4 ? 16 : 4;
    if (!aligned(image, image_pitch, row, al) || !aligned(out, out_pitch, row, al))
        return fail(FF_ERR_INVALID_ARGUMENT, "lax_wendroff: image and output need aligned rows of width pixels");
    if (image == out) return fail(FF_ERR_INVALID_ARGUMENT, "lax_wendroff: the output must not be the input image");
    if (std::max(iterations, 1) > kMaxFused && (!aligned(ws, ws_pitch, row, al) || ws == image || ws == out))
        return fail(FF_ERR_INVALID_ARGUMENT,
                    "lax_wendroff: more than " + std::to_string(kMaxFused) + " iterations need a workspace image");
    return FF_OK;
}

ff_status cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return FF_OK;
    return fail(FF_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace
}  // namespace ffb

extern "C" {

int ff_lax_wendroff_max_fused(void) { return ffb::kMaxFused; }

ff_status ff_camera_perspective(float focal, int height, int width, float sensor_height, float sensor_width,
                                ff_camera* cam) {
    if (!cam) return ffb::fail(FF_ERR_INVALID_ARGUMENT, "camera_perspective: cam must not be NULL");
    const int imgX = width - 1, imgY = height - 1;
    cam->alphaX = focal * (float)imgX / sensor_width;
    cam->alphaY = focal * (float)imgY / sensor_height;
    cam->centerX = 0.5f * (float)imgX;
    cam->centerY = 0.5f * (float)imgY;
    return FF_OK;
}

ff_status ff_rotational_flow(const ff_camera* cam, float wx, float wy, float wz, float* flow, size_t flow_pitch,
                             int height, int width, void* stream) {
    if (!cam) return ffb::fail(FF_ERR_INVALID_ARGUMENT, "rotational_flow: cam must not be NULL");
    if (height < 1 || width < 1 || height > 65535 * 8) return ffb::fail(FF_ERR_SHAPE, "rotational_flow: bad size");
    if (!ffb::aligned(flow, flow_pitch, (size_t)width * 8, 8))
        return ffb::fail(FF_ERR_INVALID_ARGUMENT, "rotational_flow: flow needs 8-byte aligned rows of width float2");
    ffb::LWArgs a{};
    a.flow_out = flow;
    a.flow_out_pitch = flow_pitch;
    a.ax = cam->alphaX, a.ay = cam->alphaY, a.cx = cam->centerX, a.cy = cam->centerY;
    a.wx = wx, a.wy = wy, a.wz = wz;
    a.H = height, a.W = width;
    return ffb::cuda_status(ffb::launch_k(ffb::rotational_flow_k, dim3((width + 31) / 32, (height + 7) / 8),
                                          dim3(32, 8), 0, (cudaStream_t)stream, a),
                            "rotational_flow");
}

ff_status ff_lax_wendroff(const float* flow, size_t flow_pitch, const float* image, size_t image_pitch, int depth,
                          int height, int width, int iterations, float* out, size_t out_pitch, float* workspace,
                          size_t workspace_pitch, void* stream) {
    ff_status st = ffb::check_common(depth, height, width, iterations, image, image_pitch, out, out_pitch, workspace,
                                     workspace_pitch);
    if (st != FF_OK) return st;
    if (!ffb::aligned(flow, flow_pitch, (size_t)width * 8, 8))
        return ffb::fail(FF_ERR_INVALID_ARGUMENT, "lax_wendroff: flow needs 8-byte aligned rows of width float2");
    ffb::LWArgs a{};
    a.flow = flow;
    a.flow_pitch = flow_pitch;
    a.src = image;
    a.src_pitch = image_pitch;
    a.H = height, a.W = width;
    return ffb::cuda_status(ffb::propagate(a, depth, iterations, false, out, out_pitch, workspace, workspace_pitch,
                                           (cudaStream_t)stream),
                            "lax_wendroff");
}

ff_status ff_rotational_predict(const ff_camera* cam, float wx, float wy, float wz, const float* image,
                                size_t image_pitch, int depth, int height, int width, int iterations, float* flow,
                                size_t flow_pitch, float* out, size_t out_pitch, float* workspace,
                                size_t workspace_pitch, void* stream) {
    if (!cam) return ffb::fail(FF_ERR_INVALID_ARGUMENT, "rotational_predict: cam must not be NULL");
    ff_status st = ffb::check_common(depth, height, width, iterations, image, image_pitch, out, out_pitch, workspace,
                                     workspace_pitch);
    if (st != FF_OK) return st;
    if (!ffb::aligned(flow, flow_pitch, (size_t)width * 8, 8))
        return ffb::fail(FF_ERR_INVALID_ARGUMENT, "rotational_predict: flow needs 8-byte aligned rows of width float2");
    ffb::LWArgs a{};
    a.flow_out = flow;
    a.flow_out_pitch = flow_pitch;
    a.ax = cam->alphaX, a.ay = cam->alphaY, a.cx = cam->centerX, a.cy = cam->centerY;
    a.wx = wx, a.wy = wy, a.wz = wz;
    a.src = image;
    a.src_pitch = image_pitch;
    a.H = height, a.W = width;
    return ffb::cuda_status(ffb::propagate(a, depth, iterations, true, out, out_pitch, workspace, workspace_pitch,
                                           (cudaStream_t)stream),
                            "rotational_predict");
}

}  // extern "C"
