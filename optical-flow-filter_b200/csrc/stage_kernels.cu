// Per-stage kernels: one thread per output pixel, clamp-to-edge global reads.
//
// These are the unfused building blocks of the hot path.  They serve the stage API
// (ff_stage_*), the phase API of the filters (computeImageModel / Propagation /
// Update) and every (iterations, smoothing) combination the fused level kernels are
// not instantiated for.  Results are identical, bit for bit, to the fused kernels.
#include <cstdlib>

#include "common.cuh"
#include "kernels.h"
#include "launch.cuh"

namespace ffb {

namespace {

constexpr int BX = 32, BY = 8;

inline dim3 grid_for(int w, int h) { return dim3((w + BX - 1) / BX, (h + BY - 1) / BY); }

// imageDownX then imageDownY fused (pyramid_px, common.cuh).  Output (H/2) x (W/2).
template <typename P>
__global__ void pyramid_down_k(CView<P> in, View<P> out) {
    grid_dep_wait();
    grid_dep_launch();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= out.w || y >= out.h) return;
    pyramid_px(in, out, x, y);
}

// Two pyramid steps in one launch: a block stages the level-0 pixels under its 64 x 16
// level-1 tile, plus those the one-pixel level-1 ring around it reads (at clamped
// coordinates), in shared memory with one batch of loads; computes the tile and the ring
// into shared memory, stores the tile, and computes the 32 x 8 level-2 pixels under it from
// the ring: the same values as two pyramid_down_k launches.  Level 1 is H1 x W1 =
// (H/2) x (W/2), level 2 (H1/2) x (W1/2).
constexpr int P2X = 2 * BX, P2Y = 2 * BY;  // level-1 tile
constexpr int S0Y = 2 * P2Y + 5;           // staged level-0 rows: 3 before the tile's, 2 after
constexpr int S0X = 2 * P2X + 8;           // staged level-0 columns: from 4 before the tile's
template <typename P>
__global__ void __launch_bounds__(BX * BY) pyramid_down2_k(CView<P> in, View<P> out1, View<P> out2) {
    __shared__ __align__(16) P s0[S0Y][S0X];
    __shared__ P ring[P2Y + 2][P2X + 2];
    grid_dep_wait();
    grid_dep_launch();
    const int x1 = blockIdx.x * P2X, y1 = blockIdx.y * P2Y;  // level-1 tile origin
    const int H1 = out1.h, W1 = out1.w, H = in.h, W = in.w;
    const int X0 = 2 * x1 - 4, Y0 = 2 * y1 - 3;  // staged level-0 origin (unclamped)
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    constexpr int T = BX * BY;
    // 4-byte words of uint8 rows whose pitch keeps them aligned, else single pixels
    const bool words = sizeof(P) == 1 && (in.pitch & 3) == 0 && ((uintptr_t)in.ptr & 3) == 0;
    if (words) {
        constexpr int WQ = S0X / 4, NS = (S0Y * WQ + T - 1) / T;
        uint32_t v[NS];
#pragma unroll
        for (int u = 0; u < NS; ++u) {
            const int e = tid + T * u, r = e / WQ, c = e - r * WQ;
            if (e < S0Y * WQ) {
                const uint8_t* row = reinterpret_cast<const uint8_t*>(in.row(min(max(Y0 + r, 0), H - 1)));
                const int x = X0 + 4 * c;
                if (x >= 0 && x + 3 < W) {
                    v[u] = __ldg(reinterpret_cast<const uint32_t*>(row + x));
                } else {  // a word beyond an edge: its clamped pixels
                    uint32_t w = 0;
#pragma unroll
                    for (int q = 0; q < 4; ++q) w |= (uint32_t)__ldg(row + min(max(x + q, 0), W - 1)) << (8 * q);
                    v[u] = w;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < NS; ++u) {
            const int e = tid + T * u, r = e / WQ, c = e - r * WQ;
            if (e < S0Y * WQ) reinterpret_cast<uint32_t*>(&s0[r][0])[c] = v[u];
        }
    } else {
        constexpr int NS = (S0Y * S0X + T - 1) / T;
        P v[NS];
#pragma unroll
        for (int u = 0; u < NS; ++u) {
            const int e = tid + T * u, r = e / S0X, c = e - r * S0X;
            if (e < S0Y * S0X) v[u] = in.clamped(X0 + c, Y0 + r);
        }
#pragma unroll
        for (int u = 0; u < NS; ++u) {
            const int e = tid + T * u, r = e / S0X, c = e - r * S0X;
            if (e < S0Y * S0X) s0[r][c] = v[u];
        }
    }
    __syncthreads();
    for (int k = tid; k < (P2X + 2) * (P2Y + 2); k += T) {
        const int i = k % (P2X + 2), j = k / (P2X + 2);
        const int ux = x1 - 1 + i, uy = y1 - 1 + j;  // unclamped level-1 position
        const int cx = min(max(ux, 0), W1 - 1), cy = min(max(uy, 0), H1 - 1);
        // pyramid_val at (cx, cy): level-0 rows 2cy-1..2cy+1, columns 2cx-1..2cx+1, clamped
        float xs[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const P* row = &s0[2 * cy - 1 + q - Y0][2 * cx - 1 - X0];
            const float sv = down3(Pix<P>::get(row[0]), Pix<P>::get(row[1]), Pix<P>::get(row[2]));
            if constexpr (sizeof(P) == 1) xs[q] = u8_to_unit(quantize_u8(sv));
            else xs[q] = sv;
        }
        const float sv = down3(xs[0], xs[1], xs[2]);
        P v;
        if constexpr (sizeof(P) == 1) v = quantize_u8(sv);
        else v = sv;
        ring[j][i] = v;
        if (ux == cx && uy == cy && ux >= x1 && ux < x1 + P2X && uy >= y1 && uy < y1 + P2Y) out1.at(ux, uy) = v;
    }
    __syncthreads();
    const int x2 = x1 / 2 + threadIdx.x, y2 = y1 / 2 + threadIdx.y;
    if (x2 >= out2.w || y2 >= out2.h) return;
    // pyramid_val over level 1, whose clamped reads the ring already holds
    float xs[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const int r = 2 * y2 - 1 + j - (y1 - 1);
        const int c = 2 * x2 - 1 - (x1 - 1);
        const float s = down3(Pix<P>::get(ring[r][c]), Pix<P>::get(ring[r][c + 1]), Pix<P>::get(ring[r][c + 2]));
        if constexpr (sizeof(P) == 1) xs[j] = u8_to_unit(quantize_u8(s));
        else xs[j] = s;
    }
    const float s = down3(xs[0], xs[1], xs[2]);
    if constexpr (sizeof(P) == 1) out2.at(x2, y2) = quantize_u8(s);
    else out2.at(x2, y2) = s;
}

// scalarProductF2_k (misc_k.cu:18-38): every float2 of a field times a scalar
__global__ void scale_flow_k(CView<float2> in, float k, View<float2> out) {
    grid_dep_wait();
    grid_dep_launch();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= out.w || y >= out.h) return;
    const float2 v = in.at(x, y);
    out.at(x, y) = make_float2(__fmul_rn(k, v.x), __fmul_rn(k, v.y));
}

// imagePrefilter_k + imageModel_k fused per pixel (imagemodel_k.cu:31-133):
// bY = Y-blur, bX = X-blur of the input; a0 = X-blur(bY), ax = X-diff(bY), ay = Y-diff(bX).
template <typename P>
__global__ void image_model_k(CView<P> img, View<float> a0, View<float2> grad) {
    grid_dep_wait();
    grid_dep_launch();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a0.w || y >= a0.h) return;
    const int W = img.w, H = img.h;
    float by[5], bx[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        // prefilter output at (x + c - 2, y), clamped as a texture read of it
        const int xc = min(max(x + c - 2, 0), W - 1);
        float v[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) v[r] = Pix<P>::get(img.clamped(xc, y + r - 2));
        by[c] = smooth5(v[0], v[1], v[2], v[3], v[4]);
    }
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        const int yr = min(max(y + r - 2, 0), H - 1);
        float v[5];
#pragma unroll
        for (int c = 0; c < 5; ++c) v[c] = Pix<P>::get(img.clamped(x + c - 2, yr));
        bx[r] = smooth5(v[0], v[1], v[2], v[3], v[4]);
    }
    a0.at(x, y) = smooth5(by[0], by[1], by[2], by[3], by[4]);
    grad.at(x, y) = make_float2(diff5(by[0], by[1], by[2], by[3], by[4]), diff5(bx[0], bx[1], bx[2], bx[3], bx[4]));
}

// One direction of an upwind sub-step (flowPropagate{X,Y}_k, flowPropagatePayload{X,Y}_k,
// propagation_k.cu:16-334).  AXIS 0 = X, 1 = Y.  Payload pointers may be null.
template <int AXIS, bool PAYLOAD>
__global__ void propagate_pass_k(CView<float2> fl, CView<float> sc, CView<float2> ve, View<float2> ofl,
                                 View<float> osc, View<float2> ove, float dt, int border) {
    grid_dep_wait();
    grid_dep_launch();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int W = ofl.w, H = ofl.h;
    if (x >= W || y >= H) return;
    const int xm = AXIS == 0 ? x - 1 : x, xp = AXIS == 0 ? x + 1 : x;
    const int ym = AXIS == 1 ? y - 1 : y, yp = AXIS == 1 ? y + 1 : y;
    const float2 fm = fl.clamped(xm, ym), f0 = fl.clamped(x, y), fp = fl.clamped(xp, yp);
    const float dv = AXIS == 0 ? dominant(fm.x, fp.x) : dominant(fm.y, fp.y);
    const float t = __fmul_rn(dt, dv);
    const bool in = (x >= border && x < W - border) && (y >= border && y < H - border);
    float2 o;
    o.x = in ? upwind(t, dv, fm.x, f0.x, fp.x) : f0.x;
    if constexpr (PAYLOAD) o.y = in ? upwind(t, dv, fm.y, f0.y, fp.y) : f0.y;
    else o.y = in ? upwind_unfused(t, dv, fm.y, f0.y, fp.y) : f0.y;
    ofl.at(x, y) = o;
    if constexpr (PAYLOAD) {
        const float sm = sc.clamped(xm, ym), s0 = sc.clamped(x, y), sp = sc.clamped(xp, yp);
        osc.at(x, y) = in ? upwind(t, dv, sm, s0, sp) : s0;
        const float2 vm = ve.clamped(xm, ym), v0 = ve.clamped(x, y), vp = ve.clamped(xp, yp);
        float2 ov;
        ov.x = in ? upwind(t, dv, vm.x, v0.x, vp.x) : v0.x;
        ov.y = in ? upwind_unfused(t, dv, vm.y, v0.y, vp.y) : v0.y;
        ove.at(x, y) = ov;
    }
}

// flowUpdate_k (update_k.cu:15-79).  `first` substitutes the old image by a0, as the
// first-frame copy does (flowfilter.cu:132-141).  a0_old may alias out_image only
// when each pixel is read before it is written (true here: one thread per pixel).
__global__ void update_k(CView<float> a0, CView<float2> grad, CView<float> a0_old, CView<float2> flow,
                         View<float2> out_flow, View<float> out_image, float gamma, float maxflow, int first) {
    grid_dep_wait();
    grid_dep_launch();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= out_flow.w || y >= out_flow.h) return;
    const float2 a = grad.at(x, y);
    const float c = a0.at(x, y);
    const float old = first ? c : a0_old.at(x, y);
    const float2 f = flow.at(x, y);
    float ox, oy;
    solve2(gamma, a.x, a.y, __fsub_rn(old, c), f.x, f.y, ox, oy);
    out_flow.at(x, y) = make_float2(sanitize(clampm(ox, maxflow)), sanitize(clampm(oy, maxflow)));
    out_image.at(x, y) = c;
}

// deltaFlowUpdate_k (update_k.cu:82-173); `first` as above (flowfilter.cu:484-494).
__global__ void delta_update_k(CView<float> a0, CView<float2> grad, CView<float> a0_old, CView<float2> delta,
                               CView<float2> coarse, View<float2> out_flow, View<float2> out_delta,
                               View<float> out_image, float gamma, float maxflow, int first) {
    grid_dep_wait();
    grid_dep_launch();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int W = out_flow.w, H = out_flow.h;
    if (x >= W || y >= H) return;
    const float2 a = grad.at(x, y);
    const float c = a0.at(x, y);
    const float old = first ? c : a0_old.at(x, y);
    const float2 d = delta.at(x, y);
    float dx, dy;
    solve2(gamma, a.x, a.y, __fsub_rn(old, c), d.x, d.y, dx, dy);
    const float hm = __fmul_rn(0.5f, maxflow);
    dx = clampm(sanitize(dx), hm);
    dy = clampm(sanitize(dy), hm);
    const float2 up = coarse.at(upmap_index(x, W, coarse.w), upmap_index(y, H, coarse.h));
    const float fx = __fadd_rn(dx, __fmul_rn(2.0f, up.x));
    const float fy = __fadd_rn(dy, __fmul_rn(2.0f, up.y));
    out_delta.at(x, y) = make_float2(dx, dy);
    out_flow.at(x, y) = make_float2(clampm(fx, maxflow), clampm(fy, maxflow));
    out_image.at(x, y) = c;
}

// flowSmooth{X,Y}_k (flowsmoothing_k.cu:21-87)
template <int AXIS>
__global__ void smooth_pass_k(CView<float2> in, View<float2> out) {
    grid_dep_wait();
    grid_dep_launch();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= out.w || y >= out.h) return;
    float2 v[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) v[k] = AXIS == 0 ? in.clamped(x + k - 2, y) : in.clamped(x, y + k - 2);
    out.at(x, y) = make_float2(box5(v[0].x, v[1].x, v[2].x, v[3].x, v[4].x),
                               box5(v[0].y, v[1].y, v[2].y, v[3].y, v[4].y));
}

template <typename T>
CView<T> cv(const View<T>& v) {
    return CView<T>{v.ptr, v.pitch, v.h, v.w};
}

}  // namespace

// ------------------------------------------------------------------ launchers
bool pdl_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("FFB_PDL");
        return !(v && v[0] == '0');
    }();
    return on;
}

cudaError_t launch_scale_flow(const float* in, size_t in_pitch, int H, int W, float k, float* out, size_t out_pitch,
                              cudaStream_t s) {
    return launch_k(scale_flow_k, grid_for(W, H), dim3(BX, BY), 0, s, CView<float2>{(const float2*)in, in_pitch, H, W},
                    k, View<float2>{(float2*)out, out_pitch, H, W});
}

cudaError_t launch_pyramid_down2(const void* in, size_t in_pitch, int item, int H, int W, void* out1,
                                 size_t out1_pitch, void* out2, size_t out2_pitch, cudaStream_t s) {
    const int h1 = H / 2, w1 = W / 2, h2 = h1 / 2, w2 = w1 / 2;
    if (h2 <= 0 || w2 <= 0) return cudaErrorInvalidValue;
    const dim3 grid((w1 + P2X - 1) / P2X, (h1 + P2Y - 1) / P2Y);
    if (item == 1)
        return launch_k(pyramid_down2_k<uint8_t>, grid, dim3(BX, BY), 0, s,
                        CView<uint8_t>{(const uint8_t*)in, in_pitch, H, W},
                        View<uint8_t>{(uint8_t*)out1, out1_pitch, h1, w1}, View<uint8_t>{(uint8_t*)out2, out2_pitch, h2, w2});
    return launch_k(pyramid_down2_k<float>, grid, dim3(BX, BY), 0, s, CView<float>{(const float*)in, in_pitch, H, W},
                    View<float>{(float*)out1, out1_pitch, h1, w1}, View<float>{(float*)out2, out2_pitch, h2, w2});
}

cudaError_t launch_pyramid_down(const void* in, size_t in_pitch, int item, int H, int W, void* out,
                                size_t out_pitch, cudaStream_t s) {
    const int h = H / 2, w = W / 2;
    if (h <= 0 || w <= 0) return cudaSuccess;
    if (item == 1) {
        return launch_k(pyramid_down_k<uint8_t>, grid_for(w, h), dim3(BX, BY), 0, s,
                        CView<uint8_t>{(const uint8_t*)in, in_pitch, H, W}, View<uint8_t>{(uint8_t*)out, out_pitch, h, w});
    } else {
        return launch_k(pyramid_down_k<float>, grid_for(w, h), dim3(BX, BY), 0, s,
                        CView<float>{(const float*)in, in_pitch, H, W}, View<float>{(float*)out, out_pitch, h, w});
    }
    return cudaGetLastError();
}

cudaError_t launch_image_model(const void* img, size_t pitch, int item, int H, int W, float* a0, size_t a0p,
                               float* grad, size_t gp, cudaStream_t s) {
    View<float> A{a0, a0p, H, W};
    View<float2> G{(float2*)grad, gp, H, W};
    if (item == 1)
        return launch_k(image_model_k<uint8_t>, grid_for(W, H), dim3(BX, BY), 0, s,
                        CView<uint8_t>{(const uint8_t*)img, pitch, H, W}, A, G);
    return launch_k(image_model_k<float>, grid_for(W, H), dim3(BX, BY), 0, s,
                    CView<float>{(const float*)img, pitch, H, W}, A, G);
}

// N sub-steps ping-ponging between `out` and the workspace `tmp` (same shape as out):
// X: in -> tmp, Y: tmp -> out, then X: out -> tmp, Y: tmp -> out, ...
cudaError_t launch_propagate(const float* flow, size_t fp, int H, int W, int N, int border, float* out, size_t op,
                             float* tmp, size_t tp, cudaStream_t s) {
    const float dt = 1.0f / (float)N;  // FlowPropagator::setIterations (propagation.cu:146-147)
    CView<float> nsc{nullptr, 0, H, W};
    CView<float2> nve{nullptr, 0, H, W};
    View<float> nosc{nullptr, 0, H, W};
    View<float2> nove{nullptr, 0, H, W};
    View<float2> O{(float2*)out, op, H, W}, T{(float2*)tmp, tp, H, W};
    CView<float2> src{(const float2*)flow, fp, H, W};
    for (int n = 0; n < N; ++n) {
        cudaError_t e = launch_k(propagate_pass_k<0, false>, grid_for(W, H), dim3(BX, BY), 0, s, src, nsc, nve, T,
                                 nosc, nove, dt, border);
        if (e != cudaSuccess) return e;
        e = launch_k(propagate_pass_k<1, false>, grid_for(W, H), dim3(BX, BY), 0, s, cv(T), nsc, nve, O, nosc, nove,
                     dt, border);
        if (e != cudaSuccess) return e;
        src = cv(O);
    }
    return cudaSuccess;
}

cudaError_t launch_propagate_payload(const float* flow, size_t fp, const float* sc, size_t sp, const float* ve,
                                     size_t vp, int H, int W, int N, int border, float* of, size_t ofp, float* os,
                                     size_t osp, float* ov, size_t ovp, float* tf, size_t tfp, float* ts, size_t tsp,
                                     float* tv, size_t tvp, cudaStream_t s) {
    const float dt = 1.0f / (float)N;
    View<float2> OF{(float2*)of, ofp, H, W}, TF{(float2*)tf, tfp, H, W};
    View<float> OS{os, osp, H, W}, TS{ts, tsp, H, W};
    View<float2> OV{(float2*)ov, ovp, H, W}, TV{(float2*)tv, tvp, H, W};
    CView<float2> sf{(const float2*)flow, fp, H, W};
    CView<float> ss{sc, sp, H, W};
    CView<float2> sv{(const float2*)ve, vp, H, W};
    for (int n = 0; n < N; ++n) {
        cudaError_t e = launch_k(propagate_pass_k<0, true>, grid_for(W, H), dim3(BX, BY), 0, s, sf, ss, sv, TF, TS, TV,
                                 dt, border);
        if (e != cudaSuccess) return e;
        e = launch_k(propagate_pass_k<1, true>, grid_for(W, H), dim3(BX, BY), 0, s, cv(TF), cv(TS), cv(TV), OF, OS,
                     OV, dt, border);
        if (e != cudaSuccess) return e;
        sf = cv(OF);
        ss = cv(OS);
        sv = cv(OV);
    }
    return cudaSuccess;
}

cudaError_t launch_update(const float* a0, size_t a0p, const float* grad, size_t gp, const float* old, size_t olp,
                          const float* flow, size_t fp, int H, int W, float gamma, float maxflow, float* of,
                          size_t ofp, float* oi, size_t oip, int first, cudaStream_t s) {
    return launch_k(
        update_k, grid_for(W, H), dim3(BX, BY), 0, s, CView<float>{a0, a0p, H, W}, CView<float2>{(const float2*)grad, gp, H, W}, CView<float>{old, olp, H, W},
        CView<float2>{(const float2*)flow, fp, H, W}, View<float2>{(float2*)of, ofp, H, W}, View<float>{oi, oip, H, W},
        gamma, maxflow, first);
}

cudaError_t launch_delta_update(const float* a0, size_t a0p, const float* grad, size_t gp, const float* old,
                                size_t olp, const float* delta, size_t dp, const float* coarse, size_t cp, int Hc,
                                int Wc, int H, int W, float gamma, float maxflow, float* of, size_t ofp, float* od,
                                size_t odp, float* oi, size_t oip, int first, cudaStream_t s) {
    return launch_k(
        delta_update_k, grid_for(W, H), dim3(BX, BY), 0, s, CView<float>{a0, a0p, H, W}, CView<float2>{(const float2*)grad, gp, H, W}, CView<float>{old, olp, H, W},
        CView<float2>{(const float2*)delta, dp, H, W}, CView<float2>{(const float2*)coarse, cp, Hc, Wc},
        View<float2>{(float2*)of, ofp, H, W}, View<float2>{(float2*)od, odp, H, W}, View<float>{oi, oip, H, W}, gamma,
        maxflow, first);
}

// S iterations: X: in -> tmp, Y: tmp -> out, X: out -> tmp, ...
cudaError_t launch_smooth(const float* flow, size_t fp, int H, int W, int S, float* out, size_t op, float* tmp,
                          size_t tp, cudaStream_t s) {
    View<float2> O{(float2*)out, op, H, W}, T{(float2*)tmp, tp, H, W};
    CView<float2> src{(const float2*)flow, fp, H, W};
    for (int k = 0; k < S; ++k) {
        cudaError_t e = launch_k(smooth_pass_k<0>, grid_for(W, H), dim3(BX, BY), 0, s, src, T);
        if (e != cudaSuccess) return e;
        e = launch_k(smooth_pass_k<1>, grid_for(W, H), dim3(BX, BY), 0, s, cv(T), O);
        if (e != cudaSuccess) return e;
        src = cv(O);
    }
    return cudaSuccess;
}

}  // namespace ffb
