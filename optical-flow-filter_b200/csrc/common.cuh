// Device-side building blocks shared by the flow-filter kernels.
//
// Arithmetic is written with explicit round-to-nearest intrinsics (__fmaf_rn,
// __fmul_rn, __fadd_rn, ...) so that nvcc never contracts or reorders it: the
// results are fixed operation by operation, and each helper states the
// reference expression it reproduces.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ffb {

// ---------------------------------------------------------------- views
template <typename T>
struct View {
    T* ptr;
    size_t pitch;  // bytes
    int h, w;
    __host__ __device__ __forceinline__ T* row(int y) const {
        return reinterpret_cast<T*>(reinterpret_cast<char*>(ptr) + (size_t)y * pitch);
    }
    __host__ __device__ __forceinline__ T& at(int x, int y) const { return row(y)[x]; }
};

template <typename T>
struct CView {
    const T* ptr;
    size_t pitch;
    int h, w;
    __host__ __device__ __forceinline__ const T* row(int y) const {
        return reinterpret_cast<const T*>(reinterpret_cast<const char*>(ptr) + (size_t)y * pitch);
    }
    __host__ __device__ __forceinline__ const T& at(int x, int y) const { return row(y)[x]; }
    // clamp-to-edge read: the reference's textures use cudaAddressModeClamp
    __device__ __forceinline__ T clamped(int x, int y) const {
        x = min(max(x, 0), w - 1);
        y = min(max(y, 0), h - 1);
        return __ldg(row(y) + x);
    }
};

// ---------------------------------------------------------------- arithmetic
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// uint8 -> float exactly as a normalised texture read returns it: v/255 rounded to
// nearest.  q = v*fl(1/255) is refined by one residual step; exhaustive over 0..255
// this equals the correctly rounded quotient.
__device__ __forceinline__ float u8_to_unit(uint32_t v) {
    const float r = 0.0039215688593685627f;  // fl(1/255)
    float fv = (float)v;
    float q = __fmul_rn(fv, r);
    float e = __fmaf_rn(-q, 255.0f, fv);
    return __fmaf_rn(e, r, q);
}

// image read as float: uint8 normalised (v/255) or float as stored
template <typename P>
struct Pix;
template <>
struct Pix<uint8_t> {
    __device__ __forceinline__ static float get(uint8_t v) { return u8_to_unit(v); }
};
template <>
struct Pix<float> {
    __device__ __forceinline__ static float get(float v) { return v; }
};

// imageDown{X,Y}: s = 0.5*c + 0.25*(m + p) in double, stored as float
// (pyramid_k.cu:38, 72).  0.5*c and 0.25*fl(m+p) are exact and their exact sum
// rounds once, so one fused multiply-add over floats gives the same value.
__device__ __forceinline__ float down3(float m, float c, float p) {
    return __fmaf_rn(0.5f, c, __fmul_rn(0.25f, __fadd_rn(m, p)));
}
// (unsigned char)(255*s), truncating (pyramid_k.cu:43, 77)
__device__ __forceinline__ uint8_t quantize_u8(float s) {
    return (uint8_t)__float2uint_rz(__fmul_rn(255.0f, s));
}

// One pixel of the next pyramid level: imageDownX then imageDownY (pyramid_k.cu:14-145),
// the X-pass value at (2x+k, 2y+j) recomputed in registers; the next level is
// (H/2) x (W/2) of in.
template <typename P>
__device__ __forceinline__ P pyramid_val(const CView<P>& in, int x, int y) {
    float xs[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const int sy = min(max(2 * y - 1 + j, 0), in.h - 1);  // X-pass image height = in.h
        float m = Pix<P>::get(in.clamped(2 * x - 1, sy));
        float c = Pix<P>::get(in.clamped(2 * x, sy));
        float p = Pix<P>::get(in.clamped(2 * x + 1, sy));
        float s = down3(m, c, p);
        if constexpr (sizeof(P) == 1) xs[j] = u8_to_unit(quantize_u8(s));
        else xs[j] = s;
    }
    float s = down3(xs[0], xs[1], xs[2]);
    if constexpr (sizeof(P) == 1) return quantize_u8(s);
    else return s;
}
template <typename P>
__device__ __forceinline__ void pyramid_px(const CView<P>& in, const View<P>& out, int x, int y) {
    out.at(x, y) = pyramid_val(in, x, y);
}

// dominant velocity: |v+| - |v-| > 0 ? v+ : v-   (propagation_k.cu:37-40)
__device__ __forceinline__ float dominant(float vm, float vp) {
    return __fsub_rn(fabsf(vp), fabsf(vm)) > 0.0f ? vp : vm;
}

// One upwind sub-step f0 - t*(dv >= 0 ? f0 - fm : fp - f0), t = dt*dv
// (propagation_k.cu:50-53, 175-207).  The reference build fuses the multiply into the
// subtraction for every channel except the last one each kernel writes (flow .y of
// flowPropagate{X,Y}_k, vector .y of flowPropagatePayload{X,Y}_k), so both forms exist.
__device__ __forceinline__ float upwind(float t, float dv, float fm, float f0, float fp) {
    float d = dv >= 0.0f ? __fsub_rn(f0, fm) : __fsub_rn(fp, f0);
    return __fmaf_rn(-t, d, f0);
}
__device__ __forceinline__ float upwind_unfused(float t, float dv, float fm, float f0, float fp) {
    float d = dv >= 0.0f ? __fsub_rn(f0, fm) : __fsub_rn(fp, f0);
    return __fsub_rn(f0, __fmul_rn(t, d));
}

// closed-form 2x2 regularised solve (update_k.cu:43-63, 114-134):
// (gamma I + a a^T)^-1 (gamma f + a Yt) = adj * q / (gamma (gamma + ax^2 + ay^2)).
// Fusion as in the reference build: qx = fma(g, fx, ax*Yt) but qy = fma(ay, Yt, g*fy).
__device__ __forceinline__ void solve2(float gamma, float ax, float ay, float yt, float fx, float fy,
                                       float& ox, float& oy) {
    float n00 = __fmaf_rn(ay, ay, gamma);
    float n11 = __fmaf_rn(ax, ax, gamma);
    float den = __fmaf_rn(ay, ay, n11);
    float n01 = __fmul_rn(-ax, ay);
    float rdet = __frcp_rn(__fmul_rn(gamma, den));
    float qx = __fmaf_rn(gamma, fx, __fmul_rn(ax, yt));
    float qy = __fmaf_rn(ay, yt, __fmul_rn(gamma, fy));
    float ix = __fmaf_rn(n00, qx, __fmul_rn(n01, qy));
    float iy = __fmaf_rn(n01, qx, __fmul_rn(n11, qy));
    ox = __fmul_rn(ix, rdet);
    oy = __fmul_rn(iy, rdet);
}

// max(-m, min(v, m)) with CUDA's fminf/fmaxf NaN rules (update_k.cu:66-67)
__device__ __forceinline__ float clampm(float v, float m) { return fmaxf(-m, fminf(v, m)); }
// isinf + isnan > 0 ? 0 : v  (update_k.cu:70-71)
__device__ __forceinline__ float sanitize(float v) { return (isinf(v) || isnan(v)) ? 0.0f : v; }

// Coarse texel chosen by a normalised-coordinate, point-sampled, clamped texture read
// at u = x/(W-1) over Wc texels (update_k.cu:151-155, texture update.cu:308-313).
// The texture unit truncates u to 21 fractional bits before scaling (measured on
// B200 for every W <= 4200 on both axes); the index is computed here in integers.
__device__ __forceinline__ int upmap_index(int x, int W, int Wc) {
    float u = __fdiv_rn((float)x, (float)(W - 1));
    if (!(u == u)) return 0;
    long long q = (long long)floorf(__fmul_rn(u, 2097152.0f));
    long long i = (q * (long long)Wc) >> 21;
    return (int)min(max(i, 0ll), (long long)(Wc - 1));
}

// image model masks (imagemodel_k.cu:21-22) and box weight (flowsmoothing_k.cu:18-19)
constexpr float kS0 = 0.0625f, kS1 = 0.25f, kS2 = 0.375f;
constexpr float kD0 = -0.125f, kD1 = -0.25f;
constexpr float kBox = 0.2f;

// 5-tap chains accumulated in tap order from +0 as the reference's loops do
// (imagemodel_k.cu:47-50, 100-111; flowsmoothing_k.cu:38-44); the first tap is
// fma(k, a, +0), which differs from k*a only in the sign of a zero result.
__device__ __forceinline__ float smooth5(float a, float b, float c, float d, float e) {
    float s = __fmaf_rn(kS0, a, 0.0f);
    s = __fmaf_rn(kS1, b, s);
    s = __fmaf_rn(kS2, c, s);
    s = __fmaf_rn(kS1, d, s);
    return __fmaf_rn(kS0, e, s);
}
// diff mask {-1/8, -1/4, 0, 1/4, 1/8}: the 0 tap adds 0*c, which leaves the sum unchanged
// for finite c; it is kept so non-finite inputs propagate as in the reference
__device__ __forceinline__ float diff5(float a, float b, float c, float d, float e) {
    float s = __fmaf_rn(kD0, a, 0.0f);
    s = __fmaf_rn(kD1, b, s);
    s = __fmaf_rn(0.0f, c, s);
    s = __fmaf_rn(-kD1, d, s);
    return __fmaf_rn(-kD0, e, s);
}
__device__ __forceinline__ float box5(float a, float b, float c, float d, float e) {
    float s = __fmaf_rn(kBox, a, 0.0f);
    s = __fmaf_rn(kBox, b, s);
    s = __fmaf_rn(kBox, c, s);
    s = __fmaf_rn(kBox, d, s);
    return __fmaf_rn(kBox, e, s);
}

// 5-tap chains on two lanes at once with sm_100's packed two-lane FP32 instructions (two
// channels of a pixel, or one channel of two pixels): each lane is the same IEEE fma.rn as
// the scalar chain's, so the results are identical
__device__ __forceinline__ float2 chain5_pair(float k0, float k1, float k2, float k3, float k4, float2 a, float2 b,
                                              float2 c, float2 d, float2 e) {
    float2 s = __ffma2_rn(make_float2(k0, k0), a, make_float2(0.0f, 0.0f));
    s = __ffma2_rn(make_float2(k1, k1), b, s);
    s = __ffma2_rn(make_float2(k2, k2), c, s);
    s = __ffma2_rn(make_float2(k3, k3), d, s);
    return __ffma2_rn(make_float2(k4, k4), e, s);
}
__device__ __forceinline__ float2 box5_pair(float2 a, float2 b, float2 c, float2 d, float2 e) {
    return chain5_pair(kBox, kBox, kBox, kBox, kBox, a, b, c, d, e);
}
__device__ __forceinline__ float2 smooth5_pair(float2 a, float2 b, float2 c, float2 d, float2 e) {
    return chain5_pair(kS0, kS1, kS2, kS1, kS0, a, b, c, d, e);
}
__device__ __forceinline__ float2 diff5_pair(float2 a, float2 b, float2 c, float2 d, float2 e) {
    return chain5_pair(kD0, kD1, 0.0f, -kD1, -kD0, a, b, c, d, e);
}

// upwind() of both channels of a flow pixel (both fused, as for the payload kernels' flow),
// with packed two-lane instructions; lane for lane the same operations as upwind()
__device__ __forceinline__ float2 upwind_pair(float t, float dv, float2 fm, float2 f0, float2 fp) {
    const float2 back = __fadd2_rn(f0, make_float2(-fm.x, -fm.y));
    const float2 fwd = __fadd2_rn(fp, make_float2(-f0.x, -f0.y));
    const float2 d = dv >= 0.0f ? back : fwd;
    return __ffma2_rn(make_float2(-t, -t), d, f0);
}

}  // namespace ffb
