// Differentiable stages: forward and adjoint (backward) kernels of every stage of the
// float-input filter, in float and in double, over a batch of B images (no reference
// counterpart; the forward recurrence is the reference's, float path).
//
// Layout: dense arrays, scalar fields [B][H][W], two-channel fields [B][H][W][2].  The float
// forward kernels repeat the per-stage kernels' arithmetic operation for operation
// (stage_kernels.cu), so with the default 0.2 smoothing weights the float forward equals the
// reference.  The smoothing weights (5 per level) and gamma (1 per level) are device
// scalars, so they can be trained without a host round trip.
//
// Backward kernels take the forward inputs (the forward is recomputed locally), follow the
// branch the forward took at every upwind, dominant-velocity and clamp decision (the
// gradient of a clamped or sanitised value is zero) and ADD into the input gradients:
// gradient buffers start at zero (or hold earlier contributions).  Stencil adjoints are in
// gather form (each input pixel collects from the outputs that read it, clamps included), so
// they need no atomics and are deterministic; only the coarse-flow gradient of the delta
// update is scattered with atomics.  Gradients of the per-level scalars are reduced per
// block, then added once per block.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <initializer_list>
#include <stdexcept>
#include <string>
#include <vector>

#include "common.cuh"
#include "ffb200.h"
#include "kernels.h"
#include "launch.cuh"

namespace ffb {
namespace diff {

// ------------------------------------------------------------------ arithmetic per type
template <typename T>
struct Ar;
template <>
struct Ar<float> {
    __device__ static float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
    __device__ static float add(float a, float b) { return __fadd_rn(a, b); }
    __device__ static float sub(float a, float b) { return __fsub_rn(a, b); }
    __device__ static float rcp(float a) { return __frcp_rn(a); }
    __device__ static bool finite(float a) { return isfinite(a); }
};
template <>
struct Ar<double> {
    __device__ static double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
    __device__ static double mul(double a, double b) { return __dmul_rn(a, b); }
    __device__ static double add(double a, double b) { return __dadd_rn(a, b); }
    __device__ static double sub(double a, double b) { return __dsub_rn(a, b); }
    __device__ static double rcp(double a) { return __drcp_rn(a); }
    __device__ static bool finite(double a) { return isfinite(a); }
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }

template <typename T>
__device__ __forceinline__ T down3(T m, T c, T p) {
    return Ar<T>::fma(T(0.5), c, Ar<T>::mul(T(0.25), Ar<T>::add(m, p)));
}
template <typename T>
__device__ __forceinline__ T chain5(const T* k, T a, T b, T c, T d, T e) {
    T s = Ar<T>::fma(k[0], a, T(0));
    s = Ar<T>::fma(k[1], b, s);
    s = Ar<T>::fma(k[2], c, s);
    s = Ar<T>::fma(k[3], d, s);
    return Ar<T>::fma(k[4], e, s);
}
template <typename T>
struct Masks {
    T s[5], d[5];
    __device__ Masks() {
        s[0] = T(0.0625); s[1] = T(0.25); s[2] = T(0.375); s[3] = T(0.25); s[4] = T(0.0625);
        d[0] = T(-0.125); d[1] = T(-0.25); d[2] = T(0); d[3] = T(0.25); d[4] = T(0.125);
    }
};
template <typename T>
__device__ __forceinline__ T dominant(T vm, T vp) {
    return Ar<T>::sub(fabs(vp), fabs(vm)) > T(0) ? vp : vm;
}
template <typename T>
__device__ __forceinline__ T upwind(T t, T dv, T fm, T f0, T fp) {
    T d = dv >= T(0) ? Ar<T>::sub(f0, fm) : Ar<T>::sub(fp, f0);
    return Ar<T>::fma(-t, d, f0);
}
template <typename T>
__device__ __forceinline__ T upwind_unfused(T t, T dv, T fm, T f0, T fp) {
    T d = dv >= T(0) ? Ar<T>::sub(f0, fm) : Ar<T>::sub(fp, f0);
    return Ar<T>::sub(f0, Ar<T>::mul(t, d));
}
template <typename T>
__device__ __forceinline__ T clampm(T v, T m) {
    return fmax(-m, fmin(v, m));
}
template <typename T>
__device__ __forceinline__ T sanitize(T v) {
    return Ar<T>::finite(v) ? v : T(0);
}

// the 2x2 solve with its intermediates (update_k.cu:43-63)
template <typename T>
struct Solve {
    T n00, n11, n01, rdet, ox, oy;
    __device__ Solve(T g, T ax, T ay, T yt, T fx, T fy) {
        n00 = Ar<T>::fma(ay, ay, g);
        n11 = Ar<T>::fma(ax, ax, g);
        const T den = Ar<T>::fma(ay, ay, n11);
        n01 = Ar<T>::mul(-ax, ay);
        rdet = Ar<T>::rcp(Ar<T>::mul(g, den));
        const T qx = Ar<T>::fma(g, fx, Ar<T>::mul(ax, yt));
        const T qy = Ar<T>::fma(ay, yt, Ar<T>::mul(g, fy));
        const T ix = Ar<T>::fma(n00, qx, Ar<T>::mul(n01, qy));
        const T iy = Ar<T>::fma(n01, qx, Ar<T>::mul(n11, qy));
        ox = Ar<T>::mul(ix, rdet);
        oy = Ar<T>::mul(iy, rdet);
    }
};

// adjoint of o = (g I + a a^T)^-1 (g f + a yt) for the output gradient (gx, gy)
template <typename T>
struct SolveGrad {
    T gfx, gfy, gyt, gax, gay, gg;
    __device__ SolveGrad(const Solve<T>& s, T g, T ax, T ay, T yt, T fx, T fy, T gx, T gy) {
        const T lx = s.rdet * (s.n00 * gx + s.n01 * gy);
        const T ly = s.rdet * (s.n01 * gx + s.n11 * gy);
        gfx = g * lx;
        gfy = g * ly;
        gyt = ax * lx + ay * ly;
        const T oa = s.ox * ax + s.oy * ay, la = lx * ax + ly * ay;
        gax = yt * lx - lx * oa - s.ox * la;
        gay = yt * ly - ly * oa - s.oy * la;
        gg = (fx * lx + fy * ly) - (lx * s.ox + ly * s.oy);
    }
};

template <typename T>
__device__ __forceinline__ void atomic_add(T* p, T v) {
    atomicAdd(p, v);
}

// block-wide sum of one value per thread, added once per block into *dst
template <typename T>
__device__ __forceinline__ void block_add(T v, T* dst) {
    __shared__ T part[32];
    const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
    const int warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) part[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x * blockDim.y + 31) >> 5;
    if (warp == 0) {
        T s = lane < nw ? part[lane] : T(0);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) atomicAdd(dst, s);
    }
}

// block-wide sums of NV values per thread in one pass; thread k < NV writes sum k to dst[k]
// (added atomically if `atomic`, else stored: one slot set per block, reduced later)
template <typename T, int NV>
__device__ __forceinline__ void block_sum(const T (&v)[NV], T* dst, bool atomic) {
    __shared__ T part[NV][32];
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    const int nw = (blockDim.x * blockDim.y + 31) >> 5;
    for (int k = 0; k < NV; ++k) {
        T x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) part[k][warp] = x;
    }
    __syncthreads();
    if (t < NV) {
        T acc = T(0);
        for (int w = 0; w < nw; ++w) acc += part[t][w];
        if (atomic) atomicAdd(&dst[t], acc);
        else dst[t] = acc;
    }
}

__device__ __forceinline__ size_t block_linear() {
    return blockIdx.x + (size_t)gridDim.x * (blockIdx.y + (size_t)gridDim.y * blockIdx.z);
}

// a pair of T (the two channels of a flow pixel) as one vector access
template <typename T>
struct Pair;
template <>
struct Pair<float> {
    using V = float2;
};
template <>
struct Pair<double> {
    using V = double2;
};
template <typename T>
__device__ __forceinline__ typename Pair<T>::V ld2(const T* p, size_t k) {
    return reinterpret_cast<const typename Pair<T>::V*>(p)[k];
}

// write or add one gradient value
template <bool ACC, typename T>
__device__ __forceinline__ void put(T& dst, T v) {
    if constexpr (ACC) dst += v;
    else dst = v;
}

#define PIX_SETUP                                              \
    const int x = blockIdx.x * blockDim.x + threadIdx.x;       \
    const int y = blockIdx.y * blockDim.y + threadIdx.y;       \
    const size_t b = blockIdx.z;                               \
    const bool live = x < W && y < H;

// ------------------------------------------------------------------ pyramid (float path)
template <typename T>
__global__ void pyr_fwd_k(const T* __restrict__ in, T* __restrict__ out, int H, int W) {
    grid_dep_wait();
    grid_dep_launch();
    const int h = H / 2, w = W / 2;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    const size_t b = blockIdx.z;
    if (x >= w || y >= h) return;
    const T* I = in + b * H * W;
    T xs[3];
    for (int j = 0; j < 3; ++j) {
        const int sy = clampi(2 * y - 1 + j, 0, H - 1);
        xs[j] = down3(I[sy * W + clampi(2 * x - 1, 0, W - 1)], I[sy * W + clampi(2 * x, 0, W - 1)],
                      I[sy * W + clampi(2 * x + 1, 0, W - 1)]);
    }
    out[(b * h + y) * w + x] = down3(xs[0], xs[1], xs[2]);
}

// gather form: input pixel (X, Y) sums the contributions of the outputs whose 3x3 stencil
// (after clamping) reads it; outputs x in [X/2 - 1, X/2 + 1] cover every case
template <typename T>
__global__ void pyr_bwd_k(const T* __restrict__ gout, T* gin, int H, int W) {
    grid_dep_wait();
    grid_dep_launch();
    const int h = H / 2, w = W / 2;
    PIX_SETUP
    if (!live) return;
    const T wt[3] = {T(0.25), T(0.5), T(0.25)};
    const T* G = gout + b * h * w;
    T acc = T(0);
    for (int yo = max(y / 2 - 1, 0); yo <= min(y / 2 + 1, h - 1); ++yo) {
        T wy = T(0);
        for (int j = 0; j < 3; ++j)
            if (clampi(2 * yo - 1 + j, 0, H - 1) == y) wy += wt[j];
        if (wy == T(0)) continue;
        for (int xo = max(x / 2 - 1, 0); xo <= min(x / 2 + 1, w - 1); ++xo) {
            T wx = T(0);
            for (int k = 0; k < 3; ++k)
                if (clampi(2 * xo - 1 + k, 0, W - 1) == x) wx += wt[k];
            if (wx != T(0)) acc += G[yo * w + xo] * wy * wx;
        }
    }
    gin[(b * H + y) * W + x] += acc;
}

// ------------------------------------------------------------------ image model
template <typename T>
__global__ void model_fwd_k(const T* __restrict__ img, T* __restrict__ a0, T* __restrict__ grad, int H, int W) {
    grid_dep_wait();
    grid_dep_launch();
    PIX_SETUP
    if (!live) return;
    const Masks<T> M;
    const T* I = img + b * H * W;
    T by[5], bx[5];
    for (int c = 0; c < 5; ++c) {
        const int xc = clampi(x + c - 2, 0, W - 1);
        T v[5];
        for (int r = 0; r < 5; ++r) v[r] = I[clampi(y + r - 2, 0, H - 1) * W + xc];
        by[c] = chain5(M.s, v[0], v[1], v[2], v[3], v[4]);
    }
    for (int r = 0; r < 5; ++r) {
        const int yr = clampi(y + r - 2, 0, H - 1);
        T v[5];
        for (int c = 0; c < 5; ++c) v[c] = I[yr * W + clampi(x + c - 2, 0, W - 1)];
        bx[r] = chain5(M.s, v[0], v[1], v[2], v[3], v[4]);
    }
    const size_t k = (b * H + y) * W + x;
    a0[k] = chain5(M.s, by[0], by[1], by[2], by[3], by[4]);
    grad[2 * k] = chain5(M.d, by[0], by[1], by[2], by[3], by[4]);
    grad[2 * k + 1] = chain5(M.d, bx[0], bx[1], bx[2], bx[3], bx[4]);
}

// weight of tap k of a clamped 5-tap stencil centred at output i that lands on index j
// (several taps land on the edge index at the borders), summed over taps
template <typename T>
__device__ __forceinline__ T tap_weight(const T* w, int i, int j, int n) {
    T acc = T(0);
    for (int k = 0; k < 5; ++k)
        if (clampi(i + k - 2, 0, n - 1) == j) acc += w[k];
    return acc;
}

// tap_weight where the stencil cannot reach a clamp (j - 2 .. j + 2 inside): the one tap j - i + 2
template <typename T>
__device__ __forceinline__ T tap_w(const T* w, int i, int j, int n, bool inner) {
    return inner ? w[j - i + 2] : tap_weight(w, i, j, n);
}

// step 1 (gather): gradients of the Y blur by (used by a0 and ax along X) and of the X blur
// bx (used by ay along Y) at this pixel
template <typename T>
__global__ void model_bwd1_k(const T* __restrict__ ga0, const T* __restrict__ ggrad, T* gby, T* gbx, int H, int W) {
    grid_dep_wait();
    grid_dep_launch();
    PIX_SETUP
    if (!live) return;
    const Masks<T> M;
    const size_t row = (b * H + y) * W;
    const bool ix = x >= 2 && x + 2 <= W - 1, iy = y >= 2 && y + 2 <= H - 1;
    T aby = T(0), abx = T(0);
    for (int i = max(x - 2, 0); i <= min(x + 2, W - 1); ++i) {
        const T ws = tap_w(M.s, i, x, W, ix), wd = tap_w(M.d, i, x, W, ix);
        aby += ws * ga0[row + i] + wd * ggrad[2 * (row + i)];
    }
    for (int i = max(y - 2, 0); i <= min(y + 2, H - 1); ++i)
        abx += tap_w(M.d, i, y, H, iy) * ggrad[2 * ((b * H + i) * W + x) + 1];
    gby[row + x] = aby;
    gbx[row + x] = abx;
}

// step 2 (gather): by = Y blur of the image, bx = X blur of the image
template <typename T, bool ACC = true>
__global__ void model_bwd2_k(const T* __restrict__ gby, const T* __restrict__ gbx, T* gimg, int H, int W) {
    grid_dep_wait();
    grid_dep_launch();
    PIX_SETUP
    if (!live) return;
    const Masks<T> M;
    const bool ix = x >= 2 && x + 2 <= W - 1, iy = y >= 2 && y + 2 <= H - 1;
    T acc = T(0);
    for (int i = max(y - 2, 0); i <= min(y + 2, H - 1); ++i) acc += tap_w(M.s, i, y, H, iy) * gby[(b * H + i) * W + x];
    const size_t row = (b * H + y) * W;
    for (int i = max(x - 2, 0); i <= min(x + 2, W - 1); ++i) acc += tap_w(M.s, i, x, W, ix) * gbx[row + i];
    put<ACC>(gimg[row + x], acc);
}

// ------------------------------------------------------------------ propagation sub-step
template <typename T, int AXIS, bool PAYLOAD>
__global__ void prop_fwd_k(const T* __restrict__ f, const T* __restrict__ s, const T* __restrict__ v, T* __restrict__ fo,
                           T* __restrict__ so, T* __restrict__ vo, int H, int W, T dt, int border) {
    grid_dep_wait();
    grid_dep_launch();
    PIX_SETUP
    if (!live) return;
    const int xm = AXIS == 0 ? max(x - 1, 0) : x, xp = AXIS == 0 ? min(x + 1, W - 1) : x;
    const int ym = AXIS == 1 ? max(y - 1, 0) : y, yp = AXIS == 1 ? min(y + 1, H - 1) : y;
    const size_t k = (b * H + y) * W + x, km = (b * H + ym) * W + xm, kp = (b * H + yp) * W + xp;
    const T fmx = f[2 * km], fmy = f[2 * km + 1], f0x = f[2 * k], f0y = f[2 * k + 1], fpx = f[2 * kp], fpy = f[2 * kp + 1];
    const T dv = AXIS == 0 ? dominant(fmx, fpx) : dominant(fmy, fpy);
    const T t = Ar<T>::mul(dt, dv);
    const bool in = x >= border && x < W - border && y >= border && y < H - border;
    fo[2 * k] = in ? upwind(t, dv, fmx, f0x, fpx) : f0x;
    fo[2 * k + 1] = in ? (PAYLOAD ? upwind(t, dv, fmy, f0y, fpy) : upwind_unfused(t, dv, fmy, f0y, fpy)) : f0y;
    if constexpr (PAYLOAD) {
        so[k] = in ? upwind(t, dv, s[km], s[k], s[kp]) : s[k];
        vo[2 * k] = in ? upwind(t, dv, v[2 * km], v[2 * k], v[2 * kp]) : v[2 * k];
        vo[2 * k + 1] = in ? upwind_unfused(t, dv, v[2 * km + 1], v[2 * k + 1], v[2 * kp + 1]) : v[2 * k + 1];
    }
}

// Gather-form adjoint of one upwind sub-step at position j of a line of n positions along
// the sub-step's axis: the gradients of the input channels at j, collected from the outputs
// i in {j-1, j, j+1} whose clamped stencil (i-1, i, i+1) reads j, recomputing each output's
// dominant velocity, upwind branch and border freeze.  chan(p, o): every input channel at
// position p into o; gchan(p, o): every output-gradient channel at p (p always inside the
// line).  Channels: flow x, flow y [, scalar, vector x, vector y]; line_in: the line lies
// inside the border across the axis.
template <typename T, int AXIS, bool PAYLOAD, typename CH, typename GO>
__device__ __forceinline__ void prop_adj_at(int j, int n, bool line_in, int border, T dt, const CH& chan,
                                            const GO& gchan, T (&acc)[PAYLOAD ? 5 : 2]) {
    constexpr int NC = PAYLOAD ? 5 : 2;
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] = T(0);
    if (j >= 2 && j + 2 <= n - 1) {
        // away from the line ends no index clamps: the five positions j-2..j+2 in registers,
        // the same results as the general loop below
        T px[5][NC], gx[3][NC];
#pragma unroll
        for (int p = 0; p < 5; ++p) chan(j - 2 + p, px[p]);
#pragma unroll
        for (int q = 0; q < 3; ++q) gchan(j - 1 + q, gx[q]);
        // branch-free: every lane runs the same instructions, the upwind branch, the border
        // freeze and the dominant-neighbour choice are per-lane selects (a frozen output
        // passes its gradient through: coefficient 1 at q == 1, 0 elsewhere).  The upwind
        // differences of neighbouring positions are shared by the three outputs.
        T dif[4][NC];  // dif[p] = position p+1 minus position p
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int c = 0; c < NC; ++c) dif[p][c] = px[p + 1][c] - px[p][c];
#pragma unroll
        for (int q = 0; q < 3; ++q) {  // output i = j - 1 + q reads positions q, q+1, q+2
            const int i = j - 1 + q;
            const bool in = line_in && i >= border && i < n - border;
            const T vm_ = px[q][AXIS], vp_ = px[q + 2][AXIS];
            const bool take_p = Ar<T>::sub(fabs(vp_), fabs(vm_)) > T(0);
            const T dv = take_p ? vp_ : vm_;
            const T t = dt * dv;
            const bool pos = dv >= T(0);
            const T dtq = in ? dt : T(0);
            T coef;  // weight of this output's gradient at j
            if (q == 1) coef = in ? (pos ? T(1) - t : T(1) + t) : T(1);
            else if (q == 2) coef = in && pos ? t : T(0);
            else coef = in && !pos ? -t : T(0);
            T gdv = T(0);
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const T g_o = gx[q][c];
                acc[c] += g_o * coef;
                gdv -= g_o * dtq * (pos ? dif[q][c] : dif[q + 1][c]);  // upwind difference
            }
            // the dominant velocity is the chosen neighbour's AXIS component (position 2 = j)
            if (q != 1) acc[AXIS] += (q == 0 ? take_p : !take_p) ? gdv : T(0);
        }
        return;
    }
    for (int i = max(j - 1, 0); i <= min(j + 1, n - 1); ++i) {
        const bool in = line_in && i >= border && i < n - border;
        T go[NC];
        gchan(i, go);
        if (!in) {
            if (i == j)
                for (int c = 0; c < NC; ++c) acc[c] += go[c];
            continue;
        }
        const int im = max(i - 1, 0), ip = min(i + 1, n - 1);
        T pm[NC], p0[NC], pp[NC];
        chan(im, pm);
        chan(i, p0);
        chan(ip, pp);
        const T vm_ = pm[AXIS], vp_ = pp[AXIS];
        const bool take_p = Ar<T>::sub(fabs(vp_), fabs(vm_)) > T(0);
        const T dv = take_p ? vp_ : vm_;
        const T t = dt * dv;
        T gdv = T(0);
        for (int c = 0; c < NC; ++c) {
            if (dv >= T(0)) {
                if (i == j) acc[c] += go[c] * (T(1) - t);
                if (im == j) acc[c] += go[c] * t;
                gdv -= go[c] * dt * (p0[c] - pm[c]);
            } else {
                if (i == j) acc[c] += go[c] * (T(1) + t);
                if (ip == j) acc[c] -= go[c] * t;
                gdv -= go[c] * dt * (pp[c] - p0[c]);
            }
        }
        // the dominant velocity is the chosen neighbour's AXIS component
        if ((take_p ? ip : im) == j) acc[AXIS] += gdv;
    }
}

// every channel of one pixel of a propagated field (f pairs, s scalars, v pairs) at index k
template <typename T, bool PAYLOAD>
__device__ __forceinline__ void field_px(const T* __restrict__ f, const T* __restrict__ s, const T* __restrict__ v,
                                         size_t k, T (&o)[PAYLOAD ? 5 : 2]) {
    const auto a = ld2(f, k);
    o[0] = a.x;
    o[1] = a.y;
    if constexpr (PAYLOAD) {
        const auto b = ld2(v, k);
        o[2] = s[k];
        o[3] = b.x;
        o[4] = b.y;
    }
}

// Adjoint of one upwind sub-step, one thread per input pixel (prop_adj_at over global memory)
template <typename T, int AXIS, bool PAYLOAD, bool ACC = true>
__global__ void prop_bwd_k(const T* __restrict__ f, const T* __restrict__ s, const T* __restrict__ v,
                           const T* __restrict__ gfo, const T* __restrict__ gso, const T* __restrict__ gvo, T* gf, T* gs,
                           T* gv, int H, int W, T dt, int border) {
    grid_dep_wait();
    grid_dep_launch();
    PIX_SETUP
    if (!live) return;
    constexpr int NC = PAYLOAD ? 5 : 2;
    // linear index of position p along the axis, on this pixel's line
    auto at = [&](int p) -> size_t { return AXIS == 0 ? (b * H + y) * W + p : (b * H + p) * W + x; };
    const bool line_in = AXIS == 0 ? (y >= border && y < H - border) : (x >= border && x < W - border);
    T acc[NC];
    prop_adj_at<T, AXIS, PAYLOAD>(
        AXIS == 0 ? x : y, AXIS == 0 ? W : H, line_in, border, dt,
        [&](int p, T(&o)[NC]) { field_px<T, PAYLOAD>(f, s, v, at(p), o); },
        [&](int p, T(&o)[NC]) { field_px<T, PAYLOAD>(gfo, gso, gvo, at(p), o); }, acc);
    const size_t kj = at(AXIS == 0 ? x : y);
    put<ACC>(gf[2 * kj], acc[0]);
    put<ACC>(gf[2 * kj + 1], acc[1]);
    if constexpr (PAYLOAD) {
        put<ACC>(gs[kj], acc[2]);
        put<ACC>(gv[2 * kj], acc[3]);
        put<ACC>(gv[2 * kj + 1], acc[4]);
    }
}

// ------------------------------------------------------------------ update (top level)
template <typename T>
__global__ void update_fwd_k(const T* __restrict__ a0, const T* __restrict__ grad, const T* __restrict__ old,
                             const T* __restrict__ fh, const T* __restrict__ gamma, T* __restrict__ out, int H, int W,
                             T maxflow) {
    grid_dep_wait();
    grid_dep_launch();
    PIX_SETUP
    if (!live) return;
    const size_t k = (b * H + y) * W + x;
    const T g = *gamma, c = a0[k];
    const Solve<T> s(g, grad[2 * k], grad[2 * k + 1], Ar<T>::sub(old[k], c), fh[2 * k], fh[2 * k + 1]);
    out[2 * k] = sanitize(clampm(s.ox, maxflow));
    out[2 * k + 1] = sanitize(clampm(s.oy, maxflow));
}

template <typename T>
__device__ __forceinline__ bool passes(T o, T m) {
    return Ar<T>::finite(o) && o < m && o > -m;
}

template <typename T>
__global__ void update_bwd_k(const T* __restrict__ a0, const T* __restrict__ grad, const T* __restrict__ old,
                             const T* __restrict__ fh, const T* __restrict__ gamma, const T* __restrict__ gout, T* ga0,
                             T* ggrad, T* gold, T* gfh, T* ggamma, int H, int W, T maxflow) {
    grid_dep_wait();
    grid_dep_launch();
    PIX_SETUP
    T gg = T(0);
    if (live) {
        const size_t k = (b * H + y) * W + x;
        const T g = *gamma, c = a0[k], ax = grad[2 * k], ay = grad[2 * k + 1], yt = Ar<T>::sub(old[k], c);
        const T fx = fh[2 * k], fy = fh[2 * k + 1];
        const Solve<T> s(g, ax, ay, yt, fx, fy);
        const T gx = passes(s.ox, maxflow) ? gout[2 * k] : T(0);
        const T gy = passes(s.oy, maxflow) ? gout[2 * k + 1] : T(0);
        const SolveGrad<T> d(s, g, ax, ay, yt, fx, fy, gx, gy);
        // one thread per pixel writes these: plain adds
        gfh[2 * k] += d.gfx;
        gfh[2 * k + 1] += d.gfy;
        gold[k] += d.gyt;
        ga0[k] -= d.gyt;
        ggrad[2 * k] += d.gax;
        ggrad[2 * k + 1] += d.gay;
        gg = d.gg;
    }
    block_add(gg, ggamma);
}

// ------------------------------------------------------------------ delta update
template <typename T>
__global__ void dupdate_fwd_k(const T* __restrict__ a0, const T* __restrict__ grad, const T* __restrict__ old,
                              const T* __restrict__ dh, const T* __restrict__ coarse, const T* __restrict__ gamma,
                              T* __restrict__ flow, T* __restrict__ delta, int H, int W, int Hc, int Wc, T maxflow) {
    grid_dep_wait();
    grid_dep_launch();
    PIX_SETUP
    if (!live) return;
    const size_t k = (b * H + y) * W + x;
    const T g = *gamma, c = a0[k];
    const Solve<T> s(g, grad[2 * k], grad[2 * k + 1], Ar<T>::sub(old[k], c), dh[2 * k], dh[2 * k + 1]);
    const T hm = Ar<T>::mul(T(0.5), maxflow);
    const T dx = clampm(sanitize(s.ox), hm), dy = clampm(sanitize(s.oy), hm);
    const size_t kc = (b * Hc + upmap_index(y, H, Hc)) * Wc + upmap_index(x, W, Wc);
    delta[2 * k] = dx;
    delta[2 * k + 1] = dy;
    flow[2 * k] = clampm(Ar<T>::add(dx, Ar<T>::mul(T(2), coarse[2 * kc])), maxflow);
    flow[2 * k + 1] = clampm(Ar<T>::add(dy, Ar<T>::mul(T(2), coarse[2 * kc + 1])), maxflow);
}

template <typename T>
__global__ void dupdate_bwd_k(const T* __restrict__ a0, const T* __restrict__ grad, const T* __restrict__ old,
                              const T* __restrict__ dh, const T* __restrict__ coarse, const T* __restrict__ gamma,
                              const T* __restrict__ gflow, const T* __restrict__ gdelta, T* ga0, T* ggrad, T* gold,
                              T* gdh, T* gcoarse, T* ggamma, int H, int W, int Hc, int Wc, T maxflow) {
    grid_dep_wait();
    grid_dep_launch();
    PIX_SETUP
    T gg = T(0);
    if (live) {
        const size_t k = (b * H + y) * W + x;
        const T g = *gamma, c = a0[k], ax = grad[2 * k], ay = grad[2 * k + 1], yt = Ar<T>::sub(old[k], c);
        const T fx = dh[2 * k], fy = dh[2 * k + 1];
        const Solve<T> s(g, ax, ay, yt, fx, fy);
        const T hm = Ar<T>::mul(T(0.5), maxflow);
        const T dx = clampm(sanitize(s.ox), hm), dy = clampm(sanitize(s.oy), hm);
        const size_t kc = (b * Hc + upmap_index(y, H, Hc)) * Wc + upmap_index(x, W, Wc);
        const T ux = Ar<T>::add(dx, Ar<T>::mul(T(2), coarse[2 * kc]));
        const T uy = Ar<T>::add(dy, Ar<T>::mul(T(2), coarse[2 * kc + 1]));
        const T gux = passes(ux, maxflow) ? gflow[2 * k] : T(0);
        const T guy = passes(uy, maxflow) ? gflow[2 * k + 1] : T(0);
        atomic_add(&gcoarse[2 * kc], T(2) * gux);
        atomic_add(&gcoarse[2 * kc + 1], T(2) * guy);
        const T gx = passes(s.ox, hm) ? gdelta[2 * k] + gux : T(0);
        const T gy = passes(s.oy, hm) ? gdelta[2 * k + 1] + guy : T(0);
        const SolveGrad<T> d(s, g, ax, ay, yt, fx, fy, gx, gy);
        // one thread per pixel writes these: plain adds (the coarse flow above needs atomics)
        gdh[2 * k] += d.gfx;
        gdh[2 * k + 1] += d.gfy;
        gold[k] += d.gyt;
        ga0[k] -= d.gyt;
        ggrad[2 * k] += d.gax;
        ggrad[2 * k + 1] += d.gay;
        gg = d.gg;
    }
    block_add(gg, ggamma);
}

// ------------------------------------------------------------------ weighted smoothing pass
template <typename T, int AXIS>
__global__ void smooth_fwd_k(const T* __restrict__ w5, const T* __restrict__ in, T* __restrict__ out, int H, int W,
                             T* __restrict__ out2 = nullptr) {
    grid_dep_wait();
    grid_dep_launch();
    PIX_SETUP
    if (!live) return;
    T w[5];
    for (int i = 0; i < 5; ++i) w[i] = w5[i];
    size_t kk[5];
    for (int i = 0; i < 5; ++i)
        kk[i] = AXIS == 0 ? (b * H + y) * W + clampi(x + i - 2, 0, W - 1) : (b * H + clampi(y + i - 2, 0, H - 1)) * W + x;
    const size_t k = (b * H + y) * W + x;
    for (int ch = 0; ch < 2; ++ch) {
        const T v = chain5(w, in[2 * kk[0] + ch], in[2 * kk[1] + ch], in[2 * kk[2] + ch], in[2 * kk[3] + ch],
                           in[2 * kk[4] + ch]);
        out[2 * k + ch] = v;
        if (out2) out2[2 * k + ch] = v;  // a second copy (the frame driver's level-0 output)
    }
}

// Blocks of 32 x 8 threads cover 32 x 32 pixels (kSmoothRows rows per thread), so the
// weight gradient is reduced once per 1024 pixels.
// PART: gw5 is a partial-sum array, this block stores its 5 sums at gw5[5 * block]
constexpr int kSmoothRows = 4;
template <typename T, int AXIS, bool ACC = true, bool PART = false>
__global__ void smooth_bwd_k(const T* __restrict__ w5, const T* __restrict__ in, const T* __restrict__ gout, T* gin,
                             T* gw5, int H, int W) {
    grid_dep_wait();
    grid_dep_launch();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t b = blockIdx.z;
    T gw[5] = {T(0), T(0), T(0), T(0), T(0)};
    for (int rr = 0; rr < kSmoothRows; ++rr) {
        const int y = (blockIdx.y * kSmoothRows + rr) * blockDim.y + threadIdx.y;
        if (x < W && y < H) {
            T w[5];
            for (int i = 0; i < 5; ++i) w[i] = w5[i];
            const int n = AXIS == 0 ? W : H;
            const int j = AXIS == 0 ? x : y;
            auto at = [&](int p) -> size_t { return AXIS == 0 ? (b * H + y) * W + p : (b * H + p) * W + x; };
            // input gradient at this pixel: outputs i in [j-2, j+2] whose clamped taps land on j
            T a0 = T(0), a1 = T(0);
            if (j >= 2 && j + 2 <= n - 1) {
                // no clamps: output i reads j through tap j - i + 2 only
    #pragma unroll
                for (int q = 0; q < 5; ++q) {
                    const T wt = w[4 - q];
                    if (wt != T(0)) {
                        const auto gv = ld2(gout, at(j - 2 + q));
                        a0 += wt * gv.x;
                        a1 += wt * gv.y;
                    }
                }
            } else
            for (int i = max(j - 2, 0); i <= min(j + 2, n - 1); ++i) {
                const T wt = tap_weight(w, i, j, n);
                if (wt != T(0)) {
                    a0 += wt * gout[2 * at(i)];
                    a1 += wt * gout[2 * at(i) + 1];
                }
            }
            put<ACC>(gin[2 * at(j)], a0);
            put<ACC>(gin[2 * at(j) + 1], a1);
            // weight gradient: this pixel as an output
            const auto g01 = ld2(gout, at(j));
            const T g0 = g01.x, g1 = g01.y;
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                const auto iv = ld2(in, at(clampi(j + k - 2, 0, n - 1)));
                gw[k] += g0 * iv.x + g1 * iv.y;
            }
        }
    }
    block_sum<T, 5>(gw, PART ? gw5 + 5 * block_linear() : gw5, !PART);
}

// Adjoint of one smoothing iteration (X pass, then Y pass) of a 32 x 32 tile in one block of
// the frame driver.  Every input the tile needs is staged in shared memory first, in one
// batch of independent loads: the output gradient on the tile and two halo rows and columns,
// the Y pass's input (the tape) on the tile's columns and the halo rows, the X pass's input
// on the tile's rows and the halo columns (both at clamped coordinates).  Then the Y adjoint
// on the tile's rows and the halo columns (shared), and the X adjoint from it into gin
// (stored, or added when ACC).  The weight gradients of both passes are summed over the
// tile's own pixels (each pass's output gradient times its clamped input taps) and stored as
// 5 sums at part[5 * block].  Gradient halo entries outside the image are never read: the
// gathers visit only the outputs inside the image.
constexpr int kST = 32;
constexpr int kSW = kST + 4;
inline dim3 grid_tile32(int w, int h, int B) { return dim3((w + kST - 1) / kST, (h + kST - 1) / kST, B); }
template <typename T>
constexpr size_t smooth_iter_smem() {
    return sizeof(typename Pair<T>::V) * (size_t)(kSW * kSW + 3 * kST * kSW);
}
// G2: a second output gradient gout2 is added to gout (image b at gout2 + b * g2_bstride)
template <typename T, bool ACC, bool G2>
__global__ void __launch_bounds__(256) smooth_iter_bwd_k(const T* __restrict__ w5, const T* __restrict__ xin,
                                                         const T* __restrict__ xmid, const T* __restrict__ gout,
                                                         const T* __restrict__ gout2, long long g2_bstride,
                                                         T* __restrict__ gin, T* __restrict__ part, int H, int W) {
    grid_dep_wait();
    using V = typename Pair<T>::V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V(*sg)[kSW] = reinterpret_cast<V(*)[kSW]>(smem_raw);          // gout: rows y0-2.., cols x0-2..
    V(*sym)[kST] = reinterpret_cast<V(*)[kST]>(sg + kSW);        // xmid: rows y0-2.., cols x0..
    V(*sxi)[kSW] = reinterpret_cast<V(*)[kSW]>(sym + kSW);       // xin: rows y0.., cols x0-2..
    V(*sm)[kSW] = sxi + kST;                                      // gradient of the X pass output
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int x0 = blockIdx.x * kST, y0 = blockIdx.y * kST;
    const size_t base = (size_t)blockIdx.z * H * W;
    const V* go = reinterpret_cast<const V*>(gout) + base;
    const V* xi = reinterpret_cast<const V*>(xin) + base;
    const V* xm = reinterpret_cast<const V*>(xmid) + base;
    V* gi = reinterpret_cast<V*>(gin) + base;
    T w[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) w[k] = w5[k];
    {
        constexpr int NG = (kSW * kSW + 255) / 256, NT = (kST * kSW + 255) / 256;
        V a[NG], bm[NT], bi[NT];
#pragma unroll
        for (int u = 0; u < NG; ++u) {
            const int e = tid + 256 * u, r = e / kSW, c = e - r * kSW;
            const int y = y0 - 2 + r, x = x0 - 2 + c;
            if (e < kSW * kSW && y >= 0 && y < H && x >= 0 && x < W) {
                a[u] = go[(size_t)y * W + x];
                if constexpr (G2) {
                    const V b2 = reinterpret_cast<const V*>(gout2 + blockIdx.z * g2_bstride)[(size_t)y * W + x];
                    a[u].x += b2.x;
                    a[u].y += b2.y;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < NT; ++u) {
            const int e = tid + 256 * u;
            const int rm = e / kST, cm = e - rm * kST;   // xmid: kSW rows x kST columns
            const int rx = e / kSW, cx = e - rx * kSW;   // xin: kST rows x kSW columns
            if (e < kST * kSW) {
                const int ym = clampi(y0 - 2 + rm, 0, H - 1), xm_ = x0 + cm;
                if (xm_ < W) bm[u] = xm[(size_t)ym * W + xm_];
                const int yx = y0 + rx, xx = clampi(x0 - 2 + cx, 0, W - 1);
                if (yx < H) bi[u] = xi[(size_t)yx * W + xx];
            }
        }
#pragma unroll
        for (int u = 0; u < NG; ++u) {
            const int e = tid + 256 * u, r = e / kSW, c = e - r * kSW;
            const int y = y0 - 2 + r, x = x0 - 2 + c;
            if (e < kSW * kSW && y >= 0 && y < H && x >= 0 && x < W) sg[r][c] = a[u];
        }
#pragma unroll
        for (int u = 0; u < NT; ++u) {
            const int e = tid + 256 * u;
            const int rm = e / kST, cm = e - rm * kST, rx = e / kSW, cx = e - rx * kSW;
            if (e < kST * kSW) {
                if (x0 + cm < W) sym[rm][cm] = bm[u];
                if (y0 + rx < H) sxi[rx][cx] = bi[u];
            }
        }
    }
    __syncthreads();
    T gw[5] = {T(0), T(0), T(0), T(0), T(0)};
    for (int e = tid; e < kST * kSW; e += 256) {
        const int r = e / kSW, c = e - r * kSW;
        const int y = y0 + r, x = x0 - 2 + c;
        if (y >= H || x < 0 || x >= W) continue;
        T ax = T(0), ay = T(0);
        if (y >= 2 && y + 2 <= H - 1) {
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const V v = sg[r + q][c];
                ax += w[4 - q] * v.x;
                ay += w[4 - q] * v.y;
            }
        } else {
            for (int i = max(y - 2, 0); i <= min(y + 2, H - 1); ++i) {
                const T wt = tap_weight(w, i, y, H);
                const V v = sg[i - y0 + 2][c];
                ax += wt * v.x;
                ay += wt * v.y;
            }
        }
        V m;
        m.x = ax;
        m.y = ay;
        sm[r][c] = m;
        if (c >= 2 && c < kST + 2) {  // the Y pass's output (y, x) is this tile's pixel
            const V g = sg[r + 2][c];
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                const V iv = sym[r + k][c - 2];  // row clamp(y + k - 2)
                gw[k] += g.x * iv.x + g.y * iv.y;
            }
        }
    }
    __syncthreads();
    grid_dep_launch();  // the next kernel's blocks may now take this block's place
    for (int e = tid; e < kST * kST; e += 256) {
        const int r = e / kST, c = e - r * kST;
        const int y = y0 + r, x = x0 + c;
        if (y >= H || x >= W) continue;
        T ax = T(0), ay = T(0);
        if (x >= 2 && x + 2 <= W - 1) {
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const V v = sm[r][c + q];
                ax += w[4 - q] * v.x;
                ay += w[4 - q] * v.y;
            }
        } else {
            for (int i = max(x - 2, 0); i <= min(x + 2, W - 1); ++i) {
                const T wt = tap_weight(w, i, x, W);
                const V v = sm[r][i - x0 + 2];
                ax += wt * v.x;
                ay += wt * v.y;
            }
        }
        const size_t k = (size_t)y * W + x;
        V o;
        if constexpr (ACC) {
            o = gi[k];
            o.x += ax;
            o.y += ay;
        } else {
            o.x = ax;
            o.y = ay;
        }
        gi[k] = o;
        const V g = sm[r][c + 2];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const V iv = sxi[r][c + q];  // column clamp(x + q - 2)
            gw[q] += g.x * iv.x + g.y * iv.y;
        }
    }
    block_sum<T, 5>(gw, part + 5 * block_linear(), false);
}

// asynchronous global -> shared copy of N bytes (4, 8 or 16; both addresses N-aligned)
template <int N>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Adjoint of one propagation iteration (X sub-step, then Y sub-step) of a 32 x 32 tile in one
// block of the frame driver.  Staged in shared memory in one batch of asynchronous copies:
// the gradient of the Y sub-step's output on the tile and one halo row and column, the Y
// sub-step's input on the tile's columns plus one and the rows plus two each side, the X
// sub-step's input on the tile's rows and the columns plus two each side (the tape, or the
// state before the first sub-step).  Then the Y adjoint on the tile's rows and the halo
// columns (shared), and the X adjoint from it into the X sub-step's input gradient (stored,
// or added when ACC).  Entries outside the image are never read.
constexpr int kPG = kST + 2;
constexpr int kPropThreads = 512;  // 32 x 16
template <typename T, bool PAYLOAD>
struct PropTile {
    using V = typename Pair<T>::V;
    static constexpr int NC = PAYLOAD ? 5 : 2;
    // pixel fields of a staged region: f pairs [, s, v pairs]
    template <int R, int C>
    struct Field {
        V f[R][C];
        T s[PAYLOAD ? R : 1][PAYLOAD ? C : 1];
        V v[PAYLOAD ? R : 1][PAYLOAD ? C : 1];
    };
    Field<kPG, kPG> go;      // output gradient: rows y0-1.., cols x0-1..
    Field<kST + 4, kPG> ty;  // Y sub-step input: rows y0-2.., cols x0-1..
    Field<kST, kST + 4> tx;  // X sub-step input: rows y0.., cols x0-2..
    T mid[NC][kST][kPG];     // gradient of the X sub-step's output: rows y0.., cols x0-1..
};

// copy pixel k of a field into slot (r, c) of a staged region
template <typename T, bool PAYLOAD, typename F>
__device__ __forceinline__ void stage_px(F& dst, int r, int c, const T* f, const T* s, const T* v, size_t k) {
    constexpr int P = 2 * sizeof(T);
    if (f) {
        cp_async<P>(&dst.f[r][c], f + 2 * k);
    } else {  // an absent gradient: zeros
        dst.f[r][c].x = T(0);
        dst.f[r][c].y = T(0);
    }
    if constexpr (PAYLOAD) {
        cp_async<sizeof(T)>(&dst.s[r][c], s + k);
        cp_async<P>(&dst.v[r][c], v + 2 * k);
    }
}
template <typename T, bool PAYLOAD, typename F>
__device__ __forceinline__ void read_px(const F& src, int r, int c, T (&o)[PAYLOAD ? 5 : 2]) {
    o[0] = src.f[r][c].x;
    o[1] = src.f[r][c].y;
    if constexpr (PAYLOAD) {
        o[2] = src.s[r][c];
        o[3] = src.v[r][c].x;
        o[4] = src.v[r][c].y;
    }
}

template <typename T, bool PAYLOAD, bool ACC>
__global__ void __launch_bounds__(kPropThreads) prop_iter_bwd_k(const T* __restrict__ xf, const T* __restrict__ xs,
                                                                const T* __restrict__ xv, const T* __restrict__ yf,
                                                                const T* __restrict__ ys, const T* __restrict__ yv,
                                                                const T* __restrict__ gfo, const T* __restrict__ gso,
                                                                const T* __restrict__ gvo, T* __restrict__ gf,
                                                                T* __restrict__ gs, T* __restrict__ gv, int H, int W,
                                                                T dt, int border) {
    grid_dep_wait();
    using Tile = PropTile<T, PAYLOAD>;
    constexpr int NC = Tile::NC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Tile& S = *reinterpret_cast<Tile*>(smem_raw);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int x0 = blockIdx.x * kST, y0 = blockIdx.y * kST;
    const size_t base = (size_t)blockIdx.z * H * W;
    for (int e = tid; e < kPG * kPG; e += kPropThreads) {
        const int r = e / kPG, c = e - r * kPG, y = y0 - 1 + r, x = x0 - 1 + c;
        if (y >= 0 && y < H && x >= 0 && x < W)
            stage_px<T, PAYLOAD>(S.go, r, c, gfo, gso, gvo, base + (size_t)y * W + x);
    }
    for (int e = tid; e < (kST + 4) * kPG; e += kPropThreads) {
        const int r = e / kPG, c = e - r * kPG, y = y0 - 2 + r, x = x0 - 1 + c;
        if (y >= 0 && y < H && x >= 0 && x < W) stage_px<T, PAYLOAD>(S.ty, r, c, yf, ys, yv, base + (size_t)y * W + x);
    }
    for (int e = tid; e < kST * (kST + 4); e += kPropThreads) {
        const int r = e / (kST + 4), c = e - r * (kST + 4), y = y0 + r, x = x0 - 2 + c;
        if (y < H && x >= 0 && x < W) stage_px<T, PAYLOAD>(S.tx, r, c, xf, xs, xv, base + (size_t)y * W + x);
    }
    cp_async_wait_all();
    __syncthreads();
    // Y adjoint at rows y0.., columns x0-1..
    for (int e = tid; e < kST * kPG; e += kPropThreads) {
        const int r = e / kPG, c = e - r * kPG;
        const int y = y0 + r, x = x0 - 1 + c;
        if (y >= H || x < 0 || x >= W) continue;
        T acc[NC];
        prop_adj_at<T, 1, PAYLOAD>(
            y, H, x >= border && x < W - border, border, dt,
            [&](int p, T(&o)[NC]) { read_px<T, PAYLOAD>(S.ty, p - y0 + 2, c, o); },
            [&](int p, T(&o)[NC]) { read_px<T, PAYLOAD>(S.go, p - y0 + 1, c, o); }, acc);
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) S.mid[ch][r][c] = acc[ch];
    }
    __syncthreads();
    grid_dep_launch();  // the next kernel's blocks may now take this block's place
    // X adjoint at the tile's pixels
    for (int e = tid; e < kST * kST; e += kPropThreads) {
        const int r = e / kST, c = e - r * kST;
        const int y = y0 + r, x = x0 + c;
        if (y >= H || x >= W) continue;
        T acc[NC];
        prop_adj_at<T, 0, PAYLOAD>(
            x, W, y >= border && y < H - border, border, dt,
            [&](int p, T(&o)[NC]) { read_px<T, PAYLOAD>(S.tx, r, p - x0 + 2, o); },
            [&](int p, T(&o)[NC]) {
#pragma unroll
                for (int ch = 0; ch < NC; ++ch) o[ch] = S.mid[ch][r][p - x0 + 1];
            },
            acc);
        const size_t k = base + (size_t)y * W + x;
        put<ACC>(gf[2 * k], acc[0]);
        put<ACC>(gf[2 * k + 1], acc[1]);
        if constexpr (PAYLOAD) {
            put<ACC>(gs[k], acc[2]);
            put<ACC>(gv[2 * k], acc[3]);
            put<ACC>(gv[2 * k + 1], acc[4]);
        }
    }
}

// The image model's adjoint (model_bwd1_k then model_bwd2_k) of a 32 x 32 tile in one block
// of the frame driver: the gradients of a0 and of the image gradient on the tile and two halo
// rows and columns staged in shared memory in one batch of loads; the gradients of the Y
// blur (rows y0-2.., the tile's columns) and of the X blur (the tile's rows, columns x0-2..)
// in shared memory; the image gradient from them, stored (or added when ACC).
template <typename T>
constexpr size_t model_tile_smem() {
    return sizeof(T) * (size_t)(kSW * kSW + 2 * kSW * kSW + 2 * kST * kSW);
}
template <typename T, bool ACC>
__global__ void __launch_bounds__(256) model_tile_bwd_k(const T* __restrict__ ga0, const T* __restrict__ ggrad,
                                                        T* __restrict__ gimg, int H, int W) {
    grid_dep_wait();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T(*sa)[kSW] = reinterpret_cast<T(*)[kSW]>(smem_raw);         // ga0: rows y0-2.., cols x0-2..
    T(*sgx)[kSW] = sa + kSW;                                      // ggrad x: same
    T(*sgy)[kSW] = sgx + kSW;                                     // ggrad y: same
    T(*sby)[kST] = reinterpret_cast<T(*)[kST]>(sgy + kSW);       // gby: rows y0-2.., cols x0..
    T(*sbx)[kSW] = reinterpret_cast<T(*)[kSW]>(sby + kSW);       // gbx: rows y0.., cols x0-2..
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int x0 = blockIdx.x * kST, y0 = blockIdx.y * kST;
    const size_t base = (size_t)blockIdx.z * H * W;
    const T* a0g = ga0 + base;
    const typename Pair<T>::V* gg = reinterpret_cast<const typename Pair<T>::V*>(ggrad) + base;
    const Masks<T> M;
    {
        constexpr int NG = (kSW * kSW + 255) / 256;
        T va[NG];
        typename Pair<T>::V vg[NG];
#pragma unroll
        for (int u = 0; u < NG; ++u) {
            const int e = tid + 256 * u, r = e / kSW, c = e - r * kSW;
            const int y = y0 - 2 + r, x = x0 - 2 + c;
            if (e < kSW * kSW && y >= 0 && y < H && x >= 0 && x < W) {
                const size_t k = (size_t)y * W + x;
                va[u] = a0g[k];
                vg[u] = gg[k];
            }
        }
#pragma unroll
        for (int u = 0; u < NG; ++u) {
            const int e = tid + 256 * u, r = e / kSW, c = e - r * kSW;
            const int y = y0 - 2 + r, x = x0 - 2 + c;
            if (e < kSW * kSW && y >= 0 && y < H && x >= 0 && x < W) {
                sa[r][c] = va[u];
                sgx[r][c] = vg[u].x;
                sgy[r][c] = vg[u].y;
            }
        }
    }
    __syncthreads();
    // gby at rows y0-2.. (X gathers of a0 and the x gradient), gbx at columns x0-2.. (Y gather
    // of the y gradient)
    for (int e = tid; e < kSW * kST; e += 256) {
        {
            const int r = e / kST, c = e - r * kST;
            const int y = y0 - 2 + r, x = x0 + c;
            if (y >= 0 && y < H && x < W) {
                T acc = T(0);
                if (x >= 2 && x + 2 <= W - 1) {
#pragma unroll
                    for (int q = 0; q < 5; ++q) acc += M.s[4 - q] * sa[r][c + q] + M.d[4 - q] * sgx[r][c + q];
                } else {
                    for (int i = max(x - 2, 0); i <= min(x + 2, W - 1); ++i)
                        acc += tap_weight(M.s, i, x, W) * sa[r][i - x0 + 2] + tap_weight(M.d, i, x, W) * sgx[r][i - x0 + 2];
                }
                sby[r][c] = acc;
            }
        }
        {
            const int r = e / kSW, c = e - r * kSW;
            const int y = y0 + r, x = x0 - 2 + c;
            if (y < H && x >= 0 && x < W) {
                T acc = T(0);
                if (y >= 2 && y + 2 <= H - 1) {
#pragma unroll
                    for (int q = 0; q < 5; ++q) acc += M.d[4 - q] * sgy[r + q][c];
                } else {
                    for (int i = max(y - 2, 0); i <= min(y + 2, H - 1); ++i)
                        acc += tap_weight(M.d, i, y, H) * sgy[i - y0 + 2][c];
                }
                sbx[r][c] = acc;
            }
        }
    }
    __syncthreads();
    grid_dep_launch();  // the next kernel's blocks may now take this block's place
    T* gi = gimg + base;
    for (int e = tid; e < kST * kST; e += 256) {
        const int r = e / kST, c = e - r * kST;
        const int y = y0 + r, x = x0 + c;
        if (y >= H || x >= W) continue;
        T acc = T(0);
        if (y >= 2 && y + 2 <= H - 1) {
#pragma unroll
            for (int q = 0; q < 5; ++q) acc += M.s[4 - q] * sby[r + q][c];
        } else {
            for (int i = max(y - 2, 0); i <= min(y + 2, H - 1); ++i) acc += tap_weight(M.s, i, y, H) * sby[i - y0 + 2][c];
        }
        if (x >= 2 && x + 2 <= W - 1) {
#pragma unroll
            for (int q = 0; q < 5; ++q) acc += M.s[4 - q] * sbx[r][c + q];
        } else {
            for (int i = max(x - 2, 0); i <= min(x + 2, W - 1); ++i) acc += tap_weight(M.s, i, x, W) * sbx[r][i - x0 + 2];
        }
        put<ACC>(gi[(size_t)y * W + x], acc);
    }
}

// Store-mode update adjoints of the frame driver: every per-pixel gradient is stored (the
// destinations start undefined), the gradient of a0 as a state output (ga0_out, nullable)
// is folded in, `first` (old image == a0) cancels the yt path, gold is added (a caller's
// input-state gradient) or stored, and the gamma gradient goes to one partial per block.
template <typename T>
struct FrameAdj {
    const T* ga0_out;
    int first;
    int gold_acc;
    T* part;
    __device__ void write(size_t k, const SolveGrad<T>& d, T* ga0, T* ggrad, T* gold, T* gfh) const {
        const T gyt = first ? T(0) : d.gyt;
        ga0[k] = (ga0_out ? ga0_out[k] : T(0)) - gyt;
        ggrad[2 * k] = d.gax;
        ggrad[2 * k + 1] = d.gay;
        gfh[2 * k] = d.gfx;
        gfh[2 * k + 1] = d.gfy;
        if (gold_acc) {
            if (!first) gold[k] += gyt;
        } else {
            gold[k] = gyt;
        }
    }
};

template <typename T>
__global__ void update_bwd_frame_k(const T* __restrict__ a0, const T* __restrict__ grad, const T* __restrict__ old,
                                   const T* __restrict__ fh, const T* __restrict__ gamma, const T* __restrict__ gout,
                                   T* ga0, T* ggrad, T* gold, T* gfh, FrameAdj<T> fa, int H, int W, T maxflow) {
    grid_dep_wait();
    grid_dep_launch();
    PIX_SETUP
    T gg[1] = {T(0)};
    if (live) {
        const size_t k = (b * H + y) * W + x;
        const T g = *gamma, c = a0[k], ax = grad[2 * k], ay = grad[2 * k + 1], yt = Ar<T>::sub(old[k], c);
        const T fx = fh[2 * k], fy = fh[2 * k + 1];
        const Solve<T> s(g, ax, ay, yt, fx, fy);
        const T gx = passes(s.ox, maxflow) ? gout[2 * k] : T(0);
        const T gy = passes(s.oy, maxflow) ? gout[2 * k + 1] : T(0);
        const SolveGrad<T> d(s, g, ax, ay, yt, fx, fy, gx, gy);
        fa.write(k, d, ga0, ggrad, gold, gfh);
        gg[0] = d.gg;
    }
    block_sum<T, 1>(gg, fa.part + block_linear(), false);
}

template <typename T>
__global__ void dupdate_bwd_frame_k(const T* __restrict__ a0, const T* __restrict__ grad, const T* __restrict__ old,
                                    const T* __restrict__ dh, const T* __restrict__ coarse,
                                    const T* __restrict__ gamma, const T* __restrict__ gflow,
                                    const T* __restrict__ gdelta, T* ga0, T* ggrad, T* gold, T* gdh, T* gcoarse,
                                    FrameAdj<T> fa, int H, int W, int Hc, int Wc, T maxflow) {
    grid_dep_wait();
    grid_dep_launch();
    PIX_SETUP
    T gg[1] = {T(0)};
    // a warp is 32 consecutive pixels of one row and the coarse column is monotone in x, so
    // lanes sharing a coarse pixel form runs: each run's sum is added by its first lane
    unsigned long long key = ~0ull - threadIdx.x;  // distinct for pixels outside the image
    T cx = T(0), cy = T(0);
    size_t kc = 0;
    if (live) {
        const size_t k = (b * H + y) * W + x;
        const T g = *gamma, c = a0[k], ax = grad[2 * k], ay = grad[2 * k + 1], yt = Ar<T>::sub(old[k], c);
        const T fx = dh[2 * k], fy = dh[2 * k + 1];
        const Solve<T> s(g, ax, ay, yt, fx, fy);
        const T hm = Ar<T>::mul(T(0.5), maxflow);
        const T dx = clampm(sanitize(s.ox), hm), dy = clampm(sanitize(s.oy), hm);
        kc = (b * Hc + upmap_index(y, H, Hc)) * Wc + upmap_index(x, W, Wc);
        key = kc;
        const T ux = Ar<T>::add(dx, Ar<T>::mul(T(2), coarse[2 * kc]));
        const T uy = Ar<T>::add(dy, Ar<T>::mul(T(2), coarse[2 * kc + 1]));
        const T gux = passes(ux, maxflow) ? gflow[2 * k] : T(0);
        const T guy = passes(uy, maxflow) ? gflow[2 * k + 1] : T(0);
        cx = T(2) * gux;
        cy = T(2) * guy;
        const T gx = passes(s.ox, hm) ? gdelta[2 * k] + gux : T(0);
        const T gy = passes(s.oy, hm) ? gdelta[2 * k + 1] + guy : T(0);
        const SolveGrad<T> d(s, g, ax, ay, yt, fx, fy, gx, gy);
        fa.write(k, d, ga0, ggrad, gold, gdh);
        gg[0] = d.gg;
    }
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x;  // blocks are 32 wide
    const unsigned run = __match_any_sync(full, key);
    const unsigned longest = __reduce_max_sync(full, (unsigned)__popc(run));
    T sx = cx, sy = cy;
    for (unsigned d = 1; d < longest; ++d) {
        const T ox = __shfl_down_sync(full, cx, d), oy = __shfl_down_sync(full, cy, d);
        if (lane + d < 32 && ((run >> (lane + d)) & 1u)) {
            sx += ox;
            sy += oy;
        }
    }
    if (live && lane == __ffs(run) - 1) {
        atomic_add(&gcoarse[2 * kc], sx);
        atomic_add(&gcoarse[2 * kc + 1], sy);
    }
    block_sum<T, 1>(gg, fa.part + block_linear(), false);
}

// dst[v] += sum over i < n of part[i * NV + v], one block (fixed order: deterministic)
template <typename T, int NV>
__global__ void reduce_parts_k(const T* __restrict__ part, int n, T* dst) {
    grid_dep_wait();
    grid_dep_launch();
    T acc[NV];
    for (int v = 0; v < NV; ++v) acc[v] = T(0);
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        for (int v = 0; v < NV; ++v) acc[v] += part[(size_t)i * NV + v];
    __shared__ T tot[NV];
    block_sum<T, NV>(acc, tot, false);
    __syncthreads();
    if (threadIdx.x < NV) dst[threadIdx.x] += tot[threadIdx.x];
}

// The per-block partial sums of one frame's backward, reduced in one launch: block j adds
// the sum of its segment (n[j] rows of nv[j] values) to dst[j] (fixed order: deterministic)
template <typename T>
struct ReduceJobs {
    static constexpr int kMax = 2 * FF_DIFF_MAX_LEVELS;
    const T* part[kMax];
    T* dst[kMax];
    int n[kMax], nv[kMax];
    int count = 0;
};
template <typename T>
__global__ void __launch_bounds__(1024) reduce_jobs_k(ReduceJobs<T> J) {
    grid_dep_wait();
    grid_dep_launch();
    const int j = blockIdx.x;
    const T* part = J.part[j];
    const int n = J.n[j], nv = J.nv[j];
    T acc[5] = {T(0), T(0), T(0), T(0), T(0)};
    if (nv == 5) {
        for (int i = threadIdx.x; i < n; i += blockDim.x)
#pragma unroll
            for (int v = 0; v < 5; ++v) acc[v] += part[(size_t)i * 5 + v];
    } else {
        for (int i = threadIdx.x; i < n; i += blockDim.x) acc[0] += part[i];
    }
    __shared__ T tot[5];
    block_sum<T, 5>(acc, tot, false);
    __syncthreads();
    if ((int)threadIdx.x < nv) J.dst[j][threadIdx.x] += tot[threadIdx.x];
}

// dst = (ACC ? dst : 0) + a + b over B images of `per` elements; a dense (nullable, zero),
// image i of b at b + i * bstride
template <typename T, bool ACC>
__global__ void sum2_k(T* __restrict__ dst, const T* __restrict__ a, const T* __restrict__ b, long long bstride,
                       long long per, int B) {
    grid_dep_wait();
    grid_dep_launch();
    const long long n = (long long)B * per;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long img = i / per;
        const T v = a ? a[i] + b[img * bstride + (i - img * per)] : b[img * bstride + (i - img * per)];
        dst[i] = ACC ? dst[i] + v : v;
    }
}

// dst += src over n elements
template <typename T>
__global__ void add_k(T* __restrict__ dst, const T* __restrict__ src, size_t n) {
    grid_dep_wait();
    grid_dep_launch();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] += src[i];
}

// ------------------------------------------------------------------ endpoint-error loss
// flows (B, T, P, 2) dense (P = H * W pixels); truth element (b, t, p, c) at
// truth[b * tb + t * tt + 2 p + c] (tt = 0: one truth frame for every t).  Frames t >= first
// count.  Forward: per-block partial sums of sqrt(dx^2 + dy^2 + eps), one per block, reduced
// in fixed order (deterministic).  Backward: the flow gradient d g / (count |d|) for every
// element (zero before `first`, and where |d| = 0).
struct EpeGeom {
    int B, T, first;
    long long P, tb, tt;
};
constexpr int kEpeThreads = 256, kEpeBlocks = 1024;
template <typename T>
__global__ void __launch_bounds__(kEpeThreads) epe_fwd_k(const T* __restrict__ flows, const T* __restrict__ truth,
                                                         EpeGeom g, T eps, T* __restrict__ part) {
    grid_dep_wait();
    grid_dep_launch();
    using V = typename Pair<T>::V;
    const long long tf = g.T - g.first, n = (long long)g.B * tf * g.P;
    T acc[1] = {T(0)};
    for (long long i = blockIdx.x * (long long)kEpeThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kEpeThreads) {
        const long long p = i % g.P, bt = i / g.P, t = g.first + bt % tf, b = bt / tf;
        const V f = reinterpret_cast<const V*>(flows)[(b * g.T + t) * g.P + p];
        const V r = *reinterpret_cast<const V*>(truth + b * g.tb + t * g.tt + 2 * p);
        const T dx = f.x - r.x, dy = f.y - r.y;
        acc[0] += sqrt(dx * dx + dy * dy + eps);
    }
    block_sum<T, 1>(acc, part + blockIdx.x, false);
}
template <typename T>
__global__ void __launch_bounds__(1024) epe_sum_k(const T* __restrict__ part, int n, T inv_count, T* loss) {
    grid_dep_wait();
    grid_dep_launch();
    T acc[1] = {T(0)};
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc[0] += part[i];
    __shared__ T tot[1];
    block_sum<T, 1>(acc, tot, false);
    __syncthreads();
    if (threadIdx.x == 0) *loss = tot[0] * inv_count;
}
template <typename T>
__global__ void __launch_bounds__(kEpeThreads) epe_bwd_k(const T* __restrict__ flows, const T* __restrict__ truth,
                                                         EpeGeom g, T eps, const T* __restrict__ gloss, T inv_count,
                                                         T* __restrict__ gflows) {
    grid_dep_wait();
    grid_dep_launch();
    using V = typename Pair<T>::V;
    const T s = *gloss * inv_count;
    const long long n = (long long)g.B * g.T * g.P;
    for (long long i = blockIdx.x * (long long)kEpeThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kEpeThreads) {
        const long long p = i % g.P, bt = i / g.P, t = bt % g.T, b = bt / g.T;
        V o;
        o.x = T(0);
        o.y = T(0);
        if (t >= g.first) {
            const V f = reinterpret_cast<const V*>(flows)[i];
            const V r = *reinterpret_cast<const V*>(truth + b * g.tb + t * g.tt + 2 * p);
            const T dx = f.x - r.x, dy = f.y - r.y;
            const T m = sqrt(dx * dx + dy * dy + eps);
            if (m > T(0)) {
                const T k = s / m;
                o.x = dx * k;
                o.y = dy * k;
            }
        }
        reinterpret_cast<V*>(gflows)[i] = o;
    }
}

inline dim3 grid3(int w, int h, int B) { return dim3((w + 31) / 32, (h + 7) / 8, B); }
// the smoothing adjoint's grid (32 x 8 threads over 32 x 32 pixels)
inline dim3 grid_smooth(int w, int h, int B) { return dim3((w + 31) / 32, (h + 8 * kSmoothRows - 1) / (8 * kSmoothRows), B); }
const dim3 kBlock(32, 8);

template <typename T>
cudaError_t pyramid(bool bwd, int B, int H, int W, const void* a, void* o, cudaStream_t s) {
    const int h = H / 2, w = W / 2;
    if (h <= 0 || w <= 0) return cudaSuccess;
    // the adjoint runs one thread per INPUT pixel (gather), the forward one per output pixel
    if (bwd) return launch_k(pyr_bwd_k<T>, grid3(W, H, B), kBlock, 0, s, (const T*)a, (T*)o, H, W);
    return launch_k(pyr_fwd_k<T>, grid3(w, h, B), kBlock, 0, s, (const T*)a, (T*)o, H, W);
}

}  // namespace diff
}  // namespace ffb

// ------------------------------------------------------------------ C ABI
ff_status ffb_fail(ff_status s, const std::string& msg);  // capi.cu: last error + log

using namespace ffb;
using namespace ffb::diff;

namespace {

template <typename F>
ff_status run(int dtype, F&& f) {
    if (dtype != 0 && dtype != 1) {
        return ffb_fail(FF_ERR_INVALID_ARGUMENT, "dtype must be 0 (float32) or 1 (float64)");
    }
    cudaError_t e = f();
    if (e != cudaSuccess) {
        return ffb_fail(FF_ERR_CUDA, std::string("CUDA: ") + cudaGetErrorString(e));
    }
    return FF_OK;
}

ff_status check_shape(int B, int H, int W) {
    if (B <= 0 || H <= 0 || W <= 0) {
        return ffb_fail(FF_ERR_INVALID_ARGUMENT, "batch, height and width must be positive");
    }
    return FF_OK;
}

}  // namespace

// two-channel fields are read as one vector per pixel: their base must be aligned to a pair
bool pairs_aligned(int dtype, std::initializer_list<const void*> ps) {
    const uintptr_t a = dtype ? 16 : 8;
    for (const void* p : ps)
        if (p && (uintptr_t)p % a) return false;
    return true;
}

#define PAIRS_OR_RETURN(dtype, ...)                                                                   \
    do {                                                                                              \
        if (!pairs_aligned(dtype, {__VA_ARGS__})) {                                                   \
            return ffb_fail(FF_ERR_INVALID_ARGUMENT, "two-channel fields must be aligned to two elements (8 or 16 bytes)");                                                           \
        }                                                                                             \
    } while (0)

#define SHAPE_OR_RETURN(B, H, W)                   \
    do {                                           \
        ff_status st_ = check_shape(B, H, W);      \
        if (st_ != FF_OK) return st_;              \
    } while (0)

extern "C" {

ff_status ff_diff_pyramid(int dtype, int B, int H, int W, const void* in, void* out, void* stream) {
    SHAPE_OR_RETURN(B, H, W);
    return run(dtype, [&] {
        return dtype ? pyramid<double>(false, B, H, W, in, out, (cudaStream_t)stream)
                     : pyramid<float>(false, B, H, W, in, out, (cudaStream_t)stream);
    });
}

ff_status ff_diff_pyramid_bwd(int dtype, int B, int H, int W, const void* gout, void* gin, void* stream) {
    SHAPE_OR_RETURN(B, H, W);
    return run(dtype, [&] {
        return dtype ? pyramid<double>(true, B, H, W, gout, gin, (cudaStream_t)stream)
                     : pyramid<float>(true, B, H, W, gout, gin, (cudaStream_t)stream);
    });
}

ff_status ff_diff_model(int dtype, int B, int H, int W, const void* img, void* a0, void* grad, void* stream) {
    SHAPE_OR_RETURN(B, H, W);
    cudaStream_t s = (cudaStream_t)stream;
    return run(dtype, [&] {
        if (dtype) return launch_k(model_fwd_k<double>, grid3(W, H, B), kBlock, 0, s, (const double*)img, (double*)a0,
                                   (double*)grad, H, W);
        return launch_k(model_fwd_k<float>, grid3(W, H, B), kBlock, 0, s, (const float*)img, (float*)a0, (float*)grad,
                        H, W);
    });
}

ff_status ff_diff_model_bwd(int dtype, int B, int H, int W, const void* ga0, const void* ggrad, void* gby, void* gbx,
                            void* gimg, void* stream) {
    SHAPE_OR_RETURN(B, H, W);
    cudaStream_t s = (cudaStream_t)stream;
    return run(dtype, [&] {
        cudaError_t e;
        if (dtype) {
            e = launch_k(model_bwd1_k<double>, grid3(W, H, B), kBlock, 0, s, (const double*)ga0, (const double*)ggrad,
                         (double*)gby, (double*)gbx, H, W);
            if (e == cudaSuccess)
                e = launch_k(model_bwd2_k<double>, grid3(W, H, B), kBlock, 0, s, (const double*)gby,
                             (const double*)gbx, (double*)gimg, H, W);
            return e;
        }
        e = launch_k(model_bwd1_k<float>, grid3(W, H, B), kBlock, 0, s, (const float*)ga0, (const float*)ggrad,
                     (float*)gby, (float*)gbx, H, W);
        if (e == cudaSuccess)
            e = launch_k(model_bwd2_k<float>, grid3(W, H, B), kBlock, 0, s, (const float*)gby, (const float*)gbx,
                         (float*)gimg, H, W);
        return e;
    });
}

ff_status ff_diff_propagate(int dtype, int B, int H, int W, int axis, int payload, double dt, int border,
                            const void* f, const void* sc, const void* v, void* fo, void* so, void* vo,
                            void* stream) {
    SHAPE_OR_RETURN(B, H, W);
    if ((axis != 0 && axis != 1) || border < 0) {
        return ffb_fail(FF_ERR_INVALID_ARGUMENT, "axis must be 0 or 1 and border >= 0");
    }
    cudaStream_t s = (cudaStream_t)stream;
    return run(dtype, [&] {
        const dim3 g = grid3(W, H, B);
#define PROP_F(T, A, P)                                                                                          \
    launch_k(prop_fwd_k<T, A, P>, g, kBlock, 0, s, (const T*)f, (const T*)sc, (const T*)v, (T*)fo, (T*)so, (T*)vo, H, \
             W, (T)dt, border)
        if (dtype) {
            if (axis == 0) return payload ? PROP_F(double, 0, true) : PROP_F(double, 0, false);
            return payload ? PROP_F(double, 1, true) : PROP_F(double, 1, false);
        }
        if (axis == 0) return payload ? PROP_F(float, 0, true) : PROP_F(float, 0, false);
        return payload ? PROP_F(float, 1, true) : PROP_F(float, 1, false);
#undef PROP_F
    });
}

ff_status ff_diff_propagate_bwd(int dtype, int B, int H, int W, int axis, int payload, double dt, int border,
                                const void* f, const void* sc, const void* v, const void* gfo, const void* gso,
                                const void* gvo, void* gf, void* gs, void* gv, void* stream) {
    SHAPE_OR_RETURN(B, H, W);
    PAIRS_OR_RETURN(dtype, f, v, gfo, gvo, gf, gv);
    if ((axis != 0 && axis != 1) || border < 0) {
        return ffb_fail(FF_ERR_INVALID_ARGUMENT, "axis must be 0 or 1 and border >= 0");
    }
    cudaStream_t s = (cudaStream_t)stream;
    return run(dtype, [&] {
        const dim3 g = grid3(W, H, B);
#define PROP_B(T, A, P)                                                                                         \
    launch_k(prop_bwd_k<T, A, P>, g, kBlock, 0, s, (const T*)f, (const T*)sc, (const T*)v, (const T*)gfo,        \
             (const T*)gso, (const T*)gvo, (T*)gf, (T*)gs, (T*)gv, H, W, (T)dt, border)
        if (dtype) {
            if (axis == 0) return payload ? PROP_B(double, 0, true) : PROP_B(double, 0, false);
            return payload ? PROP_B(double, 1, true) : PROP_B(double, 1, false);
        }
        if (axis == 0) return payload ? PROP_B(float, 0, true) : PROP_B(float, 0, false);
        return payload ? PROP_B(float, 1, true) : PROP_B(float, 1, false);
#undef PROP_B
    });
}

ff_status ff_diff_update(int dtype, int B, int H, int W, const void* a0, const void* grad, const void* old,
                         const void* fhat, const void* gamma, double maxflow, void* out, void* stream) {
    SHAPE_OR_RETURN(B, H, W);
    cudaStream_t s = (cudaStream_t)stream;
    return run(dtype, [&] {
        if (dtype)
            return launch_k(update_fwd_k<double>, grid3(W, H, B), kBlock, 0, s, (const double*)a0, (const double*)grad,
                            (const double*)old, (const double*)fhat, (const double*)gamma, (double*)out, H, W,
                            maxflow);
        return launch_k(update_fwd_k<float>, grid3(W, H, B), kBlock, 0, s, (const float*)a0, (const float*)grad,
                        (const float*)old, (const float*)fhat, (const float*)gamma, (float*)out, H, W, (float)maxflow);
    });
}

ff_status ff_diff_update_bwd(int dtype, int B, int H, int W, const void* a0, const void* grad, const void* old,
                             const void* fhat, const void* gamma, double maxflow, const void* gout, void* ga0,
                             void* ggrad, void* gold, void* gfhat, void* ggamma, void* stream) {
    SHAPE_OR_RETURN(B, H, W);
    cudaStream_t s = (cudaStream_t)stream;
    return run(dtype, [&] {
        if (dtype)
            return launch_k(update_bwd_k<double>, grid3(W, H, B), kBlock, 0, s, (const double*)a0, (const double*)grad,
                            (const double*)old, (const double*)fhat, (const double*)gamma, (const double*)gout,
                            (double*)ga0, (double*)ggrad, (double*)gold, (double*)gfhat, (double*)ggamma, H, W,
                            maxflow);
        return launch_k(update_bwd_k<float>, grid3(W, H, B), kBlock, 0, s, (const float*)a0, (const float*)grad,
                        (const float*)old, (const float*)fhat, (const float*)gamma, (const float*)gout, (float*)ga0,
                        (float*)ggrad, (float*)gold, (float*)gfhat, (float*)ggamma, H, W, (float)maxflow);
    });
}

ff_status ff_diff_delta_update(int dtype, int B, int H, int W, int Hc, int Wc, const void* a0, const void* grad,
                               const void* old, const void* dhat, const void* coarse, const void* gamma,
                               double maxflow, void* flow, void* delta, void* stream) {
    SHAPE_OR_RETURN(B, H, W);
    SHAPE_OR_RETURN(B, Hc, Wc);
    cudaStream_t s = (cudaStream_t)stream;
    return run(dtype, [&] {
        if (dtype)
            return launch_k(dupdate_fwd_k<double>, grid3(W, H, B), kBlock, 0, s, (const double*)a0,
                            (const double*)grad, (const double*)old, (const double*)dhat, (const double*)coarse,
                            (const double*)gamma, (double*)flow, (double*)delta, H, W, Hc, Wc, maxflow);
        return launch_k(dupdate_fwd_k<float>, grid3(W, H, B), kBlock, 0, s, (const float*)a0, (const float*)grad,
                        (const float*)old, (const float*)dhat, (const float*)coarse, (const float*)gamma, (float*)flow,
                        (float*)delta, H, W, Hc, Wc, (float)maxflow);
    });
}

ff_status ff_diff_delta_update_bwd(int dtype, int B, int H, int W, int Hc, int Wc, const void* a0, const void* grad,
                                   const void* old, const void* dhat, const void* coarse, const void* gamma,
                                   double maxflow, const void* gflow, const void* gdelta, void* ga0, void* ggrad,
                                   void* gold, void* gdhat, void* gcoarse, void* ggamma, void* stream) {
    SHAPE_OR_RETURN(B, H, W);
    SHAPE_OR_RETURN(B, Hc, Wc);
    cudaStream_t s = (cudaStream_t)stream;
    return run(dtype, [&] {
        if (dtype)
            return launch_k(dupdate_bwd_k<double>, grid3(W, H, B), kBlock, 0, s, (const double*)a0,
                            (const double*)grad, (const double*)old, (const double*)dhat, (const double*)coarse,
                            (const double*)gamma, (const double*)gflow, (const double*)gdelta, (double*)ga0,
                            (double*)ggrad, (double*)gold, (double*)gdhat, (double*)gcoarse, (double*)ggamma, H, W, Hc,
                            Wc, maxflow);
        return launch_k(dupdate_bwd_k<float>, grid3(W, H, B), kBlock, 0, s, (const float*)a0, (const float*)grad,
                        (const float*)old, (const float*)dhat, (const float*)coarse, (const float*)gamma,
                        (const float*)gflow, (const float*)gdelta, (float*)ga0, (float*)ggrad, (float*)gold,
                        (float*)gdhat, (float*)gcoarse, (float*)ggamma, H, W, Hc, Wc, (float)maxflow);
    });
}

ff_status ff_diff_smooth(int dtype, int B, int H, int W, int axis, const void* w5, const void* in, void* out,
                         void* stream) {
    SHAPE_OR_RETURN(B, H, W);
    if (axis != 0 && axis != 1) {
        return ffb_fail(FF_ERR_INVALID_ARGUMENT, "axis must be 0 or 1");
    }
    cudaStream_t s = (cudaStream_t)stream;
    return run(dtype, [&] {
        const dim3 g = grid3(W, H, B);
        if (dtype)
            return axis == 0 ? launch_k(smooth_fwd_k<double, 0>, g, kBlock, 0, s, (const double*)w5,
                                        (const double*)in, (double*)out, H, W, (double*)nullptr)
                             : launch_k(smooth_fwd_k<double, 1>, g, kBlock, 0, s, (const double*)w5,
                                        (const double*)in, (double*)out, H, W, (double*)nullptr);
        return axis == 0 ? launch_k(smooth_fwd_k<float, 0>, g, kBlock, 0, s, (const float*)w5, (const float*)in,
                                    (float*)out, H, W, (float*)nullptr)
                         : launch_k(smooth_fwd_k<float, 1>, g, kBlock, 0, s, (const float*)w5, (const float*)in,
                                    (float*)out, H, W, (float*)nullptr);
    });
}

ff_status ff_diff_smooth_bwd(int dtype, int B, int H, int W, int axis, const void* w5, const void* in,
                             const void* gout, void* gin, void* gw5, void* stream) {
    SHAPE_OR_RETURN(B, H, W);
    PAIRS_OR_RETURN(dtype, in, gout, gin);
    if (axis != 0 && axis != 1) {
        return ffb_fail(FF_ERR_INVALID_ARGUMENT, "axis must be 0 or 1");
    }
    cudaStream_t s = (cudaStream_t)stream;
    return run(dtype, [&] {
        const dim3 g = grid_smooth(W, H, B);
        if (dtype)
            return axis == 0 ? launch_k(smooth_bwd_k<double, 0>, g, kBlock, 0, s, (const double*)w5,
                                        (const double*)in, (const double*)gout, (double*)gin, (double*)gw5, H, W)
                             : launch_k(smooth_bwd_k<double, 1>, g, kBlock, 0, s, (const double*)w5,
                                        (const double*)in, (const double*)gout, (double*)gin, (double*)gw5, H, W);
        return axis == 0 ? launch_k(smooth_bwd_k<float, 0>, g, kBlock, 0, s, (const float*)w5, (const float*)in,
                                    (const float*)gout, (float*)gin, (float*)gw5, H, W)
                         : launch_k(smooth_bwd_k<float, 1>, g, kBlock, 0, s, (const float*)w5, (const float*)in,
                                    (const float*)gout, (float*)gin, (float*)gw5, H, W);
    });
}

}  // extern "C"

extern "C" {

size_t ff_diff_epe_scratch_bytes(int dtype) { return (size_t)ffb::diff::kEpeBlocks * (dtype ? 8 : 4); }

ff_status ff_diff_epe(int dtype, int B, int T, int H, int W, int first, double eps, const void* flows,
                      const void* truth, long long truth_bstride, long long truth_tstride, void* loss, void* scratch,
                      void* stream) {
    using namespace ffb::diff;
    if (dtype != 0 && dtype != 1) return ffb_fail(FF_ERR_INVALID_ARGUMENT, "dtype must be 0 (float32) or 1 (float64)");
    if (B < 1 || T < 1 || H < 1 || W < 1 || first < 0 || first >= T || !(eps >= 0))
        return ffb_fail(FF_ERR_INVALID_ARGUMENT, "ff_diff_epe: bad shape, first frame or eps");
    if (!flows || !truth || !loss || !scratch) return ffb_fail(FF_ERR_INVALID_ARGUMENT, "ff_diff_epe: null pointer");
    if (!::pairs_aligned(dtype, {flows, truth}) || (truth_bstride | truth_tstride) & 1)
        return ffb_fail(FF_ERR_INVALID_ARGUMENT, "ff_diff_epe: flow pairs must be aligned to two elements");
    const EpeGeom g{B, T, first, (long long)H * W, truth_bstride, truth_tstride};
    const double inv = 1.0 / ((double)B * (T - first) * H * W);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    if (dtype) {
        e = ffb::launch_k(epe_fwd_k<double>, dim3(kEpeBlocks), dim3(kEpeThreads), 0, s, (const double*)flows,
                          (const double*)truth, g, eps, (double*)scratch);
        if (e == cudaSuccess)
            e = ffb::launch_k(epe_sum_k<double>, dim3(1), dim3(1024), 0, s, (const double*)scratch, kEpeBlocks, inv,
                              (double*)loss);
    } else {
        e = ffb::launch_k(epe_fwd_k<float>, dim3(kEpeBlocks), dim3(kEpeThreads), 0, s, (const float*)flows,
                          (const float*)truth, g, (float)eps, (float*)scratch);
        if (e == cudaSuccess)
            e = ffb::launch_k(epe_sum_k<float>, dim3(1), dim3(1024), 0, s, (const float*)scratch, kEpeBlocks,
                              (float)inv, (float*)loss);
    }
    return e == cudaSuccess ? FF_OK : ffb_fail(FF_ERR_CUDA, std::string("CUDA: ") + cudaGetErrorString(e));
}

ff_status ff_diff_epe_bwd(int dtype, int B, int T, int H, int W, int first, double eps, const void* flows,
                          const void* truth, long long truth_bstride, long long truth_tstride, const void* grad_loss,
                          void* grad_flows, void* stream) {
    using namespace ffb::diff;
    if (dtype != 0 && dtype != 1) return ffb_fail(FF_ERR_INVALID_ARGUMENT, "dtype must be 0 (float32) or 1 (float64)");
    if (B < 1 || T < 1 || H < 1 || W < 1 || first < 0 || first >= T || !(eps >= 0))
        return ffb_fail(FF_ERR_INVALID_ARGUMENT, "ff_diff_epe_bwd: bad shape, first frame or eps");
    if (!flows || !truth || !grad_loss || !grad_flows)
        return ffb_fail(FF_ERR_INVALID_ARGUMENT, "ff_diff_epe_bwd: null pointer");
    if (!::pairs_aligned(dtype, {flows, truth, grad_flows}) || (truth_bstride | truth_tstride) & 1)
        return ffb_fail(FF_ERR_INVALID_ARGUMENT, "ff_diff_epe_bwd: flow pairs must be aligned to two elements");
    const EpeGeom g{B, T, first, (long long)H * W, truth_bstride, truth_tstride};
    const double inv = 1.0 / ((double)B * (T - first) * H * W);
    cudaStream_t s = (cudaStream_t)stream;
    const cudaError_t e =
        dtype ? ffb::launch_k(epe_bwd_k<double>, dim3(kEpeBlocks), dim3(kEpeThreads), 0, s, (const double*)flows,
                              (const double*)truth, g, eps, (const double*)grad_loss, inv, (double*)grad_flows)
              : ffb::launch_k(epe_bwd_k<float>, dim3(kEpeBlocks), dim3(kEpeThreads), 0, s, (const float*)flows,
                              (const float*)truth, g, (float)eps, (const float*)grad_loss, (float)inv,
                              (float*)grad_flows);
    return e == cudaSuccess ? FF_OK : ffb_fail(FF_ERR_CUDA, std::string("CUDA: ") + cudaGetErrorString(e));
}

}  // extern "C"

// ------------------------------------------------------------------ frame driver
// One frame of the differentiable pyramidal filter (and its adjoint) as one host call that
// launches every stage kernel itself: the same recurrence as flowfilter_b200.diff composes
// from the stage Functions (pyramid, then the top level, then the delta levels from L-2
// down to 0), with every intermediate the adjoint needs kept in a caller-provided tape.
namespace ffb {
namespace diff {
namespace {

struct Geo {
    int B, L, border;
    int H[FF_DIFF_MAX_LEVELS], W[FF_DIFF_MAX_LEVELS], N[FF_DIFF_MAX_LEVELS], S[FF_DIFF_MAX_LEVELS];
    double maxflow[FF_DIFF_MAX_LEVELS];
    size_t n1(int l) const { return (size_t)B * H[l] * W[l]; }
};

Geo geo_of(const ff_diff_geom* g) {
    if (!g || g->levels < 1 || g->levels > FF_DIFF_MAX_LEVELS || g->batch < 1 || g->border < 0)
        throw std::invalid_argument("bad differentiable-filter geometry");
    Geo o{};
    o.B = g->batch;
    o.L = g->levels;
    o.border = g->border;
    for (int l = 0; l < o.L; ++l) {
        o.H[l] = g->height[l];
        o.W[l] = g->width[l];
        o.N[l] = g->iterations[l];
        o.S[l] = g->smooth[l];
        o.maxflow[l] = g->maxflow[l];
        if (o.H[l] < 1 || o.W[l] < 1 || o.N[l] < 1 || o.S[l] < 0) throw std::invalid_argument("bad level geometry");
        if (l > 0 && (o.H[l] != o.H[l - 1] / 2 || o.W[l] != o.W[l - 1] / 2))
            throw std::invalid_argument("level sizes must halve");
    }
    return o;
}

// offsets (in elements of T) of the forward's intermediates.  As a tape, everything the
// adjoint reads gets its own place.  Compact (a forward without adjoint): the buffers are
// reused as soon as the forward is done with them, and only the level images and the top
// level's unsmoothed flow (the coarse flow of level L-2) stay apart.
struct Tape {
    size_t img[FF_DIFF_MAX_LEVELS] = {};                // level images, l >= 1
    size_t grad[FF_DIFF_MAX_LEVELS] = {};               // image gradients
    std::vector<size_t> prop[FF_DIFF_MAX_LEVELS];       // outputs of sub-steps 0..2N-1
    std::vector<size_t> sm[FF_DIFF_MAX_LEVELS];         // inputs of smoothing passes (sm[0] = update output)
    size_t total = 0;
    Tape(const Geo& g, bool compact = false) {
        auto take = [&](size_t n) {
            size_t at = total;
            total += (n + 31) / 32 * 32;
            return at;
        };
        if (compact) {
            size_t n1m = 0, stm = 0;
            for (int l = 0; l < g.L; ++l) {
                n1m = std::max(n1m, g.n1(l));
                stm = std::max(stm, (l < g.L - 1 ? 5 : 2) * g.n1(l));
                if (l > 0) img[l] = take(g.n1(l));
            }
            const size_t gr = take(2 * n1m), pa = take(stm), pb = take(stm), sa = take(2 * n1m), sb = take(2 * n1m);
            const size_t fu_top = take(2 * g.n1(g.L - 1));
            for (int l = 0; l < g.L; ++l) {
                grad[l] = gr;
                for (int k = 1; k <= 2 * g.N[l]; ++k) prop[l].push_back(k % 2 ? pa : pb);
                // pass j reads sm[j] and writes sm[j+1]: two buffers alternate after sm[0]
                const int ns = std::max(2 * g.S[l], 1);
                for (int k = 0; k < ns; ++k)
                    sm[l].push_back(k == 0 ? (l == g.L - 1 ? fu_top : sa) : (k % 2 ? sb : sa));
            }
            return;
        }
        for (int l = 0; l < g.L; ++l) {
            const size_t n1 = g.n1(l), n2 = 2 * n1;
            const bool delta = l < g.L - 1;
            const size_t state = delta ? n2 + n1 + n2 : n2;  // (f, s, v) or f
            if (l > 0) img[l] = take(n1);
            grad[l] = take(n2);
            for (int k = 1; k <= 2 * g.N[l]; ++k) prop[l].push_back(take(state));
            for (int k = 0; k < std::max(2 * g.S[l], 1); ++k) sm[l].push_back(take(n2));
        }
    }
};

inline size_t blocks_of(const Geo& g, int l) {
    const dim3 d = grid3(g.W[l], g.H[l], g.B);
    return (size_t)d.x * d.y * d.z;
}

// blocks of the fused smoothing adjoint at level l
inline size_t tiles32_of(const Geo& g, int l) {
    const dim3 d = grid_tile32(g.W[l], g.H[l], g.B);
    return (size_t)d.x * d.y * d.z;
}

// backward scratch (elements of T)
struct Scratch {
    size_t gimg[FF_DIFF_MAX_LEVELS] = {};  // image gradients of levels >= 1
    // per-block partial sums: weight gradients (S iterations x tiles x 5) and gamma gradient
    // (update blocks x 1) of each level, reduced together at the end of the frame
    size_t part_w[FF_DIFF_MAX_LEVELS] = {}, part_g[FF_DIFF_MAX_LEVELS] = {};
    size_t ga0, gg, gfu, pa, pb, sa, sb, zero;
    size_t total = 0;
    Scratch(const Geo& g) {
        auto take = [&](size_t n) {
            size_t at = total;
            total += (n + 31) / 32 * 32;
            return at;
        };
        size_t n1m = 0;
        for (int l = 0; l < g.L; ++l) {
            if (l > 0) gimg[l] = take(g.n1(l));
            n1m = std::max(n1m, g.n1(l));
            part_w[l] = take((size_t)std::max(g.S[l], 1) * tiles32_of(g, l) * 5);
            part_g[l] = take(blocks_of(g, l));
        }
        const size_t n2m = 2 * n1m, st = n2m + n1m + n2m;
        ga0 = take(n1m);
        gg = take(n2m);
        gfu = take(2 * g.n1(g.L - 1));
        pa = take(st);
        pb = take(st);
        sa = take(n2m);
        sb = take(n2m);
        zero = take(n2m);  // zeros standing in for absent output gradients
    }
};

template <typename T>
struct Driver {
    const Geo& g;
    cudaStream_t s;
    Driver(const Geo& g_, cudaStream_t s_) : g(g_), s(s_) {}
    void ok(cudaError_t e) const {
        if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
    }
    dim3 grid(int l) const { return grid3(g.W[l], g.H[l], g.B); }
    void zero(T* p, size_t n) const { ok(cudaMemsetAsync(p, 0, n * sizeof(T), s)); }
    void copy(T* dst, const T* src, size_t n) const {
        ok(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
    }
    void add(T* dst, const T* src, size_t n) const {
        ok(launch_k(add_k<T>, dim3((unsigned)std::min<size_t>((n + 255) / 256, 4096)), dim3(256), 0, s, dst, src, n));
    }
    void reduce(const ReduceJobs<T>& jobs) const {
        if (jobs.count > 0) ok(launch_k(reduce_jobs_k<T>, dim3(jobs.count), dim3(1024), 0, s, jobs));
    }
    void prop(int l, int axis, bool payload, const T* f, const T* sc, const T* v, T* fo, T* so, T* vo) const {
        const T dt = (T)(1.0 / g.N[l]);
        const int H = g.H[l], W = g.W[l], b = g.border;
        cudaError_t e;
        if (payload) {
            e = axis == 0 ? launch_k(prop_fwd_k<T, 0, true>, grid(l), kBlock, 0, s, f, sc, v, fo, so, vo, H, W, dt, b)
                          : launch_k(prop_fwd_k<T, 1, true>, grid(l), kBlock, 0, s, f, sc, v, fo, so, vo, H, W, dt, b);
        } else {
            e = axis == 0 ? launch_k(prop_fwd_k<T, 0, false>, grid(l), kBlock, 0, s, f, sc, v, fo, so, vo, H, W, dt, b)
                          : launch_k(prop_fwd_k<T, 1, false>, grid(l), kBlock, 0, s, f, sc, v, fo, so, vo, H, W, dt, b);
        }
        ok(e);
    }
    void smooth(int l, int axis, const T* w5, const T* in, T* out, T* out2 = nullptr) const {
        ok(axis == 0 ? launch_k(smooth_fwd_k<T, 0>, grid(l), kBlock, 0, s, w5, in, out, g.H[l], g.W[l], out2)
                     : launch_k(smooth_fwd_k<T, 1>, grid(l), kBlock, 0, s, w5, in, out, g.H[l], g.W[l], out2));
    }
    // one propagation iteration's adjoint (X and Y sub-step): X input x*, Y input y*, output
    // gradient g*o, X input gradient g* (stored, or added when ACC)
    template <bool PAYLOAD, bool ACC>
    void prop_iter_bwd(int l, const T* xf, const T* xs, const T* xv, const T* yf, const T* ys, const T* yv,
                       const T* gfo, const T* gso, const T* gvo, T* gf, T* gs, T* gv) const {
        constexpr size_t smem = sizeof(PropTile<T, PAYLOAD>);
        static bool prepared[64] = {};  // the dynamic shared-memory limit, set once per device
        int dev = 0;
        ok(cudaGetDevice(&dev));
        if (!prepared[dev & 63]) {
            ok(cudaFuncSetAttribute(prop_iter_bwd_k<T, PAYLOAD, ACC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
            prepared[dev & 63] = true;
        }
        const T dt = (T)(1.0 / g.N[l]);
        ok(launch_k(prop_iter_bwd_k<T, PAYLOAD, ACC>, grid_tile32(g.W[l], g.H[l], g.B), dim3(32, kPropThreads / 32),
                    smem, s, xf, xs, xv,
                    yf, ys, yv, gfo, gso, gvo, gf, gs, gv, g.H[l], g.W[l], dt, g.border));
    }
    // one smoothing iteration's adjoint (X and Y pass): input gradient stored (or added),
    // weight sums per block
    void smooth_iter_bwd(int l, bool acc, const T* w5, const T* xin, const T* xmid, const T* go, T* gi, T* part,
                         const T* go2 = nullptr, long long go2_bstride = 0) const {
        const dim3 gr = grid_tile32(g.W[l], g.H[l], g.B);
        const int H = g.H[l], W = g.W[l];
        constexpr size_t smem = smooth_iter_smem<T>();
        static bool prepared[64][4] = {};  // the dynamic shared-memory limit, set once per device
        int dev = 0;
        ok(cudaGetDevice(&dev));
        const int v = (acc ? 1 : 0) + (go2 ? 2 : 0);
        auto kern = v == 0 ? smooth_iter_bwd_k<T, false, false>
                  : v == 1 ? smooth_iter_bwd_k<T, true, false>
                  : v == 2 ? smooth_iter_bwd_k<T, false, true>
                           : smooth_iter_bwd_k<T, true, true>;
        if (!prepared[dev & 63][v]) {
            ok(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            prepared[dev & 63][v] = true;
        }
        ok(launch_k(kern, gr, kBlock, smem, s, w5, xin, xmid, go, go2, go2_bstride, gi, part, H, W));
    }
    void model(int l, const T* img, T* a0, T* grad) const {
        ok(launch_k(model_fwd_k<T>, grid(l), kBlock, 0, s, img, a0, grad, g.H[l], g.W[l]));
    }
    // image gradient of the image model: stored into gimg, or added when acc
    void model_bwd(int l, bool acc, const T* ga0, const T* ggrad, T* gimg) const {
        constexpr size_t smem = model_tile_smem<T>();
        static bool prepared[64][2] = {};  // the dynamic shared-memory limit, set once per device
        int dev = 0;
        ok(cudaGetDevice(&dev));
        if (!prepared[dev & 63][acc]) {
            ok(acc ? cudaFuncSetAttribute(model_tile_bwd_k<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem)
                   : cudaFuncSetAttribute(model_tile_bwd_k<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
            prepared[dev & 63][acc] = true;
        }
        const dim3 gr = grid_tile32(g.W[l], g.H[l], g.B);
        ok(acc ? launch_k(model_tile_bwd_k<T, true>, gr, kBlock, smem, s, ga0, ggrad, gimg, g.H[l], g.W[l])
               : launch_k(model_tile_bwd_k<T, false>, gr, kBlock, smem, s, ga0, ggrad, gimg, g.H[l], g.W[l]));
    }

    // ---- forward
    // y_out (nullable): a second copy of level 0's smoothed flow
    void forward(bool first, const T* frame, const T* gamma, const T* weights, const T* const* in, T* const* out,
                 T* fu_out, T* tp, bool compact = false, T* y_out = nullptr) const {
        const Tape tape(g, compact);
        const int L = g.L, top = L - 1;
        auto img = [&](int l) -> const T* { return l == 0 ? frame : tp + tape.img[l]; };
        for (int l = 1; l < L; ++l)
            ok(launch_k(pyr_fwd_k<T>, grid3(g.W[l], g.H[l], g.B), kBlock, 0, s, img(l - 1), tp + tape.img[l],
                        g.H[l - 1], g.W[l - 1]));
        // top level: flow propagation, update, smoothing
        {
            const int l = top;
            const size_t n2 = 2 * g.n1(l);
            T* a0 = out[3 * l + 1];
            T* grad = tp + tape.grad[l];
            model(l, img(l), a0, grad);
            const T* f = in[3 * l];
            for (int k = 0; k < 2 * g.N[l]; ++k) {
                T* fo = tp + tape.prop[l][k];
                prop(l, k % 2, false, f, nullptr, nullptr, fo, nullptr, nullptr);
                f = fo;
            }
            const T* old = first ? a0 : in[3 * l + 1];
            T* fu = tp + tape.sm[l][0];
            ok(launch_k(update_fwd_k<T>, grid(l), kBlock, 0, s, (const T*)a0, (const T*)grad, old, f, gamma + l, fu,
                        g.H[l], g.W[l], (T)g.maxflow[l]));
            if (fu_out) copy(fu_out, fu, n2);
            smooth_chain(l, weights + 5 * l, tape, tp, out[3 * l], l == 0 ? y_out : nullptr);
            copy(out[3 * l + 2], in[3 * l + 2], n2);
        }
        // delta levels, L-2 down to 0
        for (int l = L - 2; l >= 0; --l) {
            const size_t n1 = g.n1(l), n2 = 2 * n1;
            T* a0 = out[3 * l + 1];
            T* grad = tp + tape.grad[l];
            model(l, img(l), a0, grad);
            const T *f = in[3 * l], *sc = in[3 * l + 1], *v = in[3 * l + 2];
            for (int k = 0; k < 2 * g.N[l]; ++k) {
                T* base = tp + tape.prop[l][k];
                prop(l, k % 2, true, f, sc, v, base, base + n2, base + n2 + n1);
                f = base;
                sc = base + n2;
                v = base + n2 + n1;
            }
            const T* old = first ? a0 : sc;
            const T* coarse = l == L - 2 ? tp + tape.sm[top][0] : in[3 * (l + 1)];
            T* flow = tp + tape.sm[l][0];
            ok(launch_k(dupdate_fwd_k<T>, grid(l), kBlock, 0, s, (const T*)a0, (const T*)grad, old, v, coarse,
                        gamma + l, flow, out[3 * l + 2], g.H[l], g.W[l], g.H[l + 1], g.W[l + 1], (T)g.maxflow[l]));
            smooth_chain(l, weights + 5 * l, tape, tp, out[3 * l], l == 0 ? y_out : nullptr);
        }
    }
    // 2S passes from tape.sm[l][0]; pass j writes tape.sm[l][j+1], the last writes `last` (and
    // `last2`, when given)
    void smooth_chain(int l, const T* w5, const Tape& tape, T* tp, T* last, T* last2 = nullptr) const {
        const int n = 2 * g.S[l];
        if (n == 0) {
            copy(last, tp + tape.sm[l][0], 2 * g.n1(l));
            if (last2) copy(last2, tp + tape.sm[l][0], 2 * g.n1(l));
        }
        for (int j = 0; j < n; ++j)
            smooth(l, j % 2, w5, tp + tape.sm[l][j], j + 1 < n ? tp + tape.sm[l][j + 1] : last, j + 1 < n ? nullptr : last2);
    }

    // ---- backward: gradients of the outputs -> gradients of the inputs, ADDED into the
    // caller's buffers.  Inside, every intermediate gradient is stored by the kernel that
    // produces it (no clearing), and only the kernels writing the caller's buffers add.
    // gy (nullable): a second gradient of level 0's smoothed flow (of the forward's y_out),
    // image i at gy + i * gy_bstride
    void backward(bool first, const T* frame, const T* gamma, const T* weights, const T* const* in,
                  const T* const* out, const T* tp, const T* const* gout, const T* gfu_out, const T* gy,
                  long long gy_bstride, T* gframe, T* ggamma, T* gweights, T* const* gin, T* sc_) const {
        (void)frame;
        const Tape tape(g);
        const Scratch S_(g);
        const int L = g.L, top = L - 1;
        // image gradients: level 0's is the caller's frame gradient itself
        T* gimg[FF_DIFF_MAX_LEVELS];
        gimg[0] = gframe;
        for (int l = 1; l < L; ++l) gimg[l] = sc_ + S_.gimg[l];
        // zeros standing in for an absent output gradient, cleared at the first such use
        T* const zbuf = sc_ + S_.zero;
        bool zeroed = false;
        auto gz = [&](const T* p) {
            if (p) return p;
            if (!zeroed) zero(zbuf, 2 * g.n1(0));
            zeroed = true;
            return (const T*)zbuf;
        };
        // gradient of the top level's unsmoothed flow: the caller's, the coarse reads of level
        // L-2 (scattered by its update adjoint) and the top's smoothing adjoint, in that order
        T* gfu = sc_ + S_.gfu;
        if (gfu_out) copy(gfu, gfu_out, 2 * g.n1(top));
        else zero(gfu, 2 * g.n1(top));
        T *ga0 = sc_ + S_.ga0, *ggr = sc_ + S_.gg;
        T *pa = sc_ + S_.pa, *pb = sc_ + S_.pb, *sa = sc_ + S_.sa, *sb = sc_ + S_.sb;
        // the partial sums of the weight and gamma gradients, reduced in one launch at the end
        ReduceJobs<T> jobs;
        auto jobs_add = [&](const T* part, int n, int nv, T* dst) {
            jobs.part[jobs.count] = part;
            jobs.n[jobs.count] = n;
            jobs.nv[jobs.count] = nv;
            jobs.dst[jobs.count] = dst;
            ++jobs.count;
        };

        // adjoint of the 2S smoothing passes of level l, from the gradient of the smoothed
        // flow; the gradient of the pass-0 input goes to dst (added if acc) and is returned.
        // Pass j > 0 writes bufs[j % 2]; pass 1 writes sb, so dst may be sa.
        auto smooth_back = [&](int l, const T* g_last, T* dst, bool acc) -> const T* {
            const int n = 2 * g.S[l];
            const T* g2 = l == 0 ? gy : nullptr;  // level 0: the second gradient joins here
            const T* gcur = gz(g_last);
            if (n == 0) {
                if (g2) {
                    const long long per = 2LL * g.H[l] * g.W[l];
                    const unsigned nb = (unsigned)std::min<long long>((g.B * per + 255) / 256, 4096);
                    ok(acc ? launch_k(sum2_k<T, true>, dim3(nb), dim3(256), 0, s, dst, g_last, g2, gy_bstride, per, g.B)
                           : launch_k(sum2_k<T, false>, dim3(nb), dim3(256), 0, s, dst, g_last, g2, gy_bstride, per,
                                      g.B));
                    return dst;
                }
                if (!acc) return gcur;
                add(dst, gcur, 2 * g.n1(l));
                return dst;
            }
            // iteration i reads the tape's pass inputs sm[2i] (X) and sm[2i+1] (Y); iteration
            // i > 0 writes bufs[i % 2], iteration 1 writes sb, so dst may be sa
            const size_t nb = tiles32_of(g, l);
            T* part = sc_ + S_.part_w[l];
            T* bufs[2] = {sa, sb};
            for (int i = g.S[l] - 1; i >= 0; --i) {
                T* o = i == 0 ? dst : bufs[i % 2];
                smooth_iter_bwd(l, i == 0 && acc, weights + 5 * l, tp + tape.sm[l][2 * i], tp + tape.sm[l][2 * i + 1],
                                gcur, o, part + i * nb * 5, i == g.S[l] - 1 ? g2 : nullptr, gy_bstride);
                gcur = o;
            }
            jobs_add(part, (int)(g.S[l] * nb), 5, gweights + 5 * l);
            return gcur;
        };

        for (int l = 0; l <= L - 2; ++l) {
            const size_t n1 = g.n1(l), n2 = 2 * n1;
            const T* a0 = out[3 * l + 1];
            const T* grad = tp + tape.grad[l];
            const int last = 2 * g.N[l] - 1;
            const T* fh_base = tp + tape.prop[l][last];
            const T* sh = fh_base + n2;
            const T* vh = fh_base + n2 + n1;
            const T* old = first ? a0 : sh;
            const T* coarse = l == L - 2 ? tp + tape.sm[top][0] : in[3 * (l + 1)];
            const T* gflow = smooth_back(l, gout[3 * l], sa, false);
            // gradients of the propagated (f, s, v): f is not read after propagation (zero),
            // s is the old image unless first, v the delta input of the solve
            T* gsh = pa + n2;
            T* gvh = pa + n2 + n1;
            T* gco = l == L - 2 ? gfu : gin[3 * (l + 1)];
            const FrameAdj<T> fa{gout[3 * l + 1], first ? 1 : 0, 0, sc_ + S_.part_g[l]};
            ok(launch_k(dupdate_bwd_frame_k<T>, grid(l), kBlock, 0, s, a0, grad, old, vh, coarse, gamma + l, gflow,
                        gz(gout[3 * l + 2]), ga0, ggr, gsh, gvh, gco, fa, g.H[l], g.W[l], g.H[l + 1], g.W[l + 1],
                        (T)g.maxflow[l]));
            jobs_add(sc_ + S_.part_g[l], (int)blocks_of(g, l), 1, ggamma + l);
            // iterations N-1 .. 0: the Y sub-step 2i+1 reads tape entry 2i, the X sub-step 2i
            // reads entry 2i-1 (the input state for i = 0, whose gradient goes to the caller's)
            const T *cf = nullptr, *cs = gsh, *cv = gvh;  // f is not read after propagation: no gradient
            T* bufs[2] = {pb, pa};
            for (int i = g.N[l] - 1; i >= 0; --i) {
                const T* yb = tp + tape.prop[l][2 * i];
                if (i == 0) {
                    prop_iter_bwd<true, true>(l, in[3 * l], in[3 * l + 1], in[3 * l + 2], yb, yb + n2, yb + n2 + n1, cf,
                                              cs, cv, gin[3 * l], gin[3 * l + 1], gin[3 * l + 2]);
                    break;
                }
                const T* xb = tp + tape.prop[l][2 * i - 1];
                T* o = bufs[(g.N[l] - 1 - i) % 2];
                prop_iter_bwd<true, false>(l, xb, xb + n2, xb + n2 + n1, yb, yb + n2, yb + n2 + n1, cf, cs, cv, o,
                                           o + n2, o + n2 + n1);
                cf = o;
                cs = o + n2;
                cv = o + n2 + n1;
            }
            model_bwd(l, l == 0, ga0, ggr, gimg[l]);
        }
        {
            const int l = top;
            const size_t n2 = 2 * g.n1(l);
            const T* a0 = out[3 * l + 1];
            const T* grad = tp + tape.grad[l];
            const int last = 2 * g.N[l] - 1;
            const T* fh = tp + tape.prop[l][last];
            const T* old = first ? a0 : in[3 * l + 1];
            smooth_back(l, gout[3 * l], gfu, true);
            T* gh = pa;
            const FrameAdj<T> fa{gout[3 * l + 1], first ? 1 : 0, 1, sc_ + S_.part_g[l]};
            ok(launch_k(update_bwd_frame_k<T>, grid(l), kBlock, 0, s, a0, grad, old, fh, gamma + l, (const T*)gfu, ga0,
                        ggr, gin[3 * l + 1], gh, fa, g.H[l], g.W[l], (T)g.maxflow[l]));
            jobs_add(sc_ + S_.part_g[l], (int)blocks_of(g, l), 1, ggamma + l);
            if (gout[3 * l + 2]) add(gin[3 * l + 2], gout[3 * l + 2], n2);
            const T* cur = gh;
            T* bufs[2] = {pb, pa};
            for (int i = g.N[l] - 1; i >= 0; --i) {
                const T* yb = tp + tape.prop[l][2 * i];
                if (i == 0) {
                    prop_iter_bwd<false, true>(l, in[3 * l], nullptr, nullptr, yb, nullptr, nullptr, cur, nullptr,
                                               nullptr, gin[3 * l], nullptr, nullptr);
                    break;
                }
                T* o = bufs[(g.N[l] - 1 - i) % 2];
                prop_iter_bwd<false, false>(l, tp + tape.prop[l][2 * i - 1], nullptr, nullptr, yb, nullptr, nullptr,
                                            cur, nullptr, nullptr, o, nullptr, nullptr);
                cur = o;
            }
            model_bwd(l, l == 0, ga0, ggr, gimg[l]);
        }
        // pyramid adjoint, coarse to fine, added into the finer level's image gradient
        for (int l = L - 1; l >= 1; --l)
            ok(launch_k(pyr_bwd_k<T>, grid3(g.W[l - 1], g.H[l - 1], g.B), kBlock, 0, s, (const T*)gimg[l], gimg[l - 1],
                        g.H[l - 1], g.W[l - 1]));
        reduce(jobs);
    }
};

template <typename F>
ff_status run_frame(F&& f) {
    try {
        f();
        return FF_OK;
    } catch (const std::invalid_argument& e) {
        return ffb_fail(FF_ERR_INVALID_ARGUMENT, e.what());
    } catch (const std::exception& e) {
        return ffb_fail(FF_ERR_CUDA, std::string("CUDA: ") + e.what());
    }
}

}  // namespace
}  // namespace diff
}  // namespace ffb

extern "C" {

size_t ff_diff_frame_tape_bytes(int dtype, const ff_diff_geom* geom) {
    try {
        return ffb::diff::Tape(ffb::diff::geo_of(geom)).total * (dtype ? 8 : 4);
    } catch (...) {
        return 0;
    }
}

size_t ff_diff_frame_scratch_bytes(int dtype, const ff_diff_geom* geom) {
    try {
        return ffb::diff::Scratch(ffb::diff::geo_of(geom)).total * (dtype ? 8 : 4);
    } catch (...) {
        return 0;
    }
}

ff_status ff_diff_frame_forward(int dtype, const ff_diff_geom* geom, int first, const void* frame, const void* gamma,
                                const void* weights, const void* const* state_in, void* const* state_out,
                                void* fu_out, void* y_out, void* tape, void* stream) {
    return ffb::diff::run_frame([&] {
        const ffb::diff::Geo g = ffb::diff::geo_of(geom);
        if (dtype != 0 && dtype != 1) throw std::invalid_argument("dtype must be 0 (float32) or 1 (float64)");
        if (!frame || !gamma || !weights || !state_in || !state_out || !tape)
            throw std::invalid_argument("null pointer argument");
        for (int k = 0; k < 3 * g.L; ++k)
            if (!::pairs_aligned(dtype, {state_in[k], state_out[k]}))
                throw std::invalid_argument("state fields must be aligned to two elements (8 or 16 bytes)");
        if (!::pairs_aligned(dtype, {y_out})) throw std::invalid_argument("y_out must be aligned to two elements");
        if (dtype) {
            ffb::diff::Driver<double>(g, (cudaStream_t)stream)
                .forward(first != 0, (const double*)frame, (const double*)gamma, (const double*)weights,
                         (const double* const*)state_in, (double* const*)state_out, (double*)fu_out, (double*)tape,
                         false, (double*)y_out);
        } else {
            ffb::diff::Driver<float>(g, (cudaStream_t)stream)
                .forward(first != 0, (const float*)frame, (const float*)gamma, (const float*)weights,
                         (const float* const*)state_in, (float* const*)state_out, (float*)fu_out, (float*)tape, false,
                         (float*)y_out);
        }
    });
}

size_t ff_diff_frame_infer_bytes(int dtype, const ff_diff_geom* geom) {
    try {
        return ffb::diff::Tape(ffb::diff::geo_of(geom), true).total * (dtype ? 8 : 4);
    } catch (...) {
        return 0;
    }
}

ff_status ff_diff_frame_infer(int dtype, const ff_diff_geom* geom, int first, const void* frame, const void* gamma,
                              const void* weights, const void* const* state_in, void* const* state_out, void* fu_out,
                              void* scratch, void* stream) {
    return ffb::diff::run_frame([&] {
        const ffb::diff::Geo g = ffb::diff::geo_of(geom);
        if (dtype != 0 && dtype != 1) throw std::invalid_argument("dtype must be 0 (float32) or 1 (float64)");
        if (!frame || !gamma || !weights || !state_in || !state_out || !scratch)
            throw std::invalid_argument("null pointer argument");
        for (int k = 0; k < 3 * g.L; ++k)
            if (!::pairs_aligned(dtype, {state_in[k], state_out[k]}))
                throw std::invalid_argument("state fields must be aligned to two elements (8 or 16 bytes)");
        if (dtype) {
            ffb::diff::Driver<double>(g, (cudaStream_t)stream)
                .forward(first != 0, (const double*)frame, (const double*)gamma, (const double*)weights,
                         (const double* const*)state_in, (double* const*)state_out, (double*)fu_out,
                         (double*)scratch, true);
        } else {
            ffb::diff::Driver<float>(g, (cudaStream_t)stream)
                .forward(first != 0, (const float*)frame, (const float*)gamma, (const float*)weights,
                         (const float* const*)state_in, (float* const*)state_out, (float*)fu_out, (float*)scratch,
                         true);
        }
    });
}

ff_status ff_diff_frame_backward(int dtype, const ff_diff_geom* geom, int first, const void* frame, const void* gamma,
                                 const void* weights, const void* const* state_in, const void* const* state_out,
                                 const void* tape, const void* const* grad_state_out, const void* grad_fu,
                                 const void* grad_y, long long grad_y_bstride, void* grad_frame, void* grad_gamma,
                                 void* grad_weights, void* const* grad_state_in, void* scratch, void* stream) {
    return ffb::diff::run_frame([&] {
        const ffb::diff::Geo g = ffb::diff::geo_of(geom);
        if (dtype != 0 && dtype != 1) throw std::invalid_argument("dtype must be 0 (float32) or 1 (float64)");
        if (!frame || !gamma || !weights || !state_in || !state_out || !tape || !grad_state_out || !grad_frame ||
            !grad_gamma || !grad_weights || !grad_state_in || !scratch)
            throw std::invalid_argument("null pointer argument");
        for (int k = 0; k < 3 * g.L; ++k)
            if (!::pairs_aligned(dtype, {state_in[k], state_out[k], grad_state_out[k], grad_state_in[k]}))
                throw std::invalid_argument("state fields must be aligned to two elements (8 or 16 bytes)");
        if (!::pairs_aligned(dtype, {grad_y}) || (grad_y && (grad_y_bstride & 1)))
            throw std::invalid_argument("grad_y must be aligned to two elements, with an even image stride");
        if (dtype) {
            ffb::diff::Driver<double>(g, (cudaStream_t)stream)
                .backward(first != 0, (const double*)frame, (const double*)gamma, (const double*)weights,
                          (const double* const*)state_in, (const double* const*)state_out, (const double*)tape,
                          (const double* const*)grad_state_out, (const double*)grad_fu, (const double*)grad_y,
                          grad_y_bstride, (double*)grad_frame,
                          (double*)grad_gamma, (double*)grad_weights, (double* const*)grad_state_in, (double*)scratch);
        } else {
            ffb::diff::Driver<float>(g, (cudaStream_t)stream)
                .backward(first != 0, (const float*)frame, (const float*)gamma, (const float*)weights,
                          (const float* const*)state_in, (const float* const*)state_out, (const float*)tape,
                          (const float* const*)grad_state_out, (const float*)grad_fu, (const float*)grad_y,
                          grad_y_bstride, (float*)grad_frame,
                          (float*)grad_gamma, (float*)grad_weights, (float* const*)grad_state_in, (float*)scratch);
        }
    });
}

}  // extern "C"
