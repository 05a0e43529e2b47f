// Device side of the tile-fused level step (tile_level.cu, batch.cu): one CTA computes one
// output tile of a pyramid level for one frame.
//
// The CTA loads the previous frame's state (smoothed flow, old image and delta flow for
// delta levels) over the tile plus a halo of R = N + 2S pixels into shared memory, and
// then runs every stage of the level there, each stage over a region one stencil radius
// smaller than the one before:
//
//   N x (upwind X sub-step, upwind Y sub-step)    radius R     -> 2S   (one pass per pair, A <-> B)
//   image model of the new frame                  radius 2S + 2 -> 2S  (in the spare buffer)
//   update (2x2 solve, clamps, coarse upsample)   radius 2S            (in place)
//   S x (5-tap box X, 5-tap box Y)                radius 2S    -> 0    (ping-pong, last pass to HBM)
//
// Reads outside the image are clamped to the edge, as the reference's textures do
// (cudaAddressModeClamp), so a region that touches the image border simply stops there.
// Every stage is spread over all threads of the CTA (up to 512) with one barrier between
// stages: the work of a small level is bound neither by the serial row recurrence of the
// streaming kernel nor by per-stage launch latency.
//
// The arithmetic is the per-stage kernels' (stage_kernels.cu) operation for operation, so
// the results are bit-identical to them and to the reference.
#pragma once

#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "kernels.h"
#include "launch.cuh"

namespace ffb {
namespace tile {

struct Geom {
    int TW, TH;    // output tile
    int N, S, R;   // propagation sub-steps, smoothing iterations, state halo N + 2S
    int SW, SH;    // state region (TW + 2R) x (TH + 2R)
    int tiles_x;
    int offB;      // byte offset of buffer B
    int offC;      // byte offset of the coarse column table (delta levels)
};

// Shared-memory bytes of one tile.  Buffers A and B each hold the state fields over the
// state region: float2 flow, then for delta levels float2 delta and float old image.  The
// buffer that does not hold the propagated state hosts the image model (the image, its Y
// blur and its X blur) between the propagation and the update.
struct Layout {
    size_t a, b, c, total;
};
inline Layout layout(bool delta, int N, int S, int tw, int th) {
    const size_t R = (size_t)N + 2 * (size_t)S;
    const size_t ns = ((size_t)tw + 2 * R) * ((size_t)th + 2 * R);
    const size_t fb = delta ? 20 : 8;
    const size_t rI = 2 * (size_t)S + 2;
    const size_t iw = tw + 2 * rI, ih = th + 2 * rI;
    const size_t model = (iw * ih + (th + 4 * (size_t)S) * iw + ih * (tw + 4 * (size_t)S)) * 4;
    Layout L;
    // the propagated state ends in A or in B (one swap per sub-step pair), and the image
    // model then lives in the other buffer: both are sized for either use
    L.a = (std::max(ns * fb, model) + 15) / 16 * 16;
    L.b = L.a;
    L.c = delta ? ((size_t)tw + 4 * (size_t)S) * 4 : 0;
    L.total = L.a + L.b + L.c;
    return L;
}

template <typename T>
__device__ __forceinline__ void swap2(T& a, T& b) {
    T t = a;
    a = b;
    b = t;
}

template <typename T>
__device__ __forceinline__ const T* grow(const void* base, size_t pitch, int y) {
    return reinterpret_cast<const T*>(reinterpret_cast<const char*>(base) + (size_t)y * pitch);
}
template <typename T>
__device__ __forceinline__ T* growm(void* base, size_t pitch, int y) {
    return reinterpret_cast<T*>(reinterpret_cast<char*>(base) + (size_t)y * pitch);
}

// Visits every pixel of [xa, xb) x [ya, yb): lane l of each warp takes the columns
// xa + l, xa + l + 32, ..., warp w the rows ya + w, ya + w + nw, ...  k is the pixel's index
// in an array of row stride `stride` whose (xa, ya) element is k0.  load(x, y, k) reads a
// pixel's inputs and done(x, y, k, in) computes and stores; two rows are visited per
// iteration with both loads issued before either store, so their latencies overlap.
// Every loop bound is uniform across the warp: in the last column chunk the lanes past
// xb repeat column xb - 1, computing and storing the same value as the lane that owns it,
// so no lane diverges.
template <typename Load, typename Done>
__device__ __forceinline__ void walk(int xa, int xb, int ya, int yb, int stride, int k0, Load&& load, Done&& done) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int dk = nw * stride;
    for (int cx = xa; cx < xb; cx += 32) {
        const int x = min(cx + lane, xb - 1);
        int y = ya + w;
        int k = k0 + (x - xa) + w * stride;
        for (; y + nw < yb; y += 2 * nw, k += 2 * dk) {
            const auto p = load(x, y, k);
            const auto q = load(x, y + nw, k + dk);
            done(x, y, k, p);
            done(x, y + nw, k + dk, q);
        }
        if (y < yb) {
            const auto p = load(x, y, k);
            done(x, y, k, p);
        }
    }
}

struct PropIn {
    float2 fm, f0, fp;
    float sm, s0, sp;
    float2 vm, v0, vp;
};

template <bool DELTA>
__device__ __forceinline__ PropIn prop_load(const float2* fs, const float2* ds, const float* is, int k, int km,
                                            int kp) {
    PropIn p;
    p.fm = fs[km];
    p.f0 = fs[k];
    p.fp = fs[kp];
    if constexpr (DELTA) {
        p.sm = is[km];
        p.s0 = is[k];
        p.sp = is[kp];
        p.vm = ds[km];
        p.v0 = ds[k];
        p.vp = ds[kp];
    }
    return p;
}

// the state fields of one pixel
struct PropOut {
    float2 f;
    float s;
    float2 v;
};

// One upwind sub-step at one pixel: propagate_pass_k<AXIS, DELTA> (stage_kernels.cu).
template <int AXIS, bool DELTA>
__device__ __forceinline__ PropOut prop_eval(const PropIn& p, float dt, bool in) {
    const float dv = AXIS == 0 ? dominant(p.fm.x, p.fp.x) : dominant(p.fm.y, p.fp.y);
    const float t = __fmul_rn(dt, dv);
    PropOut o;
    if constexpr (DELTA) {
        o.f = in ? upwind_pair(t, dv, p.fm, p.f0, p.fp) : p.f0;
    } else {
        o.f.x = in ? upwind(t, dv, p.fm.x, p.f0.x, p.fp.x) : p.f0.x;
        o.f.y = in ? upwind_unfused(t, dv, p.fm.y, p.f0.y, p.fp.y) : p.f0.y;
    }
    if constexpr (DELTA) {
        o.s = in ? upwind(t, dv, p.sm, p.s0, p.sp) : p.s0;
        o.v.x = in ? upwind(t, dv, p.vm.x, p.v0.x, p.vp.x) : p.v0.x;
        o.v.y = in ? upwind_unfused(t, dv, p.vm.y, p.v0.y, p.vp.y) : p.v0.y;
    }
    return o;
}

struct Five {
    float2 v0, v1, v2, v3, v4;
};
__device__ __forceinline__ float2 box5_2(const Five& f) { return box5_pair(f.v0, f.v1, f.v2, f.v3, f.v4); }

// One CTA's work: output tile `tile` (row-major over the tile grid) of the level step
// described by (a, g), in the dynamic shared memory `sm`.
template <bool DELTA, typename P>
__device__ __forceinline__ void tile_body(const LevelArgs& a, const Geom& g, int tile, unsigned char* sm) {
    // Ordering with the preceding kernel (PDL): by default wait for it before anything.  With
    // pdl_late_wait (a delta level launched right after its top level) the state load,
    // propagation and image model read only the previous frame's state and an image that
    // was complete before the preceding kernel passed its own wait, so the wait moves to
    // just before the update, the first stage that reads the coarse flow.
    const bool late_wait = a.pdl_late_wait != 0;
    if (!late_wait) grid_dep_wait();
    if (a.pdl_early_trigger) grid_dep_launch();
    const int W = a.W, H = a.H;
    const int tx = tile % g.tiles_x, ty = tile / g.tiles_x;
    const int x0 = tx * g.TW, y0 = ty * g.TH;
    const int x1 = min(x0 + g.TW, W), y1 = min(y0 + g.TH, H);
    const int ox = x0 - g.R, oy = y0 - g.R;  // state region origin (may lie outside the image)
    const int SW = g.SW, NS = g.SW * g.SH;
    const int B = a.border;
    // kernel parameters used per pixel, held in registers
    const float2* __restrict__ fs_in = reinterpret_cast<const float2*>(a.fs_in);
    const float2* __restrict__ d_in = reinterpret_cast<const float2*>(a.d_in);
    const float* __restrict__ io_in = a.io_in;
    const size_t fs_in_p = a.fs_in_pitch, d_in_p = a.d_in_pitch, io_in_p = a.io_in_pitch;
    const P* __restrict__ img_in = reinterpret_cast<const P*>(a.img);
    const size_t img_p = a.img_pitch;
    const float2* __restrict__ coarse = reinterpret_cast<const float2*>(a.coarse);
    const size_t coarse_p = a.coarse_pitch;
    const int* __restrict__ coarse_rows = a.coarse_rows;
    float* const d_out = a.d_out;
    float* const io_out = a.io_out;
    float* const fu_out = a.fu_out;
    float* const fs_out = a.fs_out;
    const size_t d_out_p = a.d_out_pitch, io_out_p = a.io_out_pitch, fu_out_p = a.fu_out_pitch,
                 fs_out_p = a.fs_out_pitch;
    const bool first = a.first != 0;

    float2* fA = reinterpret_cast<float2*>(sm);
    float2* fB = reinterpret_cast<float2*>(sm + g.offB);
    float2* dA = fA + NS;  // delta levels only
    float2* dB = fB + NS;
    float* iA = reinterpret_cast<float*>(dA + NS);
    float* iB = reinterpret_cast<float*>(dB + NS);

    auto sidx = [&](int x, int y) { return (y - oy) * SW + (x - ox); };
    // region of radius r around the output tile, clipped to the image
    auto xa = [&](int r) { return max(x0 - r, 0); };
    auto xb = [&](int r) { return min(x1 + r, W); };
    auto ya = [&](int r) { return max(y0 - r, 0); };
    auto yb = [&](int r) { return min(y1 + r, H); };
    auto row_in = [&](int y) { return y >= B && y < H - B; };
    auto col_in = [&](int x) { return x >= B && x < W - B; };

    // ---- previous frame's state over radius R
    {
        struct In {
            float2 f, d;
            float i;
        };
        walk(
            xa(g.R), xb(g.R), ya(g.R), yb(g.R), SW, sidx(xa(g.R), ya(g.R)),
            [&](int x, int y, int) {
                In v;
                v.f = __ldg(grow<float2>(fs_in, fs_in_p, y) + x);
                if constexpr (DELTA) {
                    v.d = __ldg(grow<float2>(d_in, d_in_p, y) + x);
                    v.i = __ldg(grow<float>(io_in, io_in_p, y) + x);
                }
                return v;
            },
            [&](int, int, int k, const In& v) {
                fA[k] = v.f;
                if constexpr (DELTA) {
                    dA[k] = v.d;
                    iA[k] = v.i;
                }
            });
    }
    __syncthreads();

    // ---- propagation: N x (X, Y) sub-steps, dt = 1/N (propagation.cu:146-147).  Each X/Y
    // pair is one pass: a warp takes a 32-column chunk and a band of rows, computes the X
    // sub-step for rows y-1, y, y+1 into a rolling register window and the Y sub-step from
    // it, so the X result never goes through shared memory (one barrier per pair).
    const float dt = 1.0f / (float)g.N;
    float2 *fs = fA, *fd = fB, *ds = dA, *dd = dB;
    float *is = iA, *id = iB;
    // A tile whose whole state region lies inside the propagation border (x, y in [B, size-B))
    // has no frozen pixel: its sub-steps skip the border test and its selects.
    const bool interior = x0 - g.R >= B && x1 + g.R <= W - B && y0 - g.R >= B && y1 + g.R <= H - B;
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        for (int j = 1; j <= g.N; ++j) {
            const int r = g.R - j;  // output radius of this pair; its X sub-step reads radius r + 1
            const int cxa = xa(r), cxb = xb(r), rya = ya(r), ryb = yb(r);
            const int nc = (cxb - cxa + 31) >> 5;
            const int nb = max(1, nw / nc);
            const int K = (ryb - rya + nb - 1) / nb;
            for (int item = warp; item < nc * nb; item += nw) {
                const int band = item / nc, c = item - band * nc;
                const int x = min(cxa + c * 32 + lane, cxb - 1);  // spare lanes repeat the last column
                const int by0 = rya + band * K, by1 = min(by0 + K, ryb);
                if (by0 >= by1) continue;
                const int kc = x - ox;
                const int dxm = x > 0 ? 1 : 0, dxp = x < W - 1 ? 1 : 0;
                const bool cin = col_in(x);
                // one band of rows: X sub-step into a rolling window of rows y-1, y, y+1, then
                // the Y sub-step from it; FREE = no pixel of the tile is frozen at the border
                auto band_pass = [&](auto free_tag) {
                    constexpr bool FREE = decltype(free_tag)::value;
                    auto xstep = [&](int row) {
                        const int k = (row - oy) * SW + kc;
                        // a free tile lies inside the border, so its X neighbours are never clamped:
                        // constant offsets let the loads share one address
                        const PropIn p = FREE ? prop_load<DELTA>(fs, ds, is, k, k - 1, k + 1)
                                              : prop_load<DELTA>(fs, ds, is, k, k - dxm, k + dxp);
                        return FREE ? prop_eval<0, DELTA>(p, dt, true) : prop_eval<0, DELTA>(p, dt, cin && row_in(row));
                    };
                    PropOut cur = xstep(by0);
                    PropOut prev = by0 > 0 ? xstep(by0 - 1) : cur;  // row -1 clamps to row 0
                    for (int y = by0; y < by1; ++y) {
                        const PropOut nxt = y + 1 < H ? xstep(y + 1) : cur;  // row H clamps to H - 1
                        PropIn q;
                        q.fm = prev.f;
                        q.f0 = cur.f;
                        q.fp = nxt.f;
                        if constexpr (DELTA) {
                            q.sm = prev.s;
                            q.s0 = cur.s;
                            q.sp = nxt.s;
                            q.vm = prev.v;
                            q.v0 = cur.v;
                            q.vp = nxt.v;
                        }
                        const PropOut o =
                            FREE ? prop_eval<1, DELTA>(q, dt, true) : prop_eval<1, DELTA>(q, dt, cin && row_in(y));
                        const int k = (y - oy) * SW + kc;
                        fd[k] = o.f;
                        if constexpr (DELTA) {
                            id[k] = o.s;
                            dd[k] = o.v;
                        }
                        prev = cur;
                        cur = nxt;
                    }
                };
                if (interior) band_pass(std::true_type{});
                else band_pass(std::false_type{});
            }
            __syncthreads();
            swap2(fs, fd);
            swap2(ds, dd);
            swap2(is, id);
        }
    }
    // the propagated state is in fs/is/ds (buffer A for even N, B for odd N); the image model
    // goes to the other buffer
    unsigned char* const spare = reinterpret_cast<unsigned char*>(fd);

    // ---- image model of the new frame (imagemodel_k.cu:31-133) over radius 2S, in B
    const int S2 = 2 * g.S, rI = S2 + 2;
    const int IW = g.TW + 2 * rI, BXW = g.TW + 2 * S2;
    const int IH = g.TH + 2 * rI;
    float* img = reinterpret_cast<float*>(spare);        // origin (x0 - rI, y0 - rI), IW x IH
    float* byv = img + IW * IH;                          // Y blur, origin (x0 - rI, y0 - 2S), IW wide
    float* bxv = byv + (g.TH + 2 * S2) * IW;             // X blur, origin (x0 - 2S, y0 - rI), BXW wide
    int* ccol = reinterpret_cast<int*>(sm + g.offC);     // coarse column of each column, origin x0 - 2S
    auto iidx = [&](int x, int y) { return (y - y0 + rI) * IW + (x - x0 + rI); };
    if (a.pyr_src) {
        // fused pyramid step: this level's image from the finer one (pyramid_down_k)
        const CView<P> fine{reinterpret_cast<const P*>(a.pyr_src), a.pyr_src_pitch, a.pyr_src_H, a.pyr_src_W};
        walk(
            xa(rI), xb(rI), ya(rI), yb(rI), IW, iidx(xa(rI), ya(rI)),
            [&](int x, int y, int) { return pyramid_val(fine, x, y); },
            [&](int x, int y, int k, P v) {
                img[k] = Pix<P>::get(v);
                if (x >= x0 && x < x1 && y >= y0 && y < y1) growm<P>(const_cast<void*>(a.img), img_p, y)[x] = v;
            });
    } else {
        walk(
            xa(rI), xb(rI), ya(rI), yb(rI), IW, iidx(xa(rI), ya(rI)),
            [&](int x, int y, int) { return __ldg(grow<P>(img_in, img_p, y) + x); },
            [&](int, int, int k, P v) { img[k] = Pix<P>::get(v); });
    }
    if constexpr (DELTA) {
        for (int x = xa(S2) + (int)threadIdx.x; x < xb(S2); x += blockDim.x) ccol[x - x0 + S2] = upmap_index(x, W, a.Wc);
    }
    __syncthreads();
    {
        struct Col5 {
            float v0, v1, v2, v3, v4;
        };
        // Y blur at (x, y): rows y-2..y+2 clamped to the image
        walk(
            xa(rI), xb(rI), ya(S2), yb(S2), IW, (ya(S2) - y0 + S2) * IW + (xa(rI) - x0 + rI),
            [&](int x, int y, int) {
                const int ki = iidx(x, y);
                Col5 c;
                c.v0 = img[ki - min(y, 2) * IW];
                c.v1 = img[ki - min(y, 1) * IW];
                c.v2 = img[ki];
                c.v3 = img[ki + min(H - 1 - y, 1) * IW];
                c.v4 = img[ki + min(H - 1 - y, 2) * IW];
                return c;
            },
            [&](int, int, int k, const Col5& c) { byv[k] = smooth5(c.v0, c.v1, c.v2, c.v3, c.v4); });
        // X blur at (x, y): columns x-2..x+2 clamped to the image
        walk(
            xa(S2), xb(S2), ya(rI), yb(rI), BXW, (ya(rI) - y0 + rI) * BXW + (xa(S2) - x0 + S2),
            [&](int x, int y, int) {
                const int ki = iidx(x, y);
                Col5 c;
                c.v0 = img[ki - min(x, 2)];
                c.v1 = img[ki - min(x, 1)];
                c.v2 = img[ki];
                c.v3 = img[ki + min(W - 1 - x, 1)];
                c.v4 = img[ki + min(W - 1 - x, 2)];
                return c;
            },
            [&](int, int, int k, const Col5& c) { bxv[k] = smooth5(c.v0, c.v1, c.v2, c.v3, c.v4); });
    }
    __syncthreads();

    if (late_wait) grid_dep_wait();

    // ---- update over radius 2S: the new flow goes to the propagated flow field in place
    {
        const float gamma = a.gamma, maxflow = a.maxflow;
        struct UpdIn {
            float b0, b1, b2, b3, b4, c0, c1, c2, c3, c4;
            float old;
            float2 f;  // propagated delta (delta levels) or propagated flow (top levels)
            float2 up;
        };
        walk(
            xa(S2), xb(S2), ya(S2), yb(S2), SW, sidx(xa(S2), ya(S2)),
            [&](int x, int y, int k) {
                UpdIn u;
                const int kb = (y - y0 + S2) * IW + (x - x0 + rI);
                u.b0 = byv[kb - min(x, 2)];
                u.b1 = byv[kb - min(x, 1)];
                u.b2 = byv[kb];
                u.b3 = byv[kb + min(W - 1 - x, 1)];
                u.b4 = byv[kb + min(W - 1 - x, 2)];
                const int kx = (y - y0 + rI) * BXW + (x - x0 + S2);
                u.c0 = bxv[kx - min(y, 2) * BXW];
                u.c1 = bxv[kx - min(y, 1) * BXW];
                u.c2 = bxv[kx];
                u.c3 = bxv[kx + min(H - 1 - y, 1) * BXW];
                u.c4 = bxv[kx + min(H - 1 - y, 2) * BXW];
                if constexpr (DELTA) {
                    u.old = is[k];
                    u.f = ds[k];
                    const int cr = __ldg(coarse_rows + y);
                    u.up = __ldg(grow<float2>(coarse, coarse_p, cr) + ccol[x - x0 + S2]);
                } else {
                    u.old = __ldg(grow<float>(io_in, io_in_p, y) + x);
                    u.f = fs[k];
                }
                return u;
            },
            [&](int x, int y, int k, const UpdIn& u) {
                const float c = smooth5(u.b0, u.b1, u.b2, u.b3, u.b4);
                const float ax = diff5(u.b0, u.b1, u.b2, u.b3, u.b4);
                const float ay = diff5(u.c0, u.c1, u.c2, u.c3, u.c4);
                const float old = first ? c : u.old;
                const bool out = x >= x0 && x < x1 && y >= y0 && y < y1;
                float fx, fy;
                solve2(gamma, ax, ay, __fsub_rn(old, c), u.f.x, u.f.y, fx, fy);
                if constexpr (DELTA) {
                    // deltaFlowUpdate_k (update_k.cu:82-173)
                    const float hm = __fmul_rn(0.5f, maxflow);
                    const float dx = clampm(sanitize(fx), hm);
                    const float dy = clampm(sanitize(fy), hm);
                    const float gx = __fadd_rn(dx, __fmul_rn(2.0f, u.up.x));
                    const float gy = __fadd_rn(dy, __fmul_rn(2.0f, u.up.y));
                    fs[k] = make_float2(clampm(gx, maxflow), clampm(gy, maxflow));
                    if (out) {
                        growm<float2>(d_out, d_out_p, y)[x] = make_float2(dx, dy);
                        growm<float>(io_out, io_out_p, y)[x] = c;
                    }
                } else {
                    // flowUpdate_k (update_k.cu:15-79); the old image is the previous frame's a0
                    const float2 o = make_float2(sanitize(clampm(fx, maxflow)), sanitize(clampm(fy, maxflow)));
                    fs[k] = o;
                    if (out) {
                        if (fu_out) growm<float2>(fu_out, fu_out_p, y)[x] = o;
                        growm<float>(io_out, io_out_p, y)[x] = c;
                    }
                }
            });
    }
    __syncthreads();

    // ---- smoothing: S x (box X, box Y) (flowsmoothing_k.cu:21-87); the last pass writes HBM
    for (int s = 1; s <= g.S; ++s) {
        const int r = 2 * (g.S - s);
        walk(
            xa(r), xb(r), ya(r + 2), yb(r + 2), SW, sidx(xa(r), ya(r + 2)),
            [&](int x, int, int k) {
                Five f;
                f.v0 = fs[k - min(x, 2)];
                f.v1 = fs[k - min(x, 1)];
                f.v2 = fs[k];
                f.v3 = fs[k + min(W - 1 - x, 1)];
                f.v4 = fs[k + min(W - 1 - x, 2)];
                return f;
            },
            [&](int, int, int k, const Five& f) { fd[k] = box5_2(f); });
        __syncthreads();
        const bool last = s == g.S;
        // the next kernel in the stream may start scheduling its blocks from here on
        if (last && !a.pdl_early_trigger) grid_dep_launch();
        walk(
            xa(r), xb(r), ya(r), yb(r), SW, sidx(xa(r), ya(r)),
            [&](int, int y, int k) {
                Five f;
                f.v0 = fd[k - min(y, 2) * SW];
                f.v1 = fd[k - min(y, 1) * SW];
                f.v2 = fd[k];
                f.v3 = fd[k + min(H - 1 - y, 1) * SW];
                f.v4 = fd[k + min(H - 1 - y, 2) * SW];
                return f;
            },
            [&](int x, int y, int k, const Five& f) {
                const float2 o = box5_2(f);
                if (last) growm<float2>(fs_out, fs_out_p, y)[x] = o;
                else fs[k] = o;
            });
        if (!last) __syncthreads();
    }
}

}  // namespace tile
}  // namespace ffb
