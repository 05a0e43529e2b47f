// Fused per-level kernel: image model + N propagation sub-steps + update + S smoothing
// iterations of one pyramid level in a single pass over HBM.
//
// Mapping.  A warp owns a window of 64 columns (two adjacent pixels per lane, held as
// float2 pairs .x = column c0, .y = column c0+1) and streams down a band of rows.
// Every stage that reads vertical neighbours keeps a small window of its input rows in
// registers (2 rows for a 3-tap upwind step, 4 rows for a 5-tap filter); horizontal
// neighbours come from the adjacent lanes through warp shuffles.  Each stage therefore
// runs a fixed number of rows behind the newest loaded row:
//
//   state row i loaded            (smoothed flow, old image, delta flow of the last frame)
//   X sub-step k  -> row i-k+1,  Y sub-step k -> row i-k          (k = 1..N)
//   image row i-N+2 loaded -> X/Y blur -> a0, ax, ay at row i-N
//   update at row i-N             -> delta / old image / unsmoothed flow stored
//   smoothing s: X at row i-N-2(s-1), Y at row i-N-2s              (s = 1..S)
//   smoothed flow stored at row i-N-2S
//
// The window overlaps its neighbours by HX = 2S + max(N, 2) columns on each side and
// the band starts 2S + max(N, 4-N) rows early, so the halo pixels are recomputed
// rather than exchanged; reads are clamp-to-edge, and at the image edges each stage
// substitutes the edge pixel for missing neighbours exactly as the reference's
// per-stage texture reads do.  Arithmetic is the same operation sequence as the
// per-stage kernels (common.cuh), so results are bit-identical.
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace ffb {
namespace lvl {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarpsPerBlock = 4;

// lane-constant geometry and arguments of one warp
struct Ctx {
    int W, H;
    int c0, c1;            // pixel columns of this lane
    int cc0, cc1;          // clamped load columns
    bool vec;              // pixels adjacent and inside: vector loads/stores
    bool out0, out1;       // pixels stored by this warp
    bool col0, col1;       // pixels outside the propagation border (x in [b, W-b))
    int ix0, ix1;          // coarse-flow columns (delta levels)
    int ys, ye;            // output rows of the band
    int border;
    int first;
    float dt, gamma, maxflow, half_maxflow;
    // X-neighbour sources for the edge path: index into {L.x, L.y, v.x, v.y, R.x, R.y}
    // of the clamped column c+o, per pixel p and offset o in {-2, -1, +1, +2}
    int8_t nb[2][4];
};

__device__ __forceinline__ float pick6(int k, float a, float b, float c, float d, float e, float f) {
    float r = a;
    r = (k == 1) ? b : r;
    r = (k == 2) ? c : r;
    r = (k == 3) ? d : r;
    r = (k == 4) ? e : r;
    r = (k == 5) ? f : r;
    return r;
}

__device__ __forceinline__ float2 shfl_up2(float2 v) {
    return make_float2(__shfl_up_sync(kFull, v.x, 1), __shfl_up_sync(kFull, v.y, 1));
}
__device__ __forceinline__ float2 shfl_dn2(float2 v) {
    return make_float2(__shfl_down_sync(kFull, v.x, 1), __shfl_down_sync(kFull, v.y, 1));
}

// minus/plus neighbours (offset -1/+1) of both pixels of a pair
template <bool EDGE>
__device__ __forceinline__ void nb3(const Ctx& c, float2 v, float2& m, float2& p) {
    const float ly = __shfl_up_sync(kFull, v.y, 1);
    const float rx = __shfl_down_sync(kFull, v.x, 1);
    if (!EDGE) {
        m = make_float2(ly, v.x);
        p = make_float2(v.y, rx);
    } else {
        m = make_float2(pick6(c.nb[0][1], 0.f, ly, v.x, v.y, rx, 0.f), pick6(c.nb[1][1], 0.f, ly, v.x, v.y, rx, 0.f));
        p = make_float2(pick6(c.nb[0][2], 0.f, ly, v.x, v.y, rx, 0.f), pick6(c.nb[1][2], 0.f, ly, v.x, v.y, rx, 0.f));
    }
}

// offsets -2..+2 of both pixels; t[k] holds the pair for offset k-2
template <bool EDGE>
__device__ __forceinline__ void nb5(const Ctx& c, float2 v, float2 (&t)[5]) {
    const float2 L = shfl_up2(v), R = shfl_dn2(v);
    if (!EDGE) {
        t[0] = make_float2(L.x, L.y);
        t[1] = make_float2(L.y, v.x);
        t[2] = v;
        t[3] = make_float2(v.y, R.x);
        t[4] = make_float2(R.x, R.y);
    } else {
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            const int k = o < 2 ? o : o + 1;
            t[k] = make_float2(pick6(c.nb[0][o], L.x, L.y, v.x, v.y, R.x, R.y),
                               pick6(c.nb[1][o], L.x, L.y, v.x, v.y, R.x, R.y));
        }
        t[2] = v;
    }
}

// raw neighbours -2..+2 of an input loaded at clamped columns (no substitution needed:
// a raw image column < 0 already holds column 0's value)
__device__ __forceinline__ void nb5_raw(float2 v, float2 (&t)[5]) {
    const float2 L = shfl_up2(v), R = shfl_dn2(v);
    t[0] = make_float2(L.x, L.y);
    t[1] = make_float2(L.y, v.x);
    t[2] = v;
    t[3] = make_float2(v.y, R.x);
    t[4] = make_float2(R.x, R.y);
}

__device__ __forceinline__ float2 smooth5p(const float2 (&t)[5]) {
    return make_float2(smooth5(t[0].x, t[1].x, t[2].x, t[3].x, t[4].x), smooth5(t[0].y, t[1].y, t[2].y, t[3].y, t[4].y));
}
__device__ __forceinline__ float2 diff5p(const float2 (&t)[5]) {
    return make_float2(diff5(t[0].x, t[1].x, t[2].x, t[3].x, t[4].x), diff5(t[0].y, t[1].y, t[2].y, t[3].y, t[4].y));
}
__device__ __forceinline__ float2 box5p(const float2 (&t)[5]) {
    return make_float2(box5(t[0].x, t[1].x, t[2].x, t[3].x, t[4].x), box5(t[0].y, t[1].y, t[2].y, t[3].y, t[4].y));
}

// upwind step of a pair: n = vel >= 0 ? m : p; d = v - n; v - |t|*d (fused or not).
// Equals the reference's v - t*(vel >= 0 ? v - m : p - v) bit for bit: for vel < 0,
// t = -|t| and p - v = -(v - p) exactly.
template <bool FUSED>
__device__ __forceinline__ float2 upwind2(float2 v, float2 m, float2 p, float2 vel, float2 at) {
    const float d0 = __fsub_rn(v.x, vel.x >= 0.0f ? m.x : p.x);
    const float d1 = __fsub_rn(v.y, vel.y >= 0.0f ? m.y : p.y);
    if (FUSED) return make_float2(__fmaf_rn(-at.x, d0, v.x), __fmaf_rn(-at.y, d1, v.y));
    return make_float2(__fsub_rn(v.x, __fmul_rn(at.x, d0)), __fsub_rn(v.y, __fmul_rn(at.y, d1)));
}

__device__ __forceinline__ float2 abs_t(float dt, float2 vel) {
    return make_float2(fabsf(__fmul_rn(dt, vel.x)), fabsf(__fmul_rn(dt, vel.y)));
}

template <typename T>
__device__ __forceinline__ const T* rowp(const void* base, size_t pitch, int y) {
    return reinterpret_cast<const T*>(reinterpret_cast<const char*>(base) + (size_t)y * pitch);
}
template <typename T>
__device__ __forceinline__ T* rowp_w(void* base, size_t pitch, int y) {
    return reinterpret_cast<T*>(reinterpret_cast<char*>(base) + (size_t)y * pitch);
}

// pair of interleaved float2 pixels (c0, c1) -> (x pair, y pair)
__device__ __forceinline__ void load_f2pair(const Ctx& c, const float* base, size_t pitch, int y, float2& xs,
                                            float2& ysv) {
    const float2* row = rowp<float2>(base, pitch, y);
    if (c.vec) {
        const float4 q = __ldg(reinterpret_cast<const float4*>(row + c.cc0));
        xs = make_float2(q.x, q.z);
        ysv = make_float2(q.y, q.w);
    } else {
        const float2 a = __ldg(row + c.cc0), b = __ldg(row + c.cc1);
        xs = make_float2(a.x, b.x);
        ysv = make_float2(a.y, b.y);
    }
}
__device__ __forceinline__ float2 load_f1pair(const Ctx& c, const float* base, size_t pitch, int y) {
    const float* row = rowp<float>(base, pitch, y);
    if (c.vec) return __ldg(reinterpret_cast<const float2*>(row + c.cc0));
    return make_float2(__ldg(row + c.cc0), __ldg(row + c.cc1));
}
__device__ __forceinline__ void store_f2pair(const Ctx& c, float* base, size_t pitch, int y, float2 xs, float2 ysv) {
    float2* row = rowp_w<float2>(base, pitch, y);
    if (c.out1) {
        *reinterpret_cast<float4*>(row + c.c0) = make_float4(xs.x, ysv.x, xs.y, ysv.y);
    } else if (c.out0) {
        row[c.c0] = make_float2(xs.x, ysv.x);
    }
}
__device__ __forceinline__ void store_f1pair(const Ctx& c, float* base, size_t pitch, int y, float2 v) {
    float* row = rowp_w<float>(base, pitch, y);
    if (c.out1) {
        *reinterpret_cast<float2*>(row + c.c0) = v;
    } else if (c.out0) {
        row[c.c0] = v.x;
    }
}

template <typename P>
__device__ __forceinline__ float2 load_image(const Ctx& c, const void* img, size_t pitch, int y) {
    const P* row = rowp<P>(img, pitch, y);
    return make_float2(Pix<P>::get(__ldg(row + c.cc0)), Pix<P>::get(__ldg(row + c.cc1)));
}

// The pipeline of one warp.  DELTA: delta level (flow, old image and delta flow are
// propagated; the update refines the coarse flow).  Otherwise a top level (flow is
// propagated; old image read in place).
template <bool DELTA, int N, int S, typename P, bool EDGE>
struct Pipe {
    // propagated channels: U, V (flow) [, I old image, DX, DY delta flow]
    static constexpr int NC = DELTA ? 5 : 2;
    static constexpr int CU = 0, CV = 1, CI = 2, CDX = 3, CDY = 4;
    // channels whose upwind step the reference build fuses into one fma: all but the
    // last channel each reference kernel writes (flow .y of flowPropagate{X,Y}_k,
    // vector .y of flowPropagatePayload{X,Y}_k)
    static constexpr bool fused(int ch) { return DELTA ? ch != CDY : ch != CV; }

    float2 pw[N][2][NC];  // Y sub-step windows: rows (q-1, q) of the X sub-step output
    float2 imw[4];        // image rows j-4 .. j-1
    float2 bxw[4];        // X-blurred image rows j-4 .. j-1
    float2 sw[S][4][2];   // smoothing windows: rows q-2 .. q+1 of the X pass, (U, V)

    __device__ __forceinline__ void init() {
#pragma unroll
        for (int k = 0; k < N; ++k)
#pragma unroll
            for (int r = 0; r < 2; ++r)
#pragma unroll
                for (int ch = 0; ch < NC; ++ch) pw[k][r][ch] = make_float2(0.f, 0.f);
#pragma unroll
        for (int r = 0; r < 4; ++r) imw[r] = bxw[r] = make_float2(0.f, 0.f);
#pragma unroll
        for (int s = 0; s < S; ++s)
#pragma unroll
            for (int r = 0; r < 4; ++r) sw[s][r][0] = sw[s][r][1] = make_float2(0.f, 0.f);
    }

    // border freeze (propagation_k.cu:59-65): pixels within `border` of an edge keep v
    __device__ __forceinline__ static void freeze(const Ctx& c, int q, float2 (&out)[NC], const float2 (&v)[NC]) {
        if (!EDGE) return;
        const bool row_ok = q >= c.border && q < c.H - c.border;
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) {
            out[ch].x = (row_ok && c.col0) ? out[ch].x : v[ch].x;
            out[ch].y = (row_ok && c.col1) ? out[ch].y : v[ch].y;
        }
    }

    // X sub-step in place on row q (flowPropagateX_k / flowPropagatePayloadX_k)
    __device__ __forceinline__ static void prop_x(const Ctx& c, int q, float2 (&v)[NC]) {
        float2 m[NC], p[NC];
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) nb3<EDGE>(c, v[ch], m[ch], p[ch]);
        const float2 vel = make_float2(dominant(m[CU].x, p[CU].x), dominant(m[CU].y, p[CU].y));
        const float2 at = abs_t(c.dt, vel);
        float2 o[NC];
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) {
            if (fused(ch)) o[ch] = upwind2<true>(v[ch], m[ch], p[ch], vel, at);
            else o[ch] = upwind2<false>(v[ch], m[ch], p[ch], vel, at);
        }
        freeze(c, q, o, v);
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) v[ch] = o[ch];
    }

    // Y sub-step producing row q from rows q-1 (prev), q (cur), q+1 (next)
    __device__ __forceinline__ static void prop_y(const Ctx& c, int q, const float2 (&prev)[NC],
                                                  const float2 (&cur)[NC], const float2 (&next)[NC],
                                                  float2 (&o)[NC]) {
        const bool top = EDGE && q == 0, bot = EDGE && q == c.H - 1;
        float2 m[NC], p[NC];
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) {
            m[ch] = top ? cur[ch] : prev[ch];
            p[ch] = bot ? cur[ch] : next[ch];
        }
        const float2 vel = make_float2(dominant(m[CV].x, p[CV].x), dominant(m[CV].y, p[CV].y));
        const float2 at = abs_t(c.dt, vel);
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) {
            if (fused(ch)) o[ch] = upwind2<true>(cur[ch], m[ch], p[ch], vel, at);
            else o[ch] = upwind2<false>(cur[ch], m[ch], p[ch], vel, at);
        }
        freeze(c, q, o, cur);
    }

    // one streamed row
    __device__ __forceinline__ void step(const Ctx& c, const LevelArgs& a, int i) {
        const int H = c.H;
        // ---- state row i
        float2 x[NC];
        {
            const int r = min(max(i, 0), H - 1);
            load_f2pair(c, a.fs_in, a.fs_in_pitch, r, x[CU], x[CV]);
            if constexpr (DELTA) {
                x[CI] = load_f1pair(c, a.io_in, a.io_in_pitch, r);
                load_f2pair(c, a.d_in, a.d_in_pitch, r, x[CDX], x[CDY]);
            }
        }
        // ---- N propagation sub-steps
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const int q = i - k;  // row of this X sub-step
            prop_x(c, q, x);
            float2 y[NC];
            prop_y(c, q - 1, pw[k][0], pw[k][1], x, y);
#pragma unroll
            for (int ch = 0; ch < NC; ++ch) {
                pw[k][0][ch] = pw[k][1][ch];
                pw[k][1][ch] = x[ch];
                x[ch] = y[ch];
            }
        }
        const int r = i - N;  // row of the update
        // ---- image model at row r (imagemodel_k.cu:31-133)
        float2 a0, ax, ay;
        {
            const int j = r + 2;
            const float2 im = load_image<P>(c, a.img, a.img_pitch, min(max(j, 0), H - 1));
            float2 t[5];
            nb5_raw(im, t);
            const float2 bx = smooth5p(t);
            float2 by, rows[5] = {imw[0], imw[1], imw[2], imw[3], im};
            by = smooth5p(rows);
            float2 brows[5] = {bxw[0], bxw[1], bxw[2], bxw[3], bx};
            ay = diff5p(brows);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                imw[k] = imw[k + 1];
                bxw[k] = bxw[k + 1];
            }
            imw[3] = im;
            bxw[3] = bx;
            float2 tb[5];
            nb5_raw(by, tb);
            a0 = smooth5p(tb);
            ax = diff5p(tb);
        }
        // ---- update at row r
        float2 fu, fv;
        const bool store_r = r >= c.ys && r < c.ye;
        {
            const int rc = min(max(r, 0), H - 1);
            float2 old;
            if constexpr (DELTA) old = x[CI];
            else old = load_f1pair(c, a.io_in, a.io_in_pitch, rc);
            if (c.first) old = a0;
            float2 fx, fy;
            if constexpr (DELTA) {
                fx = x[CDX];
                fy = x[CDY];
            } else {
                fx = x[CU];
                fy = x[CV];
            }
            float2 ox, oy;
            solve2(c.gamma, ax.x, ay.x, __fsub_rn(old.x, a0.x), fx.x, fy.x, ox.x, oy.x);
            solve2(c.gamma, ax.y, ay.y, __fsub_rn(old.y, a0.y), fx.y, fy.y, ox.y, oy.y);
            if constexpr (DELTA) {
                // deltaFlowUpdate_k (update_k.cu:136-164)
                ox = make_float2(clampm(sanitize(ox.x), c.half_maxflow), clampm(sanitize(ox.y), c.half_maxflow));
                oy = make_float2(clampm(sanitize(oy.x), c.half_maxflow), clampm(sanitize(oy.y), c.half_maxflow));
                const int iy = upmap_index(rc, H, a.Hc);
                const float2* crow = rowp<float2>(a.coarse, a.coarse_pitch, iy);
                const float2 u0 = __ldg(crow + c.ix0), u1 = __ldg(crow + c.ix1);
                fu = make_float2(clampm(__fadd_rn(ox.x, __fmul_rn(2.0f, u0.x)), c.maxflow),
                                 clampm(__fadd_rn(ox.y, __fmul_rn(2.0f, u1.x)), c.maxflow));
                fv = make_float2(clampm(__fadd_rn(oy.x, __fmul_rn(2.0f, u0.y)), c.maxflow),
                                 clampm(__fadd_rn(oy.y, __fmul_rn(2.0f, u1.y)), c.maxflow));
                if (store_r) {
                    store_f2pair(c, a.d_out, a.d_out_pitch, r, ox, oy);
                    store_f1pair(c, a.io_out, a.io_out_pitch, r, a0);
                }
            } else {
                // flowUpdate_k (update_k.cu:65-78)
                fu = make_float2(sanitize(clampm(ox.x, c.maxflow)), sanitize(clampm(ox.y, c.maxflow)));
                fv = make_float2(sanitize(clampm(oy.x, c.maxflow)), sanitize(clampm(oy.y, c.maxflow)));
                if (store_r) {
                    store_f1pair(c, a.io_out, a.io_out_pitch, r, a0);
                    if (a.fu_out) store_f2pair(c, a.fu_out, a.fu_out_pitch, r, fu, fv);
                }
            }
        }
        // ---- S smoothing iterations (flowsmoothing_k.cu:21-87)
#pragma unroll
        for (int s = 0; s < S; ++s) {
            float2 tu[5], tv[5];
            nb5<EDGE>(c, fu, tu);
            nb5<EDGE>(c, fv, tv);
            const float2 sxu = box5p(tu), sxv = box5p(tv);
            const int q = r - 2 * s - 2;  // row of this Y pass
            float2 ru[5] = {sw[s][0][0], sw[s][1][0], sw[s][2][0], sw[s][3][0], sxu};
            float2 rv[5] = {sw[s][0][1], sw[s][1][1], sw[s][2][1], sw[s][3][1], sxv};
            if (EDGE && (q < 2 || q > H - 3)) {
                // clamp-to-edge rows: slot k holds row q-2+k
                float2 cu[5], cv[5];
#pragma unroll
                for (int k = 0; k < 5; ++k) {
                    const int src = min(max(q - 2 + k, 0), H - 1) - (q - 2);
                    cu[k] = ru[0];
                    cv[k] = rv[0];
#pragma unroll
                    for (int m = 1; m < 5; ++m) {
                        cu[k] = src == m ? ru[m] : cu[k];
                        cv[k] = src == m ? rv[m] : cv[k];
                    }
                }
                fu = box5p(cu);
                fv = box5p(cv);
            } else {
                fu = box5p(ru);
                fv = box5p(rv);
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                sw[s][k][0] = sw[s][k + 1][0];
                sw[s][k][1] = sw[s][k + 1][1];
            }
            sw[s][3][0] = sxu;
            sw[s][3][1] = sxv;
        }
        const int rs = r - 2 * S;
        if (rs >= c.ys && rs < c.ye) store_f2pair(c, a.fs_out, a.fs_out_pitch, rs, fu, fv);
    }
};

template <bool DELTA, int N, int S, typename P, bool EDGE>
__device__ __forceinline__ void run_warp(const LevelArgs& a, Ctx& c, int i0, int iters) {
    Pipe<DELTA, N, S, P, EDGE> pipe;
    pipe.init();
    // iters is a multiple of 4: windows of 2 and 4 rows rotate back in place every 4 rows
    for (int it = 0; it < iters; it += 4) {
        pipe.step(c, a, i0 + it);
        pipe.step(c, a, i0 + it + 1);
        pipe.step(c, a, i0 + it + 2);
        pipe.step(c, a, i0 + it + 3);
    }
}

// halo widths of a level: columns on each side (even) and rows before the band
__host__ __device__ constexpr int halo_x(int N, int S) { return ((2 * S + (N > 2 ? N : 2)) + 1) & ~1; }
__host__ __device__ constexpr int lead_rows(int N, int S) { return 2 * S + (N > 4 - N ? N : 4 - N); }

template <bool DELTA, int N, int S, typename P>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) level_k(LevelArgs a, int nwx, int nby, int band) {
    constexpr int HX = halo_x(N, S);
    constexpr int OX = 64 - 2 * HX;
    const int warp = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    if (warp >= nwx * nby) return;  // whole warps exit together
    const int lane = threadIdx.x & 31;
    const int wx = warp % nwx, by = warp / nwx;
    const int W = a.W, H = a.H;

    Ctx c;
    c.W = W;
    c.H = H;
    const int xo = wx * OX, x0 = xo - HX;
    c.c0 = x0 + 2 * lane;
    c.c1 = c.c0 + 1;
    c.cc0 = min(max(c.c0, 0), W - 1);
    c.cc1 = min(max(c.c1, 0), W - 1);
    c.vec = c.cc1 == c.cc0 + 1;
    const int xe = min(xo + OX, W);
    c.out0 = c.c0 >= xo && c.c0 < xe;
    c.out1 = c.c1 >= xo && c.c1 < xe;
    c.border = a.border;
    c.col0 = c.c0 >= a.border && c.c0 < W - a.border;
    c.col1 = c.c1 >= a.border && c.c1 < W - a.border;
    c.ys = by * band;
    c.ye = min(c.ys + band, H);
    c.first = a.first;
    c.dt = 1.0f / (float)N;  // FlowPropagator::setIterations (propagation.cu:146-147)
    c.gamma = a.gamma;
    c.maxflow = a.maxflow;
    c.half_maxflow = __fmul_rn(0.5f, a.maxflow);
    if (DELTA) {
        c.ix0 = upmap_index(c.cc0, W, a.Wc);
        c.ix1 = upmap_index(c.cc1, W, a.Wc);
    } else {
        c.ix0 = c.ix1 = 0;
    }
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        const int cp = p == 0 ? c.c0 : c.c1;
        const int offs[4] = {-2, -1, 1, 2};
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            const int src = min(max(cp + offs[o], 0), W - 1) - (c.c0 - 2);
            c.nb[p][o] = (int8_t)min(max(src, 0), 5);
        }
    }
    const int i0 = c.ys - lead_rows(N, S);
    const int last = c.ye - 1 + N + 2 * S;
    const int iters = (last - i0 + 1 + 3) & ~3;
    // interior warps: no clamping, substitution or border freeze can reach them
    const int m = (a.border > 2 ? a.border : 2) + 1;
    const int rlo = i0 - N - 2 * S - 2, rhi = i0 + iters + 2;
    const bool interior = x0 >= m && x0 + 64 <= W - m && rlo >= m && rhi <= H - m;
    if (interior) run_warp<DELTA, N, S, P, false>(a, c, i0, iters);
    else run_warp<DELTA, N, S, P, true>(a, c, i0, iters);
}

template <bool DELTA, int N, int S, typename P>
cudaError_t launch(const LevelArgs& a, cudaStream_t s) {
    constexpr int HX = halo_x(N, S);
    constexpr int OX = 64 - 2 * HX;
    const int nwx = (a.W + OX - 1) / OX;
    // bands sized for about 8 resident warps per SM across 148 SMs
    int band = a.band > 0 ? a.band : (int)(((long)a.H * nwx + 1183) / 1184);
    band = band < 8 ? 8 : band;
    band = band > a.H ? a.H : band;
    const int nby = (a.H + band - 1) / band;
    const int warps = nwx * nby;
    const int blocks = (warps + kWarpsPerBlock - 1) / kWarpsPerBlock;
    level_k<DELTA, N, S, P><<<blocks, kWarpsPerBlock * 32, 0, s>>>(a, nwx, nby, band);
    return cudaGetLastError();
}

}  // namespace lvl
}  // namespace ffb
