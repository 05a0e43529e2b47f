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

#include <atomic>

#include "common.cuh"
#include "kernels.h"
#include "launch.cuh"

namespace ffb {
namespace lvl {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarpsPerBlock = 4;
#ifndef FFB_ROW_UNROLL
#define FFB_ROW_UNROLL 1  // rows per loop body (2: the propagation windows rotate without moves, twice the code)
#endif
#ifndef FFB_BLOCKS_PER_SM
#define FFB_BLOCKS_PER_SM 2
#endif
constexpr int kBlocksPerSM = FFB_BLOCKS_PER_SM;  // resident blocks per SM the register budget targets
#ifndef FFB_PIPE_DELAY
#define FFB_PIPE_DELAY 0
#endif
// rows the update and smoothing of a step run behind its propagation (1: the update chain of
// the previous row runs beside the propagation chain of this one)
constexpr int kDelay = FFB_PIPE_DELAY;

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
    // edge lanes (clamp-to-edge substitution of horizontal neighbours):
    // e_l: c0 == 0; e_r1: c1 == W-1; e_r0: c0 == W-1 (odd W); e_r2: c1 == W-2 (odd W)
    bool e_l, e_r1, e_r0, e_r2;
    bool freeze_cols;      // some lane of this warp lies within the propagation border
    bool any_edge;         // some lane of this warp needs horizontal edge substitution
    bool any_split;        // some lane's two pixels are not the loaded pair (b0, b0+1)
    int b0;                // even base column of the lane's loaded pair
    unsigned o8, o16;      // this warp's shared memory (lvl_smem offset) + 8 / 16 bytes per lane
    unsigned smem_s;       // this warp's shared memory as a shared-state-space address
    int lane;
};

__device__ __forceinline__ float2 shfl_up2(float2 v) {
    return make_float2(__shfl_up_sync(kFull, v.x, 1), __shfl_up_sync(kFull, v.y, 1));
}
__device__ __forceinline__ float2 shfl_dn2(float2 v) {
    return make_float2(__shfl_down_sync(kFull, v.x, 1), __shfl_down_sync(kFull, v.y, 1));
}

// minus/plus neighbours (offset -1/+1) of both pixels of a pair.  At the image edges
// the missing neighbour is the edge pixel itself (clamp-to-edge reads of this stage's
// input): only the lanes holding columns 0, W-1 substitute.
template <bool EDGE>
__device__ __forceinline__ void nb3(const Ctx& c, float2 v, float2& m, float2& p) {
    const float ly = __shfl_up_sync(kFull, v.y, 1);
    const float rx = __shfl_down_sync(kFull, v.x, 1);
    m = make_float2(ly, v.x);
    p = make_float2(v.y, rx);
    if (EDGE && c.any_edge) {  // warp-uniform
        m.x = c.e_l ? v.x : m.x;
        p.x = c.e_r0 ? v.x : p.x;
        p.y = c.e_r1 ? v.y : p.y;
    }
}

// offsets -2..+2 of both pixels; t[k] holds the pair for offset k-2
template <bool EDGE>
__device__ __forceinline__ void nb5(const Ctx& c, float2 v, float2 (&t)[5]) {
    const float2 L = shfl_up2(v), R = shfl_dn2(v);
    t[0] = make_float2(L.x, L.y);
    t[1] = make_float2(L.y, v.x);
    t[2] = v;
    t[3] = make_float2(v.y, R.x);
    t[4] = make_float2(R.x, R.y);
    if (EDGE && c.any_edge) {  // warp-uniform
        // left edge: columns -2, -1 read column 0
        t[0].x = c.e_l ? v.x : t[0].x;
        t[1].x = c.e_l ? v.x : t[1].x;
        t[0].y = c.e_l ? v.x : t[0].y;
        // right edge, even W: columns W, W+1 read column W-1 = v.y of the last lane
        t[4].x = c.e_r1 ? v.y : t[4].x;
        t[3].y = c.e_r1 ? v.y : t[3].y;
        t[4].y = c.e_r1 ? v.y : t[4].y;
        // right edge, odd W: the last lane holds column W-1 in v.x
        t[3].x = c.e_r0 ? v.x : t[3].x;
        t[4].x = c.e_r0 ? v.x : t[4].x;
        // odd W, lane before the last: column W reads column W-1 = R.x
        t[4].y = c.e_r2 ? R.x : t[4].y;
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

// the pixel pair's 5-tap chains as packed two-lane instructions (lane = pixel)
__device__ __forceinline__ float2 smooth5p(const float2 (&t)[5]) { return smooth5_pair(t[0], t[1], t[2], t[3], t[4]); }
__device__ __forceinline__ float2 diff5p(const float2 (&t)[5]) { return diff5_pair(t[0], t[1], t[2], t[3], t[4]); }
__device__ __forceinline__ float2 box5p(const float2 (&t)[5]) { return box5_pair(t[0], t[1], t[2], t[3], t[4]); }

// upwind step of a pair: n = vel >= 0 ? m : p; d = v - n; v - |t|*d (fused or not).
// Equals the reference's v - t*(vel >= 0 ? v - m : p - v) bit for bit: for vel < 0,
// t = -|t| and p - v = -(v - p) exactly.
// fw = (vel >= 0) per pixel, at = |t| per pixel
// (packed two-lane instructions, lane = pixel; each lane the scalar operation)
#ifndef FFB_PACKED_UPWIND
#define FFB_PACKED_UPWIND 1
#endif
template <bool FUSED>
__device__ __forceinline__ float2 upwind2(float2 v, float2 m, float2 p, bool fw0, bool fw1, float2 at) {
    const float2 n = make_float2(fw0 ? m.x : p.x, fw1 ? m.y : p.y);
#if FFB_PACKED_UPWIND
    const float2 d = __fadd2_rn(v, make_float2(-n.x, -n.y));
    if (FUSED) return __ffma2_rn(make_float2(-at.x, -at.y), d, v);
    const float2 q = __fmul2_rn(at, d);
    return __fadd2_rn(v, make_float2(-q.x, -q.y));
#else
    const float dx = __fsub_rn(v.x, n.x), dy = __fsub_rn(v.y, n.y);
    if (FUSED) return make_float2(__fmaf_rn(-at.x, dx, v.x), __fmaf_rn(-at.y, dy, v.y));
    return make_float2(__fsub_rn(v.x, __fmul_rn(at.x, dx)), __fsub_rn(v.y, __fmul_rn(at.y, dy)));
#endif
}

__device__ __forceinline__ float2 abs_t(float dt, float2 vel) {
    return make_float2(fabsf(__fmul_rn(dt, vel.x)), fabsf(__fmul_rn(dt, vel.y)));
}

// row y >= 0 of a pitched image; pitches are below 2^32 bytes, so the offset is one
// 32 x 32 -> 64-bit multiply
template <typename T>
__device__ __forceinline__ const T* rowp(const void* base, size_t pitch, int y) {
    return reinterpret_cast<const T*>(reinterpret_cast<const char*>(base) +
                                      (unsigned long long)(unsigned)y * (unsigned)pitch);
}
template <typename T>
__device__ __forceinline__ T* rowp_w(void* base, size_t pitch, int y) {
    return reinterpret_cast<T*>(reinterpret_cast<char*>(base) + (unsigned long long)(unsigned)y * (unsigned)pitch);
}

// ---------------------------------------------------------------- cp.async staging
// Every input row a stage needs is copied into a per-warp shared-memory ring kDepth
// rows ahead of its use (cp.async: the data is in flight without occupying registers).
// Each lane copies and later reads only its own bytes, so no warp barrier is needed.
constexpr int kDepth = 4;
struct Slot {
    static constexpr int FLOW = 0;      // 32 lanes x 16 B: (u0, v0, u1, v1) of the state row
    static constexpr int IO = 512;      // 32 x 8 B: old image (delta: state row; top: update row)
    static constexpr int IMG = 768;     // 32 x 8 B: image row (uint8 words or float pair)
    static constexpr int DELTA = 1024;  // 32 x 16 B: delta flow of the state row
    static constexpr int COARSE = 1536; // 32 x 16 B: coarse flow at the update row
    static constexpr int TOP_BYTES = 1024, DELTA_BYTES = 2048;
};

// dst: a shared-memory address (state space .shared, 32 bits)
__device__ __forceinline__ void cp16(unsigned dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp8(unsigned dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp4(unsigned dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// pair of interleaved float2 pixels (c0, c1) -> (x pair, y pair).  EX: a lane may store
// c0 alone (odd right edge); otherwise both pixels of a lane are stored or neither
template <bool EX>
__device__ __forceinline__ void store_f2pair(const Ctx& c, float* base, size_t pitch, int y, float2 xs, float2 ysv) {
    float2* row = rowp_w<float2>(base, pitch, y);
    if (c.out1) {
        *reinterpret_cast<float4*>(row + c.c0) = make_float4(xs.x, ysv.x, xs.y, ysv.y);
    } else if (EX && c.out0) {
        row[c.c0] = make_float2(xs.x, ysv.x);
    }
}
template <bool EX>
__device__ __forceinline__ void store_f1pair(const Ctx& c, float* base, size_t pitch, int y, float2 v) {
    float* row = rowp_w<float>(base, pitch, y);
    if (c.out1) {
        *reinterpret_cast<float2*>(row + c.c0) = v;
    } else if (EX && c.out0) {
        row[c.c0] = v.x;
    }
}

// ---------------------------------------------------------------- per-warp shared memory
// [input ring: kDepth slots] [image-model window: 4 rows] [smoothing windows: S x 4 rows].
// A window row is two planes of 32 lanes x 8 B (one float2 pixel pair per lane): the image
// and its X blur for the model, the X-pass U and V for a smoothing iteration.  Row y of a
// window lives in slot y & 3; every lane reads back only what it wrote itself.
constexpr int kPlane = 32 * 8;
constexpr int kWinRow = 2 * kPlane;
template <bool DELTA, int S>
struct WarpMem {
    static constexpr int SLOT = DELTA ? Slot::DELTA_BYTES : Slot::TOP_BYTES;
    static constexpr int MODEL = kDepth * SLOT;
    static constexpr int SMOOTH = MODEL + 4 * kWinRow;
    static constexpr int BYTES = SMOOTH + S * 4 * kWinRow;
};

// The block's dynamic shared memory, addressed by 32-bit byte offsets (the kernels below
// declare the same array)
extern __shared__ __align__(16) char lvl_smem[];
__device__ __forceinline__ float2 lds2(unsigned off) { return *reinterpret_cast<const float2*>(lvl_smem + off); }
__device__ __forceinline__ void sts2(unsigned off, float2 v) { *reinterpret_cast<float2*>(lvl_smem + off) = v; }
__device__ __forceinline__ float4 lds4(unsigned off) { return *reinterpret_cast<const float4*>(lvl_smem + off); }

// The pipeline of one warp.  DELTA: delta level (flow, old image and delta flow are
// propagated; the update refines the coarse flow).  Otherwise a top level (flow is
// propagated; old image read in place).
// EX: the warp's window reaches an image edge or the propagation border columns (column
// substitution, per-lane freeze, lanes outside the image).  EY (per row, see run_warp):
// the rows of this step reach the top/bottom edge or border rows (row clamping,
// substitution and freeze).  Interior warps and rows compile without any of it.
// The propagation windows (two rows per sub-step) stay in registers and swap roles with
// the row parity PAR (the row loop is unrolled by two), so they rotate without moves;
// the 4-row windows of the 5-tap vertical filters live in shared memory.
template <bool DELTA, int N, int S, typename P, bool EX>
struct Pipe {
    // propagated channels: U, V (flow) [, I old image, DX, DY delta flow]
    static constexpr int NC = DELTA ? 5 : 2;
    static constexpr int CU = 0, CV = 1, CI = 2, CDX = 3, CDY = 4;
    // channels whose upwind step the reference build fuses into one fma: all but the
    // last channel each reference kernel writes (flow .y of flowPropagate{X,Y}_k,
    // vector .y of flowPropagatePayload{X,Y}_k)
    static constexpr bool fused(int ch) { return DELTA ? ch != CDY : ch != CV; }
    using M = WarpMem<DELTA, S>;

    float2 pw[N][2][NC];  // Y sub-step windows: the X sub-step output of the two rows before
    // propagated channels the update reads (DELTA: old image and delta flow; top: flow),
    // carried one row when the update runs a row behind the propagation (kDelay)
    static constexpr int NU = DELTA ? 3 : 2;
    float2 xu[NU];
    int cr_next;  // delta levels: coarse row of the update row the next step stages

    // coarse row (upmap_index of the row, from the level's table) read by the update of the
    // row that step i stages
    __device__ __forceinline__ static int coarse_row(const Ctx& c, const LevelArgs& a, int i) {
        return __ldg(a.coarse_rows + min(max(i - N - kDelay, 0), c.H - 1));
    }

    __device__ __forceinline__ void init(const Ctx& c) {
#pragma unroll
        for (int k = 0; k < N; ++k)
#pragma unroll
            for (int r = 0; r < 2; ++r)
#pragma unroll
                for (int ch = 0; ch < NC; ++ch) pw[k][r][ch] = make_float2(0.f, 0.f);
#pragma unroll
        for (int u = 0; u < NU; ++u) xu[u] = make_float2(0.f, 0.f);
        const unsigned w = c.o8 + M::MODEL;
#pragma unroll
        for (int r = 0; r < 4 * (1 + S); ++r) {
            sts2(w + r * kWinRow, make_float2(0.f, 0.f));
            sts2(w + r * kWinRow + kPlane, make_float2(0.f, 0.f));
        }
    }

    // border freeze (propagation_k.cu:59-65): pixels within `border` of an edge keep v
    template <bool EY>
    __device__ __forceinline__ static void freeze(const Ctx& c, int q, float2 (&out)[NC], const float2 (&v)[NC]) {
        if (EY && (q < c.border || q >= c.H - c.border)) {  // warp-uniform
#pragma unroll
            for (int ch = 0; ch < NC; ++ch) out[ch] = v[ch];
        } else if (EX && c.freeze_cols) {  // warp-uniform
#pragma unroll
            for (int ch = 0; ch < NC; ++ch) {
                out[ch].x = c.col0 ? out[ch].x : v[ch].x;
                out[ch].y = c.col1 ? out[ch].y : v[ch].y;
            }
        }
    }

    // X sub-step in place on row q (flowPropagateX_k / flowPropagatePayloadX_k).  The minus
    // and plus neighbours of the pair (c0, c1) are (lane-1's c1, c0) and (c1, lane+1's c0);
    // the upwind neighbour is selected per pixel straight from them.
    template <bool EY>
    __device__ __forceinline__ static void prop_x(const Ctx& c, int q, float2 (&v)[NC]) {
        float2 m[NC], p[NC];
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) nb3<EX>(c, v[ch], m[ch], p[ch]);
        const float2 vel = make_float2(dominant(m[CU].x, p[CU].x), dominant(m[CU].y, p[CU].y));
        const float2 at = abs_t(c.dt, vel);
        const bool fw0 = vel.x >= 0.0f, fw1 = vel.y >= 0.0f;
        float2 o[NC];
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) {
            if (fused(ch)) o[ch] = upwind2<true>(v[ch], m[ch], p[ch], fw0, fw1, at);
            else o[ch] = upwind2<false>(v[ch], m[ch], p[ch], fw0, fw1, at);
        }
        freeze<EY>(c, q, o, v);
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) v[ch] = o[ch];
    }

    // Y sub-step producing row q from rows q-1 (prev), q (cur), q+1 (next)
    template <bool EY>
    __device__ __forceinline__ static void prop_y(const Ctx& c, int q, const float2 (&prev)[NC],
                                                  const float2 (&cur)[NC], const float2 (&next)[NC],
                                                  float2 (&o)[NC]) {
        float2 m[NC], p[NC];
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) {
            m[ch] = prev[ch];
            p[ch] = next[ch];
        }
        if (EY && (q == 0 || q == c.H - 1)) {  // warp-uniform
#pragma unroll
            for (int ch = 0; ch < NC; ++ch) {
                if (q == 0) m[ch] = cur[ch];
                if (q == c.H - 1) p[ch] = cur[ch];
            }
        }
        const float2 vel = make_float2(dominant(m[CV].x, p[CV].x), dominant(m[CV].y, p[CV].y));
        const float2 at = abs_t(c.dt, vel);
        const bool fw0 = vel.x >= 0.0f, fw1 = vel.y >= 0.0f;
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) {
            if (fused(ch)) o[ch] = upwind2<true>(cur[ch], m[ch], p[ch], fw0, fw1, at);
            else o[ch] = upwind2<false>(cur[ch], m[ch], p[ch], fw0, fw1, at);
        }
        freeze<EY>(c, q, o, cur);
    }

    template <bool EY>
    __device__ __forceinline__ static int clampr(const Ctx& c, int r) { return EY ? min(max(r, 0), c.H - 1) : r; }

    // copy every input that iteration i consumes into slot `slot`.  Each lane copies the
    // aligned column pair (b0, b0+1) of every field; b0 = clamp(c0) rounded down to even,
    // so one 16/8/4-byte copy per field, and rows carry at least one column of padding.
    template <bool EY>
    // crow: the coarse row of the update row i - N - kDelay (delta levels)
    __device__ __forceinline__ static void issue(const Ctx& c, const LevelArgs& a, int slot, int i, int crow_y) {
        const unsigned sb8 = c.smem_s + 8 * c.lane + slot * M::SLOT;
        const unsigned sb16 = c.smem_s + 16 * c.lane + slot * M::SLOT;
        const int r = clampr<EY>(c, i);
        cp16(sb16 + Slot::FLOW, rowp<float2>(a.fs_in, a.fs_in_pitch, r) + c.b0);
        const int ru = clampr<EY>(c, i - N - kDelay);  // update row
        cp8(sb8 + Slot::IO, rowp<float>(a.io_in, a.io_in_pitch, DELTA ? r : ru) + c.b0);
        if constexpr (DELTA) {
            cp16(sb16 + Slot::DELTA, rowp<float2>(a.d_in, a.d_in_pitch, r) + c.b0);
            // coarse row of the update row from the level's row table (upmap_index of each row)
            const float2* crow = rowp<float2>(a.coarse, a.coarse_pitch, crow_y);
            cp8(sb16 + Slot::COARSE, crow + c.ix0);
            cp8(sb16 + Slot::COARSE + 8, crow + c.ix1);
        }
        const int rj = clampr<EY>(c, i - N + 2 - kDelay);  // image row
        if constexpr (sizeof(P) == 1) {
            // the aligned 32-bit word holding columns b0, b0+1 (image rows are 4-byte
            // aligned and padded to a multiple of 4 bytes; see fused_available)
            cp4(sb8 + Slot::IMG, reinterpret_cast<const uint8_t*>(rowp<P>(a.img, a.img_pitch, rj)) + (c.b0 & ~3));
        } else {
            cp8(sb8 + Slot::IMG, rowp<P>(a.img, a.img_pitch, rj) + c.b0);
        }
    }

    // pixel values of the lane from a loaded pair (b0, b0+1): identity unless the lane's
    // clamped columns are not (b0, b0+1) (lanes outside the image or at an odd right edge)
    __device__ __forceinline__ static float2 unpair(const Ctx& c, float lo, float hi) {
        float2 v = make_float2(lo, hi);
        if (EX && c.any_split) {  // warp-uniform
            v.x = c.cc0 == c.b0 ? lo : hi;
            v.y = c.cc1 == c.b0 ? lo : hi;
        }
        return v;
    }

    // one streamed row; its inputs wait in slot `slot`.  PAR: row parity (which register
    // of each propagation window holds the older row), or -1 when the loop body holds one
    // row and the windows shift; EA: the inputs this step stages need row clamping
    template <bool EY, bool EA, int PAR>
    __device__ __forceinline__ void step(const Ctx& c, const LevelArgs& a, int i, int slot) {
        const int H = c.H;
        cp_wait<kDepth - 1>();
        const unsigned sb8 = c.o8 + slot * M::SLOT, sb16 = c.o16 + slot * M::SLOT;
        // ---- state row i
        float2 x[NC];
        float2 io_u;  // top levels: old image at the update row
        float2 im;    // image row i-N+2
        float4 cf;    // delta levels: coarse flow (u0, v0, u1, v1) at the update row
        {
            const float4 q = lds4(sb16 + Slot::FLOW);
            x[CU] = unpair(c, q.x, q.z);
            x[CV] = unpair(c, q.y, q.w);
            const float2 iop = lds2(sb8 + Slot::IO);
            const float2 io = unpair(c, iop.x, iop.y);
            if constexpr (DELTA) {
                x[CI] = io;
                const float4 d = lds4(sb16 + Slot::DELTA);
                x[CDX] = unpair(c, d.x, d.z);
                x[CDY] = unpair(c, d.y, d.w);
                cf = lds4(sb16 + Slot::COARSE);
                io_u = make_float2(0.f, 0.f);
            } else {
                io_u = io;
                cf = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            if constexpr (sizeof(P) == 1) {
                const uint32_t w = *reinterpret_cast<const uint32_t*>(lvl_smem + sb8 + Slot::IMG);
                uint32_t v0, v1;
                if (EX) {
                    v0 = (w >> (8 * (c.cc0 & 3))) & 0xffu;
                    v1 = (w >> (8 * (c.cc1 & 3))) & 0xffu;
                } else {  // c0 even and inside: the pair is bytes sh, sh+1 of the word
                    const uint32_t sh = 8 * (c.cc0 & 2);
                    v0 = (w >> sh) & 0xffu;
                    v1 = (w >> (sh + 8)) & 0xffu;
                }
                im = make_float2(u8_to_unit(v0), u8_to_unit(v1));
            } else {
                const float2 ip = lds2(sb8 + Slot::IMG);
                im = unpair(c, ip.x, ip.y);
            }
        }
        // the slot is free again: stage the row needed kDepth iterations from now
        // the coarse row of the row staged next step is loaded a step ahead
        const int crow_y = cr_next;
        if constexpr (DELTA) cr_next = coarse_row(c, a, i + 1 + kDepth);
        issue<EA>(c, a, slot, i + kDepth, crow_y);
        cp_commit();
        // ---- N propagation sub-steps
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const int q = i - k;  // row of this X sub-step
            prop_x<EY>(c, q, x);
            float2 y[NC];
            prop_y<EY>(c, q - 1, pw[k][PAR < 0 ? 0 : PAR], pw[k][PAR < 0 ? 1 : PAR ^ 1], x, y);
#pragma unroll
            for (int ch = 0; ch < NC; ++ch) {
                if (PAR < 0) {  // one row per loop body: the window shifts
                    pw[k][0][ch] = pw[k][1][ch];
                    pw[k][1][ch] = x[ch];
                } else {
                    pw[k][PAR][ch] = x[ch];  // the newest row replaces the oldest
                }
                x[ch] = y[ch];
            }
        }
        const int r = i - N - kDelay;  // row of the update
        // the propagated channels the update reads: this row's, or the previous row's
        float2 pu[NU];
#pragma unroll
        for (int u = 0; u < NU; ++u) {
            const float2 now = x[DELTA ? CI + u : CU + u];
            pu[u] = kDelay ? xu[u] : now;
            xu[u] = now;
        }
        // window rows: slot (i + k) & 3 holds the row k steps after the oldest
        const int w0 = ((i + 0) & 3) * kWinRow, w1 = ((i + 1) & 3) * kWinRow;
        const int w2 = ((i + 2) & 3) * kWinRow, w3 = ((i + 3) & 3) * kWinRow;
        const unsigned wl = c.o8;
        // ---- image model at row r (imagemodel_k.cu:31-133)
        float2 a0, ax, ay;
        {
            const unsigned mw = wl + M::MODEL;
            float2 t[5];
            nb5_raw(im, t);
            const float2 bx = smooth5p(t);
            const float2 by = smooth5_pair(lds2(mw + w0), lds2(mw + w1), lds2(mw + w2), lds2(mw + w3), im);
            ay = diff5_pair(lds2(mw + w0 + kPlane), lds2(mw + w1 + kPlane), lds2(mw + w2 + kPlane),
                            lds2(mw + w3 + kPlane), bx);
            sts2(mw + w0, im);
            sts2(mw + w0 + kPlane, bx);
            float2 tb[5];
            nb5_raw(by, tb);
            a0 = smooth5p(tb);
            ax = diff5p(tb);
        }
        // ---- update at row r
        float2 fu, fv;
        float2 dox, doy;  // the update's stored flow: delta flow (delta levels), unsmoothed flow (top)
        {
            float2 old;
            if constexpr (DELTA) old = pu[0];
            else old = io_u;
            if (c.first) old = a0;
            float2 fx, fy;
            if constexpr (DELTA) {
                fx = pu[1];
                fy = pu[2];
            } else {
                fx = pu[0];
                fy = pu[1];
            }
            float2 ox, oy;
            solve2(c.gamma, ax.x, ay.x, __fsub_rn(old.x, a0.x), fx.x, fy.x, ox.x, oy.x);
            solve2(c.gamma, ax.y, ay.y, __fsub_rn(old.y, a0.y), fx.y, fy.y, ox.y, oy.y);
            if constexpr (DELTA) {
                // deltaFlowUpdate_k (update_k.cu:136-164)
                ox = make_float2(clampm(sanitize(ox.x), c.half_maxflow), clampm(sanitize(ox.y), c.half_maxflow));
                oy = make_float2(clampm(sanitize(oy.x), c.half_maxflow), clampm(sanitize(oy.y), c.half_maxflow));
                const float2 u0 = make_float2(cf.x, cf.y), u1 = make_float2(cf.z, cf.w);
                fu = make_float2(clampm(__fadd_rn(ox.x, __fmul_rn(2.0f, u0.x)), c.maxflow),
                                 clampm(__fadd_rn(ox.y, __fmul_rn(2.0f, u1.x)), c.maxflow));
                fv = make_float2(clampm(__fadd_rn(oy.x, __fmul_rn(2.0f, u0.y)), c.maxflow),
                                 clampm(__fadd_rn(oy.y, __fmul_rn(2.0f, u1.y)), c.maxflow));
                dox = ox;
                doy = oy;
            } else {
                // flowUpdate_k (update_k.cu:65-78)
                fu = make_float2(sanitize(clampm(ox.x, c.maxflow)), sanitize(clampm(ox.y, c.maxflow)));
                fv = make_float2(sanitize(clampm(oy.x, c.maxflow)), sanitize(clampm(oy.y, c.maxflow)));
                dox = fu;
                doy = fv;
            }
        }
        // ---- S smoothing iterations (flowsmoothing_k.cu:21-87)
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const unsigned sw = wl + M::SMOOTH + s * 4 * kWinRow;
            float2 tu[5], tv[5];
            nb5<EX>(c, fu, tu);
            nb5<EX>(c, fv, tv);
            const float2 sxu = box5p(tu), sxv = box5p(tv);
            const int q = r - 2 * s - 2;  // row of this Y pass
            float2 ru[5] = {lds2(sw + w0), lds2(sw + w1), lds2(sw + w2), lds2(sw + w3), sxu};
            float2 rv[5] = {lds2(sw + w0 + kPlane), lds2(sw + w1 + kPlane), lds2(sw + w2 + kPlane),
                            lds2(sw + w3 + kPlane), sxv};
            sts2(sw + w0, sxu);
            sts2(sw + w0 + kPlane, sxv);
            if (EY && (q < 2 || q > H - 3)) {
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
        }
        // ---- stores, after all arithmetic of the step
        if (r >= c.ys && r < c.ye) {  // warp-uniform
            store_f1pair<EX>(c, a.io_out, a.io_out_pitch, r, a0);
            if (DELTA) store_f2pair<EX>(c, a.d_out, a.d_out_pitch, r, dox, doy);
            else if (a.fu_out) store_f2pair<EX>(c, a.fu_out, a.fu_out_pitch, r, dox, doy);
        }
        const int rs = r - 2 * S;
        if (rs >= c.ys && rs < c.ye) store_f2pair<EX>(c, a.fs_out, a.fs_out_pitch, rs, fu, fv);
    }
};

// Rows [lo, hi] of a level are interior for the streaming pipeline when a step there and
// the inputs it stages need no row clamping, substitution or freeze.  A step at row i
// stages row i+kDepth, whose loads reach rows i+kDepth-N (update) up to i+kDepth (state)
// and i+kDepth-N+2 (image, below the state row when N < 2); its propagation rows i-N .. i
// stay inside the border, and its smoothing windows (down to row i-N-2S-2) inside the image.
template <int N, int S>
__device__ __forceinline__ void interior_rows(int H, int border, int& lo, int& hi) {
    const int mb = border > 1 ? border : 1;
    constexpr int ahead = kDepth + (N + kDelay < 2 ? 2 - N - kDelay : 0);  // rows below i the staged loads reach
    lo = N + kDelay + (2 * S + 2 > mb ? 2 * S + 2 : mb);
    hi = H - 1 - (ahead > mb ? ahead : mb);
}

template <bool DELTA, int N, int S, typename P, bool EX>
__device__ __forceinline__ void run_warp(const LevelArgs& a, Ctx& c, int i0, int iters) {
    using Pp = Pipe<DELTA, N, S, P, EX>;
    Pp pipe;
    pipe.init(c);
    pipe.cr_next = DELTA ? Pp::coarse_row(c, a, i0 + kDepth) : 0;
#pragma unroll
    for (int u = 0; u < kDepth; ++u) {
        Pp::template issue<true>(c, a, u, i0 + u, DELTA ? Pp::coarse_row(c, a, i0 + u) : 0);
        cp_commit();
    }
    // rows [lo, hi] are interior (no row clamping, substitution or freeze)
    int lo, hi;
    interior_rows<N, S>(c.H, c.border, lo, hi);
#if FFB_ROW_UNROLL == 2
    // two rows per loop body (the propagation windows swap roles instead of moving); a body
    // is interior when both of its rows are.  kDepth is a multiple of 2, so the slot index
    // of step it is it & (kDepth - 1)
#pragma unroll 1
    for (int it = 0; it < iters; it += 2) {
        const int i = i0 + it;
        if (i >= lo && i + 1 <= hi) {  // warp-uniform
            pipe.template step<false, false, 0>(c, a, i, it & (kDepth - 1));
            pipe.template step<false, false, 1>(c, a, i + 1, (it + 1) & (kDepth - 1));
        } else {
            pipe.template step<true, true, 0>(c, a, i, it & (kDepth - 1));
            pipe.template step<true, true, 1>(c, a, i + 1, (it + 1) & (kDepth - 1));
        }
    }
#else
    // one row per loop body, kept small for the instruction cache: the edge rows before and
    // after the interior ones run one loop, the interior rows another
    int it_a = lo - i0, it_b = hi - i0 + 1;
    it_a = it_a < 0 ? 0 : (it_a > iters ? iters : it_a);
    it_b = it_b < it_a ? it_a : (it_b > iters ? iters : it_b);
    int it = 0;
#pragma unroll 1
    for (int ph = 0; ph < 3; ++ph) {
        const int end = ph == 0 ? it_a : (ph == 1 ? it_b : iters);
        if (ph == 1) {
#pragma unroll 1
            for (; it < end; ++it) pipe.template step<false, false, -1>(c, a, i0 + it, it & (kDepth - 1));
        } else {
#pragma unroll 1
            for (; it < end; ++it) pipe.template step<true, true, -1>(c, a, i0 + it, it & (kDepth - 1));
        }
    }
#endif
    cp_wait<0>();
}

// halo widths of a level: columns on each side (even) and rows before the band
__host__ __device__ constexpr int halo_x(int N, int S) { return ((2 * S + (N > 2 ? N : 2)) + 1) & ~1; }
__host__ __device__ constexpr int lead_rows(int N, int S) { return 2 * S + (N > 4 - N ? N : 4 - N); }

// The warps of a level: nwx windows of 64 columns, each cut into bands of `band` rows.
// The first and last windows (where the image edges are, and the column handling makes a
// row dearer) are cut into bands of half the height, so their warps finish with the rest.
struct WarpGrid {
    int nwx, band, nby;   // interior windows: nby bands of `band` rows
    int ne, band_e, nby_e;  // edge windows (ne of them): nby_e bands of band_e rows
    __host__ __device__ WarpGrid(int nwx_, int band_, int H) : nwx(nwx_), band(band_) {
        nby = (H + band - 1) / band;
        ne = nwx < 2 ? nwx : 2;
        band_e = (band + 1) / 2 < 8 ? (band < 8 ? band : 8) : (band + 1) / 2;
        nby_e = (H + band_e - 1) / band_e;
    }
    __host__ __device__ int warps() const { return ne * nby_e + (nwx - ne) * nby; }
    // window column, first row and row count of warp w
    __host__ __device__ void at(int w, int& wx, int& ys, int& rows) const {
        if (w < ne * nby_e) {
            wx = w < nby_e ? 0 : nwx - 1;
            ys = (w % nby_e) * band_e;
            rows = band_e;
        } else {
            w -= ne * nby_e;
            wx = 1 + w % (nwx - ne);
            ys = (w / (nwx - ne)) * band;
            rows = band;
        }
    }
};

// warp `warp` of a level's WarpGrid of (64-column window, band) warps
template <bool DELTA, int N, int S, typename P>
__device__ __forceinline__ void level_warp(const LevelArgs& a, int nwx, int band, int warp) {
    constexpr int HX = halo_x(N, S);
    constexpr int OX = 64 - 2 * HX;
    const WarpGrid g(nwx, band, a.H);
    if (warp >= g.warps()) return;  // whole warps exit together
    const int lane = threadIdx.x & 31;
    int wx, ys0, rows;
    g.at(warp, wx, ys0, rows);
    const int W = a.W, H = a.H;

    Ctx c;
    c.W = W;
    c.H = H;
    c.lane = lane;
    const unsigned so = (threadIdx.x >> 5) * WarpMem<DELTA, S>::BYTES;
    c.o8 = so + 8 * lane;
    c.o16 = so + 16 * lane;
    c.smem_s = (unsigned)__cvta_generic_to_shared(lvl_smem) + so;
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
    c.ys = ys0;
    c.ye = min(ys0 + rows, H);
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
    c.e_l = c.c0 == 0;
    c.e_r1 = c.c1 == W - 1;
    c.e_r0 = c.c0 == W - 1;
    c.e_r2 = c.c1 == W - 2 && (W & 1);
    c.freeze_cols = __any_sync(kFull, !(c.col0 && c.col1));
    c.b0 = min(max(c.c0, 0), (W - 1) & ~1);
    c.any_edge = __any_sync(kFull, c.e_l || c.e_r0 || c.e_r1 || c.e_r2);
    c.any_split = __any_sync(kFull, c.cc0 != c.b0 || c.cc1 != c.b0 + 1);
    const int i0 = c.ys - lead_rows(N, S);
    const int last = c.ye - 1 + N + kDelay + 2 * S;
    // rows of the band's pipeline (an even count when the loop body holds two rows)
    const int iters = FFB_ROW_UNROLL == 2 ? (last - i0 + 2) & ~1 : last - i0 + 1;
    // Warps whose 64 columns lie inside the image and outside the border columns (all but
    // the first and last window of each band) run the pipeline without column handling.
    if (c.any_edge || c.freeze_cols || c.any_split)  // warp-uniform
        run_warp<DELTA, N, S, P, true>(a, c, i0, iters);
    else
        run_warp<DELTA, N, S, P, false>(a, c, i0, iters);
}

template <bool DELTA, int N, int S, typename P>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kBlocksPerSM) level_k(LevelArgs a, int nwx, int band) {
    grid_dep_wait();
    grid_dep_launch();
    level_warp<DELTA, N, S, P>(a, nwx, band, blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5));
}

template <bool DELTA, int N, int S, typename P>
cudaError_t launch(const LevelArgs& a, cudaStream_t s) {
    constexpr int HX = halo_x(N, S);
    constexpr int OX = 64 - 2 * HX;
    const int smem = kWarpsPerBlock * WarpMem<DELTA, S>::BYTES;
    // row offsets are computed as 32 x 32-bit products (rowp)
    for (size_t p : {a.img_pitch, a.fs_in_pitch, a.io_in_pitch, a.d_in_pitch, a.fs_out_pitch, a.io_out_pitch,
                     a.d_out_pitch, a.fu_out_pitch, a.coarse_pitch})
        if (p >> 32) return cudaErrorInvalidPitchValue;
    // resident warps on this device, queried once per instantiation and device (the
    // function attributes are set per device as well)
    static int resident[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    int& resident_warps = resident[dev & 63];
    if (resident_warps == 0) {
        int sms = 0, per_sm = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        // full shared carve-out, as for the tile kernels: SMs running this kernel can then
        // also host the tile kernels of the levels that run beside it
        cudaFuncSetAttribute(level_k<DELTA, N, S, P>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
        const cudaError_t e =
            cudaFuncSetAttribute(level_k<DELTA, N, S, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, level_k<DELTA, N, S, P>, kWarpsPerBlock * 32, smem);
        resident_warps = (sms > 0 ? sms : 148) * (per_sm > 0 ? per_sm : 1) * kWarpsPerBlock;
    }
    const int nwx = (a.W + OX - 1) / OX;
    // bands: as few as fill the resident warps once (every extra band restarts a pipeline);
    // the edge windows' half-height bands count twice
    int band = a.band;
    if (band <= 0) {
        const int cols = nwx + (nwx < 2 ? nwx : 2);
        const int bands = resident_warps / cols > 0 ? resident_warps / cols : 1;
        band = (a.H + bands - 1) / bands;
        while (band < a.H && WarpGrid(nwx, band, a.H).warps() > resident_warps) ++band;
    }
    band = band < 8 ? 8 : band;
    band = band > a.H ? a.H : band;
    const int warps = WarpGrid(nwx, band, a.H).warps();
    const int blocks = (warps + kWarpsPerBlock - 1) / kWarpsPerBlock;
    return launch_k(level_k<DELTA, N, S, P>, dim3(blocks), dim3(kWarpsPerBlock * 32), smem, s, a, nwx, band);
}

}  // namespace lvl
}  // namespace ffb
