// Tile-fused level step: launch side.  The device code is in tile_body.cuh; this file
// chooses the tile shape of a level (from the SM count, or by the autotuner) and launches
// one CTA per output tile.
#include <algorithm>
#include <atomic>

#include "tile_body.cuh"

namespace ffb {
namespace tile {

template <bool DELTA, typename P>
__global__ void __launch_bounds__(1024) tile_k(LevelArgs a, Geom g) {
    extern __shared__ __align__(16) unsigned char sm[];
    tile_body<DELTA, P>(a, g, blockIdx.x, sm);
}

struct DeviceInfo {
    int sms = 0;
    size_t smem_optin = 0;
};

DeviceInfo device_info() {
    static DeviceInfo cache[64];
    int dev = 0;
    cudaGetDevice(&dev);
    DeviceInfo& d = cache[dev & 63];
    if (d.sms == 0) {
        int sms = 0, optin = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        d.smem_optin = (size_t)(optin > 0 ? optin : 48 * 1024);
        d.sms = sms > 0 ? sms : 148;
    }
    return d;
}

// A tile-shape choice is a tile width, a number of tiles resident per SM and the threads of
// a tile; the tile height follows so that the tiles fill whole waves of the GPU (as few as
// fit in shared memory).  Index 0 is the automatic choice.
struct Choice {
    int tw, per_sm, threads;
};
constexpr Choice kChoices[] = {{0, 0, 0},     {32, 1, 512},  {32, 2, 512},  {32, 3, 256},  {48, 1, 512},
                               {48, 2, 512},  {48, 3, 256},  {64, 1, 512},  {64, 2, 512},  {64, 3, 256},
                               {96, 1, 512},  {96, 2, 512},  {128, 1, 512}, {32, 1, 1024}, {48, 1, 1024},
                               {64, 1, 1024}, {96, 1, 1024}, {128, 1, 1024}};
constexpr int kNumChoices = sizeof(kChoices) / sizeof(kChoices[0]);
constexpr size_t kSmemPerSM = 228 * 1024;  // B200 shared memory per SM
constexpr size_t kSmemReserve = 1024;      // per resident block

struct Cfg {
    int tw = 0, th = 0, threads = 0, waves = 0, per_sm = 0;
};

Cfg shape_of(Choice c, bool delta, int N, int S, int W, int H) {
    Cfg out;
    if (c.tw <= 0) return out;
    const DeviceInfo d = device_info();
    const int threads = c.threads;
    if (threads * c.per_sm > 2048) return out;
    const int tiles_x = (W + c.tw - 1) / c.tw;
    for (int waves = 1; waves <= 256; ++waves) {
        const long slots = (long)d.sms * c.per_sm * waves;
        const long rows = std::max(1L, slots / tiles_x);
        int th = (int)((H + rows - 1) / rows);
        th = std::max(1, std::min(th, H));
        const size_t smem = layout(delta, N, S, c.tw, th).total;
        if (smem <= d.smem_optin && (smem + kSmemReserve) * c.per_sm <= kSmemPerSM) {
            out.tw = c.tw;
            out.th = th;
            out.threads = threads;
            out.waves = waves;
            out.per_sm = c.per_sm;
            return out;
        }
        if (th == 1) break;
    }
    return out;
}

// automatic shape: the least halo-inflated work per SM over the waves it takes
Cfg auto_cfg(bool delta, int N, int S, int W, int H) {
    const int R = N + 2 * S;
    Cfg best;
    double best_cost = 0;
    for (int i = 1; i < kNumChoices; ++i) {
        const Cfg c = shape_of(kChoices[i], delta, N, S, W, H);
        if (c.tw == 0) continue;
        const double cost = (double)c.waves * c.per_sm * (c.tw + R) * (c.th + R);
        if (best.tw == 0 || cost < best_cost) {
            best = c;
            best_cost = cost;
        }
    }
    return best;
}

Cfg cfg_of(int index, bool delta, int N, int S, int W, int H) {
    if (index < 0 || index >= kNumChoices) return Cfg{};
    return index == 0 ? auto_cfg(delta, N, S, W, H) : shape_of(kChoices[index], delta, N, S, W, H);
}

template <bool DELTA, typename P>
cudaError_t launch_t(const LevelArgs& a, int N, int S, Cfg c, cudaStream_t s) {
    static std::atomic<unsigned long long> prepared{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    const Layout L = layout(DELTA, N, S, c.tw, c.th);
    if (!(prepared.load() & bit)) {
        cudaError_t e = cudaFuncSetAttribute(tile_k<DELTA, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)device_info().smem_optin);
        if (e != cudaSuccess) return e;
        // An SM's L1/shared split is fixed while blocks run on it.  A small tile (the top
        // level's) would otherwise get a small shared carve-out, and the next level's large
        // tiles, launched early to overlap it, could not share its SMs: ask for the full
        // shared-memory carve-out for every tile kernel.
        e = cudaFuncSetAttribute(tile_k<DELTA, P>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
        prepared.fetch_or(bit);
    }
    Geom g;
    g.TW = c.tw;
    g.TH = c.th;
    g.N = N;
    g.S = S;
    g.R = N + 2 * S;
    g.SW = c.tw + 2 * g.R;
    g.SH = c.th + 2 * g.R;
    g.tiles_x = (a.W + c.tw - 1) / c.tw;
    g.offB = (int)L.a;
    g.offC = (int)(L.a + L.b);
    const int tiles = g.tiles_x * ((a.H + c.th - 1) / c.th);
    return launch_k(tile_k<DELTA, P>, dim3(tiles), dim3(c.threads), L.total, s, a, g);
}

}  // namespace tile

int tile_config_count() { return tile::kNumChoices; }

bool tile_available(bool delta, int N, int S, int W, int H, int cfg) {
    if (N < 1 || S < 1 || W < 1 || H < 1) return false;
    return tile::cfg_of(cfg, delta, N, S, W, H).tw > 0;
}

void tile_shape(bool delta, int N, int S, int W, int H, int cfg, int* tw, int* th) {
    const tile::Cfg c = tile::cfg_of(cfg, delta, N, S, W, H);
    *tw = c.tw;
    *th = c.th;
}

cudaError_t launch_tile_level(bool delta, int N, int S, const LevelArgs& a, int cfg, cudaStream_t s) {
    if (N < 1 || S < 1) return cudaErrorInvalidConfiguration;
    const tile::Cfg c = tile::cfg_of(cfg, delta, N, S, a.W, a.H);
    if (c.tw == 0) return cudaErrorInvalidConfiguration;
    if (delta) {
        return a.item == 1 ? tile::launch_t<true, uint8_t>(a, N, S, c, s) : tile::launch_t<true, float>(a, N, S, c, s);
    }
    return a.item == 1 ? tile::launch_t<false, uint8_t>(a, N, S, c, s) : tile::launch_t<false, float>(a, N, S, c, s);
}

}  // namespace ffb
