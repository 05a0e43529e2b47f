// Dispatch to the fused per-level kernels (level_pipe.cuh, instantiated in level_n*.cu).
#include "level_pipe.cuh"

namespace ffb {

cudaError_t launch_level_n1(bool delta, int item, int S, const LevelArgs& a, cudaStream_t s);
cudaError_t launch_level_n2(bool delta, int item, int S, const LevelArgs& a, cudaStream_t s);
cudaError_t launch_level_n3(bool delta, int item, int S, const LevelArgs& a, cudaStream_t s);
cudaError_t launch_level_n4(bool delta, int item, int S, const LevelArgs& a, cudaStream_t s);

// instantiated: propagation iterations 1..4, smoothing iterations 1..4; delta levels on
// uint8 images, top levels on uint8 or float images.  Other combinations run the
// per-stage kernels, which give identical results.
bool fused_available(bool delta, int item, int N, int S) {
    if (N < 1 || N > 4 || S < 1 || S > 4) return false;
    if (delta && item != 1) return false;
    return item == 1 || item == 4;
}

cudaError_t launch_fused_level(bool delta, int N, int S, const LevelArgs& a, cudaStream_t s) {
    switch (N) {
        case 1: return launch_level_n1(delta, a.item, S, a, s);
        case 2: return launch_level_n2(delta, a.item, S, a, s);
        case 3: return launch_level_n3(delta, a.item, S, a, s);
        case 4: return launch_level_n4(delta, a.item, S, a, s);
    }
    return cudaErrorNotSupported;
}

int fused_warp_grid(int N, int S, int W, int H, int band, int* nwx, int* nby) {
    const int ox = 64 - 2 * lvl::halo_x(N, S);
    band = band < 8 ? 8 : band;
    band = band > H ? H : band;
    *nwx = (W + ox - 1) / ox;
    *nby = (H + band - 1) / band;
    return (lvl::WarpGrid(*nwx, band, H).warps() + lvl::kWarpsPerBlock - 1) / lvl::kWarpsPerBlock;
}

int fused_resident_warps() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (sms > 0 ? sms : 148) * lvl::kBlocksPerSM * lvl::kWarpsPerBlock;
}

}  // namespace ffb
