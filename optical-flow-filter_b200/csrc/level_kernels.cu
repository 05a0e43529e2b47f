// Dispatch to the fused per-level kernels (level_pipe.cuh, instantiated in level_n*.cu).
#include "kernels.h"

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

}  // namespace ffb
