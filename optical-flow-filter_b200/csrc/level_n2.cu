// Instantiations of the fused level kernel for 2 propagation iteration(s).
#include "level_pipe.cuh"

namespace ffb {

cudaError_t launch_level_n2(bool delta, int item, int S, const LevelArgs& a, cudaStream_t s) {
    using lvl::launch;
    if (delta) {
        if (item != 1) return cudaErrorNotSupported;
        switch (S) {
            case 1: return launch<true, 2, 1, uint8_t>(a, s);
            case 2: return launch<true, 2, 2, uint8_t>(a, s);
            case 3: return launch<true, 2, 3, uint8_t>(a, s);
            case 4: return launch<true, 2, 4, uint8_t>(a, s);
        }
    } else if (item == 1) {
        switch (S) {
            case 1: return launch<false, 2, 1, uint8_t>(a, s);
            case 2: return launch<false, 2, 2, uint8_t>(a, s);
            case 3: return launch<false, 2, 3, uint8_t>(a, s);
            case 4: return launch<false, 2, 4, uint8_t>(a, s);
        }
    } else {
        switch (S) {
            case 1: return launch<false, 2, 1, float>(a, s);
            case 2: return launch<false, 2, 2, float>(a, s);
            case 3: return launch<false, 2, 3, float>(a, s);
            case 4: return launch<false, 2, 4, float>(a, s);
        }
    }
    return cudaErrorNotSupported;
}

}  // namespace ffb
