// Fused per-level kernels (placeholder until the streaming kernels land).
#include "common.cuh"
#include "kernels.h"

namespace ffb {

bool fused_available(bool, int, int, int) { return false; }

cudaError_t launch_fused_level(bool, int, int, const LevelArgs&, cudaStream_t) { return cudaErrorNotSupported; }

}  // namespace ffb
