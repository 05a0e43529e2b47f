// One launch for the streaming level steps of many levels with different (delta, iterations,
// smoothing): the batched step's phase kernel.  Each job (one stream-level) is a contiguous
// range of blocks; a block finds its job by binary search and runs the level's warps through
// the instantiation of level_warp for the job's (delta, N, S), each instantiation a separate
// non-inlined function, so one kernel serves every combination without the launches
// multiplying with the combinations present.  The kernel's register budget is the largest
// instantiation's (the launch bounds cap it); its shared memory is the largest of the jobs'.
#include "level_pipe.cuh"

namespace ffb {
namespace lvl {
namespace {

template <bool DELTA, int N, int S>
__device__ __forceinline__ void warp_fn(const LevelArgs& a, int nwx, int band, int warp) {
    level_warp<DELTA, N, S, uint8_t>(a, nwx, band, warp);
}

// (delta, N, S) -> one call; kind = delta * 16 + (N - 1) * 4 + (S - 1)
template <int K>
__device__ __forceinline__ void call_kind(const LevelArgs& a, int nwx, int band, int warp) {
    warp_fn<(K >> 4) != 0, ((K >> 2) & 3) + 1, (K & 3) + 1>(a, nwx, band, warp);
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32, kBlocksPerSM)
    level_mega_k(const StreamJob* __restrict__ jobs, int n) {
    grid_dep_wait();
    grid_dep_launch();
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].first_block <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const StreamJob& j = jobs[lo];
    const int warp = ((int)blockIdx.x - j.first_block) * kWarpsPerBlock + (threadIdx.x >> 5);
    const int kind = j.kind;
#define FFB_KIND(K) \
    case K: call_kind<K>(j.a, j.nwx, j.band, warp); break;
    switch (kind) {
        FFB_KIND(0) FFB_KIND(1) FFB_KIND(2) FFB_KIND(3) FFB_KIND(4) FFB_KIND(5) FFB_KIND(6) FFB_KIND(7)
        FFB_KIND(8) FFB_KIND(9) FFB_KIND(10) FFB_KIND(11) FFB_KIND(12) FFB_KIND(13) FFB_KIND(14) FFB_KIND(15)
        FFB_KIND(16) FFB_KIND(17) FFB_KIND(18) FFB_KIND(19) FFB_KIND(20) FFB_KIND(21) FFB_KIND(22) FFB_KIND(23)
        FFB_KIND(24) FFB_KIND(25) FFB_KIND(26) FFB_KIND(27) FFB_KIND(28) FFB_KIND(29) FFB_KIND(30) FFB_KIND(31)
        default: break;
    }
#undef FFB_KIND
}

template <bool DELTA, int N, int S>
constexpr int block_smem() {
    return kWarpsPerBlock * WarpMem<DELTA, S>::BYTES;
}

}  // namespace
}  // namespace lvl

int stream_kind(bool delta, int N, int S) { return (delta ? 16 : 0) + (N - 1) * 4 + (S - 1); }

int stream_block_smem(bool delta, int S) {
    if (delta) {
        switch (S) {
            case 1: return lvl::block_smem<true, 1, 1>();
            case 2: return lvl::block_smem<true, 1, 2>();
            case 3: return lvl::block_smem<true, 1, 3>();
            default: return lvl::block_smem<true, 1, 4>();
        }
    }
    switch (S) {
        case 1: return lvl::block_smem<false, 1, 1>();
        case 2: return lvl::block_smem<false, 1, 2>();
        case 3: return lvl::block_smem<false, 1, 3>();
        default: return lvl::block_smem<false, 1, 4>();
    }
}

cudaError_t launch_stream_mega(const StreamJob* jobs, int n, int blocks, int smem, cudaStream_t s) {
    // the kernel's shared-memory limit and carve-out, set once per device
    static std::atomic<unsigned long long> prepared{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(prepared.load() & bit)) {
        cudaError_t e = cudaFuncSetAttribute(lvl::level_mega_k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                             (int)cudaSharedmemCarveoutMaxShared);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(lvl::level_mega_k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     stream_block_smem(true, 4));
        if (e != cudaSuccess) return e;
        prepared.fetch_or(bit);
    }
    return launch_k(lvl::level_mega_k, dim3(blocks), dim3(lvl::kWarpsPerBlock * 32), (size_t)smem, s, jobs, n);
}

}  // namespace ffb
