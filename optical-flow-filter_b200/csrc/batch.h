// Batched step over many independent flow-filter streams (no reference counterpart).
//
// A Batch owns one pyramidal Filter per stream; streams differ in size, levels and
// parameters.  One step advances every stream by one frame with a number of kernel launches
// that does not grow with the number of streams:
//
//   ingest      one kernel copies every stream's frame out of one packed device buffer
//   pyramid     one launch per pyramid depth, over all streams that have that level
//   levels A    every top level and every delta level that reads the previous frame's
//               coarse flow (levels 0..L-3)
//   levels B    the levels L-2, which read this frame's unsmoothed top-level flow
//
// In each phase the small levels go to one tile-fused launch, and the large ones (as
// large as the levels a single filter streams) to one streaming-kernel launch per
// (delta, propagation iterations, smoothing iterations) group; the launches of a phase
// are branches of the step graph that run side by side.  Each batched launch walks a
// device table of jobs (one per stream-level), each job a contiguous range of CTAs.  The
// pyramid and level launches of a step are replayed from a CUDA graph.  Every stream's
// results are those of the same stream filtered alone.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "filter.h"

namespace ffb {

struct TileJob;
struct PyrJob;
struct IngestJob;

class Batch {
public:
    Batch(int n, const int* heights, const int* widths, const int* levels);
    ~Batch();
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;

    int size() const { return (int)f_.size(); }
    Filter& stream(int i);
    // byte offset of stream i's frame (rows of width bytes, no padding) in a packed buffer
    size_t frame_offset(int i) const;
    size_t frame_bytes() const { return total_; }
    // kernel launches of one batched step (ingest included)
    int launches_per_step() const;
    // advance every stream by one frame read from `frames` (frame_bytes() bytes on the device)
    void step(const void* frames, cudaStream_t s);
    // levels of at least min_pixels pixels (< 0: the single filter's threshold) run the
    // streaming kernel in bands of `band` rows (<= 0: chosen per phase); the others the
    // tile kernel
    void set_tuning(long min_pixels, int band);

private:
    struct Table;
    void init(int n, const int* heights, const int* widths, const int* levels);
    void build(Table& t);
    bool matches(const Table& t) const;
    void release_table(Table& t);
    bool streamed(const Filter& f, int l) const;

    std::vector<std::unique_ptr<Filter>> f_;
    std::vector<size_t> off_;
    size_t total_ = 0;
    IngestJob* d_ingest_ = nullptr;
    int ingest_blocks_ = 0;
    std::unique_ptr<Table> tab_[2];
    cudaStream_t cap_ = nullptr;
    int max_levels_ = 0;
    long min_px_ = -1;
    int band_ = 0;
    unsigned long long tune_gen_ = 0;
    std::vector<cudaStream_t> side_;  // capture branches of the streaming launches
    std::vector<cudaEvent_t> ev_;     // fork and join events of those branches
};

}  // namespace ffb
