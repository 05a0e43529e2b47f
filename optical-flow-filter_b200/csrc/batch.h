// Batched step over many independent flow-filter streams (no reference counterpart).
//
// A Batch owns one pyramidal Filter per stream; streams differ in size, levels and
// parameters.  One step advances every stream by one frame with a number of kernel launches
// that does not grow with the number of streams nor with their parameters:
//
//   ingest      one kernel copies every stream's frame out of one packed device buffer into
//               its level-0 image and builds pyramid levels 1 and 2 from it
//   (deeper pyramid levels, when a stream has more than 3: one launch per depth)
//   levels A    one streaming-kernel launch over every top level and every delta level that
//               reads the previous frame's coarse flow (levels 0..L-3)
//   levels B    one streaming-kernel launch over the levels L-2, which read this frame's
//               unsmoothed top-level flow
//
// A phase launch walks a device table of jobs (one per stream-level), each job a contiguous
// range of blocks running the instantiation of the streaming kernel for its (delta,
// iterations, smoothing) (level_mega.cu).  Levels the streaming kernel does not cover (more
// than 4 iterations or smoothing passes) go to one tile-kernel launch per phase.  The phase
// launches of a step are replayed from a CUDA graph.  Every stream's results are those of the
// same stream filtered alone, whatever the tuning.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <utility>
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
    // phase-A levels of fewer than min_pixels pixels (< 0: kDefaultTileBelow) run the tile
    // kernel, every other level the streaming kernel covers runs it, in bands of `band` rows
    // (<= 0: chosen per step)
    void set_tuning(long min_pixels, int band);
    static constexpr long kDefaultTileBelow = 200000;
    // levels of height x width pixels run in bands of `band` rows (<= 0: no override)
    void set_level_band(int height, int width, int band);

private:
    struct Table;
    void init(int n, const int* heights, const int* widths, const int* levels);
    void build(Table& t);
    bool matches(const Table& t) const;
    void release_table(Table& t);
    bool streamed(const Filter& f, int l) const;
    int band_of(const Level& v, int rule_band) const;

    std::vector<std::unique_ptr<Filter>> f_;
    std::vector<size_t> off_;
    size_t total_ = 0;
    IngestJob* d_ingest_ = nullptr;
    unsigned short* d_ingest_block_ = nullptr;  // job of each ingest block
    int ingest_blocks_ = 0;
    std::unique_ptr<Table> tab_[2];
    cudaStream_t cap_ = nullptr;
    cudaStream_t side_ = nullptr;  // capture branch of phase A's tile launch
    cudaEvent_t fork_ = nullptr, join_ = nullptr;
    int max_levels_ = 0;
    long min_px_ = -1;
    int band_ = 0;
    std::map<std::pair<int, int>, int> level_band_;  // (height, width) -> band rows
    unsigned long long tune_gen_ = 0;
};

}  // namespace ffb
