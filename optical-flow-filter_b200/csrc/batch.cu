// Batched step over many independent streams: job tables, batched kernels and the step
// graph (see batch.h).
#include "batch.h"

#include <algorithm>
#include <atomic>
#include <map>
#include <string>
#include <tuple>

#include "tile_body.cuh"

namespace ffb {

struct TileJob {
    LevelArgs a;
    tile::Geom g;
    int delta;
    int first_block;
};

struct PyrJob {
    const uint8_t* in;
    size_t in_pitch;
    int H, W;  // finer level
    uint8_t* out;
    size_t out_pitch;
    int h, w;  // coarser level
    int bx;    // 32-column block columns
    int first_block;
};

struct IngestJob {
    size_t src;  // byte offset of the frame in the packed buffer (rows of W bytes)
    uint8_t* dst;
    size_t dst_pitch;
    int H, W;
    int rows_per_block;
    int first_block;
};

namespace {

constexpr int kTileThreads = 512;
constexpr size_t kBatchSmemCap = 228 * 1024 / 2 - 1024;  // two tiles resident per SM

// the job whose block range holds block b (jobs sorted by first_block, the first at 0)
template <typename J>
__device__ __forceinline__ int job_of(const J* jobs, int n, int b) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].first_block <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// copies every stream's frame out of the packed buffer into its filter's input image
__global__ void __launch_bounds__(256) ingest_k(const uint8_t* __restrict__ frames, const IngestJob* __restrict__ jobs,
                                                int n) {
    grid_dep_wait();
    grid_dep_launch();
    const IngestJob j = jobs[job_of(jobs, n, blockIdx.x)];
    const int r0 = (blockIdx.x - j.first_block) * j.rows_per_block;
    const int r1 = min(r0 + j.rows_per_block, j.H);
    for (int r = r0; r < r1; ++r) {
        const uint8_t* src = frames + j.src + (size_t)r * j.W;
        uint8_t* dst = j.dst + (size_t)r * j.dst_pitch;
        if ((j.W & 15) == 0 && ((uintptr_t)src & 15) == 0 && ((uintptr_t)dst & 15) == 0) {
            const int n16 = j.W >> 4;
            for (int c = threadIdx.x; c < n16; c += blockDim.x)
                reinterpret_cast<uint4*>(dst)[c] = __ldg(reinterpret_cast<const uint4*>(src) + c);
        } else {
            for (int c = threadIdx.x; c < j.W; c += blockDim.x) dst[c] = __ldg(src + c);
        }
    }
}

// one pyramid depth over every stream that has it: pyramid_down_k per job
__global__ void __launch_bounds__(256) pyramid_batch_k(const PyrJob* __restrict__ jobs, int n) {
    grid_dep_wait();
    grid_dep_launch();
    const PyrJob j = jobs[job_of(jobs, n, blockIdx.x)];
    const int b = blockIdx.x - j.first_block;
    const int x = (b % j.bx) * 32 + (int)(threadIdx.x & 31);
    const int y = (b / j.bx) * 8 + (int)(threadIdx.x >> 5);
    if (x >= j.w || y >= j.h) return;
    pyramid_px(CView<uint8_t>{j.in, j.in_pitch, j.H, j.W}, View<uint8_t>{j.out, j.out_pitch, j.h, j.w}, x, y);
}

// tile-fused level steps of many streams and levels in one launch
__global__ void __launch_bounds__(kTileThreads, 2) tile_batch_k(const TileJob* __restrict__ jobs, int n) {
    extern __shared__ __align__(16) unsigned char sm[];
    const TileJob& j = jobs[job_of(jobs, n, blockIdx.x)];
    const int t = blockIdx.x - j.first_block;
    if (j.delta) tile::tile_body<true, uint8_t>(j.a, j.g, t, sm);
    else tile::tile_body<false, uint8_t>(j.a, j.g, t, sm);
}

// tile shape of one level inside a batch: the least halo overhead whose shared memory
// lets two tiles share an SM (the batch supplies the parallelism, not the tile count)
tile::Geom batch_geom(bool delta, int N, int S, int W, int H, size_t* smem) {
    const int R = N + 2 * S;
    tile::Geom best{};
    double best_eff = -1;
    const int tws[] = {32, 48, 64, 96, 128};
    const int ths[] = {8, 12, 16, 20, 24, 32, 40, 48, 64};
    for (int tw0 : tws) {
        for (int th0 : ths) {
            const int tw = std::min(tw0, W), th = std::min(th0, H);
            const tile::Layout L = tile::layout(delta, N, S, tw, th);
            if (L.total > kBatchSmemCap) continue;
            const long tiles = (long)((W + tw - 1) / tw) * ((H + th - 1) / th);
            // useful pixels per unit of tile work, with whole tiles counted
            const double eff = (double)W * H / ((double)tiles * (tw + 2 * R) * (th + 2 * R));
            if (eff > best_eff) {
                best_eff = eff;
                best.TW = tw;
                best.TH = th;
                *smem = L.total;
            }
        }
    }
    if (best.TW == 0) throw Error(FF_ERR_UNSUPPORTED, "batch: a level's tile does not fit in shared memory");
    best.N = N;
    best.S = S;
    best.R = R;
    best.SW = best.TW + 2 * R;
    best.SH = best.TH + 2 * R;
    best.tiles_x = (W + best.TW - 1) / best.TW;
    const tile::Layout L = tile::layout(delta, N, S, best.TW, best.TH);
    best.offB = (int)L.a;
    best.offC = (int)(L.a + L.b);
    return best;
}

template <typename T>
T* to_device(const std::vector<T>& v) {
    if (v.empty()) return nullptr;
    T* d = nullptr;
    check_cuda(device_malloc((void**)&d, v.size() * sizeof(T)), "batch tables");
    const cudaError_t e = cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) cudaFree(d);
    check_cuda(e, "batch tables");
    return d;
}

}  // namespace

struct Batch::Table {
    std::vector<int> parity;
    std::vector<unsigned long long> gen;
    unsigned long long tune_gen = 0;
    PyrJob* d_pyr = nullptr;
    TileJob* d_tile = nullptr;
    StreamJob* d_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
};

// the streaming-kernel launches of a step: (phase, delta, N, S) -> its jobs
using StreamGroups = std::map<std::tuple<int, int, int, int>, std::vector<StreamJob>>;

Batch::Batch(int n, const int* heights, const int* widths, const int* levels) {
    if (n <= 0) throw Error(FF_ERR_INVALID_ARGUMENT, "batch: stream count must be positive");
    if (!heights || !widths || !levels) throw Error(FF_ERR_INVALID_ARGUMENT, "batch: null shape arrays");
    try {
        init(n, heights, widths, levels);
    } catch (...) {
        // a failed constructor runs no destructor: release what init made (the streams'
        // filters go with f_)
        if (d_ingest_) cudaFree(d_ingest_);
        if (cap_) cudaStreamDestroy(cap_);
        throw;
    }
}

void Batch::init(int n, const int* heights, const int* widths, const int* levels) {
    check_cuda(cudaStreamCreateWithFlags(&cap_, cudaStreamNonBlocking), "cudaStreamCreate");
    std::vector<IngestJob> ing;
    int blocks = 0;
    for (int i = 0; i < n; ++i) {
        f_.emplace_back(new Filter(Kind::Pyramidal, heights[i], widths[i], levels[i], 1, true));
        max_levels_ = std::max(max_levels_, levels[i]);
        off_.push_back(total_);
        total_ += ((size_t)heights[i] * widths[i] + 255) / 256 * 256;
        const Level& v = f_.back()->level(0);
        IngestJob j{};
        j.src = off_.back();
        j.dst = (uint8_t*)v.img;
        j.dst_pitch = v.img_pitch;
        j.H = v.H;
        j.W = v.W;
        j.rows_per_block = std::max(1, 16384 / v.W);
        j.first_block = blocks;
        blocks += (v.H + j.rows_per_block - 1) / j.rows_per_block;
        ing.push_back(j);
    }
    d_ingest_ = to_device(ing);
    ingest_blocks_ = blocks;
    for (auto& t : tab_) t.reset(new Table);
    check_cuda(cudaFuncSetAttribute(tile_batch_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBatchSmemCap),
               "cudaFuncSetAttribute");
    // full shared carve-out, so the L-2 launch's blocks can share SMs with the top launch's
    check_cuda(cudaFuncSetAttribute(tile_batch_k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    (int)cudaSharedmemCarveoutMaxShared),
               "cudaFuncSetAttribute");
}

void Batch::release_table(Table& t) {
    if (t.graph) cudaGraphExecDestroy(t.graph);
    if (t.d_pyr) cudaFree(t.d_pyr);
    if (t.d_tile) cudaFree(t.d_tile);
    if (t.d_stream) cudaFree(t.d_stream);
    t = Table{};
}

Batch::~Batch() {
    // the step graphs read the job tables: wait for every stream's last step first
    for (auto& f : f_) {
        try {
            f->wait_done();
        } catch (...) {
        }
    }
    for (auto& t : tab_)
        if (t) release_table(*t);
    if (d_ingest_) cudaFree(d_ingest_);
    if (cap_) cudaStreamDestroy(cap_);
    for (cudaStream_t q : side_) cudaStreamDestroy(q);
    for (cudaEvent_t e : ev_) cudaEventDestroy(e);
}

Filter& Batch::stream(int i) {
    if (i < 0 || i >= size()) throw Error(FF_ERR_OUT_OF_RANGE, "batch stream index out of bounds: " + std::to_string(i));
    return *f_[i];
}

size_t Batch::frame_offset(int i) const {
    if (i < 0 || i >= (int)off_.size())
        throw Error(FF_ERR_OUT_OF_RANGE, "batch stream index out of bounds: " + std::to_string(i));
    return off_[i];
}

bool Batch::streamed(const Filter& f, int l) const {
    const Level& v = f.level(l);
    const long min_px = min_px_ >= 0 ? min_px_ : Filter::kFusedMinPixels;
    return v.item == 1 && (long)v.H * v.W >= min_px && f.streaming_ok(l);
}

void Batch::set_tuning(long min_pixels, int band) {
    min_px_ = min_pixels < 0 ? -1 : min_pixels;
    band_ = band > 0 ? band : 0;
    ++tune_gen_;
}

int Batch::launches_per_step() const {
    bool tile_a = false, tile_b = false;
    std::map<std::tuple<int, int, int, int>, int> groups;
    for (auto& f : f_) {
        const int L = f->levels();
        for (int l = 0; l < L; ++l) {
            const Level& v = f->level(l);
            const int late = L >= 2 && l == L - 2;
            if (streamed(*f, l)) groups[{late, v.delta, v.iters, v.smooth}] = 1;
            else (late ? tile_b : tile_a) = true;
        }
    }
    return 1 + (max_levels_ - 1) + (int)tile_a + (int)tile_b + (int)groups.size();
}

bool Batch::matches(const Table& t) const {
    if (!t.graph || t.tune_gen != tune_gen_) return false;
    for (size_t i = 0; i < f_.size(); ++i)
        if (t.parity[i] != f_[i]->parity() || t.gen[i] != f_[i]->config_generation()) return false;
    return true;
}

void Batch::build(Table& t) {
    release_table(t);
    std::vector<PyrJob> pyr;
    std::vector<int> pyr_first(max_levels_, 0), pyr_count(max_levels_, 0), pyr_blocks(max_levels_, 0);
    for (int d = 1; d < max_levels_; ++d) {
        pyr_first[d] = (int)pyr.size();
        int blocks = 0;
        for (auto& f : f_) {
            if (f->levels() <= d) continue;
            const Level& fine = f->level(d - 1);
            const Level& coarse = f->level(d);
            PyrJob j{};
            j.in = (const uint8_t*)fine.img;
            j.in_pitch = fine.img_pitch;
            j.H = fine.H;
            j.W = fine.W;
            j.out = (uint8_t*)coarse.img;
            j.out_pitch = coarse.img_pitch;
            j.h = coarse.H;
            j.w = coarse.W;
            j.bx = (coarse.W + 31) / 32;
            j.first_block = blocks;
            blocks += j.bx * ((coarse.H + 7) / 8);
            pyr.push_back(j);
        }
        pyr_count[d] = (int)pyr.size() - pyr_first[d];
        pyr_blocks[d] = blocks;
    }
    // phase A: top levels and levels 0..L-3; phase B: levels L-2.  Large levels go to the
    // streaming launches of their phase, the others to the phase's tile launch.
    std::vector<TileJob> ja, jb;
    int blocks_a = 0, blocks_b = 0;
    size_t smem_a = 0, smem_b = 0;
    StreamGroups groups;
    std::map<std::tuple<int, int, int, int>, int> group_blocks;
    // Band rows: every band recomputes (2S + N)-row lead and tail windows, so long bands
    // waste less, while the streaming branches need enough warps to balance over the SMs.
    // One band for the step: the longest of 256..32 rows that gives phase A's streaming
    // levels (phase B's when A has none) kWaves waves of resident warps (fitted to the
    // 64-stream and single-size 640x480 .. 1920x1080 mixes on B200).
    constexpr int kBands[] = {256, 128, 64, 32};
    constexpr double kWaves = 3.5;
    int band = band_;
    if (band <= 0) {
        const double resident = (double)fused_resident_warps();
        auto warps_at = [&](int phase, int b) {
            long warps = 0;
            for (auto& f : f_) {
                const int L = f->levels();
                for (int l = 0; l < L; ++l) {
                    if ((L >= 2 && l == L - 2) != (phase == 1) || !streamed(*f, l)) continue;
                    const Level& v = f->level(l);
                    int nwx = 0, nby = 0;
                    fused_warp_grid(v.iters, v.smooth, v.W, v.H, b, &nwx, &nby);
                    warps += (long)nwx * nby;
                }
            }
            return warps;
        };
        const int phase = warps_at(0, 8) > 0 ? 0 : 1;
        band = 32;
        for (int b : kBands)
            if (warps_at(phase, b) >= kWaves * resident) {
                band = b;
                break;
            }
    }
    // which launch of phase A holds each stream's top level (a group key, or the tile
    // launch), and the streams of each phase-B launch: a phase-B launch waits only for the
    // phase-A launches holding its streams' top levels
    std::vector<std::tuple<int, int, int, int>> top_key(f_.size());
    std::vector<char> top_tiled(f_.size(), 0);
    std::map<std::tuple<int, int, int, int>, std::vector<int>> group_streams;
    std::vector<int> jb_streams;
    for (size_t si = 0; si < f_.size(); ++si) {
        Filter* f = f_[si].get();
        const int L = f->levels();
        for (int l = 0; l < L; ++l) {
            const Level& v = f->level(l);
            const std::tuple<int, int, int, int> key{L >= 2 && l == L - 2, v.delta, v.iters, v.smooth};
            if (l == L - 1) {
                top_key[si] = key;
                top_tiled[si] = !streamed(*f, l);
            }
            if (streamed(*f, l)) {
                group_streams[key].push_back((int)si);
                StreamJob j{};
                j.a = f->level_args(l);
                j.band = std::min(std::max(band, 8), v.H);
                int& blocks = group_blocks[key];
                j.first_block = blocks;
                blocks += fused_warp_grid(v.iters, v.smooth, v.W, v.H, j.band, &j.nwx, &j.nby);
                groups[key].push_back(j);
                continue;
            }
            TileJob j{};
            j.a = f->level_args(l);
            j.delta = v.delta ? 1 : 0;
            size_t smem = 0;
            j.g = batch_geom(v.delta, v.iters, v.smooth, v.W, v.H, &smem);
            const int tiles = j.g.tiles_x * ((v.H + j.g.TH - 1) / j.g.TH);
            const bool late = L >= 2 && l == L - 2;
            // the tile launch of phase B follows that of phase A on one stream: its jobs wait
            // for it only before their update, and A lets B's blocks start at once
            j.a.pdl_late_wait = late ? 1 : 0;
            j.a.pdl_early_trigger = late ? 0 : 1;
            if (late) {
                jb_streams.push_back((int)si);
                j.first_block = blocks_b;
                blocks_b += tiles;
                smem_b = std::max(smem_b, smem);
                jb.push_back(j);
            } else {
                j.first_block = blocks_a;
                blocks_a += tiles;
                smem_a = std::max(smem_a, smem);
                ja.push_back(j);
            }
        }
    }
    std::vector<TileJob> all(ja);
    all.insert(all.end(), jb.begin(), jb.end());
    std::vector<StreamJob> sall;
    std::vector<size_t> sfirst;
    for (auto& kv : groups) {
        sfirst.push_back(sall.size());
        sall.insert(sall.end(), kv.second.begin(), kv.second.end());
    }
    t.d_pyr = to_device(pyr);
    t.d_tile = to_device(all);
    t.d_stream = to_device(sall);
    t.parity.clear();
    t.gen.clear();
    for (auto& f : f_) {
        t.parity.push_back(f->parity());
        t.gen.push_back(f->config_generation());
    }
    t.tune_gen = tune_gen_;
    const int ngroups = (int)groups.size();
    while ((int)side_.size() < ngroups) {
        cudaStream_t q = nullptr;
        check_cuda(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking), "cudaStreamCreate");
        side_.push_back(q);
    }
    while ((int)ev_.size() < 2 + ngroups) {
        cudaEvent_t ev = nullptr;
        check_cuda(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
        ev_.push_back(ev);
    }
    // phase-A launches each phase-B launch waits for (-1: the tile launch)
    std::map<std::tuple<int, int, int, int>, int> gindex;
    for (auto& kv : groups) {
        const int i = (int)gindex.size();
        gindex[kv.first] = i;
    }
    auto deps_of = [&](const std::vector<int>& streams) {
        std::vector<int> d;
        for (int si : streams) {
            const int k = top_tiled[si] ? -1 : gindex.at(top_key[si]);
            if (std::find(d.begin(), d.end(), k) == d.end()) d.push_back(k);
        }
        return d;
    };
    // capture: pyramid depths; phase A: the tile launch on the capture stream and each
    // streaming group on a branch forked after the pyramid; phase B: the tile launch on the
    // capture stream after phase A's tile launch, and each streaming group on a branch; a
    // phase-B launch waits for the phase-A launches holding its streams' top levels; join
    cudaGraph_t g = nullptr;
    check_cuda(cudaStreamBeginCapture(cap_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    for (int d = 1; d < max_levels_; ++d)
        if (pyr_count[d] > 0)
            ok(launch_k(pyramid_batch_k, dim3(pyr_blocks[d]), dim3(256), 0, cap_,
                        (const PyrJob*)(t.d_pyr + pyr_first[d]), pyr_count[d]));
    ok(cudaEventRecord(ev_[0], cap_));
    auto branch = [&](int i, const std::tuple<int, int, int, int>& key, const std::vector<StreamJob>& jobs) {
        ok(launch_fused_batch(std::get<1>(key) != 0, std::get<2>(key), std::get<3>(key), t.d_stream + sfirst[i],
                              (int)jobs.size(), group_blocks.at(key), side_[i]));
        ok(cudaEventRecord(ev_[2 + i], side_[i]));
    };
    for (auto& kv : groups) {
        const int i = gindex[kv.first];
        if (std::get<0>(kv.first) != 0) continue;
        ok(cudaStreamWaitEvent(side_[i], ev_[0], 0));
        branch(i, kv.first, kv.second);
    }
    if (!ja.empty())
        ok(launch_k(tile_batch_k, dim3(blocks_a), dim3(kTileThreads), smem_a, cap_, (const TileJob*)t.d_tile,
                    (int)ja.size()));
    ok(cudaEventRecord(ev_[1], cap_));  // phase A's tile launch (or the pyramid) done
    for (auto& kv : groups) {
        const int i = gindex[kv.first];
        if (std::get<0>(kv.first) != 1) continue;
        ok(cudaStreamWaitEvent(side_[i], ev_[1], 0));
        for (int k : deps_of(group_streams.at(kv.first)))
            if (k >= 0) ok(cudaStreamWaitEvent(side_[i], ev_[2 + k], 0));
        branch(i, kv.first, kv.second);
    }
    if (!jb.empty()) {
        for (int k : deps_of(jb_streams))
            if (k >= 0) ok(cudaStreamWaitEvent(cap_, ev_[2 + k], 0));
        ok(launch_k(tile_batch_k, dim3(blocks_b), dim3(kTileThreads), smem_b, cap_,
                    (const TileJob*)(t.d_tile + ja.size()), (int)jb.size()));
    }
    for (int i = 0; i < ngroups; ++i) ok(cudaStreamWaitEvent(cap_, ev_[2 + i], 0));
    cudaError_t ec = cudaStreamEndCapture(cap_, &g);
    check_cuda(e, "batch capture");
    check_cuda(ec, "cudaStreamEndCapture");
    e = cudaGraphInstantiateWithFlags(&t.graph, g, 0);
    cudaGraphDestroy(g);
    check_cuda(e, "cudaGraphInstantiate");
    log_message(FF_LOG_INFO, "batch: step graph built for " + std::to_string(f_.size()) + " streams, " +
                                 std::to_string(launches_per_step()) + " launches, streaming band " +
                                 std::to_string(band) + " rows");
}

void Batch::step(const void* frames, cudaStream_t s) {
    if (!frames) throw Error(FF_ERR_INVALID_ARGUMENT, "batch: null frame buffer");
    if ((uintptr_t)frames % 16) throw Error(FF_ERR_INVALID_ARGUMENT, "batch: the frame buffer must be 16-byte aligned");
    for (auto& f : f_) f->batch_begin(s);
    check_cuda(launch_k(ingest_k, dim3(ingest_blocks_), dim3(256), 0, s, (const uint8_t*)frames,
                        (const IngestJob*)d_ingest_, size()),
               "batch ingest");
    bool first = false;
    for (auto& f : f_) first |= f->any_first();
    if (first) {
        // frame 0 seeds every level's old image from this frame (first-frame rule of the
        // reference); each stream takes its own path once, then joins the batch
        for (auto& f : f_) f->compute_async(s);
        return;
    }
    Table* t = nullptr;
    for (auto& c : tab_)
        if (matches(*c)) t = c.get();
    if (!t) {
        t = tab_[f_[0]->parity()].get();
        check_cuda(cudaStreamSynchronize(s), "batch rebuild");  // the old tables may still be in use
        build(*t);
    }
    check_cuda(cudaGraphLaunch(t->graph, s), "cudaGraphLaunch");
    for (auto& f : f_) f->batch_end(s);
}

}  // namespace ffb
