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

// one stream's frame: copied into its level-0 image, with levels 1 and 2 of its pyramid
// built from it in the same blocks (tiles of P2X x P2Y level-1 pixels; a one-level stream's
// blocks copy tiles of 2 P2X x 2 P2Y level-0 pixels)
struct IngestJob {
    size_t src;  // byte offset of the frame in the packed buffer (rows of W bytes)
    uint8_t* dst;
    size_t dst_pitch;
    int H, W;
    uint8_t* out1;
    size_t out1_pitch;
    int h1, w1;
    uint8_t* out2;
    size_t out2_pitch;
    int h2, w2;
    int levels;  // levels this launch fills: 1, 2 or 3
    int tiles_x, tiles_y;
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

constexpr int P2X = 64, P2Y = 16;  // level-1 tile of the ingest launch (blocks of 32 x 8 threads)

// Every stream's frame out of the packed buffer into its level-0 image, and levels 1 and 2
// of its pyramid from the frame.  A block stages the level-0 pixels under its level-1 tile
// and the one-pixel level-1 ring around it (at clamped coordinates) in shared memory with
// one batch of loads, copies its part of level 0 out of it, computes the level-1 tile plus
// ring from it (pyramid_px, common.cuh: the values of a pyramid_down_k pass), and the
// level-2 pixels under the tile from the ring.  The last tile row and column of a stream also
// copy the level-0 remainder (odd sizes).
// staged level-0 rows and columns: the tile's 2 P2Y x 2 P2X pixels, 3 before and 2 after in
// each direction, the columns from a 4-byte boundary (4 before)
constexpr int S0Y = 2 * P2Y + 5, S0X = 2 * P2X + 8;
// block_job[b]: the job of block b (a table, so a block finds its job in one load)
__global__ void __launch_bounds__(256, 6) ingest_pyr_k(const uint8_t* __restrict__ frames,
                                                       const IngestJob* __restrict__ jobs,
                                                       const unsigned short* __restrict__ block_job) {
    __shared__ __align__(16) uint8_t s0[S0Y][S0X];
    __shared__ uint8_t ring[P2Y + 2][P2X + 2];
    grid_dep_wait();
    grid_dep_launch();
    const IngestJob& j = jobs[block_job[blockIdx.x]];
    const int b = blockIdx.x - j.first_block;
    const int tx = b % j.tiles_x, ty = b / j.tiles_x;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const uint8_t* src = frames + j.src;
    const int W = j.W, H = j.H;
    const bool words = (W & 3) == 0 && (j.dst_pitch & 3) == 0;  // rows are 4-byte aligned
    if (j.levels < 2) {  // block-uniform: a one-level stream's tile is a plain copy
        const int x0 = tx * 2 * P2X, y0 = ty * 2 * P2Y;
        const int xe = tx == j.tiles_x - 1 ? W : min(x0 + 2 * P2X, W);
        const int ye = ty == j.tiles_y - 1 ? H : min(y0 + 2 * P2Y, H);
        const int wv = xe - x0, rows = ye - y0;
        if (words) {
            const int wq = wv >> 2;
            for (int k = tid; k < rows * wq; k += 256) {
                const int r = k / wq, c = k - r * wq;
                reinterpret_cast<uint32_t*>(j.dst + (size_t)(y0 + r) * j.dst_pitch + x0)[c] =
                    __ldg(reinterpret_cast<const uint32_t*>(src + (size_t)(y0 + r) * W + x0) + c);
            }
        } else {
            for (int k = tid; k < rows * wv; k += 256) {
                const int r = k / wv, c = k - r * wv;
                j.dst[(size_t)(y0 + r) * j.dst_pitch + x0 + c] = __ldg(src + (size_t)(y0 + r) * W + x0 + c);
            }
        }
        return;
    }
    const int x1 = tx * P2X, y1 = ty * P2Y;
    const int X0 = 2 * x1 - 4, Y0 = 2 * y1 - 3;  // staged level-0 origin (unclamped)
    if (words) {
        constexpr int WQ = S0X / 4, NS = (S0Y * WQ + 255) / 256;
        uint32_t v[NS];
#pragma unroll
        for (int u = 0; u < NS; ++u) {
            const int e = tid + 256 * u, r = e / WQ, c = e - r * WQ;
            if (e < S0Y * WQ) {
                const uint8_t* row = src + (size_t)min(max(Y0 + r, 0), H - 1) * W;
                const int x = X0 + 4 * c;
                if (x >= 0 && x + 3 < W) {
                    v[u] = __ldg(reinterpret_cast<const uint32_t*>(row + x));
                } else {  // a word beyond an edge: its clamped bytes
                    uint32_t w = 0;
#pragma unroll
                    for (int q = 0; q < 4; ++q) w |= (uint32_t)__ldg(row + min(max(x + q, 0), W - 1)) << (8 * q);
                    v[u] = w;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < NS; ++u) {
            const int e = tid + 256 * u, r = e / WQ, c = e - r * WQ;
            if (e < S0Y * WQ) reinterpret_cast<uint32_t*>(s0[r])[c] = v[u];
        }
    } else {
        constexpr int NS = (S0Y * S0X + 255) / 256;
        uint8_t v[NS];
#pragma unroll
        for (int u = 0; u < NS; ++u) {
            const int e = tid + 256 * u, r = e / S0X, c = e - r * S0X;
            if (e < S0Y * S0X) v[u] = __ldg(src + (size_t)min(max(Y0 + r, 0), H - 1) * W + min(max(X0 + c, 0), W - 1));
        }
#pragma unroll
        for (int u = 0; u < NS; ++u) {
            const int e = tid + 256 * u, r = e / S0X, c = e - r * S0X;
            if (e < S0Y * S0X) s0[r][c] = v[u];
        }
    }
    __syncthreads();
    {
        const int x0 = 2 * x1, y0 = 2 * y1;
        const int xe = tx == j.tiles_x - 1 ? W : min(x0 + 2 * P2X, W);
        const int ye = ty == j.tiles_y - 1 ? H : min(y0 + 2 * P2Y, H);
        const int wv = xe - x0, rows = ye - y0;
        if (words) {  // x0 - X0 = 4: word-aligned in s0 as in the image row
            const int wq = wv >> 2;
            for (int k = tid; k < rows * wq; k += 256) {
                const int r = k / wq, c = k - r * wq;
                reinterpret_cast<uint32_t*>(j.dst + (size_t)(y0 + r) * j.dst_pitch + x0)[c] =
                    reinterpret_cast<const uint32_t*>(s0[y0 + r - Y0] + 4)[c];
            }
        } else {
            for (int k = tid; k < rows * wv; k += 256) {
                const int r = k / wv, c = k - r * wv;
                j.dst[(size_t)(y0 + r) * j.dst_pitch + x0 + c] = s0[y0 + r - Y0][x0 + c - X0];
            }
        }
    }
    for (int k = tid; k < (P2X + 2) * (P2Y + 2); k += 256) {
        const int i = k % (P2X + 2), r = k / (P2X + 2);
        const int ux = x1 - 1 + i, uy = y1 - 1 + r;  // unclamped level-1 position
        const int cx = min(max(ux, 0), j.w1 - 1), cy = min(max(uy, 0), j.h1 - 1);
        // pyramid_val at (cx, cy): rows 2cy-1..2cy+1, columns 2cx-1..2cx+1 of level 0, clamped
        float xs[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const uint8_t* row = s0[2 * cy - 1 + q - Y0] + (2 * cx - 1 - X0);
            const float sv = down3(u8_to_unit(row[0]), u8_to_unit(row[1]), u8_to_unit(row[2]));
            xs[q] = u8_to_unit(quantize_u8(sv));
        }
        const uint8_t val = quantize_u8(down3(xs[0], xs[1], xs[2]));
        ring[r][i] = val;
        if (ux == cx && uy == cy && ux >= x1 && ux < x1 + P2X && uy >= y1 && uy < y1 + P2Y)
            j.out1[(size_t)uy * j.out1_pitch + ux] = val;
    }
    if (j.levels < 3) return;  // block-uniform
    __syncthreads();
    const int x2 = x1 / 2 + threadIdx.x, y2 = y1 / 2 + threadIdx.y;
    if (x2 >= j.w2 || y2 >= j.h2) return;
    // pyramid_val over level 1, whose clamped reads the ring holds
    float xs[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const int r = 2 * y2 - 1 + q - (y1 - 1);
        const int c = 2 * x2 - 1 - (x1 - 1);
        const float sv = down3(u8_to_unit(ring[r][c]), u8_to_unit(ring[r][c + 1]), u8_to_unit(ring[r][c + 2]));
        xs[q] = u8_to_unit(quantize_u8(sv));
    }
    j.out2[(size_t)y2 * j.out2_pitch + x2] = quantize_u8(down3(xs[0], xs[1], xs[2]));
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
    int launches = 0;  // kernel launches of the graph
};

Batch::Batch(int n, const int* heights, const int* widths, const int* levels) {
    if (n <= 0) throw Error(FF_ERR_INVALID_ARGUMENT, "batch: stream count must be positive");
    if (!heights || !widths || !levels) throw Error(FF_ERR_INVALID_ARGUMENT, "batch: null shape arrays");
    try {
        init(n, heights, widths, levels);
    } catch (...) {
        // a failed constructor runs no destructor: release what init made (the streams'
        // filters go with f_)
        if (d_ingest_) cudaFree(d_ingest_);
        if (d_ingest_block_) cudaFree(d_ingest_block_);
        if (cap_) cudaStreamDestroy(cap_);
        if (side_) cudaStreamDestroy(side_);
        if (fork_) cudaEventDestroy(fork_);
        if (join_) cudaEventDestroy(join_);
        throw;
    }
}

void Batch::init(int n, const int* heights, const int* widths, const int* levels) {
    check_cuda(cudaStreamCreateWithFlags(&cap_, cudaStreamNonBlocking), "cudaStreamCreate");
    check_cuda(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking), "cudaStreamCreate");
    check_cuda(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "cudaEventCreate");
    check_cuda(cudaEventCreateWithFlags(&join_, cudaEventDisableTiming), "cudaEventCreate");
    std::vector<IngestJob> ing;
    int blocks = 0;
    for (int i = 0; i < n; ++i) {
        f_.emplace_back(new Filter(Kind::Pyramidal, heights[i], widths[i], levels[i], 1, true));
        Filter& f = *f_.back();
        max_levels_ = std::max(max_levels_, levels[i]);
        off_.push_back(total_);
        total_ += ((size_t)heights[i] * widths[i] + 255) / 256 * 256;
        const Level& v = f.level(0);
        IngestJob j{};
        j.src = off_.back();
        j.dst = (uint8_t*)v.img;
        j.dst_pitch = v.img_pitch;
        j.H = v.H;
        j.W = v.W;
        j.levels = std::min(f.levels(), 3);
        if (j.levels >= 2) {
            const Level& v1 = f.level(1);
            j.out1 = (uint8_t*)v1.img;
            j.out1_pitch = v1.img_pitch;
            j.h1 = v1.H;
            j.w1 = v1.W;
            j.tiles_x = (v1.W + P2X - 1) / P2X;
            j.tiles_y = (v1.H + P2Y - 1) / P2Y;
        } else {
            j.tiles_x = (v.W + 2 * P2X - 1) / (2 * P2X);
            j.tiles_y = (v.H + 2 * P2Y - 1) / (2 * P2Y);
        }
        if (j.levels >= 3) {
            const Level& v2 = f.level(2);
            j.out2 = (uint8_t*)v2.img;
            j.out2_pitch = v2.img_pitch;
            j.h2 = v2.H;
            j.w2 = v2.W;
        }
        j.first_block = blocks;
        blocks += j.tiles_x * j.tiles_y;
        ing.push_back(j);
    }
    d_ingest_ = to_device(ing);
    ingest_blocks_ = blocks;
    if (n > 65535) throw Error(FF_ERR_UNSUPPORTED, "batch: at most 65535 streams");
    std::vector<unsigned short> block_job(blocks);
    for (int i = 0; i < n; ++i)
        for (int b = ing[i].first_block; b < ing[i].first_block + ing[i].tiles_x * ing[i].tiles_y; ++b)
            block_job[b] = (unsigned short)i;
    d_ingest_block_ = to_device(block_job);
    for (auto& t : tab_) t.reset(new Table);
    check_cuda(cudaFuncSetAttribute(tile_batch_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBatchSmemCap),
               "cudaFuncSetAttribute");
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
    if (d_ingest_block_) cudaFree(d_ingest_block_);
    if (cap_) cudaStreamDestroy(cap_);
    if (side_) cudaStreamDestroy(side_);
    if (fork_) cudaEventDestroy(fork_);
    if (join_) cudaEventDestroy(join_);
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

// Phase-B levels (L-2) always stream when the kernel covers them, so only phase A has a tile
// launch unless a phase-B level has more iterations or smoothing passes than the kernel's 4
bool Batch::streamed(const Filter& f, int l) const {
    const Level& v = f.level(l);
    const int L = f.levels();
    const bool late = L >= 2 && l == L - 2;
    const long min_px = min_px_ >= 0 ? min_px_ : kDefaultTileBelow;
    return v.item == 1 && (late || (long)v.H * v.W >= min_px) && f.streaming_ok(l);
}

void Batch::set_tuning(long min_pixels, int band) {
    min_px_ = min_pixels < 0 ? -1 : min_pixels;
    band_ = band > 0 ? band : 0;
    ++tune_gen_;
}

void Batch::set_level_band(int height, int width, int band) {
    if (band > 0) level_band_[{height, width}] = band;
    else level_band_.erase({height, width});
    ++tune_gen_;
}

int Batch::launches_per_step() const {
    bool stream_a = false, stream_b = false, tile_a = false, tile_b = false;
    for (auto& f : f_) {
        const int L = f->levels();
        for (int l = 0; l < L; ++l) {
            const bool late = L >= 2 && l == L - 2;
            (streamed(*f, l) ? (late ? stream_b : stream_a) : (late ? tile_b : tile_a)) = true;
        }
    }
    // the ingest and pyramid launch, one per pyramid depth beyond 2, one per phase and kernel
    return 1 + std::max(max_levels_ - 3, 0) + (int)stream_a + (int)stream_b + (int)tile_a + (int)tile_b;
}

bool Batch::matches(const Table& t) const {
    if (!t.graph || t.tune_gen != tune_gen_) return false;
    for (size_t i = 0; i < f_.size(); ++i)
        if (t.parity[i] != f_[i]->parity() || t.gen[i] != f_[i]->config_generation()) return false;
    return true;
}

// band rows of a streamed level: its size's override, the batch's band, or the default rule
int Batch::band_of(const Level& v, int rule_band) const {
    const auto it = level_band_.find({v.H, v.W});
    const int b = it != level_band_.end() ? it->second : (band_ > 0 ? band_ : rule_band);
    return std::min(std::max(b, 8), v.H);
}

void Batch::build(Table& t) {
    release_table(t);
    // pyramid depths beyond 2 (levels 1 and 2 come with the ingest launch): one launch each
    std::vector<PyrJob> pyr;
    std::vector<int> pyr_first(max_levels_, 0), pyr_count(max_levels_, 0), pyr_blocks(max_levels_, 0);
    for (int d = 3; d < max_levels_; ++d) {
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
    // Default band: one for the step, the longest of 256..32 rows that gives phase A's
    // streamed levels kWaves waves of resident warps (every band recomputes (2S + N)-row
    // lead and tail windows, so long bands waste less, while the phase needs enough warps to
    // balance over the SMs).  Sizes with an override (set_level_band) keep theirs.
    constexpr int kBands[] = {256, 128, 64, 32};
    constexpr double kWaves = 3.5;
    int rule = 32;
    {
        const double resident = (double)fused_resident_warps();
        auto warps_at = [&](int phase, int b) {
            long warps = 0;
            for (auto& f : f_) {
                const int L = f->levels();
                for (int l = 0; l < L; ++l) {
                    if ((L >= 2 && l == L - 2) != (phase == 1) || !streamed(*f, l)) continue;
                    const Level& v = f->level(l);
                    int nwx = 0, nby = 0;
                    fused_warp_grid(v.iters, v.smooth, v.W, v.H, std::min(std::max(b, 8), v.H), &nwx, &nby);
                    warps += (long)nwx * nby;
                }
            }
            return warps;
        };
        const int phase = warps_at(0, 8) > 0 ? 0 : 1;
        for (int b : kBands)
            if (warps_at(phase, b) >= kWaves * resident) {
                rule = b;
                break;
            }
    }
    // phase A: top levels and levels 0..L-3 (they read the previous frame's coarse flow);
    // phase B: levels L-2 (they read this frame's top-level flow).  Streamed levels go to the
    // phase's streaming launch, the others to its tile launch.
    std::vector<StreamJob> sj[2];
    std::vector<TileJob> tj[2];
    int sblocks[2] = {0, 0}, ssmem[2] = {0, 0}, tblocks[2] = {0, 0};
    size_t tsmem[2] = {0, 0};
    for (auto& fp : f_) {
        Filter* f = fp.get();
        const int L = f->levels();
        for (int l = 0; l < L; ++l) {
            const Level& v = f->level(l);
            const int ph = L >= 2 && l == L - 2 ? 1 : 0;
            if (streamed(*f, l)) {
                StreamJob j{};
                j.a = f->level_args(l);
                j.band = band_of(v, rule);
                j.kind = stream_kind(v.delta, v.iters, v.smooth);
                if (v.iters < 1 || v.iters > 4 || v.smooth < 1 || v.smooth > 4)  // the phase kernel's instantiations
                    throw Error(FF_ERR_LOGIC, "batch: a streamed level outside the streaming kernel's range");
                j.first_block = sblocks[ph];
                sblocks[ph] += fused_warp_grid(v.iters, v.smooth, v.W, v.H, j.band, &j.nwx, &j.nby);
                ssmem[ph] = std::max(ssmem[ph], stream_block_smem(v.delta, v.smooth));
                sj[ph].push_back(j);
                continue;
            }
            TileJob j{};
            j.a = f->level_args(l);
            j.a.pdl_late_wait = 0;
            j.a.pdl_early_trigger = 0;
            j.delta = v.delta ? 1 : 0;
            size_t smem = 0;
            j.g = batch_geom(v.delta, v.iters, v.smooth, v.W, v.H, &smem);
            j.first_block = tblocks[ph];
            tblocks[ph] += j.g.tiles_x * ((v.H + j.g.TH - 1) / j.g.TH);
            tsmem[ph] = std::max(tsmem[ph], smem);
            tj[ph].push_back(j);
        }
    }
    // longest warps first: blocks start in index order, so the phase's tail is short warps
    // (a warp's time ~ its pipeline rows x the stages per row)
    for (auto& v : sj) {
        auto cost = [&](const StreamJob& j) {
            const int N = ((j.kind >> 2) & 3) + 1, S = (j.kind & 3) + 1;
            return (long)(j.band + 2 * N + 4 * S) * (2 * N + 2 * S + 4);
        };
        std::stable_sort(v.begin(), v.end(), [&](const StreamJob& x, const StreamJob& y) { return cost(x) > cost(y); });
        int blocks = 0;
        for (auto& j : v) {
            j.first_block = blocks;
            int nwx = 0, nby = 0;
            blocks += fused_warp_grid(((j.kind >> 2) & 3) + 1, (j.kind & 3) + 1, j.a.W, j.a.H, j.band, &nwx, &nby);
        }
    }
    std::vector<StreamJob> sall(sj[0]);
    sall.insert(sall.end(), sj[1].begin(), sj[1].end());
    std::vector<TileJob> tall(tj[0]);
    tall.insert(tall.end(), tj[1].begin(), tj[1].end());
    t.d_pyr = to_device(pyr);
    t.d_tile = to_device(tall);
    t.d_stream = to_device(sall);
    t.parity.clear();
    t.gen.clear();
    for (auto& f : f_) {
        t.parity.push_back(f->parity());
        t.gen.push_back(f->config_generation());
    }
    t.tune_gen = tune_gen_;
    // capture: the deeper pyramid depths; phase A's streaming launch, with its tile launch on
    // a branch beside it (the small levels fill the streaming launch's tail); phase B's
    // launches after both
    cudaGraph_t g = nullptr;
    check_cuda(cudaStreamBeginCapture(cap_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    int launches = 0;
    for (int d = 3; d < max_levels_; ++d)
        if (pyr_count[d] > 0) {
            ok(launch_k(pyramid_batch_k, dim3(pyr_blocks[d]), dim3(256), 0, cap_,
                        (const PyrJob*)(t.d_pyr + pyr_first[d]), pyr_count[d]));
            ++launches;
        }
    for (int ph = 0; ph < 2; ++ph) {
        const bool branch = ph == 0 && !tj[0].empty() && !sj[0].empty();
        if (branch) {
            ok(cudaEventRecord(fork_, cap_));
            ok(cudaStreamWaitEvent(side_, fork_, 0));
        }
        if (!sj[ph].empty()) {
            ok(launch_stream_mega(t.d_stream + (ph ? sj[0].size() : 0), (int)sj[ph].size(), sblocks[ph], ssmem[ph],
                                  cap_));
            ++launches;
        }
        if (!tj[ph].empty()) {
            ok(launch_k(tile_batch_k, dim3(tblocks[ph]), dim3(kTileThreads), tsmem[ph], branch ? side_ : cap_,
                        (const TileJob*)(t.d_tile + (ph ? tj[0].size() : 0)), (int)tj[ph].size()));
            ++launches;
        }
        if (branch) {
            ok(cudaEventRecord(join_, side_));
            ok(cudaStreamWaitEvent(cap_, join_, 0));
        }
    }
    cudaError_t ec = cudaStreamEndCapture(cap_, &g);
    check_cuda(e, "batch capture");
    check_cuda(ec, "cudaStreamEndCapture");
    e = cudaGraphInstantiateWithFlags(&t.graph, g, 0);
    cudaGraphDestroy(g);
    check_cuda(e, "cudaGraphInstantiate");
    t.launches = launches;
    log_message(FF_LOG_INFO, "batch: step graph built for " + std::to_string(f_.size()) + " streams, " +
                                 std::to_string(1 + launches) + " launches, default streaming band " +
                                 std::to_string(rule) + " rows");
}

void Batch::step(const void* frames, cudaStream_t s) {
    if (!frames) throw Error(FF_ERR_INVALID_ARGUMENT, "batch: null frame buffer");
    if ((uintptr_t)frames % 16) throw Error(FF_ERR_INVALID_ARGUMENT, "batch: the frame buffer must be 16-byte aligned");
    for (auto& f : f_) f->batch_begin(s);
    check_cuda(launch_k(ingest_pyr_k, dim3(ingest_blocks_), dim3(32, 8), 0, s, (const uint8_t*)frames,
                        (const IngestJob*)d_ingest_, (const unsigned short*)d_ingest_block_),
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
