// Filter objects: buffers, parameter rules and the per-frame schedule.
//
// Reference schedule (src/gpu/flowfilter.cu:685-716): pyramid; image model and
// propagation of every level; top update; delta updates finest first.  Because the
// finest levels update before coarser ones, a delta level h < L-2 reads level h+1's
// smoothed flow of the PREVIOUS frame, and level L-2 reads the top level's
// UNSMOOTHED flow of this frame (flowfilter.cu:663-672).  With ping-pong state this
// is: coarse(h) = fs[cur] of level h+1, or fu of the top level for h = L-2.
#include "filter.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <vector>

#include "kernels.h"

namespace ffb {

void check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    ff_status s = (e == cudaErrorMemoryAllocation) ? FF_ERR_OUT_OF_MEMORY : FF_ERR_CUDA;
    throw Error(s, std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {
std::atomic<long long> g_alloc_fail_after{-1};

// true for the allocation that the injection fails (one-shot)
bool allocation_fails() {
    long long n = g_alloc_fail_after.load();
    while (n >= 0)
        if (g_alloc_fail_after.compare_exchange_weak(n, n - 1)) return n == 0;
    return false;
}
}  // namespace

void inject_allocation_failure(long long n) { g_alloc_fail_after.store(n < 0 ? -1 : n); }

cudaError_t device_malloc(void** p, size_t bytes) {
    if (allocation_fails()) return cudaErrorMemoryAllocation;
    return cudaMalloc(p, bytes);
}

cudaError_t device_malloc_pitch(void** p, size_t* pitch, size_t width_bytes, size_t height) {
    if (allocation_fails()) return cudaErrorMemoryAllocation;
    return cudaMallocPitch(p, pitch, width_bytes, height);
}

// Rows are allocated with room for one extra pixel (and a 4-byte multiple), so the fused
// kernels' aligned pair copies of columns (W-1, W) stay inside the allocation.
void Buf::alloc(int h_, int w_, int bpp_) {
    release();
    h = h_;
    w = w_;
    bpp = bpp_;
    if (h <= 0 || w <= 0) return;
    const size_t row = ((size_t)(w + 1) * bpp + 3) & ~(size_t)3;
    check_cuda(device_malloc_pitch(&p, &pitch, row, (size_t)h), "cudaMallocPitch");
    check_cuda(cudaMemset2D(p, pitch, 0, row, (size_t)h), "cudaMemset2D");
}

void Buf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    pitch = 0;
}

void Buf::clear(cudaStream_t s) {
    if (p) check_cuda(cudaMemset2DAsync(p, pitch, 0, row_bytes(), (size_t)h, s), "cudaMemset2DAsync");
}

void Level::alloc_state() {
    for (int k = 0; k < 2; ++k) {
        fs[k].alloc(H, W, 8);
        io[k].alloc(H, W, 4);
        if (delta) d[k].alloc(H, W, 8);
    }
    if (!delta) fu.alloc(H, W, 8);
}

// Same index as the device's upmap_index (common.cuh): u = x/(W-1) rounded to float,
// truncated to 21 fractional bits, times the coarse size.  IEEE float division on the
// host rounds like __fdiv_rn.
static int upmap_index_host(int x, int W, int Wc) {
    const float u = (float)x / (float)(W - 1);
    if (!(u == u)) return 0;
    const long long q = (long long)std::floor(u * 2097152.0f);
    long long i = (q * (long long)Wc) >> 21;
    if (i < 0) i = 0;
    if (i > Wc - 1) i = Wc - 1;
    return (int)i;
}

void Level::build_coarse_rows() {
    if (!delta || Hc <= 0) return;
    std::vector<int> t(H);
    for (int y = 0; y < H; ++y) t[y] = upmap_index_host(y, H, Hc);
    coarse_rows.alloc(1, H, 4);
    check_cuda(cudaMemcpy(coarse_rows.p, t.data(), t.size() * sizeof(int), cudaMemcpyHostToDevice), "coarse rows");
}

void Level::alloc_scratch() {
    if (a0.p) return;
    a0.alloc(H, W, 4);
    grad.alloc(H, W, 8);
    fp.alloc(H, W, 8);
    t1.alloc(H, W, 8);
    if (delta) {
        ip.alloc(H, W, 4);
        dp.alloc(H, W, 8);
        t2.alloc(H, W, 4);
        t3.alloc(H, W, 8);
        fut.alloc(H, W, 8);
    }
}

void Level::release() {
    for (int k = 0; k < 2; ++k) {
        fs[k].release();
        io[k].release();
        d[k].release();
    }
    for (Buf* b : {&fu, &a0, &grad, &fp, &ip, &dp, &t1, &t2, &t3, &fut, &coarse_rows}) b->release();
}

Filter::Filter(Kind kind, int H, int W, int levels, int item, bool own_input)
    : kind_(kind), H_(H), W_(W), L_(levels), item_(item) {
    if (H <= 0) throw Error(FF_ERR_INVALID_ARGUMENT, "height should be greater than zero, got: " + std::to_string(H));
    if (W <= 0) throw Error(FF_ERR_INVALID_ARGUMENT, "width should be greater than zero, got: " + std::to_string(W));
    if (levels <= 0) throw Error(FF_ERR_INVALID_ARGUMENT, "levels should be greater than zero, got: " + std::to_string(levels));
    if (item != 1 && item != 4) throw Error(FF_ERR_INVALID_ARGUMENT, "item size should be 1 or 4: " + std::to_string(item));
    if (kind != Kind::Pyramidal && levels != 1) throw Error(FF_ERR_INVALID_ARGUMENT, "single-level filter with levels != 1");
    try {
        check_cuda(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
        own_stream_ = true;
        check_cuda(cudaEventCreate(&ev0_), "cudaEventCreate");
        check_cuda(cudaEventCreate(&ev1_), "cudaEventCreate");
        // the frame graph's chain pyramid -> top -> level L-2 (captured on cap_) at the highest
        // stream priority, level 0 (on side_) at the lowest: when both have blocks waiting,
        // the latency-bound chain's are dispatched first (graphs keep node priorities)
        int lo_p = 0, hi_p = 0;
        check_cuda(cudaDeviceGetStreamPriorityRange(&lo_p, &hi_p), "cudaDeviceGetStreamPriorityRange");
        check_cuda(cudaStreamCreateWithPriority(&side_, cudaStreamNonBlocking, lo_p), "cudaStreamCreate");
        check_cuda(cudaStreamCreateWithPriority(&cap_, cudaStreamNonBlocking, hi_p), "cudaStreamCreate");
        for (cudaEvent_t* e : {&ev_fork_, &ev_pyr_, &ev_join_, &done_})
            check_cuda(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate");
        check_cuda(cudaEventRecord(done_, stream_), "cudaEventRecord");
        lv_.resize(L_);
        if (kind == Kind::Pyramidal) {
            // ImagePyramid::configure: integer halving, X then Y (pyramid.cu:74-83)
            input_.alloc(H, W, item);
            int h = H, w = W;
            pyr_.resize(L_ - 1);
            for (int l = 0; l < L_; ++l) {
                if (l > 0) {
                    w /= 2;
                    h /= 2;
                    if (h <= 0 || w <= 0)
                        throw Error(FF_ERR_INVALID_ARGUMENT, "pyramid level " + std::to_string(l) + " has zero size");
                    pyr_[l - 1].alloc(h, w, item);
                }
                Level& v = lv_[l];
                v.delta = l < L_ - 1;
                v.H = h;
                v.W = w;
                v.item = item;
                v.img = l == 0 ? input_.p : pyr_[l - 1].p;
                v.img_pitch = l == 0 ? input_.pitch : pyr_[l - 1].pitch;
                v.img_owned = true;
            }
            for (int l = 0; l < L_ - 1; ++l) {
                lv_[l].Hc = lv_[l + 1].H;
                lv_[l].Wc = lv_[l + 1].W;
                lv_[l].build_coarse_rows();
            }
        } else {
            Level& v = lv_[0];
            v.delta = kind == Kind::Delta;
            v.H = H;
            v.W = W;
            v.item = item;
            if (own_input) {
                input_.alloc(H, W, item);
                v.img = input_.p;
                v.img_pitch = input_.pitch;
                v.img_owned = true;
            }
        }
        // configure() defaults: FlowUpdate/DeltaFlowUpdate(gamma 1, maxflow 1),
        // FlowSmoother(1), FlowPropagator(1), border 3 (flowfilter.cu:100-107, 393-402)
        for (Level& v : lv_) v.alloc_state();
        check_cuda(cudaDeviceSynchronize(), "configure");
    } catch (...) {
        for (Level& v : lv_) v.release();
        for (Buf& b : pyr_) b.release();
        input_.release();
        release_runtime();
        throw;
    }
}

Filter::HostPipe::~HostPipe() {
    if (out) cudaStreamSynchronize(out);
    if (in) cudaStreamSynchronize(in);
    for (int k = 0; k < 2; ++k) {
        for (cudaEvent_t e : {h2d[k], computed[k], d2h[k]})
            if (e) cudaEventDestroy(e);
        staging[k].release();
    }
    if (last_d2h) cudaEventDestroy(last_d2h);
    if (in) cudaStreamDestroy(in);
    if (out) cudaStreamDestroy(out);
}

void Filter::leave_pipe_mode() {
    if (!pipe_mode_) return;
    lv_[0].img = input_.p;
    lv_[0].img_pitch = input_.pitch;
    pipe_mode_ = false;
    drop_graphs();
}

void Filter::synchronize() {
    check_cuda(cudaEventSynchronize(done_), "synchronize");
    if (pipe_) {
        check_cuda(cudaStreamSynchronize(pipe_->out), "synchronize");
        check_cuda(cudaStreamSynchronize(pipe_->in), "synchronize");
        pipe_->pending = false;
    }
}

void Filter::process_host_async(const ff_image& in, ff_image& out, cudaStream_t s) {
    if (!input_.p || lv_[0].img_owned == false)
        throw Error(FF_ERR_UNSUPPORTED, "pipelined host processing needs a filter that owns its input image");
    check_image_shape(in.height, in.width, in.depth, (int)in.itemSize);
    if (!in.data) throw Error(FF_ERR_INVALID_ARGUMENT, "null image data");
    if (out.height != H_ || out.width != W_ || out.depth != 2 || out.itemSize != 4)
        throw Error(FF_ERR_SHAPE, "flow buffer should be [" + std::to_string(H_) + ", " + std::to_string(W_) + ", 2][4]");
    if (!out.data) throw Error(FF_ERR_INVALID_ARGUMENT, "null flow buffer");
    if (!pipe_) {
        std::unique_ptr<HostPipe> p(new HostPipe);
        check_cuda(cudaStreamCreateWithFlags(&p->in, cudaStreamNonBlocking), "cudaStreamCreate");
        check_cuda(cudaStreamCreateWithFlags(&p->out, cudaStreamNonBlocking), "cudaStreamCreate");
        for (int k = 0; k < 2; ++k) {
            p->staging[k].alloc(H_, W_, item_);
            for (cudaEvent_t* e : {&p->h2d[k], &p->computed[k], &p->d2h[k]}) {
                check_cuda(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate");
                check_cuda(cudaEventRecord(*e, stream_), "cudaEventRecord");
            }
        }
        check_cuda(cudaEventCreateWithFlags(&p->last_d2h, cudaEventDisableTiming), "cudaEventCreate");
        pipe_ = std::move(p);
    }
    HostPipe& P = *pipe_;
    if (!pipe_mode_) {
        drop_graphs();
        pipe_mode_ = true;
    }
    const int p = cur_;
    // upload into this parity's staging image once the frame two steps back stopped reading it
    check_cuda(cudaStreamWaitEvent(P.in, P.computed[p], 0), "cudaStreamWaitEvent");
    check_cuda(cudaMemcpy2DAsync(P.staging[p].p, P.staging[p].pitch, in.data, in.pitch, (size_t)W_ * item_, (size_t)H_,
                                 cudaMemcpyHostToDevice, P.in),
               "upload");
    check_cuda(cudaEventRecord(P.h2d[p], P.in), "cudaEventRecord");
    // compute: after the upload, and after the download of the frame two steps back, whose
    // result buffer this frame overwrites
    lv_[0].img = P.staging[p].p;
    lv_[0].img_pitch = P.staging[p].pitch;
    check_cuda(cudaStreamWaitEvent(s, P.h2d[p], 0), "cudaStreamWaitEvent");
    check_cuda(cudaStreamWaitEvent(s, P.d2h[p], 0), "cudaStreamWaitEvent");
    in_pipe_ = true;
    try {
        compute_async(s);
    } catch (...) {
        in_pipe_ = false;
        throw;
    }
    in_pipe_ = false;
    check_cuda(cudaEventRecord(P.computed[p], s), "cudaEventRecord");
    // download the smoothed level-0 flow of this frame
    const Buf& r = lv_[0].fs[cur_];
    check_cuda(cudaStreamWaitEvent(P.out, P.computed[p], 0), "cudaStreamWaitEvent");
    check_cuda(cudaMemcpy2DAsync(out.data, out.pitch, r.p, r.pitch, r.row_bytes(), (size_t)r.h, cudaMemcpyDeviceToHost,
                                 P.out),
               "download");
    check_cuda(cudaEventRecord(P.d2h[p], P.out), "cudaEventRecord");
    check_cuda(cudaEventRecord(P.last_d2h, P.out), "cudaEventRecord");
    P.pending = true;
}

void Filter::release_runtime() {
    pipe_.reset();
    drop_graphs();
    for (cudaEvent_t e : prof_ev_) cudaEventDestroy(e);
    prof_ev_.clear();
    for (cudaEvent_t* e : {&ev0_, &ev1_, &ev_fork_, &ev_pyr_, &ev_join_, &done_}) {
        if (*e) cudaEventDestroy(*e);
        *e = nullptr;
    }
    if (side_) cudaStreamDestroy(side_);
    if (cap_) cudaStreamDestroy(cap_);
    side_ = cap_ = nullptr;
    if (own_stream_ && stream_) cudaStreamDestroy(stream_);
    stream_ = nullptr;
}

Filter::~Filter() {
    if (done_) cudaEventSynchronize(done_);
    if (stream_) cudaStreamSynchronize(stream_);
    if (side_) cudaStreamSynchronize(side_);
    release_runtime();
    for (Level& v : lv_) v.release();
    for (Buf& b : pyr_) b.release();
    input_.release();
}

// Every operation on the filter, on whichever stream, starts after the previous one
// finished (event done_) and marks its own end; blocking calls use the filter's stream.
void Filter::begin_on(cudaStream_t s) {
    check_cuda(cudaStreamWaitEvent(s, done_, 0), "cudaStreamWaitEvent");
    // work outside the pipelined path must not overwrite a result still being downloaded
    if (pipe_ && pipe_->pending && !in_pipe_) {
        check_cuda(cudaStreamWaitEvent(s, pipe_->last_d2h, 0), "cudaStreamWaitEvent");
        pipe_->pending = false;
    }
}
void Filter::end_on(cudaStream_t s) {
    check_cuda(cudaEventRecord(done_, s), "cudaEventRecord");
    ++ops_;
}

void Filter::wait_done() const { check_cuda(cudaEventSynchronize(done_), "wait"); }

bool Filter::any_first() const {
    for (const Level& v : lv_)
        if (v.first) return true;
    return false;
}

void Filter::batch_begin(cudaStream_t s) {
    if (ops_ != batch_seen_) begin_on(s);
}

void Filter::batch_end(cudaStream_t s) {
    end_on(s);
    batch_seen_ = ops_;
    cur_ ^= 1;
    for (Level& v : lv_) v.first = false;
    phase_ = 0;
}

Level& Filter::level(int l) {
    if (l < 0 || l >= L_) throw Error(FF_ERR_OUT_OF_RANGE, "level index out of bounds: " + std::to_string(l));
    return lv_[l];
}
const Level& Filter::level(int l) const {
    if (l < 0 || l >= L_) throw Error(FF_ERR_OUT_OF_RANGE, "level index out of bounds: " + std::to_string(l));
    return lv_[l];
}

// FlowFilter::setGamma / DeltaFlowFilter::setGamma: gamma/255^2 for uint8 input
// (flowfilter.cu:276-285, 559-568); FlowUpdate::setGamma rejects gamma <= 0 (update.cu:124-132)
void Filter::set_gamma(int l, float g) {
    drop_graphs();
    Level& v = level(l);
    const float eff = v.item == 1 ? g / (255.0f * 255.0f) : g;
    if (!(eff > 0.0f)) throw Error(FF_ERR_INVALID_ARGUMENT, "gamma should be greater than zero: " + std::to_string(g));
    v.gamma = eff;
}
float Filter::gamma(int l) const { return level(l).gamma; }

// setMaxFlow: iterations = int(ceilf(maxflow)) must be > 0 (propagation.cu:137-148);
// pyramids halve per level, top = maxflow / 2^(L-1) (flowfilter.cu:849-866)
void Filter::set_max_flow(float m) {
    drop_graphs();
    for (Level& v : lv_) v.tuned_path = -1;
    float ml = m;
    std::vector<float> per(L_);
    if (L_ == 1) {
        per[0] = m;
    } else {
        for (int l = 0; l < L_ - 1; ++l) {
            per[l] = ml;
            ml /= 2.0f;
        }
        per[L_ - 1] = ml;
    }
    for (float x : per)
        if (!((int)ceilf(x) > 0))
            throw Error(FF_ERR_INVALID_ARGUMENT, "propagation iterations should be greater than zero, maxflow: " + std::to_string(m));
    for (int l = 0; l < L_; ++l) {
        lv_[l].maxflow = per[l];
        lv_[l].iters = (int)ceilf(per[l]);
    }
}
float Filter::max_flow() const { return lv_[0].maxflow; }

void Filter::set_smooth(int l, int n) {
    drop_graphs();
    for (Level& v : lv_) v.tuned_path = -1;
    Level& v = level(l);
    if (n <= 0) throw Error(FF_ERR_INVALID_ARGUMENT, "smooth iterations should be greater than zero: " + std::to_string(n));
    v.smooth = n;
}
int Filter::smooth(int l) const { return level(l).smooth; }

void Filter::set_border(int b) {
    drop_graphs();
    if (b < 0) throw Error(FF_ERR_INVALID_ARGUMENT, "border should be greater or equal zero: " + std::to_string(b));
    for (Level& v : lv_) v.border = b;
}
int Filter::border() const { return lv_[L_ - 1].border; }
int Filter::iterations(int l) const { return level(l).iters; }

void Filter::set_stream(cudaStream_t s) {
    check_cuda(cudaEventSynchronize(done_), "set_stream");
    if (own_stream_ && stream_) {
        cudaStreamSynchronize(stream_);
        cudaStreamDestroy(stream_);
    }
    own_stream_ = false;
    stream_ = s;
}

void Filter::check_image_shape(int h, int w, int depth, int item) const {
    if (h != H_ || w != W_ || depth != 1 || item != item_)
        throw Error(FF_ERR_SHAPE, "GPUImage::upload(): shapes do not match. Required: [" + std::to_string(H_) + ", " +
                                      std::to_string(W_) + ", 1][" + std::to_string(item_) + "], passed: [" +
                                      std::to_string(h) + ", " + std::to_string(w) + ", " + std::to_string(depth) +
                                      "][" + std::to_string(item) + "]");
}

void Filter::load_host(const ff_image& img) {
    leave_pipe_mode();
    check_image_shape(img.height, img.width, img.depth, (int)img.itemSize);
    if (!img.data) throw Error(FF_ERR_INVALID_ARGUMENT, "null image data");
    Level& v = lv_[0];
    if (!v.img) throw Error(FF_ERR_LOGIC, "input image has not been set");
    begin_on(stream_);
    check_cuda(cudaMemcpy2DAsync(const_cast<void*>(v.img), v.img_pitch, img.data, img.pitch, (size_t)W_ * item_,
                                 (size_t)H_, cudaMemcpyHostToDevice, stream_),
               "upload");
    end_on(stream_);
    check_cuda(cudaStreamSynchronize(stream_), "upload");
}

void Filter::load_device_async(const void* img, size_t pitch, cudaStream_t s) {
    leave_pipe_mode();
    Level& v = lv_[0];
    if (!v.img) throw Error(FF_ERR_LOGIC, "input image has not been set");
    if (!img) throw Error(FF_ERR_INVALID_ARGUMENT, "null image pointer");
    begin_on(s);
    check_cuda(cudaMemcpy2DAsync(const_cast<void*>(v.img), v.img_pitch, img, pitch, (size_t)W_ * item_, (size_t)H_,
                                 cudaMemcpyDeviceToDevice, s),
               "load_device");
    end_on(s);
}

void Filter::bind_device(const void* img, size_t pitch) {
    pipe_mode_ = false;
    drop_graphs();
    if (!img) throw Error(FF_ERR_INVALID_ARGUMENT, "null image pointer");
    if (pitch < (size_t)W_ * item_) throw Error(FF_ERR_INVALID_ARGUMENT, "pitch smaller than a row");
    if (((uintptr_t)img % item_) || (pitch % item_))
        throw Error(FF_ERR_INVALID_ARGUMENT, "image rows must be aligned to the item size");
    lv_[0].img = img;
    lv_[0].img_pitch = pitch;
    lv_[0].img_owned = false;
}

void Filter::set_external_image(const void* img, size_t pitch) { bind_device(img, pitch); }

void Filter::set_external_coarse(const void* flow, size_t pitch, int Hc, int Wc) {
    drop_graphs();
    if (!flow) throw Error(FF_ERR_INVALID_ARGUMENT, "null coarse flow");
    if (Hc <= 0 || Wc <= 0) throw Error(FF_ERR_INVALID_ARGUMENT, "coarse flow shape");
    if (pitch < (size_t)Wc * 8) throw Error(FF_ERR_INVALID_ARGUMENT, "coarse pitch smaller than a row");
    Level& v = lv_[0];
    v.coarse = flow;
    v.coarse_pitch = pitch;
    v.Hc = Hc;
    v.Wc = Wc;
    v.build_coarse_rows();
}

void Filter::coarse_of(int l, const void** p, size_t* pitch, int* Hc, int* Wc) const {
    const Level& v = lv_[l];
    if (kind_ != Kind::Pyramidal) {
        *p = v.coarse;
        *pitch = v.coarse_pitch;
    } else if (l == L_ - 2) {
        *p = lv_[L_ - 1].fu.p;
        *pitch = lv_[L_ - 1].fu.pitch;
    } else {
        *p = lv_[l + 1].fs[cur_].p;
        *pitch = lv_[l + 1].fs[cur_].pitch;
    }
    *Hc = v.Hc;
    *Wc = v.Wc;
}

// ------------------------------------------------------------------ unfused path
void Filter::model_unfused(int l, cudaStream_t s) {
    Level& v = lv_[l];
    v.alloc_scratch();
    check_cuda(launch_image_model(v.img, v.img_pitch, v.item, v.H, v.W, (float*)v.a0.p, v.a0.pitch,
                                  (float*)v.grad.p, v.grad.pitch, s),
               "image model");
}

void Filter::propagate_unfused(int l, cudaStream_t s) {
    Level& v = lv_[l];
    v.alloc_scratch();
    const Buf& fs = v.fs[cur_];
    if (!v.delta) {
        check_cuda(launch_propagate((const float*)fs.p, fs.pitch, v.H, v.W, v.iters, v.border, (float*)v.fp.p,
                                    v.fp.pitch, (float*)v.t1.p, v.t1.pitch, s),
                   "propagate");
    } else {
        const Buf& io = v.io[cur_];
        const Buf& d = v.d[cur_];
        check_cuda(launch_propagate_payload((const float*)fs.p, fs.pitch, (const float*)io.p, io.pitch,
                                            (const float*)d.p, d.pitch, v.H, v.W, v.iters, v.border, (float*)v.fp.p,
                                            v.fp.pitch, (float*)v.ip.p, v.ip.pitch, (float*)v.dp.p, v.dp.pitch,
                                            (float*)v.t1.p, v.t1.pitch, (float*)v.t2.p, v.t2.pitch, (float*)v.t3.p,
                                            v.t3.pitch, s),
                   "propagate payload");
    }
}

void Filter::update_unfused(int l, cudaStream_t s) {
    Level& v = lv_[l];
    v.alloc_scratch();
    const int nxt = cur_ ^ 1;
    if (!v.delta) {
        const Buf& io = v.io[cur_];
        check_cuda(launch_update((const float*)v.a0.p, v.a0.pitch, (const float*)v.grad.p, v.grad.pitch,
                                 (const float*)io.p, io.pitch, (const float*)v.fp.p, v.fp.pitch, v.H, v.W, v.gamma,
                                 v.maxflow, (float*)v.fu.p, v.fu.pitch, (float*)v.io[nxt].p, v.io[nxt].pitch,
                                 v.first ? 1 : 0, s),
                   "update");
        check_cuda(launch_smooth((const float*)v.fu.p, v.fu.pitch, v.H, v.W, v.smooth, (float*)v.fs[nxt].p,
                                 v.fs[nxt].pitch, (float*)v.t1.p, v.t1.pitch, s),
                   "smooth");
    } else {
        const void* cp;
        size_t cpitch;
        int Hc, Wc;
        coarse_of(l, &cp, &cpitch, &Hc, &Wc);
        if (!cp) throw Error(FF_ERR_LOGIC, "DeltaFlowFilter: input flow not set");
        check_cuda(launch_delta_update((const float*)v.a0.p, v.a0.pitch, (const float*)v.grad.p, v.grad.pitch,
                                       (const float*)v.ip.p, v.ip.pitch, (const float*)v.dp.p, v.dp.pitch,
                                       (const float*)cp, cpitch, Hc, Wc, v.H, v.W, v.gamma, v.maxflow,
                                       (float*)v.fut.p, v.fut.pitch, (float*)v.d[nxt].p, v.d[nxt].pitch,
                                       (float*)v.io[nxt].p, v.io[nxt].pitch, v.first ? 1 : 0, s),
                   "delta update");
        check_cuda(launch_smooth((const float*)v.fut.p, v.fut.pitch, v.H, v.W, v.smooth, (float*)v.fs[nxt].p,
                                 v.fs[nxt].pitch, (float*)v.t1.p, v.t1.pitch, s),
                   "smooth");
    }
}

void Filter::step_level_unfused(int l, cudaStream_t s) {
    model_unfused(l, s);
    propagate_unfused(l, s);
    update_unfused(l, s);
}

// can the fused kernel run this level (instantiated, aligned image rows, coarse flow)?
bool Filter::fused_ok(int l) const {
    const Level& v = lv_[l];
    // the fused kernels stage rows with 4- and 8-byte cp.async copies: the image rows must
    // be aligned, and uint8 rows readable up to the next multiple of 4 bytes
    const uintptr_t ib = (uintptr_t)v.img;
    const bool img_ok = v.item == 1 ? (ib % 4 == 0 && v.img_pitch % 4 == 0 && (v.img_owned || v.W % 4 == 0))
                                    : (ib % 8 == 0 && v.img_pitch % 8 == 0 &&
                                       (v.img_owned || v.W % 2 == 0 || v.img_pitch >= (size_t)(v.W + 1) * 4));
    bool coarse_ok = true;
    if (v.delta) {
        const void* cpp = nullptr;
        size_t cpitch = 0;
        int chh = 0, cww = 0;
        coarse_of(l, &cpp, &cpitch, &chh, &cww);
        coarse_ok = cpp && (uintptr_t)cpp % 8 == 0 && cpitch % 8 == 0;
    }
    return img_ok && coarse_ok && fused_available(v.delta, v.item, v.iters, v.smooth);
}

bool Filter::tile_ok(int l, int cfg) const {
    const Level& v = lv_[l];
    if (v.delta) {
        const void* cpp = nullptr;
        size_t cpitch = 0;
        int chh = 0, cww = 0;
        coarse_of(l, &cpp, &cpitch, &chh, &cww);
        if (!cpp || (uintptr_t)cpp % 8 != 0 || cpitch % 8 != 0) return false;
    }
    if (v.item == 4 && ((uintptr_t)v.img % 4 != 0 || v.img_pitch % 4 != 0)) return false;
    return tile_available(v.delta, v.iters, v.smooth, v.W, v.H, cfg);
}

LevelArgs Filter::level_args(int l) const {
    const Level& v = lv_[l];
    const int nxt = cur_ ^ 1;
    LevelArgs a{};
    a.H = v.H;
    a.W = v.W;
    a.item = v.item;
    a.img = v.img;
    a.img_pitch = v.img_pitch;
    a.fs_in = (const float*)v.fs[cur_].p;
    a.fs_in_pitch = v.fs[cur_].pitch;
    a.io_in = (const float*)v.io[cur_].p;
    a.io_in_pitch = v.io[cur_].pitch;
    a.fs_out = (float*)v.fs[nxt].p;
    a.fs_out_pitch = v.fs[nxt].pitch;
    a.io_out = (float*)v.io[nxt].p;
    a.io_out_pitch = v.io[nxt].pitch;
    if (v.delta) {
        a.d_in = (const float*)v.d[cur_].p;
        a.d_in_pitch = v.d[cur_].pitch;
        a.d_out = (float*)v.d[nxt].p;
        a.d_out_pitch = v.d[nxt].pitch;
        const void* cp;
        coarse_of(l, &cp, &a.coarse_pitch, &a.Hc, &a.Wc);
        a.coarse = (const float*)cp;
        a.coarse_rows = (const int*)v.coarse_rows.p;
    } else {
        a.fu_out = (float*)v.fu.p;
        a.fu_out_pitch = v.fu.pitch;
    }
    a.gamma = v.gamma;
    a.maxflow = v.maxflow;
    a.border = v.border;
    a.first = v.first ? 1 : 0;
    return a;
}

void Filter::launch_fused(int l, int band, cudaStream_t s) {
    const Level& v = lv_[l];
    LevelArgs a = level_args(l);
    a.band = band;
    check_cuda(launch_fused_level(v.delta, v.iters, v.smooth, a, s), "fused level");
}

void Filter::launch_tile(int l, int cfg, cudaStream_t s) {
    const Level& v = lv_[l];
    LevelArgs a = level_args(l);
    // In a pyramid frame the top level's tile kernel is followed on the same stream by level
    // L-2's, which reads the top's output only from its update on: the top lets it start at
    // once, and it waits only before its update (so its propagation overlaps the top level).
    if (kind_ == Kind::Pyramidal && L_ >= 2 && pdl_chain_) {
        int p_top = 0, p_next = 0;
        const bool top_tile = path_of(L_ - 1, &p_top) == kTile, next_tile = path_of(L_ - 2, &p_next) == kTile;
        if (l == L_ - 1 && next_tile) a.pdl_early_trigger = 1;
        if (l == L_ - 2 && top_tile) a.pdl_late_wait = 1;
    }
    if (fuse_pyramid_ && l == L_ - 1) {
        const Level& fine = lv_[0];
        a.pyr_src = fine.img;
        a.pyr_src_pitch = fine.img_pitch;
        a.pyr_src_H = fine.H;
        a.pyr_src_W = fine.W;
    }
    check_cuda(launch_tile_level(v.delta, v.iters, v.smooth, a, cfg, s), "tile level");
}

void Filter::step_level(int l, cudaStream_t s) {
    Level& v = lv_[l];
    if (!v.img) throw Error(FF_ERR_LOGIC, "input image has not been set");
    if (v.delta) {
        const void* cp;
        size_t cpitch;
        int hc, wc;
        coarse_of(l, &cp, &cpitch, &hc, &wc);
        if (!cp) throw Error(FF_ERR_LOGIC, "DeltaFlowFilter: input flow not set");
    }
    int param = 0;
    switch (path_of(l, &param)) {
        case kStream: launch_fused(l, param, s); break;
        case kTile: launch_tile(l, param, s); break;
        default: step_level_unfused(l, s);
    }
}

// the path a level step takes now; *param = band rows (streaming) or tile shape (tile)
int Filter::path_of(int l, int* param) const {
    const Level& v = lv_[l];
    int dummy = 0;
    int& p = param ? *param : dummy;
    p = 0;
    switch (fused_mode_) {
        case 0: return kPerStage;
        case 1:
            p = band_;
            return fused_ok(l) ? kStream : kPerStage;
        case 3: return tile_ok(l, 0) ? kTile : kPerStage;
        default: break;
    }
    if (v.tuned_path == kStream && fused_ok(l)) {
        p = v.tuned_band > 0 ? v.tuned_band : band_;
        return kStream;
    }
    if (v.tuned_path == kTile && tile_ok(l, v.tuned_band)) {
        p = v.tuned_band;
        return kTile;
    }
    if (v.tuned_path == kPerStage) return kPerStage;
    // untuned: the streaming kernel keeps large levels in one pass over HBM; below
    // kFusedMinPixels its warps are few and latency-bound, and the tile kernel spreads
    // each stage over whole CTAs instead
    if ((long)v.H * v.W >= kFusedMinPixels && fused_ok(l)) {
        p = band_;
        return kStream;
    }
    if (tile_ok(l, 0)) return kTile;
    return kPerStage;
}

void Filter::autotune(int reps, void* flush, size_t flush_bytes) {
    if (reps < 1) throw Error(FF_ERR_INVALID_ARGUMENT, "autotune repetitions must be >= 1");
    for (const Level& v : lv_)
        if (v.first) throw Error(FF_ERR_LOGIC, "autotune needs at least one computed frame");
    check_cuda(cudaEventSynchronize(done_), "autotune");
    drop_graphs();
    // the top level's unsmoothed flow is a result (getFlow) and an input of level L-2:
    // keep this frame's copy and restore it afterwards
    Buf keep;
    Level& top = lv_[L_ - 1];
    if (!top.delta && top.fu.p) {
        keep.alloc(top.fu.h, top.fu.w, top.fu.bpp);
        check_cuda(cudaMemcpy2DAsync(keep.p, keep.pitch, top.fu.p, top.fu.pitch, top.fu.row_bytes(), top.fu.h,
                                     cudaMemcpyDeviceToDevice, stream_), "autotune");
    }
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
    // candidates are timed as captured graphs of `reps` level steps, as the frame step
    // replays them, so launch gaps do not penalise the multi-kernel per-stage path
    auto time_it = [&](auto&& run) {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        check_cuda(cudaStreamBeginCapture(cap_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        try {
            for (int k = 0; k < reps; ++k) run(cap_);
        } catch (...) {
            cudaStreamEndCapture(cap_, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        check_cuda(cudaStreamEndCapture(cap_, &g), "cudaStreamEndCapture");
        cudaError_t e = cudaGraphInstantiateWithFlags(&ge, g, 0);
        cudaGraphDestroy(g);
        check_cuda(e, "cudaGraphInstantiate");
        check_cuda(cudaGraphLaunch(ge, stream_), "cudaGraphLaunch");  // warm-up
        check_cuda(cudaEventRecord(e0, stream_), "cudaEventRecord");
        check_cuda(cudaGraphLaunch(ge, stream_), "cudaGraphLaunch");
        check_cuda(cudaEventRecord(e1, stream_), "cudaEventRecord");
        check_cuda(cudaEventSynchronize(e1), "autotune");
        cudaGraphExecDestroy(ge);
        float ms = 0.f;
        check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
        return ms;
    };
    // Stage 1, every level alone: each choice timed as a graph of `reps` level steps.
    // top level first: level L-2 reads its unsmoothed flow
    struct Choice {
        float ms;
        int path, band;
    };
    std::vector<std::vector<Choice>> timed(L_);
    for (int l = L_ - 1; l >= 0; --l) {
        Level& v = lv_[l];
        v.alloc_scratch();  // allocations cannot happen inside a capture
        std::vector<Choice>& c = timed[l];
        c.push_back({time_it([&](cudaStream_t st) { step_level_unfused(l, st); }), kPerStage, 0});
        if (fused_ok(l)) {
            const int rows[] = {0, 8, 10, 12, 16, 24, 32, 48, 64, 96, 128};
            for (int b : rows) {
                if (b > v.H) continue;
                c.push_back({time_it([&](cudaStream_t st) { launch_fused(l, b, st); }), kStream, b});
            }
        }
        for (int k = 0; k < tile_config_count(); ++k) {
            if (!tile_ok(l, k)) continue;
            c.push_back({time_it([&](cudaStream_t st) { launch_tile(l, k, st); }), kTile, k});
        }
        std::stable_sort(c.begin(), c.end(), [](const Choice& a, const Choice& b) { return a.ms < b.ms; });
        v.tuned_path = c[0].path;
        v.tuned_band = c[0].band;
    }
    if (keep.p) {
        check_cuda(cudaMemcpy2DAsync(top.fu.p, top.fu.pitch, keep.p, keep.pitch, top.fu.row_bytes(), top.fu.h,
                                     cudaMemcpyDeviceToDevice, stream_), "autotune");
    }
    // Stage 2, whole frames: the levels of a frame share the GPU (level 0 runs beside the
    // chain pyramid -> top level -> level L-2 on a side stream), so the fastest level alone is
    // not always the fastest beside the others: a streaming level 0 in long bands leaves
    // room on every SM for the latency-bound small levels.  Combinations of each level's
    // three best choices (and, for a streaming level 0, longer bands) are timed as replayed
    // frames from a snapshot of the state, which is restored afterwards.
    if (L_ > 1) {
        check_cuda(cudaStreamSynchronize(stream_), "autotune");
        // per level: the three best choices, and the two best of each fused kernel
        std::vector<std::vector<Choice>> cand(L_);
        for (int l = 0; l < L_; ++l) {
            auto have = [&](const Choice& c) {
                for (const Choice& d : cand[l])
                    if (d.path == c.path && d.band == c.band) return true;
                return false;
            };
            for (const Choice& c : timed[l])
                if (cand[l].size() < 3) cand[l].push_back(c);
            for (int path : {(int)kStream, (int)kTile}) {
                int n = 0;
                for (const Choice& c : timed[l])
                    if (c.path == path && n < 2) {
                        ++n;
                        if (!have(c)) cand[l].push_back(c);
                    }
            }
        }
        if (fused_ok(0)) {
            for (int b : {48, 64, 80, 96}) {
                if (b > lv_[0].H) continue;
                bool have = false;
                for (const Choice& c : cand[0]) have |= c.path == kStream && c.band == b;
                if (!have) cand[0].push_back({0.f, kStream, b});
            }
        }
        std::vector<unsigned char> snap(state_bytes());
        export_state(snap.data(), snap.size());
        const bool graphs_was = graphs_;
        graphs_ = true;
        // a combination's score: the median of its timed frames
        auto score = [&](const std::vector<size_t>& pick, int frames) {
            for (int l = 0; l < L_; ++l) {
                lv_[l].tuned_path = cand[l][pick[l]].path;
                lv_[l].tuned_band = cand[l][pick[l]].band;
            }
            drop_graphs();
            // two frames capture both parities' graphs, then `frames` replays are timed one
            // by one (with `flush` overwritten before each, outside the timing, if given)
            compute_async(stream_);
            compute_async(stream_);
            std::vector<float> t(frames);
            for (int k = 0; k < frames; ++k) {
                if (flush && flush_bytes)
                    check_cuda(cudaMemsetAsync(flush, k & 0xff, flush_bytes, stream_), "flush");
                check_cuda(cudaEventRecord(e0, stream_), "cudaEventRecord");
                compute_async(stream_);
                check_cuda(cudaEventRecord(e1, stream_), "cudaEventRecord");
                check_cuda(cudaEventSynchronize(e1), "autotune");
                check_cuda(cudaEventElapsedTime(&t[k], e0, e1), "cudaEventElapsedTime");
            }
            std::nth_element(t.begin(), t.begin() + frames / 2, t.end());
            return t[frames / 2];
        };
        const int frames = std::max(reps, 7);
        std::vector<std::pair<float, std::vector<size_t>>> scored;
        std::vector<size_t> idx(L_, 0);
        for (;;) {
            const float ms = score(idx, frames);
            scored.push_back({ms, idx});
            int l = 0;
            while (l < L_ && ++idx[l] == cand[l].size()) idx[l++] = 0;
            if (l == L_) break;
        }
        // the six best again, in five interleaved rounds (clock or thermal drift during the
        // rounds then touches every finalist alike); a finalist's score is the median of its
        // rounds' medians
        std::sort(scored.begin(), scored.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        const size_t K = std::min<size_t>(scored.size(), 6);
        constexpr int kRounds = 5;
        std::vector<std::vector<float>> rounds(K);
        for (int r = 0; r < kRounds; ++r)
            for (size_t k = 0; k < K; ++k) rounds[k].push_back(score(scored[k].second, frames));
        std::vector<size_t> best_idx = scored[0].second;
        float best_ms = -1.f;
        for (size_t k = 0; k < K; ++k) {
            std::nth_element(rounds[k].begin(), rounds[k].begin() + kRounds / 2, rounds[k].end());
            const float ms = rounds[k][kRounds / 2];
            if (best_ms < 0.f || ms < best_ms) {
                best_ms = ms;
                best_idx = scored[k].second;
            }
        }
        for (int l = 0; l < L_; ++l) {
            lv_[l].tuned_path = cand[l][best_idx[l]].path;
            lv_[l].tuned_band = cand[l][best_idx[l]].band;
        }
        graphs_ = graphs_was;
        import_state(snap.data(), snap.size());
    }
    check_cuda(cudaStreamSynchronize(stream_), "autotune");
    keep.release();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    end_on(stream_);
}

float Filter::time_level(int l, int reps, void* flush, size_t flush_bytes) {
    level(l);
    if (reps < 1) throw Error(FF_ERR_INVALID_ARGUMENT, "repetitions must be >= 1");
    for (const Level& v : lv_)
        if (v.first) throw Error(FF_ERR_LOGIC, "timing a level needs at least one computed frame");
    check_cuda(cudaEventSynchronize(done_), "time_level");
    Level& top = lv_[L_ - 1];
    Buf keep;
    if (!top.delta && top.fu.p) {  // getFlow() result / coarse input: restored afterwards
        keep.alloc(top.fu.h, top.fu.w, top.fu.bpp);
        check_cuda(cudaMemcpy2DAsync(keep.p, keep.pitch, top.fu.p, top.fu.pitch, top.fu.row_bytes(), top.fu.h,
                                     cudaMemcpyDeviceToDevice, stream_), "time_level");
    }
    if (path_of(l, nullptr) == kPerStage) lv_[l].alloc_scratch();
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    check_cuda(cudaStreamBeginCapture(cap_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    try {
        step_level(l, cap_);
    } catch (...) {
        cudaStreamEndCapture(cap_, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    check_cuda(cudaStreamEndCapture(cap_, &g), "cudaStreamEndCapture");
    cudaError_t e = cudaGraphInstantiateWithFlags(&ge, g, 0);
    cudaGraphDestroy(g);
    check_cuda(e, "cudaGraphInstantiate");
    std::vector<cudaEvent_t> ev(2 * (size_t)reps);
    for (auto& x : ev) check_cuda(cudaEventCreate(&x), "cudaEventCreate");
    check_cuda(cudaGraphLaunch(ge, stream_), "cudaGraphLaunch");  // warm-up
    for (int k = 0; k < reps; ++k) {
        if (flush && flush_bytes) check_cuda(cudaMemsetAsync(flush, k & 0xff, flush_bytes, stream_), "flush");
        check_cuda(cudaEventRecord(ev[2 * k], stream_), "cudaEventRecord");
        check_cuda(cudaGraphLaunch(ge, stream_), "cudaGraphLaunch");
        check_cuda(cudaEventRecord(ev[2 * k + 1], stream_), "cudaEventRecord");
    }
    check_cuda(cudaEventSynchronize(ev.back()), "time_level");
    float total = 0.f;
    for (int k = 0; k < reps; ++k) {
        float ms = 0.f;
        check_cuda(cudaEventElapsedTime(&ms, ev[2 * k], ev[2 * k + 1]), "cudaEventElapsedTime");
        total += ms;
    }
    for (auto& x : ev) cudaEventDestroy(x);
    cudaGraphExecDestroy(ge);
    if (keep.p)
        check_cuda(cudaMemcpy2DAsync(top.fu.p, top.fu.pitch, keep.p, keep.pitch, top.fu.row_bytes(), top.fu.h,
                                     cudaMemcpyDeviceToDevice, stream_), "time_level");
    check_cuda(cudaStreamSynchronize(stream_), "time_level");
    keep.release();
    end_on(stream_);
    return total;
}

std::string Filter::tuning() const {
    std::string out;
    for (int l = 0; l < L_; ++l) {
        const Level& v = lv_[l];
        int param = 0;
        const int path = path_of(l, &param);
        std::string what;
        if (path == kStream) {
            what = "fused band " + (param ? std::to_string(param) : std::string("auto"));
        } else if (path == kTile) {
            int tw = 0, th = 0;
            tile_shape(v.delta, v.iters, v.smooth, v.W, v.H, param, &tw, &th);
            what = "tile " + std::to_string(tw) + "x" + std::to_string(th);
        } else {
            what = "per-stage";
        }
        if (v.tuned_path < 0 && fused_mode_ == 2) what += " (untuned)";
        out += "level " + std::to_string(l) + ": " + what + (l + 1 < L_ ? "; " : "");
    }
    return out;
}

// One frame's launches on `s` for the current state parity.  Levels 0..L-3 do not
// depend on this frame's top level, so they run on a side stream concurrently with the
// pyramid -> top -> level L-2 chain (level 0 also without waiting for the pyramid).
void Filter::enqueue_frame(cudaStream_t s) {
    const bool prof = prof_count_ < prof_cap_;
    auto level_on = [&](int l, cudaStream_t st) {
        if (prof) check_cuda(cudaEventRecord(prof_ev_[((size_t)prof_count_ * L_ + l) * 2], st), "cudaEventRecord");
        step_level(l, st);
        if (prof) check_cuda(cudaEventRecord(prof_ev_[((size_t)prof_count_ * L_ + l) * 2 + 1], st), "cudaEventRecord");
    };
    const int side_levels = kind_ == Kind::Pyramidal && L_ > 2 ? L_ - 2 : 0;  // levels 0 .. L-3
    if (side_levels > 0) {
        check_cuda(cudaEventRecord(ev_fork_, s), "cudaEventRecord");
        check_cuda(cudaStreamWaitEvent(side_, ev_fork_, 0), "cudaStreamWaitEvent");
        level_on(0, side_);
    }
    // a two-level pyramid whose top level runs the tile kernel computes its level image
    // inside that kernel (the pyramid step needs no launch of its own)
    int p_top = 0;
    fuse_pyramid_ = kind_ == Kind::Pyramidal && L_ == 2 && path_of(1, &p_top) == kTile;
    if (kind_ == Kind::Pyramidal && !fuse_pyramid_) {
        int l = 1;
        if (L_ >= 3 && lv_[2].H >= 1 && lv_[2].W >= 1) {  // levels 1 and 2 in one launch
            const Level& fine = lv_[0];
            check_cuda(launch_pyramid_down2(fine.img, fine.img_pitch, item_, fine.H, fine.W, pyr_[0].p, pyr_[0].pitch,
                                            pyr_[1].p, pyr_[1].pitch, s),
                       "pyramid");
            l = 3;
        }
        for (; l < L_; ++l) {
            const Level& fine = lv_[l - 1];
            check_cuda(launch_pyramid_down(fine.img, fine.img_pitch, item_, fine.H, fine.W, pyr_[l - 1].p,
                                           pyr_[l - 1].pitch, s),
                       "pyramid");
        }
    }
    if (side_levels > 1) {
        check_cuda(cudaEventRecord(ev_pyr_, s), "cudaEventRecord");
        check_cuda(cudaStreamWaitEvent(side_, ev_pyr_, 0), "cudaStreamWaitEvent");
        for (int l = 1; l < side_levels; ++l) level_on(l, side_);
    }
    // top first (level L-2 reads its fresh unsmoothed flow); with profiling events between
    // the launches there is no programmatic edge to exploit
    pdl_chain_ = !prof;
    for (int l = L_ - 1; l >= side_levels; --l) level_on(l, s);
    pdl_chain_ = false;
    fuse_pyramid_ = false;
    if (side_levels > 0) {
        check_cuda(cudaEventRecord(ev_join_, side_), "cudaEventRecord");
        check_cuda(cudaStreamWaitEvent(s, ev_join_, 0), "cudaStreamWaitEvent");
    }
    if (prof) ++prof_count_;
}

void Filter::drop_graphs() {
    ++config_gen_;
    for (int k = 0; k < 2; ++k) {
        if (graph_exec_[k]) cudaGraphExecDestroy(graph_exec_[k]);
        graph_exec_[k] = nullptr;
    }
}

void Filter::compute_async(cudaStream_t s) {
    begin_on(s);
    bool any_first = false;
    for (const Level& v : lv_) any_first |= v.first;
    if (graphs_ && !any_first && prof_count_ >= prof_cap_) {
        cudaGraphExec_t& ge = graph_exec_[cur_];
        if (!ge) {
            // per-stage levels need their scratch before the capture (no allocation inside it)
            for (int l = 0; l < L_; ++l)
                if (path_of(l, nullptr) == kPerStage) lv_[l].alloc_scratch();
            // capture this parity's frame once; the buffers it names alternate per frame
            check_cuda(cudaStreamBeginCapture(cap_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
            try {
                enqueue_frame(cap_);
            } catch (...) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(cap_, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            cudaGraph_t g = nullptr;
            check_cuda(cudaStreamEndCapture(cap_, &g), "cudaStreamEndCapture");
            cudaError_t e = cudaGraphInstantiateWithFlags(&ge, g, cudaGraphInstantiateFlagUseNodePriority);
            cudaGraphDestroy(g);
            check_cuda(e, "cudaGraphInstantiate");
        }
        check_cuda(cudaGraphLaunch(ge, s), "cudaGraphLaunch");
    } else {
        enqueue_frame(s);
    }
    end_on(s);
    cur_ ^= 1;
    for (Level& v : lv_) v.first = false;
    phase_ = 0;
}

void Filter::set_graphs(bool on) {
    graphs_ = on;
    if (!on) drop_graphs();
}

void Filter::set_profiling(int frames) {
    if (frames < 0) throw Error(FF_ERR_INVALID_ARGUMENT, "profiling frame count must be >= 0");
    check_cuda(cudaStreamSynchronize(stream_), "profiling");
    for (cudaEvent_t e : prof_ev_) cudaEventDestroy(e);
    prof_ev_.clear();
    prof_cap_ = frames;
    prof_count_ = 0;
    prof_ev_.resize((size_t)frames * L_ * 2, nullptr);
    for (auto& e : prof_ev_) check_cuda(cudaEventCreate(&e), "cudaEventCreate");
}

void Filter::level_kernel_ms(int l, float* total, int* frames) {
    level(l);
    float sum = 0.0f;
    for (int k = 0; k < prof_count_; ++k) {
        cudaEvent_t a = prof_ev_[((size_t)k * L_ + l) * 2], b = prof_ev_[((size_t)k * L_ + l) * 2 + 1];
        check_cuda(cudaEventSynchronize(b), "cudaEventSynchronize");
        float ms = 0.0f;
        check_cuda(cudaEventElapsedTime(&ms, a, b), "cudaEventElapsedTime");
        sum += ms;
    }
    *total = sum;
    *frames = prof_count_;
}

void Filter::compute() {
    check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    compute_async(stream_);
    check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(ev1_), "compute");
    check_cuda(cudaEventElapsedTime(&elapsed_, ev0_, ev1_), "cudaEventElapsedTime");
}

// phase API (FlowFilter / DeltaFlowFilter computeImageModel / Propagation / Update)
void Filter::phase_model() {
    if (kind_ == Kind::Pyramidal) throw Error(FF_ERR_UNSUPPORTED, "phase API is for single-level filters");
    if (!lv_[0].img) throw Error(FF_ERR_LOGIC, "input image has not been set");
    check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    begin_on(stream_);
    model_unfused(0, stream_);
    end_on(stream_);
    check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(ev1_), "computeImageModel");
    check_cuda(cudaEventElapsedTime(&elapsed_, ev0_, ev1_), "cudaEventElapsedTime");
    phase_ = 1;
}

void Filter::phase_propagation() {
    if (kind_ == Kind::Pyramidal) throw Error(FF_ERR_UNSUPPORTED, "phase API is for single-level filters");
    check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    begin_on(stream_);
    propagate_unfused(0, stream_);
    end_on(stream_);
    check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(ev1_), "computePropagation");
    check_cuda(cudaEventElapsedTime(&elapsed_, ev0_, ev1_), "cudaEventElapsedTime");
    phase_ = 2;
}

void Filter::phase_update() {
    if (kind_ == Kind::Pyramidal) throw Error(FF_ERR_UNSUPPORTED, "phase API is for single-level filters");
    check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    begin_on(stream_);
    update_unfused(0, stream_);
    end_on(stream_);
    check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(ev1_), "computeUpdate");
    check_cuda(cudaEventElapsedTime(&elapsed_, ev0_, ev1_), "cudaEventElapsedTime");
    cur_ ^= 1;
    lv_[0].first = false;
    phase_ = 0;
}

// ------------------------------------------------------------------ results
void Filter::result(int which, void** p, size_t* pitch) {
    const Level& v = lv_[0];
    const Buf* b = nullptr;
    switch (which) {
        case 0: b = &v.fs[cur_]; break;
        case 1:
            if (kind_ == Kind::Single || (kind_ == Kind::Pyramidal && L_ == 1)) b = &v.fu;
            else b = &v.fs[cur_];
            break;
        case 2: b = &v.io[cur_]; break;
        default: throw Error(FF_ERR_INVALID_ARGUMENT, "unknown result selector " + std::to_string(which));
    }
    *p = b->p;
    *pitch = b->pitch;
}

void Filter::download_flow(ff_image& out) {
    if (out.height != H_ || out.width != W_ || out.depth != 2 || out.itemSize != 4)
        throw Error(FF_ERR_SHAPE, "GPUImage::download(): shapes do not match. Required: [" + std::to_string(H_) + ", " +
                                      std::to_string(W_) + ", 2][4]");
    if (!out.data) throw Error(FF_ERR_INVALID_ARGUMENT, "null flow buffer");
    const Buf& b = lv_[0].fs[cur_];
    begin_on(stream_);
    check_cuda(cudaMemcpy2DAsync(out.data, out.pitch, b.p, b.pitch, b.row_bytes(), (size_t)b.h, cudaMemcpyDeviceToHost,
                                 stream_),
               "downloadFlow");
    end_on(stream_);
    check_cuda(cudaStreamSynchronize(stream_), "downloadFlow");
}

void Filter::download_image(ff_image& out) {
    if (out.height != H_ || out.width != W_ || out.depth != 1 || out.itemSize != 4)
        throw Error(FF_ERR_SHAPE, "GPUImage::download(): shapes do not match. Required: [" + std::to_string(H_) + ", " +
                                      std::to_string(W_) + ", 1][4]");
    if (!out.data) throw Error(FF_ERR_INVALID_ARGUMENT, "null image buffer");
    const Buf& b = lv_[0].io[cur_];
    begin_on(stream_);
    check_cuda(cudaMemcpy2DAsync(out.data, out.pitch, b.p, b.pitch, b.row_bytes(), (size_t)b.h, cudaMemcpyDeviceToHost,
                                 stream_),
               "downloadImage");
    end_on(stream_);
    check_cuda(cudaStreamSynchronize(stream_), "downloadImage");
}

void Filter::level_state(int l, int which, void* dst, size_t dst_pitch) {
    const Level& v = level(l);
    const Buf* b = nullptr;
    switch (which) {
        case 0: b = &v.fs[cur_]; break;
        case 1: b = v.delta ? nullptr : &v.fu; break;
        case 2: b = &v.io[cur_]; break;
        case 3: b = v.delta ? &v.d[cur_] : nullptr; break;
        default: break;
    }
    if (!b || !b->p) throw Error(FF_ERR_UNSUPPORTED, "level state " + std::to_string(which) + " not kept for level " + std::to_string(l));
    if (!dst) throw Error(FF_ERR_INVALID_ARGUMENT, "null destination");
    begin_on(stream_);
    check_cuda(cudaMemcpy2DAsync(dst, dst_pitch, b->p, b->pitch, b->row_bytes(), (size_t)b->h, cudaMemcpyDeviceToHost,
                                 stream_),
               "level state");
    end_on(stream_);
    check_cuda(cudaStreamSynchronize(stream_), "level state");
}

// ------------------------------------------------------------------ state export / import
// Layout: StateHeader, then per level a StateLevel, then per level the rows of its smoothed
// flow (W float2), old image (W float) and delta flow (delta levels) or unsmoothed flow
// (the top level, read by getFlow of a single-level filter) (W float2), each packed without
// padding.
namespace {
constexpr char kStateMagic[8] = {'F', 'F', 'B', 'S', 'T', 'A', 'T', 'E'};
constexpr uint32_t kStateVersion = 1;
struct StateHeader {
    char magic[8];
    uint32_t version, kind, levels, reserved;
};
struct StateLevel {
    uint32_t H, W, delta, first;
};
}  // namespace

size_t Filter::state_bytes() const {
    size_t n = sizeof(StateHeader) + (size_t)L_ * sizeof(StateLevel);
    for (const Level& v : lv_) n += (size_t)v.H * v.W * (8 + 4 + 8);
    return n;
}

void Filter::export_state(void* host, size_t bytes) const {
    if (!host) throw Error(FF_ERR_INVALID_ARGUMENT, "null state buffer");
    if (bytes < state_bytes())
        throw Error(FF_ERR_INVALID_ARGUMENT, "state buffer too small: " + std::to_string(bytes) + " < " +
                                                 std::to_string(state_bytes()));
    if (phase_ != 0) throw Error(FF_ERR_LOGIC, "the state can be exported between frames only");
    // every frame computed so far, and the pipelined downloads of their flows, have finished
    wait_done();
    if (pipe_) {
        check_cuda(cudaStreamSynchronize(pipe_->out), "export state");
        check_cuda(cudaStreamSynchronize(pipe_->in), "export state");
    }
    unsigned char* out = static_cast<unsigned char*>(host);
    StateHeader h{};
    std::memcpy(h.magic, kStateMagic, sizeof(h.magic));
    h.version = kStateVersion;
    h.kind = (uint32_t)kind_;
    h.levels = (uint32_t)L_;
    std::memcpy(out, &h, sizeof(h));
    out += sizeof(h);
    for (const Level& v : lv_) {
        const StateLevel sl{(uint32_t)v.H, (uint32_t)v.W, v.delta ? 1u : 0u, v.first ? 1u : 0u};
        std::memcpy(out, &sl, sizeof(sl));
        out += sizeof(sl);
    }
    for (const Level& v : lv_) {
        const Buf* bufs[3] = {&v.fs[cur_], &v.io[cur_], v.delta ? &v.d[cur_] : &v.fu};
        for (const Buf* b : bufs) {
            const size_t row = b->row_bytes();
            check_cuda(cudaMemcpy2DAsync(out, row, b->p, b->pitch, row, (size_t)b->h, cudaMemcpyDeviceToHost,
                                         stream_),
                       "export state");
            out += row * b->h;
        }
    }
    check_cuda(cudaStreamSynchronize(stream_), "export state");
}

void Filter::import_state(const void* host, size_t bytes) {
    if (!host) throw Error(FF_ERR_INVALID_ARGUMENT, "null state buffer");
    if (phase_ != 0) throw Error(FF_ERR_LOGIC, "the state can be imported between frames only");
    const unsigned char* in = static_cast<const unsigned char*>(host);
    StateHeader h{};
    if (bytes < sizeof(h)) throw Error(FF_ERR_SHAPE, "state image too short");
    std::memcpy(&h, in, sizeof(h));
    if (std::memcmp(h.magic, kStateMagic, sizeof(h.magic)) != 0 || h.version != kStateVersion)
        throw Error(FF_ERR_INVALID_ARGUMENT, "not a filter state image (or another version)");
    if (h.kind != (uint32_t)kind_ || h.levels != (uint32_t)L_)
        throw Error(FF_ERR_SHAPE, "state image of another filter kind or level count");
    if (bytes != state_bytes())
        throw Error(FF_ERR_SHAPE, "state image size " + std::to_string(bytes) + ", this filter's is " +
                                      std::to_string(state_bytes()));
    in += sizeof(h);
    std::vector<StateLevel> sl(L_);
    for (int l = 0; l < L_; ++l) {
        std::memcpy(&sl[l], in, sizeof(StateLevel));
        in += sizeof(StateLevel);
        const Level& v = lv_[l];
        if (sl[l].H != (uint32_t)v.H || sl[l].W != (uint32_t)v.W || sl[l].delta != (v.delta ? 1u : 0u))
            throw Error(FF_ERR_SHAPE, "state image level " + std::to_string(l) + " has another size");
    }
    // a pipelined download may still be reading the buffers the copies below overwrite
    synchronize();
    for (int l = 0; l < L_; ++l) {
        Level& v = lv_[l];
        Buf* bufs[3] = {&v.fs[cur_], &v.io[cur_], v.delta ? &v.d[cur_] : &v.fu};
        for (Buf* b : bufs) {
            const size_t row = b->row_bytes();
            check_cuda(cudaMemcpy2DAsync(b->p, b->pitch, in, row, row, (size_t)b->h, cudaMemcpyHostToDevice,
                                         stream_),
                       "import state");
            in += row * b->h;
        }
        v.first = sl[l].first != 0;
    }
    // the copies are complete before any later work on any stream reads the state
    check_cuda(cudaStreamSynchronize(stream_), "import state");
    // the frame graphs hold the levels' first-frame flags; a batch rebuilds its tables
    drop_graphs();
}

}  // namespace ffb
