// C++ drop-in classes (include/flowfilter/...) over the C ABI of libffb200.so.
//
// Each class keeps the reference's names, arguments and error types; all device work is
// done by the ff_* entry points.  Built as libflowfilter_gpu.so, the library name the
// reference's callers link against.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <stdexcept>
#include <string>

#include "ffb200.h"
#include "flowfilter/colorwheel.h"
#include "flowfilter/gpu/camera.h"
#include "flowfilter/gpu/display.h"
#include "flowfilter/gpu/flowfilter.h"
#include "flowfilter/gpu/flowsmoothing.h"
#include "flowfilter/gpu/image.h"
#include "flowfilter/gpu/imagemodel.h"
#include "flowfilter/gpu/pipeline.h"
#include "flowfilter/gpu/propagation.h"
#include "flowfilter/gpu/pyramid.h"
#include "flowfilter/gpu/rotation.h"
#include "flowfilter/gpu/update.h"

static_assert(sizeof(flowfilter::gpu::perspectiveCamera) == sizeof(ff_camera), "perspectiveCamera / ff_camera");

// flowfilter::image_t is passed to the C ABI as an ff_image: same fields, same layout
static_assert(sizeof(flowfilter::image_t) == sizeof(ff_image), "image_t / ff_image size");
static_assert(offsetof(flowfilter::image_t, height) == offsetof(ff_image, height), "image_t.height");
static_assert(offsetof(flowfilter::image_t, width) == offsetof(ff_image, width), "image_t.width");
static_assert(offsetof(flowfilter::image_t, depth) == offsetof(ff_image, depth), "image_t.depth");
static_assert(offsetof(flowfilter::image_t, pitch) == offsetof(ff_image, pitch), "image_t.pitch");
static_assert(offsetof(flowfilter::image_t, itemSize) == offsetof(ff_image, itemSize), "image_t.itemSize");
static_assert(offsetof(flowfilter::image_t, data) == offsetof(ff_image, data), "image_t.data");

namespace flowfilter {

// the library's colour wheel, filled when the library loads
unsigned char COLOR_WHEEL_D[COLOR_WHEEL_HEIGHT * COLOR_WHEEL_WIDTH * COLOR_WHEEL_DEPTH];
namespace {
const bool wheel_filled = ff_color_wheel_default(COLOR_WHEEL_D) == FF_OK;
}  // namespace

image_t getColorWheelRGBA() {
    image_t img;
    img.height = COLOR_WHEEL_HEIGHT;
    img.width = COLOR_WHEEL_WIDTH;
    img.depth = COLOR_WHEEL_DEPTH;
    img.itemSize = 1;
    img.pitch = (std::size_t)COLOR_WHEEL_WIDTH * COLOR_WHEEL_DEPTH;
    img.data = wheel_filled ? COLOR_WHEEL_D : nullptr;
    return img;
}

namespace gpu {

namespace {

// ff_status -> the exception type the reference throws for the same condition
void check(ff_status s, const char* where) {
    if (s == FF_OK) return;
    const std::string msg = std::string(where) + ": " + ff_last_error();
    switch (s) {
        case FF_ERR_INVALID_ARGUMENT:
        case FF_ERR_SHAPE: throw std::invalid_argument(msg);
        case FF_ERR_OUT_OF_RANGE: throw std::out_of_range(msg);
        case FF_ERR_LOGIC: throw std::logic_error(msg);
        default: throw std::runtime_error(msg);
    }
}

ff_image* as_ff(flowfilter::image_t& img) { return reinterpret_cast<ff_image*>(&img); }

void require(ff_filter* f, const char* where) {
    if (!f) throw std::logic_error(std::string(where) + ": the filter has not been configured");
}

}  // namespace

// ------------------------------------------------------------------ GPUImage
GPUImage::GPUImage() = default;

GPUImage::GPUImage(const int height, const int width, const int depth, const int itemSize) {
    if (height <= 0 || width <= 0 || depth <= 0 || itemSize <= 0)
        throw std::invalid_argument("GPUImage: height, width, depth and itemSize must be positive");
    h_ = (std::size_t)height;
    w_ = (std::size_t)width;
    depth_ = (std::size_t)depth;
    item_ = (std::size_t)itemSize;
    void* p = nullptr;
    check(ff_malloc_pitch(&p, &pitch_, w_ * depth_ * item_, h_), "GPUImage");
    buf_ = std::shared_ptr<void>(p, [](void* q) { ff_free(q); });
    clear();
}

GPUImage::~GPUImage() = default;

int GPUImage::height() const { return (int)h_; }
int GPUImage::width() const { return (int)w_; }
int GPUImage::depth() const { return (int)depth_; }
int GPUImage::pitch() const { return (int)pitch_; }
int GPUImage::itemSize() const { return (int)item_; }
void* GPUImage::data() { return buf_.get(); }
std::shared_ptr<void> GPUImage::getDeviceBuffer() { return buf_; }

bool GPUImage::compareShape(const flowfilter::image_t& img) const {
    return (std::size_t)img.height == h_ && (std::size_t)img.width == w_ && (std::size_t)img.depth == depth_ &&
           img.itemSize == item_;
}

bool GPUImage::compareShapeGPU(const flowfilter::gpu::GPUImage& img) const {
    return img.h_ == h_ && img.w_ == w_ && img.depth_ == depth_ && img.item_ == item_;
}

void GPUImage::upload(flowfilter::image_t& img) {
    if (!compareShape(img)) throw std::invalid_argument("GPUImage::upload(): shapes do not match");
    check(ff_memcpy2d(buf_.get(), pitch_, img.data, img.pitch, w_ * depth_ * item_, h_, 0), "GPUImage::upload");
}

void GPUImage::download(flowfilter::image_t& img) const {
    if (!compareShape(img)) throw std::invalid_argument("GPUImage::download(): shapes do not match");
    check(ff_memcpy2d(img.data, img.pitch, buf_.get(), pitch_, w_ * depth_ * item_, h_, 1), "GPUImage::download");
}

void GPUImage::copyFrom(flowfilter::gpu::GPUImage& img) {
    if (!compareShapeGPU(img)) throw std::invalid_argument("GPUImage::copyFrom(): shapes do not match");
    check(ff_memcpy2d(buf_.get(), pitch_, img.buf_.get(), img.pitch_, w_ * depth_ * item_, h_, 2),
          "GPUImage::copyFrom");
}

void GPUImage::clear() {
    if (buf_) check(ff_memset2d(buf_.get(), pitch_, 0, w_ * depth_ * item_, h_), "GPUImage::clear");
}

// ------------------------------------------------------------------ Stage
struct Stage::Events {
    cudaEvent_t start = nullptr, stop = nullptr;
    ~Events() {
        if (start) cudaEventDestroy(start);
        if (stop) cudaEventDestroy(stop);
    }
};

Stage::Stage() = default;
Stage::Stage(void* stream) : stream_(stream) {}
Stage::~Stage() = default;

void Stage::startTiming() {
    if (!events_) {
        auto e = std::make_shared<Events>();
        if (cudaEventCreate(&e->start) != cudaSuccess || cudaEventCreate(&e->stop) != cudaSuccess)
            throw std::runtime_error("Stage: cudaEventCreate failed");
        events_ = e;
    }
    if (cudaEventRecord(events_->start, (cudaStream_t)stream_) != cudaSuccess)
        throw std::runtime_error("Stage::startTiming(): cudaEventRecord failed");
}

void Stage::stopTiming() {
    if (!events_) throw std::logic_error("Stage::stopTiming(): startTiming() was not called");
    if (cudaEventRecord(events_->stop, (cudaStream_t)stream_) != cudaSuccess ||
        cudaEventSynchronize(events_->stop) != cudaSuccess ||
        cudaEventElapsedTime(&elapsed_, events_->start, events_->stop) != cudaSuccess)
        throw std::runtime_error("Stage::stopTiming(): CUDA event failure");
}

float Stage::elapsedTime() const { return elapsed_; }

EmptyStage::EmptyStage() = default;
void EmptyStage::configure() {}
void EmptyStage::compute() {
    startTiming();
    stopTiming();
}

// ------------------------------------------------------------------ ImageModel
ImageModel::ImageModel() = default;

ImageModel::ImageModel(GPUImage inputImage) {
    setInputImage(inputImage);
    configure();
}

ImageModel::~ImageModel() = default;

void ImageModel::setInputImage(GPUImage img) {
    if (img.depth() != 1) throw std::invalid_argument("ImageModel::setInputImage(): input image should have depth 1");
    if (img.itemSize() != 1 && img.itemSize() != 4)
        throw std::invalid_argument("ImageModel::setInputImage(): item size should be 1 or 4");
    input_ = img;
    configured_ = false;
}

void ImageModel::configure() {
    if (!input_.data()) throw std::logic_error("ImageModel::configure(): input image has not been set");
    constant_ = GPUImage(input_.height(), input_.width(), 1, sizeof(float));
    gradient_ = GPUImage(input_.height(), input_.width(), 2, sizeof(float));
    configured_ = true;
}

void ImageModel::compute() {
    if (!configured_) throw std::logic_error("ImageModel::compute(): stage not configured");
    startTiming();
    check(ff_stage_image_model(input_.data(), input_.pitch(), input_.itemSize(), input_.height(), input_.width(),
                               (float*)constant_.data(), constant_.pitch(), (float*)gradient_.data(),
                               gradient_.pitch(), stream_),
          "ImageModel::compute");
    stopTiming();
}

GPUImage ImageModel::getImageConstant() { return constant_; }
GPUImage ImageModel::getImageGradient() { return gradient_; }

// ------------------------------------------------------------------ stage classes
namespace {

// a device scratch buffer of at least `bytes` (reused while large enough)
GPUImage scratch(GPUImage& ws, std::size_t bytes) {
    const int w = (int)std::max<std::size_t>(bytes, 1);
    if (!ws.data() || (std::size_t)ws.pitch() < (std::size_t)w) ws = GPUImage(1, w, 1, 1);
    return ws;
}

void need_flow(GPUImage& img, const char* where) {
    if (img.depth() != 2 || img.itemSize() != 4)
        throw std::invalid_argument(std::string(where) + ": a flow field should have depth 2 of float");
}
void need_scalar(GPUImage& img, const char* where) {
    if (img.depth() != 1 || img.itemSize() != 4)
        throw std::invalid_argument(std::string(where) + ": the field should have depth 1 of float");
}
void same_shape(GPUImage& a, GPUImage& b, const char* where) {
    if (a.height() != b.height() || a.width() != b.width())
        throw std::invalid_argument(std::string(where) + ": input buffers do not match height and width");
}

}  // namespace

// FlowSmoother (flowsmoothing.cu:20-127)
FlowSmoother::FlowSmoother() = default;
FlowSmoother::FlowSmoother(GPUImage inputFlow, const int iterations) {
    setIterations(iterations);
    setInputFlow(inputFlow);
    configure();
}
FlowSmoother::~FlowSmoother() = default;
void FlowSmoother::configure() {
    if (!input_.data()) throw std::logic_error("FlowSmoother::configure(): input flow not set");
    smoothed_ = GPUImage(input_.height(), input_.width(), 2, sizeof(float));
    smoothed_.clear();
    configured_ = true;
}
void FlowSmoother::compute() {
    if (!configured_) throw std::logic_error("FlowSmoother::compute(): stage not configured");
    GPUImage ws = scratch(workspace_, ff_stage_smooth_workspace_size(input_.height(), input_.width()));
    startTiming();
    check(ff_stage_smooth((const float*)input_.data(), input_.pitch(), input_.height(), input_.width(), iterations_,
                          (float*)smoothed_.data(), smoothed_.pitch(), ws.data(), stream_),
          "FlowSmoother::compute");
    stopTiming();
}
int FlowSmoother::getIterations() const { return iterations_; }
void FlowSmoother::setIterations(const int N) {
    if (N <= 0)
        throw std::invalid_argument("FlowSmoother::setIterations(): iterations should be greater than zero: " +
                                    std::to_string(N));
    iterations_ = N;
}
void FlowSmoother::setInputFlow(GPUImage inputFlow) {
    need_flow(inputFlow, "FlowSmoother::setInputFlow()");
    input_ = inputFlow;
}
GPUImage FlowSmoother::getSmoothedFlow() { return smoothed_; }

// ImagePyramid (pyramid.cu:20-219)
ImagePyramid::ImagePyramid() = default;
ImagePyramid::ImagePyramid(GPUImage image, const int levels) {
    setInputImage(image);
    setLevels(levels);
    configure();
}
ImagePyramid::~ImagePyramid() = default;
void ImagePyramid::configure() {
    if (!input_.data()) throw std::logic_error("ImagePyramid::configure(): input image not set");
    images_.clear();
    int h = input_.height(), w = input_.width();
    for (int l = 1; l < levels_; ++l) {
        h /= 2;
        w /= 2;
        if (h < 1 || w < 1) throw std::invalid_argument("ImagePyramid::configure(): too many levels for the image");
        images_.emplace_back(h, w, 1, input_.itemSize());
        images_.back().clear();
    }
    configured_ = true;
}
void ImagePyramid::compute() {
    if (!configured_) throw std::logic_error("ImagePyramid::compute(): stage not configured");
    startTiming();
    GPUImage prev = input_;
    for (GPUImage& img : images_) {
        check(ff_stage_pyramid_down(prev.data(), prev.pitch(), prev.itemSize(), prev.height(), prev.width(),
                                    img.data(), img.pitch(), stream_),
              "ImagePyramid::compute");
        prev = img;
    }
    stopTiming();
}
void ImagePyramid::setInputImage(GPUImage img) {
    if (img.depth() != 1 || (img.itemSize() != 1 && img.itemSize() != 4))
        throw std::invalid_argument("ImagePyramid::setInputImage(): image should have depth 1 of uint8 or float");
    input_ = img;
    configured_ = false;
}
void ImagePyramid::setLevels(const int levels) {
    if (levels <= 0)
        throw std::invalid_argument("ImagePyramid::setLevels(): levels should be greater than zero: " +
                                    std::to_string(levels));
    levels_ = levels;
    configured_ = false;
}
GPUImage ImagePyramid::getImage(int level) {
    if (level < 0 || level >= levels_)
        throw std::out_of_range("ImagePyramid::getImage(): level index out of bounds: " + std::to_string(level));
    if (level == 0) return input_;
    if (!configured_) throw std::logic_error("ImagePyramid::getImage(): stage not configured");
    return images_[level - 1];
}
int ImagePyramid::getLevels() const { return levels_; }

// FlowPropagator (propagation.cu:20-210)
FlowPropagator::FlowPropagator() = default;
FlowPropagator::FlowPropagator(GPUImage inputFlow, const int iterations) {
    setIterations(iterations);
    setInputFlow(inputFlow);
    configure();
}
FlowPropagator::~FlowPropagator() = default;
void FlowPropagator::configure() {
    if (!input_.data()) throw std::logic_error("FlowPropagator::configure(): input flow not set");
    propagated_ = GPUImage(input_.height(), input_.width(), 2, sizeof(float));
    propagated_.clear();
    configured_ = true;
}
void FlowPropagator::compute() {
    if (!configured_) throw std::logic_error("FlowPropagator::compute(): stage not configured");
    GPUImage ws = scratch(workspace_, ff_stage_propagate_workspace_size(input_.height(), input_.width()));
    GPUImage src = input_;
    startTiming();
    if (invert_) {  // scalarProductF2_k with -1 (propagation.cu:92-96)
        if (!negated_.data() || negated_.height() != input_.height() || negated_.width() != input_.width())
            negated_ = GPUImage(input_.height(), input_.width(), 2, sizeof(float));
        check(ff_stage_scale_flow((const float*)input_.data(), input_.pitch(), input_.height(), input_.width(), -1.0f,
                                  (float*)negated_.data(), negated_.pitch(), stream_),
              "FlowPropagator::compute");
        src = negated_;
    }
    check(ff_stage_propagate((const float*)src.data(), src.pitch(), src.height(), src.width(), iterations_, border_,
                             (float*)propagated_.data(), propagated_.pitch(), ws.data(), stream_),
          "FlowPropagator::compute");
    stopTiming();
}
void FlowPropagator::setIterations(const int N) {
    if (N <= 0)
        throw std::invalid_argument("FlowPropagator::setIterations(): iterations should be greater than zero: " +
                                    std::to_string(N));
    iterations_ = N;
}
int FlowPropagator::getIterations() const { return iterations_; }
float FlowPropagator::getDt() const { return 1.0f / float(iterations_); }
void FlowPropagator::setBorder(const int border) {
    if (border < 0) throw std::invalid_argument("FlowPropagator::setBorder(): border should be >= 0");
    border_ = border;
}
int FlowPropagator::getBorder() const { return border_; }
void FlowPropagator::setInvertInputFlow(const bool invert) { invert_ = invert; }
bool FlowPropagator::getInvertInputFlow() const { return invert_; }
void FlowPropagator::setInputFlow(GPUImage inputFlow) {
    need_flow(inputFlow, "FlowPropagator::setInputFlow()");
    input_ = inputFlow;
}
GPUImage FlowPropagator::getPropagatedFlow() { return propagated_; }

// FlowPropagatorPayload (propagation.cu:212-412)
FlowPropagatorPayload::FlowPropagatorPayload() = default;
FlowPropagatorPayload::FlowPropagatorPayload(GPUImage inputFlow, GPUImage scalarPayload, GPUImage vectorPayload,
                                             const int iterations) {
    setIterations(iterations);
    setInputFlow(inputFlow);
    setScalarPayload(scalarPayload);
    setVectorPayload(vectorPayload);
    configure();
}
FlowPropagatorPayload::~FlowPropagatorPayload() = default;
void FlowPropagatorPayload::configure() {
    if (!flow_.data() || !scalar_.data() || !vector_.data())
        throw std::logic_error("FlowPropagatorPayload::configure(): inputs not set");
    same_shape(flow_, scalar_, "FlowPropagatorPayload::configure()");
    same_shape(flow_, vector_, "FlowPropagatorPayload::configure()");
    flowOut_ = GPUImage(flow_.height(), flow_.width(), 2, sizeof(float));
    scalarOut_ = GPUImage(flow_.height(), flow_.width(), 1, sizeof(float));
    vectorOut_ = GPUImage(flow_.height(), flow_.width(), 2, sizeof(float));
    flowOut_.clear();
    scalarOut_.clear();
    vectorOut_.clear();
    configured_ = true;
}
void FlowPropagatorPayload::compute() {
    if (!configured_) throw std::logic_error("FlowPropagatorPayload::compute(): stage not configured");
    GPUImage ws = scratch(workspace_, ff_stage_propagate_payload_workspace_size(flow_.height(), flow_.width()));
    startTiming();
    check(ff_stage_propagate_payload((const float*)flow_.data(), flow_.pitch(), (const float*)scalar_.data(),
                                     scalar_.pitch(), (const float*)vector_.data(), vector_.pitch(), flow_.height(),
                                     flow_.width(), iterations_, border_, (float*)flowOut_.data(), flowOut_.pitch(),
                                     (float*)scalarOut_.data(), scalarOut_.pitch(), (float*)vectorOut_.data(),
                                     vectorOut_.pitch(), ws.data(), stream_),
          "FlowPropagatorPayload::compute");
    stopTiming();
}
void FlowPropagatorPayload::setIterations(const int N) {
    if (N <= 0)
        throw std::invalid_argument("FlowPropagatorPayload::setIterations(): iterations should be greater than zero: " +
                                    std::to_string(N));
    iterations_ = N;
}
int FlowPropagatorPayload::getIterations() const { return iterations_; }
float FlowPropagatorPayload::getDt() const { return 1.0f / float(iterations_); }
void FlowPropagatorPayload::setBorder(const int border) {
    if (border < 0) throw std::invalid_argument("FlowPropagatorPayload::setBorder(): border should be >= 0");
    border_ = border;
}
int FlowPropagatorPayload::getBorder() const { return border_; }
void FlowPropagatorPayload::setInputFlow(GPUImage img) {
    need_flow(img, "FlowPropagatorPayload::setInputFlow()");
    flow_ = img;
}
void FlowPropagatorPayload::setScalarPayload(GPUImage img) {
    need_scalar(img, "FlowPropagatorPayload::setScalarPayload()");
    scalar_ = img;
}
void FlowPropagatorPayload::setVectorPayload(GPUImage img) {
    need_flow(img, "FlowPropagatorPayload::setVectorPayload()");
    vector_ = img;
}
GPUImage FlowPropagatorPayload::getPropagatedFlow() { return flowOut_; }
GPUImage FlowPropagatorPayload::getPropagatedScalar() { return scalarOut_; }
GPUImage FlowPropagatorPayload::getPropagatedVector() { return vectorOut_; }

// FlowUpdate (update.cu:20-210)
FlowUpdate::FlowUpdate() = default;
FlowUpdate::FlowUpdate(GPUImage inputFlow, GPUImage inputImage, GPUImage inputImageGradient, const float gamma,
                       const float maxflow) {
    setGamma(gamma);
    setMaxFlow(maxflow);
    setInputFlow(inputFlow);
    setInputImage(inputImage);
    setInputImageGradient(inputImageGradient);
    configure();
}
FlowUpdate::~FlowUpdate() = default;
void FlowUpdate::configure() {
    if (!flow_.data() || !image_.data() || !gradient_.data())
        throw std::logic_error("FlowUpdate::configure(): inputs not set");
    same_shape(flow_, image_, "FlowUpdate::configure()");
    same_shape(flow_, gradient_, "FlowUpdate::configure()");
    flowUpdated_ = GPUImage(flow_.height(), flow_.width(), 2, sizeof(float));
    imageUpdated_ = GPUImage(flow_.height(), flow_.width(), 1, sizeof(float));
    flowUpdated_.clear();
    imageUpdated_.clear();
    configured_ = true;
}
void FlowUpdate::compute() {
    if (!configured_) throw std::logic_error("FlowUpdate::compute(): stage not configured");
    startTiming();
    // the old image is read from, and the new image constant written to, the updated image
    check(ff_stage_update((const float*)image_.data(), image_.pitch(), (const float*)gradient_.data(),
                          gradient_.pitch(), (const float*)imageUpdated_.data(), imageUpdated_.pitch(),
                          (const float*)flow_.data(), flow_.pitch(), flow_.height(), flow_.width(), gamma_, maxflow_,
                          (float*)flowUpdated_.data(), flowUpdated_.pitch(), (float*)imageUpdated_.data(),
                          imageUpdated_.pitch(), stream_),
          "FlowUpdate::compute");
    stopTiming();
}
float FlowUpdate::getGamma() const { return gamma_; }
void FlowUpdate::setGamma(const float gamma) {
    if (!(gamma > 0))
        throw std::invalid_argument("FlowUpdate::setGamma(): gamma should be greater than zero: " +
                                    std::to_string(gamma));
    gamma_ = gamma;
}
float FlowUpdate::getMaxFlow() const { return maxflow_; }
void FlowUpdate::setMaxFlow(const float maxflow) { maxflow_ = maxflow; }
void FlowUpdate::setInputFlow(GPUImage inputFlow) {
    need_flow(inputFlow, "FlowUpdate::setInputFlow()");
    flow_ = inputFlow;
}
void FlowUpdate::setInputImage(GPUImage image) {
    need_scalar(image, "FlowUpdate::setInputImage()");
    image_ = image;
}
void FlowUpdate::setInputImageGradient(GPUImage imageGradient) {
    need_flow(imageGradient, "FlowUpdate::setInputImageGradient()");
    gradient_ = imageGradient;
}
GPUImage FlowUpdate::getUpdatedFlow() { return flowUpdated_; }
GPUImage FlowUpdate::getUpdatedImage() { return imageUpdated_; }

// DeltaFlowUpdate (update.cu:212-420)
DeltaFlowUpdate::DeltaFlowUpdate() = default;
DeltaFlowUpdate::DeltaFlowUpdate(GPUImage inputFlow, GPUImage inputDeltaFlow, GPUImage inputOldImage,
                                 GPUImage inputImage, GPUImage inputImageGradient, const float gamma,
                                 const float maxflow) {
    setGamma(gamma);
    setMaxFlow(maxflow);
    setInputDeltaFlow(inputDeltaFlow);
    setInputFlow(inputFlow);
    setInputImageOld(inputOldImage);
    setInputImage(inputImage);
    setInputImageGradient(inputImageGradient);
    configure();
}
DeltaFlowUpdate::~DeltaFlowUpdate() = default;
void DeltaFlowUpdate::configure() {
    if (!coarse_.data() || !delta_.data() || !oldImage_.data() || !image_.data() || !gradient_.data())
        throw std::logic_error("DeltaFlowUpdate::configure(): inputs not set");
    same_shape(delta_, oldImage_, "DeltaFlowUpdate::configure()");
    same_shape(delta_, image_, "DeltaFlowUpdate::configure()");
    same_shape(delta_, gradient_, "DeltaFlowUpdate::configure()");
    flowUpdated_ = GPUImage(delta_.height(), delta_.width(), 2, sizeof(float));
    deltaUpdated_ = GPUImage(delta_.height(), delta_.width(), 2, sizeof(float));
    imageUpdated_ = GPUImage(delta_.height(), delta_.width(), 1, sizeof(float));
    flowUpdated_.clear();
    deltaUpdated_.clear();
    imageUpdated_.clear();
    configured_ = true;
}
void DeltaFlowUpdate::compute() {
    if (!configured_) throw std::logic_error("DeltaFlowUpdate::compute(): stage not configured");
    startTiming();
    check(ff_stage_delta_update((const float*)image_.data(), image_.pitch(), (const float*)gradient_.data(),
                                gradient_.pitch(), (const float*)oldImage_.data(), oldImage_.pitch(),
                                (const float*)delta_.data(), delta_.pitch(), (const float*)coarse_.data(),
                                coarse_.pitch(), coarse_.height(), coarse_.width(), delta_.height(), delta_.width(),
                                gamma_, maxflow_, (float*)flowUpdated_.data(), flowUpdated_.pitch(),
                                (float*)deltaUpdated_.data(), deltaUpdated_.pitch(), (float*)imageUpdated_.data(),
                                imageUpdated_.pitch(), stream_),
          "DeltaFlowUpdate::compute");
    stopTiming();
}
float DeltaFlowUpdate::getGamma() const { return gamma_; }
void DeltaFlowUpdate::setGamma(const float gamma) {
    if (!(gamma > 0))
        throw std::invalid_argument("DeltaFlowUpdate::setGamma(): gamma should be greater than zero: " +
                                    std::to_string(gamma));
    gamma_ = gamma;
}
float DeltaFlowUpdate::getMaxFlow() const { return maxflow_; }
void DeltaFlowUpdate::setMaxFlow(const float maxflow) { maxflow_ = maxflow; }
void DeltaFlowUpdate::setInputFlow(GPUImage inputFlow) {
    need_flow(inputFlow, "DeltaFlowUpdate::setInputFlow()");
    coarse_ = inputFlow;
}
void DeltaFlowUpdate::setInputDeltaFlow(GPUImage inputDeltaFlow) {
    need_flow(inputDeltaFlow, "DeltaFlowUpdate::setInputDeltaFlow()");
    delta_ = inputDeltaFlow;
}
void DeltaFlowUpdate::setInputImageOld(GPUImage image) {
    need_scalar(image, "DeltaFlowUpdate::setInputImageOld()");
    oldImage_ = image;
}
void DeltaFlowUpdate::setInputImage(GPUImage image) {
    need_scalar(image, "DeltaFlowUpdate::setInputImage()");
    image_ = image;
}
void DeltaFlowUpdate::setInputImageGradient(GPUImage imageGradient) {
    need_flow(imageGradient, "DeltaFlowUpdate::setInputImageGradient()");
    gradient_ = imageGradient;
}
GPUImage DeltaFlowUpdate::getUpdatedFlow() { return flowUpdated_; }
GPUImage DeltaFlowUpdate::getUpdatedDeltaFlow() { return deltaUpdated_; }
GPUImage DeltaFlowUpdate::getUpdatedImage() { return imageUpdated_; }

// ------------------------------------------------------------------ FlowToColor
FlowToColor::FlowToColor() = default;

FlowToColor::FlowToColor(GPUImage inputFlow, const float maxflow) {
    setInputFlow(inputFlow);
    setMaxFlow(maxflow);
    configure();
}

FlowToColor::~FlowToColor() = default;

void FlowToColor::configure() {
    if (!inputFlowSet_) throw std::logic_error("FlowToColor::configure(): input flow not set");
    colorFlow_ = GPUImage(inputFlow_.height(), inputFlow_.width(), 4, sizeof(unsigned char));
    configured_ = true;
}

void FlowToColor::compute() {
    if (!configured_) throw std::logic_error("FlowToColor::compute(): Stage not configured");
    startTiming();
    check(ff_flow_to_color((const float*)inputFlow_.data(), inputFlow_.pitch(), inputFlow_.height(),
                           inputFlow_.width(), maxflow_, (const unsigned char*)wheel_.data(),
                           (unsigned char*)colorFlow_.data(), colorFlow_.pitch(), stream_),
          "FlowToColor::compute");
    stopTiming();
}

void FlowToColor::downloadColorFlow(flowfilter::image_t& colorFlow) { colorFlow_.download(colorFlow); }

void FlowToColor::setInputFlow(GPUImage inputFlow) {
    if (inputFlow.depth() != 2 || inputFlow.itemSize() != sizeof(float))
        throw std::invalid_argument("FlowToColor::setInputFlow(): input flow should have depth 2 of float");
    inputFlow_ = inputFlow;
    inputFlowSet_ = true;
}

GPUImage FlowToColor::getColorFlow() { return colorFlow_; }

float FlowToColor::getMaxFlow() const { return maxflow_; }

void FlowToColor::setMaxFlow(const float maxflow) {
    if (!(maxflow > 0.0f))
        throw std::invalid_argument("FlowToColor::setMaxFlow(): maxflow should be greater than 0.0: " +
                                    std::to_string(maxflow));
    maxflow_ = maxflow;
}

void FlowToColor::setColorWheel(flowfilter::image_t& wheel) {
    if (wheel.height != COLOR_WHEEL_HEIGHT || wheel.width != COLOR_WHEEL_WIDTH || wheel.depth != COLOR_WHEEL_DEPTH ||
        wheel.itemSize != 1)
        throw std::invalid_argument("FlowToColor::setColorWheel(): the wheel should be 256x256 RGBA uint8");
    // a dense device copy (ff_flow_to_color reads the wheel as 256 rows of 1 KB)
    GPUImage w(COLOR_WHEEL_HEIGHT, COLOR_WHEEL_WIDTH, COLOR_WHEEL_DEPTH, 1);
    if ((std::size_t)w.pitch() != (std::size_t)COLOR_WHEEL_WIDTH * COLOR_WHEEL_DEPTH)
        throw std::runtime_error("FlowToColor::setColorWheel(): unexpected device row pitch");
    w.upload(wheel);
    wheel_ = w;
}

// ------------------------------------------------------------------ camera
perspectiveCamera createPerspectiveCamera(const float focalLength, const int height, const int width,
                                          const float sensorHeight, const float sensorWidth) {
    perspectiveCamera cam;
    check(ff_camera_perspective(focalLength, height, width, sensorHeight, sensorWidth,
                                reinterpret_cast<ff_camera*>(&cam)),
          "createPerspectiveCamera");
    return cam;
}

namespace {
// a second image like `like` when the run needs more than one launch, else an empty one
GPUImage lw_workspace(GPUImage& ws, GPUImage& like, int iterations) {
    if ((iterations > 0 ? iterations : 1) <= ff_lax_wendroff_max_fused()) return GPUImage();
    if (!ws.data() || !ws.compareShapeGPU(like)) ws = GPUImage(like.height(), like.width(), like.depth(), 4);
    return ws;
}
}  // namespace

// ------------------------------------------------------------------ LaxWendroffPropagator
LaxWendroffPropagator::LaxWendroffPropagator() = default;

LaxWendroffPropagator::LaxWendroffPropagator(GPUImage inputFlow, GPUImage inputImage) {
    setInputFlow(inputFlow);
    setInputImage(inputImage);
    configure();
}

LaxWendroffPropagator::~LaxWendroffPropagator() = default;

void LaxWendroffPropagator::configure() {
    if (!inputFlowSet_) throw std::logic_error("LaxWendroffPropagator::configure(): input flow has not been set");
    if (!inputImageSet_) throw std::logic_error("LaxWendroffPropagator::configure(): input image has not been set");
    propagated_ = GPUImage(inputFlow_.height(), inputFlow_.width(), inputImage_.depth(), sizeof(float));
    configured_ = true;
}

void LaxWendroffPropagator::compute() {
    if (!configured_) throw std::logic_error("LaxWendroffPropagator::compute(): stage not configured");
    GPUImage ws = lw_workspace(workspace_, propagated_, iterations_);
    startTiming();
    check(ff_lax_wendroff((const float*)inputFlow_.data(), inputFlow_.pitch(), (const float*)inputImage_.data(),
                          inputImage_.pitch(), inputImage_.depth(), inputImage_.height(), inputImage_.width(),
                          iterations_, (float*)propagated_.data(), propagated_.pitch(), (float*)ws.data(),
                          ws.data() ? ws.pitch() : 0, stream_),
          "LaxWendroffPropagator::compute");
    stopTiming();
}

void LaxWendroffPropagator::setIterations(const int N) {
    if (N <= 0)
        throw std::invalid_argument("LaxWendroffPropagator::setIterations(): iterations less than zero: " +
                                    std::to_string(N));
    iterations_ = N;
    dt_ = 1.0f / float(N);
}

int LaxWendroffPropagator::getIterations() const { return iterations_; }
float LaxWendroffPropagator::getDt() const { return dt_; }

void LaxWendroffPropagator::setInputFlow(GPUImage inputFlow) {
    if (inputFlow.depth() != 2 || inputFlow.itemSize() != 4)
        throw std::invalid_argument("LaxWendroffPropagator::setInputFlow(): input flow should have depth 2 of float");
    inputFlow_ = inputFlow;
    inputFlowSet_ = true;
}

void LaxWendroffPropagator::setInputImage(GPUImage img) {
    if ((img.depth() != 1 && img.depth() != 4) || img.itemSize() != 4)
        throw std::invalid_argument("LaxWendroffPropagator::setInputImage(): input image should have depth 1 or 4 "
                                    "of float");
    if (img.height() != inputFlow_.height() || img.width() != inputFlow_.width())
        throw std::invalid_argument("LaxWendroffPropagator::setInputImage(): image shape does not match with input "
                                    "flow");
    inputImage_ = img;
    inputImageSet_ = true;
}

GPUImage LaxWendroffPropagator::getFlow() { return inputFlow_; }
GPUImage LaxWendroffPropagator::getPropagatedImage() { return propagated_; }

// ------------------------------------------------------------------ RotationalFlowImagePredictor
RotationalFlowImagePredictor::RotationalFlowImagePredictor() = default;

RotationalFlowImagePredictor::RotationalFlowImagePredictor(perspectiveCamera cam) { setCamera(cam); }

RotationalFlowImagePredictor::RotationalFlowImagePredictor(perspectiveCamera cam, GPUImage inputImage) {
    setCamera(cam);
    setInputImage(inputImage);
    configure();
}

RotationalFlowImagePredictor::~RotationalFlowImagePredictor() = default;

void RotationalFlowImagePredictor::configure() {
    if (!inputImageSet_) throw std::logic_error("RotationalFlowImagePredictor::configure(): input image not set");
    opticalFlow_ = GPUImage(inputImage_.height(), inputImage_.width(), 2, sizeof(float));
    predicted_ = GPUImage(inputImage_.height(), inputImage_.width(), inputImage_.depth(), sizeof(float));
    iterations_ = 0;  // a new propagator, as the reference's configure() makes
    configured_ = true;
}

void RotationalFlowImagePredictor::compute() {
    if (!configured_) throw std::logic_error("RotationalFlowImagePredictor::compute(): stage not configured");
    GPUImage ws = lw_workspace(workspace_, predicted_, iterations_);
    startTiming();
    check(ff_rotational_predict(reinterpret_cast<const ff_camera*>(&camera_), w_[0], w_[1], w_[2],
                                (const float*)inputImage_.data(), inputImage_.pitch(), inputImage_.depth(),
                                inputImage_.height(), inputImage_.width(), iterations_, (float*)opticalFlow_.data(),
                                opticalFlow_.pitch(), (float*)predicted_.data(), predicted_.pitch(), (float*)ws.data(),
                                ws.data() ? ws.pitch() : 0, stream_),
          "RotationalFlowImagePredictor::compute");
    stopTiming();
}

void RotationalFlowImagePredictor::setInputImage(GPUImage inputImage) {
    if ((inputImage.depth() != 1 && inputImage.depth() != 4) || inputImage.itemSize() != 4)
        throw std::invalid_argument("RotationalFlowImagePredictor::setInputImage(): input image should have depth 1 "
                                    "or 4 of float");
    inputImage_ = inputImage;
    inputImageSet_ = true;
}

GPUImage RotationalFlowImagePredictor::getPredictedImage() { return predicted_; }
GPUImage RotationalFlowImagePredictor::getOpticalFlow() { return opticalFlow_; }
void RotationalFlowImagePredictor::setCamera(perspectiveCamera cam) { camera_ = cam; }

void RotationalFlowImagePredictor::setAngularVelocity(const float wx, const float wy, const float wz) {
    w_[0] = wx;
    w_[1] = wy;
    w_[2] = wz;
}

void RotationalFlowImagePredictor::setIterations(const int iterations) {
    if (iterations <= 0)
        throw std::invalid_argument("LaxWendroffPropagator::setIterations(): iterations less than zero: " +
                                    std::to_string(iterations));
    iterations_ = iterations;
}

int RotationalFlowImagePredictor::getIterations() const { return iterations_; }

// ------------------------------------------------------------------ FilterHandle
FilterHandle::~FilterHandle() { reset(nullptr); }

ff_filter* FilterHandle::get() const { return f_; }

void FilterHandle::reset(ff_filter* f) {
    if (f_) ff_filter_destroy(f_);
    f_ = f;
    for (int k = 0; k < 3; ++k) {
        has_alias_[k] = false;
        alias_[k] = GPUImage();
    }
}

GPUImage FilterHandle::alias(int which, int depth) {
    if (!has_alias_[which]) {
        int h = 0, w = 0, l = 0;
        check(ff_filter_shape(f_, &h, &w, &l), "getFlow");
        alias_[which] = GPUImage(h, w, depth, sizeof(float));
        has_alias_[which] = true;
        refresh();
    }
    return alias_[which];
}

// the filter's current results live in buffers that alternate between frames; the
// GPUImages handed out keep their own buffer and are brought up to date here
void FilterHandle::refresh() {
    for (int k = 0; k < 3; ++k) {
        if (!has_alias_[k]) continue;
        void* p = nullptr;
        std::size_t pitch = 0;
        check(ff_filter_device_result(f_, k, &p, &pitch), "getFlow");
        GPUImage& a = alias_[k];
        check(ff_memcpy2d(a.data(), a.pitch(), p, pitch, (std::size_t)a.width() * a.depth() * a.itemSize(),
                          a.height(), 2),
              "getFlow");
    }
}

// ------------------------------------------------------------------ FlowFilter
FlowFilter::FlowFilter() = default;

FlowFilter::FlowFilter(GPUImage inputImage) {
    setInputImage(inputImage);
    configure();
}

FlowFilter::FlowFilter(const int height, const int width) : FlowFilter(height, width, 1, 1.0f, 1.0f) {}

FlowFilter::FlowFilter(const int height, const int width, const int smoothIterations, const float maxflow,
                       const float gamma) {
    ff_filter* f = nullptr;
    check(ff_filter_create(height, width, smoothIterations, maxflow, gamma, &f), "FlowFilter::FlowFilter");
    h_.reset(f);
    height_ = height;
    width_ = width;
}

FlowFilter::~FlowFilter() = default;

ff_filter* FlowFilter::handle() const {
    require(h_.get(), "FlowFilter");
    return h_.get();
}

void FlowFilter::setInputImage(GPUImage inputImage) {
    if (inputImage.depth() != 1)
        throw std::invalid_argument("FlowFilter::setInputImage(): input image should have depth 1, got: " +
                                    std::to_string(inputImage.depth()));
    if (inputImage.itemSize() != 1 && inputImage.itemSize() != 4)
        throw std::invalid_argument("FlowFilter::setInputImage(): item size should be 1 or 4: " +
                                    std::to_string(inputImage.itemSize()));
    input_ = inputImage;
}

void FlowFilter::configure() {
    if (!input_.data()) {
        if (h_.get()) return;  // FlowFilter(h, w, ...) owns its input and is configured
        throw std::logic_error("FlowFilter::configure(): input image has not been set");
    }
    ff_filter* f = nullptr;
    check(ff_filter_create_on_device_image(input_.data(), input_.pitch(), input_.itemSize(), input_.height(),
                                           input_.width(), &f),
          "FlowFilter::configure");
    h_.reset(f);
    height_ = input_.height();
    width_ = input_.width();
}

void FlowFilter::compute() {
    check(ff_filter_compute(handle()), "FlowFilter::compute");
    check(ff_filter_elapsed_ms(handle(), &elapsed_), "FlowFilter::compute");
    h_.refresh();
}

void FlowFilter::computeImageModel() { check(ff_filter_compute_image_model(handle()), "FlowFilter::computeImageModel"); }
void FlowFilter::computePropagation() {
    check(ff_filter_compute_propagation(handle()), "FlowFilter::computePropagation");
}
void FlowFilter::computeUpdate() {
    check(ff_filter_compute_update(handle()), "FlowFilter::computeUpdate");
    h_.refresh();
}

GPUImage FlowFilter::getFlow() { return h_.alias(1, 2); }

void FlowFilter::loadImage(flowfilter::image_t& image) {
    check(ff_filter_load_image_host(handle(), as_ff(image)), "FlowFilter::loadImage");
}
void FlowFilter::downloadFlow(flowfilter::image_t& flow) {
    check(ff_filter_download_flow_host(handle(), as_ff(flow)), "FlowFilter::downloadFlow");
}
void FlowFilter::downloadImage(flowfilter::image_t& image) {
    check(ff_filter_download_image_host(handle(), as_ff(image)), "FlowFilter::downloadImage");
}

float FlowFilter::getGamma() const {
    float g = 0.f;
    check(ff_filter_get_gamma(handle(), 0, &g), "FlowFilter::getGamma");
    return g;
}
void FlowFilter::setGamma(const float gamma) { check(ff_filter_set_gamma(handle(), 0, gamma), "FlowFilter::setGamma"); }
float FlowFilter::getMaxFlow() const {
    float m = 0.f;
    check(ff_filter_get_max_flow(handle(), &m), "FlowFilter::getMaxFlow");
    return m;
}
void FlowFilter::setMaxFlow(const float maxflow) {
    check(ff_filter_set_max_flow(handle(), maxflow), "FlowFilter::setMaxFlow");
}
int FlowFilter::getSmoothIterations() const {
    int n = 0;
    check(ff_filter_get_smooth_iterations(handle(), 0, &n), "FlowFilter::getSmoothIterations");
    return n;
}
void FlowFilter::setSmoothIterations(const int N) {
    check(ff_filter_set_smooth_iterations(handle(), 0, N), "FlowFilter::setSmoothIterations");
}
void FlowFilter::setPropagationBorder(const int border) {
    check(ff_filter_set_propagation_border(handle(), border), "FlowFilter::setPropagationBorder");
}
int FlowFilter::getPropagationBorder() const {
    int b = 0;
    check(ff_filter_get_propagation_border(handle(), &b), "FlowFilter::getPropagationBorder");
    return b;
}
int FlowFilter::getPropagationIterations() const {
    int n = 0;
    check(ff_filter_get_propagation_iterations(handle(), 0, &n), "FlowFilter::getPropagationIterations");
    return n;
}
int FlowFilter::height() const { return height_; }
int FlowFilter::width() const { return width_; }

// ------------------------------------------------------------------ DeltaFlowFilter
DeltaFlowFilter::DeltaFlowFilter() = default;

DeltaFlowFilter::DeltaFlowFilter(GPUImage inputImage, GPUImage inputFlow) {
    setInputImage(inputImage);
    setInputFlow(inputFlow);
    configure();
}

DeltaFlowFilter::~DeltaFlowFilter() = default;

ff_filter* DeltaFlowFilter::handle() const {
    require(h_.get(), "DeltaFlowFilter");
    return h_.get();
}

void DeltaFlowFilter::setInputImage(GPUImage inputImage) {
    if (inputImage.depth() != 1) throw std::invalid_argument("DeltaFlowFilter::setInputImage(): depth should be 1");
    if (inputImage.itemSize() != 1 && inputImage.itemSize() != 4)
        throw std::invalid_argument("DeltaFlowFilter::setInputImage(): item size should be 1 or 4");
    input_ = inputImage;
}

void DeltaFlowFilter::setInputFlow(GPUImage inputFlow) {
    if (inputFlow.depth() != 2 || inputFlow.itemSize() != 4)
        throw std::invalid_argument("DeltaFlowFilter::setInputFlow(): the flow should be 2 float channels");
    flow_ = inputFlow;
}

void DeltaFlowFilter::configure() {
    if (!input_.data()) throw std::logic_error("DeltaFlowFilter::configure(): input image has not been set");
    if (!flow_.data()) throw std::logic_error("DeltaFlowFilter::configure(): input flow has not been set");
    ff_filter* f = nullptr;
    check(ff_delta_filter_create(input_.data(), input_.pitch(), input_.itemSize(), input_.height(), input_.width(),
                                 flow_.data(), flow_.pitch(), flow_.height(), flow_.width(), &f),
          "DeltaFlowFilter::configure");
    h_.reset(f);
}

void DeltaFlowFilter::compute() {
    check(ff_filter_compute(handle()), "DeltaFlowFilter::compute");
    check(ff_filter_elapsed_ms(handle(), &elapsed_), "DeltaFlowFilter::compute");
    h_.refresh();
}
void DeltaFlowFilter::computeImageModel() {
    check(ff_filter_compute_image_model(handle()), "DeltaFlowFilter::computeImageModel");
}
void DeltaFlowFilter::computePropagation() {
    check(ff_filter_compute_propagation(handle()), "DeltaFlowFilter::computePropagation");
}
void DeltaFlowFilter::computeUpdate() {
    check(ff_filter_compute_update(handle()), "DeltaFlowFilter::computeUpdate");
    h_.refresh();
}

GPUImage DeltaFlowFilter::getFlow() { return h_.alias(1, 2); }
GPUImage DeltaFlowFilter::getImage() { return h_.alias(2, 1); }

float DeltaFlowFilter::getGamma() const {
    float g = 0.f;
    check(ff_filter_get_gamma(handle(), 0, &g), "DeltaFlowFilter::getGamma");
    return g;
}
void DeltaFlowFilter::setGamma(const float gamma) {
    check(ff_filter_set_gamma(handle(), 0, gamma), "DeltaFlowFilter::setGamma");
}
float DeltaFlowFilter::getMaxFlow() const {
    float m = 0.f;
    check(ff_filter_get_max_flow(handle(), &m), "DeltaFlowFilter::getMaxFlow");
    return m;
}
void DeltaFlowFilter::setMaxFlow(const float maxflow) {
    check(ff_filter_set_max_flow(handle(), maxflow), "DeltaFlowFilter::setMaxFlow");
}
int DeltaFlowFilter::getSmoothIterations() const {
    int n = 0;
    check(ff_filter_get_smooth_iterations(handle(), 0, &n), "DeltaFlowFilter::getSmoothIterations");
    return n;
}
void DeltaFlowFilter::setSmoothIterations(const int N) {
    check(ff_filter_set_smooth_iterations(handle(), 0, N), "DeltaFlowFilter::setSmoothIterations");
}
void DeltaFlowFilter::setPropagationBorder(const int border) {
    check(ff_filter_set_propagation_border(handle(), border), "DeltaFlowFilter::setPropagationBorder");
}
int DeltaFlowFilter::getPropagationBorder() const {
    int b = 0;
    check(ff_filter_get_propagation_border(handle(), &b), "DeltaFlowFilter::getPropagationBorder");
    return b;
}
int DeltaFlowFilter::getPropagationIterations() const {
    int n = 0;
    check(ff_filter_get_propagation_iterations(handle(), 0, &n), "DeltaFlowFilter::getPropagationIterations");
    return n;
}
int DeltaFlowFilter::height() const { return input_.height(); }
int DeltaFlowFilter::width() const { return input_.width(); }

// ------------------------------------------------------------------ PyramidalFlowFilter
PyramidalFlowFilter::PyramidalFlowFilter() = default;

PyramidalFlowFilter::PyramidalFlowFilter(const int height, const int width, const int levels) {
    ff_filter* f = nullptr;
    check(ff_pyramidal_create(height, width, levels, &f), "PyramidalFlowFilter::PyramidalFlowFilter");
    h_.reset(f);
    height_ = height;
    width_ = width;
    levels_ = levels;
}

PyramidalFlowFilter::~PyramidalFlowFilter() = default;

ff_filter* PyramidalFlowFilter::handle() const {
    require(h_.get(), "PyramidalFlowFilter");
    return h_.get();
}

void PyramidalFlowFilter::configure() { handle(); }

void PyramidalFlowFilter::compute() {
    check(ff_filter_compute(handle()), "PyramidalFlowFilter::compute");
    check(ff_filter_elapsed_ms(handle(), &elapsed_), "PyramidalFlowFilter::compute");
    h_.refresh();
}

GPUImage PyramidalFlowFilter::getFlow() { return h_.alias(1, 2); }

void PyramidalFlowFilter::loadImage(flowfilter::image_t& image) {
    check(ff_filter_load_image_host(handle(), as_ff(image)), "PyramidalFlowFilter::loadImage");
}
void PyramidalFlowFilter::downloadFlow(flowfilter::image_t& flow) {
    check(ff_filter_download_flow_host(handle(), as_ff(flow)), "PyramidalFlowFilter::downloadFlow");
}
void PyramidalFlowFilter::downloadImage(flowfilter::image_t& image) {
    check(ff_filter_download_image_host(handle(), as_ff(image)), "PyramidalFlowFilter::downloadImage");
}

float PyramidalFlowFilter::getGamma(const int level) const {
    float g = 0.f;
    check(ff_filter_get_gamma(handle(), level, &g), "PyramidalFlowFilter::getGamma");
    return g;
}
void PyramidalFlowFilter::setGamma(const int level, const float gamma) {
    check(ff_filter_set_gamma(handle(), level, gamma), "PyramidalFlowFilter::setGamma");
}
void PyramidalFlowFilter::setGamma(const std::vector<float>& gamma) {
    if ((int)gamma.size() != levels_)
        throw std::invalid_argument("PyramidalFlowFilter::setGamma(): gamma vector should be size " +
                                    std::to_string(levels_) + ", got: " + std::to_string(gamma.size()));
    for (int l = 0; l < levels_; ++l) setGamma(l, gamma[l]);
}
float PyramidalFlowFilter::getMaxFlow() const {
    float m = 0.f;
    check(ff_filter_get_max_flow(handle(), &m), "PyramidalFlowFilter::getMaxFlow");
    return m;
}
void PyramidalFlowFilter::setMaxFlow(const float maxflow) {
    check(ff_filter_set_max_flow(handle(), maxflow), "PyramidalFlowFilter::setMaxFlow");
}
int PyramidalFlowFilter::getSmoothIterations(const int level) const {
    int n = 0;
    check(ff_filter_get_smooth_iterations(handle(), level, &n), "PyramidalFlowFilter::getSmoothIterations");
    return n;
}
void PyramidalFlowFilter::setSmoothIterations(const int level, const int N) {
    check(ff_filter_set_smooth_iterations(handle(), level, N), "PyramidalFlowFilter::setSmoothIterations");
}
void PyramidalFlowFilter::setSmoothIterations(const std::vector<int>& iterations) {
    if ((int)iterations.size() != levels_)
        throw std::invalid_argument("PyramidalFlowFilter::setSmoothIterations(): vector should be size " +
                                    std::to_string(levels_) + ", got: " + std::to_string(iterations.size()));
    for (int l = 0; l < levels_; ++l) setSmoothIterations(l, iterations[l]);
}
void PyramidalFlowFilter::setPropagationBorder(const int border) {
    check(ff_filter_set_propagation_border(handle(), border), "PyramidalFlowFilter::setPropagationBorder");
}
int PyramidalFlowFilter::getPropagationBorder() const {
    int b = 0;
    check(ff_filter_get_propagation_border(handle(), &b), "PyramidalFlowFilter::getPropagationBorder");
    return b;
}
int PyramidalFlowFilter::height() const { return height_; }
int PyramidalFlowFilter::width() const { return width_; }
int PyramidalFlowFilter::levels() const { return levels_; }

}  // namespace gpu
}  // namespace flowfilter
