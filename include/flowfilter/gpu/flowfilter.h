/*
 * flowfilter::gpu::{FlowFilter, DeltaFlowFilter, PyramidalFlowFilter} for the B200
 * drop-in C++ API (reference: include/flowfilter/gpu/flowfilter.h:31-332,
 * src/gpu/flowfilter.cu:23-897).
 *
 * Same constructors, methods, parameter rules and results as the reference classes; the
 * work runs in libffb200.so through the C ABI of ffb200.h.  compute() returns when the
 * frame is done, as in the reference.  getFlow() returns a GPUImage that keeps showing
 * the filter's latest flow after every later compute() (the reference returns its
 * internal buffer); downloadFlow() copies the smoothed level-0 flow to the host.
 *
 * Errors: std::invalid_argument for bad arguments and shapes, std::logic_error for calls
 * in the wrong state, std::out_of_range for level indices, std::runtime_error for CUDA
 * failures (where the reference exits the process).
 */
#ifndef FLOWFILTER_B200_GPU_FLOWFILTER_H_
#define FLOWFILTER_B200_GPU_FLOWFILTER_H_

#include <vector>

#include "flowfilter/gpu/image.h"
#include "flowfilter/gpu/pipeline.h"
#include "flowfilter/image.h"

struct ff_filter;

namespace flowfilter {
namespace gpu {

// state shared by the three filter classes (a handle on one ff_filter)
class FLOWFILTER_API FilterHandle {
public:
    FilterHandle() = default;
    ~FilterHandle();
    FilterHandle(const FilterHandle&) = delete;
    FilterHandle& operator=(const FilterHandle&) = delete;

    ff_filter* get() const;
    void reset(ff_filter* f);
    // GPUImage that getFlow() handed out, refreshed after every compute
    GPUImage alias(int which, int depth);
    void refresh();

private:
    ff_filter* f_ = nullptr;
    GPUImage alias_[3];
    bool has_alias_[3] = {false, false, false};
};

class FLOWFILTER_API FlowFilter : public Stage {
public:
    FlowFilter();
    explicit FlowFilter(flowfilter::gpu::GPUImage inputImage);
    FlowFilter(const int height, const int witdh);
    FlowFilter(const int height, const int witdh, const int smoothIterations, const float maxflow,
               const float gamma);
    ~FlowFilter();

    void configure();
    void compute() override;
    void computeImageModel();
    void computePropagation();
    void computeUpdate();

    void setInputImage(flowfilter::gpu::GPUImage inputImage);
    flowfilter::gpu::GPUImage getFlow();  // unsmoothed updated flow (flowfilter.cu:266-268)
    void loadImage(flowfilter::image_t& image);
    void downloadFlow(flowfilter::image_t& flow);
    void downloadImage(flowfilter::image_t& image);

    float getGamma() const;
    void setGamma(const float gamma);
    float getMaxFlow() const;
    void setMaxFlow(const float maxflow);
    int getSmoothIterations() const;
    void setSmoothIterations(const int N);
    void setPropagationBorder(const int border);
    int getPropagationBorder() const;
    int getPropagationIterations() const;
    int height() const;
    int width() const;

private:
    ff_filter* handle() const;
    FilterHandle h_;
    GPUImage input_;
    int height_ = 0, width_ = 0;
};

class FLOWFILTER_API DeltaFlowFilter : public Stage {
public:
    DeltaFlowFilter();
    DeltaFlowFilter(flowfilter::gpu::GPUImage inputImage, flowfilter::gpu::GPUImage inputFlow);
    ~DeltaFlowFilter();

    void configure();
    void compute() override;
    void computeImageModel();
    void computePropagation();
    void computeUpdate();

    void setInputImage(flowfilter::gpu::GPUImage inputImage);
    void setInputFlow(flowfilter::gpu::GPUImage inputFlow);
    flowfilter::gpu::GPUImage getFlow();   // smoothed flow (flowfilter.cu:545-547)
    flowfilter::gpu::GPUImage getImage();  // updated image

    float getGamma() const;
    void setGamma(const float gamma);
    float getMaxFlow() const;
    void setMaxFlow(const float maxflow);
    int getSmoothIterations() const;
    void setSmoothIterations(const int N);
    void setPropagationBorder(const int border);
    int getPropagationBorder() const;
    int getPropagationIterations() const;
    int height() const;
    int width() const;

private:
    ff_filter* handle() const;
    FilterHandle h_;
    GPUImage input_, flow_;
};

class FLOWFILTER_API PyramidalFlowFilter : public Stage {
public:
    PyramidalFlowFilter();
    PyramidalFlowFilter(const int height, const int width, const int levels);
    ~PyramidalFlowFilter();

    void configure();
    void compute() override;

    flowfilter::gpu::GPUImage getFlow();  // level-0 flow (flowfilter.cu:718-725)
    void loadImage(flowfilter::image_t& image);
    void downloadFlow(flowfilter::image_t& flow);
    void downloadImage(flowfilter::image_t& image);

    float getGamma(const int level) const;
    void setGamma(const int level, const float gamma);
    void setGamma(const std::vector<float>& gamma);
    float getMaxFlow() const;
    void setMaxFlow(const float maxflow);
    int getSmoothIterations(const int level) const;
    void setSmoothIterations(const int level, const int N);
    void setSmoothIterations(const std::vector<int>& iterations);
    void setPropagationBorder(const int border);
    int getPropagationBorder() const;
    int height() const;
    int width() const;
    int levels() const;

private:
    ff_filter* handle() const;
    FilterHandle h_;
    int height_ = 0, width_ = 0, levels_ = 0;
};

}  // namespace gpu
}  // namespace flowfilter

#endif  // FLOWFILTER_B200_GPU_FLOWFILTER_H_
