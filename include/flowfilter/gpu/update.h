/*
 * flowfilter::gpu::FlowUpdate and DeltaFlowUpdate for the B200 drop-in C++ API
 * (reference: include/flowfilter/gpu/update.h:21-169, src/gpu/update.cu:20-420).
 *
 * FlowUpdate: the regularised 2x2 update of a top level, (gamma I + a a^T)^-1 (gamma f +
 * a (old - a0)), clamped to +-maxflow; the old image is the stage's own updated-image buffer,
 * read and then overwritten with the new image constant by every compute().
 * DeltaFlowUpdate: the same solve on a propagated delta flow, clamped to +-maxflow/2, plus
 * twice the coarse flow (`inputFlow`, half the size, point-sampled at normalised
 * coordinates), clamped to +-maxflow.  Gamma is used as given (the filters scale it for uint8
 * images).  Outputs are the stage's own buffers.  Errors: std::invalid_argument for bad inputs
 * or gamma <= 0, std::logic_error for configure()/compute() out of order.
 */
#ifndef FLOWFILTER_B200_GPU_UPDATE_H_
#define FLOWFILTER_B200_GPU_UPDATE_H_

#include "flowfilter/gpu/image.h"
#include "flowfilter/gpu/pipeline.h"

namespace flowfilter {
namespace gpu {

class FLOWFILTER_API FlowUpdate : public Stage {
public:
    FlowUpdate();
    FlowUpdate(flowfilter::gpu::GPUImage inputFlow, flowfilter::gpu::GPUImage inputImage,
               flowfilter::gpu::GPUImage inputImageGradient, const float gamma = 1.0, const float maxflow = 1.0);
    ~FlowUpdate();

    void configure();
    void compute() override;

    float getGamma() const;
    void setGamma(const float gamma);
    float getMaxFlow() const;
    void setMaxFlow(const float maxflow);

    void setInputFlow(flowfilter::gpu::GPUImage inputFlow);
    void setInputImage(flowfilter::gpu::GPUImage image);
    void setInputImageGradient(flowfilter::gpu::GPUImage imageGradient);

    flowfilter::gpu::GPUImage getUpdatedFlow();
    flowfilter::gpu::GPUImage getUpdatedImage();

private:
    float gamma_ = 1.0f, maxflow_ = 1.0f;
    bool configured_ = false;
    GPUImage flow_, image_, gradient_, flowUpdated_, imageUpdated_;
};

class FLOWFILTER_API DeltaFlowUpdate : public Stage {
public:
    DeltaFlowUpdate();
    DeltaFlowUpdate(flowfilter::gpu::GPUImage inputFlow, flowfilter::gpu::GPUImage inputDeltaFlow,
                    flowfilter::gpu::GPUImage inputOldImage, flowfilter::gpu::GPUImage inputImage,
                    flowfilter::gpu::GPUImage inputImageGradient, const float gamma = 1.0,
                    const float maxflow = 1.0);
    ~DeltaFlowUpdate();

    void configure();
    void compute() override;

    float getGamma() const;
    void setGamma(const float gamma);
    float getMaxFlow() const;
    void setMaxFlow(const float maxflow);

    void setInputFlow(flowfilter::gpu::GPUImage inputFlow);
    void setInputDeltaFlow(flowfilter::gpu::GPUImage inputDeltaFlow);
    void setInputImageOld(flowfilter::gpu::GPUImage image);
    void setInputImage(flowfilter::gpu::GPUImage image);
    void setInputImageGradient(flowfilter::gpu::GPUImage imageGradient);

    flowfilter::gpu::GPUImage getUpdatedFlow();
    flowfilter::gpu::GPUImage getUpdatedDeltaFlow();
    flowfilter::gpu::GPUImage getUpdatedImage();

private:
    float gamma_ = 1.0f, maxflow_ = 1.0f;
    bool configured_ = false;
    GPUImage coarse_, delta_, oldImage_, image_, gradient_, flowUpdated_, deltaUpdated_, imageUpdated_;
};

}  // namespace gpu
}  // namespace flowfilter

#endif  // FLOWFILTER_B200_GPU_UPDATE_H_
