/*
 * flowfilter::gpu::LaxWendroffPropagator for the B200 drop-in C++ API
 * (reference: include/flowfilter/gpu/propagation.h:218-282, src/gpu/propagation.cu:506-716).
 *
 * Propagates an image (depth 1 or 4, float) along a flow field (depth 2, float) with
 * `iterations` Lax-Wendroff Y-then-X pass pairs, dt = 1/iterations; before setIterations()
 * one pass pair with dt = 0 runs, as in the reference.  The reference's FlowPropagator and
 * FlowPropagatorPayload stages are the filter's internals here (ff_stage_propagate*).
 * Errors: std::invalid_argument for bad inputs or iterations <= 0, std::logic_error for
 * configure()/compute() out of order (the reference throws bare std::exception).
 */
#ifndef FLOWFILTER_B200_GPU_PROPAGATION_H_
#define FLOWFILTER_B200_GPU_PROPAGATION_H_

#include "flowfilter/gpu/image.h"
#include "flowfilter/gpu/pipeline.h"

namespace flowfilter {
namespace gpu {

class FLOWFILTER_API LaxWendroffPropagator : public Stage {
public:
    LaxWendroffPropagator();
    LaxWendroffPropagator(flowfilter::gpu::GPUImage inputFlow, flowfilter::gpu::GPUImage inputImage);
    ~LaxWendroffPropagator();

    void configure();
    void compute() override;

    void setIterations(const int N);
    int getIterations() const;
    float getDt() const;

    void setInputFlow(flowfilter::gpu::GPUImage inputFlow);
    void setInputImage(flowfilter::gpu::GPUImage img);

    flowfilter::gpu::GPUImage getFlow();
    flowfilter::gpu::GPUImage getPropagatedImage();

private:
    int iterations_ = 0;
    float dt_ = 0.0f;
    bool inputFlowSet_ = false, inputImageSet_ = false, configured_ = false;
    GPUImage inputFlow_, inputImage_, propagated_, workspace_;
};

}  // namespace gpu
}  // namespace flowfilter

#endif  // FLOWFILTER_B200_GPU_PROPAGATION_H_
