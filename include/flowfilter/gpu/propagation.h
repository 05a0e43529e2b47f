/*
 * flowfilter::gpu::FlowPropagator, FlowPropagatorPayload and LaxWendroffPropagator for the
 * B200 drop-in C++ API (reference: include/flowfilter/gpu/propagation.h:26-282,
 * src/gpu/propagation.cu:20-716).
 *
 * FlowPropagator: `iterations` upwind X-then-Y sub-step pairs of a flow field by itself,
 * dt = 1/iterations, pixels within `border` (3) of the edge frozen; setInvertInputFlow
 * propagates the negated input.  FlowPropagatorPayload: the same, carrying a scalar and a
 * 2-vector field with the flow's velocities.  Outputs are the stages' own buffers.
 * LaxWendroffPropagator: an image (depth 1 or 4, float) along a flow field (depth 2, float)
 * with `iterations` Lax-Wendroff Y-then-X pass pairs, dt = 1/iterations; before
 * setIterations() one pass pair with dt = 0 runs, as in the reference.
 * Errors: std::invalid_argument for bad inputs or iterations <= 0, std::logic_error for
 * configure()/compute() out of order (the reference throws bare std::exception).
 */
#ifndef FLOWFILTER_B200_GPU_PROPAGATION_H_
#define FLOWFILTER_B200_GPU_PROPAGATION_H_

#include "flowfilter/gpu/image.h"
#include "flowfilter/gpu/pipeline.h"

namespace flowfilter {
namespace gpu {

class FLOWFILTER_API FlowPropagator : public Stage {
public:
    FlowPropagator();
    FlowPropagator(flowfilter::gpu::GPUImage inputFlow, const int iterations = 1);
    ~FlowPropagator();

    void configure();
    void compute() override;

    void setIterations(const int N);
    int getIterations() const;
    float getDt() const;
    void setBorder(const int border);
    int getBorder() const;
    void setInvertInputFlow(const bool invert);
    bool getInvertInputFlow() const;

    void setInputFlow(flowfilter::gpu::GPUImage inputFlow);
    flowfilter::gpu::GPUImage getPropagatedFlow();

private:
    int iterations_ = 1, border_ = 3;
    bool invert_ = false, configured_ = false;
    GPUImage input_, negated_, propagated_, workspace_;
};

class FLOWFILTER_API FlowPropagatorPayload : public Stage {
public:
    FlowPropagatorPayload();
    FlowPropagatorPayload(flowfilter::gpu::GPUImage inputFlow, flowfilter::gpu::GPUImage scalarPayload,
                          flowfilter::gpu::GPUImage vectorPayload, const int iterations = 1);
    ~FlowPropagatorPayload();

    void configure();
    void compute() override;

    void setIterations(const int N);
    int getIterations() const;
    float getDt() const;
    void setBorder(const int border);
    int getBorder() const;

    void setInputFlow(flowfilter::gpu::GPUImage img);
    void setScalarPayload(flowfilter::gpu::GPUImage img);
    void setVectorPayload(flowfilter::gpu::GPUImage img);

    flowfilter::gpu::GPUImage getPropagatedFlow();
    flowfilter::gpu::GPUImage getPropagatedScalar();
    flowfilter::gpu::GPUImage getPropagatedVector();

private:
    int iterations_ = 1, border_ = 3;
    bool configured_ = false;
    GPUImage flow_, scalar_, vector_, flowOut_, scalarOut_, vectorOut_, workspace_;
};

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
