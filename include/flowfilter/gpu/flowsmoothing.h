/*
 * flowfilter::gpu::FlowSmoother for the B200 drop-in C++ API
 * (reference: include/flowfilter/gpu/flowsmoothing.h:22-79, src/gpu/flowsmoothing.cu:20-127).
 *
 * `iterations` passes of the 5-tap box filter (weights 0.2) along X then Y over a float2
 * flow image, clamp-to-edge.  getSmoothedFlow() is the stage's own output buffer, written
 * in place by every compute().  Errors: std::invalid_argument for a bad input or
 * iterations <= 0, std::logic_error for configure()/compute() out of order (the reference
 * throws bare std::exception, or exits in compute()).
 */
#ifndef FLOWFILTER_B200_GPU_FLOWSMOOTHING_H_
#define FLOWFILTER_B200_GPU_FLOWSMOOTHING_H_

#include "flowfilter/gpu/image.h"
#include "flowfilter/gpu/pipeline.h"

namespace flowfilter {
namespace gpu {

class FLOWFILTER_API FlowSmoother : public Stage {
public:
    FlowSmoother();
    FlowSmoother(flowfilter::gpu::GPUImage inputFlow, const int iterations);
    ~FlowSmoother();

    void configure();
    void compute() override;

    int getIterations() const;
    void setIterations(const int N);

    void setInputFlow(flowfilter::gpu::GPUImage inputFlow);
    flowfilter::gpu::GPUImage getSmoothedFlow();

private:
    int iterations_ = 1;
    bool configured_ = false;
    GPUImage input_, smoothed_, workspace_;
};

}  // namespace gpu
}  // namespace flowfilter

#endif  // FLOWFILTER_B200_GPU_FLOWSMOOTHING_H_
