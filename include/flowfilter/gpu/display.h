/*
 * flowfilter::gpu::FlowToColor for the B200 drop-in C++ API
 * (reference: include/flowfilter/gpu/display.h:21-93, src/gpu/display.cu:20-142).
 *
 * Colour-encodes a float2 flow image into an RGBA uint8 image through a 256x256 colour
 * wheel read at (flow + maxflow) / (2 maxflow), as the reference's texture lookup does.
 * The wheel is the library's default (getColorWheelRGBA(), the reference's table) unless
 * setColorWheel() gives another table.  The reference throws bare std::exception;
 * here the same conditions throw std::invalid_argument (bad input flow, maxflow <= 0) or
 * std::logic_error (configure without an input, compute before configure), both of which
 * derive from std::exception.
 */
#ifndef FLOWFILTER_B200_GPU_DISPLAY_H_
#define FLOWFILTER_B200_GPU_DISPLAY_H_

#include "flowfilter/gpu/image.h"
#include "flowfilter/gpu/pipeline.h"
#include "flowfilter/image.h"

namespace flowfilter {
namespace gpu {

class FLOWFILTER_API FlowToColor : public Stage {
public:
    FlowToColor();
    FlowToColor(flowfilter::gpu::GPUImage inputFlow, const float maxflow);
    ~FlowToColor();

    void configure();
    void compute() override;

    void downloadColorFlow(flowfilter::image_t& colorFlow);
    void setInputFlow(flowfilter::gpu::GPUImage inputFlow);
    flowfilter::gpu::GPUImage getColorFlow();

    float getMaxFlow() const;
    void setMaxFlow(const float maxflow);

    // not in the reference: another 256x256 RGBA wheel (host image, depth 4, itemSize 1)
    void setColorWheel(flowfilter::image_t& wheel);

private:
    bool configured_ = false;
    bool inputFlowSet_ = false;
    float maxflow_ = 1.0f;
    GPUImage inputFlow_, colorFlow_, wheel_;
};

}  // namespace gpu
}  // namespace flowfilter

#endif  // FLOWFILTER_B200_GPU_DISPLAY_H_
