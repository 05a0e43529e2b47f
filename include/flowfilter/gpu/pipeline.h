/*
 * flowfilter::gpu::Stage for the B200 drop-in C++ API
 * (reference: include/flowfilter/gpu/pipeline.h:29-82, src/gpu/pipeline.cu:20-88).
 *
 * Base of the filter classes: compute() and elapsedTime(), the device milliseconds of
 * the last compute().  startTiming()/stopTiming() time any work the caller queues on the
 * stage's stream in between (stopTiming waits for it).
 */
#ifndef FLOWFILTER_B200_GPU_PIPELINE_H_
#define FLOWFILTER_B200_GPU_PIPELINE_H_

#include <memory>

#include "flowfilter/image.h"

namespace flowfilter {
namespace gpu {

class FLOWFILTER_API Stage {
public:
    Stage();
    explicit Stage(void* stream);  // a cudaStream_t; nullptr = the legacy default stream
    virtual ~Stage();

    void startTiming();
    void stopTiming();
    virtual void compute() = 0;
    float elapsedTime() const;

protected:
    void* stream_ = nullptr;
    float elapsed_ = 0.0f;

private:
    struct Events;
    std::shared_ptr<Events> events_;
};

class FLOWFILTER_API EmptyStage : public Stage {
public:
    EmptyStage();
    void configure();
    void compute() override;
};

}  // namespace gpu
}  // namespace flowfilter

#endif  // FLOWFILTER_B200_GPU_PIPELINE_H_
