/*
 * flowfilter::gpu::RotationalFlowImagePredictor for the B200 drop-in C++ API
 * (reference: include/flowfilter/gpu/rotation.h:21-90, src/gpu/rotation.cu:22-124).
 *
 * The optical flow a camera rotating at (wx, wy, wz) sees (camera model from
 * createPerspectiveCamera) and the input image propagated along it with the
 * Lax-Wendroff scheme, both in one launch (ff_rotational_predict).  As in the reference,
 * configure() starts a new propagator: the iterations go back to 0 (one pass pair with
 * dt = 0) until setIterations() is called again.
 */
#ifndef FLOWFILTER_B200_GPU_ROTATION_H_
#define FLOWFILTER_B200_GPU_ROTATION_H_

#include "flowfilter/gpu/camera.h"
#include "flowfilter/gpu/image.h"
#include "flowfilter/gpu/pipeline.h"

namespace flowfilter {
namespace gpu {

class FLOWFILTER_API RotationalFlowImagePredictor : public Stage {
public:
    RotationalFlowImagePredictor();
    explicit RotationalFlowImagePredictor(perspectiveCamera cam);
    RotationalFlowImagePredictor(perspectiveCamera cam, flowfilter::gpu::GPUImage inputImage);
    ~RotationalFlowImagePredictor();

    void configure();
    void compute() override;

    void setInputImage(flowfilter::gpu::GPUImage inputImage);
    flowfilter::gpu::GPUImage getPredictedImage();
    flowfilter::gpu::GPUImage getOpticalFlow();

    void setCamera(perspectiveCamera cam);
    void setAngularVelocity(const float wx, const float wy, const float wz);
    void setIterations(const int iterations);
    int getIterations() const;

private:
    bool configured_ = false, inputImageSet_ = false;
    perspectiveCamera camera_{};
    float w_[3] = {0.0f, 0.0f, 0.0f};
    int iterations_ = 0;
    GPUImage inputImage_, opticalFlow_, predicted_, workspace_;
};

}  // namespace gpu
}  // namespace flowfilter

#endif  // FLOWFILTER_B200_GPU_ROTATION_H_
