/*
 * flowfilter::gpu::ImageModel for the B200 drop-in C++ API
 * (reference: include/flowfilter/gpu/imagemodel.h:22-91, src/gpu/imagemodel.cu:25-113).
 *
 * From a uint8 or float image: the constant term a0 (float, Gaussian-smoothed image)
 * and the gradient (float2: X and Y central differences of the smoothed image).
 */
#ifndef FLOWFILTER_B200_GPU_IMAGEMODEL_H_
#define FLOWFILTER_B200_GPU_IMAGEMODEL_H_

#include "flowfilter/gpu/image.h"
#include "flowfilter/gpu/pipeline.h"

namespace flowfilter {
namespace gpu {

class FLOWFILTER_API ImageModel : public Stage {
public:
    ImageModel();
    explicit ImageModel(flowfilter::gpu::GPUImage inputImage);
    ~ImageModel();

    void configure();
    void compute() override;
    void setInputImage(flowfilter::gpu::GPUImage img);
    flowfilter::gpu::GPUImage getImageConstant();
    flowfilter::gpu::GPUImage getImageGradient();

private:
    GPUImage input_, constant_, gradient_;
    bool configured_ = false;
};

}  // namespace gpu
}  // namespace flowfilter

#endif  // FLOWFILTER_B200_GPU_IMAGEMODEL_H_
