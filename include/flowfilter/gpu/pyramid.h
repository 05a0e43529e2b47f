/*
 * flowfilter::gpu::ImagePyramid for the B200 drop-in C++ API
 * (reference: include/flowfilter/gpu/pyramid.h:27-90, src/gpu/pyramid.cu:20-219).
 *
 * Levels of a uint8 or float image by repeated [1/4, 1/2, 1/4] X then Y passes at stride 2
 * (uint8 levels are truncated after each pass, as the reference's normalised texture reads
 * and uchar stores do).  getImage(0) is the input image itself; the other levels are the
 * stage's own buffers, written in place by every compute().  Errors: std::invalid_argument
 * for a bad input or level count, std::out_of_range for a level index outside the pyramid,
 * std::logic_error for configure()/compute() out of order.
 */
#ifndef FLOWFILTER_B200_GPU_PYRAMID_H_
#define FLOWFILTER_B200_GPU_PYRAMID_H_

#include <vector>

#include "flowfilter/gpu/image.h"
#include "flowfilter/gpu/pipeline.h"

namespace flowfilter {
namespace gpu {

class FLOWFILTER_API ImagePyramid : public Stage {
public:
    ImagePyramid();
    ImagePyramid(flowfilter::gpu::GPUImage image, const int levels);
    ~ImagePyramid();

    void configure();
    void compute() override;

    void setInputImage(flowfilter::gpu::GPUImage img);
    void setLevels(const int levels);

    flowfilter::gpu::GPUImage getImage(int level);
    int getLevels() const;

private:
    int levels_ = 1;
    bool configured_ = false;
    GPUImage input_;
    std::vector<GPUImage> images_;  // levels 1 .. levels-1
};

}  // namespace gpu
}  // namespace flowfilter

#endif  // FLOWFILTER_B200_GPU_PYRAMID_H_
