/*
 * flowfilter::gpu::GPUImage for the B200 drop-in C++ API
 * (reference: include/flowfilter/gpu/image.h:28-123, src/gpu/image.cu:24-200).
 *
 * A pitched device buffer held by a shared handle: copies of a GPUImage alias the same
 * memory, which is released when the last copy goes.  upload/download/copyFrom are
 * synchronous 2-D copies that honour the host image's pitch, as in the reference.
 * Errors throw std::invalid_argument (shape mismatch) or std::runtime_error (CUDA).
 */
#ifndef FLOWFILTER_B200_GPU_IMAGE_H_
#define FLOWFILTER_B200_GPU_IMAGE_H_

#include <cstddef>
#include <memory>

#include "flowfilter/image.h"

namespace flowfilter {
namespace gpu {

// typed device view of a GPUImage (reference gpuimage_t<T>)
template <typename T>
struct gpuimage_t {
    int height;
    int width;
    std::size_t pitch;
    T* data;
};

class FLOWFILTER_API GPUImage {
public:
    GPUImage();
    GPUImage(const int height, const int width, const int depth = 1, const int itemSize = sizeof(char));
    ~GPUImage();

    int height() const;
    int width() const;
    int depth() const;
    int pitch() const;
    int itemSize() const;
    void* data();

    template <typename T>
    gpuimage_t<T> wrap() {
        gpuimage_t<T> v;
        v.height = (int)h_;
        v.width = (int)w_;
        v.pitch = pitch_;
        v.data = static_cast<T*>(buf_.get());
        return v;
    }

    void upload(flowfilter::image_t& img);
    void download(flowfilter::image_t& img) const;
    void copyFrom(flowfilter::gpu::GPUImage& img);
    void clear();
    std::shared_ptr<void> getDeviceBuffer();
    bool compareShape(const flowfilter::image_t& img) const;
    bool compareShapeGPU(const flowfilter::gpu::GPUImage& img) const;

private:
    std::size_t h_ = 0, w_ = 0, depth_ = 0, pitch_ = 0, item_ = 0;
    std::shared_ptr<void> buf_;
};

}  // namespace gpu
}  // namespace flowfilter

#endif  // FLOWFILTER_B200_GPU_IMAGE_H_
