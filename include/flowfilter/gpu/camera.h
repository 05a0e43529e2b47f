/*
 * Camera model for the B200 drop-in C++ API
 * (reference: include/flowfilter/gpu/camera.h:14-33, src/gpu/camera.cu:15-31).
 */
#ifndef FLOWFILTER_B200_GPU_CAMERA_H_
#define FLOWFILTER_B200_GPU_CAMERA_H_

#include "flowfilter/image.h"

namespace flowfilter {
namespace gpu {

// same fields and layout as ff_camera in ffb200.h
typedef struct {
    float alphaX;
    float alphaY;
    float centerX;
    float centerY;
} perspectiveCamera;

FLOWFILTER_API perspectiveCamera createPerspectiveCamera(const float focalLength, const int height, const int width,
                                                         const float sensorHeight, const float sensorWidth);

}  // namespace gpu
}  // namespace flowfilter

#endif  // FLOWFILTER_B200_GPU_CAMERA_H_
