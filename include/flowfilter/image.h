/*
 * flowfilter::image_t for the B200 drop-in C++ API.
 *
 * Same fields, order and meaning as the reference's host image descriptor
 * (include/flowfilter/image.h:30-49), and the same layout as ff_image in ffb200.h, so
 * one can be passed where the other is expected.  The memory is the caller's.
 */
#ifndef FLOWFILTER_B200_IMAGE_H_
#define FLOWFILTER_B200_IMAGE_H_

#include <cstddef>

#if defined(__GNUC__)
#define FLOWFILTER_API __attribute__((visibility("default")))
#else
#define FLOWFILTER_API
#endif

namespace flowfilter {

typedef struct {
    int height;            // pixels
    int width;             // pixels
    int depth;             // channels per pixel
    std::size_t pitch;     // bytes per row
    std::size_t itemSize;  // bytes per channel item (1 for uint8, 4 for float)
    void* data;            // host buffer
} image_t;

}  // namespace flowfilter

#endif  // FLOWFILTER_B200_IMAGE_H_
