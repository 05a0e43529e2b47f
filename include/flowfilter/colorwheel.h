/*
 * Colour wheel for the B200 drop-in C++ API (reference: include/flowfilter/colorwheel.h:14-27).
 *
 * The same names and sizes as the reference: a 256x256 RGBA table COLOR_WHEEL_D and
 * getColorWheelRGBA() viewing it, with the reference's values (ff_color_wheel_default).
 */
#ifndef FLOWFILTER_B200_COLORWHEEL_H_
#define FLOWFILTER_B200_COLORWHEEL_H_

#include "flowfilter/image.h"

namespace flowfilter {

FLOWFILTER_API extern unsigned char COLOR_WHEEL_D[];

const int COLOR_WHEEL_HEIGHT = 256;
const int COLOR_WHEEL_WIDTH = 256;
const int COLOR_WHEEL_DEPTH = 4;

FLOWFILTER_API image_t getColorWheelRGBA();

}  // namespace flowfilter

#endif  // FLOWFILTER_B200_COLORWHEEL_H_
