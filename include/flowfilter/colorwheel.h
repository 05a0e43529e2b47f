/*
 * Colour wheel for the B200 drop-in C++ API (reference: include/flowfilter/colorwheel.h:14-27).
 *
 * The same names and sizes as the reference: a 256x256 RGBA table COLOR_WHEEL_D and
 * getColorWheelRGBA() viewing it.  The values are this library's wheel (the Middlebury
 * colour code computed at texel centres, ff_color_wheel_default), a different image of the
 * same code than the reference's embedded table.
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
