#ifndef TMFQS_HOST_CORE_MATH_H
#define TMFQS_HOST_CORE_MATH_H

#include "tmfqs/core/types.h"

namespace tmfqs {

// Complex helpers (include/tmfqs/core/math.h; src/tmfqs/core/math.cpp:7-29).
Amplitude amplitudeAdd(Amplitude a, Amplitude b);
Amplitude amplitudeMultiply(Amplitude a, Amplitude b);
Amplitude complexExp(Amplitude exponent);

}  // namespace tmfqs

#endif
