#ifndef TMFQS_HOST_CORE_CONSTANTS_H
#define TMFQS_HOST_CORE_CONSTANTS_H

namespace tmfqs {
// The reference's kPi (include/tmfqs/core/constants.h:6): the double nearest pi.
inline constexpr double kPi = 3.14159265358979323846;
}

#endif
