// TEST INFRASTRUCTURE ONLY -- stand-in for the reference's
// rtcore/cpu/Device.h (which needs embree), reduced to the declarations that
// rtcore/cpu/Texture.h uses.
#pragma once
#include "barney_rtc.h"

namespace BARNEY_NS {
namespace rtc {
struct Device {};
}  // namespace rtc
}  // namespace BARNEY_NS
