// TEST INFRASTRUCTURE ONLY -- stand-in for the reference's CPU-backend
// barney_rtc.h (rtcore/cpu/barney_rtc.h), reduced to what the compiled
// reference files need: device-code markers that expand to nothing (the CPU
// backend compiles device code as plain C++, rtcore/cpu/embree-common.h:10-11),
// rtc::float4 as a 4-float vector with rtc::load, and rtc::tex3D, which calls
// the reference's own CPU texture samplers (rtcore/cpu/Texture.cpp).
#pragma once
#define RTC_DEVICE_CODE 1
#define __rtc_device
#define __rtc_both
#define __rtc_global
#define BARNEY_RTC_CPU 1
#include "rtcore/common/rtcore-common.h"

namespace BARNEY_NS {
namespace rtc {
struct Device;
struct Buffer;
struct Group;
struct Geom;
struct GeomType;
struct TraceKernel2D;
using float4 = owl::common::vec4f;
inline owl::common::vec4f load(const float4 &v) { return v; }
float tex3D1f(TextureObject to, float x, float y, float z);
template <typename T>
T tex3D(TextureObject to, float x, float y, float z);
template <>
inline float tex3D<float>(TextureObject to, float x, float y, float z) { return tex3D1f(to, x, y, z); }
}  // namespace rtc
}  // namespace BARNEY_NS
