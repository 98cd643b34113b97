// barney_shim.hpp -- C++ source-level drop-in for Barney's native API.
//
// Barney's own header (barney/native/include/barney.h) declares its bn*
// functions as C++ functions inside namespace BARNEY_NS (barney_cuda,
// barney_optix or barney_cpu, chosen by barneyConfig.h.in:31-36), with
// default arguments.  Code written against that header can be rebuilt
// against barney_b200 by including this file instead: it re-exports the
// extern "C" symbols of bn_volume.h inside the same namespace, with the
// reference's default arguments.  Every bn* entry point of barney.h is
// declared; outside the structured-volume and isosurface path they record
// an "unsupported" error instead of rendering.
#pragma once
#include "bn_volume.h"

#ifndef BARNEY_NS
#define BARNEY_NS barney_cuda
#endif

namespace BARNEY_NS {
using ::BNCamera;
using ::BNContext;
using ::BNData;
using ::BNDataType;
using ::BNFrameBuffer;
using ::BNFrameBufferChannel;
using ::BNGeom;
using ::BNGroup;
using ::BNMaterial;
using ::BNSampler;
using ::BNTexture2D;
using ::BNTexture3D;
using ::BNTextureAddressMode;
using ::BNTextureColorSpace;
using ::BNTextureFilterMode;
using ::BNLight;
using ::BNModel;
using ::BNObject;
using ::BNRenderer;
using ::BNScalarField;
using ::BNTextureData;
using ::BNTransform;
using ::BNVolume;
using ::bn_float2;
using ::bn_float3;
using ::bn_float4;

using ::bnAccumReset;
using ::bnAddReference;
using ::bnBuild;
using ::bnCameraCreate;
using ::bnCommit;
using ::bnContextCreate;
using ::bnContextDestroy;
using ::bnDataCreate;
using ::bnDataSet;
using ::bnGeometryCreate;
using ::bnMaterialCreate;
using ::bnSamplerCreate;
using ::bnSet4x3fv;
using ::bnSet4x4fv;
using ::bnSetInstanceAttributes;
using ::bnSetString;
using ::bnTextureData2DCreate;
using ::bnUpdateInstanceTransforms;
using ::bnFrameBufferGetSize;
using ::bnFrameBufferRead;
using ::bnGroupBuild;
using ::bnGroupCreate;
using ::bnLightCreate;
using ::bnModelCreate;
using ::bnPhysicalDeviceCount;
using ::bnRelease;
using ::bnRender;
using ::bnScalarFieldCreate;
using ::bnSet1f;
using ::bnSet1i;
using ::bnSet2f;
using ::bnSet2i;
using ::bnSet3f;
using ::bnSet3i;
using ::bnSet4f;
using ::bnSet4i;
using ::bnSetData;
using ::bnSetInstances;
using ::bnSetObject;
using ::bnTextureData3DCreate;
using ::bnVolumeCreate;
using ::bnVolumeSetXF;

// barney.h default arguments
inline BNFrameBuffer bnFrameBufferCreate(BNContext c, int deprecated = 0) { return ::bnFrameBufferCreate(c, deprecated); }
inline BNRenderer bnRendererCreate(BNContext c, const char *type = "default") { return ::bnRendererCreate(c, type); }
inline void bnFrameBufferResize(BNFrameBuffer fb, BNDataType fmt, int sx, int sy,
                                uint32_t channels = BN_FB_COLOR) {
  ::bnFrameBufferResize(fb, fmt, sx, sy, channels);
}
inline BNTexture2D bnTexture2DCreate(BNContext c, int slot, BNDataType fmt, uint32_t sx, uint32_t sy,
                                     const void *texels, BNTextureFilterMode filter = BN_TEXTURE_LINEAR,
                                     BNTextureAddressMode ax = BN_TEXTURE_WRAP,
                                     BNTextureAddressMode ay = BN_TEXTURE_WRAP,
                                     BNTextureColorSpace cs = BN_COLOR_SPACE_LINEAR) {
  return ::bnTexture2DCreate(c, slot, fmt, sx, sy, texels, filter, ax, ay, cs);
}
inline BNTexture3D bnTexture3DCreate(BNContext c, int slot, BNDataType fmt, uint32_t sx, uint32_t sy, uint32_t sz,
                                     const void *texels, BNTextureFilterMode filter = BN_TEXTURE_LINEAR,
                                     BNTextureAddressMode a = BN_TEXTURE_CLAMP) {
  return ::bnTexture3DCreate(c, slot, fmt, sx, sy, sz, texels, filter, a);
}
// barney.h polymorphic setters
inline void bnSet(BNObject o, const char *n, bn_float2 v) { ::bnSet2f(o, n, v.x, v.y); }
inline void bnSet(BNObject o, const char *n, bn_float3 v) { ::bnSet3f(o, n, v.x, v.y, v.z); }
inline void bnSet(BNObject o, const char *n, bn_float4 v) { ::bnSet4f(o, n, v.x, v.y, v.z, v.w); }
}  // namespace BARNEY_NS
