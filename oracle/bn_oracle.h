// bn_oracle.h -- TEST INFRASTRUCTURE ONLY: scene description shared by the
// FP32 restatement (bn_oracle.cpp), the FP64 expectation (bn_fp64.cpp) and the
// Python harness (oracle/__init__.py).
#pragma once
#include <cstdint>

extern "C" {
typedef struct {
  const void *voxels;
  int dtype;              // 0 f32, 1 u8 unorm (/255), 2 f16, 3 bf16, 4 u16 unorm (/65535)
  int dims[3];
  float origin[3];
  float spacing[3];
  const float *tf;        // tfN x rgba
  int tfN;
  float domain[2];
  float baseDensity;
  float camPos[3], camDir[3], camUp[3];
  float fovy;
  float bgColor[4];
  float ambientRadiance;
  float cutPlane[4];
  int numDirLights;
  const float *dirLights; // per light: direction xyz, radiance, color rgb
  int phaseMode;          // 0 SimplePhase(0.7*rgb) (default build); 1 HGPhase (multi-scatter build)
  float anisotropy;
  float scatteringAlbedo;
  int emissionAbsorption; // 1: collision contributes TF rgb, no shadow ray (extension)
  int exactLog;           // 1: -logf instead of fastLog (extension)
  int majorantRoundUp;    // 1: majorant bumped one ulp up (precision forms)
  int compensatedAccum;   // 1: Neumaier-compensated accumulation across waves (precision forms)
  int maxVolumeBounces;   // with phaseMode 1: up to this many volume bounces (multi-scatter build)
  // principled volume coefficients (PrincipledVolume.h), enabled by `principled`
  int principled;
  float pDensity, pDensityThreshold, pDensityScale, pValueRange[2];
  float pEmissionStrength, pBlackbodyIntensity, pTemperature;
  float pScatterColor[3], pAbsorptionColor[3], pEmissionColor[3], pBlackbodyTint[3];
  // isoSurface geometry on the same field (MCIsoSurfaceAccel) with an
  // AnariMatte material of constant color and opacity, enabled by `iso`
  int iso;
  float isoValue;
  float isoColor[4];      // AnariMatte "color" (rgba; a float3 set gives alpha 1)
  float isoOpacity;       // AnariMatte "opacity"
  int noVolume;           // 1: the group holds the isosurface alone (no volume)
  int width, height;
} OrcScene;
}
