// bn_kernels.cu -- sm_100a kernels of the structured-volume path.
//
//   mcBuildKernel      macrocell scalar ranges + majorants (StructuredData.cu:31-96,
//                      MCGrid.cu:97-141), fused
//   mcMapKernel        majorant re-map after a transfer-function change (mapMCs)
//   renderKernel       persistent megakernel: ray generation (generateRays.cu:43-244),
//                      box test + 3D-DDA over the macrocell grid (MCAccelerator.h:552-689,
//                      DDA.h:61-201), Woodcock tracking with software trilinear sampling
//                      and TF lookup (Volume.h:62-203, StructuredData.h:101-112,
//                      rtcore/cpu/Texture.cpp:324-416, TransferFunction.h:68-87),
//                      single-scatter shading with one shadow ray (shadeRays.cu:294-880),
//                      shadow transmittance, and per-pixel accumulation
//                      (shadeRays.cu:996-1040) -- rays never leave registers
//   resolveKernel      accum * 1/accumID -> float4 / rgba8 / sRGB (TiledFB.cu:13-52)
//
// Numerics: compiled with --fmad=false and IEEE division/sqrt so every
// expression is evaluated exactly as the reference source writes it; the
// results are bit-identical to the FP32 CPU restatement in oracle/.
//
// Work decomposition: one warp owns an 8x4 pixel tile for all waves of the
// launch; each lane owns one pixel and accumulates it in registers in wave
// order (the order the reference's per-generation launches add in).  Warps
// fetch tiles from a global counter.  Each loop iteration performs at most
// one Woodcock step, so lanes on different rays, waves or generations keep
// executing the sampling code together.
#include "bn_device.h"

#include <cuda_fp16.h>
#include <cstdint>
#include <mutex>

namespace bnb {
// The fast-math object (-DBNB_FAST_MATH, compiled with FMA contraction and
// approximate division and square root) holds the plain render kernels and
// their launchers in bnb::fastmath; macrocell builds, resolves and the
// no-allocation path exist only in the exact object.
#ifdef BNB_FAST_MATH
namespace fastmath {
#endif

#define DEV __device__ __forceinline__

// Bounds-checked build (-DBNB_BOUNDS_CHECK, libbarney_b200_bc.so): every
// indexed access of the render and macrocell kernels is checked first; an
// index outside its array is counted in g_boundsViolations and the access is
// skipped.  In the normal build BNB_IN is true and the checks compile away.
#ifdef BNB_BOUNDS_CHECK
__device__ unsigned long long g_boundsViolations;
__device__ __forceinline__ bool bnbIn(long long i, long long n) {
  if (i >= 0 && i < n) return true;
  atomicAdd(&g_boundsViolations, 1ull);
  return false;
}
#define BNB_IN(i, n) bnbIn((long long)(i), (long long)(n))
#else
#define BNB_IN(i, n) true
#endif

#define kInf __int_as_float(0x7f800000)
// math.h:13-18
#define ONE_PI_F 3.14159265358979323846f
static constexpr float kFourPi = 4.f * ONE_PI_F;
static constexpr float kOneOverFourPi = 1.f / kFourPi;

// ---------------------------------------------------------------------------
// RNG (barney-common.h:21-67)
// ---------------------------------------------------------------------------
static constexpr uint64_t kRngMul = 6364136223846793005ull;
static constexpr uint64_t kRngInit = 0xcafef00dd15ea5e5ull;

DEV uint32_t rngNext(uint64_t &state) {
  uint64_t x = state;
  unsigned count = (unsigned)(x >> 61);
  state = x * kRngMul;
  x ^= x >> 22;
  return (uint32_t)(x >> (22 + count));
}
DEV float rngFloat(uint64_t &state) { return (rngNext(state) & 0x00FFFFFFu) * (1.f / 16777216.f); }
DEV uint64_t rngSeed2(uint32_t a, uint32_t b) {
  uint64_t st = kRngInit;
  st ^= (uint32_t)(2u * a + 1u);
  rngNext(st);
  st ^= (uint32_t)(2u * b);
  rngNext(st);
  return st;
}
// Random2(RNGSeed &parent, b): child copies parent, parent advances once,
// child mixes in b.
DEV uint64_t rngDerive(uint64_t &parent, uint64_t b) {
  uint64_t child = parent;
  parent = parent * kRngMul;
  child ^= ((b ? b : 290374ull) << 1);
  rngNext(child);
  return child;
}
// hash(0,0,0) of barney-common.h:88-104: instance 0, geometry 0
static constexpr uint64_t kHash000 = (0xcbf29ce484222325ULL * 0x100000001b3ULL) * 0x100000001b3ULL;

// Volume.h:154-164
DEV float fastLog(float f) {
  f = (f - 1.f) / (f + 1.f);
  float f2 = f * f;
  float s = f;
  f *= f2;
  s += (1.f / 3.f) * f;
  f *= f2;
  s += (1.f / 5.f) * f;
  return s + s;
}

// Natural logarithm of a normal binary32 x > 0, for the exact-log free-flight
// step (bnx.exactLog).  logf differs in its last bits between CUDA and host
// libm, so the oracle and the CUDA kernels share this one evaluation:
// x = m 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s) with
// s = (m-1)/(m+1) (|s| <= 0.1716) as an odd series to s^11, plus e ln2 with
// ln2 split as 0.693145751953125 (16 significant bits, so e times it is
// exact) + 1.42860682e-6.  Within 1.7 ulp of log over (0, 1].
DEV float logPortable(float x) {
  const uint32_t b = __float_as_uint(x);
  int e = (int)((b >> 23) & 0xffu) - 127;
  float m = __uint_as_float((b & 0x7fffffu) | 0x3f800000u);
  if (m > 1.41421356f) {
    m = m * 0.5f;
    e += 1;
  }
  const float s = (m - 1.f) / (m + 1.f);
  const float z = s * s;
  const float p = 0.666666667f + z * (0.4f + z * (0.285714286f + z * (0.222222222f + z * 0.181818182f)));
  const float lm = 2.f * s + s * (z * p);
  const float fe = (float)e;
  return fe * 0.693145751953125f + (fe * 1.42860682e-6f + lm);
}

// e^x for |x| < 87 (the blackbody colour's powf), shared with the oracle like
// logPortable: k = rint(x / ln2), r = x - k ln2 (split ln2, |r| <= 0.347),
// e^r as the Taylor series to r^8 (truncation below 3e-9), times 2^k by
// exponent arithmetic.
DEV float expPortable(float x) {
  const float k = rintf(x * 1.44269504f);
  const float r = (x - k * 0.693145751953125f) - k * 1.42860682e-6f;
  const float p = 1.f + r * (1.f + r * (0.5f + r * (1.66666667e-1f + r * (4.16666667e-2f + r * (8.33333333e-3f +
                  r * (1.38888889e-3f + r * (1.98412698e-4f + r * 2.48015873e-5f)))))));
  return p * __uint_as_float((uint32_t)((int)k + 127) << 23);
}
// x^y for x > 0 (PrincipledVolume.h's powf), as e^(y log x)
DEV float powPortable(float x, float y) { return expPortable(y * logPortable(x)); }


DEV float fmin_(float a, float b) { return fminf(a, b); }
DEV float fmax_(float a, float b) { return fmaxf(a, b); }
DEV float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
DEV float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
DEV float3 normalize3(float3 v) {
  float s = 1.f / sqrtf(dot3(v, v));
  return f3(v.x * s, v.y * s, v.z * s);
}

// ---------------------------------------------------------------------------
// field sampling
// ---------------------------------------------------------------------------
template <int T>
DEV float loadVoxel(const void *p, int64_t i, const float *u8lut) {
  if (T == VOX_F32) return __ldg((const float *)p + i);
  if (T == VOX_U8) return u8lut[__ldg((const uint8_t *)p + i)];
  if (T == VOX_F16) return __half2float(__ushort_as_half(__ldg((const unsigned short *)p + i)));
  if (T == VOX_U16) {
    // x / 65535 (unorm16) without a division: q + (x - 65535 q) / 65535,
    // evaluated unfused, equals the correctly rounded quotient for every
    // 16-bit x (checked exhaustively in tests/test_oracle_kat.py)
    const float x = (float)__ldg((const unsigned short *)p + i);
    const float r = __fdiv_rn(1.f, 65535.f);
    const float q = __fmul_rn(x, r);
    return __fadd_rn(q, __fmul_rn(__fsub_rn(x, __fmul_rn(q, 65535.f)), r));
  }
  return __uint_as_float((uint32_t)__ldg((const unsigned short *)p + i) << 16);
}

// Texture.cpp:324-336
DEV void lerpCoords(int &i0, int &d, float &f, int N, float tc) {
  float u = tc - .5f;
  if (u <= 0.f) { i0 = 0; d = 0; f = 0.f; return; }
  if (u >= (float)(N - 1)) { i0 = N - 1; d = 0; f = 0.f; return; }
  int iu = (int)u;
  f = u - (float)iu;
  i0 = iu;
  d = 1;
}
// (1 - f) a + f b with each operation rounded (never fused): the trilinear
// and TF interpolations keep the reference's evaluation in the fast-math
// build too, so samples and TF lookups stay within the bar set for them
DEV float lerp_l(float f, float a, float b) { return __fadd_rn(__fmul_rn(1.f - f, a), __fmul_rn(f, b)); }

// StructuredDataSampler::DD::sample + CPU LINEAR tex3D; returns NaN outside
// The cell-space position is rounded explicitly (__fmul_rn is never fused
// into the following +.5): in the fast-math build a fused form would move the
// texel coordinate, and so the interpolation weights, by far more than the
// 2 ulp allowed for a sample.  In the exact build it is the same product.
template <int T>
DEV float sampleField(const VolumeDD &v, float3 P, const float *u8lut) {
  float rx = __fmul_rn(P.x - v.gridOrigin.x, v.rcpSpacing.x);
  float ry = __fmul_rn(P.y - v.gridOrigin.y, v.rcpSpacing.y);
  float rz = __fmul_rn(P.z - v.gridOrigin.z, v.rcpSpacing.z);
  if (rx < 0.f || ry < 0.f || rz < 0.f) return __int_as_float(0x7fc00000);
  if (rx >= (float)v.numCells.x || ry >= (float)v.numCells.y || rz >= (float)v.numCells.z)
    return __int_as_float(0x7fc00000);
  int x0, y0, z0, dx, dy, dz;
  float fx, fy, fz;
  lerpCoords(x0, dx, fx, v.numScalars.x, rx + .5f);
  lerpCoords(y0, dy, fy, v.numScalars.y, ry + .5f);
  lerpCoords(z0, dz, fz, v.numScalars.z, rz + .5f);
  const int64_t nx = v.numScalars.x, nxy = (int64_t)v.numScalars.x * v.numScalars.y;
  const int64_t b = (int64_t)x0 + nx * y0 + nxy * z0;
  const int64_t oy = dy ? nx : 0, oz = dz ? nxy : 0;
  if (!BNB_IN(b, nxy * v.numScalars.z) || !BNB_IN(b + oz + oy + dx, nxy * v.numScalars.z))
    return __int_as_float(0x7fc00000);
  float v000 = loadVoxel<T>(v.voxels, b, u8lut);
  float v001 = loadVoxel<T>(v.voxels, b + dx, u8lut);
  float v010 = loadVoxel<T>(v.voxels, b + oy, u8lut);
  float v011 = loadVoxel<T>(v.voxels, b + oy + dx, u8lut);
  float v100 = loadVoxel<T>(v.voxels, b + oz, u8lut);
  float v101 = loadVoxel<T>(v.voxels, b + oz + dx, u8lut);
  float v110 = loadVoxel<T>(v.voxels, b + oz + oy, u8lut);
  float v111 = loadVoxel<T>(v.voxels, b + oz + oy + dx, u8lut);
  float v00 = lerp_l(fx, v000, v001);
  float v01 = lerp_l(fx, v010, v011);
  float v10 = lerp_l(fx, v100, v101);
  float v11 = lerp_l(fx, v110, v111);
  float w0 = lerp_l(fy, v00, v01);
  float w1 = lerp_l(fy, v10, v11);
  return lerp_l(fz, w0, w1);
}

// ---------------------------------------------------------------------------
// macrocells (StructuredData.cu:31-62 + MCGrid.cu:97-113 + TransferFunction.h:93-117)
// ---------------------------------------------------------------------------
DEV float tfMajorant(const VolumeDD &v, float lo, float hi) {
  if (lo > hi) return 0.f;
  float span = v.domHi - v.domLo;
  float f_lo = (lo - v.domLo) / span;
  float f_hi = (hi - v.domLo) / span;
  f_lo = fmin_(1.f, fmax_(0.f, f_lo));
  f_hi = fmin_(1.f, fmax_(0.f, f_hi));
  f_lo *= (float)(v.tfN - 1);
  f_hi *= (float)(v.tfN - 1);
  int i_lo = min(v.tfN - 2, max(0, (int)f_lo));
  int i_hi = min(v.tfN - 2, max(0, (int)f_hi));
  f_lo -= (float)i_lo;
  f_hi -= (float)i_hi;
  float lerp_lo = (1.f - f_lo) * v.tf[i_lo].w + f_lo * v.tf[i_lo + 1].w;
  float lerp_hi = (1.f - f_hi) * v.tf[i_hi].w + f_hi * v.tf[i_hi + 1].w;
  float m = 0.f;
  m = fmax_(m, lerp_lo);
  m = fmax_(m, lerp_hi);
  for (int i = i_lo + 1; i <= i_hi; i++) m = fmax_(m, v.tf[i].w);
  return m * v.baseDensity;
}

// ---- principled volumes (PrincipledVolume.h:55-175) ----
DEV float clampF(float f, float lo, float hi) { return fmin_(hi, fmax_(lo, f)); }  // math.h:127
DEV float rmax3(float3 a) { return fmax_(fmax_(a.x, a.y), a.z); }
DEV float principledDensityFactor(const PrincipledDD &p, float scalar) {
  const float x = clampF(scalar, p.valueLo, p.valueHi);
  if (p.densityThreshold > 0.f && x < p.densityThreshold) return 0.f;
  return p.density * fmax_(x, 0.f) * p.densityScale;
}
DEV float3 principledSigma(float d, float3 color) { return f3(d * color.x, d * color.y, d * color.z); }
DEV float principledSigmaT(const PrincipledDD &p, float scalar) {
  const float d = principledDensityFactor(p, scalar);
  const float3 s = principledSigma(d, p.scatterColor), a = principledSigma(d, p.absorptionColor);
  return rmax3(f3(s.x + a.x, s.y + a.y, s.z + a.z));
}
// principledSampleMap's tint (its w is principledSigmaT), times rgb; not
// inlined, so that the Woodcock loop keeps its registers
__device__ __noinline__ float3 principledTintTimes(const PrincipledDD &p, float scalar, float3 rgb) {
  const float d = principledDensityFactor(p, scalar);
  const float3 s = principledSigma(d, p.scatterColor), a = principledSigma(d, p.absorptionColor);
  float3 tint = f3(1.f, 1.f, 1.f);
  if (rmax3(f3(s.x + a.x, s.y + a.y, s.z + a.z)) > 0.f) {
    const float ms = rmax3(s);
    if (ms > 0.f) tint = f3(s.x / ms, s.y / ms, s.z / ms);
  }
  return f3(tint.x * rgb.x, tint.y * rgb.y, tint.z * rgb.z);
}
DEV float3 principledBlackbodyColor(float kelvin) {
  kelvin = clampF(kelvin, 1000.f, 40000.f);
  const float t = kelvin / 100.f;
  float r, g, b;
  if (t <= 66.f) {
    r = 1.f;
    g = clampF(0.390081578f * logPortable(t) - 0.631841444f, 0.f, 1.f);
  } else {
    r = clampF(1.292936186f * powPortable(t - 60.f, -0.1332047592f), 0.f, 1.f);
    g = clampF(1.129890860f * powPortable(t - 60.f, -0.0755148492f), 0.f, 1.f);
  }
  if (t >= 66.f) b = 1.f;
  else if (t <= 19.f) b = 0.f;
  else b = clampF(0.543206789f * logPortable(t - 10.f) - 1.196254089f, 0.f, 1.f);
  return f3(r, g, b);
}
DEV float3 principledEmission(const PrincipledDD &p, float scalar) {
  const float d = principledDensityFactor(p, scalar);
  float3 Le = f3(p.emissionStrength * p.emissionColor.x * d, p.emissionStrength * p.emissionColor.y * d,
                 p.emissionStrength * p.emissionColor.z * d);
  if (p.blackbodyIntensity > 0.f && p.temperature > 0.f) {
    const float3 bb = principledBlackbodyColor(p.temperature);
    Le = f3(Le.x + p.blackbodyIntensity * p.blackbodyTint.x * bb.x * d,
            Le.y + p.blackbodyIntensity * p.blackbodyTint.y * bb.y * d,
            Le.z + p.blackbodyIntensity * p.blackbodyTint.z * bb.z * d);
  }
  return Le;
}
// sampled, not a guaranteed bound, as in the reference
DEV float principledMajorant(const PrincipledDD &p, float lo, float hi) {
  if (lo > hi) return 0.f;
  float m = 0.f;
  for (int i = 0; i <= 8; ++i) {
    const float t = float(i) / float(8);
    m = fmax_(m, principledSigmaT(p, lo + t * (hi - lo)));
  }
  return m;
}
// mapMCs (MCGrid.cu:97-113)
DEV float mapMajorant(const VolumeDD &v, float lo, float hi) {
  const float tfMaj = tfMajorant(v, lo, hi);
  return v.pv.enabled ? principledMajorant(v.pv, lo, hi) * tfMaj : tfMaj;
}

DEV float roundUpMajorant(float m, int roundUp) {
  return (roundUp && m > 0.f) ? __int_as_float(__float_as_int(m) + 1) : m;
}

#ifndef BNB_FAST_MATH
template <int T>
__global__ void __launch_bounds__(128) mcBuildKernel(VolumeDD v, float2 *ranges, float *majorants, int roundUp) {
  __shared__ float u8lut[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) u8lut[i] = __fdiv_rn((float)i * 1.f, 255.f);
  __syncthreads();
  const int64_t n = (int64_t)v.mcDims.x * v.mcDims.y * v.mcDims.z;
  for (int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; tid < n; tid += (int64_t)gridDim.x * blockDim.x) {
    const int mx = (int)(tid % v.mcDims.x);
    const int my = (int)((tid / v.mcDims.x) % v.mcDims.y);
    const int mz = (int)(tid / ((int64_t)v.mcDims.x * v.mcDims.y));
    const int x0 = mx * kCellsPerMC, y0 = my * kCellsPerMC, z0 = mz * kCellsPerMC;
    const int x1 = min(x0 + kCellsPerMC, v.numScalars.x - 1);
    const int y1 = min(y0 + kCellsPerMC, v.numScalars.y - 1);
    const int z1 = min(z0 + kCellsPerMC, v.numScalars.z - 1);
    float lo = kInf, hi = -kInf;
    const int64_t nx = v.numScalars.x, nxy = (int64_t)v.numScalars.x * v.numScalars.y;
    if (!BNB_IN(x1 + nx * y1 + nxy * z1, nxy * v.numScalars.z)) {
      // (bounds-checked build) a counted violation: an empty range and a
      // zero majorant, so the macrocell reads as empty
      ranges[tid] = make_float2(kInf, -kInf);
      if (majorants) majorants[tid] = 0.f;
      continue;
    }
    for (int z = z0; z <= z1; z++)
      for (int y = y0; y <= y1; y++) {
        const int64_t row = nx * y + nxy * z;
        for (int x = x0; x <= x1; x++) {
          float f = loadVoxel<T>(v.voxels, row + x, u8lut);
          lo = fmin_(lo, f);
          hi = fmax_(hi, f);
        }
      }
    ranges[tid] = make_float2(lo, hi);
    if (majorants) majorants[tid] = roundUpMajorant(mapMajorant(v, lo, hi), roundUp);
  }
}

__global__ void mcMapKernel(VolumeDD v, const float2 *ranges, float *majorants, int roundUp) {
  const int64_t n = (int64_t)v.mcDims.x * v.mcDims.y * v.mcDims.z;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float2 r = ranges[i];
    majorants[i] = roundUpMajorant(mapMajorant(v, r.x, r.y), roundUp);
  }
}
#endif  // !BNB_FAST_MATH

// ---------------------------------------------------------------------------
// render megakernel
// ---------------------------------------------------------------------------

// Per-lane state of the ray being traced.
struct TraceState {
  float3 org, dir;      // object-space ray, zero components of dir set to 1e-6
  float rayTMax;        // ray.tMax (PRD), clamps every Woodcock range
  float ddaTMax;        // tRange.upper after the box test, DDA's tMax
  float rayT0;          // DDA ray_t0
  float nextCellBegin;
  float3 tNext, tStep;
  int cx, cy, cz;
  int bits;             // 1/2/4: DDA direction > 0 on x/y/z; 8/16/32: component fixed up from 0
  uint64_t rng;         // Random rng of isProg
  float t, tUpper, maj; // current Woodcock range
};

// Ray.h:170-181
DEV bool boxTest(float3 org, float3 dir, float &t0, float &t1, float3 lo, float3 hi) {
  float rx = 1.f / dir.x, ry = 1.f / dir.y, rz = 1.f / dir.z;
  float lx = (lo.x - org.x) * rx, ly = (lo.y - org.y) * ry, lz = (lo.z - org.z) * rz;
  float hx = (hi.x - org.x) * rx, hy = (hi.y - org.y) * ry, hz = (hi.z - org.z) * rz;
  float nx = fmin_(lx, hx), ny = fmin_(ly, hy), nz = fmin_(lz, hz);
  float fx = fmax_(lx, hx), fy = fmax_(ly, hy), fz = fmax_(lz, hz);
  t0 = fmax_(t0, fmax_(fmax_(nx, ny), nz));
  t1 = fmin_(t1, fmin_(fmin_(fx, fy), fz));
  return t0 <= t1;
}

// TraceRays::run fix-up + isProg prologue + dda3 set-up (DDA.h:68-171).
// Returns false if the ray has no cell to visit.  raySeed is advanced when
// the box test passes (Random rng(ray.rngSeed, ...), MCAccelerator.h:592).
DEV bool traceBegin(const VolumeDD &v, TraceState &ts, float3 org, float3 dir, float tMax, uint64_t &raySeed) {
  const int fixed = (dir.x == 0.f ? 8 : 0) | (dir.y == 0.f ? 16 : 0) | (dir.z == 0.f ? 32 : 0);
  if (dir.x == 0.f) dir.x = 1e-6f;
  if (dir.y == 0.f) dir.y = 1e-6f;
  if (dir.z == 0.f) dir.z = 1e-6f;
  ts.org = org;
  ts.dir = dir;
  ts.rayTMax = tMax;
  float t0 = 0.f, t1 = tMax;
  if (!boxTest(org, dir, t0, t1, v.boundsLo, v.boundsHi)) return false;
  const float3 o = f3((org.x - v.mcOrigin.x) * v.rcpMcSpacing.x, (org.y - v.mcOrigin.y) * v.rcpMcSpacing.y,
                      (org.z - v.mcOrigin.z) * v.rcpMcSpacing.z);
  const float3 d = f3(dir.x * v.rcpMcSpacing.x, dir.y * v.rcpMcSpacing.y, dir.z * v.rcpMcSpacing.z);
  ts.rng = rngDerive(raySeed, kHash000);
  ts.ddaTMax = t1;
  // dda3
  const float3 rcpd = f3(1.f / d.x, 1.f / d.y, 1.f / d.z);
  const float3 fs = f3((float)v.mcDims.x, (float)v.mcDims.y, (float)v.mcDims.z);
  float lx = (0.f - o.x) * rcpd.x, ly = (0.f - o.y) * rcpd.y, lz = (0.f - o.z) * rcpd.z;
  float hx = (fs.x - o.x) * rcpd.x, hy = (fs.y - o.y) * rcpd.y, hz = (fs.z - o.z) * rcpd.z;
  float nx = fmin_(lx, hx), ny = fmin_(ly, hy), nz = fmin_(lz, hz);
  float fx = fmax_(lx, hx), fy = fmax_(ly, hy), fz = fmax_(lz, hz);
  if (d.x == 0.f) { if (o.x < 0.f || o.x > fs.x) return false; nx = -kInf; fx = kInf; }
  if (d.y == 0.f) { if (o.y < 0.f || o.y > fs.y) return false; ny = -kInf; fy = kInf; }
  if (d.z == 0.f) { if (o.z < 0.f || o.z > fs.z) return false; nz = -kInf; fz = kInf; }
  const float ray_t0 = fmax_(0.f, fmax_(fmax_(nx, ny), nz));
  const float ray_t1 = fmin_(t1, fmin_(fmin_(fx, fy), fz));
  if (ray_t0 > ray_t1) return false;
  const float3 oi = f3(o.x + ray_t0 * d.x, o.y + ray_t0 * d.y, o.z + ray_t0 * d.z);
  const float3 fc = f3(fmax_(0.f, fmin_(fs.x - 1.f, floorf(oi.x))), fmax_(0.f, fmin_(fs.y - 1.f, floorf(oi.y))),
                       fmax_(0.f, fmin_(fs.z - 1.f, floorf(oi.z))));
  const float3 fe = f3(d.x > 0.f ? fc.x + 1.f : fc.x, d.y > 0.f ? fc.y + 1.f : fc.y, d.z > 0.f ? fc.z + 1.f : fc.z);
  ts.tStep = f3(fabsf(rcpd.x), fabsf(rcpd.y), fabsf(rcpd.z));
  ts.tNext = f3(d.x == 0.f ? kInf : fabsf(fe.x - oi.x) * ts.tStep.x, d.y == 0.f ? kInf : fabsf(fe.y - oi.y) * ts.tStep.y,
                d.z == 0.f ? kInf : fabsf(fe.z - oi.z) * ts.tStep.z);
  // bits 0-2: DDA direction > 0 on x/y/z; bits 3-5: that component of the
  // ray direction was exactly 0 and was replaced by 1e-6 above
  ts.bits = (d.x > 0.f ? 1 : 0) | (d.y > 0.f ? 2 : 0) | (d.z > 0.f ? 4 : 0) | fixed;
  ts.cx = (int)fc.x;
  ts.cy = (int)fc.y;
  ts.cz = (int)fc.z;
  ts.rayT0 = ray_t0;
  ts.nextCellBegin = 0.f;
  return true;
}

// DDA.h:184-199: leave the current cell; false when the grid is exited
DEV bool ddaStep(const VolumeDD &v, TraceState &ts, float tClosest) {
  ts.nextCellBegin = tClosest;
  if (ts.tNext.x == tClosest) {
    ts.tNext.x += ts.tStep.x;
    ts.cx += (ts.bits & 1) ? 1 : -1;
    if (ts.cx == ((ts.bits & 1) ? v.mcDims.x : -1)) return false;
  }
  if (ts.tNext.y == tClosest) {
    ts.tNext.y += ts.tStep.y;
    ts.cy += (ts.bits & 2) ? 1 : -1;
    if (ts.cy == ((ts.bits & 2) ? v.mcDims.y : -1)) return false;
  }
  if (ts.tNext.z == tClosest) {
    ts.tNext.z += ts.tStep.z;
    ts.cz += (ts.bits & 4) ? 1 : -1;
    if (ts.cz == ((ts.bits & 4) ? v.mcDims.z : -1)) return false;
  }
  return true;
}

struct LightSample {
  float3 dir, radiance;
  float pdf;
};

// DG.h:183-193
DEV float3 randomDirection(uint64_t &rng) {
  while (true) {
    float x = 1.f - 2.f * rngFloat(rng);
    float y = 1.f - 2.f * rngFloat(rng);
    float z = 1.f - 2.f * rngFloat(rng);
    float3 v = f3(x, y, z);
    if (dot3(v, v) <= 1.f) return normalize3(v);
  }
}

// Phase.h:51-58
DEV float hgPhase(float g, float cosTheta) {
  if (fabsf(g) < 1e-3f) return kOneOverFourPi;
  float g2 = g * g;
  float denom = 1.f + g2 - 2.f * g * cosTheta;
  return kOneOverFourPi * (1.f - g2) / (denom * sqrtf(denom));
}

// sin and cos of x in [0, 2pi] (the HG sampler's azimuth).  The reference
// calls cosf/sinf, whose last bits differ between CUDA and host libm; the
// oracle and these kernels share one binary32 evaluation instead:
// Cody-Waite reduction by pi/2 = P1 + P2 + P3 (P1 has 8 significant bits, so
// j*P1 is exact) to |r| <= pi/4, then the Taylor series of sin to r^11 and
// of cos to r^12 (truncation error below 1e-10) in Horner form.
DEV void sincosPortable(float x, float &sn, float &cs) {
  const float j = rintf(x * 0.636619772f);
  const float r = ((x - j * 1.5703125f) - j * 4.83751296997070312e-4f) - j * 7.54978995e-8f;
  const float r2 = r * r;
  const float sp = r + r * (r2 * (-1.66666667e-1f + r2 * (8.33333333e-3f + r2 * (-1.98412698e-4f +
                   r2 * (2.75573192e-6f + r2 * -2.50521084e-8f)))));
  const float cp = 1.f + r2 * (-0.5f + r2 * (4.16666667e-2f + r2 * (-1.38888889e-3f + r2 * (2.48015873e-5f +
                   r2 * (-2.75573192e-7f + r2 * 2.08767570e-9f)))));
  switch ((int)j & 3) {
  case 0: sn = sp; cs = cp; break;
  case 1: sn = cp; cs = -sp; break;
  case 2: sn = -sp; cs = -cp; break;
  default: sn = -cp; cs = sp; break;
  }
}

DEV float3 cross3(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// HGPhase::sampleDirection, Phase.h:76-101 (cosf/sinf via sincosPortable)
DEV float3 hgSampleDirection(float3 wi_in, float g, uint64_t &random) {
  const float u0 = rngFloat(random);
  const float u1 = rngFloat(random);
  float cosTheta;
  if (fabsf(g) < 1e-3f) cosTheta = 1.f - 2.f * u0;
  else {
    const float sqrTerm = (1.f - g * g) / (1.f + g - 2.f * g * u0);
    cosTheta = (1.f + g * g - sqrTerm * sqrTerm) / (2.f * g);
  }
  const float sinTheta = sqrtf(fmax_(0.f, 1.f - cosTheta * cosTheta));
  const float phi = (2.f * ONE_PI_F) * u1;
  float sinPhi, cosPhi;
  sincosPortable(phi, sinPhi, cosPhi);
  const float3 local = f3(cosPhi * sinTheta, sinPhi * sinTheta, cosTheta);
  const float3 w = normalize3(wi_in);
  const float3 u = fabsf(w.x) > 0.1f ? normalize3(cross3(f3(0.f, 1.f, 0.f), w)) : normalize3(cross3(f3(1.f, 0.f, 0.f), w));
  const float3 vv = cross3(w, u);
  return normalize3(f3(local.x * u.x + local.y * vv.x + local.z * w.x, local.x * u.y + local.y * vv.y + local.z * w.y,
                       local.x * u.z + local.y * vv.z + local.z * w.z));
}

// shadeRays.cu:294-402 restricted to the constant environment and
// directional lights.  N = 0 for a volume hit; SURF instantiations take the
// front-facing normal N of a surface hit.  Returns false if no light sample;
// sets lightNeedsMIS / lightIsDirLight.
template <bool SURF = false>
DEV bool sampleLights(const FrameDD &fr, uint64_t &random, LightSample &ls, bool &needsMIS, bool &isDir,
                      float3 N = make_float3(0.f, 0.f, 0.f)) {
  needsMIS = false;
  isDir = false;
  const bool nZero = !SURF || (N.x == 0.f && N.y == 0.f && N.z == 0.f);
  // sampleEnvLight: the sphere for N = 0, else the hemisphere about N
  float3 eDir = randomDirection(random);
  if (!nZero && dot3(eDir, N) < 0.f) eDir = f3(-eDir.x, -eDir.y, -eDir.z);
  const float eRad = (nZero ? kFourPi : 2.f * ONE_PI_F) * fr.ambientRadiance;
  float elsWeight = eRad;  // reduce_max of a grey radiance
  float dlsWeight = 0.f;
  float3 dDir = f3(0.f, 0.f, 0.f), dRad = f3(0.f, 0.f, 0.f);
  if (fr.numDirLights > 0) {
    int lID[2];
    float w[2];
    float sumW = 0.f;
    for (int i = 0; i < 2; i++) {
      lID[i] = min(int(rngFloat(random) * fr.numDirLights), fr.numDirLights - 1);
      w[i] = 0.f;
      const DirLightDD &L = fr.dirLights[lID[i]];
      float3 rad = f3(L.color.x * L.radiance, L.color.y * L.radiance, L.color.z * L.radiance);
      float weight = nZero ? 1.f : dot3(L.toLight, N);
      if (!nZero && weight <= 1e-3f) continue;
      weight *= fmax_(fmax_(rad.x, rad.y), rad.z);
      if (weight <= 1e-3f) continue;
      w[i] = weight;
      sumW += weight;
    }
    if (sumW != 0.f) {
      float r = rngFloat(random) * sumW;
      int i = 0;
      while (i < 2 && r >= w[i]) { r -= w[i]; ++i; }
      if (i < 2) {
        const DirLightDD &L = fr.dirLights[lID[i]];
        dDir = L.toLight;
        const float den = w[i] / sumW * fr.dirLightPick;  // (2.f / float(numDirLights)), formed on the host
        dRad = f3(L.color.x * L.radiance * 1.f / den, L.color.y * L.radiance * 1.f / den,
                  L.color.z * L.radiance * 1.f / den);
        if (w[i] != 0.f) dlsWeight = fmax_(fmax_(dRad.x, dRad.y), dRad.z);
      }
    }
  }
  float sumWeights = 0.f + dlsWeight + elsWeight + 0.f;
  if (sumWeights == 0.f) return false;
  elsWeight *= 1.f / sumWeights;
  const float alsWeight = 0.f * (1.f / sumWeights);
  dlsWeight *= 1.f / sumWeights;
  const float plsWeight = 0.f * (1.f / sumWeights);
  const float r = rngFloat(random);
  if (r <= alsWeight) return false;  // area-light slot of an empty light list: pdf 0
  if (r <= alsWeight + elsWeight) {
    const float s = 1.f / elsWeight;
    ls.dir = eDir;
    ls.radiance = f3(eRad * s, eRad * s, eRad * s);
    ls.pdf = nZero ? kOneOverFourPi : 1.f / (2.f * ONE_PI_F);
    needsMIS = true;
    return true;
  }
  if (r <= alsWeight + elsWeight + plsWeight) return false;
  if (dlsWeight == 0.f) return false;
  const float s = 1.f / dlsWeight;
  ls.dir = dDir;
  ls.radiance = f3(dRad.x * s, dRad.y * s, dRad.z * s);
  ls.pdf = kInf;
  isDir = true;
  return true;
}

DEV float roundHalf(float x) { return __half2float(__float2half_rn(x)); }

// Neumaier-compensated sum (precision forms): sum += x, error kept in c.
DEV void neumaier(float &sum, float &c, float x) {
  const float t = sum + x;
  c += fabsf(sum) >= fabsf(x) ? (sum - t) + x : (x - t) + sum;
  sum = t;
}
DEV void accAdd(float &sum, float &c, float x, bool comp) {
  if (comp) neumaier(sum, c, x);
  else sum += x;
}

// TransferFunction::DD::map's table coordinate of a non-NaN scalar
// (TransferFunction.h:74-83): entry idx and fraction f.  The division and the
// scaling are rounded explicitly, as in sampleField: in the fast-math build an
// approximate quotient or a fused scale would move f by up to 2^-16 over a
// 256-entry table.  x/1 == x exactly, so a unit domain skips the division.
DEV void tfLocate(const VolumeDD &v, float s, int &idx, float &f) {
  const float span = v.domHi - v.domLo;
  f = span == 1.f ? (s - v.domLo) : __fdiv_rn(s - v.domLo, span);
  f = fmin_(1.f, fmax_(0.f, f));
  f = __fmul_rn(f, (float)(v.tfN - 1));
  idx = min(v.tfN - 2, max(0, (int)f));
  f -= (float)idx;
}

// Field sample of a job: compile-time voxel type, or (T < 0) the job's type.
template <int T>
DEV float sampleJob(const VolumeDD &v, float3 P, const float *u8lut) {
  if (T >= 0) return sampleField<(T < 0 ? 0 : T)>(v, P, u8lut);
  switch (v.type) {
  case VOX_F32: return sampleField<VOX_F32>(v, P, u8lut);
  case VOX_U8: return sampleField<VOX_U8>(v, P, u8lut);
  case VOX_F16: return sampleField<VOX_F16>(v, P, u8lut);
  case VOX_U16: return sampleField<VOX_U16>(v, P, u8lut);
  default: return sampleField<VOX_BF16>(v, P, u8lut);
  }
}

// ---------------------------------------------------------------------------
// isoSurface geometry (MCIsoSurfaceAccel::isProg, MCAccelerator.h:325-548)
// ---------------------------------------------------------------------------
static constexpr float kTwoPi = 2.f * ONE_PI_F;
static constexpr float kOneOverPi = 1.f / ONE_PI_F;
static constexpr float kOneOverTwoPi = 1.f / kTwoPi;

// (float)i / 10.f for i = 0..10, each the correctly rounded quotient (the
// literals below are those quotients)
__constant__ float kIsoTenths[11] = {0.f, .1f, .2f, .3f, .4f, .5f, .6f, .7f, .8f, .9f, 1.f};

// The isosurface's intersection program for one ray: box test, its own RNG
// derived from the ray's seed (which this advances), a DDA over the
// macrocell scalar ranges and, in every macrocell whose range holds the iso
// value, ten linear steps from the cell's entry to its exit, intersecting the
// first segment whose end values bracket the iso value.  The program reports
// no intersection to the traversal; it lowers only the ray's own tMax.
// dir: the ray direction after the zero fix-up; tMax: the ray's tMax.
// Returns tHit < tMax on a hit, else tMax; *seed is the ray's RNG seed,
// advanced when the box test passes.
//
// Warp-cooperative: the lanes that call it together walk their own
// macrocells, but the eleven field samples of every lane's current
// candidate macrocell are spread over all those lanes (a lane whose ray is
// done keeps sampling for the others), each taking the owner's ray through
// shuffles, into the warp's slice of isoBuf (32 x 11 floats).  Each owner
// then runs the reference's segment test over its eleven values in order.
// A sample has no side effects, so taking all eleven where the reference may
// stop early gives the same hit.  jobs/job: the ray's job (batch kernels
// sample the owner's volume).
constexpr int kIsoBufPerWarp = 32 * 11;
template <int T, bool BATCH>
DEV float isoIntersect(const JobDD *jobs, int job, const VolumeDD &v, float3 org, float3 dir, float tMax,
                       uint64_t *seed, const float *u8lut, float *isoBuf) {
  const unsigned mask = __activemask();
  const int lane = threadIdx.x & 31;
  float tHit = tMax;
  bool walking = false;  // the ray still has macrocells to walk
  uint64_t rng = 0;
  float t1 = tMax, ray_t0 = 0.f, nextCellBegin = 0.f;
  float3 tNext = f3(0.f, 0.f, 0.f), tStep = f3(0.f, 0.f, 0.f);
  int cx = 0, cy = 0, cz = 0, sx = 0, sy = 0, sz = 0, ex = 0, ey = 0, ez = 0;
  const float iso = v.iso.isoValue;
  {
    float t0 = 0.f;
    if (boxTest(org, dir, t0, t1, v.boundsLo, v.boundsHi)) {
      uint64_t raySeed = *seed;
      const float3 o = f3((org.x - v.mcOrigin.x) * v.rcpMcSpacing.x, (org.y - v.mcOrigin.y) * v.rcpMcSpacing.y,
                          (org.z - v.mcOrigin.z) * v.rcpMcSpacing.z);
      const float3 d = f3(dir.x * v.rcpMcSpacing.x, dir.y * v.rcpMcSpacing.y, dir.z * v.rcpMcSpacing.z);
      rng = rngDerive(raySeed, kHash000);  // hash(instance 0, geometry 0, primitive 0)
      *seed = raySeed;
      // dda3 (DDA.h:61-201), tMax = the box test's t1
      const float3 rcpd = f3(1.f / d.x, 1.f / d.y, 1.f / d.z);
      const float3 fs = f3((float)v.mcDims.x, (float)v.mcDims.y, (float)v.mcDims.z);
      float lx = (0.f - o.x) * rcpd.x, ly = (0.f - o.y) * rcpd.y, lz = (0.f - o.z) * rcpd.z;
      float hx = (fs.x - o.x) * rcpd.x, hy = (fs.y - o.y) * rcpd.y, hz = (fs.z - o.z) * rcpd.z;
      float nx = fmin_(lx, hx), ny = fmin_(ly, hy), nz = fmin_(lz, hz);
      float fx = fmax_(lx, hx), fy = fmax_(ly, hy), fz = fmax_(lz, hz);
      walking = true;
      if (d.x == 0.f) { if (o.x < 0.f || o.x > fs.x) walking = false; nx = -kInf; fx = kInf; }
      if (d.y == 0.f) { if (o.y < 0.f || o.y > fs.y) walking = false; ny = -kInf; fy = kInf; }
      if (d.z == 0.f) { if (o.z < 0.f || o.z > fs.z) walking = false; nz = -kInf; fz = kInf; }
      ray_t0 = fmax_(0.f, fmax_(fmax_(nx, ny), nz));
      const float ray_t1 = fmin_(t1, fmin_(fmin_(fx, fy), fz));
      if (ray_t0 > ray_t1) walking = false;
      const float3 oi = f3(o.x + ray_t0 * d.x, o.y + ray_t0 * d.y, o.z + ray_t0 * d.z);
      const float3 fc = f3(fmax_(0.f, fmin_(fs.x - 1.f, floorf(oi.x))), fmax_(0.f, fmin_(fs.y - 1.f, floorf(oi.y))),
                           fmax_(0.f, fmin_(fs.z - 1.f, floorf(oi.z))));
      const float3 fe = f3(d.x > 0.f ? fc.x + 1.f : fc.x, d.y > 0.f ? fc.y + 1.f : fc.y, d.z > 0.f ? fc.z + 1.f : fc.z);
      tStep = f3(fabsf(rcpd.x), fabsf(rcpd.y), fabsf(rcpd.z));
      tNext = f3(d.x == 0.f ? kInf : fabsf(fe.x - oi.x) * tStep.x, d.y == 0.f ? kInf : fabsf(fe.y - oi.y) * tStep.y,
                 d.z == 0.f ? kInf : fabsf(fe.z - oi.z) * tStep.z);
      cx = (int)fc.x; cy = (int)fc.y; cz = (int)fc.z;
      sx = d.x > 0.f ? 1 : -1; sy = d.y > 0.f ? 1 : -1; sz = d.z > 0.f ? 1 : -1;
      ex = d.x > 0.f ? v.mcDims.x : -1; ey = d.y > 0.f ? v.mcDims.y : -1; ez = d.z > 0.f ? v.mcDims.z : -1;
    }
  }
  // every step leaves one cell and the grid has < 2^31 cells, so each walk
  // ends; the bound only guards against a non-finite step
  int iter = 0;
  // leave the current cell (DDA.h:184-199); false when the grid is left
  auto stepCell = [&](float tClosest) -> bool {
    nextCellBegin = tClosest;
    if (tNext.x == tClosest) { tNext.x += tStep.x; cx += sx; if (cx == ex) return false; }
    if (tNext.y == tClosest) { tNext.y += tStep.y; cy += sy; if (cy == ey) return false; }
    if (tNext.z == tClosest) { tNext.z += tStep.z; cz += sz; if (cz == ez) return false; }
    return true;
  };
  const int workers = __popc(mask);
  const int wrank = __popc(mask & ((1u << lane) - 1u));
  float *buf = isoBuf;
  while (true) {
    // 1. each walking ray moves to its next candidate macrocell (range holds
    //    the iso value) or leaves the grid
    bool cand = false;
    float ct0 = 0.f, ct1 = 0.f, tClosest = 0.f;
    while (walking) {
      tClosest = fmin_(fmin_(tNext.x, tNext.y), tNext.z);
      ct0 = ray_t0 + nextCellBegin;
      ct1 = ray_t0 + fmin_(tClosest, t1);
      // the macrocell callback
      const float upper = fmin_(ct1, tMax);
      if (ct0 < upper) {
        const int rci = cx + v.mcDims.x * (cy + v.mcDims.y * cz);
        const float2 rg = BNB_IN(rci, (long long)v.mcDims.x * v.mcDims.y * v.mcDims.z)
                              ? __ldg(v.iso.ranges + rci)
                              : make_float2(1.f, 0.f);  // (bounds-checked build: an empty range)
        if (iso >= rg.x && iso <= rg.y) {
          cand = true;
          break;
        }
      }
      if (++iter >= (1 << 24) || !stepCell(tClosest)) walking = false;
    }
    const unsigned cmask = __ballot_sync(mask, cand);
    if (!cmask) break;
    // 2. the eleven samples of every candidate, spread over the warp: sample
    //    point i is the entry for i = 0, else (1 - i/10) ct0 + (i/10) ct1
    const int tasks = 11 * __popc(cmask);
    for (int k0 = 0; k0 < tasks; k0 += workers) {
      const int k = k0 + wrank;
      const int r = k < tasks ? k / 11 : 0;
      const int i = k < tasks ? k - 11 * r : 0;
      const int owner = __fns(cmask, 0, r + 1);
      const float ox = __shfl_sync(mask, org.x, owner), oy = __shfl_sync(mask, org.y, owner);
      const float oz = __shfl_sync(mask, org.z, owner);
      const float dx = __shfl_sync(mask, dir.x, owner), dy = __shfl_sync(mask, dir.y, owner);
      const float dz = __shfl_sync(mask, dir.z, owner);
      const float c0 = __shfl_sync(mask, ct0, owner), c1 = __shfl_sync(mask, ct1, owner);
      const int oj = BATCH ? __shfl_sync(mask, job, owner) : 0;
      if (k < tasks) {
        const float fi = kIsoTenths[i];
        const float tt = i == 0 ? c0 : (1.f - fi) * c0 + fi * c1;
        const VolumeDD &vo = BATCH ? jobs[oj].v : v;
        buf[owner * 11 + i] = sampleJob<T>(vo, f3(ox + tt * dx, oy + tt * dy, oz + tt * dz), u8lut);
      }
    }
    __syncwarp(mask);
    // 3. each candidate's segments in order (MCAccelerator.h:325-548): the
    //    first that brackets the iso value and lies below tMax is the hit
    if (cand) {
      float tt1 = ct0;
      float ff1 = buf[lane * 11];
      bool done = false;
#pragma unroll 1
      for (int i = 1; i <= 10; i++) {
        const float tt0 = tt1;
        const float ff0 = ff1;
        const float fi = kIsoTenths[i];  // (float)i / 10.f
        tt1 = (1.f - fi) * ct0 + fi * ct1;
        ff1 = buf[lane * 11 + i];
        if (isnan(ff0) || isnan(ff1)) continue;
        if (iso >= fmin_(ff0, ff1) && iso <= fmax_(ff0, ff1)) {
          float t = (iso - ff0) / (ff1 - ff0);
          t = (1.f - t) * tt0 + t * tt1;
          tHit = (t < tHit) ? t : tHit;  // a 0/0 segment (NaN) keeps tHit
          if (tHit < tMax) { done = true; break; }
        }
      }
      // a hit ends the walk; otherwise on to the next macrocell
      if (done || ++iter >= (1 << 24) || !stepCell(tClosest)) walking = false;
    }
    __syncwarp(mask);  // the buffer is read before the next round writes it
  }
  if (!(tHit < tMax)) return tMax;
  if (v.iso.alpha < 1.f && rngFloat(rng) > v.iso.alpha) return tMax;  // Lambertian::getOpacity
  return tHit;
}

// The hit normal (MCAccelerator.h:444-478): central differences over
// +-normalDelta, one-sided where a neighbour lies outside the field, and
// -normalize(dir) for a zero gradient; returned normalized and rounded to
// binary16, as Ray::packNormal stores it.
// pre: the seven field values at P and P -/+ normalDelta along x, y, z
// (isoNormalSamples, taken by the whole warp), or null to sample here
template <int T>
__device__ __noinline__ float3 isoNormal(const VolumeDD &v, float3 P, float3 dir, const float *u8lut,
                                         const float *pre) {
  const float dl = v.iso.normalDelta;
  const float fP = pre ? pre[0] : sampleJob<T>(v, P, u8lut);
  // central differences: samples at P -/+ dl along x, then y, then z (one
  // copy of the sampler in a loop); an axis whose sample is NaN (outside the
  // field) uses fP instead and halves its step count
  float3 n = f3(0.f, 0.f, 0.f);
  float fLo = 0.f;
#pragma unroll 1
  for (int i = 0; i < 6; i++) {
    const int axis = i >> 1;
    const float o = (i & 1) ? dl : -dl;
    const float fv = pre ? pre[1 + i]
                         : sampleJob<T>(v, f3(P.x + (axis == 0 ? o : 0.f), P.y + (axis == 1 ? o : 0.f),
                                              P.z + (axis == 2 ? o : 0.f)), u8lut);
    if (!(i & 1)) {
      fLo = fv;
      continue;
    }
    float f0 = fLo, f1 = fv, d = 2.f;
    if (isnan(f0)) { d -= 1.f; f0 = fP; }
    if (isnan(f1)) { d -= 1.f; f1 = fP; }
    const float c = d == 0.f ? 0.f : (f1 - f0) / d;
    if (axis == 0) n.x = c;
    else if (axis == 1) n.y = c;
    else n.z = c;
  }
  if (n.x == 0.f && n.y == 0.f && n.z == 0.f) {
    const float3 dn = normalize3(dir);
    n = f3(-dn.x, -dn.y, -dn.z);
  }
  n = normalize3(n);
  return f3(roundHalf(n.x), roundHalf(n.y), roundHalf(n.z));
}

// owl::common::frame(N) (embree's LinearSpace3 frame(): dx from the larger
// of (0, N.z, -N.y) and (-N.z, 0, N.x), dy = normalize(cross(N, dx))) applied
// to v: dx * v.x + dy * v.y + N * v.z
DEV float3 frameXfm(float3 N, float3 v) {
  const float3 dx0 = f3(0.f, N.z, -N.y);
  const float3 dx1 = f3(-N.z, 0.f, N.x);
  const float3 dx = normalize3(dot3(dx0, dx0) > dot3(dx1, dx1) ? dx0 : dx1);
  const float3 dy = normalize3(cross3(N, dx));
  return f3(dx.x * v.x + dy.x * v.y + N.x * v.z, dx.y * v.x + dy.y * v.y + N.y * v.z,
            dx.z * v.x + dy.z * v.y + N.z * v.z);
}

// Lambertian::pdf (Lambertian.h:45-54): cosine pdf about the normal turned toward wi
DEV float lambertPdf(float3 Ng, float3 wi) {
  float3 N = Ng;
  if (dot3(wi, N) < 0.f) N = f3(-N.x, -N.y, -N.z);
  return fmax_(dot3(wi, N), 0.f) * kOneOverPi;
}

// Lane phases of the render loop.
enum LanePhase : int {
  LP_IDLE = 0,      // no pixel
  LP_NEWSAMPLE = 1, // the next wave of its pixel needs a primary ray
  LP_CELL = 2,      // a ray needs its next macrocell with a non-zero majorant
  LP_WOODCOCK = 3,  // inside a Woodcock range
  LP_HIT = 4,       // collision found, waiting to be shaded
  LP_ENDED = 5,     // ray left the grid (primary: background; shadow: reached the light)
  LP_BEGIN = 6      // a new primary or shadow ray (ts.org, ts.dir, ts.rayTMax) needs its set-up
};

constexpr int kChunk = 32;  // pixels a warp takes at a time (one 8x4 tile)

// A principled volume's hit in the multi-scatter build (MCAccelerator.h:621-659):
// tint, scattering albedo and emission from the field value at P (sampled
// again: it is the collision's value).  Not inlined, so that the render loop
// keeps its registers when principled volumes are off.
template <int T>
__device__ __noinline__ void principledAtHit(const VolumeDD &v, float3 P, const float4 *tfTab, const float *u8lut,
                                             float3 &tint, float &hitAlb, float3 &emission) {
  const float scalar = sampleJob<T>(v, P, u8lut);
  const float d = principledDensityFactor(v.pv, scalar);
  float3 ss = principledSigma(d, v.pv.scatterColor), sa = principledSigma(d, v.pv.absorptionColor);
  // the TF at the hit (TransferFunction::map)
  const float span = v.domHi - v.domLo;
  float tf = span == 1.f ? (scalar - v.domLo) : (scalar - v.domLo) / span;
  tf = fmin_(1.f, fmax_(0.f, tf));
  tf *= (float)(v.tfN - 1);
  const int ti = min(v.tfN - 2, max(0, (int)tf));
  tf -= (float)ti;
  const float4 ta = tfTab[ti], tb = tfTab[ti + 1];
  const float tw = ((1.f - tf) * ta.w + tf * tb.w) * v.baseDensity;
  if (tw > 0.f) {
    ss = f3(ss.x * tw, ss.y * tw, ss.z * tw);
    sa = f3(sa.x * tw, sa.y * tw, sa.z * tw);
    tint = f3(tint.x * ((1.f - tf) * ta.x + tf * tb.x), tint.y * ((1.f - tf) * ta.y + tf * tb.y),
              tint.z * ((1.f - tf) * ta.z + tf * tb.z));
  } else {
    ss = f3(0.f, 0.f, 0.f);
    sa = f3(0.f, 0.f, 0.f);
  }
  const float st = rmax3(f3(ss.x + sa.x, ss.y + sa.y, ss.z + sa.z));
  if (st > 0.f) {
    const float ms = rmax3(ss);
    if (ms > 0.f) tint = f3(ss.x / ms, ss.y / ms, ss.z / ms);
    hitAlb = rmax3(ss) / st;
  }
  emission = principledEmission(v.pv, scalar);
}

// shadeRays.cu:17-41 (MAX_PATH_DEPTH)
constexpr int kMaxPathDepth = 10;

// bounce() for a hit on the isosurface (shadeRays.cu:540-878) with the
// Lambertian BSDF of its AnariMatte material (Lambertian.h:45-86): a shadow
// ray toward a light sample, weighted by f_r and the surface's cosine, then,
// within the path depth and the one diffuse bounce allowed
// (MAX_DIFFUSE_BOUNCES), a cosine-sampled scattered ray.  A sample of pdf 0
// sends the ray out again unchanged from its own origin (the reference keeps
// the cleared ray, :757-768).  cosineSampleHemisphere (DG.h:162-168) draws
// its two numbers in argument order; its sincosf is sincosPortable.  Not
// inlined, so that the render loop keeps its registers.
struct SurfaceBounce {
  uint64_t shadowSeed;  // the shadow ray's RNG seed (the ray's, after its bounce RNG was derived)
  uint64_t seed;        // the ray's RNG seed after the bounce
  float3 shadowOrg, shadowTp;
  float3 lightDir;
  float shadowMis;
  float3 scatOrg, scatDir, pathTp;
  float pathMis;
  int flags;            // 1 shadow ray, 2 scattered ray, 4 it re-traces the incoming ray, 8 a diffuse bounce
};
template <int T>
__device__ __noinline__ SurfaceBounce surfaceBounce(const VolumeDD &v, const FrameDD &fr, float3 P, float tHit,
                                                    float3 dirFixed, float3 inOrg, float3 dir, float3 pathTp,
                                                    uint64_t raySeed, int depth, int nDifB, const float *u8lut,
                                                    const float *normalSamples) {
  SurfaceBounce out;
  out.flags = 0;
  out.shadowMis = 1.f;
  out.pathTp = pathTp;
  out.pathMis = 1.f;
  uint64_t random = rngDerive(raySeed, (uint64_t)__float_as_uint(tHit));
  out.shadowSeed = raySeed;
  const float3 Ng = normalize3(isoNormal<T>(v, P, dirFixed, u8lut, normalSamples));
  const bool hitWasOnFront = dot3(dir, Ng) < 0.f;
  const float3 Ngff = hitWasOnFront ? Ng : f3(-Ng.x, -Ng.y, -Ng.z);
  const float3 won = normalize3(dir);
  const float3 woN = f3(-won.x, -won.y, -won.z);  // dg.wo
  const float offsetEpsilon = fmax_(1e-4f, 1e-6f * fmax_(fmax_(fabsf(P.x), fabsf(P.y)), fabsf(P.z)));
  const float3 alb = v.iso.albedo;
  LightSample ls;
  bool needsMIS, isDir;
  if (sampleLights<true>(fr, random, ls, needsMIS, isDir, Ngff)) {
    // Lambertian::eval: the cosine against the shading normal, not turned
    const float cosThetaI = fmax_(dot3(ls.dir, Ng), 0.f);
    const float fpdf = cosThetaI * kOneOverPi;
    float3 fv = f3(alb.x * kOneOverPi * cosThetaI, alb.y * kOneOverPi * cosThetaI, alb.z * kOneOverPi * cosThetaI);
    if (fpdf > 0.f && !(fmax_(fmax_(fv.x, fv.y), fv.z) < 1e-4f)) {
      fv = f3(fmin_(fv.x, 13.f), fmin_(fv.y, 13.f), fmin_(fv.z, 13.f));
      const float ip = isinf(ls.pdf) ? 1.f : (1.f / ls.pdf);
      const float cl = kOneOverPi * fabsf(dot3(Ng, ls.dir));
      const float3 tp = f3(pathTp.x * ip * fv.x * ls.radiance.x * cl, pathTp.y * ip * fv.y * ls.radiance.y * cl,
                           pathTp.z * ip * fv.z * ls.radiance.z * cl);
      // shadowRay.rngSeed = ray.rngSeed; ray.rngSeed.next(tMax)
      raySeed = (raySeed ^ ((uint64_t)__float_as_uint(tHit) << 1)) * kRngMul;
      bool alive = true;
      if (!isDir && needsMIS) {
        const float pl = kOneOverFourPi;
        const float ps = lambertPdf(Ng, ls.dir);
        out.shadowMis = pl / (pl + ps + 1e-10f);
        if (out.shadowMis < 1e-5f) alive = false;
      }
      if (alive && kInf * (1.f - 2.f * offsetEpsilon) > 0.f) {
        out.shadowTp = f3(roundHalf(tp.x), roundHalf(tp.y), roundHalf(tp.z));
        out.shadowOrg = f3(P.x + offsetEpsilon * Ngff.x, P.y + offsetEpsilon * Ngff.y, P.z + offsetEpsilon * Ngff.z);
        out.lightDir = ls.dir;
        out.flags |= 1;
      }
    }
  }
  out.seed = raySeed;
  if (depth >= kMaxPathDepth) return out;
  // Lambertian::scatter
  float3 N = Ng;
  if (dot3(woN, N) < 0.f) N = f3(-N.x, -N.y, -N.z);
  const float su = rngFloat(random);
  const float sv = rngFloat(random);
  const float cosTheta = sqrtf(sv);
  const float sinTheta = sqrtf(1.0f - sv);
  float sinPhi, cosPhi;
  sincosPortable(kTwoPi * su, sinPhi, cosPhi);
  const float3 local = f3(cosPhi * sinTheta, sinPhi * sinTheta, cosTheta);
  const float pdf = local.z * kOneOverPi;
  if (!(pdf > 0.f) || pdf <= 1e-6f) {  // the same ray again, tMax infinite
    out.scatOrg = inOrg;
    out.scatDir = dir;
    out.flags |= 2 | 4;
    return out;
  }
  if (nDifB >= 1) return out;
  out.scatDir = normalize3(frameXfm(N, local));
  const float c = fabsf(dot3(Ng, normalize3(out.scatDir)));
  const float denom = isinf(pdf) ? 1.f : (pdf + 1e-10f);
  out.pathTp = f3(roundHalf(pathTp.x * fmin_((alb.x * c) / denom, 2.5f)),
                  roundHalf(pathTp.y * fmin_((alb.y * c) / denom, 2.5f)),
                  roundHalf(pathTp.z * fmin_((alb.z * c) / denom, 2.5f)));
  if (needsMIS && !isinf(pdf)) {
    const float ps = lambertPdf(Ng, out.scatDir);
    out.pathMis = ps / (ps + kOneOverFourPi);
  }
  out.scatOrg = f3(P.x + (1.f * offsetEpsilon) * Ngff.x, P.y + (1.f * offsetEpsilon) * Ngff.y,
                   P.z + (1.f * offsetEpsilon) * Ngff.z);
  out.flags |= 2 | 8;
  return out;
}

// The seven field samples of the normal (isoNormal) of every lane with
// need, spread over all 32 lanes of the warp: for lane L, buf[7 L] at P and
// buf[7 L + 1 + i] at P -/+ normalDelta along axis i / 2 (the points
// isoNormal samples, formed by the same expressions).  Called by the whole
// warp; P: the lane's hit point (ignored without need).
template <int T, bool BATCH>
DEV void isoNormalSamples(const JobDD *jobs, int job, const VolumeDD &v, float3 P, bool need, const float *u8lut,
                          float *buf) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned nmask = __ballot_sync(FULL, need);
  if (!nmask) return;
  const int tasks = 7 * __popc(nmask);
  for (int k0 = 0; k0 < tasks; k0 += 32) {
    const int k = k0 + lane;
    const int r = k < tasks ? k / 7 : 0;
    const int i = k < tasks ? k - 7 * r : 0;
    const int owner = __fns(nmask, 0, r + 1);
    const float px = __shfl_sync(FULL, P.x, owner), py = __shfl_sync(FULL, P.y, owner);
    const float pz = __shfl_sync(FULL, P.z, owner);
    const int oj = BATCH ? __shfl_sync(FULL, job, owner) : 0;
    if (k < tasks) {
      const VolumeDD &vo = BATCH ? jobs[oj].v : v;
      float3 Q = f3(px, py, pz);
      if (i > 0) {
        const int axis = (i - 1) >> 1;
        const float dl = vo.iso.normalDelta;
        const float o = ((i - 1) & 1) ? dl : -dl;
        Q = f3(px + (axis == 0 ? o : 0.f), py + (axis == 1 ? o : 0.f), pz + (axis == 2 ? o : 0.f));
      }
      buf[owner * 7 + i] = sampleJob<T>(vo, Q, u8lut);
    }
  }
  __syncwarp();
}

// The render loop shared by the single-frame kernel (one job, read from a
// __grid_constant__ parameter, TF staged in shared memory) and the batch
// kernel (a job table in global memory, chunks of all jobs in one counter).
// LOG: 0 fastLog (Volume.h:154-164), 1 -logf (bnx.exactLog), 2 per job (batch)
// EXT: 0 the plain kernels; 1 multi-scatter paths and principled volumes;
// 2 also isosurfaces (ISO); 3 isosurfaces (with their diffuse bounce)
// without volume bounces or principled volumes
// CMP: compensated sums (fr.comp) in no job (0: compiled out), in the jobs
// that carry terms (1: a test per sum), or in every job (2)
template <int T, bool BATCH, int LOG, int EXT, int CMP>
// isoBuf: the warp's isosurface sample buffer (kIsoBufPerWarp floats in
// shared memory; isosurface kernels only)
DEV void renderLoop(const JobDD *__restrict__ jobs, const int *__restrict__ chunkStart, int numJobs, int numChunks, const SchedDD &sd,
                    LaunchCounters *ctr, const float4 *sTF, const float *u8lut, float *isoBuf) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  constexpr bool ISO = EXT >= 2;
  constexpr bool PVMS = EXT == 1 || EXT == 2;  // principled volumes and volume bounces compiled in

  // lane work counters, 32-bit, flushed to the launch counters (below)
  unsigned nSamples = 0, nVisits = 0, nRays = 0;
  unsigned errBits = 0;

  // warp-uniform work chunk
  int chunkJob = 0, chunkBase = 0, chunkLeft = 0;
  bool exhausted = false;

  // lane state
  int phase = LP_IDLE;
  int job = 0, ix = 0, iy = 0, k = 0;  // the pixel's index iy * width + ix is formed where it is used
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  float4 comp = make_float4(0.f, 0.f, 0.f, 0.f);
  TraceState ts{};  // defined in every lane: the warp-wide passes read idle lanes' too
  uint64_t raySeed = 0;
  float3 primDir = f3(0.f, 0.f, 0.f);
  // shadowFrag: the fragment a shadow ray adds when it reaches the light
  // (min(MIS weight x throughput, clamp)), formed when the ray is spawned.
  // The plain kernels keep it in hitRGB's registers: a primary ray's TF
  // colour is dead once its collision is shaded, and a shadow ray's own
  // collision colour is never read.
  float3 hitRGB = f3(0.f, 0.f, 0.f);
  float3 shadowFragStore = f3(0.f, 0.f, 0.f);
  float3 &shadowFrag = EXT ? shadowFragStore : hitRGB;
  bool shadowRay = false;
  unsigned steps = 0;
  // EXT (the instantiation for multi-scatter paths and principled volumes;
  // the plain kernels compile neither): the path's throughput, rounded to binary16 like
  // PathState::throughput (Ray.h:17-23); the MIS weight of the path ray; its
  // generation; the volume and diffuse bounces taken; and a scattered ray
  // that waits while its generation's shadow ray is traced (pend 1: it
  // starts where the shadow ray starts; pend 2: at the origin kept in hitRGB;
  // in direction primDir, with RNG seed pendSeed).  A ray that hits the
  // isosurface carries bit 64 of ts.bits, its hit distance in ts.rayTMax.
  float3 pathTp = f3(1.f, 1.f, 1.f);
  float pathMis = 1.f;
  int depth = 0, nVolB = 0, nDifB = 0;
  int pend = 0;
  uint64_t pendSeed = 0;

  // Each round: (A) one service pass over the lanes whose ray needs host
  // work -- shading, accumulation, a new pixel, ray generation, ray set-up --
  // then (B) a tight loop that only steps macrocells and Woodcock ranges
  // until at least sd.serviceBatch lanes (or every busy lane) need service.
  while (true) {
    // between two service passes a lane traces at most one ray (< 2^24
    // counter increments), so 32-bit lane counters flushed from 2^31 on never wrap
    if ((nSamples | nVisits | nRays) >= 0x80000000u) {
      atomicAdd(&ctr->samples, (unsigned long long)nSamples);
      atomicAdd(&ctr->mcVisits, (unsigned long long)nVisits);
      atomicAdd(&ctr->rays, (unsigned long long)nRays);
      nSamples = nVisits = nRays = 0;
    }
    {
      const JobDD &J = jobs[BATCH ? job : 0];
      const VolumeDD &v = J.v;
      const FrameDD &fr = J.fr;
      // a ray that left the volume behind its isosurface hit has hit the surface
      if (ISO && phase == LP_ENDED && (ts.bits & 64)) {
        ts.t = ts.rayTMax;
        phase = LP_HIT;
      }
      // the field samples of this pass's surface normals, taken by the whole
      // warp (the lanes that shade a surface hit would take them one by one)
      if (ISO)
        isoNormalSamples<T, BATCH>(jobs, job, v,
                                   f3(ts.org.x + ts.t * ts.dir.x, ts.org.y + ts.t * ts.dir.y, ts.org.z + ts.t * ts.dir.z),
                                   phase == LP_HIT && !shadowRay && (ts.bits & 64) && !fr.emissionAbsorption, u8lut,
                                   isoBuf);
      // ------------------------------------------------------------------
      // A1. collisions: shading and shadow-ray spawn (shadeRays.cu:608-746)
      // ------------------------------------------------------------------
      if (phase == LP_HIT) {
        const int accumID = fr.accumID0 + k;
        const float clampMax = 10.f * (1 + accumID);
        const bool cmp = CMP == 2 || (CMP == 1 && fr.comp != nullptr);
        const bool surf = ISO && (ts.bits & 64);  // the hit is on the isosurface
        bool spawned = false;
        if (!shadowRay) {
          if (!EXT) {  // primary hit: generation-0 accumulation (fragment 0, alpha 1)
            if (accumID == 0) {
              acc = make_float4(0.f, 0.f, 0.f, 1.f);
              comp = make_float4(0.f, 0.f, 0.f, 0.f);
            } else {
              accAdd(acc.w, comp.w, 1.f, cmp);
            }
          }
          const float tHit = ts.t;
          const float3 P = f3(ts.org.x + tHit * ts.dir.x, ts.org.y + tHit * ts.dir.y, ts.org.z + tHit * ts.dir.z);
          // the multi-scatter build re-derives a principled volume's tint,
          // albedo and emission from the field value at the hit
          // (MCAccelerator.h:621-659); the field is sampled again at the same
          // point instead of keeping the value in a register
          float3 tint = hitRGB;
          float hitAlb = v.scatteringAlbedo;
          if (EXT) {
            float3 frag = f3(0.f, 0.f, 0.f);
            if (PVMS && v.phase == PHASE_HG && v.pv.enabled && !fr.emissionAbsorption && !surf) {
              float3 e;
              principledAtHit<T>(v, P, BATCH ? v.tf : sTF, u8lut, tint, hitAlb, e);
              // emission of the HGPhase hit: incomingThroughput * emission (shadeRays.cu:613-617)
              if (rmax3(e) > 0.f) frag = f3(pathTp.x * e.x, pathTp.y * e.y, pathTp.z * e.z);
            }
            const float fx = fmin_(frag.x, clampMax), fy = fmin_(frag.y, clampMax), fz = fmin_(frag.z, clampMax);
            if (depth == 0) {  // generation 0: the fragment and alpha 1
              if (accumID == 0) {
                acc = make_float4(fx, fy, fz, 1.f);
                comp = make_float4(0.f, 0.f, 0.f, 0.f);
              } else {
                accAdd(acc.w, comp.w, 1.f, cmp);
                if (fx > 0.f) accAdd(acc.x, comp.x, fx, cmp);
                if (fy > 0.f) accAdd(acc.y, comp.y, fy, cmp);
                if (fz > 0.f) accAdd(acc.z, comp.z, fz, cmp);
              }
            } else {  // a scattered ray's hit: its emission, if any
              if (fx > 0.f) accAdd(acc.x, comp.x, fx, cmp);
              if (fy > 0.f) accAdd(acc.y, comp.y, fy, cmp);
              if (fz > 0.f) accAdd(acc.z, comp.z, fz, cmp);
            }
          }
          if (fr.emissionAbsorption) {
            const float ex = fmin_(hitRGB.x, clampMax), ey = fmin_(hitRGB.y, clampMax), ez = fmin_(hitRGB.z, clampMax);
            if (accumID == 0) acc = make_float4(ex, ey, ez, 1.f);
            else {
              if (ex > 0.f) accAdd(acc.x, comp.x, ex, cmp);
              if (ey > 0.f) accAdd(acc.y, comp.y, ey, cmp);
              if (ez > 0.f) accAdd(acc.z, comp.z, ez, cmp);
            }
          } else if (ISO && surf) {
            const SurfaceBounce sb = surfaceBounce<T>(v, fr, P, tHit, ts.dir, ts.org, primDir, pathTp, raySeed, depth,
                                                      nDifB, u8lut, isoBuf + lane * 7);
            raySeed = (sb.flags & 1) ? sb.shadowSeed : sb.seed;
            if (sb.flags & 1) {  // makeShadowRay (Ray.h:147-157)
              shadowFrag = f3(fmin_(sb.shadowMis * sb.shadowTp.x, clampMax), fmin_(sb.shadowMis * sb.shadowTp.y, clampMax),
                              fmin_(sb.shadowMis * sb.shadowTp.z, clampMax));
              ts.org = sb.shadowOrg;
              ts.dir = sb.lightDir;
              ts.rayTMax = kInf;
              shadowRay = true;
              spawned = true;
              nRays++;
              steps = 0;
              phase = LP_BEGIN;
            }
            if (sb.flags & 2) {
              if (sb.flags & 8) {
                nDifB++;
                pathTp = sb.pathTp;
                pathMis = sb.pathMis;
              }
              depth++;
              primDir = sb.scatDir;
              if (spawned) {  // after the shadow ray: from its origin, or from the one kept in hitRGB
                pend = (sb.flags & 4) ? 2 : 1;
                if (sb.flags & 4) hitRGB = sb.scatOrg;
                pendSeed = sb.seed;
              } else {
                ts.org = sb.scatOrg;
                ts.dir = primDir;
                ts.rayTMax = kInf;
                shadowRay = false;
                spawned = true;
                nRays++;
                steps = 0;
                phase = LP_BEGIN;
              }
            }
          } else {
            // bounce() volume-hit branch, shadeRays.cu:608-746
            uint64_t random = rngDerive(raySeed, (uint64_t)__float_as_uint(tHit));
            // the ray's own direction: the plain kernels undo the zero fix-up
            // of traceBegin instead of keeping a copy in registers
            const float3 won = normalize3(EXT ? primDir
                                              : f3((ts.bits & 8) ? 0.f : ts.dir.x, (ts.bits & 16) ? 0.f : ts.dir.y,
                                                   (ts.bits & 32) ? 0.f : ts.dir.z));
            const float3 woN = f3(-won.x, -won.y, -won.z);  // dg.wo
            const float offsetEpsilon = fmax_(1e-4f, 1e-6f * fmax_(fmax_(fabsf(P.x), fabsf(P.y)), fabsf(P.z)));
            LightSample ls;
            bool needsMIS, isDir;
            uint64_t scatSeed = raySeed;  // the path ray's seed after the shadow ray took its copy
            if (sampleLights(fr, random, ls, needsMIS, isDir)) {
              float3 alb;
              float fpdf;
              if (v.phase == PHASE_SIMPLE) {
                alb = f3(.7f * tint.x, .7f * tint.y, .7f * tint.z);
                fpdf = kOneOverFourPi;
              } else {
                const float a = EXT ? hitAlb : v.scatteringAlbedo;  // plain kernels read it here, not earlier
                alb = f3(a * tint.x, a * tint.y, a * tint.z);
                // HGPhase::pdf (Phase.h:51-58) is 1/4pi for |g| < 1e-3 whatever the
                // angle: the directions are normalised only when it is not
                if (fabsf(v.anisotropy) < 1e-3f) {
                  fpdf = kOneOverFourPi;
                } else {
                  const float3 wi_in = normalize3(f3(-woN.x, -woN.y, -woN.z));
                  fpdf = hgPhase(v.anisotropy, dot3(wi_in, normalize3(ls.dir)));
                }
              }
              float3 fv = f3(fpdf * alb.x, fpdf * alb.y, fpdf * alb.z);
              if (fpdf > 0.f && !(fmax_(fmax_(fv.x, fv.y), fv.z) < 1e-4f)) {
                fv = f3(fmin_(fv.x, 13.f), fmin_(fv.y, 13.f), fmin_(fv.z, 13.f));
                const float ip = isinf(ls.pdf) ? 1.f : (1.f / ls.pdf);
                const float3 tin = EXT ? pathTp : f3(1.f, 1.f, 1.f);  // incomingThroughput
                const float3 tp = f3(tin.x * ip * fv.x * ls.radiance.x * 1.f, tin.y * ip * fv.y * ls.radiance.y * 1.f,
                                     tin.z * ip * fv.z * ls.radiance.z * 1.f);
                // shadowRay.rngSeed = ray.rngSeed; ray.rngSeed.next(tMax)
                if (EXT) scatSeed = (raySeed ^ ((uint64_t)__float_as_uint(tHit) << 1)) * kRngMul;
                float misWeight = 1.f;
                bool alive = true;
                if (!isDir && needsMIS) {
                  // the phase pdf of the light sample's direction is fpdf
                  // (the same expression: 1/4pi, or hgPhase of the same vectors)
                  misWeight = kOneOverFourPi / (kOneOverFourPi + fpdf + 1e-10f);
                  if (misWeight < 1e-5f) alive = false;
                }
                const float sTMax = kInf * (1.f - 2.f * offsetEpsilon);
                if (alive && sTMax > 0.f) {
                  shadowFrag = f3(fmin_(misWeight * roundHalf(tp.x), clampMax), fmin_(misWeight * roundHalf(tp.y), clampMax),
                                  fmin_(misWeight * roundHalf(tp.z), clampMax));
                  // makeShadowRay (Ray.h:147-157); its RNG seed is the primary's,
                  // which is not used again by this wave
                  ts.org = f3(P.x + offsetEpsilon * woN.x, P.y + offsetEpsilon * woN.y, P.z + offsetEpsilon * woN.z);
                  ts.dir = ls.dir;
                  ts.rayTMax = sTMax;
                  shadowRay = true;
                  spawned = true;
                  nRays++;
                  steps = 0;
                  phase = LP_BEGIN;
                }
              }
            }
            // multi-scatter build: HGPhase::scatter and the volume-bounce
            // budget (shadeRays.cu:749-878).  A sample with pdf <= 1e-6 would
            // end the path here (the reference re-traces the old ray); with
            // anisotropy clamped to [-0.99, 0.99] (Volume.cpp:55-57) the HG
            // pdf stays above 2e-4, so neither can happen.
            if (PVMS && fr.maxVolumeBounces > 0 && depth < kMaxPathDepth) {
              const float3 wi_in = normalize3(f3(-woN.x, -woN.y, -woN.z));
              const float3 sdir = hgSampleDirection(wi_in, v.anisotropy, random);
              const float pdf = hgPhase(v.anisotropy, dot3(wi_in, sdir));
              const float3 alb = f3(hitAlb * tint.x, hitAlb * tint.y, hitAlb * tint.z);
              const float3 f_r = f3(alb.x * pdf, alb.y * pdf, alb.z * pdf);
              if (pdf > 0.f && !(pdf <= 1e-6f) && nVolB < fr.maxVolumeBounces) {
                nVolB++;
                depth++;
                primDir = normalize3(sdir);
                const float denom = isinf(pdf) ? 1.f : (pdf + 1e-10f);
                pathTp = f3(roundHalf(pathTp.x * fmin_((f_r.x * 1.f) / denom, 2.5f)),
                            roundHalf(pathTp.y * fmin_((f_r.y * 1.f) / denom, 2.5f)),
                            roundHalf(pathTp.z * fmin_((f_r.z * 1.f) / denom, 2.5f)));
                if (needsMIS && !isinf(pdf)) {
                  const float ps = hgPhase(v.anisotropy, dot3(normalize3(f3(-woN.x, -woN.y, -woN.z)), normalize3(primDir)));
                  pathMis = ps / (ps + kOneOverFourPi);
                } else {
                  pathMis = 1.f;
                }
                if (spawned) {  // after the shadow ray, from the shadow ray's origin
                  pend = 1;
                  pendSeed = scatSeed;
                } else {
                  ts.org = f3(P.x + (1.f * offsetEpsilon) * woN.x, P.y + (1.f * offsetEpsilon) * woN.y,
                              P.z + (1.f * offsetEpsilon) * woN.z);
                  ts.dir = primDir;
                  ts.rayTMax = kInf;
                  raySeed = scatSeed;
                  shadowRay = false;
                  spawned = true;
                  nRays++;
                  steps = 0;
                  phase = LP_BEGIN;
                }
              }
            }
          }
        }
        if (!spawned) {
          if (EXT && pend) {  // the shadow ray was occluded: the scattered ray goes next
            if (pend == 2) ts.org = hitRGB;
            ts.dir = primDir;
            ts.rayTMax = kInf;
            raySeed = pendSeed;
            pend = 0;
            shadowRay = false;
            nRays++;
            steps = 0;
            phase = LP_BEGIN;
          } else if (++k == fr.spp) {  // no ray left: the wave is done
            const int64_t pix = (int64_t)iy * fr.width + ix;
            if (BNB_IN(pix, (long long)fr.width * fr.height)) {
              fr.accum[pix] = acc;
              if (cmp) fr.comp[pix] = comp;
            }
            phase = LP_IDLE;
          } else {
            phase = LP_NEWSAMPLE;
          }
        }
      }

      // ------------------------------------------------------------------
      // A2. rays that left the grid: bounce() without intersection
      //    (shadeRays.cu:507-600) and accumulation (:996-1040)
      // ------------------------------------------------------------------
      if (phase == LP_ENDED) {
        const int accumID = fr.accumID0 + k;
        const float clampMax = 10.f * (1 + accumID);
        const bool cmp = CMP == 2 || (CMP == 1 && fr.comp != nullptr);
        if (!shadowRay && (!EXT || depth == 0)) {
          // the primary ray's miss colour (generateRays.cu:217-227), computed here
          // rather than kept in registers for the whole wave
          float4 bg = fr.bgColor;
          if (!(fr.bgColor.w >= 0.f)) {
            const float t = (iy + .5f) / float(fr.height);
            bg = make_float4((1.0f - t) * 0.9f + t * 0.15f, (1.0f - t) * 0.9f + t * 0.25f, (1.0f - t) * 0.9f + t * .8f,
                             (1.0f - t) * 1.f + t * 1.f);
          }
          const float f0x = fmin_(bg.x, clampMax), f0y = fmin_(bg.y, clampMax), f0z = fmin_(bg.z, clampMax);
          if (accumID == 0) {
            acc = make_float4(f0x, f0y, f0z, bg.w);
            comp = make_float4(0.f, 0.f, 0.f, 0.f);
          } else {
            if (bg.w > 0.f) accAdd(acc.w, comp.w, bg.w, cmp);
            if (f0x > 0.f) accAdd(acc.x, comp.x, f0x, cmp);
            if (f0y > 0.f) accAdd(acc.y, comp.y, f0y, cmp);
            if (f0z > 0.f) accAdd(acc.z, comp.z, f0z, cmp);
          }
        } else if (!shadowRay) {  // a scattered ray left into the environment (shadeRays.cu:529-557)
          const float fx = fmin_(pathTp.x * fr.ambientRadiance * pathMis, clampMax);
          const float fy = fmin_(pathTp.y * fr.ambientRadiance * pathMis, clampMax);
          const float fz = fmin_(pathTp.z * fr.ambientRadiance * pathMis, clampMax);
          if (fx > 0.f) accAdd(acc.x, comp.x, fx, cmp);
          if (fy > 0.f) accAdd(acc.y, comp.y, fy, cmp);
          if (fz > 0.f) accAdd(acc.z, comp.z, fz, cmp);
        } else {  // the shadow ray reached the light
          const float f1x = shadowFrag.x, f1y = shadowFrag.y, f1z = shadowFrag.z;
          if (f1x > 0.f) accAdd(acc.x, comp.x, f1x, cmp);
          if (f1y > 0.f) accAdd(acc.y, comp.y, f1y, cmp);
          if (f1z > 0.f) accAdd(acc.z, comp.z, f1z, cmp);
        }
        if (EXT && shadowRay && pend) {  // the scattered ray goes next, from the shadow ray's origin
          if (pend == 2) ts.org = hitRGB;
          ts.dir = primDir;
          ts.rayTMax = kInf;
          raySeed = pendSeed;
          pend = 0;
          shadowRay = false;
          nRays++;
          steps = 0;
          phase = LP_BEGIN;
        } else if (++k == fr.spp) {
          const int64_t pix = (int64_t)iy * fr.width + ix;
          if (BNB_IN(pix, (long long)fr.width * fr.height)) {
            fr.accum[pix] = acc;
            if (cmp) fr.comp[pix] = comp;
          }
          phase = LP_IDLE;
        } else {
          phase = LP_NEWSAMPLE;
        }
      }

    }
    // ------------------------------------------------------------------
    // A3. lanes without a pixel take the next ones of the warp's chunk
    // ------------------------------------------------------------------
    unsigned need = __ballot_sync(FULL, phase == LP_IDLE);
    while (need && !exhausted) {
      if (chunkLeft == 0) {
        int c = 0, ab = 0;
        if (lane == 0) {
          c = (int)atomicAdd(&ctr->nextPixel, 1u);
          ab = (int)*(volatile unsigned *)&ctr->abort;
        }
        c = __shfl_sync(FULL, c, 0);
        ab = __shfl_sync(FULL, ab, 0);
        if (ab) { errBits |= ERR_ABORTED; exhausted = true; break; }
        if (c >= numChunks) { exhausted = true; break; }
        int j = 0;
        if (BATCH) {  // last job whose first chunk is <= c
          int lo = 0, hi = numJobs - 1;
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (chunkStart[mid] <= c) lo = mid; else hi = mid - 1;
          }
          j = lo;
        }
        const int first = BATCH ? chunkStart[j] : 0;
        const int npix = jobs[j].fr.width * jobs[j].fr.height;
        if (!BATCH && jobs[j].fr.partCount > 1)  // this rank's k-th chunk -> the frame's chunk
          c = (c / kPartTileChunks * jobs[j].fr.partCount + jobs[j].fr.partRank) * kPartTileChunks +
              c % kPartTileChunks;
        chunkJob = j;
        chunkBase = (c - first) * kChunk;
        chunkLeft = min(kChunk, npix - chunkBase);
      }
      const int n = __popc(need);
      const int take = min(n, chunkLeft);
      const int rank = __popc(need & ((1u << lane) - 1u));
      if (((need >> lane) & 1u) && rank < take) {
        const FrameDD &fr = jobs[chunkJob].fr;
        const int W = fr.width, H = fr.height;
        // pixel order: 4-row bands, column-major inside a band (8x4 tiles per 32 pixels)
        const int w = chunkBase + rank;
        const int band = w / (4 * W);
        const int rows = min(4, H - 4 * band);
        const int within = w - band * 4 * W;
        job = chunkJob;
        ix = within / rows;
        iy = 4 * band + within % rows;
        const int64_t pix = (int64_t)iy * W + ix;
        k = 0;
        const bool pixIn = BNB_IN(pix, (long long)fr.width * fr.height);
        acc = (fr.accumID0 > 0 && pixIn) ? fr.accum[pix] : make_float4(0.f, 0.f, 0.f, 0.f);
        comp = (CMP && fr.accumID0 > 0 && (CMP == 2 || fr.comp) && pixIn) ? fr.comp[pix] : make_float4(0.f, 0.f, 0.f, 0.f);
        phase = LP_NEWSAMPLE;
      }
      for (int i = 0; i < take; i++) need &= need - 1u;
      chunkBase += take;
      chunkLeft -= take;
    }
    if (!__ballot_sync(FULL, phase != LP_IDLE)) break;  // no work left for this warp
    {
      const JobDD &J = jobs[BATCH ? job : 0];
      const VolumeDD &v = J.v;
      const FrameDD &fr = J.fr;
      // ------------------------------------------------------------------
      // A4. primary rays
      //    (generateRays.cu:71-243)
      // ------------------------------------------------------------------
      if (phase == LP_NEWSAMPLE) {
        const int W = fr.width, H = fr.height;
        const int accumID = fr.accumID0 + k;
        // 32-bit wrap-around arithmetic, as the reference's ints do on the GPU
        const unsigned uAcc = (unsigned)accumID;
        uint64_t rnd = rngSeed2((unsigned)ix + (unsigned)W * uAcc, (unsigned)iy + (unsigned)H * uAcc);
        raySeed = rngSeed2((unsigned)ix + uAcc * (unsigned)W, (uint32_t)iy);
        const float pixel_u = (accumID == 0) ? .5f : rngFloat(rnd);
        const float pixel_v = (accumID == 0) ? .5f : rngFloat(rnd);
        const float image_u = ((ix + pixel_u) / float(W));
        const float image_v = ((iy + pixel_v) / float(H));
        const float aspect = fr.aspect;  // W / float(H), formed on the host
        const float su = 1.f * aspect * (image_u - .5f), sv = 1.f * (image_v - .5f);
        float3 d = f3(fr.dir00.x + su * fr.dirdu.x + sv * fr.dirdv.x, fr.dir00.y + su * fr.dirdu.y + sv * fr.dirdv.y,
                      fr.dir00.z + su * fr.dirdu.z + sv * fr.dirdv.z);
        d = normalize3(d);
        float3 o = fr.lens00;
        float tMax = 1e30f;
        if (fr.cutPlane.w > -1e28f) {
          const float3 N = f3(fr.cutPlane.x, fr.cutPlane.y, fr.cutPlane.z);
          const float dist_org = dot3(N, o) + fr.cutPlane.w;
          const float denom = dot3(N, d);
          if (dist_org >= 0.f) {
            if (denom < 0.f) tMax = fmin_(tMax, -dist_org / denom);
          } else {
            if (denom > 0.f) {
              const float te = -dist_org / denom;
              o = f3(o.x + te * d.x, o.y + te * d.y, o.z + te * d.z);
            } else tMax = 0.f;
          }
        }
        if (EXT) primDir = d;
        shadowRay = false;
        if (EXT) {
          pathTp = f3(1.f, 1.f, 1.f);
          pathMis = 1.f;
          depth = 0;
          nVolB = 0;
          nDifB = 0;
          pend = 0;
        }
        nRays++;
        steps = 0;
        ts.org = o;
        ts.dir = d;
        ts.rayTMax = tMax;
        phase = LP_BEGIN;
      }

      // ------------------------------------------------------------------
      // A5. ray set-up, primary and shadow rays together
      // ------------------------------------------------------------------
      if (phase == LP_BEGIN) {
        if (ISO && v.iso.enabled) {
          // the traversal calls the isosurface first; its hit lowers only the
          // ray's own tMax, so the volume's box test and DDA run to the
          // traversal's tMax while its Woodcock ranges stop at the surface.  A
          // shadow ray that hits the surface is occluded.
          const float3 dF = f3(ts.dir.x == 0.f ? 1e-6f : ts.dir.x, ts.dir.y == 0.f ? 1e-6f : ts.dir.y,
                               ts.dir.z == 0.f ? 1e-6f : ts.dir.z);
          const float tIso = isoIntersect<T, BATCH>(jobs, job, v, ts.org, dF, ts.rayTMax, &raySeed, u8lut, isoBuf);
          const bool isoHit = tIso < ts.rayTMax;
          if (isoHit && shadowRay) {
            phase = LP_HIT;
          } else {
            const bool inVol = v.hasVolume && traceBegin(v, ts, ts.org, ts.dir, ts.rayTMax, raySeed);
            ts.dir = dF;
            ts.bits = isoHit ? (ts.bits | 64) : (ts.bits & ~64);
            if (isoHit) ts.rayTMax = tIso;
            if (inVol) phase = LP_CELL;
            else if (isoHit) { ts.t = tIso; phase = LP_HIT; }
            else phase = LP_ENDED;
          }
        } else {
          phase = traceBegin(v, ts, ts.org, ts.dir, ts.rayTMax, raySeed) ? LP_CELL : LP_ENDED;
          if (ISO) ts.bits &= ~64;
        }
      }

    }
    {
      const JobDD &J = jobs[BATCH ? job : 0];
      const VolumeDD &v = J.v;
      const FrameDD &fr = J.fr;
      while (true) {
        // ------------------------------------------------------------------
        // B1. next macrocell with a non-zero majorant (DDA.h:172-200,
        //    MCAccelerator.h:596-612)
        // ------------------------------------------------------------------
        if (phase == LP_CELL) {
          while (true) {
            const float tClosest = fmin_(fmin_(ts.tNext.x, ts.tNext.y), ts.tNext.z);
            // cell indices are inside the grid here and the grid has < 2^31 cells
            const int ci = ts.cx + v.mcDims.x * (ts.cy + v.mcDims.y * ts.cz);
            const bool occupied = BNB_IN(ci, (long long)v.mcDims.x * v.mcDims.y * v.mcDims.z) &&
                                  ((__ldg(v.mcOccupied + (ci >> 5)) >> (ci & 31)) & 1u);
            nVisits++;
            if (!occupied) {  // majorant == 0
              if (!ddaStep(v, ts, tClosest)) { phase = LP_ENDED; break; }
              if (++steps > (1u << 22)) { errBits |= ERR_ITER_CAP; phase = LP_ENDED; break; }
            } else {
              // no collision can precede a surface hit at or before this cell's start
              if (ISO && (ts.bits & 64) && ts.rayT0 + ts.nextCellBegin >= ts.rayTMax) { phase = LP_ENDED; break; }
              ts.maj = __ldg(v.majorants + ci);
              ts.t = ts.rayT0 + ts.nextCellBegin;
              ts.tUpper = fmin_(ts.rayT0 + fmin_(tClosest, ts.ddaTMax), ts.rayTMax);
              phase = LP_WOODCOCK;
              break;
            }
          }
        }
        // ------------------------------------------------------------------
        // B2. one Woodcock step (Volume.h:180-201)
        // ------------------------------------------------------------------
        if (phase == LP_WOODCOCK) {
          const float r = rngFloat(ts.rng);
          const bool exact = LOG == 1 || (LOG == 2 && fr.exactLog);
          const float dt = exact ? (-logPortable(1.f - r) / ts.maj) : (-fastLog(1.f - r) / ts.maj);
          ts.t += dt;
          if (ts.t >= ts.tUpper) {
            const float tClosest = fmin_(fmin_(ts.tNext.x, ts.tNext.y), ts.tNext.z);
            phase = ddaStep(v, ts, tClosest) ? LP_CELL : LP_ENDED;
          } else {
            const float3 P = f3(ts.org.x + ts.t * ts.dir.x, ts.org.y + ts.t * ts.dir.y, ts.org.z + ts.t * ts.dir.z);
            const float s = sampleJob<T>(v, P, u8lut);
            nSamples++;
            float w = 0.f, f = 0.f, tfw = 0.f;
            int idx = 0;
            if (!isnan(s)) {
              tfLocate(v, s, idx, f);
              if (!BNB_IN(idx, v.tfN - 1)) idx = 0;
              const float w0 = BATCH ? __ldg(&v.tf[idx].w) : sTF[idx].w;
              const float w1 = BATCH ? __ldg(&v.tf[idx + 1].w) : sTF[idx + 1].w;
              w = __fmul_rn(lerp_l(f, w0, w1), v.baseDensity);
              if (PVMS) {  // principled volume (Volume.h:66-72): density sigma_t times the TF's
                tfw = w;
                if (v.pv.enabled) w = tfw <= 0.f ? 0.f : principledSigmaT(v.pv, s) * tfw;
              }
            }
            if (w >= rngFloat(ts.rng) * ts.maj) {
              if (ISO) ts.bits &= ~64;  // a volume collision before the surface
              // (with isosurfaces a shadow ray keeps hitRGB: it may hold a waiting ray's origin)
              if (!(ISO && shadowRay)) hitRGB = f3(0.f, 0.f, 0.f);
              if (!(ISO && shadowRay) && !isnan(s) && !((PVMS && v.pv.enabled) && tfw <= 0.f)) {
                const float4 a = BATCH ? __ldg(&v.tf[idx]) : sTF[idx];
                const float4 b = BATCH ? __ldg(&v.tf[idx + 1]) : sTF[idx + 1];
                hitRGB = f3(lerp_l(f, a.x, b.x), lerp_l(f, a.y, b.y), lerp_l(f, a.z, b.z));
                if ((PVMS && v.pv.enabled)) hitRGB = principledTintTimes(v.pv, s, hitRGB);
              }
              phase = LP_HIT;
            }
          }
          if (++steps > (1u << 22)) {  // iteration cap: end this ray as if it left the grid
            errBits |= ERR_ITER_CAP;
            phase = LP_ENDED;
          }
        }

        const bool moving = phase == LP_WOODCOCK || phase == LP_CELL;
        const int nMoving = __popc(__ballot_sync(FULL, moving));
        const int nWaiting = __popc(__ballot_sync(FULL, !moving && (phase != LP_IDLE || !exhausted)));
        if (nMoving == 0 || nWaiting >= sd.serviceBatch) break;
      }
    }
  }

  // counters: warp reduction in 64 bits, one atomic per warp
  unsigned long long wSamples = nSamples, wVisits = nVisits, wRays = nRays;
  for (int o = 16; o > 0; o >>= 1) {
    wSamples += __shfl_down_sync(FULL, wSamples, o);
    wVisits += __shfl_down_sync(FULL, wVisits, o);
    wRays += __shfl_down_sync(FULL, wRays, o);
    errBits |= __shfl_down_sync(FULL, errBits, o);
  }
  if (lane == 0) {
    atomicAdd(&ctr->samples, wSamples);
    atomicAdd(&ctr->mcVisits, wVisits);
    atomicAdd(&ctr->rays, wRays);
    if (errBits) atomicOr(&ctr->errorFlags, (unsigned long long)errBits);
  }
}

// Chunks of a frame of numChunks chunks that partition rank `rank` of
// `count` renders: whole tiles of kPartTileChunks chunks, t % count == rank.
__host__ __device__ inline int partitionChunks(int numChunks, int rank, int count) {
  const int tiles = (numChunks + kPartTileChunks - 1) / kPartTileChunks;
  if (rank >= tiles) return 0;
  const int mine = (tiles - 1 - rank) / count + 1;
  const int last = rank + (mine - 1) * count;
  return (mine - 1) * kPartTileChunks + min(kPartTileChunks, numChunks - last * kPartTileChunks);
}

template <int T, int LOG, int EXT, int CMP>
__global__ void __launch_bounds__(kRenderMaxThreads, EXT >= 2     ? kRenderMinBlocksIso
                                                     : EXT        ? kRenderMinBlocksExt
                                                     : CMP == 1   ? kRenderMinBlocksMixedComp
                                                                  : kRenderMinBlocks)
    renderKernel(const __grid_constant__ JobDD job, const __grid_constant__ SchedDD sd, LaunchCounters *ctr) {
  extern __shared__ float4 sTF[];
  __shared__ float u8lut[256];
  __shared__ float sIsoBuf[EXT >= 2 ? kRenderMaxThreads / 32 * kIsoBufPerWarp : 1];
  for (int i = threadIdx.x; i < job.v.tfN; i += blockDim.x) sTF[i] = job.v.tf[i];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) u8lut[i] = __fdiv_rn((float)i * 1.f, 255.f);
  __syncthreads();
  int numChunks = (job.fr.width * job.fr.height + kChunk - 1) / kChunk;
  if (job.fr.partCount > 1) numChunks = partitionChunks(numChunks, job.fr.partRank, job.fr.partCount);
  renderLoop<T, false, LOG, EXT, CMP>(&job, nullptr, 1, numChunks, sd, ctr, sTF, u8lut,
                                      EXT >= 2 ? sIsoBuf + (threadIdx.x >> 5) * kIsoBufPerWarp : nullptr);
}

// ---------------------------------------------------------------------------
// Regrouped render kernel (plain single-frame jobs)
// ---------------------------------------------------------------------------
// A CTA owns kAQSlots pixel slots.  A slot's whole state -- its pixel and
// wave, the accumulator and the ray in flight -- lives in shared memory, so
// any thread of the CTA can advance any slot.  Every slot waits in one of
// four ring queues in shared memory:
//   idle   no pixel: the next pixels of the frame go to these slots;
//   trace  a ray to be walked through the macrocells and Woodcock ranges;
//   hit    a primary ray's collision, to be shaded;
//   end    a primary ray that left the volume, or a shadow ray that reached
//          the light or was occluded: accumulation.
// Each warp runs on its own, with no barrier: it picks the queue with the
// most work and takes up to 32 slots from it, one per lane.
//   fetch, hit and end passes: the slots' service (renderLoop's A1-A3), then
//          primary-ray generation (A4) and ray set-up (A5) where needed; each
//          slot then joins the queue of its next step;
//   trace pass: lanes step their rays (B1, B2); a lane whose ray needs
//          service hands the slot to the hit or end queue and takes the next
//          ray of the trace queue, until that queue is empty and fewer than
//          kAQMinHeld lanes still hold rays while service work waits.
// Each slot runs exactly the state machine of a renderLoop lane (plain
// kernels: no isosurface, multi-scatter or principled volume), in the same
// order per pixel, so frames and work counters are the same bit for bit;
// only which thread executes a step changes.
//
// Queues: kAQRing cells per queue and two counters.  A producer reserves
// cells with atomicAdd on tail and fills each with a compare-and-swap once
// the cell is empty; a consumer reserves cells with a compare-and-swap on
// head (never past tail) and empties each with an exchange once it is
// filled.  A slot is in at most one queue, so a queue never holds more than
// kAQSlots entries.  Every wait for a cell is bounded (kAQSpinCap); running
// past the bound ends the launch with the iteration-cap error.
constexpr int kAQThreads = 256;
constexpr int kAQSlots = 384;
constexpr int kAQRing = 512;  // cells per queue: a power of two >= kAQSlots
constexpr int kAQMinBlocks = 3;
constexpr int kAQMinHeld = 16;
constexpr int kAQServeMin = 16;
constexpr unsigned kAQSpinCap = 1u << 20;
constexpr unsigned kAQIdleCap = 1u << 24;
enum AQQueue : int { AQ_IDLE = 0, AQ_TRACE = 1, AQ_HIT = 2, AQ_END = 3 };
constexpr int kAQDrop = 15;  // a slot left out of every queue (the frame's pixels are all taken)

struct AQShared {
  float4 acc[kAQSlots];
  float ox[kAQSlots], oy[kAQSlots], oz[kAQSlots];   // ray origin
  float dx[kAQSlots], dy[kAQSlots], dz[kAQSlots];   // ray direction (zero components fixed up by the set-up)
  float rayTMax[kAQSlots];
  unsigned seedLo[kAQSlots], seedHi[kAQSlots];      // the ray's RNG seed
  int meta[kAQSlots];  // bits 0-3 LanePhase at the hand-off, bit 4 shadow ray, bits 8-13 TraceState::bits
  int ix[kAQSlots], iy[kAQSlots], k[kAQSlots];       // pixel and wave of the launch
  float fx[kAQSlots], fy[kAQSlots], fz[kAQSlots];    // TF colour at a primary hit; a shadow ray's fragment
  float ddaTMax[kAQSlots], rayT0[kAQSlots], ncb[kAQSlots];
  float tnx[kAQSlots], tny[kAQSlots], tnz[kAQSlots];
  float tsx[kAQSlots], tsy[kAQSlots], tsz[kAQSlots];
  int cx[kAQSlots], cy[kAQSlots], cz[kAQSlots];
  unsigned rngLo[kAQSlots], rngHi[kAQSlots];         // the Woodcock RNG
  float t[kAQSlots], tUpper[kAQSlots], maj[kAQSlots];
  unsigned steps[kAQSlots];
  unsigned cell[4][kAQRing];  // slot + 1, or 0 when empty
  unsigned head[4], tail[4];
  int live;       // slots holding a pixel
  int exhausted;  // no pixel of the frame is left to take
  int aborted;
  int failed;     // a bounded wait ran out: every warp leaves
};

DEV uint64_t wfJoin(unsigned lo, unsigned hi) { return (uint64_t)lo | ((uint64_t)hi << 32); }
DEV unsigned aqLoad(const unsigned *p) { return *(const volatile unsigned *)p; }
DEV int aqLoadI(const int *p) { return *(const volatile int *)p; }

// Slot s joins queue q for every lane with put.  Called by all lanes of the
// warp.  False (that lane) when the wait for an empty cell ran out.
DEV bool aqPush(AQShared &sh, int q, bool put, int s) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned m = __ballot_sync(FULL, put);
  if (!m) return true;
  const int leader = __ffs(m) - 1;
  unsigned base = 0;
  if (lane == leader) base = atomicAdd(&sh.tail[q], (unsigned)__popc(m));
  base = __shfl_sync(FULL, base, leader);
  if (!put) return true;
  const unsigned c = (base + (unsigned)__popc(m & ((1u << lane) - 1u))) & (kAQRing - 1);
  __threadfence_block();  // the slot's state is visible before its cell
  for (unsigned spins = 0; atomicCAS(&sh.cell[q][c], 0u, (unsigned)s + 1u) != 0u;)
    if (++spins > kAQSpinCap) return false;
  return true;
}

// Lanes with want take one slot each from queue q, as many as it holds;
// -1 for the others.  Called by all lanes of the warp.  ok turns false when
// the wait for a filled cell ran out.
DEV int aqPop(AQShared &sh, int q, bool want, bool &ok) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned m = __ballot_sync(FULL, want);
  if (!m) return -1;
  int got = 0;
  unsigned base = 0;
  if (lane == 0) {
    const int n = __popc(m);
    unsigned h = aqLoad(&sh.head[q]);
    for (int tries = 0; tries < 1024; tries++) {
      const int avail = (int)(aqLoad(&sh.tail[q]) - h);
      const int take = min(n, avail);
      if (take <= 0) break;
      const unsigned old = atomicCAS(&sh.head[q], h, h + (unsigned)take);
      if (old == h) {
        got = take;
        base = h;
        break;
      }
      h = old;
    }
  }
  got = __shfl_sync(FULL, got, 0);
  base = __shfl_sync(FULL, base, 0);
  const int r = __popc(m & ((1u << lane) - 1u));
  if (!want || r >= got) return -1;
  const unsigned c = (base + (unsigned)r) & (kAQRing - 1);
  unsigned v = 0;
  for (unsigned spins = 0; (v = atomicExch(&sh.cell[q][c], 0u)) == 0u;)
    if (++spins > kAQSpinCap) {
      ok = false;
      return -1;
    }
  __threadfence_block();  // the slot's state is read after its cell
  return (int)v - 1;
}

// bytes of dynamic shared memory: the slots and queues, then the TF table
__host__ __device__ inline size_t wfSlotsBytes() { return (sizeof(AQShared) + 15) & ~(size_t)15; }

template <int T, int LOG>
__global__ void __launch_bounds__(kAQThreads, kAQMinBlocks)
    renderKernelWF(const __grid_constant__ JobDD job, LaunchCounters *ctr) {
  extern __shared__ __align__(16) unsigned char wfSmem[];
  __shared__ float u8lut[256];
  AQShared &sh = *reinterpret_cast<AQShared *>(wfSmem);
  float4 *sTF = reinterpret_cast<float4 *>(wfSmem + wfSlotsBytes());
  const VolumeDD &v = job.v;
  const FrameDD &fr = job.fr;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const unsigned FULL = 0xffffffffu;
  for (int i = tid; i < v.tfN; i += blockDim.x) sTF[i] = v.tf[i];
  for (int i = tid; i < 256; i += blockDim.x) u8lut[i] = __fdiv_rn((float)i * 1.f, 255.f);
  for (int i = tid; i < 4 * kAQRing; i += blockDim.x) (&sh.cell[0][0])[i] = 0u;
  __syncthreads();
  for (int s = tid; s < kAQSlots; s += blockDim.x) sh.cell[AQ_IDLE][s] = (unsigned)s + 1u;
  if (tid < 4) {
    sh.head[tid] = 0u;
    sh.tail[tid] = tid == AQ_IDLE ? (unsigned)kAQSlots : 0u;
  }
  if (tid == 0) {
    sh.live = 0;
    sh.exhausted = 0;
    sh.aborted = 0;
    sh.failed = 0;
  }
  __syncthreads();
  const int W = fr.width, H = fr.height;
  const int npix = W * H;
  const int frameChunks = (npix + kChunk - 1) / kChunk;
  const int numChunks = fr.partCount > 1 ? partitionChunks(frameChunks, fr.partRank, fr.partCount) : frameChunks;
  const unsigned totalPix = (unsigned)numChunks * (unsigned)kChunk;  // pixel indices of this rank's chunks
  const bool cmp = fr.comp != nullptr;
  unsigned nSamples = 0, nVisits = 0, nRays = 0, errBits = 0;
  // this rank's chunk c -> the frame's chunk, and the pixels it holds
  auto frameChunk = [&](int c) {
    return fr.partCount > 1 ? (c / kPartTileChunks * fr.partCount + fr.partRank) * kPartTileChunks + c % kPartTileChunks
                            : c;
  };
  auto chunkPixels = [&](int c) { return min(kChunk, npix - frameChunk(c) * kChunk); };
  bool ok = true;
  unsigned idlePolls = 0;  // polls without work since the live-slot count last changed
  int lastLive = -1;

  while (true) {
    if ((nSamples | nVisits | nRays) >= 0x80000000u) {
      atomicAdd(&ctr->samples, (unsigned long long)nSamples);
      atomicAdd(&ctr->mcVisits, (unsigned long long)nVisits);
      atomicAdd(&ctr->rays, (unsigned long long)nRays);
      nSamples = nVisits = nRays = 0;
    }
    // the queue to work on: a full warp of service work first, then rays
    int pend[4] = {0, 0, 0, 0};
    int exhausted = 0, live = 0, failed = 0;
    if (lane == 0) {
      for (int q = 0; q < 4; q++) pend[q] = (int)(aqLoad(&sh.tail[q]) - aqLoad(&sh.head[q]));
      exhausted = aqLoadI(&sh.exhausted);
      __threadfence_block();
      live = aqLoadI(&sh.live);
      failed = aqLoadI(&sh.failed);
    }
    for (int q = 0; q < 4; q++) pend[q] = __shfl_sync(FULL, pend[q], 0);
    exhausted = __shfl_sync(FULL, exhausted, 0);
    live = __shfl_sync(FULL, live, 0);
    failed = __shfl_sync(FULL, failed, 0);
    if (failed) break;
    if (exhausted) pend[AQ_IDLE] = 0;
    // a full warp of service work first, then rays
    int q = -1;
    if (pend[AQ_HIT] >= 32) q = AQ_HIT;
    else if (pend[AQ_END] >= 32) q = AQ_END;
    else if (pend[AQ_IDLE] >= 32) q = AQ_IDLE;
    else if (pend[AQ_TRACE] > 0) q = AQ_TRACE;
    else if (pend[AQ_HIT] > 0) q = AQ_HIT;
    else if (pend[AQ_END] > 0) q = AQ_END;
    else if (pend[AQ_IDLE] > 0) q = AQ_IDLE;
    if (q < 0) {
      if (exhausted && live == 0) break;  // the frame is done
      if (live != lastLive) {  // other warps are finishing pixels: still progress
        lastLive = live;
        idlePolls = 0;
      }
      if (++idlePolls > kAQIdleCap) {
        errBits |= ERR_ITER_CAP;
        if (lane == 0) atomicExch(&sh.failed, 1);
        break;
      }
      __nanosleep(128);
      continue;
    }
    idlePolls = 0;

    if (q == AQ_TRACE) {
      // ---------------------------------------------------------------- trace
      int s = -1, phase = LP_IDLE, meta = 0;
      unsigned steps = 0;
      TraceState ts;
      while (true) {
        const bool need = s < 0;
        if (__any_sync(FULL, need)) {
          int avail = 0;
          if (lane == 0) avail = (int)(aqLoad(&sh.tail[AQ_TRACE]) - aqLoad(&sh.head[AQ_TRACE]));
          if (__shfl_sync(FULL, avail, 0) > 0) {
            const int ns = aqPop(sh, AQ_TRACE, need, ok);
            if (ns >= 0) {
              s = ns;
              meta = sh.meta[s];
              phase = meta & 15;
              steps = sh.steps[s];
              ts.org = f3(sh.ox[s], sh.oy[s], sh.oz[s]);
              ts.dir = f3(sh.dx[s], sh.dy[s], sh.dz[s]);
              ts.rayTMax = sh.rayTMax[s];
              ts.ddaTMax = sh.ddaTMax[s];
              ts.rayT0 = sh.rayT0[s];
              ts.nextCellBegin = sh.ncb[s];
              ts.tNext = f3(sh.tnx[s], sh.tny[s], sh.tnz[s]);
              ts.tStep = f3(sh.tsx[s], sh.tsy[s], sh.tsz[s]);
              ts.cx = sh.cx[s];
              ts.cy = sh.cy[s];
              ts.cz = sh.cz[s];
              ts.bits = (meta >> 8) & 63;
              ts.rng = wfJoin(sh.rngLo[s], sh.rngHi[s]);
              ts.t = sh.t[s];
              ts.tUpper = sh.tUpper[s];
              ts.maj = sh.maj[s];
            }
          }
        }
        if (!__any_sync(FULL, s >= 0)) break;
        if (s >= 0) {
          // B1 (DDA.h:172-200, MCAccelerator.h:596-612)
          if (phase == LP_CELL) {
            while (true) {
              const float tClosest = fmin_(fmin_(ts.tNext.x, ts.tNext.y), ts.tNext.z);
              const int ci = ts.cx + v.mcDims.x * (ts.cy + v.mcDims.y * ts.cz);
              const bool occupied = BNB_IN(ci, (long long)v.mcDims.x * v.mcDims.y * v.mcDims.z) &&
                                    ((__ldg(v.mcOccupied + (ci >> 5)) >> (ci & 31)) & 1u);
              nVisits++;
              if (!occupied) {
                if (!ddaStep(v, ts, tClosest)) { phase = LP_ENDED; break; }
                if (++steps > (1u << 22)) { errBits |= ERR_ITER_CAP; phase = LP_ENDED; break; }
              } else {
                ts.maj = __ldg(v.majorants + ci);
                ts.t = ts.rayT0 + ts.nextCellBegin;
                ts.tUpper = fmin_(ts.rayT0 + fmin_(tClosest, ts.ddaTMax), ts.rayTMax);
                phase = LP_WOODCOCK;
                break;
              }
            }
          }
          // B2 (Volume.h:180-201)
          if (phase == LP_WOODCOCK) {
            const float r = rngFloat(ts.rng);
            const float dt = LOG == 1 ? (-logPortable(1.f - r) / ts.maj) : (-fastLog(1.f - r) / ts.maj);
            ts.t += dt;
            if (ts.t >= ts.tUpper) {
              const float tClosest = fmin_(fmin_(ts.tNext.x, ts.tNext.y), ts.tNext.z);
              phase = ddaStep(v, ts, tClosest) ? LP_CELL : LP_ENDED;
            } else {
              const float3 P = f3(ts.org.x + ts.t * ts.dir.x, ts.org.y + ts.t * ts.dir.y, ts.org.z + ts.t * ts.dir.z);
              const float smp = sampleField<T>(v, P, u8lut);
              nSamples++;
              float w = 0.f, f = 0.f;
              int idx = 0;
              if (!isnan(smp)) {
                tfLocate(v, smp, idx, f);
                if (!BNB_IN(idx, v.tfN - 1)) idx = 0;
                w = __fmul_rn(lerp_l(f, sTF[idx].w, sTF[idx + 1].w), v.baseDensity);
              }
              if (w >= rngFloat(ts.rng) * ts.maj) {
                if (!(meta & 16)) {  // a primary ray's collision keeps its TF colour for the shading
                  float3 hit = f3(0.f, 0.f, 0.f);
                  if (!isnan(smp)) {
                    const float4 a = sTF[idx], b = sTF[idx + 1];
                    hit = f3(lerp_l(f, a.x, b.x), lerp_l(f, a.y, b.y), lerp_l(f, a.z, b.z));
                  }
                  sh.fx[s] = hit.x;
                  sh.fy[s] = hit.y;
                  sh.fz[s] = hit.z;
                }
                phase = LP_HIT;
              }
            }
            if (++steps > (1u << 22)) {
              errBits |= ERR_ITER_CAP;
              phase = LP_ENDED;
            }
          }
        }
        // rays that need service go to the hit (a primary ray's collision)
        // or end queue (everything else)
        const bool fin = s >= 0 && phase != LP_CELL && phase != LP_WOODCOCK;
        const bool toHit = fin && phase == LP_HIT && !(meta & 16);
        if (fin) {
          sh.t[s] = ts.t;
          sh.meta[s] = (meta & ~15) | phase;
        }
        ok &= aqPush(sh, AQ_HIT, toHit, s);
        ok &= aqPush(sh, AQ_END, fin && !toHit, s);
        if (fin) s = -1;
        // under kAQMinHeld busy lanes with the trace queue empty and service
        // work waiting, the rays in hand go back to the trace queue
        const int held = __popc(__ballot_sync(FULL, s >= 0));
        if (held == 0 || held >= kAQMinHeld) continue;
        int tAvail = 0, sAvail = 0;
        if (lane == 0) {
          tAvail = (int)(aqLoad(&sh.tail[AQ_TRACE]) - aqLoad(&sh.head[AQ_TRACE]));
          sAvail = (int)(aqLoad(&sh.tail[AQ_HIT]) - aqLoad(&sh.head[AQ_HIT])) +
                   (int)(aqLoad(&sh.tail[AQ_END]) - aqLoad(&sh.head[AQ_END]));
          if (!aqLoadI(&sh.exhausted)) sAvail += (int)(aqLoad(&sh.tail[AQ_IDLE]) - aqLoad(&sh.head[AQ_IDLE]));
        }
        tAvail = __shfl_sync(FULL, tAvail, 0);
        sAvail = __shfl_sync(FULL, sAvail, 0);
        if (tAvail > 0 || sAvail < kAQServeMin) continue;
        if (s >= 0) {
          sh.ncb[s] = ts.nextCellBegin;
          sh.tnx[s] = ts.tNext.x;
          sh.tny[s] = ts.tNext.y;
          sh.tnz[s] = ts.tNext.z;
          sh.cx[s] = ts.cx;
          sh.cy[s] = ts.cy;
          sh.cz[s] = ts.cz;
          sh.rngLo[s] = (unsigned)ts.rng;
          sh.rngHi[s] = (unsigned)(ts.rng >> 32);
          sh.t[s] = ts.t;
          sh.tUpper[s] = ts.tUpper;
          sh.maj[s] = ts.maj;
          sh.steps[s] = steps;
          sh.meta[s] = (meta & ~15) | phase;
        }
        ok &= aqPush(sh, AQ_TRACE, s >= 0, s);
        break;
      }
    } else {
      // ---------------------------------------------------------- fetch / hit / end
      int s = aqPop(sh, q, true, ok);
      int phase = kAQDrop;  // where the slot goes after this pass
      int meta = 0, kk = 0, px = 0, py = 0;
      float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
      float4 comp = make_float4(0.f, 0.f, 0.f, 0.f);
      int64_t pix = 0;
      uint64_t raySeed = 0;
      float3 org = f3(0.f, 0.f, 0.f), dir = f3(0.f, 0.f, 0.f);
      float tMax = 0.f;
      bool dirty = false;  // acc / k changed
      if (q == AQ_IDLE) {
        // A3: the next pixels of this rank's chunks, in chunk order
        // the slots count as live before they take pixels, so that no warp
        // sees the frame exhausted with none live while these are assigned
        const unsigned m = __ballot_sync(FULL, s >= 0);
        unsigned base = 0;
        int ab = 0;
        if (lane == 0 && m) {
          atomicAdd(&sh.live, __popc(m));
          __threadfence_block();
          base = atomicAdd(&ctr->nextPixel, (unsigned)__popc(m));
          ab = (int)*(volatile unsigned *)&ctr->abort;
        }
        base = __shfl_sync(FULL, base, 0);
        ab = __shfl_sync(FULL, ab, 0);
        bool ends = false;
        if (s >= 0) {
          const unsigned p = base + (unsigned)__popc(m & ((1u << lane) - 1u));
          if (ab || p >= totalPix) {
            ends = true;  // nothing left for this slot: it stays out of every queue
          } else {
            const int c = (int)(p / kChunk), o = (int)(p % kChunk);
            if (o >= chunkPixels(c)) {
              phase = LP_IDLE;  // past the frame's last pixel: back to the idle queue
            } else {
              // pixel order: 4-row bands, column-major inside a band (8x4 tiles per 32 pixels)
              const int wf = frameChunk(c) * kChunk + o;
              const int band = wf / (4 * W);
              const int rows = min(4, H - 4 * band);
              const int within = wf - band * 4 * W;
              px = within / rows;
              py = 4 * band + within % rows;
              pix = (int64_t)py * W + px;
              const bool pixIn = BNB_IN(pix, (long long)npix);
              kk = 0;
              acc = (fr.accumID0 > 0 && pixIn) ? fr.accum[pix] : make_float4(0.f, 0.f, 0.f, 0.f);
              if (cmp && pixIn && fr.accumID0 == 0) fr.comp[pix] = make_float4(0.f, 0.f, 0.f, 0.f);
              sh.ix[s] = px;
              sh.iy[s] = py;
              dirty = true;
              phase = LP_NEWSAMPLE;
            }
          }
        }
        const unsigned noPix = __ballot_sync(FULL, s >= 0 && phase != LP_NEWSAMPLE);
        const unsigned ended = __ballot_sync(FULL, ends);
        if (lane == 0) {
          if (ab) atomicExch(&sh.aborted, 1);
          if (ended) atomicExch(&sh.exhausted, 1);
          __threadfence_block();
          if (noPix) atomicSub(&sh.live, __popc(noPix));
        }
      } else if (s >= 0) {
        meta = sh.meta[s];
        kk = sh.k[s];
        acc = sh.acc[s];
        px = sh.ix[s];
        py = sh.iy[s];
        pix = (int64_t)py * W + px;
        if (cmp && BNB_IN(pix, (long long)npix)) comp = fr.comp[pix];
        const bool shadowRay = (meta >> 4) & 1;
        const int accumID = fr.accumID0 + kk;
        const float clampMax = 10.f * (1 + accumID);
        dirty = true;
        bool spawned = false;
        if (q == AQ_HIT) {
          // A1 (shadeRays.cu:608-746): a primary ray's collision
          if (accumID == 0) {
            acc = make_float4(0.f, 0.f, 0.f, 1.f);
            comp = make_float4(0.f, 0.f, 0.f, 0.f);
          } else {
            accAdd(acc.w, comp.w, 1.f, cmp);
          }
          const float tHit = sh.t[s];
          const float3 o0 = f3(sh.ox[s], sh.oy[s], sh.oz[s]);
          const float3 d0 = f3(sh.dx[s], sh.dy[s], sh.dz[s]);
          const float3 P = f3(o0.x + tHit * d0.x, o0.y + tHit * d0.y, o0.z + tHit * d0.z);
          const float3 hitRGB = f3(sh.fx[s], sh.fy[s], sh.fz[s]);
          raySeed = wfJoin(sh.seedLo[s], sh.seedHi[s]);
          if (fr.emissionAbsorption) {
            const float ex = fmin_(hitRGB.x, clampMax), ey = fmin_(hitRGB.y, clampMax), ez = fmin_(hitRGB.z, clampMax);
            if (accumID == 0) acc = make_float4(ex, ey, ez, 1.f);
            else {
              if (ex > 0.f) accAdd(acc.x, comp.x, ex, cmp);
              if (ey > 0.f) accAdd(acc.y, comp.y, ey, cmp);
              if (ez > 0.f) accAdd(acc.z, comp.z, ez, cmp);
            }
          } else {
            uint64_t random = rngDerive(raySeed, (uint64_t)__float_as_uint(tHit));
            const int bits = (meta >> 8) & 63;
            const float3 won = normalize3(f3((bits & 8) ? 0.f : d0.x, (bits & 16) ? 0.f : d0.y, (bits & 32) ? 0.f : d0.z));
            const float3 woN = f3(-won.x, -won.y, -won.z);
            const float offsetEpsilon = fmax_(1e-4f, 1e-6f * fmax_(fmax_(fabsf(P.x), fabsf(P.y)), fabsf(P.z)));
            LightSample ls;
            bool needsMIS, isDir;
            if (sampleLights(fr, random, ls, needsMIS, isDir)) {
              float3 alb;
              float fpdf;
              if (v.phase == PHASE_SIMPLE) {
                alb = f3(.7f * hitRGB.x, .7f * hitRGB.y, .7f * hitRGB.z);
                fpdf = kOneOverFourPi;
              } else {
                const float a = v.scatteringAlbedo;
                alb = f3(a * hitRGB.x, a * hitRGB.y, a * hitRGB.z);
                // HGPhase::pdf (Phase.h:51-58) is 1/4pi for |g| < 1e-3 whatever the
                // angle: the directions are normalised only when it is not
                if (fabsf(v.anisotropy) < 1e-3f) {
                  fpdf = kOneOverFourPi;
                } else {
                  const float3 wi_in = normalize3(f3(-woN.x, -woN.y, -woN.z));
                  fpdf = hgPhase(v.anisotropy, dot3(wi_in, normalize3(ls.dir)));
                }
              }
              float3 fv = f3(fpdf * alb.x, fpdf * alb.y, fpdf * alb.z);
              if (fpdf > 0.f && !(fmax_(fmax_(fv.x, fv.y), fv.z) < 1e-4f)) {
                fv = f3(fmin_(fv.x, 13.f), fmin_(fv.y, 13.f), fmin_(fv.z, 13.f));
                const float ip = isinf(ls.pdf) ? 1.f : (1.f / ls.pdf);
                const float3 tp = f3(1.f * ip * fv.x * ls.radiance.x * 1.f, 1.f * ip * fv.y * ls.radiance.y * 1.f,
                                     1.f * ip * fv.z * ls.radiance.z * 1.f);
                float misWeight = 1.f;
                bool alive = true;
                if (!isDir && needsMIS) {
                  // the light sample's phase pdf is fpdf (the same expression)
                  misWeight = kOneOverFourPi / (kOneOverFourPi + fpdf + 1e-10f);
                  if (misWeight < 1e-5f) alive = false;
                }
                const float sTMax = kInf * (1.f - 2.f * offsetEpsilon);
                if (alive && sTMax > 0.f) {
                  // the fragment the shadow ray adds if it reaches the light
                  sh.fx[s] = fmin_(misWeight * roundHalf(tp.x), clampMax);
                  sh.fy[s] = fmin_(misWeight * roundHalf(tp.y), clampMax);
                  sh.fz[s] = fmin_(misWeight * roundHalf(tp.z), clampMax);
                  // makeShadowRay (Ray.h:147-157)
                  org = f3(P.x + offsetEpsilon * woN.x, P.y + offsetEpsilon * woN.y, P.z + offsetEpsilon * woN.z);
                  dir = ls.dir;
                  tMax = sTMax;
                  meta |= 16;
                  spawned = true;
                  nRays++;
                  phase = LP_BEGIN;
                }
              }
            }
          }
        } else {
          // A2 (shadeRays.cu:507-600, 996-1040): a ray that ended
          const int endPhase = meta & 15;
          if (!shadowRay) {
            float4 bg = fr.bgColor;
            if (!(fr.bgColor.w >= 0.f)) {
              const float tt = (py + .5f) / float(H);
              bg = make_float4((1.0f - tt) * 0.9f + tt * 0.15f, (1.0f - tt) * 0.9f + tt * 0.25f,
                               (1.0f - tt) * 0.9f + tt * .8f, (1.0f - tt) * 1.f + tt * 1.f);
            }
            const float f0x = fmin_(bg.x, clampMax), f0y = fmin_(bg.y, clampMax), f0z = fmin_(bg.z, clampMax);
            if (accumID == 0) {
              acc = make_float4(f0x, f0y, f0z, bg.w);
              comp = make_float4(0.f, 0.f, 0.f, 0.f);
            } else {
              if (bg.w > 0.f) accAdd(acc.w, comp.w, bg.w, cmp);
              if (f0x > 0.f) accAdd(acc.x, comp.x, f0x, cmp);
              if (f0y > 0.f) accAdd(acc.y, comp.y, f0y, cmp);
              if (f0z > 0.f) accAdd(acc.z, comp.z, f0z, cmp);
            }
          } else if (endPhase == LP_ENDED) {  // the shadow ray reached the light
            const float f1x = sh.fx[s], f1y = sh.fy[s], f1z = sh.fz[s];
            if (f1x > 0.f) accAdd(acc.x, comp.x, f1x, cmp);
            if (f1y > 0.f) accAdd(acc.y, comp.y, f1y, cmp);
            if (f1z > 0.f) accAdd(acc.z, comp.z, f1z, cmp);
          }
          // an occluded shadow ray adds nothing
        }
        if (!spawned) {
          if (++kk == fr.spp) {  // the pixel's last wave
            if (BNB_IN(pix, (long long)npix)) {
              fr.accum[pix] = acc;
              if (cmp) fr.comp[pix] = comp;
            }
            phase = LP_IDLE;
          } else {
            phase = LP_NEWSAMPLE;
          }
        }
        if (cmp && phase != LP_IDLE && BNB_IN(pix, (long long)npix)) fr.comp[pix] = comp;
      }
      const unsigned doneNow = __ballot_sync(FULL, q != AQ_IDLE && s >= 0 && phase == LP_IDLE);
      if (lane == 0 && doneNow) atomicSub(&sh.live, __popc(doneNow));
      // A4: primary rays (generateRays.cu:71-243)
      if (phase == LP_NEWSAMPLE) {
        const int accumID = fr.accumID0 + kk;
        const unsigned uAcc = (unsigned)accumID;
        uint64_t rnd = rngSeed2((unsigned)px + (unsigned)W * uAcc, (unsigned)py + (unsigned)H * uAcc);
        raySeed = rngSeed2((unsigned)px + uAcc * (unsigned)W, (uint32_t)py);
        const float pixel_u = (accumID == 0) ? .5f : rngFloat(rnd);
        const float pixel_v = (accumID == 0) ? .5f : rngFloat(rnd);
        const float image_u = ((px + pixel_u) / float(W));
        const float image_v = ((py + pixel_v) / float(H));
        const float aspect = fr.aspect;  // W / float(H), formed on the host
        const float su = 1.f * aspect * (image_u - .5f), sv = 1.f * (image_v - .5f);
        float3 d = f3(fr.dir00.x + su * fr.dirdu.x + sv * fr.dirdv.x, fr.dir00.y + su * fr.dirdu.y + sv * fr.dirdv.y,
                      fr.dir00.z + su * fr.dirdu.z + sv * fr.dirdv.z);
        d = normalize3(d);
        float3 o = fr.lens00;
        tMax = 1e30f;
        if (fr.cutPlane.w > -1e28f) {
          const float3 N = f3(fr.cutPlane.x, fr.cutPlane.y, fr.cutPlane.z);
          const float dist_org = dot3(N, o) + fr.cutPlane.w;
          const float denom = dot3(N, d);
          if (dist_org >= 0.f) {
            if (denom < 0.f) tMax = fmin_(tMax, -dist_org / denom);
          } else {
            if (denom > 0.f) {
              const float te = -dist_org / denom;
              o = f3(o.x + te * d.x, o.y + te * d.y, o.z + te * d.z);
            } else tMax = 0.f;
          }
        }
        meta &= ~16;  // a primary ray
        nRays++;
        org = o;
        dir = d;
        phase = LP_BEGIN;
      }
      // A5: TraceRays::run fix-up, isProg prologue, dda3 set-up
      if (phase == LP_BEGIN) {
        TraceState ts;
        const bool inside = traceBegin(v, ts, org, dir, tMax, raySeed);
        sh.ox[s] = ts.org.x;
        sh.oy[s] = ts.org.y;
        sh.oz[s] = ts.org.z;
        sh.dx[s] = ts.dir.x;
        sh.dy[s] = ts.dir.y;
        sh.dz[s] = ts.dir.z;
        sh.rayTMax[s] = ts.rayTMax;
        sh.seedLo[s] = (unsigned)raySeed;
        sh.seedHi[s] = (unsigned)(raySeed >> 32);
        if (inside) {
          sh.ddaTMax[s] = ts.ddaTMax;
          sh.rayT0[s] = ts.rayT0;
          sh.ncb[s] = ts.nextCellBegin;
          sh.tnx[s] = ts.tNext.x;
          sh.tny[s] = ts.tNext.y;
          sh.tnz[s] = ts.tNext.z;
          sh.tsx[s] = ts.tStep.x;
          sh.tsy[s] = ts.tStep.y;
          sh.tsz[s] = ts.tStep.z;
          sh.cx[s] = ts.cx;
          sh.cy[s] = ts.cy;
          sh.cz[s] = ts.cz;
          sh.rngLo[s] = (unsigned)ts.rng;
          sh.rngHi[s] = (unsigned)(ts.rng >> 32);
          sh.steps[s] = 0;
          meta = (meta & ~(15 | (63 << 8))) | LP_CELL | (ts.bits << 8);
          phase = LP_CELL;
        } else {
          // rays that miss keep only their fix-up bits (none are read at a miss)
          meta = (meta & ~15) | LP_ENDED;
          phase = LP_ENDED;
        }
      }
      if (s >= 0 && phase != kAQDrop) {
        if (dirty) {
          sh.acc[s] = acc;
          sh.k[s] = kk;
        }
        if (phase != LP_IDLE) sh.meta[s] = meta;
      }
      const bool keep = s >= 0 && phase != kAQDrop;
      ok &= aqPush(sh, AQ_TRACE, keep && phase == LP_CELL, s);
      ok &= aqPush(sh, AQ_END, keep && phase == LP_ENDED, s);
      ok &= aqPush(sh, AQ_IDLE, keep && phase == LP_IDLE, s);
    }
    if (!__all_sync(FULL, ok)) {
      errBits |= ERR_ITER_CAP;
      if (lane == 0) atomicExch(&sh.failed, 1);
      break;
    }
  }
  if (threadIdx.x == 0 && aqLoadI(&sh.aborted)) errBits |= ERR_ABORTED;
  unsigned long long wSamples = nSamples, wVisits = nVisits, wRays = nRays;
  for (int o = 16; o > 0; o >>= 1) {
    wSamples += __shfl_down_sync(FULL, wSamples, o);
    wVisits += __shfl_down_sync(FULL, wVisits, o);
    wRays += __shfl_down_sync(FULL, wRays, o);
    errBits |= __shfl_down_sync(FULL, errBits, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&ctr->samples, wSamples);
    atomicAdd(&ctr->mcVisits, wVisits);
    atomicAdd(&ctr->rays, wRays);
    if (errBits) atomicOr(&ctr->errorFlags, (unsigned long long)errBits);
  }
}

// T: the voxel type every job of the batch has, or -1 (mixed: a switch per sample)
template <int T, int EXT, int CMP>
__global__ void __launch_bounds__(kRenderMaxThreads, EXT >= 2     ? kRenderMinBlocksIso
                                                     : EXT        ? kRenderMinBlocksExt
                                                     : CMP == 1   ? kRenderMinBlocksMixedComp
                                                                  : kRenderMinBlocks)
    renderBatchKernel(const JobDD *__restrict__ jobs, const int *__restrict__ chunkStart, int numJobs, const __grid_constant__ SchedDD sd,
                      LaunchCounters *ctr) {
  __shared__ float u8lut[256];
  __shared__ float sIsoBuf[EXT >= 2 ? kRenderMaxThreads / 32 * kIsoBufPerWarp : 1];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) u8lut[i] = __fdiv_rn((float)i * 1.f, 255.f);
  __syncthreads();
  // plain batch kernels draw free-flight distances with fastLog only; batches
  // with an exact-log job run the extended kernel, which chooses per job
  renderLoop<T, true, EXT ? 2 : 0, EXT, CMP>(jobs, chunkStart, numJobs, __ldg(chunkStart + numJobs), sd, ctr, nullptr,
                                             u8lut, EXT >= 2 ? sIsoBuf + (threadIdx.x >> 5) * kIsoBufPerWarp : nullptr);
}

// Field samples and transfer-function lookups at given points
// (bnxVolumeSample): the structured sampler (NaN outside) and sampleAndMap
// (Volume.h:62-74), with the expressions of the render loop's Woodcock step.
template <int T>
__global__ void sampleProbeKernel(VolumeDD v, const float3 *P, int n, float *scalar, float4 *rgba) {
  __shared__ float u8lut[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) u8lut[i] = __fdiv_rn((float)i * 1.f, 255.f);
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float s = sampleField<T>(v, P[i], u8lut);
    float4 m = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!isnan(s)) {
      int idx;
      float f;
      tfLocate(v, s, idx, f);
      const float4 a = v.tf[idx], b = v.tf[idx + 1];
      float3 rgb = f3(lerp_l(f, a.x, b.x), lerp_l(f, a.y, b.y), lerp_l(f, a.z, b.z));
      float w = __fmul_rn(lerp_l(f, a.w, b.w), v.baseDensity);
      if (v.pv.enabled) {  // principled: TF density 0 maps to 0, else sigma_t and tint times the TF's
        if (w <= 0.f) {
          rgb = f3(0.f, 0.f, 0.f);
          w = 0.f;
        } else {
          rgb = principledTintTimes(v.pv, s, rgb);
          w = principledSigmaT(v.pv, s) * w;
        }
      }
      m = make_float4(rgb.x, rgb.y, rgb.z, w);
    }
    scalar[i] = s;
    rgba[i] = m;
  }
}

#ifndef BNB_FAST_MATH
// ---------------------------------------------------------------------------
// resolve (TiledFB.cu:13-52, math.h:61-125)
// ---------------------------------------------------------------------------
DEV float linearToSrgb(float x) {
  if (x <= 0.0031308f) return 12.92f * x;
  return 1.055f * powf(x, 1.f / 2.4f) - 0.055f;
}
DEV uint32_t make8(float f) { return (uint32_t)min(255, max(0, int(f * 256.f))); }

__global__ void resolveKernel(const float4 *accum, const float4 *comp, int n, float accumScale, int fmt, void *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 a = accum[i];
    if (comp) {  // compensated accumulation: add the running error back before scaling
      const float4 c = comp[i];
      a = make_float4(a.x + c.x, a.y + c.y, a.z + c.z, a.w + c.w);
    }
    float4 c = make_float4(a.x * accumScale, a.y * accumScale, a.z * accumScale, a.w * accumScale);
    if (fmt == FMT_FLOAT4) {
      ((float4 *)out)[i] = c;
    } else {
      if (fmt == FMT_RGBA8_SRGB) { c.x = linearToSrgb(c.x); c.y = linearToSrgb(c.y); c.z = linearToSrgb(c.z); }
      ((uint32_t *)out)[i] = (make8(c.x) << 0) + (make8(c.y) << 8) + (make8(c.z) << 16) + (make8(c.w) << 24);
    }
  }
}

// batch resolve: one 32-thread group per pixel chunk of any job
__global__ void resolveBatchKernel(const JobDD *jobs, const int *chunkStart, int numJobs, int numChunks) {
  const int groupsPerBlock = blockDim.x / 32;
  const int sub = threadIdx.x & 31;
  for (int c = blockIdx.x * groupsPerBlock + threadIdx.x / 32; c < numChunks; c += gridDim.x * groupsPerBlock) {
    int lo = 0, hi = numJobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(chunkStart + mid) <= c) lo = mid; else hi = mid - 1;
    }
    const FrameDD &fr = jobs[lo].fr;
    const int i = (c - __ldg(chunkStart + lo)) * 32 + sub;
    if (i >= fr.width * fr.height) continue;
    // pixel i of the chunk order maps to the same pixel as in the render loop
    const int W = fr.width, H = fr.height;
    const int band = i / (4 * W);
    const int rows = min(4, H - 4 * band);
    const int within = i - band * 4 * W;
    const int64_t p = (int64_t)(4 * band + within % rows) * W + within / rows;
    float4 a = fr.accum[p];
    if (fr.comp) {
      const float4 cc = fr.comp[p];
      a = make_float4(a.x + cc.x, a.y + cc.y, a.z + cc.z, a.w + cc.w);
    }
    const float accumScale = 1.f / (fr.accumID0 + fr.spp);
    float4 col = make_float4(a.x * accumScale, a.y * accumScale, a.z * accumScale, a.w * accumScale);
    if (fr.colorFormat == FMT_FLOAT4) {
      ((float4 *)fr.color)[p] = col;
    } else {
      if (fr.colorFormat == FMT_RGBA8_SRGB) { col.x = linearToSrgb(col.x); col.y = linearToSrgb(col.y); col.z = linearToSrgb(col.z); }
      ((uint32_t *)fr.color)[p] = (make8(col.x) << 0) + (make8(col.y) << 8) + (make8(col.z) << 16) + (make8(col.w) << 24);
    }
  }
}

#endif  // !BNB_FAST_MATH

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int smCount() {
  static int n = 0;
  if (!n) {
    int dev = 0, c = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
      cudaGetLastError();
      return 1;
    }
    n = c;
  }
  return n;
}

#ifndef BNB_FAST_MATH
// Occupancy bitmap of a majorant grid: one ballot per warp packs the
// "majorant != 0" flags of 32 consecutive macrocells into one word.  The
// render loop tests these bits (32 KB for a 64^3 grid, resident in L1)
// instead of loading a majorant for every macrocell it crosses.
__global__ void __launch_bounds__(256) mcOccupancyKernel(const float *majorants, int64_t n, unsigned *occupied) {
  const int lane = threadIdx.x & 31;
  const int64_t words = (n + 31) >> 5;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < words; w += warps) {
    const int64_t i = (w << 5) + lane;
    const bool occ = i < n && majorants[i] != 0.f;
    const unsigned bits = __ballot_sync(0xffffffffu, occ);
    if (lane == 0) occupied[w] = bits;
  }
}

static cudaError_t launchOccupancy(const float *majorants, int64_t n, unsigned *occupied, cudaStream_t s) {
  const int64_t words = (n + 31) >> 5;
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((words + 7) / 8, (int64_t)smCount() * 8));
  mcOccupancyKernel<<<blocks, 256, 0, s>>>(majorants, n, occupied);
  return cudaGetLastError();
}

cudaError_t launchBuildMacrocells(const VolumeDD &v, float2 *ranges, float *majorants, unsigned *occupied, int roundUp,
                                  cudaStream_t s) {
  const int64_t n = (int64_t)v.mcDims.x * v.mcDims.y * v.mcDims.z;
  const int blocks = (int)std::min<int64_t>((n + 127) / 128, (int64_t)smCount() * 16);
  switch (v.type) {
  case VOX_F32: mcBuildKernel<VOX_F32><<<blocks, 128, 0, s>>>(v, ranges, majorants, roundUp); break;
  case VOX_U8: mcBuildKernel<VOX_U8><<<blocks, 128, 0, s>>>(v, ranges, majorants, roundUp); break;
  case VOX_F16: mcBuildKernel<VOX_F16><<<blocks, 128, 0, s>>>(v, ranges, majorants, roundUp); break;
  case VOX_U16: mcBuildKernel<VOX_U16><<<blocks, 128, 0, s>>>(v, ranges, majorants, roundUp); break;
  default: mcBuildKernel<VOX_BF16><<<blocks, 128, 0, s>>>(v, ranges, majorants, roundUp); break;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !majorants) return e;
  return launchOccupancy(majorants, n, occupied, s);
}

cudaError_t launchMapMajorants(const VolumeDD &v, const float2 *ranges, float *majorants, unsigned *occupied,
                               int roundUp, cudaStream_t s) {
  const int64_t n = (int64_t)v.mcDims.x * v.mcDims.y * v.mcDims.z;
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)smCount() * 8);
  mcMapKernel<<<blocks, 256, 0, s>>>(v, ranges, majorants, roundUp);
  cudaError_t e = cudaGetLastError();
  return e != cudaSuccess ? e : launchOccupancy(majorants, n, occupied, s);
}
#endif  // !BNB_FAST_MATH

template <int T>
static cudaError_t launchRenderT(const VolumeDD &v, const FrameDD &fr, const SchedDD &sd, LaunchCounters *ctr,
                                 int bps, int tpb, cudaStream_t s) {
  const size_t smem = (size_t)v.tfN * sizeof(float4);
  const bool pvms = fr.maxVolumeBounces > 0 || v.pv.enabled;
  const int ext = v.iso.enabled ? (pvms ? 2 : 3) : pvms ? 1 : 0;
  // kernels with and without compensated sums
  const bool cmp = fr.comp != nullptr;
#ifdef BNB_FAST_MATH
  if (ext) return cudaErrorInvalidValue;  // the fast-math object holds the plain kernels only
  auto kern = cmp ? (fr.exactLog ? renderKernel<T, 1, 0, 2> : renderKernel<T, 0, 0, 2>)
                  : (fr.exactLog ? renderKernel<T, 1, 0, 0> : renderKernel<T, 0, 0, 0>);
#else
  // isosurfaces without volume bounces or principled volumes: the smaller
  // EXT 3 kernel unless the job keeps compensated sums
  auto kern = ext == 3 && !cmp ? (fr.exactLog ? renderKernel<T, 1, 3, 0> : renderKernel<T, 0, 3, 0>)
              : ext >= 2 ? (cmp ? (fr.exactLog ? renderKernel<T, 1, 2, 2> : renderKernel<T, 0, 2, 2>)
                                : (fr.exactLog ? renderKernel<T, 1, 2, 0> : renderKernel<T, 0, 2, 0>))
              : ext == 1 ? (cmp ? (fr.exactLog ? renderKernel<T, 1, 1, 2> : renderKernel<T, 0, 1, 2>)
                                : (fr.exactLog ? renderKernel<T, 1, 1, 0> : renderKernel<T, 0, 1, 0>))
              : cmp ? (fr.exactLog ? renderKernel<T, 1, 0, 2> : renderKernel<T, 0, 0, 2>)
                    : (fr.exactLog ? renderKernel<T, 1, 0, 0> : renderKernel<T, 0, 0, 0>);
#endif
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return cudaGetLastError();
  if (bps <= 0) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, tpb, smem) != cudaSuccess) return cudaGetLastError();
    bps = occ > 0 ? occ : 1;
  }
  JobDD job;
  job.v = v;
  job.fr = fr;
  kern<<<smCount() * bps, tpb, smem, s>>>(job, sd, ctr);
  return cudaGetLastError();
}

template <int T>
static cudaError_t launchRenderWFT(const VolumeDD &v, const FrameDD &fr, LaunchCounters *ctr, cudaStream_t s) {
  const size_t smem = wfSlotsBytes() + (size_t)v.tfN * sizeof(float4);
  auto kern = fr.exactLog ? renderKernelWF<T, 1> : renderKernelWF<T, 0>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return cudaGetLastError();
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kAQThreads, smem) != cudaSuccess)
    return cudaGetLastError();
  JobDD job;
  job.v = v;
  job.fr = fr;
  kern<<<smCount() * (occ > 0 ? occ : 1), kAQThreads, smem, s>>>(job, ctr);
  return cudaGetLastError();
}

cudaError_t launchRenderRegrouped(const VolumeDD &v, const FrameDD &fr, LaunchCounters *ctr, cudaStream_t s) {
  if (v.iso.enabled || fr.maxVolumeBounces > 0 || v.pv.enabled) return cudaErrorInvalidValue;  // plain jobs only
  switch (v.type) {
  case VOX_F32: return launchRenderWFT<VOX_F32>(v, fr, ctr, s);
  case VOX_U8: return launchRenderWFT<VOX_U8>(v, fr, ctr, s);
  case VOX_F16: return launchRenderWFT<VOX_F16>(v, fr, ctr, s);
  case VOX_U16: return launchRenderWFT<VOX_U16>(v, fr, ctr, s);
  default: return launchRenderWFT<VOX_BF16>(v, fr, ctr, s);
  }
}

cudaError_t launchRender(const VolumeDD &v, const FrameDD &fr, LaunchCounters *ctr, int bps, int tpb, cudaStream_t s,
                         const SchedDD &sd) {
  if (tpb <= 0) tpb = 128;
  switch (v.type) {
  case VOX_F32: return launchRenderT<VOX_F32>(v, fr, sd, ctr, bps, tpb, s);
  case VOX_U8: return launchRenderT<VOX_U8>(v, fr, sd, ctr, bps, tpb, s);
  case VOX_F16: return launchRenderT<VOX_F16>(v, fr, sd, ctr, bps, tpb, s);
  case VOX_U16: return launchRenderT<VOX_U16>(v, fr, sd, ctr, bps, tpb, s);
  default: return launchRenderT<VOX_BF16>(v, fr, sd, ctr, bps, tpb, s);
  }
}

template <int EXT, int CMP>
static auto batchKernelFor(int voxelType) {
  switch (voxelType) {
  case VOX_F32: return renderBatchKernel<VOX_F32, EXT, CMP>;
  case VOX_U8: return renderBatchKernel<VOX_U8, EXT, CMP>;
  case VOX_F16: return renderBatchKernel<VOX_F16, EXT, CMP>;
  case VOX_U16: return renderBatchKernel<VOX_U16, EXT, CMP>;
  case VOX_BF16: return renderBatchKernel<VOX_BF16, EXT, CMP>;
  default: return renderBatchKernel<-1, EXT, CMP>;
  }
}

// A batch of at most kParamJobs plain jobs passed as a kernel parameter
// (constant bank) instead of a table in global memory: the jobs' fields are
// read through the constant cache, as the single-frame kernel reads its job.
// Used for launches outside graph capture (a parameter would be frozen into
// a graph); measured 4 % more served frames/s than the table.
struct JobTableParam {
  JobDD jobs[kParamJobs];
  int chunkStart[kParamJobs + 1];
};
template <int T, int CMP>
__global__ void __launch_bounds__(kRenderMaxThreads, CMP == 1 ? kRenderMinBlocksMixedComp : kRenderMinBlocks)
    renderBatchParamKernel(const __grid_constant__ JobTableParam tab, int numJobs, const __grid_constant__ SchedDD sd,
                           LaunchCounters *ctr) {
  __shared__ float u8lut[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) u8lut[i] = __fdiv_rn((float)i * 1.f, 255.f);
  __syncthreads();
  renderLoop<T, true, 0, 0, CMP>(tab.jobs, tab.chunkStart, numJobs, tab.chunkStart[numJobs], sd, ctr, nullptr, u8lut,
                                 nullptr);
}
template <int CMP>
static auto batchParamKernelFor(int voxelType) {
  switch (voxelType) {
  case VOX_F32: return renderBatchParamKernel<VOX_F32, CMP>;
  case VOX_U8: return renderBatchParamKernel<VOX_U8, CMP>;
  case VOX_F16: return renderBatchParamKernel<VOX_F16, CMP>;
  case VOX_U16: return renderBatchParamKernel<VOX_U16, CMP>;
  case VOX_BF16: return renderBatchParamKernel<VOX_BF16, CMP>;
  default: return renderBatchParamKernel<-1, CMP>;
  }
}
cudaError_t launchRenderBatchParams(const JobDD *hostJobs, const int *hostChunkStart, int numJobs,
                                    LaunchCounters *ctr, int bps, int tpb, cudaStream_t s, const SchedDD &sd,
                                    int voxelType, int compensated) {
  if (numJobs < 1 || numJobs > kParamJobs) return cudaErrorInvalidValue;
  if (tpb <= 0) tpb = 128;
  auto kern = compensated == 2   ? batchParamKernelFor<2>(voxelType)
              : compensated == 1 ? batchParamKernelFor<1>(voxelType)
                                 : batchParamKernelFor<0>(voxelType);
  if (bps <= 0) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, tpb, 0) != cudaSuccess)
      return cudaGetLastError();
    bps = occ > 0 ? occ : 1;
  }
  // host staging of the 31 KB parameter (the launch copies it); one launch
  // at a time fills it
  static JobTableParam tab;
  static std::mutex m;
  std::lock_guard<std::mutex> l(m);
  memcpy(tab.jobs, hostJobs, numJobs * sizeof(JobDD));
  memcpy(tab.chunkStart, hostChunkStart, (numJobs + 1) * sizeof(int));
  kern<<<smCount() * bps, tpb, 0, s>>>(tab, numJobs, sd, ctr);
  return cudaGetLastError();
}

cudaError_t launchRenderBatch(const JobDD *jobs, const int *chunkStart, int numJobs, LaunchCounters *ctr, int bps,
                              int tpb, cudaStream_t s, const SchedDD &sd, int extended, int voxelType,
                              int compensated) {
  if (tpb <= 0) tpb = 128;
#ifdef BNB_FAST_MATH
  if (extended) return cudaErrorInvalidValue;  // the fast-math object holds the plain kernels only
  auto kern = compensated == 2   ? batchKernelFor<0, 2>(voxelType)
              : compensated == 1 ? batchKernelFor<0, 1>(voxelType)
                                 : batchKernelFor<0, 0>(voxelType);
#else
  auto kern = extended == 3 && !compensated ? batchKernelFor<3, 0>(voxelType)
              : extended >= 2    ? (compensated ? batchKernelFor<2, 1>(voxelType) : batchKernelFor<2, 0>(voxelType))
              : extended         ? (compensated ? batchKernelFor<1, 1>(voxelType) : batchKernelFor<1, 0>(voxelType))
              : compensated == 2 ? batchKernelFor<0, 2>(voxelType)
              : compensated == 1 ? batchKernelFor<0, 1>(voxelType)
                                 : batchKernelFor<0, 0>(voxelType);
#endif
  if (bps <= 0) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, tpb, 0) != cudaSuccess)
      return cudaGetLastError();
    bps = occ > 0 ? occ : 1;
  }
  kern<<<smCount() * bps, tpb, 0, s>>>(jobs, chunkStart, numJobs, sd, ctr);
  return cudaGetLastError();
}

cudaError_t launchSampleProbe(const VolumeDD &v, const float3 *P, int n, float *scalar, float4 *rgba, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int blocks = std::max(1, std::min((n + 255) / 256, smCount() * 8));
  switch (v.type) {
  case VOX_F32: sampleProbeKernel<VOX_F32><<<blocks, 256, 0, s>>>(v, P, n, scalar, rgba); break;
  case VOX_U8: sampleProbeKernel<VOX_U8><<<blocks, 256, 0, s>>>(v, P, n, scalar, rgba); break;
  case VOX_F16: sampleProbeKernel<VOX_F16><<<blocks, 256, 0, s>>>(v, P, n, scalar, rgba); break;
  case VOX_U16: sampleProbeKernel<VOX_U16><<<blocks, 256, 0, s>>>(v, P, n, scalar, rgba); break;
  default: sampleProbeKernel<VOX_BF16><<<blocks, 256, 0, s>>>(v, P, n, scalar, rgba); break;
  }
  return cudaGetLastError();
}

#ifdef BNB_BOUNDS_CHECK
// out-of-range accesses counted by this object's kernels since the last call
long long readBoundsViolationsHere() {
  unsigned long long n = 0, zero = 0;
  if (cudaMemcpyFromSymbol(&n, g_boundsViolations, sizeof n) != cudaSuccess) return -2;
  if (cudaMemcpyToSymbol(g_boundsViolations, &zero, sizeof zero) != cudaSuccess) return -2;
  return (long long)n;
}
#endif

#ifndef BNB_FAST_MATH
cudaError_t launchResolveBatch(const JobDD *jobs, const int *chunkStart, int numJobs, int numChunks, cudaStream_t s) {
  const int blocks = std::max(1, std::min((numChunks + 7) / 8, smCount() * 8));
  resolveBatchKernel<<<blocks, 256, 0, s>>>(jobs, chunkStart, numJobs, numChunks);
  return cudaGetLastError();
}

cudaError_t launchResolve(const float4 *accum, int n, int accumID, int fmt, void *out, cudaStream_t s,
                          const float4 *comp) {
  const float accumScale = 1.f / accumID;
  const int blocks = std::max(1, std::min((n + 255) / 256, smCount() * 8));
  resolveKernel<<<blocks, 256, 0, s>>>(accum, comp, n, accumScale, fmt, out);
  return cudaGetLastError();
}

bool boundsCheckedBuild() {
#ifdef BNB_BOUNDS_CHECK
  return true;
#else
  return false;
#endif
}

// Out-of-range accesses the bounds-checked build has counted (and resets
// the count); -1 in the normal build.
long long readBoundsViolations() {
#ifdef BNB_BOUNDS_CHECK
  const long long a = readBoundsViolationsHere(), b = fastmath::readBoundsViolationsHere();
  return (a < 0 || b < 0) ? -2 : a + b;
#else
  return -1;
#endif
}

// ---------------------------------------------------------------------------
// No-allocation render (bnxRenderStructuredNoAlloc)
//
// Scratch of this path -- the macrocell majorant grid, its occupancy bitmap
// and the launch counters -- lives in the file-scope array below instead of
// in memory the context allocates.  It is sized for kNoAllocMaxMacrocells
// macrocells (64^3, i.e. grids up to 513^3 scalars) and is held by every GPU
// that loads the library until the process exits: 1 MiB of majorants +
// 32 KiB of bitmap + 256 bytes of counters.  All calls share it, so calls whose work overlaps on the GPU
// race; each call overwrites the majorants it needs and clears the counters.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocCountersBytes = 256;
constexpr size_t kNoAllocMajorantBytes = kNoAllocMaxMacrocells * sizeof(float);
static __device__ __align__(256) unsigned char
    g_noAllocScratch[kNoAllocCountersBytes + kNoAllocMajorantBytes + kNoAllocMaxMacrocells / 8];

// Majorant grid straight from the voxels: the fused build of mcBuildKernel
// without storing the scalar ranges.
template <int T>
__global__ void __launch_bounds__(128) mcMajorantScratchKernel(VolumeDD v, int roundUp) {
  __shared__ float u8lut[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) u8lut[i] = __fdiv_rn((float)i * 1.f, 255.f);
  __syncthreads();
  float *majorants = (float *)(g_noAllocScratch + kNoAllocCountersBytes);
  const int64_t n = (int64_t)v.mcDims.x * v.mcDims.y * v.mcDims.z;
  for (int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; tid < n; tid += (int64_t)gridDim.x * blockDim.x) {
    const int mx = (int)(tid % v.mcDims.x);
    const int my = (int)((tid / v.mcDims.x) % v.mcDims.y);
    const int mz = (int)(tid / ((int64_t)v.mcDims.x * v.mcDims.y));
    const int x0 = mx * kCellsPerMC, y0 = my * kCellsPerMC, z0 = mz * kCellsPerMC;
    const int x1 = min(x0 + kCellsPerMC, v.numScalars.x - 1);
    const int y1 = min(y0 + kCellsPerMC, v.numScalars.y - 1);
    const int z1 = min(z0 + kCellsPerMC, v.numScalars.z - 1);
    float lo = kInf, hi = -kInf;
    const int64_t nx = v.numScalars.x, nxy = (int64_t)v.numScalars.x * v.numScalars.y;
    if (!BNB_IN(x1 + nx * y1 + nxy * z1, nxy * v.numScalars.z)) {
      // (bounds-checked build) a counted violation: a zero majorant, not the
      // previous call's value left in the shared scratch
      majorants[tid] = 0.f;
      continue;
    }
    for (int z = z0; z <= z1; z++)
      for (int y = y0; y <= y1; y++) {
        const int64_t row = nx * y + nxy * z;
        for (int x = x0; x <= x1; x++) {
          float f = loadVoxel<T>(v.voxels, row + x, u8lut);
          lo = fmin_(lo, f);
          hi = fmax_(hi, f);
        }
      }
    majorants[tid] = roundUpMajorant(mapMajorant(v, lo, hi), roundUp);
  }
}

// Device address of g_noAllocScratch on the current device (the host-side
// name of the array is only a stand-in, never a device address).  Looked up
// with cudaGetSymbolAddress on every call made while stream s is not
// capturing, so that a device reset, after which the module and its array
// are loaded anew, is picked up; a call on a capturing stream uses the
// address its device's last such call found.
static void *noAllocScratchAddress(cudaStream_t s, cudaError_t *err) {
  static std::mutex m;
  static void *addr[64] = {nullptr};
  int dev = 0;
  *err = cudaGetDevice(&dev);
  if (*err != cudaSuccess) return nullptr;
  if (dev < 0 || dev >= 64) { *err = cudaErrorInvalidDevice; return nullptr; }
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  *err = cudaStreamIsCapturing(s, &capture);
  if (*err != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> l(m);
  if (capture == cudaStreamCaptureStatusNone || !addr[dev]) {
    void *p = nullptr;
    *err = cudaGetSymbolAddress(&p, g_noAllocScratch);
    if (*err != cudaSuccess) return nullptr;
    addr[dev] = p;
  }
  return addr[dev];
}

cudaError_t launchRenderNoAlloc(VolumeDD v, FrameDD fr, int fmt, void *color, int roundUp, cudaStream_t s) {
  const int64_t n = (int64_t)v.mcDims.x * v.mcDims.y * v.mcDims.z;
  if (n <= 0 || n > kNoAllocMaxMacrocells) return cudaErrorInvalidValue;
  cudaError_t e = cudaSuccess;
  unsigned char *base = (unsigned char *)noAllocScratchAddress(s, &e);
  if (!base) return e;
  LaunchCounters *ctr = (LaunchCounters *)base;
  float *majorants = (float *)(base + kNoAllocCountersBytes);
  unsigned *occupied = (unsigned *)(base + kNoAllocCountersBytes + kNoAllocMajorantBytes);
  v.majorants = majorants;
  v.mcOccupied = occupied;
  e = cudaMemsetAsync(ctr, 0, sizeof(LaunchCounters), s);
  if (e != cudaSuccess) return e;
  const int blocks = (int)std::min<int64_t>((n + 127) / 128, (int64_t)smCount() * 16);
  switch (v.type) {
  case VOX_F32: mcMajorantScratchKernel<VOX_F32><<<blocks, 128, 0, s>>>(v, roundUp); break;
  case VOX_U8: mcMajorantScratchKernel<VOX_U8><<<blocks, 128, 0, s>>>(v, roundUp); break;
  case VOX_F16: mcMajorantScratchKernel<VOX_F16><<<blocks, 128, 0, s>>>(v, roundUp); break;
  case VOX_U16: mcMajorantScratchKernel<VOX_U16><<<blocks, 128, 0, s>>>(v, roundUp); break;
  default: mcMajorantScratchKernel<VOX_BF16><<<blocks, 128, 0, s>>>(v, roundUp); break;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = launchOccupancy(majorants, n, occupied, s);
  if (e != cudaSuccess) return e;
  e = launchRender(v, fr, ctr, 0, 0, s);
  if (e != cudaSuccess) return e;
  return launchResolve(fr.accum, fr.width * fr.height, fr.accumID0 + fr.spp, fmt, color, s);
}
#endif  // !BNB_FAST_MATH

#ifdef BNB_FAST_MATH
}  // namespace fastmath
#endif
}  // namespace bnb
