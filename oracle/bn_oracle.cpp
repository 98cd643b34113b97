// bn_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of Barney's structured-volume path-tracing hot path, used
// as the parity checker for the CUDA implementation in barney_b200/.  Only
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
// legs may load this library; the product never links or calls it.
//
// Parity status: the reference cannot be compiled here (its owl, cuBQL,
// embree and optix submodules are empty and the ANARI SDK is absent) and its
// own tests hold no golden vectors for this path, so this restatement is
// "parity unpinned" against reference outputs.  It is pinned instead against
// (a) hand-derived known-answer values written into tests/test_oracle_kat.py
// and (b) the committed fixtures under tests/golden/, generated from this
// file by tests/golden/make_golden.py.
//
// Arithmetic convention: every expression is evaluated in IEEE-754 binary32
// in the order the reference source writes it, with no FMA contraction
// (built with -ffp-contract=off).  Division and sqrt are correctly rounded.
//
// Reference files followed (paths relative to the Barney source tree):
//   barney/native/common/barney-common.h:21-108   RNGSeed, Random2, hash
//   barney/native/common/math.h:13-18,61-128      constants, sRGB, make_rgba, clamp
//   barney/native/Camera.cu:82-100                perspective camera commit
//   barney/native/kernels/generateRays.cu:43-244  primary ray generation
//   barney/native/kernels/traceRays.dev.cu:26-52  zero-direction fix-up
//   barney/native/render/Ray.h:111-217            setVolumeHit, makeShadowRay, boxTest
//   barney/native/volume/MCAccelerator.h:552-689  MCVolumeAccel::isProg
//   barney/native/volume/DDA.h:61-201             dda3
//   barney/native/volume/Volume.h:62-74,154-203   sampleAndMap, fastLog, Woodcock
//   barney/native/volume/StructuredData.h:101-112 structured sampler
//   barney/rtcore/cpu/Texture.cpp:193-276,324-416 software point / linear filtering
//   barney/native/volume/TransferFunction.h:68-117 map, majorant
//   barney/native/volume/StructuredData.cu:26-96  macrocell range build
//   barney/native/volume/MCGrid.cu:97-141         mapMCs
//   barney/native/kernels/shadeRays.cu:17-402,475-1042 light sampling, bounce, accumulate
//   barney/native/packedBSDF/Phase.h:14-176       HGPhase, SimplePhase
//   barney/native/render/DG.h:162-193             cosineSampleHemisphere, randomDirection
//   barney/native/volume/MCAccelerator.h:325-548  MCIsoSurfaceAccel::isProg (isosurface hit, normal)
//   barney/native/geometry/IsoSurface.cpp:36-90   isoSurface parameters
//   barney/native/material/AnariMatte.h:49-71     matte material -> Lambertian
//   barney/native/material/HostMaterial.h:98-115  constant material parameters
//   barney/native/packedBSDF/Lambertian.h:45-86   Lambertian pdf, eval, scatter
//   barney/native/light/EnvMap.h:136-151          constant-env pdf
//   barney/native/light/DirLight.cu:11-20         directional light device data
//   barney/native/fb/TiledFB.cu:13-52, LocalFB.cpp:61-71 resolve / tonemap
//   barney/rtcore/cpu/Float16.cpp:25+             float -> half, round to nearest even
//   barney/rtcore/cpu/Compute.cpp:17-80           job-per-block thread pool (CPU baseline)

#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace orc {

// ---------------------------------------------------------------------------
// small vector math (owl::common semantics restated from their meaning)
// ---------------------------------------------------------------------------
struct vec3f { float x, y, z; };
struct vec4f { float x, y, z, w; };
struct vec3i { int x, y, z; };

static const float INF = std::numeric_limits<float>::infinity();
// math.h:13-18
static const float ONE_PI = (float)M_PI;
static const float TWO_PI = 2.f * ONE_PI;
static const float FOUR_PI = 4.f * ONE_PI;
static const float ONE_OVER_FOUR_PI = 1.f / FOUR_PI;

static inline float fmin_(float a, float b) { return a < b ? a : b; }
static inline float fmax_(float a, float b) { return b < a ? a : b; }
static inline vec3f V(float x, float y, float z) { return {x, y, z}; }
static inline vec3f V(float s) { return {s, s, s}; }
static inline vec3f operator+(vec3f a, vec3f b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline vec3f operator-(vec3f a, vec3f b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline vec3f operator*(vec3f a, vec3f b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
static inline vec3f operator*(float s, vec3f b) { return {s * b.x, s * b.y, s * b.z}; }
static inline vec3f operator*(vec3f a, float s) { return {a.x * s, a.y * s, a.z * s}; }
static inline vec3f operator/(vec3f a, float s) { return {a.x / s, a.y / s, a.z / s}; }
static inline vec3f operator-(vec3f a) { return {-a.x, -a.y, -a.z}; }
static inline vec3f rcp(vec3f a) { return {1.f / a.x, 1.f / a.y, 1.f / a.z}; }
static inline vec3f vmin(vec3f a, vec3f b) { return {fmin_(a.x, b.x), fmin_(a.y, b.y), fmin_(a.z, b.z)}; }
static inline vec3f vmax(vec3f a, vec3f b) { return {fmax_(a.x, b.x), fmax_(a.y, b.y), fmax_(a.z, b.z)}; }
static inline vec3f vabs(vec3f a) { return {fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
static inline vec3f vfloor(vec3f a) { return {floorf(a.x), floorf(a.y), floorf(a.z)}; }
static inline float reduce_max(vec3f a) { return fmax_(fmax_(a.x, a.y), a.z); }
static inline float reduce_min(vec3f a) { return fmin_(fmin_(a.x, a.y), a.z); }
static inline float dot(vec3f a, vec3f b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline vec3f cross(vec3f a, vec3f b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
static inline vec3f normalize(vec3f v) { return v * (1.f / sqrtf(dot(v, v))); }
static inline bool isZero(vec3f v) { return v.x == 0.f && v.y == 0.f && v.z == 0.f; }
static inline float clampf(float f, float lo, float hi) { return fmin_(hi, fmax_(lo, f)); }  // math.h:127
static inline int clampi(int f, int lo, int hi) { return std::min(hi, std::max(lo, f)); }
static inline uint32_t floatBits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

// float -> IEEE binary16, round to nearest even (the conversion Float16.cpp:25
// and __float2half_rn both perform), and back.
static inline uint16_t f2h(float f) {
  uint32_t x = floatBits(f);
  uint32_t sign = (x >> 16) & 0x8000u;
  uint32_t ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u) return (uint16_t)(sign | 0x7c00u | (ax > 0x7f800000u ? 0x200u : 0u));
  if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);  // rounds to >= 65520 -> inf
  if (ax < 0x38800000u) {                                     // result is subnormal or zero
    if (ax < 0x33000000u) return (uint16_t)sign;              // < 2^-25 -> zero
    uint32_t e = ax >> 23;
    uint32_t m = (ax & 0x7fffffu) | 0x800000u;
    uint32_t shift = 126u - e;                                // 14..24
    uint32_t q = m >> shift;
    uint32_t rem = m & ((1u << shift) - 1u);
    uint32_t half = 1u << (shift - 1u);
    if (rem > half || (rem == half && (q & 1u))) q++;
    return (uint16_t)(sign | q);
  }
  uint32_t e = (ax >> 23) - 112u;  // rebias 127 -> 15
  uint32_t m = ax & 0x7fffffu;
  uint32_t q = (e << 10) | (m >> 13);
  uint32_t rem = m & 0x1fffu;
  if (rem > 0x1000u || (rem == 0x1000u && (q & 1u))) q++;
  return (uint16_t)(sign | q);
}
static inline float h2f(uint16_t h) {
  uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
  uint32_t e = (h >> 10) & 0x1fu, m = h & 0x3ffu, out;
  if (e == 0) {
    if (m == 0) out = sign;
    else { float f = (float)m * (1.f / 16777216.f); uint32_t b = floatBits(f); out = sign | b; }
  } else if (e == 31) out = sign | 0x7f800000u | (m << 13);
  else out = sign | ((e + 112u) << 23) | (m << 13);
  float r; memcpy(&r, &out, 4); return r;
}
static inline float bitsFloat(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline float bf2f(uint16_t h) { uint32_t u = (uint32_t)h << 16; float r; memcpy(&r, &u, 4); return r; }
static inline vec3f halfRound(vec3f v) { return {h2f(f2h(v.x)), h2f(f2h(v.y)), h2f(f2h(v.z))}; }

// ---------------------------------------------------------------------------
// RNG and hash -- barney-common.h:21-108
// ---------------------------------------------------------------------------
struct RNGSeed {
  uint64_t state = 0xcafef00dd15ea5e5ull;
  void seed(uint32_t a, uint32_t b) {
    state ^= (uint32_t)(2u * a + 1u);
    next();
    state ^= (uint32_t)(2u * b);
    next();
  }
  uint32_t next() {
    uint64_t x = state;
    const uint64_t multiplier = 6364136223846793005ull;
    unsigned count = (unsigned)(x >> 61);
    state = x * multiplier;
    x ^= x >> 22;
    return (uint32_t)(x >> (22 + count));
  }
  uint32_t nextHashed(uint64_t h) { state ^= (h << 1); return next(); }
};
struct Random2 : RNGSeed {
  Random2(uint32_t a, uint32_t b) { seed(a, b); }
  Random2(RNGSeed &s, uint64_t b) { state = s.state; s.next(); nextHashed(b ? b : 290374ull); }
  float operator()() { return (next() & 0x00FFFFFFu) * (1.f / (float)0x01000000); }
};
static inline uint64_t hash1(uint32_t v) { return 0xcbf29ce484222325ULL ^ (0x100000001b3ULL * v); }
static inline uint64_t hash2(uint64_t h, uint32_t v) { return h * 0x100000001b3ULL ^ v; }
static inline uint64_t hash3(uint32_t a, uint32_t b, uint32_t c) { return hash2(hash2(hash1(a), b), c); }

// Volume.h:154-164
static inline float fastLog(float f) {
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
static inline float logPortable(float x) {
  const uint32_t b = floatBits(x);
  int e = (int)((b >> 23) & 0xffu) - 127;
  float m = bitsFloat((b & 0x7fffffu) | 0x3f800000u);
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

// e^x for |x| < 87 (the blackbody colour's powf), shared with the CUDA kernels
// like logPortable: k = rint(x / ln2), r = x - k ln2 (split ln2, |r| <=
// 0.347), e^r as the Taylor series to r^8 (truncation below 3e-9), times 2^k
// by exponent arithmetic.
static inline float expPortable(float x) {
  const float k = rintf(x * 1.44269504f);
  const float r = (x - k * 0.693145751953125f) - k * 1.42860682e-6f;
  const float p = 1.f + r * (1.f + r * (0.5f + r * (1.66666667e-1f + r * (4.16666667e-2f + r * (8.33333333e-3f +
                  r * (1.38888889e-3f + r * (1.98412698e-4f + r * 2.48015873e-5f)))))));
  return p * bitsFloat((uint32_t)((int)k + 127) << 23);
}
// x^y for x > 0 (PrincipledVolume.h's powf), as e^(y log x)
static inline float powPortable(float x, float y) { return expPortable(y * logPortable(x)); }


} // namespace orc

using namespace orc;

// ---------------------------------------------------------------------------
// scene description shared with the Python harness (oracle/__init__.py)
// ---------------------------------------------------------------------------
#include "bn_oracle.h"

extern "C" {

typedef struct {
  unsigned long long samples;      // sampleAndMap calls
  unsigned long long mcVisits;     // DDA cells whose majorant was read
  unsigned long long rays;         // rays traced (primary + shadow)
  unsigned long long pixelSamples;
} OrcStats;
}

namespace orc {

struct Scene {
  const OrcScene &s;
  vec3i numScalars, numCells, mcDims;
  vec3f gridOrigin, gridSpacing, mcOrigin, mcSpacing;
  vec3f boundsLo, boundsHi;
  std::vector<float> majorants;
  std::vector<float> ranges;  // per macrocell lo, hi (MCGrid scalar ranges)
  float isoDelta = 0.f;       // central-difference step of the isosurface normal
  // camera DD, Camera.cu:82-100
  vec3f dir00, dirdu, dirdv, lens00;
  explicit Scene(const OrcScene &s) : s(s) {}
};

// rtcore/cpu/Texture.cpp:193-225 (float, uchar); unorm16 follows the
// GPU backend's normalised read of BN_UFIXED16 (cudaCommon/TextureData.cu:46-51,
// x/65535; the CPU backend has no sampler for it); f16 / bf16 are the
// precision-form extensions (no reference counterpart).
static inline float texel(const OrcScene &s, int64_t idx) {
  switch (s.dtype) {
  case 0: return ((const float *)s.voxels)[idx];
  case 1: { float v = (float)((const uint8_t *)s.voxels)[idx]; return v * 1.f / 255.f; }
  case 2: return h2f(((const uint16_t *)s.voxels)[idx]);
  case 3: return bf2f(((const uint16_t *)s.voxels)[idx]);
  default: { float v = (float)((const uint16_t *)s.voxels)[idx]; return v * 1.f / 65535.f; }  // unorm16
  }
}

// Texture.cpp:324-336
static inline void lerpCoords(int &i0, int &i1, float &f, int N, float tc) {
  if (tc - .5f <= 0.f) { i0 = i1 = 0; f = 0.f; return; }
  if (tc - .5f >= N - 1) { i0 = i1 = N - 1; f = 0.f; return; }
  f = (tc - .5f) - int(tc - .5f);
  i0 = int(tc - .5f);
  i1 = i0 + 1;
}
static inline float lerp_l(float f, float a, float b) { return (1.f - f) * a + f * b; }

// Texture.cpp:339-411, LINEAR filter, unnormalized coordinates, clamp
static float tex3DLinear(const OrcScene &s, float tx, float ty, float tz) {
  const int Nx = s.dims[0], Ny = s.dims[1], Nz = s.dims[2];
  int ix0, ix1, iy0, iy1, iz0, iz1;
  float fx, fy, fz;
  lerpCoords(ix0, ix1, fx, Nx, tx);
  lerpCoords(iy0, iy1, fy, Ny, ty);
  lerpCoords(iz0, iz1, fz, Nz, tz);
  auto addr = [&](int x, int y, int z) { return (int64_t)x + (int64_t)Nx * ((int64_t)y + (int64_t)Ny * z); };
  float v000 = texel(s, addr(ix0, iy0, iz0));
  float v001 = texel(s, addr(ix1, iy0, iz0));
  float v010 = texel(s, addr(ix0, iy1, iz0));
  float v011 = texel(s, addr(ix1, iy1, iz0));
  float v100 = texel(s, addr(ix0, iy0, iz1));
  float v101 = texel(s, addr(ix1, iy0, iz1));
  float v110 = texel(s, addr(ix0, iy1, iz1));
  float v111 = texel(s, addr(ix1, iy1, iz1));
  float v00 = lerp_l(fx, v000, v001);
  float v01 = lerp_l(fx, v010, v011);
  float v10 = lerp_l(fx, v100, v101);
  float v11 = lerp_l(fx, v110, v111);
  float v0 = lerp_l(fy, v00, v01);
  float v1 = lerp_l(fy, v10, v11);
  return lerp_l(fz, v0, v1);
}

// StructuredData.h:101-112
static float sampleField(const Scene &sc, vec3f P) {
  vec3f rel = (P - sc.gridOrigin) * rcp(sc.gridSpacing);
  if (rel.x < 0.f) return NAN;
  if (rel.y < 0.f) return NAN;
  if (rel.z < 0.f) return NAN;
  if (rel.x >= sc.numCells.x) return NAN;
  if (rel.y >= sc.numCells.y) return NAN;
  if (rel.z >= sc.numCells.z) return NAN;
  return tex3DLinear(sc.s, rel.x + .5f, rel.y + .5f, rel.z + .5f);
}

static inline vec4f tfValue(const OrcScene &s, int i) {
  return {s.tf[4 * i + 0], s.tf[4 * i + 1], s.tf[4 * i + 2], s.tf[4 * i + 3]};
}

// TransferFunction.h:68-87
static vec4f tfMap(const OrcScene &s, float v) {
  float span = s.domain[1] - s.domain[0];
  float f = (v - s.domain[0]) / span;
  f = clampf(f, 0.f, 1.f);
  f *= (s.tfN - 1);
  int idx = clampi(int(f), 0, s.tfN - 2);
  f -= idx;
  vec4f v0 = tfValue(s, idx), v1 = tfValue(s, idx + 1);
  vec4f r = {(1.f - f) * v0.x + f * v1.x, (1.f - f) * v0.y + f * v1.y,
             (1.f - f) * v0.z + f * v1.z, (1.f - f) * v0.w + f * v1.w};
  r.w *= s.baseDensity;
  return r;
}

// TransferFunction.h:93-117
static float tfMajorant(const OrcScene &s, float lo, float hi) {
  if (lo > hi) return 0.f;
  float span = s.domain[1] - s.domain[0];
  float f_lo = (lo - s.domain[0]) / span;
  float f_hi = (hi - s.domain[0]) / span;
  f_lo = clampf(f_lo, 0.f, 1.f);
  f_hi = clampf(f_hi, 0.f, 1.f);
  f_lo *= (s.tfN - 1);
  f_hi *= (s.tfN - 1);
  int idx0_lo = clampi(int(f_lo), 0, s.tfN - 2);
  int idx0_hi = clampi(int(f_hi), 0, s.tfN - 2);
  f_lo -= idx0_lo;
  f_hi -= idx0_hi;
  float lerp_lo = (1.f - f_lo) * s.tf[4 * idx0_lo + 3] + f_lo * s.tf[4 * (idx0_lo + 1) + 3];
  float lerp_hi = (1.f - f_hi) * s.tf[4 * idx0_hi + 3] + f_hi * s.tf[4 * (idx0_hi + 1) + 3];
  float m = 0.f;
  m = fmax_(m, lerp_lo);
  m = fmax_(m, lerp_hi);
  for (int i = idx0_lo + 1; i <= idx0_hi; i++) m = fmax_(m, s.tf[4 * i + 3]);
  return m * s.baseDensity;
}

// ---- principled volumes (PrincipledVolume.h:55-175) ----
static inline vec3f pv3(const float *c) { return V(c[0], c[1], c[2]); }
static inline float principledDensityFactor(const OrcScene &s, float scalar) {
  float x = clampf(scalar, s.pValueRange[0], s.pValueRange[1]);
  if (s.pDensityThreshold > 0.f && x < s.pDensityThreshold) return 0.f;
  return s.pDensity * fmax_(x, 0.f) * s.pDensityScale;
}
static inline vec3f principledSigmaS(const OrcScene &s, float scalar) {
  return principledDensityFactor(s, scalar) * pv3(s.pScatterColor);
}
static inline vec3f principledSigmaA(const OrcScene &s, float scalar) {
  return principledDensityFactor(s, scalar) * pv3(s.pAbsorptionColor);
}
static inline float principledSigmaT(const OrcScene &s, float scalar) {
  return reduce_max(principledSigmaS(s, scalar) + principledSigmaA(s, scalar));
}
static inline vec4f principledSampleMap(const OrcScene &s, float scalar) {
  vec3f sigma_s = principledSigmaS(s, scalar);
  vec3f sigma_a = principledSigmaA(s, scalar);
  vec3f sigma_t = sigma_s + sigma_a;
  float sigma_t_scalar = reduce_max(sigma_t);
  vec3f tint = V(1.f);
  if (sigma_t_scalar > 0.f) {
    float ms = reduce_max(sigma_s);
    tint = ms > 0.f ? V(sigma_s.x / ms, sigma_s.y / ms, sigma_s.z / ms) : V(1.f);
  }
  return {tint.x, tint.y, tint.z, sigma_t_scalar};
}
static inline vec3f principledBlackbodyColor(float kelvin) {
  kelvin = clampf(kelvin, 1000.f, 40000.f);
  float t = kelvin / 100.f;
  float r, g, b;
  if (t <= 66.f) {
    r = 1.f;
    g = clampf(0.390081578f * logPortable(t) - 0.631841444f, 0.f, 1.f);
  } else {
    r = clampf(1.292936186f * powPortable(t - 60.f, -0.1332047592f), 0.f, 1.f);
    g = clampf(1.129890860f * powPortable(t - 60.f, -0.0755148492f), 0.f, 1.f);
  }
  if (t >= 66.f) b = 1.f;
  else if (t <= 19.f) b = 0.f;
  else b = clampf(0.543206789f * logPortable(t - 10.f) - 1.196254089f, 0.f, 1.f);
  return V(r, g, b);
}
static inline vec3f principledEmission(const OrcScene &s, float scalar) {
  float d = principledDensityFactor(s, scalar);
  vec3f Le = s.pEmissionStrength * pv3(s.pEmissionColor) * d;
  if (s.pBlackbodyIntensity > 0.f && s.pTemperature > 0.f)
    Le = Le + s.pBlackbodyIntensity * pv3(s.pBlackbodyTint) * principledBlackbodyColor(s.pTemperature) * d;
  return Le;
}
static inline float principledMajorant(const OrcScene &s, float lo, float hi) {
  if (lo > hi) return 0.f;
  float m = 0.f;
  const int steps = 8;
  for (int i = 0; i <= steps; ++i) {
    float t = float(i) / float(steps);
    float x = lo + t * (hi - lo);
    m = fmax_(m, principledSigmaT(s, x));
  }
  return m;
}
// MCGrid.cu:97-113 mapMCs, with the principled scale
static inline float mapMajorant(const OrcScene &s, float lo, float hi) {
  const float tfMaj = tfMajorant(s, lo, hi);
  return s.principled ? principledMajorant(s, lo, hi) * tfMaj : tfMaj;
}

// Volume.h:60-74
static inline vec4f sampleAndMap(const Scene &sc, vec3f P, float &scalar) {
  float f = sampleField(sc, P);
  scalar = f;
  if (std::isnan(f)) return {0.f, 0.f, 0.f, 0.f};
  if (sc.s.principled) {
    vec4f tf = tfMap(sc.s, f);
    if (tf.w <= 0.f) return {0.f, 0.f, 0.f, 0.f};
    vec4f p = principledSampleMap(sc.s, f);
    return {p.x * tf.x, p.y * tf.y, p.z * tf.z, p.w * tf.w};
  }
  return tfMap(sc.s, f);
}

// StructuredData.cu:31-62, cellsPerMC = 8, NEAREST fetch at integer coords
static void buildRangesSpan(const OrcScene &s, vec3i mcDims, float *out, int64_t begin, int64_t end) {
  for (int64_t tid = begin; tid < end; tid++) {
    vec3i mc = {(int)(tid % mcDims.x), (int)((tid / mcDims.x) % mcDims.y), (int)(tid / ((int64_t)mcDims.x * mcDims.y))};
    float lo = INF, hi = -INF;  // owl interval<float> default = empty
    for (int iiz = 0; iiz <= 8; iiz++)
      for (int iiy = 0; iiy <= 8; iiy++)
        for (int iix = 0; iix <= 8; iix++) {
          int x = mc.x * 8 + iix, y = mc.y * 8 + iiy, z = mc.z * 8 + iiz;
          if (x >= s.dims[0] || y >= s.dims[1] || z >= s.dims[2]) continue;
          float f = texel(s, (int64_t)x + (int64_t)s.dims[0] * ((int64_t)y + (int64_t)s.dims[1] * z));
          lo = fmin_(lo, f);
          hi = fmax_(hi, f);
        }
    out[2 * tid + 0] = lo;
    out[2 * tid + 1] = hi;
  }
}
// every macrocell is independent: large grids are split over the host's threads
static void buildRanges(const OrcScene &s, vec3i mcDims, float *out) {
  const int64_t n = (int64_t)mcDims.x * mcDims.y * mcDims.z;
  const int64_t nt = n < 4096 ? 1 : std::max(1u, std::thread::hardware_concurrency());
  if (nt == 1) return buildRangesSpan(s, mcDims, out, 0, n);
  std::vector<std::thread> pool;
  for (int64_t t = 0; t < nt; t++)
    pool.emplace_back(buildRangesSpan, std::cref(s), mcDims, out, n * t / nt, n * (t + 1) / nt);
  for (auto &th : pool) th.join();
}

static void setupScene(Scene &sc) {
  const OrcScene &s = sc.s;
  sc.numScalars = {s.dims[0], s.dims[1], s.dims[2]};
  sc.numCells = {s.dims[0] - 1, s.dims[1] - 1, s.dims[2] - 1};       // StructuredData.cu:146-150
  sc.gridOrigin = V(s.origin[0], s.origin[1], s.origin[2]);
  sc.gridSpacing = V(s.spacing[0], s.spacing[1], s.spacing[2]);
  sc.boundsLo = sc.gridOrigin;                                        // :177-181
  sc.boundsHi = sc.gridOrigin + sc.gridSpacing * V((float)sc.numCells.x, (float)sc.numCells.y, (float)sc.numCells.z);
  sc.mcDims = {(sc.numCells.x + 7) / 8, (sc.numCells.y + 7) / 8, (sc.numCells.z + 7) / 8};  // :74
  sc.mcOrigin = sc.boundsLo;                                          // :76
  sc.mcSpacing = V(8.f) * sc.gridSpacing;                             // :77
  int64_t n = (int64_t)sc.mcDims.x * sc.mcDims.y * sc.mcDims.z;
  std::vector<float> &ranges = sc.ranges;
  ranges.resize(2 * n);
  buildRanges(s, sc.mcDims, ranges.data());
  // MCAccelerator.h:445-447: length(bounds.size()) * .1 / (sum of macrocell dims)
  const vec3f bsize = sc.boundsHi - sc.boundsLo;
  sc.isoDelta = sqrtf(dot(bsize, bsize)) * .1f / float(sc.mcDims.x + sc.mcDims.y + sc.mcDims.z);
  sc.majorants.resize(n);
  for (int64_t i = 0; i < n; i++) {                                   // MCGrid.cu:97-113
    float m = mapMajorant(s, ranges[2 * i], ranges[2 * i + 1]);
    if (s.majorantRoundUp && m > 0.f) m = nextafterf(m, INF);
    sc.majorants[i] = m;
  }
  // Camera.cu:63-101: "direction" is normalized on set, again on commit
  vec3f direction = normalize(V(s.camDir[0], s.camDir[1], s.camDir[2]));
  vec3f up = V(s.camUp[0], s.camUp[1], s.camUp[2]);
  vec3f dir00 = normalize(direction);
  vec3f dirdu = normalize(cross(dir00, up));
  vec3f dirdv = normalize(cross(dirdu, dir00));
  dir00 = dir00 * (float)(1.f / (2.0f * tanf((0.5f * s.fovy) * (float)M_PI / 180.0f)));
  sc.dir00 = dir00; sc.dirdu = dirdu; sc.dirdv = dirdv;
  sc.lens00 = V(s.camPos[0], s.camPos[1], s.camPos[2]);
}

// Ray.h:170-181
static inline bool boxTest(vec3f org, vec3f dir, float &t0, float &t1, vec3f lo, vec3f hi) {
  vec3f t_lo = (lo - org) * rcp(dir);
  vec3f t_hi = (hi - org) * rcp(dir);
  vec3f t_nr = vmin(t_lo, t_hi);
  vec3f t_fr = vmax(t_lo, t_hi);
  t0 = fmax_(t0, reduce_max(t_nr));
  t1 = fmin_(t1, reduce_min(t_fr));
  return t0 <= t1;
}

// DDA.h:61-201
template <typename Lambda>
static void dda3(vec3f org, vec3f dir, float tMax, vec3i gridSize, const Lambda &lambda) {
  const vec3f rcp_dir = rcp(dir);
  const vec3f f_size = V((float)gridSize.x, (float)gridSize.y, (float)gridSize.z);
  vec3f t_lo = (V(0.f) - org) * rcp(dir);
  vec3f t_hi = (f_size - org) * rcp(dir);
  vec3f t_nr = vmin(t_lo, t_hi);
  vec3f t_fr = vmax(t_lo, t_hi);
  if (dir.x == 0.f) { if (org.x < 0.f || org.x > f_size.x) return; t_nr.x = -INF; t_fr.x = +INF; }
  if (dir.y == 0.f) { if (org.y < 0.f || org.y > f_size.y) return; t_nr.y = -INF; t_fr.y = +INF; }
  if (dir.z == 0.f) { if (org.z < 0.f || org.z > f_size.z) return; t_nr.z = -INF; t_fr.z = +INF; }
  float ray_t0 = fmax_(0.f, reduce_max(t_nr));
  float ray_t1 = fmin_(tMax, reduce_min(t_fr));
  if (ray_t0 > ray_t1) return;
  vec3f org_in_volume = org + ray_t0 * dir;
  vec3f f_cell = vmax(V(0.f), vmin(f_size - V(1.f), vfloor(org_in_volume)));
  vec3f f_cell_end = {dir.x > 0.f ? f_cell.x + 1.f : f_cell.x,
                      dir.y > 0.f ? f_cell.y + 1.f : f_cell.y,
                      dir.z > 0.f ? f_cell.z + 1.f : f_cell.z};
  vec3f t_step = vabs(rcp_dir);
  vec3f t_next = {(dir.x == 0.f) ? INF : (fabsf(f_cell_end.x - org_in_volume.x) * t_step.x),
                  (dir.y == 0.f) ? INF : (fabsf(f_cell_end.y - org_in_volume.y) * t_step.y),
                  (dir.z == 0.f) ? INF : (fabsf(f_cell_end.z - org_in_volume.z) * t_step.z)};
  const vec3i stop = {dir.x > 0.f ? gridSize.x : -1, dir.y > 0.f ? gridSize.y : -1, dir.z > 0.f ? gridSize.z : -1};
  const vec3i cell_delta = {dir.x > 0.f ? +1 : -1, dir.y > 0.f ? +1 : -1, dir.z > 0.f ? +1 : -1};
  vec3i cell = {(int)f_cell.x, (int)f_cell.y, (int)f_cell.z};
  float next_cell_begin = 0.f;
  while (1) {
    float t_closest = reduce_min(t_next);
    const float cell_t0 = ray_t0 + next_cell_begin;
    const float cell_t1 = ray_t0 + fmin_(t_closest, tMax);
    if (!lambda(cell, cell_t0, cell_t1)) return;
    next_cell_begin = t_closest;
    if (t_next.x == t_closest) { t_next.x += t_step.x; cell.x += cell_delta.x; if (cell.x == stop.x) return; }
    if (t_next.y == t_closest) { t_next.y += t_step.y; cell.y += cell_delta.y; if (cell.y == stop.y) return; }
    if (t_next.z == t_closest) { t_next.z += t_step.z; cell.z += cell_delta.z; if (cell.z == stop.z) return; }
  }
}

struct Ray {
  vec3f org, dir;
  float tMax;
  RNGSeed rngSeed;
  bool hadHit = false;
  bool surf = false;   // the hit is on the isosurface (else a volume collision)
  vec3f N;             // isosurface hit: normal as stored in the ray (vec3h, Ray.h:61-62)
  vec3f P;
  vec3f hitColor;  // mapped rgb at the collision (phase tint)
  float hitScalar; // field value at the collision (principled volumes)
};

struct LocalStats { uint64_t samples = 0, mcVisits = 0, rays = 0; };

// Woodcock::sampleRange, Volume.h:168-203
static bool woodcock(vec4f &sample, float &scalar, const Scene &sc, vec3f org, vec3f dir, float t_lower,
                     float &t_upper, float majorant, Random2 &rand, LocalStats &st) {
  float t = t_lower;
  while (true) {
    float r = rand();
    float dt = sc.s.exactLog ? (-logPortable(1.f - r) / majorant) : (-fastLog(1.f - r) / majorant);
    t += dt;
    if (t >= t_upper) return false;
    vec3f P = org + t * dir;
    sample = sampleAndMap(sc, P, scalar);
    st.samples++;
    if (sample.w >= rand() * majorant) { t_upper = t; return true; }
  }
}

// ---------------------------------------------------------------------------
// isoSurface geometry on the field: MCIsoSurfaceAccel::isProg
// (MCAccelerator.h:325-548) with an AnariMatte material (AnariMatte.h:49-71)
// ---------------------------------------------------------------------------
// The constant material parameters (HostMaterial.h:98-115: a NaN value reads
// as (0,0,0,1)); Lambertian albedo = .85 * color * (1/pi), alpha = color.w * opacity.x
static const float ONE_OVER_PI = 1.f / ONE_PI;
static inline vec4f isoColor(const OrcScene &s) {
  if (std::isnan(s.isoColor[0])) return {0.f, 0.f, 0.f, 1.f};
  return {s.isoColor[0], s.isoColor[1], s.isoColor[2], s.isoColor[3]};
}
static inline float isoOpacity(const OrcScene &s) { return std::isnan(s.isoOpacity) ? 0.f : s.isoOpacity; }
static inline vec3f isoAlbedo(const OrcScene &s) {
  const vec4f c = isoColor(s);
  const float reflectance = .85f;
  return V(reflectance * c.x * ONE_OVER_PI, reflectance * c.y * ONE_OVER_PI, reflectance * c.z * ONE_OVER_PI);
}
static inline float isoAlpha(const OrcScene &s) { return isoColor(s).w * isoOpacity(s); }

// The isosurface's intersection program for one ray: box test, its own RNG
// (derived from the ray's seed, which this advances), a DDA over the
// macrocell ranges and, in every macrocell whose range holds the iso value,
// ten linear steps between the cell's entry and exit, intersecting the
// segment whose end values bracket the iso value.  The program reports no
// intersection to the traversal: it only lowers the ray's own tMax.
// tMax: the traversal's ray tMax.  Returns true with tHit < ray.tMax on a hit.
static bool isoIntersect(const Scene &sc, Ray &ray, vec3f obj_org, vec3f obj_dir, float tMax, float &tHit) {
  float t0 = 0.f, t1 = tMax;
  if (!boxTest(obj_org, obj_dir, t0, t1, sc.boundsLo, sc.boundsHi)) return false;
  const vec3f dda_org = (obj_org - sc.mcOrigin) * rcp(sc.mcSpacing);
  const vec3f dda_dir = obj_dir * rcp(sc.mcSpacing);
  // Random rng(ray.rngSeed, hash(instance 0, geometry 0, primitive 0))
  Random2 rng(ray.rngSeed, hash3(0, 0, 0));
  const float iso = sc.s.isoValue;
  const float prdTMax = ray.tMax;
  tHit = prdTMax;
  dda3(dda_org, dda_dir, t1, sc.mcDims, [&](const vec3i &c, float ct0, float ct1) -> bool {
    const float lower = ct0, upper = fmin_(ct1, prdTMax);
    if (lower >= upper) return true;
    const int64_t idx = (int64_t)c.x + (int64_t)sc.mcDims.x * ((int64_t)c.y + (int64_t)sc.mcDims.y * c.z);
    const float rlo = sc.ranges[2 * idx], rhi = sc.ranges[2 * idx + 1];
    if (!(iso >= rlo && iso <= rhi)) return true;
    float tt1 = ct0;
    float ff1 = sampleField(sc, obj_org + tt1 * obj_dir);
    const int numSteps = 10;
    for (int i = 1; i <= numSteps; i++) {
      const float tt0 = tt1;
      const float ff0 = ff1;
      tt1 = lerp_l(i / float(numSteps), ct0, ct1);
      ff1 = sampleField(sc, obj_org + tt1 * obj_dir);
      if (std::isnan(ff0) || std::isnan(ff1)) continue;
      const float vlo = fmin_(ff0, ff1), vhi = fmax_(ff0, ff1);
      if (iso >= vlo && iso <= vhi) {
        float t = (iso - ff0) / (ff1 - ff0);
        t = lerp_l(t, tt0, tt1);
        tHit = (t < tHit) ? t : tHit;  // min(tHit, t); a 0/0 segment (NaN) keeps tHit
        if (tHit < prdTMax) return false;
      }
    }
    return true;
  });
  if (!(tHit < prdTMax)) return false;
  const float opacity = isoAlpha(sc.s);  // Lambertian::getOpacity
  if (opacity < 1.f && rng() > opacity) return false;
  return true;
}

// The hit normal (MCAccelerator.h:444-478): central differences of the field
// over +-delta, one-sided where a neighbour is outside; a zero gradient
// falls back to -normalize(dir).  Returned as Ray::packNormal stores it
// (normalized, rounded to binary16).
static vec3f isoNormal(const Scene &sc, vec3f osP, vec3f obj_dir) {
  const float delta = sc.isoDelta;
  const float fP = sampleField(sc, osP);
  float fPx0 = sampleField(sc, osP + V(-delta, 0.f, 0.f));
  float fPx1 = sampleField(sc, osP + V(+delta, 0.f, 0.f));
  float fPy0 = sampleField(sc, osP + V(0.f, -delta, 0.f));
  float fPy1 = sampleField(sc, osP + V(0.f, +delta, 0.f));
  float fPz0 = sampleField(sc, osP + V(0.f, 0.f, -delta));
  float fPz1 = sampleField(sc, osP + V(0.f, 0.f, +delta));
  float dx = 2.f, dy = 2.f, dz = 2.f;
  if (std::isnan(fPx0)) { dx -= 1.f; fPx0 = fP; }
  if (std::isnan(fPx1)) { dx -= 1.f; fPx1 = fP; }
  if (std::isnan(fPy0)) { dy -= 1.f; fPy0 = fP; }
  if (std::isnan(fPy1)) { dy -= 1.f; fPy1 = fP; }
  if (std::isnan(fPz0)) { dz -= 1.f; fPz0 = fP; }
  if (std::isnan(fPz1)) { dz -= 1.f; fPz1 = fP; }
  vec3f osN = V(dx == 0.f ? 0.f : (fPx1 - fPx0) / dx, dy == 0.f ? 0.f : (fPy1 - fPy0) / dy,
                dz == 0.f ? 0.f : (fPz1 - fPz0) / dz);
  if (isZero(osN)) osN = -normalize(obj_dir);
  return halfRound(normalize(osN));
}

// TraceRays::run (traceRays.dev.cu:26-52) over the group's isosurface, then
// its volume (MCVolumeAccel::isProg, MCAccelerator.h:552-689), for one
// identity instance.  The traversal calls the isosurface first: its hit
// lowers only the ray's own tMax, so the volume's box test and DDA still run
// to the traversal's tMax while its Woodcock ranges stop at the surface.  A
// shadow ray that hits the surface is occluded and skips the volume, and the
// volume's DDA stops at the first occupied macrocell that starts at or
// beyond a surface hit; neither can change the outcome.
static void traceRay(const Scene &sc, Ray &ray, LocalStats &st, bool shadowRay = false) {
  st.rays++;
  vec3f dir = ray.dir;
  if (dir.x == 0.f) dir.x = 1e-6f;
  if (dir.y == 0.f) dir.y = 1e-6f;
  if (dir.z == 0.f) dir.z = 1e-6f;
  const vec3f obj_org = ray.org, obj_dir = dir;
  const float tMax = ray.tMax;  // the traversal's tMax
  bool isoHit = false;
  if (sc.s.iso) {
    float tHit;
    if (isoIntersect(sc, ray, obj_org, obj_dir, tMax, tHit)) {
      isoHit = true;
      ray.hadHit = true;  // AnariMatte setHit -> Ray::setHit (Ray.h:88-99)
      ray.surf = true;
      ray.tMax = tHit;
      ray.P = obj_org + tHit * obj_dir;
      ray.N = isoNormal(sc, ray.P, obj_dir);
      if (shadowRay) return;
    }
  }
  if (sc.s.noVolume) return;
  float t0 = 0.f, t1 = tMax;
  if (!boxTest(obj_org, obj_dir, t0, t1, sc.boundsLo, sc.boundsHi)) return;
  vec3f dda_org = (obj_org - sc.mcOrigin) * rcp(sc.mcSpacing);
  vec3f dda_dir = obj_dir * rcp(sc.mcSpacing);
  Random2 rng(ray.rngSeed, hash3(0, 0, 0));
  dda3(dda_org, dda_dir, t1, sc.mcDims, [&](const vec3i &c, float ct0, float ct1) -> bool {
    const float majorant = sc.majorants[(int64_t)c.x + (int64_t)sc.mcDims.x * ((int64_t)c.y + (int64_t)sc.mcDims.y * c.z)];
    st.mcVisits++;
    if (majorant == 0.f) return true;
    if (isoHit && ct0 >= ray.tMax) return false;
    vec4f sample = {0, 0, 0, 0};
    float scalar = 0.f;
    float upper = fmin_(ct1, ray.tMax);
    if (!woodcock(sample, scalar, sc, obj_org, obj_dir, ct0, upper, majorant, rng, st)) return true;
    vec3f P = obj_org + upper * obj_dir;
    ray.hadHit = true;           // Ray::setVolumeHit -> setHit (Ray.h:101-144)
    ray.surf = false;
    ray.P = P;
    ray.tMax = upper;
    ray.hitColor = V(sample.x, sample.y, sample.z);
    ray.hitScalar = scalar;
    return false;
  });
}

// shadeRays.cu:17-41: MAX_PATH_DEPTH; PathState::throughput is vec3h
// (Ray.h:17-23), so every stored throughput is rounded to binary16.
static const int MAX_PATH_DEPTH = 10;

struct PixelSample {
  // generation-0 contribution
  vec3f frag0; float alpha0;
  // later generations' contributions in accumulation order: per generation
  // the shadow ray's, then the scattered ray's
  int n = 0;
  vec3f frags[2 * (MAX_PATH_DEPTH + 2)];
  void add(vec3f f) { frags[n++] = f; }
};

struct LightSample { vec3f direction, radiance; float distance; float pdf = 0.f; };

// DG.h:183-193
static vec3f randomDirection(Random2 &rng) {
  vec3f v;
  while (true) {
    v.x = 1.f - 2.f * rng();
    v.y = 1.f - 2.f * rng();
    v.z = 1.f - 2.f * rng();
    if (dot(v, v) <= 1.f) return normalize(v);
  }
}

// Phase.h:51-58
static inline float hgPhase(float g, float cosTheta) {
  if (fabsf(g) < 1e-3f) return ONE_OVER_FOUR_PI;
  float g2 = g * g;
  float denom = 1.f + g2 - 2.f * g * cosTheta;
  return ONE_OVER_FOUR_PI * (1.f - g2) / (denom * sqrtf(denom));
}

// sin and cos of x in [0, 2pi] (the phase-function samplers' azimuth).  The
// reference calls cosf/sinf, whose last bits differ between CUDA and host
// libm; this restatement and the CUDA kernels share one binary32
// evaluation instead: Cody-Waite reduction by pi/2 = P1 + P2 + P3 (P1 has 8
// significant bits, so j*P1 is exact) to |r| <= pi/4, then the Taylor series
// of sin to r^11 and of cos to r^12 (truncation error below 1e-10) in
// Horner form.
static inline void sincosPortable(float x, float &sn, float &cs) {
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

// HGPhase::sampleDirection, Phase.h:76-101 (cosf/sinf via sincosPortable)
static vec3f hgSampleDirection(vec3f wi_in, float g, Random2 &random) {
  float u0 = random();
  float u1 = random();
  float cosTheta;
  if (fabsf(g) < 1e-3f) cosTheta = 1.f - 2.f * u0;
  else {
    float sqrTerm = (1.f - g * g) / (1.f + g - 2.f * g * u0);
    cosTheta = (1.f + g * g - sqrTerm * sqrTerm) / (2.f * g);
  }
  float sinTheta = sqrtf(fmax_(0.f, 1.f - cosTheta * cosTheta));
  float phi = TWO_PI * u1;
  float sinPhi, cosPhi;
  sincosPortable(phi, sinPhi, cosPhi);
  vec3f local = V(cosPhi * sinTheta, sinPhi * sinTheta, cosTheta);
  vec3f w = normalize(wi_in);
  vec3f u, v;
  if (fabsf(w.x) > 0.1f) u = normalize(cross(V(0.f, 1.f, 0.f), w));
  else u = normalize(cross(V(1.f, 0.f, 0.f), w));
  v = cross(w, u);
  return normalize(local.x * u + local.y * v + local.z * w);
}

// shadeRays.cu:294-402 for the lights this path has: the constant
// environment (renderer.ambientRadiance, no env-map texture) and
// directional lights.  N is the zero vector for volume hits and the
// front-facing normal for surface hits.
static const float ONE_OVER_TWO_PI = 1.f / TWO_PI;
static bool sampleLights(const Scene &sc, LightSample &ls, Random2 &random, bool &lightNeedsMIS,
                         bool &lightIsDirLight, vec3f N = V(0.f)) {
  const OrcScene &s = sc.s;
  lightNeedsMIS = false;
  // sampleEnvLight :266-291
  LightSample els;
  els.direction = randomDirection(random);
  els.distance = INF;
  if (!isZero(N)) {
    els.radiance = V(TWO_PI * s.ambientRadiance);
    if (dot(els.direction, N) < 0.f) els.direction = -els.direction;
    els.pdf = ONE_OVER_TWO_PI;
  } else {
    els.radiance = V(FOUR_PI * s.ambientRadiance);
    els.pdf = ONE_OVER_FOUR_PI;
  }
  float elsWeight = reduce_max(els.radiance);
  // sampleAreaLights: none on this path -> false, no random numbers
  float alsWeight = 0.f;
  // sampleDirLights :139-189
  LightSample dls;
  float dlsWeight = 0.f;
  if (s.numDirLights > 0) {
    const int RES = 2;
    int lID[RES];
    float weights[RES];
    float sumW = 0.f;
    bool ok = true;
    for (int i = 0; i < RES; i++) {
      lID[i] = std::min(int(random() * s.numDirLights), s.numDirLights - 1);
      weights[i] = 0.f;
      const float *L = s.dirLights + 7 * lID[i];
      vec3f rad = V(L[4], L[5], L[6]) * L[3];
      const vec3f lightDir = -normalize(V(L[0], L[1], L[2]));
      float weight = isZero(N) ? 1.f : dot(lightDir, N);
      if (weight <= 1e-3f) continue;
      weight *= reduce_max(rad);
      if (weight <= 1e-3f) continue;
      weights[i] = weight;
      sumW += weight;
    }
    if (sumW == 0.f) ok = false;
    if (ok) {
      float r = random() * sumW;
      int i = 0;
      while (i < RES && r >= weights[i]) { r -= weights[i]; ++i; }
      if (i == RES) ok = false;
      else {
        const float *L = s.dirLights + 7 * lID[i];
        // DirLight.cu:11-20: direction normalized (identity instance)
        vec3f ldir = normalize(V(L[0], L[1], L[2]));
        dls.direction = -ldir;
        dls.distance = INF;
        dls.radiance = V(L[4], L[5], L[6]) * L[3] * 1.f / (weights[i] / sumW * (float(RES) / float(s.numDirLights)));
        dls.pdf = INF;
        ok = weights[i] != 0.f;
      }
    }
    dlsWeight = ok ? reduce_max(dls.radiance) : 0.f;
  }
  float plsWeight = 0.f;
  float sumWeights = alsWeight + dlsWeight + elsWeight + plsWeight;
  if (sumWeights == 0.f) return false;
  elsWeight *= 1.f / sumWeights;
  alsWeight *= 1.f / sumWeights;
  dlsWeight *= 1.f / sumWeights;
  plsWeight *= 1.f / sumWeights;
  float r = random();
  if (r <= alsWeight) {
    ls = LightSample();  // area-light sample of an empty light list: pdf 0
  } else if (r <= alsWeight + elsWeight) {
    ls = els;
    ls.radiance = ls.radiance * (1.f / elsWeight);
    lightNeedsMIS = true;
  } else if (r <= alsWeight + elsWeight + plsWeight) {
    ls = LightSample();
  } else {
    if (dlsWeight == 0.f) return false;  // no directional sample exists
    ls = dls;
    ls.radiance = ls.radiance * (1.f / dlsWeight);
    lightIsDirLight = true;
  }
  if (std::isnan(ls.pdf) || (ls.pdf <= 0.f)) return false;
  return true;
}

// ---------------------------------------------------------------------------
// surface hits: bounce() with a Lambertian BSDF (shadeRays.cu:540-878,
// packedBSDF/Lambertian.h:45-86, DG.h:162-193)
// ---------------------------------------------------------------------------
// owl::common::frame(N) (the owl submodule, absent here): the orthonormal
// basis of embree's LinearSpace3 frame() -- dx from the larger of
// (0, N.z, -N.y) and (-N.z, 0, N.x), dy = normalize(cross(N, dx)), dz = N --
// and xfmVector(frame, v) = dx * v.x + dy * v.y + dz * v.z.
static vec3f frameXfm(vec3f N, vec3f v) {
  const vec3f dx0 = V(0.f, N.z, -N.y);
  const vec3f dx1 = V(-N.z, 0.f, N.x);
  const vec3f dx = normalize(dot(dx0, dx0) > dot(dx1, dx1) ? dx0 : dx1);
  const vec3f dy = normalize(cross(N, dx));
  return dx * v.x + dy * v.y + N * v.z;
}
// Lambertian::pdf: the cosine pdf about the normal turned toward wi
static inline float lambertPdf(vec3f Ng, vec3f wi) {
  vec3f N = Ng;
  if (dot(wi, N) < 0.f) N = -N;
  const float cosThetaI = fmax_(dot(wi, N), 0.f);
  return cosThetaI * ONE_OVER_PI;
}

// bounce() for a hit on the isosurface: shadow ray toward a light sample
// with the Lambertian's f_r and the surface's cosine, then (path depth and
// the one diffuse bounce allowed, MAX_DIFFUSE_BOUNCES) a cosine-sampled
// scattered ray.  cosineSampleHemisphere draws its two numbers in argument
// order (u for the azimuth first); its sincosf is sincosPortable.
static void surfaceBounce(const Scene &sc, Ray &ray, int depth, Random2 &random, vec3f P, vec3f wo,
                          float offsetEpsilon, vec3f &tp, float &pathMis, int &numDiffuseBounces, Ray &shadow,
                          vec3f &shadowTp, float &shadowMis, bool &haveShadow, bool &haveScatter) {
  const vec3f albedo = isoAlbedo(sc.s);
  const vec3f Ng = normalize(ray.N);
  const bool hitWasOnFront = dot(ray.dir, Ng) < 0.f;
  const vec3f Ngff = hitWasOnFront ? Ng : -Ng;
  LightSample ls;
  bool lightNeedsMIS = false, lightIsDirLight = false;
  if (sampleLights(sc, ls, random, lightNeedsMIS, lightIsDirLight, Ngff)) {
    // Lambertian::eval: cosine against the shading normal (dg.Ns = Ng, not turned)
    const float cosThetaI = fmax_(dot(ls.direction, Ng), 0.f);
    const float fpdf = cosThetaI * ONE_OVER_PI;
    vec3f fval = albedo * ONE_OVER_PI * cosThetaI;
    if ((fpdf > 0.f) && !(reduce_max(fval) < 1e-4f)) {
      fval = vmin(fval, V(13.f));
      const float cosL = ONE_OVER_PI * fabsf(dot(Ng, ls.direction));
      vec3f tp_sr = tp * (std::isinf(ls.pdf) ? 1.f : (1.f / ls.pdf)) * fval * ls.radiance * cosL;
      shadow.org = P + offsetEpsilon * Ngff;
      shadow.dir = ls.direction;
      shadow.tMax = ls.distance * (1.f - 2.f * offsetEpsilon);
      shadowTp = halfRound(tp_sr);
      shadow.rngSeed = ray.rngSeed;
      ray.rngSeed.nextHashed((uint64_t)floatBits(ray.tMax));
      haveShadow = true;
      if (!lightIsDirLight && lightNeedsMIS) {
        const float pdf_light = ONE_OVER_FOUR_PI;
        const float pdf_scatter = lambertPdf(Ng, ls.direction);
        shadowMis = pdf_light / (pdf_light + pdf_scatter + 1e-10f);
        if (shadowMis < 1e-5f) haveShadow = false;
      }
      if (!(shadow.tMax > 0.f)) haveShadow = false;
    }
  }
  if (depth >= MAX_PATH_DEPTH) return;
  // Lambertian::scatter
  vec3f N = Ng;
  if (dot(wo, N) < 0.f) N = -N;
  const float su = random();
  const float sv = random();
  const float phi = TWO_PI * su;
  const float cosTheta = sqrtf(sv);
  const float sinTheta = sqrtf(1.0f - sv);
  float sinPhi, cosPhi;
  sincosPortable(phi, sinPhi, cosPhi);
  const vec3f localDir = V(cosPhi * sinTheta, sinPhi * sinTheta, cosTheta);
  const vec3f sdir = frameXfm(N, localDir);
  const float pdf = localDir.z * ONE_OVER_PI;
  if (!(pdf > 0.f) || pdf <= 1e-6f) {
    // no valid sample: the ray, cleared, goes out again unchanged (:757-768)
    ray.tMax = INF;
    ray.hadHit = false;
    ray.surf = false;
    haveScatter = true;
    return;
  }
  if (numDiffuseBounces >= 1) return;  // MAX_DIFFUSE_BOUNCES
  numDiffuseBounces++;
  ray.org = P + (1.f * offsetEpsilon) * Ngff;
  ray.dir = normalize(sdir);
  const float c = fabsf(dot(Ng, normalize(ray.dir)));
  const float denom = std::isinf(pdf) ? 1.f : (pdf + 1e-10f);
  vec3f scatterFactor = V((albedo.x * c) / denom, (albedo.y * c) / denom, (albedo.z * c) / denom);
  scatterFactor = vmin(scatterFactor, V(2.5f));
  tp = halfRound(tp * scatterFactor);
  if (lightNeedsMIS && !std::isinf(pdf)) {
    const float ps = lambertPdf(Ng, ray.dir);
    const float pl = ONE_OVER_FOUR_PI;
    pathMis = ps / (ps + pl);
  } else {
    pathMis = 1.f;
  }
  ray.tMax = INF;
  ray.hadHit = false;
  ray.surf = false;
  haveScatter = true;
}

// one wave for one pixel: generateRays.cu:43-244, trace, bounce()
// (shadeRays.cu:475-880) for generation 0, trace of the shadow ray,
// bounce() for generation 1.
static PixelSample renderPixelSample(const Scene &sc, int ix, int iy, int accumID, LocalStats &st) {
  const OrcScene &s = sc.s;
  const int W = s.width, H = s.height;
  PixelSample out{};
  Ray ray;
  // 32-bit wrap-around arithmetic, as the reference's ints do on the GPU
  const unsigned uAcc = (unsigned)accumID;
  Random2 rand((unsigned)ix + (unsigned)W * uAcc, (unsigned)iy + (unsigned)H * uAcc);
  ray.rngSeed.seed((unsigned)ix + uAcc * (unsigned)W, (unsigned)iy);
  float pixel_u = ((accumID == 0) ? .5f : rand());
  float pixel_v = ((accumID == 0) ? .5f : rand());
  float image_u = ((ix + pixel_u) / float(W));
  float image_v = ((iy + pixel_v) / float(H));
  float aspect = W / float(H);
  ray.org = sc.lens00;
  vec3f ray_dir = sc.dir00 + (1.f * aspect * (image_u - .5f)) * sc.dirdu + (1.f * (image_v - .5f)) * sc.dirdv;
  ray.dir = normalize(ray_dir);
  ray.tMax = 1e30f;
  if (s.cutPlane[3] > -1e28f) {
    vec3f N = V(s.cutPlane[0], s.cutPlane[1], s.cutPlane[2]);
    float d_plane = s.cutPlane[3];
    float dist_org = dot(N, ray.org) + d_plane;
    float denom = dot(N, ray.dir);
    if (dist_org >= 0.f) {
      if (denom < 0.f) { float t_cut = -dist_org / denom; ray.tMax = fmin_(ray.tMax, t_cut); }
    } else {
      if (denom > 0.f) { float t_entry = -dist_org / denom; ray.org = ray.org + t_entry * ray.dir; }
      else ray.tMax = 0.f;
    }
  }
  const float t = (iy + .5f) / float(H);
  vec4f bg;
  if (s.bgColor[3] >= 0.f) bg = {s.bgColor[0], s.bgColor[1], s.bgColor[2], s.bgColor[3]};
  else bg = {(1.0f - t) * 0.9f + t * 0.15f, (1.0f - t) * 0.9f + t * 0.25f, (1.0f - t) * 0.9f + t * .8f, (1.0f - t) * 1.f + t * 1.f};

  traceRay(sc, ray, st);

  // ---- generation 0: bounce() on the primary ray
  if (!ray.hadHit) {
    out.frag0 = V(bg.x, bg.y, bg.z);
    out.alpha0 = bg.w;
    return out;
  }
  out.frag0 = V(0.f);
  out.alpha0 = 1.f;
  if (s.emissionAbsorption) {  // extension: collision estimator of emission
    out.frag0 = ray.hitColor;
    return out;
  }
  // path state: throughput (vec3h), MIS weight of the path ray, bounces
  vec3f tp = V(1.f);
  float pathMis = 1.f;
  int numVolumeBounces = 0, numDiffuseBounces = 0;
  for (int depth = 0;; depth++) {
    // ---- bounce() on a hit of generation `depth` (shadeRays.cu:608-878)
    Random2 random(ray.rngSeed, (uint64_t)floatBits(ray.tMax));
    const vec3f P = ray.P;
    const vec3f wo = -normalize(ray.dir);
    const float offsetEpsilon = fmax_(1e-4f, 1e-6f * reduce_max(vabs(P)));  // safe_eps
    Ray shadow;
    vec3f shadowTp = V(0.f);
    float shadowMis = 1.f;
    bool haveShadow = false;
    bool haveScatter = false;
    if (ray.surf) {
      surfaceBounce(sc, ray, depth, random, P, wo, offsetEpsilon, tp, pathMis, numDiffuseBounces, shadow, shadowTp,
                    shadowMis, haveShadow, haveScatter);
    } else {
    // bsdf at the collision (Phase.h): SimplePhase(0.7) or HGPhase.  The
    // multi-scatter build re-derives a principled volume's tint, albedo and
    // emission from the field value at the hit (MCAccelerator.h:621-659).
    vec3f tint = ray.hitColor;
    float hitAlbedo = s.scatteringAlbedo;
    vec3f emission = V(0.f);
    if (s.phaseMode == 1 && s.principled) {
      const float scalar = ray.hitScalar;
      vec3f sigma_s = principledSigmaS(s, scalar);
      vec3f sigma_a = principledSigmaA(s, scalar);
      vec4f tf = tfMap(s, scalar);
      if (tf.w > 0.f) {
        sigma_s = sigma_s * tf.w;
        sigma_a = sigma_a * tf.w;
        tint = tint * V(tf.x, tf.y, tf.z);
      } else {
        sigma_s = V(0.f);
        sigma_a = V(0.f);
      }
      float sigma_t = reduce_max(sigma_s + sigma_a);
      if (sigma_t > 0.f) {
        float ms = reduce_max(sigma_s);
        tint = ms > 0.f ? V(sigma_s.x / ms, sigma_s.y / ms, sigma_s.z / ms) : tint;
        hitAlbedo = reduce_max(sigma_s) / sigma_t;
      }
      emission = principledEmission(s, scalar);
    }
    vec3f albedo;
    if (s.phaseMode == 0) albedo = .7f * tint;
    else albedo = hitAlbedo * tint;
    // emission of an HGPhase hit (shadeRays.cu:613-617): this generation's fragment
    if (s.phaseMode == 1 && reduce_max(emission) > 0.f) {
      if (depth == 0) out.frag0 = tp * emission;
      else out.add(tp * emission);
    }
    // shadow ray (:640-746)
    LightSample ls;
    bool lightNeedsMIS = false, lightIsDirLight = false;
    if (sampleLights(sc, ls, random, lightNeedsMIS, lightIsDirLight)) {
      float fpdf;
      if (s.phaseMode == 0) fpdf = ONE_OVER_FOUR_PI;
      else fpdf = hgPhase(s.anisotropy, dot(normalize(-wo), normalize(ls.direction)));
      vec3f fval = fpdf * albedo;
      if ((fpdf > 0.f) && !(reduce_max(fval) < 1e-4f)) {
        fval = vmin(fval, V(13.f));
        const vec3f incomingThroughput = tp;
        vec3f tp_sr = incomingThroughput * (std::isinf(ls.pdf) ? 1.f : (1.f / ls.pdf)) * fval * ls.radiance * 1.f;
        shadow.org = P + offsetEpsilon * wo;
        shadow.dir = ls.direction;
        shadow.tMax = ls.distance * (1.f - 2.f * offsetEpsilon);
        shadowTp = halfRound(tp_sr);
        shadow.rngSeed = ray.rngSeed;
        ray.rngSeed.nextHashed((uint64_t)floatBits(ray.tMax));
        haveShadow = true;
        if (!lightIsDirLight && lightNeedsMIS) {
          float pdf_light = ONE_OVER_FOUR_PI;  // EnvMap.h:142-151, no texture
          float pdf_scatter;
          if (s.phaseMode == 0) pdf_scatter = ONE_OVER_FOUR_PI;
          else pdf_scatter = hgPhase(s.anisotropy, dot(normalize(-wo), normalize(ls.direction)));
          shadowMis = pdf_light / (pdf_light + pdf_scatter + 1e-10f);
          if (shadowMis < 1e-5f) haveShadow = false;
        }
        if (!(shadow.tMax > 0.f)) haveShadow = false;
      }
    }
    // scattered ray (:749-878), multi-scatter build: HGPhase::scatter, then
    // the volume-bounce budget.  A sample with pdf <= 1e-6 would end the path
    // here (the reference re-traces the old ray); with anisotropy clamped to
    // [-0.99, 0.99] (Volume.cpp:55-57) the HG pdf stays above 2e-4.
    if (s.phaseMode == 1 && s.maxVolumeBounces > 0 && depth < MAX_PATH_DEPTH) {
      const vec3f wi_in = normalize(-wo);
      const vec3f sdir = hgSampleDirection(wi_in, s.anisotropy, random);
      const float pdf = hgPhase(s.anisotropy, dot(wi_in, sdir));
      const vec3f f_r = albedo * pdf;
      if (pdf > 0.f && !(pdf <= 1e-6f) && numVolumeBounces < s.maxVolumeBounces) {
        numVolumeBounces++;
        ray.org = P + (1.f * offsetEpsilon) * wo;
        ray.dir = normalize(sdir);
        const float denom = std::isinf(pdf) ? 1.f : (pdf + 1e-10f);
        vec3f scatterFactor = V((f_r.x * 1.f) / denom, (f_r.y * 1.f) / denom, (f_r.z * 1.f) / denom);
        scatterFactor = vmin(scatterFactor, V(2.5f));
        tp = halfRound(tp * scatterFactor);
        if (lightNeedsMIS && !std::isinf(pdf)) {
          const float ps = hgPhase(s.anisotropy, dot(normalize(-wo), normalize(ray.dir)));
          const float pl = ONE_OVER_FOUR_PI;
          pathMis = ps / (ps + pl);
        } else {
          pathMis = 1.f;
        }
        ray.tMax = INF;
        ray.hadHit = false;
        haveScatter = true;
      }
    }
    }
    // ---- generation depth+1: the shadow ray, then the scattered ray
    if (haveShadow) {
      traceRay(sc, shadow, st, true);
      out.add(shadow.hadHit ? V(0.f) : (shadowMis * shadowTp));
    }
    if (!haveScatter) return out;
    traceRay(sc, ray, st);
    if (!ray.hadHit) {  // secondary ray into the environment (:529-557)
      out.add(tp * V(s.ambientRadiance) * pathMis);
      return out;
    }
    // a secondary hit: emission of principled volumes only
  }
}

// Neumaier-compensated sum (precision forms): sum += x, error kept in c.
static inline void neumaier(float &sum, float &c, float x) {
  float t = sum + x;
  if (fabsf(sum) >= fabsf(x)) c += (sum - t) + x;
  else c += (x - t) + sum;
  sum = t;
}
static inline void addTo(float &sum, float &c, float x, bool comp) {
  if (comp) neumaier(sum, c, x);
  else sum += x;
}

// _shadeRays accumulation, shadeRays.cu:996-1040.  With compensation the
// positive adds go through neumaier() and comp holds the running error.
static inline void accumulate(vec4f &acc, vec4f &comp, const PixelSample &ps, int accumID, bool compensated) {
  float clampMax = 10.f * (1 + accumID);
  vec3f f0 = vmin(ps.frag0, V(clampMax));
  if (accumID == 0) {
    acc = {f0.x, f0.y, f0.z, ps.alpha0};
    comp = {0.f, 0.f, 0.f, 0.f};
  } else {
    if (ps.alpha0 > 0.f) addTo(acc.w, comp.w, ps.alpha0, compensated);
    if (f0.x > 0.f) addTo(acc.x, comp.x, f0.x, compensated);
    if (f0.y > 0.f) addTo(acc.y, comp.y, f0.y, compensated);
    if (f0.z > 0.f) addTo(acc.z, comp.z, f0.z, compensated);
  }
  for (int i = 0; i < ps.n; i++) {
    vec3f f1 = vmin(ps.frags[i], V(clampMax));
    if (f1.x > 0.f) addTo(acc.x, comp.x, f1.x, compensated);
    if (f1.y > 0.f) addTo(acc.y, comp.y, f1.y, compensated);
    if (f1.z > 0.f) addTo(acc.z, comp.z, f1.z, compensated);
  }
}

} // namespace orc

extern "C" {

uint32_t orc_version() { return 1; }

// RNG known-answer helpers
void orc_rng_stream(uint32_t a, uint32_t b, int n, uint32_t *out) {
  Random2 r(a, b);
  for (int i = 0; i < n; i++) out[i] = r.next();
}
void orc_rng_floats(uint32_t a, uint32_t b, int n, float *out) {
  Random2 r(a, b);
  for (int i = 0; i < n; i++) out[i] = r();
}
// Random2(seed, h) derived stream; returns the advanced parent state in *parentOut
void orc_rng_derived(uint64_t parentState, uint64_t h, int n, uint32_t *out, uint64_t *parentOut) {
  RNGSeed p;
  p.state = parentState;
  Random2 r(p, h);
  for (int i = 0; i < n; i++) out[i] = r.next();
  *parentOut = p.state;
}
uint64_t orc_hash3(uint32_t a, uint32_t b, uint32_t c) { return hash3(a, b, c); }
float orc_fastlog(float f) { return fastLog(f); }
uint16_t orc_f2h(float f) { return f2h(f); }
void orc_expp(int n, const float *x, float *out) {
  for (int i = 0; i < n; i++) out[i] = expPortable(x[i]);
}
void orc_blackbody(float kelvin, float *rgb) {
  vec3f c = principledBlackbodyColor(kelvin);
  rgb[0] = c.x; rgb[1] = c.y; rgb[2] = c.z;
}
void orc_logp(int n, const float *x, float *out) {
  for (int i = 0; i < n; i++) out[i] = logPortable(x[i]);
}
void orc_sincos(int n, const float *x, float *sn, float *cs) {
  for (int i = 0; i < n; i++) sincosPortable(x[i], sn[i], cs[i]);
}
void orc_hg_sample(const float *wi, float g, uint64_t seedState, int n, float *outDirs) {
  Random2 rng(1u, 1u);
  rng.state = seedState;
  for (int i = 0; i < n; i++) {
    vec3f d = hgSampleDirection(V(wi[0], wi[1], wi[2]), g, rng);
    outDirs[3 * i] = d.x; outDirs[3 * i + 1] = d.y; outDirs[3 * i + 2] = d.z;
  }
}
float orc_h2f(uint16_t h) { return h2f(h); }

// One ray against the scene's isosurface: *hit, the hit distance and the
// stored normal; the ray's RNG state starts at seedState.
void orc_iso_trace(const OrcScene *s, const float *org, const float *dir, float tMax, uint64_t seedState, int *hit,
                   float *tOut, float *nOut) {
  Scene sc(*s);
  setupScene(sc);
  Ray ray;
  ray.org = V(org[0], org[1], org[2]);
  ray.dir = V(dir[0], dir[1], dir[2]);
  ray.tMax = tMax;
  ray.rngSeed.state = seedState;
  float tHit = tMax;
  *hit = isoIntersect(sc, ray, ray.org, ray.dir, tMax, tHit) ? 1 : 0;
  *tOut = tHit;
  const vec3f n = *hit ? isoNormal(sc, ray.org + tHit * ray.dir, ray.dir) : V(0.f);
  nOut[0] = n.x; nOut[1] = n.y; nOut[2] = n.z;
}
// owl::common::frame(N) applied to v
void orc_frame_xfm(const float *N, const float *v, float *out) {
  const vec3f r = frameXfm(V(N[0], N[1], N[2]), V(v[0], v[1], v[2]));
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

void orc_mc_dims(const OrcScene *s, int *out3) {
  out3[0] = (s->dims[0] - 1 + 7) / 8;
  out3[1] = (s->dims[1] - 1 + 7) / 8;
  out3[2] = (s->dims[2] - 1 + 7) / 8;
}
void orc_build_ranges(const OrcScene *s, float *out) {
  vec3i d = {(s->dims[0] - 1 + 7) / 8, (s->dims[1] - 1 + 7) / 8, (s->dims[2] - 1 + 7) / 8};
  buildRanges(*s, d, out);
}
void orc_map_majorants(const OrcScene *s, const float *ranges, int64_t n, float *out) {
  for (int64_t i = 0; i < n; i++) {
    float m = mapMajorant(*s, ranges[2 * i], ranges[2 * i + 1]);
    if (s->majorantRoundUp && m > 0.f) m = nextafterf(m, INF);
    out[i] = m;
  }
}
void orc_sample_points(const OrcScene *s, int n, const float *P, float *outScalar, float *outRGBA) {
  Scene sc(*s);
  sc.numScalars = {s->dims[0], s->dims[1], s->dims[2]};
  sc.numCells = {s->dims[0] - 1, s->dims[1] - 1, s->dims[2] - 1};
  sc.gridOrigin = V(s->origin[0], s->origin[1], s->origin[2]);
  sc.gridSpacing = V(s->spacing[0], s->spacing[1], s->spacing[2]);
  for (int i = 0; i < n; i++) {
    vec3f p = V(P[3 * i], P[3 * i + 1], P[3 * i + 2]);
    outScalar[i] = sampleField(sc, p);
    float scalar;
    vec4f m = sampleAndMap(sc, p, scalar);
    outRGBA[4 * i + 0] = m.x; outRGBA[4 * i + 1] = m.y; outRGBA[4 * i + 2] = m.z; outRGBA[4 * i + 3] = m.w;
  }
}
void orc_tf_map(const OrcScene *s, int n, const float *v, float *outRGBA) {
  for (int i = 0; i < n; i++) {
    vec4f m = tfMap(*s, v[i]);
    outRGBA[4 * i + 0] = m.x; outRGBA[4 * i + 1] = m.y; outRGBA[4 * i + 2] = m.z; outRGBA[4 * i + 3] = m.w;
  }
}
// DDA cell sequence for a grid-space ray; returns number of cells written (<= maxCells)
int orc_dda_cells(const float *org, const float *dir, float tMax, const int *grid, int maxCells, int *outCells,
                  float *outT) {
  int n = 0;
  dda3(V(org[0], org[1], org[2]), V(dir[0], dir[1], dir[2]), tMax, vec3i{grid[0], grid[1], grid[2]},
       [&](const vec3i &c, float t0, float t1) -> bool {
         if (n >= maxCells) return false;
         outCells[3 * n] = c.x; outCells[3 * n + 1] = c.y; outCells[3 * n + 2] = c.z;
         outT[2 * n] = t0; outT[2 * n + 1] = t1;
         n++;
         return true;
       });
  return n;
}

// Primary-ray trace for one pixel: writes hit flag, t, rgb.
void orc_trace_primary(const OrcScene *s, int ix, int iy, int accumID, int *hit, float *t, float *rgb) {
  Scene sc(*s);
  setupScene(sc);
  LocalStats st;
  const int W = s->width, H = s->height;
  Ray ray;
  // 32-bit wrap-around arithmetic, as the reference's ints do on the GPU
  const unsigned uAcc = (unsigned)accumID;
  Random2 rand((unsigned)ix + (unsigned)W * uAcc, (unsigned)iy + (unsigned)H * uAcc);
  ray.rngSeed.seed((unsigned)ix + uAcc * (unsigned)W, (unsigned)iy);
  float pixel_u = ((accumID == 0) ? .5f : rand());
  float pixel_v = ((accumID == 0) ? .5f : rand());
  float image_u = ((ix + pixel_u) / float(W));
  float image_v = ((iy + pixel_v) / float(H));
  float aspect = W / float(H);
  ray.org = sc.lens00;
  ray.dir = normalize(sc.dir00 + (1.f * aspect * (image_u - .5f)) * sc.dirdu + (1.f * (image_v - .5f)) * sc.dirdv);
  ray.tMax = 1e30f;
  traceRay(sc, ray, st);
  *hit = ray.hadHit;
  *t = ray.tMax;
  rgb[0] = ray.hitColor.x; rgb[1] = ray.hitColor.y; rgb[2] = ray.hitColor.z;
}

// LINEAR tex3D at unnormalized texel coordinates (Texture.cpp:339-411)
void orc_tex3d(const OrcScene *s, int n, const float *tc, float *out) {
  for (int i = 0; i < n; i++) out[i] = tex3DLinear(*s, tc[3 * i], tc[3 * i + 1], tc[3 * i + 2]);
}

// One ray with an explicit RNG seed state through the volume's isProg:
// hit flag, t, rgb at the collision, and the samples / macrocell visits taken.
void orc_trace_ray(const OrcScene *s, const float *org, const float *dir, float tMax, uint64_t seedState, int *hit,
                   float *t, float *rgb, int *counts) {
  Scene sc(*s);
  setupScene(sc);
  LocalStats st;
  Ray ray;
  ray.org = V(org[0], org[1], org[2]);
  ray.dir = V(dir[0], dir[1], dir[2]);
  ray.tMax = tMax;
  ray.rngSeed.state = seedState;
  traceRay(sc, ray, st);
  *hit = ray.hadHit;
  *t = ray.hadHit ? ray.tMax : 0.f;
  rgb[0] = ray.hadHit ? ray.hitColor.x : 0.f;
  rgb[1] = ray.hadHit ? ray.hitColor.y : 0.f;
  rgb[2] = ray.hadHit ? ray.hitColor.z : 0.f;
  counts[0] = (int)st.samples;
  counts[1] = (int)st.mcVisits;
}

// The principled volume's sampleMap (tint rgb, sigma_t) and emission at scalars
void orc_principled(const OrcScene *s, int n, const float *v, float *outMap, float *outEmission) {
  for (int i = 0; i < n; i++) {
    const vec4f m = principledSampleMap(*s, v[i]);
    const vec3f e = principledEmission(*s, v[i]);
    outMap[4 * i] = m.x; outMap[4 * i + 1] = m.y; outMap[4 * i + 2] = m.z; outMap[4 * i + 3] = m.w;
    outEmission[3 * i] = e.x; outEmission[3 * i + 1] = e.y; outEmission[3 * i + 2] = e.z;
  }
}

// Render waves accumID0 .. accumID0+spp-1 over the pixel rectangle
// [x0,x1) x [y0,y1), accumulating into accum (width*height float4, linear).
// Rows are handed out to numThreads workers (Compute.cpp:17-80 scheme).
// Returns wall seconds spent.
double orc_render(const OrcScene *s, int accumID0, int spp, float *accum, float *compBuf, int x0, int y0, int x1,
                  int y1, int numThreads, OrcStats *stats) {
  auto tStart = std::chrono::steady_clock::now();
  Scene sc(*s);
  setupScene(sc);
  if (numThreads <= 0) numThreads = (int)std::thread::hardware_concurrency();
  std::atomic<int> nextRow{y0};
  std::vector<LocalStats> perThread(numThreads);
  auto worker = [&](int tid) {
    LocalStats &st = perThread[tid];
    while (true) {
      int iy = nextRow++;
      if (iy >= y1) break;
      for (int ix = x0; ix < x1; ix++) {
        const int64_t p = (int64_t)iy * s->width + ix;
        vec4f *accp = (vec4f *)(accum + 4 * p);
        vec4f acc = *accp;
        vec4f comp = compBuf ? *(vec4f *)(compBuf + 4 * p) : vec4f{0.f, 0.f, 0.f, 0.f};
        for (int k = 0; k < spp; k++) {
          int accumID = accumID0 + k;
          PixelSample ps = renderPixelSample(sc, ix, iy, accumID, st);
          accumulate(acc, comp, ps, accumID, s->compensatedAccum != 0);
        }
        *accp = acc;
        if (compBuf) *(vec4f *)(compBuf + 4 * p) = comp;
      }
    }
  };
  std::vector<std::thread> threads;
  for (int i = 0; i < numThreads; i++) threads.emplace_back(worker, i);
  for (auto &t : threads) t.join();
  if (stats) {
    OrcStats tot{0, 0, 0, 0};
    for (auto &p : perThread) { tot.samples += p.samples; tot.mcVisits += p.mcVisits; tot.rays += p.rays; }
    tot.pixelSamples = (unsigned long long)(x1 - x0) * (y1 - y0) * spp;
    *stats = tot;
  }
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - tStart).count();
}

// math.h:61-66
static inline float linear_to_srgb(float x) {
  if (x <= 0.0031308f) return 12.92f * x;
  return 1.055f * powf(x, 1.f / 2.4f) - 0.055f;
}
static inline uint32_t make_8bit(float f) { return (uint32_t)std::min(255, std::max(0, int(f * 256.f))); }

// TiledFB.cu:13-52 with accumScale = 1/accumID (LocalFB.cpp:65).
// fmt: 0 float4, 1 rgba8, 2 rgba8 sRGB
// comp (may be NULL): compensation terms of the precision forms, added
// before scaling.
void orc_resolve(const float *accum, const float *comp, int64_t numPixels, int accumID, int fmt, void *out) {
  float accumScale = 1.f / accumID;
  for (int64_t i = 0; i < numPixels; i++) {
    float a[4];
    for (int c = 0; c < 4; c++) a[c] = comp ? accum[4 * i + c] + comp[4 * i + c] : accum[4 * i + c];
    vec4f c = {a[0] * accumScale, a[1] * accumScale, a[2] * accumScale, a[3] * accumScale};
    if (fmt == 0) {
      float *o = (float *)out + 4 * i;
      o[0] = c.x; o[1] = c.y; o[2] = c.z; o[3] = c.w;
    } else {
      if (fmt == 2) { c.x = linear_to_srgb(c.x); c.y = linear_to_srgb(c.y); c.z = linear_to_srgb(c.z); }
      ((uint32_t *)out)[i] = (make_8bit(c.x) << 0) + (make_8bit(c.y) << 8) + (make_8bit(c.z) << 16) + (make_8bit(c.w) << 24);
    }
  }
}

} // extern "C"
