// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Runs the REFERENCE'S OWN hot-path code on the CPU, compiled from its
// sources where they lie (oracle/Makefile, target `ref`, output
// oracle/_ref/libbnref.so), to produce golden vectors that pin both the FP32
// restatement (bn_oracle.cpp) and the CUDA kernels.  Compiled from the
// reference, unmodified:
//
//   barney/native/common/barney-common.h:21-108   RNGSeed, Random2, hash
//   barney/native/common/math.h:61-125            linear_to_srgb, make_rgba
//   barney/native/volume/DDA.h:61-201             dda3
//   barney/native/volume/Volume.h:62-74,154-203   sampleAndMap, fastLog, Woodcock::sampleRange
//   barney/native/volume/TransferFunction.h:68-117  TF map and majorant
//   barney/native/volume/PrincipledVolume.h       principled sampling and majorant
//   barney/rtcore/cpu/Texture.cpp                 CPU NEAREST / LINEAR tex3D (own TU)
//   barney/rtcore/cpu/Float16.cpp                 float -> binary16 rounding (own TU)
//
// The include tree oracle/refshim/ stands in for the parts of the reference
// build that are absent here (OWL's math library, the CMake-generated config,
// the embree device); it defines no arithmetic of the path beyond OWL's
// elementary vector operations, which it states in its own header.
//
// What this file adds is glue, restated from the reference with file:line:
//   * StructuredDataSampler::DD::sample (StructuredData.h:101-112): the
//     world-to-cell transform and NaN outside, around the reference's tex3D;
//   * the macrocell range loop of StructuredData_computeMCs
//     (StructuredData.cu:31-62) around the reference's NEAREST tex3D and
//     range1f::extend, and mapMCs (MCGrid.cu:97-113) around the reference's
//     TF majorant / principledMajorant;
//   * PerspectiveCamera::commit (Camera.cu:82-101), the pinhole primary ray of
//     _generateRays (generateRays.cu:85-122), the zero-direction fix-up of
//     TraceRays::run (traceRays.dev.cu:38-41), and MCVolumeAccel::isProg's box
//     test, macrocell-grid transform and DDA callback (MCAccelerator.h:552-612,
//     Ray.h:171-181) around the reference's dda3, Random2, hash and
//     Woodcock::sampleRange.
#include "native/common/barney-common.h"
#include "native/common/math.h"
#include "native/volume/DDA.h"
#include "native/volume/TransferFunction.h"
#include "native/volume/Volume.h"
#include "rtcore/cpu/Float16.h"
#include "rtcore/cpu/Texture.h"

#include "bn_oracle.h"

using namespace barney_cpu;
using namespace barney_cpu::native;

namespace {

// StructuredDataSampler stand-in whose DD::sample is StructuredData.h:101-112
// over the reference's CPU LINEAR texture.
struct RefSampler {
  struct DD {
    rtc::TextureObject texObj;
    vec3f cellGridOrigin;
    vec3f cellGridSpacing;
    vec3i numCells;
    float sample(const vec3f P, bool dbg = false) const {
      (void)dbg;
      vec3f rel = (P - cellGridOrigin) * rcp(cellGridSpacing);
      if (rel.x < 0.f) return NAN;
      if (rel.y < 0.f) return NAN;
      if (rel.z < 0.f) return NAN;
      if (rel.x >= numCells.x) return NAN;
      if (rel.y >= numCells.y) return NAN;
      if (rel.z >= numCells.z) return NAN;
      return rtc::tex3D<float>(texObj, rel.x + .5f, rel.y + .5f, rel.z + .5f);
    }
  };
};

rtc::DataType texFormat(int dtype) {
  if (dtype == 0) return rtc::FLOAT;
  if (dtype == 1) return rtc::UCHAR;
  throw std::runtime_error("the reference's CPU sampler reads float and unorm8 3D textures only");
}

// One scene's reference objects: texel copy, NEAREST and LINEAR textures
// (StructuredData.cu:158-172), TF device data and the volume's DD.
struct RefScene {
  const OrcScene &s;
  vec3i numScalars, numCells, mcDims;
  vec3f gridOrigin, gridSpacing, mcOrigin, mcSpacing;
  box3f worldBounds;
  std::unique_ptr<rtc::TextureData> texData;
  std::unique_ptr<rtc::Texture> texLinear, texNearest;
  std::vector<vec4f> tfValues;
  Volume::DD<RefSampler> vol;

  explicit RefScene(const OrcScene &s) : s(s) {
    numScalars = vec3i(s.dims[0], s.dims[1], s.dims[2]);
    numCells = numScalars - vec3i(1);  // StructuredData::set3i
    gridOrigin = vec3f(s.origin[0], s.origin[1], s.origin[2]);
    gridSpacing = vec3f(s.spacing[0], s.spacing[1], s.spacing[2]);
    worldBounds.lower = gridOrigin;  // StructuredData::commit
    worldBounds.upper = gridOrigin + gridSpacing * vec3f(numCells);
    // StructuredData::buildMCs (StructuredData.cu:67-77), cellsPerMC = 8
    mcDims = vec3i((numCells.x + 7) / 8, (numCells.y + 7) / 8, (numCells.z + 7) / 8);
    mcOrigin = worldBounds.lower;
    mcSpacing = vec3f(8.f) * gridSpacing;
    texData.reset(new rtc::TextureData(nullptr, numScalars, texFormat(s.dtype), s.voxels));
    rtc::TextureDesc desc;
    desc.normalizedCoords = false;
    desc.filterMode = rtc::FILTER_MODE_LINEAR;
    texLinear.reset(texData->createTexture(desc));
    desc.filterMode = rtc::FILTER_MODE_POINT;
    texNearest.reset(texData->createTexture(desc));
    for (int i = 0; i < s.tfN; i++)
      tfValues.push_back(vec4f(s.tf[4 * i], s.tf[4 * i + 1], s.tf[4 * i + 2], s.tf[4 * i + 3]));
    vol.sfSampler.texObj = texLinear->getDD();
    vol.sfSampler.cellGridOrigin = gridOrigin;
    vol.sfSampler.cellGridSpacing = gridSpacing;
    vol.sfSampler.numCells = numCells;
    vol.sfCommon.worldBounds = worldBounds;
    vol.xf.values = tfValues.data();
    vol.xf.domain = range1f(s.domain[0], s.domain[1]);
    vol.xf.baseDensity = s.baseDensity;
    vol.xf.numValues = s.tfN;
    PrincipledVolumeParams pv;
    pv.enabled = s.principled;
    pv.density = s.pDensity;
    pv.densityThreshold = s.pDensityThreshold;
    pv.densityScale = s.pDensityScale;
    pv.valueRange = range1f(s.pValueRange[0], s.pValueRange[1]);
    pv.emissionStrength = s.pEmissionStrength;
    pv.blackbodyIntensity = s.pBlackbodyIntensity;
    pv.temperature = s.pTemperature;
    pv.scatterColor = vec3f(s.pScatterColor[0], s.pScatterColor[1], s.pScatterColor[2]);
    pv.absorptionColor = vec3f(s.pAbsorptionColor[0], s.pAbsorptionColor[1], s.pAbsorptionColor[2]);
    pv.emissionColor = vec3f(s.pEmissionColor[0], s.pEmissionColor[1], s.pEmissionColor[2]);
    pv.blackbodyTint = vec3f(s.pBlackbodyTint[0], s.pBlackbodyTint[1], s.pBlackbodyTint[2]);
    vol.principled = pv.getDD(nullptr);
    vol.anisotropy = s.anisotropy;
    vol.scatteringAlbedo = s.scatteringAlbedo;
    vol.userID = 0;
  }

  // StructuredData_computeMCs (StructuredData.cu:38-60) for macrocell tid
  range1f mcRange(int tid) const {
    vec3i mcID(tid % mcDims.x, (tid / mcDims.x) % mcDims.y, tid / (mcDims.x * mcDims.y));
    range1f scalarRange;
    for (int iiz = 0; iiz <= 8; iiz++)
      for (int iiy = 0; iiy <= 8; iiy++)
        for (int iix = 0; iix <= 8; iix++) {
          vec3i scalarID = mcID * 8 + vec3i(iix, iiy, iiz);
          if (scalarID.x >= numScalars.x) continue;
          if (scalarID.y >= numScalars.y) continue;
          if (scalarID.z >= numScalars.z) continue;
          float f = rtc::tex3D<float>(texNearest->getDD(), (float)scalarID.x, (float)scalarID.y, (float)scalarID.z);
          scalarRange.extend(f);
        }
    return scalarRange;
  }
  // mapMCs (MCGrid.cu:97-113)
  float majorant(range1f r) const {
    const float tfMaj = vol.xf.majorant(r);
    return vol.principled.enabled ? principledMajorant(r, vol.principled) * tfMaj : tfMaj;
  }
};

struct Camera {
  vec3f lens00, dir00, dirdu, dirdv;
};
// PerspectiveCamera::set3f("direction") normalizes, then commit
// (Camera.cu:72-101)
Camera commitCamera(const OrcScene &s) {
  Camera c;
  vec3f direction = normalize(vec3f(s.camDir[0], s.camDir[1], s.camDir[2]));
  vec3f up(s.camUp[0], s.camUp[1], s.camUp[2]);
  vec3f dir_00 = normalize(direction);
  vec3f dir_du = normalize(cross(dir_00, up));
  vec3f dir_dv = normalize(cross(dir_du, dir_00));
  dir_00 *= (float)(1.f / (2.0f * tanf((0.5f * s.fovy) * (float)M_PI / 180.0f)));
  c.lens00 = vec3f(s.camPos[0], s.camPos[1], s.camPos[2]);
  c.dir00 = dir_00;
  c.dirdu = dir_du;
  c.dirdv = dir_dv;
  return c;
}

struct TraceOut {
  int hit = 0;
  float t = 0.f;
  vec3f rgb = vec3f(0.f);
  int samples = 0;  // sampleAndMap calls
  int visits = 0;   // DDA callbacks
};

// One ray through MCVolumeAccel::isProg (MCAccelerator.h:552-612) of the
// single-scatter build: the first accepted Woodcock collision, if any.
TraceOut traceVolume(const RefScene &sc, const std::vector<float> &majorants, vec3f org, vec3f rayDir,
                     float rayTMax, RNGSeed raySeed) {
  TraceOut out;
  // TraceRays::run: zero components of the traced direction become 1e-6
  vec3f dir = rayDir;
  if (dir.x == 0.f) dir.x = 1e-6f;
  if (dir.y == 0.f) dir.y = 1e-6f;
  if (dir.z == 0.f) dir.z = 1e-6f;
  range1f tRange = {0.f, rayTMax};
  // boxTest (Ray.h:171-181)
  {
    const box3f &box = sc.worldBounds;
    vec3f t_lo = (box.lower - org) * rcp(dir);
    vec3f t_hi = (box.upper - org) * rcp(dir);
    vec3f t_nr = min(t_lo, t_hi);
    vec3f t_fr = max(t_lo, t_hi);
    tRange.lower = max(tRange.lower, reduce_max(t_nr));
    tRange.upper = min(tRange.upper, reduce_min(t_fr));
    if (!(tRange.lower <= tRange.upper)) return out;
  }
  vec3f dda_org = (org - sc.mcOrigin) * rcp(sc.mcSpacing);
  vec3f dda_dir = dir * rcp(sc.mcSpacing);
  Random rng(raySeed, hash(0u, 0u, 0u));
  const Volume::DD<RefSampler> &vol = sc.vol;
  // counts the samples Woodcock::sampleRange takes through sampleAndMap
  struct CountingVolume {
    const Volume::DD<RefSampler> &v;
    int *n;
    vec4f sampleAndMap(vec3f P, bool dbg = false) const {
      (*n)++;
      return v.sampleAndMap(P, dbg);
    }
  } counting{vol, &out.samples};
  dda3(dda_org, dda_dir, tRange.upper, vec3ui(sc.mcDims),
       [&](const vec3i &cellIdx, float t0, float t1) -> bool {
         out.visits++;
         const float majorant = majorants[cellIdx.x + sc.mcDims.x * (cellIdx.y + sc.mcDims.y * cellIdx.z)];
         if (majorant == 0.f) return true;
         vec4f sample = 0.f;
         range1f wRange = {t0, min(t1, rayTMax)};
         if (!Woodcock::sampleRange(sample, counting, org, dir, wRange, majorant, rng, false)) return true;
         out.hit = 1;
         out.t = wRange.upper;
         out.rgb = vec3f(sample.x, sample.y, sample.z);
         return false;
       },
       false);
  return out;
}

std::vector<float> buildMajorants(const RefScene &sc) {
  const int n = sc.mcDims.x * sc.mcDims.y * sc.mcDims.z;
  std::vector<float> m(n);
  for (int i = 0; i < n; i++) m[i] = sc.majorant(sc.mcRange(i));
  return m;
}

}  // namespace

extern "C" {

void ref_rng_stream(uint32_t a, uint32_t b, int n, uint32_t *out) {
  Random2 r(a, b);
  for (int i = 0; i < n; i++) out[i] = r.next();
}
void ref_rng_floats(uint32_t a, uint32_t b, int n, float *out) {
  Random2 r(a, b);
  for (int i = 0; i < n; i++) out[i] = r();
}
// Random2(RNGSeed &parent, uint64_t b): n outputs of the child and the
// parent's state after the derivation
void ref_rng_derived(uint64_t parentState, uint64_t h, int n, uint32_t *out, uint64_t *parentOut) {
  RNGSeed parent;
  parent.state = parentState;
  Random2 child(parent, h);
  for (int i = 0; i < n; i++) out[i] = child.next();
  *parentOut = parent.state;
}
// the ray seed of _generateRays: RNGSeed::seed(a, b) from the default state
uint64_t ref_ray_seed(uint32_t a, uint32_t b) {
  RNGSeed s;
  s.seed(a, b);
  return s.state;
}
uint64_t ref_hash3(uint32_t a, uint32_t b, uint32_t c) { return hash(a, b, c); }
void ref_fastlog(int n, const float *x, float *out) {
  for (int i = 0; i < n; i++) out[i] = fastLog(x[i]);
}
void ref_f2h(int n, const float *x, uint16_t *out) {
  for (int i = 0; i < n; i++) out[i] = float32ToFloat16(x[i]);
}
void ref_h2f(int n, const uint16_t *x, float *out) {
  for (int i = 0; i < n; i++) out[i] = float16ToFloat32(x[i]);
}
void ref_linear_to_srgb(int n, const float *x, float *out) {
  for (int i = 0; i < n; i++) out[i] = linear_to_srgb(x[i]);
}
void ref_make_rgba(int n, const float *rgba, uint32_t *out) {
  for (int i = 0; i < n; i++)
    out[i] = make_rgba(vec4f(rgba[4 * i], rgba[4 * i + 1], rgba[4 * i + 2], rgba[4 * i + 3]));
}
// tex3D at unnormalized texel coordinates, NEAREST (linear = 0) or LINEAR
void ref_tex3d(const OrcScene *s, int linear, int n, const float *tc, float *out) {
  RefScene sc(*s);
  rtc::TextureObject t = linear ? sc.texLinear->getDD() : sc.texNearest->getDD();
  for (int i = 0; i < n; i++) out[i] = rtc::tex3D<float>(t, tc[3 * i], tc[3 * i + 1], tc[3 * i + 2]);
}
// the structured sampler (NaN outside) and sampleAndMap at world points
void ref_sample_points(const OrcScene *s, int n, const float *P, float *outScalar, float *outRGBA) {
  RefScene sc(*s);
  for (int i = 0; i < n; i++) {
    const vec3f p(P[3 * i], P[3 * i + 1], P[3 * i + 2]);
    outScalar[i] = sc.vol.sampleScalar(p);
    const vec4f m = sc.vol.sampleAndMap(p);
    outRGBA[4 * i] = m.x; outRGBA[4 * i + 1] = m.y; outRGBA[4 * i + 2] = m.z; outRGBA[4 * i + 3] = m.w;
  }
}
void ref_tf_map(const OrcScene *s, int n, const float *v, float *outRGBA) {
  RefScene sc(*s);
  for (int i = 0; i < n; i++) {
    const vec4f m = sc.vol.xf.map(v[i]);
    outRGBA[4 * i] = m.x; outRGBA[4 * i + 1] = m.y; outRGBA[4 * i + 2] = m.z; outRGBA[4 * i + 3] = m.w;
  }
}
void ref_mc_dims(const OrcScene *s, int *out) {
  RefScene sc(*s);
  out[0] = sc.mcDims.x; out[1] = sc.mcDims.y; out[2] = sc.mcDims.z;
}
void ref_build_ranges(const OrcScene *s, float *out) {
  RefScene sc(*s);
  const int n = sc.mcDims.x * sc.mcDims.y * sc.mcDims.z;
  for (int i = 0; i < n; i++) {
    const range1f r = sc.mcRange(i);
    out[2 * i] = r.lower;
    out[2 * i + 1] = r.upper;
  }
}
void ref_map_majorants(const OrcScene *s, const float *ranges, int64_t n, float *out) {
  RefScene sc(*s);
  for (int64_t i = 0; i < n; i++) out[i] = sc.majorant(range1f(ranges[2 * i], ranges[2 * i + 1]));
}
// the principled volume's sampleMap (rgb tint, sigma_t) and emission at scalars
void ref_principled(const OrcScene *s, int n, const float *v, float *outMap, float *outEmission) {
  RefScene sc(*s);
  for (int i = 0; i < n; i++) {
    const vec4f m = principledSampleMap(v[i], sc.vol.principled);
    const vec3f e = principledEmission(v[i], sc.vol.principled);
    outMap[4 * i] = m.x; outMap[4 * i + 1] = m.y; outMap[4 * i + 2] = m.z; outMap[4 * i + 3] = m.w;
    outEmission[3 * i] = e.x; outEmission[3 * i + 1] = e.y; outEmission[3 * i + 2] = e.z;
  }
}
// dda3 over a grid of `grid` cells for a grid-space ray: the cells visited
// with their [t0, t1]; returns the number written (<= maxCells)
int ref_dda_cells(const float *org, const float *dir, float tMax, const int *grid, int maxCells, int *outCells,
                  float *outT) {
  int n = 0;
  dda3(vec3f(org[0], org[1], org[2]), vec3f(dir[0], dir[1], dir[2]), tMax,
       vec3ui(vec3i(grid[0], grid[1], grid[2])),
       [&](const vec3i &c, float t0, float t1) -> bool {
         if (n >= maxCells) return false;
         outCells[3 * n] = c.x; outCells[3 * n + 1] = c.y; outCells[3 * n + 2] = c.z;
         outT[2 * n] = t0; outT[2 * n + 1] = t1;
         n++;
         return true;
       },
       false);
  return n;
}
// Woodcock first collision along an explicit ray with an explicit RNG seed
// state (MCAccelerator.h:552-612): hit flag, t, TF rgb at the collision and
// the samples taken / macrocells visited.
void ref_trace_ray(const OrcScene *s, const float *org, const float *dir, float tMax, uint64_t seedState, int *hit,
                   float *t, float *rgb, int *counts) {
  RefScene sc(*s);
  const std::vector<float> maj = buildMajorants(sc);
  RNGSeed seed;
  seed.state = seedState;
  const TraceOut o = traceVolume(sc, maj, vec3f(org[0], org[1], org[2]), vec3f(dir[0], dir[1], dir[2]), tMax, seed);
  *hit = o.hit;
  *t = o.t;
  rgb[0] = o.rgb.x; rgb[1] = o.rgb.y; rgb[2] = o.rgb.z;
  counts[0] = o.samples;
  counts[1] = o.visits;
}
// The primary ray of every pixel of the frame at accumID (generateRays.cu:
// 85-122, pinhole, no cut plane) traced through isProg: per pixel hit flag,
// t, TF rgb at the first collision, and the samples / visits counts.
void ref_trace_frame(const OrcScene *s, int accumID, int *hit, float *t, float *rgb, int *counts) {
  RefScene sc(*s);
  const std::vector<float> maj = buildMajorants(sc);
  const Camera cam = commitCamera(*s);
  const vec2i fbSize(s->width, s->height);
  for (int iy = 0; iy < fbSize.y; iy++)
    for (int ix = 0; ix < fbSize.x; ix++) {
      Random rand(unsigned(ix + fbSize.x * accumID), unsigned(iy + fbSize.y * accumID));
      RNGSeed raySeed;
      raySeed.seed(ix + accumID * fbSize.x, iy);
      float pixel_u = ((accumID == 0) ? .5f : rand());
      float pixel_v = ((accumID == 0) ? .5f : rand());
      float image_u = ((ix + pixel_u) / float(fbSize.x));
      float image_v = ((iy + pixel_v) / float(fbSize.y));
      float aspect = fbSize.x / float(fbSize.y);
      vec3f ray_dir = cam.dir00 + (1.f * aspect * (image_u - .5f)) * cam.dirdu + (1.f * (image_v - .5f)) * cam.dirdv;
      ray_dir = normalize(ray_dir);
      const TraceOut o = traceVolume(sc, maj, cam.lens00, ray_dir, 1e30f, raySeed);
      const size_t p = (size_t)iy * fbSize.x + ix;
      hit[p] = o.hit;
      t[p] = o.t;
      rgb[3 * p] = o.rgb.x; rgb[3 * p + 1] = o.rgb.y; rgb[3 * p + 2] = o.rgb.z;
      counts[2 * p] = o.samples;
      counts[2 * p + 1] = o.visits;
    }
}

}  // extern "C"
