// bn_objects.h -- host object model of barney_b200 shared by the C ABI
// (bn_api.cpp) and the render server (bn_server.cpp).
//
// Mirrors the object model of Barney's native layer for the structured-volume
// path: Context (barney/native/Context.*), TextureData
// (barney/native/common/Texture.cpp:85-135), StructuredData
// (barney/native/volume/StructuredData.cu:128-181), Volume + TransferFunction
// (barney/native/volume/Volume.cpp, TransferFunction.cpp), Group / Model
// (barney/native/Group.cpp, GlobalModel.cpp, ModelSlot.cpp), DirLight
// (barney/native/light/DirLight.*), PerspectiveCamera (barney/native/Camera.cu),
// Renderer (barney/native/render/Renderer.*) and FrameBuffer
// (barney/native/fb/FrameBuffer.*).  Parameter names and defaults are the
// reference's.
#pragma once
#include "../../include/bn_volume.h"
#include "bn_device.h"

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace bnb {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};
enum : int { E_OK = 0, E_INVALID_HANDLE = 1, E_INVALID_ARG = 2, E_UNSUPPORTED = 3, E_CUDA = 4, E_STATE = 5,
             E_OOM = 6, E_INTERNAL = 7, E_TIMEOUT = 8 };
extern thread_local int g_lastError;
extern thread_local std::string g_lastErrorString;

// Host-side fault injection (bnxInjectAllocationFailure): after a countdown
// of device allocations, one fails as if the device were out of memory.  The
// failure is made on the host; no CUDA call fails and no device state changes.
inline std::atomic<int> &allocFailCountdown() {
  static std::atomic<int> c{-1};
  return c;
}
// cudaMalloc, or the injected failure
inline cudaError_t deviceMalloc(void **p, size_t n) {
  int c = allocFailCountdown().load();
  while (c >= 0) {
    if (allocFailCountdown().compare_exchange_weak(c, c - 1)) {
      if (c == 0) return cudaErrorMemoryAllocation;
      break;
    }
  }
  return cudaMalloc(p, n);
}

inline void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(e == cudaErrorMemoryAllocation ? E_OOM : E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

// host-side float3 helpers (compiled with -ffp-contract=off)
struct v3 { float x, y, z; };
inline v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline v3 operator*(v3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline v3 cross(v3 a, v3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline v3 normalize(v3 v) { return v * (1.f / sqrtf(dot(v, v))); }
inline float3 F3(v3 v) { return make_float3(v.x, v.y, v.z); }

// ---------------------------------------------------------------------------
// device buffer
// ---------------------------------------------------------------------------
struct DeviceBuffer {
  void *ptr = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  ~DeviceBuffer() { release(); }
  void release() {
    if (ptr && cudaFree(ptr) != cudaSuccess) cudaGetLastError();
    ptr = nullptr;
    bytes = 0;
  }
  void resize(size_t n) {
    if (n == bytes && ptr) return;
    release();
    if (n) ck(deviceMalloc(&ptr, n), "cudaMalloc");
    bytes = n;
  }
};

struct Context;

// NVTX range for the length of a scope: the host stages of a frame (render,
// batch, server slice, macrocell build, read-back) show up as named ranges
// in NVTX-aware tools (ncu --nvtx); without a tool attached a push/pop is a
// check of one pointer.
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

// ---------------------------------------------------------------------------
// objects (Object.h:42-56 set/commit interface)
// ---------------------------------------------------------------------------
struct Object : std::enable_shared_from_this<Object> {
  enum Kind { K_DATA, K_TEXDATA, K_FIELD, K_VOLUME, K_GROUP, K_MODEL, K_LIGHT, K_CAMERA, K_RENDERER, K_FB, K_GEOM,
              K_MATERIAL };
  Context *ctx;
  Kind kind;
  Object(Context *c, Kind k) : ctx(c), kind(k) {}
  virtual ~Object() = default;
  virtual bool set1i(const std::string &, int) { return false; }
  virtual bool set3i(const std::string &, int, int, int) { return false; }
  virtual bool set1f(const std::string &, float) { return false; }
  virtual bool set2f(const std::string &, float, float) { return false; }
  virtual bool set3f(const std::string &, float, float, float) { return false; }
  virtual bool set4f(const std::string &, float, float, float, float) { return false; }
  virtual bool setObject(const std::string &, const std::shared_ptr<Object> &) { return false; }
  virtual void commit() {}
};
using ObjectSP = std::shared_ptr<Object>;

struct Data : Object {
  std::vector<ObjectSP> items;
  explicit Data(Context *c) : Object(c, K_DATA) {}
};

struct TextureData : Object {
  int type = VOX_F32;
  int dims[3] = {0, 0, 0};
  DeviceBuffer buf;
  explicit TextureData(Context *c) : Object(c, K_TEXDATA) {}
};

// StructuredData (StructuredData.h:30-74)
struct StructuredField : Object {
  std::shared_ptr<TextureData> scalars;
  int numScalars[3] = {0, 0, 0};
  int numCells[3] = {0, 0, 0};
  v3 gridOrigin{0, 0, 0};
  v3 gridSpacing{1, 1, 1};
  v3 boundsLo{0, 0, 0}, boundsHi{0, 0, 0};
  explicit StructuredField(Context *c) : Object(c, K_FIELD) {}
  bool set3i(const std::string &m, int x, int y, int z) override {
    if (m == "dims") {
      numScalars[0] = x; numScalars[1] = y; numScalars[2] = z;
      numCells[0] = x - 1; numCells[1] = y - 1; numCells[2] = z - 1;
      return true;
    }
    return false;
  }
  bool set3f(const std::string &m, float x, float y, float z) override {
    if (m == "gridOrigin") { gridOrigin = {x, y, z}; return true; }
    if (m == "gridSpacing") { gridSpacing = {x, y, z}; return true; }
    return false;
  }
  bool setObject(const std::string &m, const ObjectSP &v) override {
    if (m == "textureData") {
      if (!v || v->kind != K_TEXDATA) throw Error(E_INVALID_ARG, "textureData must be a BNTextureData");
      scalars = std::static_pointer_cast<TextureData>(v);
      return true;
    }
    return false;
  }
  void commit() override {  // StructuredData.cu:177-181
    boundsLo = gridOrigin;
    boundsHi = {gridOrigin.x + gridSpacing.x * (float)numCells[0], gridOrigin.y + gridSpacing.y * (float)numCells[1],
                gridOrigin.z + gridSpacing.z * (float)numCells[2]};
  }
};

struct Volume : Object {
  std::shared_ptr<StructuredField> sf;
  // TransferFunction.cpp:10-24 defaults: domain [0,1], two entries of 1, density 1
  float domain[2] = {0.f, 1.f};
  std::vector<float4> tfValues{make_float4(1, 1, 1, 1), make_float4(1, 1, 1, 1)};
  float baseDensity = 1.f;
  float anisotropy = 0.6f;        // Volume.h:140
  float scatteringAlbedo = 0.9f;  // Volume.h:141
  int majorantRoundUp = 0;        // bnx.majorantRoundUp (precision forms)
  // PrincipledVolumeParams defaults (PrincipledVolume.h:17-30)
  PrincipledDD pv{0, 1.f, 0.f, 1.f, 0.f, 1.f, 0.f, 0.f, 0.f, {0.8f, 0.8f, 0.8f}, {0.f, 0.f, 0.f},
                  {1.f, 1.f, 1.f}, {1.f, 1.f, 1.f}};
  bool needsMajorantRebuild = false;
  bool built = false;
  int mcDims[3] = {0, 0, 0};
  DeviceBuffer tfBuf, ranges, majorants, occupied;
  explicit Volume(Context *c) : Object(c, K_VOLUME) {}
  bool set1i(const std::string &m, int v) override {  // Volume.cpp:36-50
    if (m == "bnx.majorantRoundUp") { majorantRoundUp = v ? 1 : 0; needsMajorantRebuild = true; return true; }
    if (m == "principledVolume") { pv.enabled = v ? 1 : 0; needsMajorantRebuild = true; return true; }
    if (m == "userID") return true;
    return false;
  }
  bool set1f(const std::string &m, float v) override {  // Volume.cpp:53-91
    if (m == "anisotropy") { anisotropy = std::min(0.99f, std::max(-0.99f, v)); return true; }
    if (m == "scatteringAlbedo") { scatteringAlbedo = std::min(1.f, std::max(0.f, v)); return true; }
    if (m == "principledDensity") { pv.density = v; needsMajorantRebuild = true; return true; }
    if (m == "principledDensityThreshold") { pv.densityThreshold = std::max(v, 0.f); needsMajorantRebuild = true; return true; }
    if (m == "principledDensityScale") { pv.densityScale = v > 0.f ? v : 1.f; needsMajorantRebuild = true; return true; }
    if (m == "principledEmissionStrength") { pv.emissionStrength = std::max(v, 0.f); return true; }
    if (m == "principledBlackbodyIntensity") { pv.blackbodyIntensity = std::max(v, 0.f); return true; }
    if (m == "principledTemperature") { pv.temperature = std::max(v, 0.f); return true; }
    return false;
  }
  bool set2f(const std::string &m, float x, float y) override {  // Volume.cpp:94-103
    if (m == "principledValueRange") { pv.valueLo = x; pv.valueHi = y; needsMajorantRebuild = true; return true; }
    return false;
  }
  bool set3f(const std::string &m, float x, float y, float z) override {  // Volume.cpp:105-126
    const float3 c = make_float3(std::max(x, 0.f), std::max(y, 0.f), std::max(z, 0.f));
    if (m == "principledScatterColor") { pv.scatterColor = c; needsMajorantRebuild = true; return true; }
    if (m == "principledAbsorptionColor") { pv.absorptionColor = c; needsMajorantRebuild = true; return true; }
    if (m == "principledEmissionColor") { pv.emissionColor = c; return true; }
    if (m == "principledBlackbodyTint") { pv.blackbodyTint = c; return true; }
    return false;
  }
  VolumeDD dd() const;
  void uploadTF();
  void build();
  void remapMajorants();
  void commit() override;
};

// AnariMatte (AnariMatte.h:15-46, AnariMatte.cpp:40-90) with constant
// parameters: "color" (float3 gives alpha 1, float4) and "opacity" (float).
// Sampler- and attribute-mapped parameters are not supported.
struct Material : Object {
  float color[4] = {.8f, .8f, .8f, 1.f};
  float opacity = 1.f;
  bool committed = false;  // HostMaterial::hasBeenCommittedAtLeastOnce
  explicit Material(Context *c) : Object(c, K_MATERIAL) {}
  bool set1f(const std::string &m, float v) override {
    if (m == "opacity") { opacity = v; return true; }
    return false;
  }
  bool set3f(const std::string &m, float x, float y, float z) override {
    if (m == "color") { color[0] = x; color[1] = y; color[2] = z; color[3] = 1.f; return true; }
    return false;
  }
  bool set4f(const std::string &m, float x, float y, float z, float w) override {
    if (m == "color") { color[0] = x; color[1] = y; color[2] = z; color[3] = w; return true; }
    return false;
  }
  void commit() override { committed = true; }
};

// "iso_surface" geometry (IsoSurface.h:27-80, IsoSurface.cpp:36-90): an iso
// value on a structured scalar field, drawn with a material.
struct IsoSurface : Object {
  float isoValue = NAN;
  ObjectSP isoValues;  // bnSetData "isoValues"
  std::shared_ptr<StructuredField> sf;
  std::shared_ptr<Material> material;
  // macrocell scalar ranges of the field, built when no volume of the group
  // provides them (StructuredData::buildMCs, StructuredData.cu:71-96)
  DeviceBuffer ranges;
  int mcDims[3] = {0, 0, 0};
  const StructuredField *rangesOf = nullptr;  // the field, texture and dims the ranges were built for
  const TextureData *rangesTex = nullptr;
  int rangesDims[3] = {0, 0, 0};
  explicit IsoSurface(Context *c) : Object(c, K_GEOM) {}
  bool set1i(const std::string &m, int) override { return m == "userID"; }
  bool set1f(const std::string &m, float v) override {
    if (m == "isoValue") { isoValue = v; return true; }
    return false;
  }
  bool setObject(const std::string &m, const ObjectSP &v) override {
    if (m == "scalarField") {
      if (!v || v->kind != K_FIELD) throw Error(E_INVALID_ARG, "'scalarField' value set on 'iso_surface' is not a scalar field");
      sf = std::static_pointer_cast<StructuredField>(v);
      return true;
    }
    if (m == "material") {
      if (v && v->kind != K_MATERIAL) throw Error(E_INVALID_ARG, "invalid material in geometry::set(\"material\")");
      material = v ? std::static_pointer_cast<Material>(v) : nullptr;
      return true;
    }
    return false;
  }
  void buildRanges();
};

struct DirLight : Object {
  v3 direction{0.f, 0.f, -1.f};  // DirLight.h:37
  float irradiance = NAN;
  float radiance = 1.f;
  v3 color{1.f, 1.f, 1.f};       // Light.h:52
  explicit DirLight(Context *c) : Object(c, K_LIGHT) {}
  bool set1f(const std::string &m, float v) override {
    if (m == "irradiance") { irradiance = v; return true; }
    if (m == "radiance") { radiance = v; return true; }
    return false;
  }
  bool set3f(const std::string &m, float x, float y, float z) override {
    if (m == "direction") { direction = {x, y, z}; return true; }
    if (m == "color") { color = {x, y, z}; return true; }
    if (m == "radiance") {  // DirLight.cu:48-54 (deprecated float3 form)
      radiance = std::max(std::max(x, y), z);
      color = {x / radiance, y / radiance, z / radiance};
      return true;
    }
    if (m == "irradiance") {
      irradiance = std::max(std::max(x, y), z);
      color = {x / irradiance, y / irradiance, z / irradiance};
      return true;
    }
    return false;
  }
  DirLightDD dd() const {  // DirLight.cu:11-20, identity instance
    DirLightDD d;
    v3 dir = normalize(direction);
    d.toLight = make_float3(-dir.x, -dir.y, -dir.z);
    d.color = F3(color);
    d.radiance = std::isnan(irradiance) ? radiance : irradiance;
    return d;
  }
};

struct Group : Object {
  std::shared_ptr<Volume> volume;     // at most one volume
  std::shared_ptr<IsoSurface> iso;    // at most one isosurface geometry
  std::shared_ptr<Data> lights;
  explicit Group(Context *c) : Object(c, K_GROUP) {}
};

struct Model : Object {
  std::shared_ptr<Group> group;
  bool built = false;
  explicit Model(Context *c) : Object(c, K_MODEL) {}
};

// PerspectiveCamera (Camera.cu:17-101)
struct Camera : Object {
  v3 position{0, 0, 0}, direction{0, 0, 1}, up{0, 1, 0};
  float aspect = 1.f, fovy = 60.f, focusDistance = 0.f, apertureRadius = 0.f;
  v3 dir00{0, 0, 1}, dirdu{1, 0, 0}, dirdv{0, 1, 0}, lens00{0, 0, 0};
  explicit Camera(Context *c) : Object(c, K_CAMERA) { commit(); }
  bool set1f(const std::string &m, float v) override {
    if (m == "aspect") { aspect = v; return true; }
    if (m == "apertureRadius") { apertureRadius = v; return true; }
    if (m == "focusDistance") { focusDistance = v; return true; }
    if (m == "fovy") { fovy = v; return true; }
    return false;
  }
  bool set3f(const std::string &m, float x, float y, float z) override {
    if (m == "position") { position = {x, y, z}; return true; }
    if (m == "direction") { direction = normalize(v3{x, y, z}); return true; }
    if (m == "up") { up = {x, y, z}; return true; }
    return false;
  }
  void commit() override {
    v3 d00 = normalize(direction);
    v3 du = normalize(cross(d00, up));
    v3 dv = normalize(cross(du, d00));
    d00 = d00 * (float)(1.f / (2.0f * tanf((0.5f * fovy) * (float)M_PI / 180.0f)));
    dir00 = d00; dirdu = du; dirdv = dv; lens00 = position;
  }
};

// Renderer (Renderer.h:17-78); staged values are committed on bnCommit.
struct Renderer : Object {
  struct Params {
    float4 bgColor = make_float4(0, 0, 0, 1);
    float4 cutPlane = make_float4(0, 0, 0, -1e30f);
    int pathsPerPixel = 1;
    float ambientRadiance = 1.f;
    int maxVolumeBounces = 0;
    int hgPhase = 0;              // bnx: multi-scatter-build phase model (HGPhase)
    int emissionAbsorption = 0;   // bnx
    int exactLog = 0;             // bnx
    int compensatedAccum = 0;     // bnx: Neumaier-compensated accumulation (precision forms)
    int fastMath = 0;             // bnx: the fast-math kernels (FMA contraction, approximate division)
  } staged, p;
  explicit Renderer(Context *c) : Object(c, K_RENDERER) {}
  bool set1i(const std::string &m, int v) override {
    if (m == "pathsPerPixel") { staged.pathsPerPixel = v; return true; }
    if (m == "maxVolumeBounces") { staged.maxVolumeBounces = v; return true; }
    if (m == "crosshairs") return true;
    if (m == "bnx.hgPhase") { staged.hgPhase = v ? 1 : 0; return true; }
    if (m == "bnx.emissionAbsorption") { staged.emissionAbsorption = v ? 1 : 0; return true; }
    if (m == "bnx.exactLog") { staged.exactLog = v ? 1 : 0; return true; }
    if (m == "bnx.compensatedAccum") { staged.compensatedAccum = v ? 1 : 0; return true; }
    if (m == "bnx.fastMath") { staged.fastMath = v ? 1 : 0; return true; }
    return false;
  }
  bool set1f(const std::string &m, float v) override {
    if (m == "ambientRadiance") { staged.ambientRadiance = v; return true; }
    return false;
  }
  bool set4f(const std::string &m, float x, float y, float z, float w) override {
    if (m == "bgColor") { staged.bgColor = make_float4(x, y, z, w); return true; }
    if (m == "cutPlane") { staged.cutPlane = make_float4(x, y, z, w); return true; }
    return false;
  }
  void commit() override { p = staged; }
};

struct FrameBuffer : Object {
  int width = 0, height = 0;
  int colorFormat = FMT_RGBA8;
  uint32_t accumID = 0;
  uint64_t anariFrameEpoch = ~0ull;  // the context's commitEpoch at this buffer's last bnxAnariRenderFrame
  DeviceBuffer accum, color, comp;
  explicit FrameBuffer(Context *c) : Object(c, K_FB) {}
};

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
struct Context {
  int device = 0;
  cudaStream_t ownStream = nullptr;
  cudaStream_t stream = nullptr;
  LaunchCounters *dCounters = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  int blocksPerSM = 0, threadsPerBlock = 128;
  SchedDD sched;
  BNXStats stats{};
  // batch path: job table + chunk prefix (device, and pinned host mirrors a
  // captured graph copies from), and the cached graph of the last batch shape
  DeviceBuffer batchJobs, batchChunks;
  JobDD *hostJobs = nullptr;
  int *hostChunks = nullptr;
  LaunchCounters *hostCounters = nullptr;
  int hostCapacity = 0;
  bool useGraphs = true;
  int timeoutMs = 0;                 // render deadline (0: none)
  uint64_t commitEpoch = 0;          // commits and builds so far (bnxAnariRenderFrame)
  int partRank = 0, partCount = 1;   // pixel-tile partition (bnxSetPixelPartition)
  cudaStream_t abortStream = nullptr;
  cudaGraphExec_t graphExec = nullptr;
  std::vector<const void *> graphKey;
  std::mutex mutex;
  std::unordered_map<Object *, std::pair<ObjectSP, int>> handles;  // app references

  explicit Context(int dev) : device(dev) {
    ck(cudaSetDevice(dev), "cudaSetDevice");
    ck(cudaStreamCreateWithFlags(&ownStream, cudaStreamNonBlocking), "cudaStreamCreate");
    stream = ownStream;
    ck(deviceMalloc((void **)&dCounters, sizeof(LaunchCounters)), "cudaMalloc counters");
    ck(cudaMemset(dCounters, 0, sizeof(LaunchCounters)), "cudaMemset");
    for (auto &e : ev) ck(cudaEventCreate(&e), "cudaEventCreate");
  }
  ~Context() {
    cudaSetDevice(device);
    cudaStreamSynchronize(stream);
    if (graphExec) cudaGraphExecDestroy(graphExec);
    if (abortStream) cudaStreamDestroy(abortStream);
    if (hostJobs) cudaFreeHost(hostJobs);
    if (hostChunks) cudaFreeHost(hostChunks);
    if (hostCounters) cudaFreeHost(hostCounters);
    handles.clear();
    for (auto &e : ev) if (e) cudaEventDestroy(e);
    if (dCounters) cudaFree(dCounters);
    if (ownStream) cudaStreamDestroy(ownStream);
    cudaGetLastError();  // nothing of a destroyed context may leak into later calls
  }
  void activate() { ck(cudaSetDevice(device), "cudaSetDevice"); }
  BNObject add(const ObjectSP &o) {
    std::lock_guard<std::mutex> l(mutex);
    handles[o.get()] = {o, 1};
    return (BNObject)o.get();
  }
};

extern std::mutex g_ctxMutex;
extern std::unordered_map<Context *, std::unique_ptr<Context>> g_contexts;

Context *getContext(BNContext c);
// handle -> live object (searches all contexts; handles are unique pointers)
ObjectSP getObject(BNObject h);

template <typename T>
inline std::shared_ptr<T> getAs(BNObject h, Object::Kind k, const char *what) {
  ObjectSP o = getObject(h);
  if (o->kind != k) throw Error(E_INVALID_HANDLE, std::string("handle is not a ") + what);
  return std::static_pointer_cast<T>(o);
}

// rendering (bn_api.cpp)
struct BatchEntry { Renderer *r; Model *m; Camera *c; FrameBuffer *fb; };
JobDD buildJob(Context *ctx, Renderer &r, Model &m, Camera &cam, FrameBuffer &fb);
void renderBatch(Context *ctx, const std::vector<BatchEntry> &entries);
void reserveBatch(Context *ctx, int numJobs);  // job tables for batches up to numJobs

}  // namespace bnb

#define BN_TRY try {
#define BN_CATCH(ret)                                              \
  }                                                                \
  catch (const bnb::Error &e) {                                    \
    bnb::g_lastError = e.code;                                     \
    bnb::g_lastErrorString = e.what();                             \
    return ret;                                                    \
  }                                                                \
  catch (const std::bad_alloc &) {                                 \
    bnb::g_lastError = bnb::E_OOM;                                 \
    bnb::g_lastErrorString = "host out of memory";                 \
    return ret;                                                    \
  }                                                                \
  catch (const std::exception &e) {                                \
    bnb::g_lastError = bnb::E_INTERNAL;                            \
    bnb::g_lastErrorString = e.what();                             \
    return ret;                                                    \
  }
