// bn_api.cpp -- extern "C" entry points of barney_b200 (declared in
// include/bn_volume.h) over the host object model of bn_objects.h, and the
// host side of rendering: macrocell builds, job set-up, single and batched
// launches.  Device work goes to the kernels in bn_kernels.cu.
#include "bn_objects.h"

#include <chrono>
#include <climits>
#include <thread>

namespace bnb {

thread_local int g_lastError = 0;
thread_local std::string g_lastErrorString;
std::mutex g_ctxMutex;
std::unordered_map<Context *, std::unique_ptr<Context>> g_contexts;

Context *getContext(BNContext c) {
  std::lock_guard<std::mutex> l(g_ctxMutex);
  auto it = g_contexts.find((Context *)c);
  if (it == g_contexts.end()) throw Error(E_INVALID_HANDLE, "invalid BNContext handle");
  return it->second.get();
}

// handle -> live object (searches all contexts; handles are unique pointers)
ObjectSP getObject(BNObject h) {
  if (!h) throw Error(E_INVALID_HANDLE, "null object handle");
  std::lock_guard<std::mutex> l(g_ctxMutex);
  for (auto &kv : g_contexts) {
    std::lock_guard<std::mutex> l2(kv.second->mutex);
    auto it = kv.second->handles.find((Object *)h);
    if (it != kv.second->handles.end()) return it->second.first;
  }
  throw Error(E_INVALID_HANDLE, "invalid or released object handle");
}

// ---------------------------------------------------------------------------
// volume: TF upload, macrocell build (MCVolumeAccel::build, MCAccelerator.h:156-195)
// ---------------------------------------------------------------------------
// The field part of the device data: voxels, grid and macrocell grid
// (StructuredData::getDD, buildMCs).
static VolumeDD fieldDD(const StructuredField &f, const int mcDims[3]) {
  VolumeDD v{};
  const TextureData &td = *f.scalars;
  v.voxels = td.buf.ptr;
  v.type = td.type;
  v.numScalars = make_int3(td.dims[0], td.dims[1], td.dims[2]);
  v.numCells = make_int3(f.numCells[0], f.numCells[1], f.numCells[2]);
  v.gridOrigin = F3(f.gridOrigin);
  v.rcpSpacing = make_float3(1.f / f.gridSpacing.x, 1.f / f.gridSpacing.y, 1.f / f.gridSpacing.z);
  v.boundsLo = F3(f.boundsLo);
  v.boundsHi = F3(f.boundsHi);
  v.mcDims = make_int3(mcDims[0], mcDims[1], mcDims[2]);
  v.mcOrigin = F3(f.boundsLo);                          // StructuredData.cu:76
  const v3 mcs = {8.f * f.gridSpacing.x, 8.f * f.gridSpacing.y, 8.f * f.gridSpacing.z};  // :77
  v.rcpMcSpacing = make_float3(1.f / mcs.x, 1.f / mcs.y, 1.f / mcs.z);
  return v;
}

// Checks a field against its texture data; returns its macrocell grid dims
// (StructuredData.cu:74) and count.
static size_t macrocellDims(const StructuredField &f, int d[3]) {
  if (!f.scalars) throw Error(E_STATE, "scalar field has no textureData");
  const TextureData &td = *f.scalars;
  for (int a = 0; a < 3; a++)
    if (f.numScalars[a] != td.dims[a] || f.numScalars[a] < 2)
      throw Error(E_INVALID_ARG, "structured field 'dims' must match the texture data and be >= 2");
  for (int a = 0; a < 3; a++) d[a] = (f.numCells[a] + kCellsPerMC - 1) / kCellsPerMC;
  const size_t n = (size_t)d[0] * d[1] * d[2];
  if (n > 0x7fffffffull) throw Error(E_INVALID_ARG, "number of macrocells cannot be expressed in 32 bits");
  return n;
}

VolumeDD Volume::dd() const {
  VolumeDD v = fieldDD(*sf, mcDims);
  v.hasVolume = 1;
  v.majorants = (const float *)majorants.ptr;
  v.mcOccupied = (const unsigned *)occupied.ptr;
  v.tf = (const float4 *)tfBuf.ptr;
  v.tfN = (int)tfValues.size();
  v.domLo = domain[0];
  v.domHi = domain[1];
  v.baseDensity = baseDensity;
  v.phase = PHASE_SIMPLE;
  v.anisotropy = anisotropy;
  v.scatteringAlbedo = scatteringAlbedo;
  v.pv = pv;
  return v;
}

void Volume::uploadTF() {
  tfBuf.resize(tfValues.size() * sizeof(float4));
  ck(cudaMemcpyAsync(tfBuf.ptr, tfValues.data(), tfBuf.bytes, cudaMemcpyHostToDevice, ctx->stream), "TF upload");
}

void Volume::build() {
  NvtxRange range("volume build");
  if (!sf || !sf->scalars) throw Error(E_STATE, "volume's scalar field has no textureData");
  if (!built) {
    int d[3];
    const size_t n = macrocellDims(*sf, d);
    memcpy(mcDims, d, sizeof d);
    ranges.resize(n * sizeof(float2));
    majorants.resize(n * sizeof(float));
    occupied.resize((n + 31) / 32 * sizeof(unsigned));
    uploadTF();
    ck(launchBuildMacrocells(dd(), (float2 *)ranges.ptr, (float *)majorants.ptr, (unsigned *)occupied.ptr,
                             majorantRoundUp, ctx->stream),
       "macrocell build");
    built = true;
    needsMajorantRebuild = false;
  } else if (needsMajorantRebuild) {
    remapMajorants();
  }
}

void Volume::remapMajorants() {
  uploadTF();
  ck(launchMapMajorants(dd(), (const float2 *)ranges.ptr, (float *)majorants.ptr, (unsigned *)occupied.ptr,
                        majorantRoundUp, ctx->stream),
     "majorant map");
  needsMajorantRebuild = false;
}

void Volume::commit() {  // Volume.cpp:26-35
  if (built && needsMajorantRebuild) remapMajorants();
}

// MCIsoSurfaceAccel::build (MCAccelerator.h:200-230): the field's macrocell
// scalar ranges, when no volume of the group has built them
void IsoSurface::buildRanges() {
  NvtxRange range("isosurface ranges");
  if (!sf) throw Error(E_STATE, "isoSurface has no scalarField");
  if (rangesOf == sf.get() && rangesTex == sf->scalars.get() && ranges.ptr &&
      !memcmp(rangesDims, sf->numScalars, sizeof rangesDims))
    return;
  int d[3];
  const size_t n = macrocellDims(*sf, d);
  memcpy(mcDims, d, sizeof d);
  ranges.resize(n * sizeof(float2));
  ck(launchBuildMacrocells(fieldDD(*sf, mcDims), (float2 *)ranges.ptr, nullptr, nullptr, 0, ctx->stream),
     "macrocell range build");
  rangesOf = sf.get();
  rangesTex = sf->scalars.get();
  memcpy(rangesDims, sf->numScalars, sizeof rangesDims);
}

// The isosurface part of a job (MCIsoSurfaceAccel::DD with the AnariMatte
// material's device data): constant parameters read as
// PossiblyMappedParameter::DD::eval does (HostMaterial.h:98-115), Lambertian
// albedo .85 * color / pi, alpha color.w * opacity (AnariMatte.h:49-71), the
// normal's step |bounds size| * .1 / (sum of macrocell dims) (MCAccelerator.h:445-447).
static IsoDD isoDD(const IsoSurface &g, const float2 *ranges, const int mcDims[3]) {
  if (!g.material) throw Error(E_STATE, "isoSurface has no material");
  if (!g.material->committed) throw Error(E_STATE, "isoSurface material has not been committed");
  IsoDD d{};
  d.enabled = 1;
  d.isoValue = g.isoValue;
  d.ranges = ranges;
  const Material &m = *g.material;
  float c[4] = {m.color[0], m.color[1], m.color[2], m.color[3]};
  if (std::isnan(c[0])) { c[0] = c[1] = c[2] = 0.f; c[3] = 1.f; }
  const float opacity = std::isnan(m.opacity) ? 0.f : m.opacity;
  const float reflectance = .85f, oneOverPi = 1.f / (float)M_PI;
  d.albedo = make_float3(reflectance * c[0] * oneOverPi, reflectance * c[1] * oneOverPi, reflectance * c[2] * oneOverPi);
  d.alpha = c[3] * opacity;
  const StructuredField &f = *g.sf;
  const v3 size = {f.boundsHi.x - f.boundsLo.x, f.boundsHi.y - f.boundsLo.y, f.boundsHi.z - f.boundsLo.z};
  d.normalDelta = sqrtf(size.x * size.x + size.y * size.y + size.z * size.z) * .1f /
                  float(mcDims[0] + mcDims[1] + mcDims[2]);
  return d;
}

// ---------------------------------------------------------------------------
// render (Context::renderTiles, Context.cpp:139-182, + finalizeFrame)
// ---------------------------------------------------------------------------
// The device job of one (renderer, model, camera, frame buffer) tuple,
// validated; fr.spp waves starting at the frame buffer's accumID.
JobDD buildJob(Context *ctx, Renderer &r, Model &m, Camera &cam, FrameBuffer &fb) {
  if (!m.built || !m.group || (!m.group->volume && !m.group->iso))
    throw Error(E_STATE, "model has no built volume or isosurface instance");
  if (fb.width <= 0 || fb.height <= 0) throw Error(E_STATE, "frame buffer has not been resized");
  if (cam.apertureRadius > 0.f) throw Error(E_UNSUPPORTED, "depth-of-field cameras are not supported");
  const Renderer::Params &p = r.p;
  JobDD job{};
  VolumeDD &v = job.v;
  Volume *vol = m.group->volume.get();
  IsoSurface *iso = m.group->iso.get();
  if (vol) {
    vol->build();  // no-op unless the TF changed
    v = vol->dd();
  }
  if (iso) {
    if (!iso->sf) throw Error(E_STATE, "isoSurface has no scalarField");
    if (p.emissionAbsorption) throw Error(E_UNSUPPORTED, "isosurfaces do not render in emission-absorption mode");
    if (vol) {
      if (iso->sf != vol->sf)
        throw Error(E_UNSUPPORTED, "an isosurface and a volume of one group must share their scalar field");
      v.iso = isoDD(*iso, (const float2 *)vol->ranges.ptr, vol->mcDims);
    } else {
      iso->buildRanges();
      v = fieldDD(*iso->sf, iso->mcDims);
      v.hasVolume = 0;
      v.iso = isoDD(*iso, (const float2 *)iso->ranges.ptr, iso->mcDims);
    }
  }
  v.phase = p.hgPhase ? PHASE_HG : PHASE_SIMPLE;
  FrameDD &fr = job.fr;
  fr.dir00 = F3(cam.dir00);
  fr.dirdu = F3(cam.dirdu);
  fr.dirdv = F3(cam.dirdv);
  fr.lens00 = F3(cam.lens00);
  fr.width = fb.width;
  fr.height = fb.height;
  fr.aspect = (float)fr.width / (float)fr.height;  // generateRays.cu: W / float(H)
  fr.bgColor = p.bgColor;
  fr.ambientRadiance = p.ambientRadiance;
  fr.cutPlane = p.cutPlane;
  fr.numDirLights = 0;
  if (m.group->lights) {
    for (auto &o : m.group->lights->items) {
      if (!o || o->kind != Object::K_LIGHT) continue;
      if (fr.numDirLights == kMaxDirLights) throw Error(E_UNSUPPORTED, "too many directional lights");
      fr.dirLights[fr.numDirLights++] = std::static_pointer_cast<DirLight>(o)->dd();
    }
  }
  fr.dirLightPick = fr.numDirLights > 0 ? 2.f / (float)fr.numDirLights : 0.f;
  fr.emissionAbsorption = p.emissionAbsorption;
  fr.exactLog = p.exactLog;
  fr.fastMath = p.fastMath;
  // maxVolumeBounces acts in the multi-scatter build only (bnx.hgPhase); the
  // default build treats a volume scatter as the end of the path
  // (shadeRays.cu:23-25,774-796), so there it has no effect, as in Barney
  fr.maxVolumeBounces = (p.hgPhase && p.maxVolumeBounces > 0) ? p.maxVolumeBounces : 0;
  fr.partRank = ctx->partRank;
  fr.partCount = ctx->partCount;
  fr.accum = (float4 *)fb.accum.ptr;
  fr.comp = nullptr;
  if (p.compensatedAccum) {
    if (!fb.comp.ptr) {
      fb.comp.resize((size_t)fb.width * fb.height * sizeof(float4));
      ck(cudaMemsetAsync(fb.comp.ptr, 0, fb.comp.bytes, ctx->stream), "compensation clear");
    }
    fr.comp = (float4 *)fb.comp.ptr;
  }
  fr.accumID0 = (int)fb.accumID;
  fr.spp = p.pathsPerPixel;
  fr.color = fb.color.ptr;
  fr.colorFormat = fb.colorFormat;
  return job;
}

// ev[0..1] bracket the render kernel, ev[1..2] the resolve; a replayed
// graph records only ev[0] and ev[2] around the whole launch (ev[1] = -1).
static void readStats(Context *ctx, const LaunchCounters &hc, unsigned long long pixelSamples, bool whole = false) {
  BNXStats &st = ctx->stats;
  st.samples = hc.samples;
  st.mcVisits = hc.mcVisits;
  st.rays = hc.rays;
  st.pixelSamples = pixelSamples;
  st.errorFlags = hc.errorFlags;
  st.renderMs = st.resolveMs = 0.f;
  if (whole) {
    if (cudaEventElapsedTime(&st.renderMs, ctx->ev[0], ctx->ev[2]) != cudaSuccess) cudaGetLastError();
  } else {
    if (cudaEventElapsedTime(&st.renderMs, ctx->ev[0], ctx->ev[1]) != cudaSuccess) cudaGetLastError();
    if (cudaEventElapsedTime(&st.resolveMs, ctx->ev[1], ctx->ev[2]) != cudaSuccess) cudaGetLastError();
  }
}

// Waits for `done` with the context's render deadline.  On expiry the abort
// word of the launch counters is raised from a side stream; every warp of the
// render kernel stops at its next pixel-chunk fetch, so the stream drains
// promptly and the context stays usable.  Returns true if aborted.
static LaunchCounters *pinnedCounters(Context *ctx) {
  if (!ctx->hostCounters)
    ck(cudaHostAlloc((void **)&ctx->hostCounters, sizeof(LaunchCounters), cudaHostAllocDefault), "pinned counters");
  return ctx->hostCounters;
}

// The deadline counts from `start`, taken before the frame's first launch: a
// launch can block the calling thread (a kernel's code is loaded on its first
// launch in a process), and that time belongs to the frame too.
static bool waitWithDeadline(Context *ctx, cudaEvent_t done, std::chrono::steady_clock::time_point start) {
  if (ctx->timeoutMs <= 0) return false;
  const auto deadline = start + std::chrono::milliseconds(ctx->timeoutMs);
  while (true) {
    cudaError_t q = cudaEventQuery(done);
    if (q == cudaSuccess) return false;
    if (q != cudaErrorNotReady) ck(q, "render");
    if (std::chrono::steady_clock::now() >= deadline) break;
    std::this_thread::sleep_for(std::chrono::microseconds(100));
  }
  if (!ctx->abortStream) ck(cudaStreamCreateWithFlags(&ctx->abortStream, cudaStreamNonBlocking), "abort stream");
  static const unsigned one = 1;
  ck(cudaMemcpyAsync(&ctx->dCounters->abort, &one, sizeof one, cudaMemcpyHostToDevice, ctx->abortStream), "abort");
  ck(cudaStreamSynchronize(ctx->abortStream), "abort");
  return true;
}

// A job that needs none of the extended kernels' features (isosurface,
// multi-scatter, principled volume) runs the fast-math kernels when its
// renderer asks for them (bnx.fastMath); every other job the exact ones.
static bool plainJob(const JobDD &job) {
  return !job.v.iso.enabled && job.fr.maxVolumeBounces <= 0 && !job.v.pv.enabled;
}
// Plain jobs run the regrouped kernel unless the context turned it off
// (bnxSetRegrouping); the per-lane kernel is the same frame.
static cudaError_t launchRenderJob(Context *ctx, const JobDD &job, cudaStream_t s) {
  const bool plain = plainJob(job);
  if (plain && ctx->sched.regrouped)
    return job.fr.fastMath ? fastmath::launchRenderRegrouped(job.v, job.fr, ctx->dCounters, s)
                           : launchRenderRegrouped(job.v, job.fr, ctx->dCounters, s);
  if (job.fr.fastMath && plain)
    return fastmath::launchRender(job.v, job.fr, ctx->dCounters, ctx->blocksPerSM, ctx->threadsPerBlock, s, ctx->sched);
  return launchRender(job.v, job.fr, ctx->dCounters, ctx->blocksPerSM, ctx->threadsPerBlock, s, ctx->sched);
}

static void render(Context *ctx, Renderer &r, Model &m, Camera &cam, FrameBuffer &fb) {
  NvtxRange range("bnRender");
  const auto start = std::chrono::steady_clock::now();
  JobDD job = buildJob(ctx, r, m, cam, fb);
  if (job.fr.spp <= 0) return;
  ck(cudaMemsetAsync(ctx->dCounters, 0, sizeof(LaunchCounters), ctx->stream), "counter reset");
  ck(cudaEventRecord(ctx->ev[0], ctx->stream), "event");
  ck(launchRenderJob(ctx, job, ctx->stream), "render kernel");
  ck(cudaEventRecord(ctx->ev[1], ctx->stream), "event");
  fb.accumID += job.fr.spp;
  ck(launchResolve((const float4 *)fb.accum.ptr, fb.width * fb.height, (int)fb.accumID, fb.colorFormat, fb.color.ptr,
                   ctx->stream, job.fr.comp),
     "resolve kernel");
  ck(cudaEventRecord(ctx->ev[2], ctx->stream), "event");
  // Pinned destination: a copy into pageable memory would block this thread
  // until the render finished, before the deadline could be checked.
  ck(cudaMemcpyAsync(pinnedCounters(ctx), ctx->dCounters, sizeof(LaunchCounters), cudaMemcpyDeviceToHost, ctx->stream),
     "counter read");
  waitWithDeadline(ctx, ctx->ev[1], start);
  ck(cudaStreamSynchronize(ctx->stream), "render");
  const LaunchCounters hc = *ctx->hostCounters;
  readStats(ctx, hc, (unsigned long long)fb.width * fb.height * job.fr.spp);
  if (hc.errorFlags & ERR_ABORTED) {
    fb.accumID = 0;  // the frame is incomplete
    throw Error(E_TIMEOUT, "render aborted: exceeded the " + std::to_string(ctx->timeoutMs) + " ms deadline");
  }
}

// Pinned and device job tables for batches of up to n jobs.
void reserveBatch(Context *ctx, int n) {
  if (n > ctx->hostCapacity) {
    if (ctx->graphExec) { cudaGraphExecDestroy(ctx->graphExec); ctx->graphExec = nullptr; ctx->graphKey.clear(); }
    if (ctx->hostJobs) cudaFreeHost(ctx->hostJobs);
    if (ctx->hostChunks) cudaFreeHost(ctx->hostChunks);
    ctx->hostJobs = nullptr;
    ctx->hostChunks = nullptr;
    const int cap = std::max(n, 2 * ctx->hostCapacity);
    ck(cudaHostAlloc((void **)&ctx->hostJobs, cap * sizeof(JobDD), cudaHostAllocDefault), "pinned job table");
    ck(cudaHostAlloc((void **)&ctx->hostChunks, (cap + 1) * sizeof(int), cudaHostAllocDefault), "pinned chunks");
    pinnedCounters(ctx);
    ctx->batchJobs.resize(cap * sizeof(JobDD));
    ctx->batchChunks.resize((cap + 1) * sizeof(int));
    ctx->hostCapacity = cap;
  }
}

// Every job's waves in one persistent launch of the batch kernel, then one
// batch resolve.  The copy-in of the job table, the counter reset, both
// kernels and the counter read-back are captured once into a CUDA graph per
// batch shape (same frame buffers, sizes and launch configuration) and
// replayed; per-frame values (cameras, accumIDs) travel in the pinned job
// table the graph copies from.  Results equal one bnRender per job.
void renderBatch(Context *ctx, const std::vector<BatchEntry> &entries) {
  NvtxRange range("bnxRenderBatch");
  const auto start = std::chrono::steady_clock::now();
  const int n = (int)entries.size();
  if (n == 0) return;
  if (ctx->partCount > 1) throw Error(E_UNSUPPORTED, "a pixel partition applies to bnRender only, not to batches");
  reserveBatch(ctx, n);
  std::vector<const void *> key;
  long long chunks = 0;
  unsigned long long pixelSamples = 0;
  int extended = 0;  // 1: multi-scatter, principled or exact log; 2: isosurfaces (the extended kernels)
  bool anyIso = false, anyPvms = false;
  int voxelType = -2;     // the type every job shares, else -1
  bool fast = true;       // every job asks for the fast-math kernels
  int compJobs = 0;  // jobs that keep compensation terms
  ctx->hostChunks[0] = 0;
  for (int i = 0; i < n; i++) {
    const BatchEntry &e = entries[i];
    JobDD job = buildJob(ctx, *e.r, *e.m, *e.c, *e.fb);
    if (job.fr.spp <= 0) throw Error(E_INVALID_ARG, "every batch job needs pathsPerPixel >= 1");
    extended = std::max(extended, job.v.iso.enabled ? 2
                                  : (job.fr.maxVolumeBounces > 0 || job.v.pv.enabled || job.fr.exactLog) ? 1 : 0);
    anyIso = anyIso || job.v.iso.enabled;
    anyPvms = anyPvms || job.fr.maxVolumeBounces > 0 || job.v.pv.enabled;
    voxelType = voxelType == -2 || voxelType == job.v.type ? job.v.type : -1;
    fast = fast && job.fr.fastMath;
    compJobs += job.fr.comp != nullptr;
    ctx->hostJobs[i] = job;
    chunks += ((long long)job.fr.width * job.fr.height + 31) / 32;
    if (chunks > 0x7fffffffLL) throw Error(E_INVALID_ARG, "batch too large");
    ctx->hostChunks[i + 1] = (int)chunks;
    pixelSamples += (unsigned long long)job.fr.width * job.fr.height * job.fr.spp;
    key.push_back(e.fb);
    key.push_back(e.fb->accum.ptr);
    key.push_back(e.fb->comp.ptr);
    key.push_back((const void *)(intptr_t)(e.fb->width * 65536 + e.fb->height));
  }
  key.push_back((const void *)(intptr_t)(ctx->blocksPerSM * 4096 + ctx->threadsPerBlock));
  key.push_back((const void *)(intptr_t)ctx->sched.serviceBatch);
  key.push_back((const void *)(intptr_t)n);
  // isosurfaces without volume bounces or principled volumes: the smaller kernel
  if (anyIso && !anyPvms) extended = 3;
  key.push_back((const void *)(intptr_t)extended);
  key.push_back((const void *)(intptr_t)voxelType);
  fast = fast && extended == 0;  // the fast-math object holds the plain kernels only
  key.push_back((const void *)(intptr_t)(fast ? 1 : 0));
  // one job without a graph (a server slice with one request, say): the
  // single-frame kernel, which takes the job as a kernel parameter and keeps
  // the TF in shared memory, and a plain resolve -- the same frame as the
  // batch kernel's, faster
  const bool solo = n == 1 && !ctx->useGraphs;
  auto enqueue = [&](cudaStream_t s, bool timed) {
    if (solo) {
      const JobDD &job = ctx->hostJobs[0];
      ck(cudaMemsetAsync(ctx->dCounters, 0, sizeof(LaunchCounters), s), "counter reset");
      if (timed) ck(cudaEventRecord(ctx->ev[0], s), "event");
      ck(launchRenderJob(ctx, job, s), "render kernel");
      if (timed) ck(cudaEventRecord(ctx->ev[1], s), "event");
      ck(launchResolve(job.fr.accum, job.fr.width * job.fr.height, job.fr.accumID0 + job.fr.spp, job.fr.colorFormat,
                       job.fr.color, s, job.fr.comp),
         "resolve kernel");
      if (timed) ck(cudaEventRecord(ctx->ev[2], s), "event");
      ck(cudaMemcpyAsync(ctx->hostCounters, ctx->dCounters, sizeof(LaunchCounters), cudaMemcpyDeviceToHost, s),
         "counter read");
      return;
    }
    ck(cudaMemcpyAsync(ctx->batchJobs.ptr, ctx->hostJobs, n * sizeof(JobDD), cudaMemcpyHostToDevice, s), "job table");
    ck(cudaMemcpyAsync(ctx->batchChunks.ptr, ctx->hostChunks, (n + 1) * sizeof(int), cudaMemcpyHostToDevice, s),
       "chunk table");
    ck(cudaMemsetAsync(ctx->dCounters, 0, sizeof(LaunchCounters), s), "counter reset");
    if (timed) ck(cudaEventRecord(ctx->ev[0], s), "event");
    const int compMode = compJobs == 0 ? 0 : compJobs == n ? 2 : 1;
    if (!ctx->useGraphs && extended == 0 && n <= kParamJobs)  // the jobs as one kernel parameter
      ck((fast ? fastmath::launchRenderBatchParams : launchRenderBatchParams)(
             ctx->hostJobs, ctx->hostChunks, n, ctx->dCounters, ctx->blocksPerSM, ctx->threadsPerBlock, s, ctx->sched,
             voxelType, compMode),
         "batch render kernel");
    else
    ck((fast ? fastmath::launchRenderBatch : launchRenderBatch)((const JobDD *)ctx->batchJobs.ptr,
                                                                (const int *)ctx->batchChunks.ptr, n, ctx->dCounters,
                                                                ctx->blocksPerSM, ctx->threadsPerBlock, s, ctx->sched,
                                                                extended, voxelType,
                                                                compJobs == 0 ? 0 : compJobs == n ? 2 : 1),
       "batch render kernel");
    if (timed) ck(cudaEventRecord(ctx->ev[1], s), "event");
    ck(launchResolveBatch((const JobDD *)ctx->batchJobs.ptr, (const int *)ctx->batchChunks.ptr, n, (int)chunks, s),
       "batch resolve kernel");
    if (timed) ck(cudaEventRecord(ctx->ev[2], s), "event");
    ck(cudaMemcpyAsync(ctx->hostCounters, ctx->dCounters, sizeof(LaunchCounters), cudaMemcpyDeviceToHost, s),
       "counter read");
  };
  if (ctx->useGraphs) {
    if (!ctx->graphExec || key != ctx->graphKey) {
      if (ctx->graphExec) { cudaGraphExecDestroy(ctx->graphExec); ctx->graphExec = nullptr; }
      cudaGraph_t g = nullptr;
      ck(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
      try {
        enqueue(ctx->stream, false);
      } catch (...) {
        cudaStreamEndCapture(ctx->stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      ck(cudaStreamEndCapture(ctx->stream, &g), "graph capture");
      cudaError_t e = cudaGraphInstantiate(&ctx->graphExec, g, 0);
      cudaGraphDestroy(g);
      ck(e, "graph instantiate");
      ctx->graphKey = key;
    }
    ck(cudaEventRecord(ctx->ev[0], ctx->stream), "event");
    ck(cudaGraphLaunch(ctx->graphExec, ctx->stream), "graph launch");
    ck(cudaEventRecord(ctx->ev[2], ctx->stream), "event");
  } else {
    enqueue(ctx->stream, true);
  }
  waitWithDeadline(ctx, ctx->ev[2], start);
  ck(cudaStreamSynchronize(ctx->stream), "batch render");
  const bool aborted = ctx->hostCounters->errorFlags & ERR_ABORTED;
  for (int i = 0; i < n; i++) entries[i].fb->accumID = aborted ? 0 : entries[i].fb->accumID + ctx->hostJobs[i].fr.spp;
  readStats(ctx, *ctx->hostCounters, pixelSamples, ctx->useGraphs);
  if (aborted)
    throw Error(E_TIMEOUT, "batch render aborted: exceeded the " + std::to_string(ctx->timeoutMs) + " ms deadline");
}

}  // namespace bnb

using namespace bnb;

// ---------------------------------------------------------------------------
// extern "C" entry points
// ---------------------------------------------------------------------------
extern "C" {

BN_API int bnGetLastError(void) { return g_lastError; }
BN_API const char *bnGetLastErrorString(void) { return g_lastErrorString.c_str(); }
BN_API void bnClearLastError(void) { g_lastError = 0; g_lastErrorString.clear(); }

BN_API int bnPhysicalDeviceCount(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return 0; }
  return n;
}

BN_API BNContext bnContextCreate(int numDataGroups, const int *dataRanks, int numGPUs, const int *gpuIDs) {
  BN_TRY
  (void)dataRanks;
  if (numDataGroups > 1) throw Error(E_UNSUPPORTED, "only one data group per context is supported");
  if (numGPUs > 1) throw Error(E_UNSUPPORTED, "only one GPU per context is supported");
  int dev = (gpuIDs && numGPUs == 1) ? gpuIDs[0] : 0;
  int n = bnPhysicalDeviceCount();
  if (dev < 0 || dev >= n) throw Error(E_INVALID_ARG, "no such CUDA device");
  auto c = std::make_unique<Context>(dev);
  Context *raw = c.get();
  std::lock_guard<std::mutex> l(g_ctxMutex);
  g_contexts[raw] = std::move(c);
  return (BNContext)raw;
  BN_CATCH(nullptr)
}

BN_API void bnContextDestroy(BNContext context) {
  BN_TRY
  Context *c = getContext(context);
  std::unique_ptr<Context> owned;
  {
    std::lock_guard<std::mutex> l(g_ctxMutex);
    owned = std::move(g_contexts[c]);
    g_contexts.erase(c);
  }
  BN_CATCH()
}

BN_API void bnRelease(BNObject object) {
  BN_TRY
  ObjectSP o = getObject(object);
  Context *c = o->ctx;
  std::lock_guard<std::mutex> l(c->mutex);
  auto it = c->handles.find(o.get());
  if (--it->second.second <= 0) c->handles.erase(it);
  BN_CATCH()
}

BN_API void bnAddReference(BNObject object) {
  BN_TRY
  ObjectSP o = getObject(object);
  std::lock_guard<std::mutex> l(o->ctx->mutex);
  o->ctx->handles[o.get()].second++;
  BN_CATCH()
}

BN_API void bnCommit(BNObject target) {
  BN_TRY
  ObjectSP o = getObject(target);
  o->ctx->activate();
  o->commit();
  o->ctx->commitEpoch++;
  BN_CATCH()
}

static void warnUnsupported(const char *name) {
  g_lastError = E_UNSUPPORTED;
  g_lastErrorString = std::string("unsupported parameter '") + (name ? name : "(null)") + "'";
}

BN_API void bnSet1i(BNObject t, const char *n, int v) {
  BN_TRY
  if (!getObject(t)->set1i(n ? n : "", v)) warnUnsupported(n);
  BN_CATCH()
}
BN_API void bnSet2i(BNObject t, const char *n, int, int) {
  BN_TRY
  getObject(t);
  warnUnsupported(n);
  BN_CATCH()
}
BN_API void bnSet3i(BNObject t, const char *n, int x, int y, int z) {
  BN_TRY
  if (!getObject(t)->set3i(n ? n : "", x, y, z)) warnUnsupported(n);
  BN_CATCH()
}
BN_API void bnSet4i(BNObject t, const char *n, int, int, int, int) {
  BN_TRY
  getObject(t);
  warnUnsupported(n);
  BN_CATCH()
}
BN_API void bnSet1f(BNObject t, const char *n, float v) {
  BN_TRY
  if (!getObject(t)->set1f(n ? n : "", v)) warnUnsupported(n);
  BN_CATCH()
}
BN_API void bnSet2f(BNObject t, const char *n, float x, float y) {
  BN_TRY
  if (!getObject(t)->set2f(n ? n : "", x, y)) warnUnsupported(n);
  BN_CATCH()
}
BN_API void bnSet3f(BNObject t, const char *n, float x, float y, float z) {
  BN_TRY
  if (!getObject(t)->set3f(n ? n : "", x, y, z)) warnUnsupported(n);
  BN_CATCH()
}
BN_API void bnSet4f(BNObject t, const char *n, float x, float y, float z, float w) {
  BN_TRY
  if (!getObject(t)->set4f(n ? n : "", x, y, z, w)) warnUnsupported(n);
  BN_CATCH()
}
BN_API void bnSetObject(BNObject t, const char *n, BNObject v) {
  BN_TRY
  ObjectSP val = v ? getObject(v) : nullptr;
  if (!getObject(t)->setObject(n ? n : "", val)) warnUnsupported(n);
  BN_CATCH()
}
BN_API void bnSetString(BNObject t, const char *n, const char *) {
  BN_TRY
  getObject(t);
  warnUnsupported(n);
  BN_CATCH()
}
BN_API void bnSet4x3fv(BNObject t, const char *n, const BNTransform *) {
  BN_TRY
  getObject(t);
  warnUnsupported(n);
  BN_CATCH()
}
BN_API void bnSet4x4fv(BNObject t, const char *n, const bn_float4 *) {
  BN_TRY
  getObject(t);
  warnUnsupported(n);
  BN_CATCH()
}
BN_API void bnSetData(BNObject t, const char *n, BNData v) {
  BN_TRY
  ObjectSP o = getObject(t);
  std::string name = n ? n : "";
  if (o->kind == Object::K_GROUP && name == "lights") {
    auto g = std::static_pointer_cast<Group>(o);
    g->lights = v ? getAs<Data>(v, Object::K_DATA, "BNData") : nullptr;
    return;
  }
  if (o->kind == Object::K_GEOM && name == "isoValues") {  // IsoSurface.cpp:60-68
    // kept, and unused: the intersection program reads isoValue only (MCAccelerator.h:325-548)
    std::static_pointer_cast<IsoSurface>(o)->isoValues = v ? getObject(v) : nullptr;
    return;
  }
  warnUnsupported(n);
  BN_CATCH()
}

BN_API void bnDataSet(BNData data, size_t n, const void *items) {  // Data::set
  BN_TRY
  auto d = getAs<Data>(data, Object::K_DATA, "BNData");
  const BNObject *objs = (const BNObject *)items;
  std::vector<ObjectSP> next;
  for (size_t i = 0; i < n; i++) next.push_back(objs && objs[i] ? getObject(objs[i]) : nullptr);
  d->items.swap(next);
  BN_CATCH()
}

static void *unsupportedObject(BNContext context, const char *what) {
  getContext(context);
  throw Error(E_UNSUPPORTED, std::string(what) + " is not supported (surface materials are not mapped)");
}
BN_API BNTextureData bnTextureData2DCreate(BNContext context, int, BNDataType, int, int, const void *) {
  BN_TRY
  return (BNTextureData)unsupportedObject(context, "bnTextureData2DCreate");
  BN_CATCH(nullptr)
}
BN_API BNTexture2D bnTexture2DCreate(BNContext context, int, BNDataType, uint32_t, uint32_t, const void *,
                                     BNTextureFilterMode, BNTextureAddressMode, BNTextureAddressMode,
                                     BNTextureColorSpace) {
  BN_TRY
  return (BNTexture2D)unsupportedObject(context, "bnTexture2DCreate");
  BN_CATCH(nullptr)
}
BN_API BNTexture3D bnTexture3DCreate(BNContext context, int, BNDataType, uint32_t, uint32_t, uint32_t, const void *,
                                     BNTextureFilterMode, BNTextureAddressMode) {
  BN_TRY
  return (BNTexture3D)unsupportedObject(context, "bnTexture3DCreate");
  BN_CATCH(nullptr)
}
BN_API BNSampler bnSamplerCreate(BNContext context, int, const char *) {
  BN_TRY
  return (BNSampler)unsupportedObject(context, "bnSamplerCreate");
  BN_CATCH(nullptr)
}

BN_API BNData bnDataCreate(BNContext context, int, BNDataType type, size_t n, const void *items) {
  BN_TRY
  Context *c = getContext(context);
  if (type != BN_OBJECT) throw Error(E_UNSUPPORTED, "only BN_OBJECT data arrays are supported");
  auto d = std::make_shared<Data>(c);
  const BNObject *objs = (const BNObject *)items;
  for (size_t i = 0; i < n; i++) d->items.push_back(objs && objs[i] ? getObject(objs[i]) : nullptr);
  return c->add(d);
  BN_CATCH(nullptr)
}

BN_API BNTextureData bnTextureData3DCreate(BNContext context, int, BNDataType fmt, int w, int h, int d,
                                           const void *texels) {
  BN_TRY
  Context *c = getContext(context);
  c->activate();
  int type;
  size_t es;
  switch ((int)fmt) {
  case BN_FLOAT32: type = VOX_F32; es = 4; break;
  case BN_UFIXED8:
  case BN_UINT8: type = VOX_U8; es = 1; break;
  case BNX_FLOAT16: type = VOX_F16; es = 2; break;
  case BNX_BFLOAT16: type = VOX_BF16; es = 2; break;
  case BN_UFIXED16: type = VOX_U16; es = 2; break;
  default: throw Error(E_UNSUPPORTED, "unsupported 3D texel format");
  }
  if (w <= 0 || h <= 0 || d <= 0) throw Error(E_INVALID_ARG, "texture dimensions must be positive");
  if (!texels) throw Error(E_INVALID_ARG, "texels pointer is null");
  auto td = std::make_shared<TextureData>(c);
  td->type = type;
  td->dims[0] = w; td->dims[1] = h; td->dims[2] = d;
  const size_t bytes = (size_t)w * h * d * es;
  td->buf.resize(bytes);
  ck(cudaMemcpyAsync(td->buf.ptr, texels, bytes, cudaMemcpyDefault, c->stream), "texture upload");
  ck(cudaStreamSynchronize(c->stream), "texture upload");  // caller may free texels on return
  return c->add(td);
  BN_CATCH(nullptr)
}

BN_API BNScalarField bnScalarFieldCreate(BNContext context, int, const char *type) {
  BN_TRY
  Context *c = getContext(context);
  if (!type || std::string(type) != "structured") throw Error(E_UNSUPPORTED, "only 'structured' scalar fields");
  return c->add(std::make_shared<StructuredField>(c));
  BN_CATCH(nullptr)
}

BN_API BNVolume bnVolumeCreate(BNContext context, int, BNScalarField sf) {
  BN_TRY
  Context *c = getContext(context);
  auto v = std::make_shared<Volume>(c);
  v->sf = getAs<StructuredField>(sf, Object::K_FIELD, "BNScalarField");
  return c->add(v);
  BN_CATCH(nullptr)
}

BN_API void bnVolumeSetXF(BNVolume volume, bn_float2 domain, const bn_float4 *values, int n, float densityAt1) {
  BN_TRY
  auto v = getAs<Volume>(volume, Object::K_VOLUME, "BNVolume");
  if (!values || n < 2) throw Error(E_INVALID_ARG, "transfer function needs at least 2 values");
  if (n > kMaxTF) throw Error(E_UNSUPPORTED, "transfer function has too many entries");
  v->domain[0] = domain.x;
  v->domain[1] = domain.y;
  v->tfValues.resize(n);
  memcpy(v->tfValues.data(), values, n * sizeof(bn_float4));
  v->baseDensity = densityAt1;
  v->needsMajorantRebuild = true;
  v->ctx->commitEpoch++;
  BN_CATCH()
}

BN_API BNLight bnLightCreate(BNContext context, int, const char *type) {
  BN_TRY
  Context *c = getContext(context);
  if (!type || std::string(type) != "directional") throw Error(E_UNSUPPORTED, "only 'directional' lights");
  return c->add(std::make_shared<DirLight>(c));
  BN_CATCH(nullptr)
}

BN_API BNGeom bnGeometryCreate(BNContext context, int, const char *type) {
  BN_TRY
  Context *c = getContext(context);
  const std::string t = type ? type : "";
  if (t != "iso_surface" && t != "isoSurface")  // Geometry.cpp:33
    throw Error(E_UNSUPPORTED, "unsupported geometry type '" + t + "' (only 'iso_surface')");
  return c->add(std::make_shared<IsoSurface>(c));
  BN_CATCH(nullptr)
}

BN_API BNMaterial bnMaterialCreate(BNContext context, int, const char *type) {
  BN_TRY
  Context *c = getContext(context);
  const std::string t = type ? type : "";
  if (t != "matte" && t != "AnariMatte")  // HostMaterial.cpp:82-95
    throw Error(E_UNSUPPORTED, "unsupported material type '" + t + "' (only 'matte' / 'AnariMatte')");
  return c->add(std::make_shared<Material>(c));
  BN_CATCH(nullptr)
}

BN_API BNGroup bnGroupCreate(BNContext context, int, BNGeom *geoms, int numGeoms, BNVolume *volumes, int numVolumes) {
  BN_TRY
  Context *c = getContext(context);
  if (numGeoms < 0 || numGeoms > 1 || (numGeoms == 1 && !geoms))
    throw Error(E_UNSUPPORTED, "at most one (isoSurface) geometry per group is supported");
  if (numVolumes < 0 || numVolumes > 1 || (numVolumes == 1 && !volumes))
    throw Error(E_UNSUPPORTED, "at most one volume per group is supported");
  if (numGeoms + numVolumes == 0) throw Error(E_UNSUPPORTED, "a group needs a volume or an isoSurface");
  auto g = std::make_shared<Group>(c);
  if (numVolumes == 1) g->volume = getAs<Volume>(volumes[0], Object::K_VOLUME, "BNVolume");
  if (numGeoms == 1) g->iso = getAs<IsoSurface>(geoms[0], Object::K_GEOM, "BNGeom");
  return c->add(g);
  BN_CATCH(nullptr)
}

static void buildGroup(Group &g) {
  if (g.volume) g.volume->build();
  if (g.iso && !(g.volume && g.iso->sf == g.volume->sf)) g.iso->buildRanges();
}

BN_API void bnGroupBuild(BNGroup group) {
  BN_TRY
  auto g = getAs<Group>(group, Object::K_GROUP, "BNGroup");
  g->ctx->activate();
  buildGroup(*g);
  ck(cudaStreamSynchronize(g->ctx->stream), "group build");
  g->ctx->commitEpoch++;
  BN_CATCH()
}

BN_API BNModel bnModelCreate(BNContext context) {
  BN_TRY
  Context *c = getContext(context);
  return c->add(std::make_shared<Model>(c));
  BN_CATCH(nullptr)
}

static bool isIdentity(const BNTransform &x) {
  return x.l.vx.x == 1 && x.l.vx.y == 0 && x.l.vx.z == 0 && x.l.vy.x == 0 && x.l.vy.y == 1 && x.l.vy.z == 0 &&
         x.l.vz.x == 0 && x.l.vz.y == 0 && x.l.vz.z == 1 && x.p.x == 0 && x.p.y == 0 && x.p.z == 0;
}

BN_API void bnSetInstances(BNModel model, int, BNGroup *groups, BNTransform *xfms, int n) {
  BN_TRY
  auto m = getAs<Model>(model, Object::K_MODEL, "BNModel");
  if (n > 1) throw Error(E_UNSUPPORTED, "only one instance is supported");
  if (n == 1 && xfms && !isIdentity(xfms[0]))
    throw Error(E_UNSUPPORTED, "only identity instance transforms are supported");
  m->group = (n == 1 && groups) ? getAs<Group>(groups[0], Object::K_GROUP, "BNGroup") : nullptr;
  m->built = false;
  m->ctx->commitEpoch++;
  BN_CATCH()
}

BN_API void bnUpdateInstanceTransforms(BNModel model, int, BNTransform *xfms, int n) {
  BN_TRY
  auto m = getAs<Model>(model, Object::K_MODEL, "BNModel");
  if (n != (m->group ? 1 : 0)) throw Error(E_INVALID_ARG, "instance count differs from bnSetInstances");
  if (n == 1 && xfms && !isIdentity(xfms[0]))
    throw Error(E_UNSUPPORTED, "only identity instance transforms are supported");
  BN_CATCH()
}

BN_API void bnSetInstanceAttributes(BNModel model, int, const char *name, BNData data) {
  BN_TRY
  getAs<Model>(model, Object::K_MODEL, "BNModel");
  if (data) warnUnsupported(name);
  BN_CATCH()
}

BN_API void bnBuild(BNModel model, int) {
  BN_TRY
  auto m = getAs<Model>(model, Object::K_MODEL, "BNModel");
  m->ctx->activate();
  if (m->group) buildGroup(*m->group);
  ck(cudaStreamSynchronize(m->ctx->stream), "model build");
  m->built = true;
  m->ctx->commitEpoch++;
  BN_CATCH()
}

BN_API BNCamera bnCameraCreate(BNContext context, const char *type) {
  BN_TRY
  Context *c = getContext(context);
  std::string t = type ? type : "";
  if (t != "perspective" && t != "pinhole") throw Error(E_UNSUPPORTED, "only perspective cameras are supported");
  return c->add(std::make_shared<Camera>(c));
  BN_CATCH(nullptr)
}

BN_API BNRenderer bnRendererCreate(BNContext context, const char *) {
  BN_TRY
  Context *c = getContext(context);
  return c->add(std::make_shared<Renderer>(c));
  BN_CATCH(nullptr)
}

BN_API BNFrameBuffer bnFrameBufferCreate(BNContext context, int) {
  BN_TRY
  Context *c = getContext(context);
  return c->add(std::make_shared<FrameBuffer>(c));
  BN_CATCH(nullptr)
}

BN_API void bnFrameBufferResize(BNFrameBuffer fbh, BNDataType fmt, int sx, int sy, uint32_t channels) {
  BN_TRY
  auto fb = getAs<FrameBuffer>(fbh, Object::K_FB, "BNFrameBuffer");
  fb->ctx->activate();
  int f;
  switch ((int)fmt) {
  case BN_FLOAT4: f = FMT_FLOAT4; break;
  case BN_UFIXED8_RGBA: f = FMT_RGBA8; break;
  case BN_UFIXED8_RGBA_SRGB: f = FMT_RGBA8_SRGB; break;
  default: throw Error(E_UNSUPPORTED, "unsupported frame buffer colour format");
  }
  if (sx <= 0 || sy <= 0) throw Error(E_INVALID_ARG, "frame buffer size must be positive");
  if ((long long)sx * sy > kMaxFramePixels)  // the kernels index pixels and chunks with 32-bit ints
    throw Error(E_INVALID_ARG, "frame buffer larger than 2^31 - 1 pixels");
  if (!(channels & BN_FB_COLOR)) throw Error(E_UNSUPPORTED, "the colour channel is required");
  // unusable until both buffers exist: a failed allocation leaves a frame
  // buffer that every render and read rejects as not resized
  fb->width = fb->height = 0;
  fb->comp.release();
  fb->accumID = 0;
  fb->accum.resize((size_t)sx * sy * sizeof(float4));
  fb->color.resize((size_t)sx * sy * (f == FMT_FLOAT4 ? 16 : 4));
  fb->width = sx;
  fb->height = sy;
  fb->colorFormat = f;
  BN_CATCH()
}

BN_API void bnFrameBufferGetSize(BNFrameBuffer fbh, int *sx, int *sy) {
  BN_TRY
  if (!sx || !sy) return;
  auto fb = getAs<FrameBuffer>(fbh, Object::K_FB, "BNFrameBuffer");
  *sx = fb->width;
  *sy = fb->height;
  BN_CATCH()
}

BN_API void bnFrameBufferRead(BNFrameBuffer fbh, BNFrameBufferChannel ch, void *ptr, BNDataType fmt) {
  NvtxRange range("bnFrameBufferRead");
  BN_TRY
  auto fb = getAs<FrameBuffer>(fbh, Object::K_FB, "BNFrameBuffer");
  if (!ptr) return;  // FrameBuffer.cu:319
  if (ch != BN_FB_COLOR) throw Error(E_UNSUPPORTED, "only the colour channel can be read");
  int f = fmt == BN_FLOAT4 ? FMT_FLOAT4 : fmt == BN_UFIXED8_RGBA ? FMT_RGBA8
        : fmt == BN_UFIXED8_RGBA_SRGB ? FMT_RGBA8_SRGB : -1;
  if (f != fb->colorFormat) throw Error(E_INVALID_ARG, "requested format differs from the frame buffer's format");
  if (fb->width <= 0 || fb->height <= 0) throw Error(E_STATE, "frame buffer has not been resized");
  fb->ctx->activate();
  ck(cudaMemcpyAsync(ptr, fb->color.ptr, fb->color.bytes, cudaMemcpyDefault, fb->ctx->stream), "frame read");
  ck(cudaStreamSynchronize(fb->ctx->stream), "frame read");
  BN_CATCH()
}

// checkpoint header of bnxFrameBufferCheckpoint
struct CheckpointHeader {
  uint32_t magic, version;
  int32_t width, height;
  uint32_t accumID, hasComp, reserved[2];
};
static_assert(sizeof(CheckpointHeader) == 32, "checkpoint header is 32 bytes");
static constexpr uint32_t kCheckpointMagic = 0x43584E42u;  // "BNXC"

BN_API size_t bnxFrameBufferCheckpointSize(BNFrameBuffer fbh) {
  BN_TRY
  auto fb = getAs<FrameBuffer>(fbh, Object::K_FB, "BNFrameBuffer");
  if (fb->width <= 0 || fb->height <= 0) throw Error(E_STATE, "frame buffer has not been resized");
  const size_t px = (size_t)fb->width * fb->height * sizeof(float4);
  return sizeof(CheckpointHeader) + px + (fb->comp.ptr ? px : 0);
  BN_CATCH(0)
}

BN_API void bnxFrameBufferCheckpoint(BNFrameBuffer fbh, void *out) {
  BN_TRY
  auto fb = getAs<FrameBuffer>(fbh, Object::K_FB, "BNFrameBuffer");
  if (!out) throw Error(E_INVALID_ARG, "null checkpoint destination");
  if (fb->width <= 0 || fb->height <= 0) throw Error(E_STATE, "frame buffer has not been resized");
  Context *ctx = fb->ctx;
  ctx->activate();
  CheckpointHeader h{kCheckpointMagic, 1u, fb->width, fb->height, fb->accumID, fb->comp.ptr ? 1u : 0u, {0u, 0u}};
  memcpy(out, &h, sizeof h);
  const size_t px = (size_t)fb->width * fb->height * sizeof(float4);
  char *dst = (char *)out + sizeof h;
  ck(cudaMemcpyAsync(dst, fb->accum.ptr, px, cudaMemcpyDeviceToHost, ctx->stream), "checkpoint");
  if (fb->comp.ptr) ck(cudaMemcpyAsync(dst + px, fb->comp.ptr, px, cudaMemcpyDeviceToHost, ctx->stream), "checkpoint");
  ck(cudaStreamSynchronize(ctx->stream), "checkpoint");
  BN_CATCH()
}

BN_API void bnxFrameBufferRestore(BNFrameBuffer fbh, const void *in, size_t bytes) {
  BN_TRY
  auto fb = getAs<FrameBuffer>(fbh, Object::K_FB, "BNFrameBuffer");
  if (!in || bytes < sizeof(CheckpointHeader)) throw Error(E_INVALID_ARG, "checkpoint too short");
  CheckpointHeader h;
  memcpy(&h, in, sizeof h);
  if (h.magic != kCheckpointMagic || h.version != 1u) throw Error(E_INVALID_ARG, "not a frame buffer checkpoint");
  if (h.width != fb->width || h.height != fb->height)
    throw Error(E_INVALID_ARG, "checkpoint size differs from the frame buffer's");
  const size_t px = (size_t)fb->width * fb->height * sizeof(float4);
  if (bytes != sizeof h + px + (h.hasComp ? px : 0)) throw Error(E_INVALID_ARG, "checkpoint length is wrong");
  // the render loop and the resolve count waves in an int
  if (h.accumID > (uint32_t)INT_MAX) throw Error(E_INVALID_ARG, "checkpoint accumID is out of range");
  Context *ctx = fb->ctx;
  ctx->activate();
  // allocate before anything is copied, so that a failed allocation leaves
  // the frame buffer as it was
  if (h.hasComp && !fb->comp.ptr) fb->comp.resize(px);
  // from here on a failed copy leaves an empty frame buffer (accumID 0: the
  // next render writes its first wave instead of adding to the buffer)
  fb->accumID = 0;
  const char *src = (const char *)in + sizeof h;
  ck(cudaMemcpyAsync(fb->accum.ptr, src, px, cudaMemcpyHostToDevice, ctx->stream), "restore");
  if (h.hasComp) {
    ck(cudaMemcpyAsync(fb->comp.ptr, src + px, px, cudaMemcpyHostToDevice, ctx->stream), "restore");
  } else if (fb->comp.ptr) {
    ck(cudaMemsetAsync(fb->comp.ptr, 0, px, ctx->stream), "restore");
  }
  fb->accumID = h.accumID;
  if (h.accumID > 0)
    ck(launchResolve((const float4 *)fb->accum.ptr, fb->width * fb->height, (int)fb->accumID, fb->colorFormat,
                     fb->color.ptr, ctx->stream, h.hasComp ? (const float4 *)fb->comp.ptr : nullptr),
       "resolve kernel");
  ck(cudaStreamSynchronize(ctx->stream), "restore");
  BN_CATCH()
}

BN_API void bnAccumReset(BNFrameBuffer fbh) {
  BN_TRY
  getAs<FrameBuffer>(fbh, Object::K_FB, "BNFrameBuffer")->accumID = 0;
  BN_CATCH()
}

BN_API void bnRender(BNRenderer rh, BNModel mh, BNCamera ch, BNFrameBuffer fbh) {
  BN_TRY
  auto r = getAs<Renderer>(rh, Object::K_RENDERER, "BNRenderer");
  auto m = getAs<Model>(mh, Object::K_MODEL, "BNModel");
  auto c = getAs<Camera>(ch, Object::K_CAMERA, "BNCamera");
  auto fb = getAs<FrameBuffer>(fbh, Object::K_FB, "BNFrameBuffer");
  fb->ctx->activate();
  render(fb->ctx, *r, *m, *c, *fb);
  BN_CATCH()
}

BN_API void bnxGetStats(BNContext context, BNXStats *stats) {
  BN_TRY
  if (stats) *stats = getContext(context)->stats;
  BN_CATCH()
}

BN_API void bnxSetStream(BNContext context, void *s) {
  BN_TRY
  Context *c = getContext(context);
  c->stream = s ? (cudaStream_t)s : c->ownStream;
  BN_CATCH()
}

BN_API void *bnxGetStream(BNContext context) {
  BN_TRY
  return (void *)getContext(context)->stream;
  BN_CATCH(nullptr)
}

BN_API void bnxSetLaunchConfig(BNContext context, int bps, int tpb) {
  BN_TRY
  Context *c = getContext(context);
  if (tpb != 0 && (tpb % 32 != 0 || tpb > kRenderMaxThreads || tpb < 32))
    throw Error(E_INVALID_ARG, "threadsPerBlock must be a multiple of 32 in [32, 128]");
  c->blocksPerSM = bps < 0 ? 0 : bps;
  c->threadsPerBlock = tpb ? tpb : 128;
  BN_CATCH()
}

BN_API void *bnxFrameBufferDevicePointer(BNFrameBuffer fbh) {
  BN_TRY
  return getAs<FrameBuffer>(fbh, Object::K_FB, "BNFrameBuffer")->color.ptr;
  BN_CATCH(nullptr)
}

BN_API void bnxVolumeGetMacrocells(BNVolume vh, int *dims3, float *rangesOut, float *majOut) {
  BN_TRY
  auto v = getAs<Volume>(vh, Object::K_VOLUME, "BNVolume");
  if (!v->built) throw Error(E_STATE, "volume has not been built");
  if (dims3) memcpy(dims3, v->mcDims, sizeof v->mcDims);
  v->ctx->activate();
  if (rangesOut) ck(cudaMemcpyAsync(rangesOut, v->ranges.ptr, v->ranges.bytes, cudaMemcpyDefault, v->ctx->stream), "copy");
  if (majOut) ck(cudaMemcpyAsync(majOut, v->majorants.ptr, v->majorants.bytes, cudaMemcpyDefault, v->ctx->stream), "copy");
  ck(cudaStreamSynchronize(v->ctx->stream), "copy");
  BN_CATCH()
}

BN_API void bnxVolumeSample(BNVolume vh, const float *points, int n, float *scalarsOut, float *rgbaOut,
                            int fastMath) {
  BN_TRY
  auto v = getAs<Volume>(vh, Object::K_VOLUME, "BNVolume");
  if (n < 0 || (n > 0 && (!points || !scalarsOut || !rgbaOut)))
    throw Error(E_INVALID_ARG, "bnxVolumeSample needs n >= 0 and, for n > 0, points and both outputs");
  if (!v->built) throw Error(E_STATE, "volume has not been built");
  if (n == 0) return;
  v->ctx->activate();
  v->build();  // no-op unless the TF changed
  const VolumeDD dd = v->dd();
  const size_t un = (size_t)n;
  DeviceBuffer dP, dS, dR;
  dP.resize(un * sizeof(float3));
  dS.resize(un * sizeof(float));
  dR.resize(un * sizeof(float4));
  cudaStream_t s = v->ctx->stream;
  ck(cudaMemcpyAsync(dP.ptr, points, un * sizeof(float3), cudaMemcpyDefault, s), "sample points");
  // principled volumes render with the exact kernels only, so they sample with them here too
  const bool fast = fastMath && !dd.pv.enabled;
  ck((fast ? fastmath::launchSampleProbe : launchSampleProbe)(dd, (const float3 *)dP.ptr, n, (float *)dS.ptr,
                                                              (float4 *)dR.ptr, s),
     "sample kernel");
  ck(cudaMemcpyAsync(scalarsOut, dS.ptr, un * sizeof(float), cudaMemcpyDefault, s), "sample read");
  ck(cudaMemcpyAsync(rgbaOut, dR.ptr, un * sizeof(float4), cudaMemcpyDefault, s), "sample read");
  ck(cudaStreamSynchronize(s), "sample");
  BN_CATCH()
}

BN_API int bnxRenderStructuredNoAlloc(const BNXNoAllocFrame *f, void *stream) {
  BN_TRY
  if (!f) throw Error(E_INVALID_ARG, "frame description is null");
  int type;
  switch ((int)f->voxelType) {
  case BN_FLOAT32: type = VOX_F32; break;
  case BN_UFIXED8:
  case BN_UINT8: type = VOX_U8; break;
  case BNX_FLOAT16: type = VOX_F16; break;
  case BNX_BFLOAT16: type = VOX_BF16; break;
  case BN_UFIXED16: type = VOX_U16; break;
  default: throw Error(E_UNSUPPORTED, "unsupported voxel type");
  }
  int fmt = f->colorFormat == BN_FLOAT4 ? FMT_FLOAT4 : f->colorFormat == BN_UFIXED8_RGBA ? FMT_RGBA8
          : f->colorFormat == BN_UFIXED8_RGBA_SRGB ? FMT_RGBA8_SRGB : -1;
  if (fmt < 0) throw Error(E_UNSUPPORTED, "unsupported colour format");
  if (!f->voxels || !f->transferFunction || !f->accum || !f->color)
    throw Error(E_INVALID_ARG, "voxels, transferFunction, accum and color must be device pointers");
  for (int a = 0; a < 3; a++)
    if (f->dims[a] < 2) throw Error(E_INVALID_ARG, "every grid dimension must be >= 2");
  if (f->numTFValues < 2 || f->numTFValues > kMaxTF) throw Error(E_INVALID_ARG, "numTFValues must be in [2, 4096]");
  if (f->width <= 0 || f->height <= 0 || f->pathsPerPixel <= 0 || f->accumID < 0)
    throw Error(E_INVALID_ARG, "width, height and pathsPerPixel must be positive, accumID >= 0");
  if ((long long)f->width * f->height > kMaxFramePixels)
    throw Error(E_INVALID_ARG, "frame larger than 2^31 - 1 pixels");
  if (f->numDirLights < 0 || f->numDirLights > kMaxDirLights || (f->numDirLights && !f->dirLights))
    throw Error(E_INVALID_ARG, "numDirLights must be in [0, 16] with a host array of lights");
  int mc[3];
  for (int a = 0; a < 3; a++) mc[a] = (f->dims[a] - 1 + kCellsPerMC - 1) / kCellsPerMC;
  const long long nMC = (long long)mc[0] * mc[1] * mc[2];
  if (nMC > kNoAllocMaxMacrocells)
    throw Error(E_INVALID_ARG, "volume needs " + std::to_string(nMC) +
                                   " macrocells; the no-allocation entry point holds at most " +
                                   std::to_string((long long)kNoAllocMaxMacrocells) + " (a 513^3 grid)");
  VolumeDD v{};
  v.hasVolume = 1;
  const v3 org = {f->gridOrigin.x, f->gridOrigin.y, f->gridOrigin.z};
  const v3 spc = {f->gridSpacing.x, f->gridSpacing.y, f->gridSpacing.z};
  v.voxels = f->voxels;
  v.type = type;
  v.numScalars = make_int3(f->dims[0], f->dims[1], f->dims[2]);
  v.numCells = make_int3(f->dims[0] - 1, f->dims[1] - 1, f->dims[2] - 1);
  v.gridOrigin = F3(org);
  v.rcpSpacing = make_float3(1.f / spc.x, 1.f / spc.y, 1.f / spc.z);
  v.boundsLo = F3(org);
  v.boundsHi = make_float3(org.x + spc.x * (float)v.numCells.x, org.y + spc.y * (float)v.numCells.y,
                           org.z + spc.z * (float)v.numCells.z);
  v.majorants = nullptr;  // set to the static scratch by the launcher
  v.mcDims = make_int3(mc[0], mc[1], mc[2]);
  v.mcOrigin = F3(org);
  v.rcpMcSpacing = make_float3(1.f / (8.f * spc.x), 1.f / (8.f * spc.y), 1.f / (8.f * spc.z));
  v.tf = (const float4 *)f->transferFunction;
  v.tfN = f->numTFValues;
  v.domLo = f->domain.x;
  v.domHi = f->domain.y;
  v.baseDensity = f->densityAt1;
  v.phase = f->hgPhase ? PHASE_HG : PHASE_SIMPLE;
  v.anisotropy = std::min(0.99f, std::max(-0.99f, f->anisotropy));
  v.scatteringAlbedo = std::min(1.f, std::max(0.f, f->scatteringAlbedo));
  Camera cam(nullptr);
  cam.set3f("position", f->cameraPosition.x, f->cameraPosition.y, f->cameraPosition.z);
  cam.set3f("direction", f->cameraDirection.x, f->cameraDirection.y, f->cameraDirection.z);
  cam.set3f("up", f->cameraUp.x, f->cameraUp.y, f->cameraUp.z);
  cam.set1f("fovy", f->fovy);
  cam.commit();
  FrameDD fr{};
  fr.dir00 = F3(cam.dir00);
  fr.dirdu = F3(cam.dirdu);
  fr.dirdv = F3(cam.dirdv);
  fr.lens00 = F3(cam.lens00);
  fr.width = f->width;
  fr.height = f->height;
  fr.aspect = (float)fr.width / (float)fr.height;
  fr.bgColor = make_float4(f->bgColor.x, f->bgColor.y, f->bgColor.z, f->bgColor.w);
  fr.ambientRadiance = f->ambientRadiance;
  fr.cutPlane = make_float4(0.f, 0.f, 0.f, -1e30f);
  fr.numDirLights = f->numDirLights;
  for (int i = 0; i < f->numDirLights; i++) {
    const float *L = f->dirLights + 7 * i;
    DirLight l(nullptr);
    l.set3f("direction", L[0], L[1], L[2]);
    l.set1f("radiance", L[3]);
    l.set3f("color", L[4], L[5], L[6]);
    fr.dirLights[i] = l.dd();
  }
  fr.dirLightPick = fr.numDirLights > 0 ? 2.f / (float)fr.numDirLights : 0.f;
  fr.accum = (float4 *)f->accum;
  fr.accumID0 = f->accumID;
  fr.spp = f->pathsPerPixel;
  ck(launchRenderNoAlloc(v, fr, fmt, f->color, 0, (cudaStream_t)stream), "no-allocation render");
  return 0;
  BN_CATCH(g_lastError)
}

BN_API void bnxInjectAllocationFailure(int afterAllocations) {
  allocFailCountdown().store(afterAllocations < 0 ? -1 : afterAllocations);
}

BN_API long long bnxBoundsViolations(BNContext context) {
  BN_TRY
  if (!boundsCheckedBuild()) return -1;  // the normal build has no checks
  getContext(context)->activate();
  return readBoundsViolations();
  BN_CATCH(-2)
}

BN_API void bnxSetRegrouping(BNContext context, int enable) {
  BN_TRY
  getContext(context)->sched.regrouped = enable ? 1 : 0;
  BN_CATCH()
}

BN_API void bnxSetScheduling(BNContext context, int serviceBatch) {
  BN_TRY
  Context *c = getContext(context);
  if (serviceBatch < 1 || serviceBatch > 32) throw Error(E_INVALID_ARG, "serviceBatch must lie in [1, 32]");
  c->sched.serviceBatch = serviceBatch;
  BN_CATCH()
}

static std::vector<BatchEntry> batchEntries(const BNXRenderJob *jobs, int n) {
  if (n < 0 || (n && !jobs)) throw Error(E_INVALID_ARG, "invalid job array");
  std::vector<BatchEntry> e;
  std::vector<ObjectSP> keep;
  for (int i = 0; i < n; i++) {
    auto r = getAs<Renderer>(jobs[i].renderer, Object::K_RENDERER, "BNRenderer");
    auto m = getAs<Model>(jobs[i].model, Object::K_MODEL, "BNModel");
    auto c = getAs<Camera>(jobs[i].camera, Object::K_CAMERA, "BNCamera");
    auto fb = getAs<FrameBuffer>(jobs[i].frameBuffer, Object::K_FB, "BNFrameBuffer");
    for (auto &p : e)
      if (p.fb == fb.get()) throw Error(E_INVALID_ARG, "a frame buffer appears twice in one batch");
    e.push_back({r.get(), m.get(), c.get(), fb.get()});
  }
  return e;
}

BN_API void bnxRenderBatch(BNContext context, const BNXRenderJob *jobs, int numJobs) {
  BN_TRY
  Context *c = getContext(context);
  c->activate();
  renderBatch(c, batchEntries(jobs, numJobs));
  BN_CATCH()
}

BN_API void bnxSetPixelPartition(BNContext context, int rank, int count) {
  BN_TRY
  Context *c = getContext(context);
  if (count < 1 || rank < 0 || rank >= count) throw Error(E_INVALID_ARG, "need 0 <= rank < count");
  c->partRank = rank;
  c->partCount = count;
  BN_CATCH()
}

BN_API void bnxPixelPartitionOwners(int width, int height, int count, int *owners) {
  BN_TRY
  if (width <= 0 || height <= 0 || count < 1 || !owners) throw Error(E_INVALID_ARG, "bad partition query");
  // pixel order of the render kernel: 4-row bands, column-major inside a
  // band, 32 pixels per chunk, kPartTileChunks chunks per tile
  for (int iy = 0; iy < height; iy++) {
    const int band = iy / 4;
    const int rows = std::min(4, height - 4 * band);
    for (int ix = 0; ix < width; ix++) {
      const long long w = (long long)band * 4 * width + (long long)ix * rows + (iy - 4 * band);
      owners[(size_t)iy * width + ix] = (int)((w / 32 / kPartTileChunks) % count);
    }
  }
  BN_CATCH()
}

BN_API void bnxSetRenderTimeout(BNContext context, int milliseconds) {
  BN_TRY
  if (milliseconds < 0) throw Error(E_INVALID_ARG, "timeout must be >= 0");
  getContext(context)->timeoutMs = milliseconds;
  BN_CATCH()
}

BN_API void bnxSetBatchGraphs(BNContext context, int enable) {
  BN_TRY
  getContext(context)->useGraphs = enable != 0;
  BN_CATCH()
}

BN_API void bnxAutotuneBatch(BNContext context, const BNXRenderJob *jobs, int numJobs, BNXLaunchConfig *best) {
  BN_TRY
  Context *c = getContext(context);
  c->activate();
  std::vector<BatchEntry> e = batchEntries(jobs, numJobs);
  std::vector<uint32_t> saved;
  for (auto &x : e) saved.push_back(x.fb->accumID);
  // blocks per SM: 0, the occupancy of the kernel the batch runs
  struct Cand { int tpb, bps, service; };
  std::vector<Cand> cands;
  for (int tpb : {64, 128})
    for (int service : {4, 8, 12, 16, 20, 24, 28})
      cands.push_back({tpb, 0, service});
  Cand bestC{c->threadsPerBlock, c->blocksPerSM, c->sched.serviceBatch};
  float bestMs = 1e30f;
  for (const Cand &k : cands) {
    c->threadsPerBlock = k.tpb;
    c->blocksPerSM = k.bps;
    c->sched.serviceBatch = k.service;
    for (size_t i = 0; i < e.size(); i++) e[i].fb->accumID = saved[i];
    renderBatch(c, e);
    if (c->stats.renderMs < bestMs) { bestMs = c->stats.renderMs; bestC = k; }
  }
  c->threadsPerBlock = bestC.tpb;
  c->blocksPerSM = bestC.bps;
  c->sched.serviceBatch = bestC.service;
  for (auto &x : e) x.fb->accumID = 0;  // tuning frames are discarded
  if (best) *best = {bestC.tpb, bestC.bps, bestC.service, bestMs};
  BN_CATCH()
}

// ---------------------------------------------------------------------------
// ANARI parameter mapping (barney/anari/SpatialField.cpp:70-157,
// barney/anari/Volume.cpp:82-234): what the ANARI device does before it
// calls the native API, restated so an ANARI front-end can be layered on
// these entry points.
// ---------------------------------------------------------------------------
BN_API int bnxAnariTransferFunction1D(const float *colors, int numColorsIn, int colorChannels,
                                      const float *opacities, int numOpacitiesIn, bn_float4 uniformColor,
                                      float uniformOpacity, bn_float4 *out) {
  BN_TRY
  if (colors && colorChannels != 3 && colorChannels != 4) throw Error(E_INVALID_ARG, "colorChannels must be 3 or 4");
  if ((colors && numColorsIn < 1) || (opacities && numOpacitiesIn < 1)) throw Error(E_INVALID_ARG, "empty array");
  const int numColors = colors ? numColorsIn : 1;
  const int numOpacities = opacities ? numOpacitiesIn : 1;
  const int tfSize = std::max(numColors, numOpacities);
  if (!out) return tfSize;
  // Volume.cpp:166-167: m_uniformOpacity = opacity * color.w
  const float uOpacity = uniformOpacity * uniformColor.w;
  for (int i = 0; i < tfSize; ++i) {
    const float colorPos = tfSize > 1 ? (float(i) / (tfSize - 1)) * (numColors - 1) : 0.f;
    const float colorFrac = colorPos - floorf(colorPos);
    float c0[4] = {uniformColor.x, uniformColor.y, uniformColor.z, uOpacity};
    float c1[4] = {uniformColor.x, uniformColor.y, uniformColor.z, uOpacity};
    if (colors) {
      const int i0 = int(floorf(colorPos)), i1 = int(ceilf(colorPos));
      for (int c = 0; c < 3; c++) {
        c0[c] = colors[colorChannels * i0 + c];
        c1[c] = colors[colorChannels * i1 + c];
      }
      if (colorChannels == 4) {
        c0[3] = colors[4 * i0 + 3];
        c1[3] = colors[4 * i1 + 3];
      }
    }
    float color[4];
    for (int c = 0; c < 4; c++) color[c] = (1.f - colorFrac) * c0[c] + colorFrac * c1[c];
    if (opacities) {
      const float alphaPos = tfSize > 1 ? (float(i) / (tfSize - 1)) * (numOpacities - 1) : 0.f;
      const float alphaFrac = alphaPos - floorf(alphaPos);
      const float a0 = opacities[int(floorf(alphaPos))];
      const float a1 = opacities[int(ceilf(alphaPos))];
      color[3] *= (1.f - alphaFrac) * a0 + alphaFrac * a1;
    }
    out[i] = {color[0], color[1], color[2], color[3]};
  }
  return tfSize;
  BN_CATCH(-1)
}

BN_API float bnxAnariDensityScale(float unitDistance) {
  return unitDistance <= 0.f ? 1.f : 1.f / unitDistance;  // Volume.cpp:99-107
}

BN_API BNScalarField bnxAnariStructuredRegular(BNContext context, int slot, BNDataType elementType, const void *data,
                                               int nx, int ny, int nz, bn_float3 origin, bn_float3 spacing) {
  BN_TRY
  BNDataType bt;
  switch ((int)elementType) {  // SpatialField.cpp:106-116: float32, or ufixed8 / uint8
  case BN_FLOAT32: bt = BN_FLOAT32; break;
  case BN_UFIXED8:
  case BN_UINT8: bt = BN_UFIXED8; break;
  default: throw Error(E_UNSUPPORTED, "structuredRegular supports float32 and uint8 / ufixed8 data");
  }
  BNScalarField sf = bnScalarFieldCreate(context, slot, "structured");
  if (!sf) return nullptr;
  BNTextureData td = bnTextureData3DCreate(context, slot, bt, nx, ny, nz, data);
  if (!td) { bnRelease(sf); return nullptr; }
  bnSetObject(sf, "textureData", td);
  bnRelease(td);  // the field keeps its own reference (SpatialField.cpp:122)
  bnSet3i(sf, "dims", nx, ny, nz);
  bnSet3f(sf, "gridOrigin", origin.x, origin.y, origin.z);
  bnSet3f(sf, "gridSpacing", spacing.x, spacing.y, spacing.z);
  bnCommit(sf);
  if (g_lastError) return nullptr;
  return sf;
  BN_CATCH(nullptr)
}

// Renderer::commitParameters, barney/anari/Renderer.cpp:22-37: each
// parameter the application did not set takes the ANARI device's default.
BN_API void bnxAnariRendererParams(const BNXAnariRenderer *in, BNXAnariRenderer *out) {
  BN_TRY
  if (!out) throw Error(E_INVALID_ARG, "bnxAnariRendererParams: out is NULL");
  BNXAnariRenderer d{};
  const unsigned set = in ? in->set : 0u;
  d.pixelSamples = (set & BNX_ANARI_PIXEL_SAMPLES) ? in->pixelSamples : 1;
  d.ambientRadiance = (set & BNX_ANARI_AMBIENT_RADIANCE) ? in->ambientRadiance : 1.f;
  d.background = (set & BNX_ANARI_BACKGROUND) ? in->background : bn_float4{0.f, 0.f, 0.f, 1.f};
  d.cutPlane = (set & BNX_ANARI_CUT_PLANE) ? in->cutPlane : bn_float4{0.f, 0.f, 0.f, 0.f};
  d.maxVolumeBounces = (set & BNX_ANARI_MAX_VOLUME_BOUNCES) ? in->maxVolumeBounces : 0;
  d.crosshairs = (set & BNX_ANARI_CROSSHAIRS) ? (in->crosshairs ? 1 : 0) : 0;
  d.set = BNX_ANARI_PIXEL_SAMPLES | BNX_ANARI_AMBIENT_RADIANCE | BNX_ANARI_BACKGROUND | BNX_ANARI_CUT_PLANE |
          BNX_ANARI_MAX_VOLUME_BOUNCES | BNX_ANARI_CROSSHAIRS;
  *out = d;
  BN_CATCH()
}

// Renderer::finalize, barney/anari/Renderer.cpp:40-51 (the background image
// and the denoiser flags are not mapped: textures and the denoiser are not
// built)
BN_API void bnxAnariRendererCommit(BNRenderer renderer, const BNXAnariRenderer *params) {
  BN_TRY
  getAs<Renderer>(renderer, Object::K_RENDERER, "BNRenderer");
  BNXAnariRenderer p;
  bnxAnariRendererParams(params, &p);
  bnSet4f(renderer, "bgColor", p.background.x, p.background.y, p.background.z, p.background.w);
  bnSet1i(renderer, "crosshairs", p.crosshairs);
  bnSet1i(renderer, "pathsPerPixel", p.pixelSamples);
  bnSet1f(renderer, "ambientRadiance", p.ambientRadiance);
  bnSet1i(renderer, "maxVolumeBounces", p.maxVolumeBounces);
  bnSet4f(renderer, "cutPlane", p.cutPlane.x, p.cutPlane.y, p.cutPlane.z, p.cutPlane.w);
  if (g_lastError) return;
  bnCommit(renderer);
  BN_CATCH()
}

// Frame::renderFrame, barney/anari/Frame.cpp:172-178 and 226-261: a frame
// after any object finalization (here: any commit or build of the context)
// starts its accumulation over
BN_API void bnxAnariRenderFrame(BNRenderer renderer, BNModel model, BNCamera camera, BNFrameBuffer frameBuffer) {
  BN_TRY
  auto fb = getAs<FrameBuffer>(frameBuffer, Object::K_FB, "BNFrameBuffer");
  if (fb->anariFrameEpoch != fb->ctx->commitEpoch) {
    fb->accumID = 0;
    fb->anariFrameEpoch = fb->ctx->commitEpoch;
  }
  bnRender(renderer, model, camera, frameBuffer);
  BN_CATCH()
}

}  // extern "C"
