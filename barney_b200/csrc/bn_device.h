// bn_device.h -- data handed from the host object model (bn_api.cpp) to the
// sm_100a kernels (bn_kernels.cu).  Plain structs passed by value as kernel
// parameters; all pointers are device pointers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bnb {

enum VoxelType : int { VOX_F32 = 0, VOX_U8 = 1, VOX_F16 = 2, VOX_BF16 = 3, VOX_U16 = 4 };
enum PhaseMode : int { PHASE_SIMPLE = 0, PHASE_HG = 1 };
enum ColorFormat : int { FMT_FLOAT4 = 0, FMT_RGBA8 = 1, FMT_RGBA8_SRGB = 2 };
enum ErrorBits : unsigned { ERR_ITER_CAP = 1u, ERR_ABORTED = 2u };

constexpr int kMaxDirLights = 16;
constexpr int kMaxTF = 4096;
constexpr int kCellsPerMC = 8;  // StructuredData.cu:26
constexpr long long kMaxFramePixels = 0x7fffffffLL;  // pixels of one frame (32-bit pixel / chunk indices)
constexpr int kPartTileChunks = 32;    // pixel-tile partition: 32 chunks of 32 pixels per tile
constexpr int kRenderMaxThreads = 128;  // __launch_bounds__ of the render kernels:
constexpr int kRenderMinBlocks = 7;     // plain: 7 x 128 threads per SM (at most 73 registers)
constexpr int kRenderMinBlocksMixedComp = 6;  // plain, compensated sums tested per job (mixed batches):
                                              // 6 x 128 (85; at 7 they spill up to 348 B)
constexpr int kRenderMinBlocksExt = 5;  // extended (multi-scatter, principled): 5 x 128 (102)
constexpr int kRenderMinBlocksIso = 4;  // extended with isosurfaces: 4 x 128 (128; with the warp-cooperative
                                        // iso scan 3 % faster than 5 x 128, which spilled up to 820 B)

// Principled volume coefficients evaluated from the field value
// (PrincipledVolumeParams::DD, PrincipledVolume.h:33-46).
struct PrincipledDD {
  int enabled;
  float density, densityThreshold, densityScale, valueLo, valueHi;
  float emissionStrength, blackbodyIntensity, temperature;
  float3 scatterColor, absorptionColor, emissionColor, blackbodyTint;
};

// isoSurface geometry on the field (MCIsoSurfaceAccel::DD,
// MCAccelerator.h:75-123) with an AnariMatte material of constant colour and
// opacity (AnariMatte.h:49-71).
struct IsoDD {
  int enabled;
  float isoValue;
  const float2 *ranges;  // macrocell scalar ranges (lo, hi) of the field, mcDims cells
  float3 albedo;         // Lambertian albedo: .85 * color * (1/pi)
  float alpha;           // color.w * opacity: below 1 a ray passes the surface with probability 1 - alpha
  float normalDelta;     // central-difference step of the normal: |bounds size| * .1 / (mcDims.x + .y + .z)
};

// Structured field + macrocell majorant grid + transfer function
// (MCVolumeAccel::DD, MCAccelerator.h:23-27).
struct VolumeDD {
  const void *voxels;   // x-fastest scalars, numScalars.x * .y * .z
  int type;             // VoxelType
  int3 numScalars;      // texture dims
  int3 numCells;        // numScalars - 1
  float3 gridOrigin;
  float3 rcpSpacing;    // 1/gridSpacing (IEEE)
  float3 boundsLo, boundsHi;
  const float *majorants;
  const unsigned *mcOccupied;  // bit (i & 31) of word i >> 5 set iff majorants[i] != 0
  int3 mcDims;
  float3 mcOrigin;
  float3 rcpMcSpacing;  // 1/(8*gridSpacing)
  const float4 *tf;     // tfN entries
  int tfN;
  float domLo, domHi;
  float baseDensity;
  int phase;            // PhaseMode
  float anisotropy;
  float scatteringAlbedo;
  PrincipledDD pv;
  int hasVolume;        // 0: the group holds an isosurface on this field and no volume
  IsoDD iso;
};

struct DirLightDD {
  float3 toLight;       // -normalize(direction)  (DirLight.cu:11-20, shadeRays.cu:180)
  float radiance;
  float3 color;
};

// One frame's worth of render parameters (Camera::DD, Renderer::DD,
// World::DD lights, frame buffer).
struct FrameDD {
  float3 dir00, dirdu, dirdv, lens00;   // PerspectiveCamera::commit, Camera.cu:82-100
  int width, height;
  float aspect;          // width / (float)height, the one IEEE quotient _generateRays forms per ray
  float4 bgColor;
  float ambientRadiance;
  float4 cutPlane;
  int numDirLights;
  float dirLightPick;    // 2.f / float(numDirLights) (shadeRays.cu's reservoir of two), 0 without lights
  DirLightDD dirLights[kMaxDirLights];
  int emissionAbsorption;
  int exactLog;
  int fastMath;          // the job asks for the fast-math kernels (host-side choice; kernels ignore it)
  int maxVolumeBounces;  // > 0: multi-scatter build (HG phase), scattered rays up to this many volume bounces
  int partRank, partCount;  // pixel-tile partition: render the tiles t with t % partCount == partRank
  float4 *accum;        // width*height, linear
  float4 *comp;         // width*height Neumaier compensation terms, or null (plain sums)
  int accumID0;         // accumID of the first wave of this launch
  int spp;              // waves in this launch
  void *color;          // resolved output (batch resolve only)
  int colorFormat;      // ColorFormat of color
};

// One render job: a volume and a frame.  The single-frame kernel takes it
// as a parameter; the batch kernel reads a table of them from HBM.
struct JobDD {
  VolumeDD v;
  FrameDD fr;
};

// Warp scheduling of the render loop: a warp keeps stepping macrocells and
// Woodcock ranges until at least serviceBatch of its lanes (or all of its
// busy lanes) need service -- shading, accumulation, a new ray -- and then
// serves them together.
struct SchedDD {
  int serviceBatch = 22;
  int regrouped = 0;  // plain single-frame jobs: the regrouped kernel (launchRenderRegrouped) instead of renderLoop's
};

// Device counters of one launch (samples, mcVisits, rays, errorFlags)
struct LaunchCounters {
  unsigned long long samples, mcVisits, rays, errorFlags;
  unsigned int nextPixel;   // work counter of the persistent render kernel
  unsigned int abort;       // host-set abort request
};

// launchers (bn_kernels.cu).  Both majorant launchers also write the
// occupancy bitmap of the new majorants, ceil(n/32) words; with majorants
// null, launchBuildMacrocells writes the scalar ranges only.
cudaError_t launchBuildMacrocells(const VolumeDD &vol, float2 *ranges, float *majorants, unsigned *occupied,
                                  int roundUp, cudaStream_t s);
cudaError_t launchMapMajorants(const VolumeDD &vol, const float2 *ranges, float *majorants, unsigned *occupied,
                               int roundUp, cudaStream_t s);
cudaError_t launchRender(const VolumeDD &vol, const FrameDD &frame, LaunchCounters *counters, int blocksPerSM,
                         int threadsPerBlock, cudaStream_t s, const SchedDD &sd = SchedDD());
// jobs / chunkStart: device arrays; chunkStart has numJobs+1 entries, the
// prefix sum of each job's ceil(width*height/32) pixel chunks.
// extended: 2 if some job has an isosurface and some job volume bounces
// (fr.maxVolumeBounces > 0) or a principled volume, 3 if some job has an
// isosurface and none has either, else 1 if some job has volume bounces, a
// principled volume or exact-log free flight, else 0 (selects the kernel
// instantiation that implements them); voxelType: the
// VoxelType all jobs share (a kernel compiled for it) or -1 (mixed);
// compensated: how many jobs carry compensation terms (fr.comp): 0 none,
// 1 some, 2 all
cudaError_t launchRenderBatch(const JobDD *jobs, const int *chunkStart, int numJobs, LaunchCounters *counters,
                              int blocksPerSM, int threadsPerBlock, cudaStream_t s, const SchedDD &sd = SchedDD(),
                              int extended = 0, int voxelType = -1, int compensated = 1);
// The same for at most kParamJobs plain jobs (extended 0) whose table and
// chunk prefix are in host memory: passed as one kernel parameter.  Not for
// stream capture (the parameter would be frozen into the graph).
constexpr int kParamJobs = 32;
cudaError_t launchRenderBatchParams(const JobDD *hostJobs, const int *hostChunkStart, int numJobs,
                                    LaunchCounters *counters, int blocksPerSM, int threadsPerBlock, cudaStream_t s,
                                    const SchedDD &sd, int voxelType, int compensated);
cudaError_t launchResolve(const float4 *accum, int numPixels, int accumID, int fmt, void *out, cudaStream_t s,
                          const float4 *comp = nullptr);
// resolves every job of a batch table into its fr.color after its waves
cudaError_t launchResolveBatch(const JobDD *jobs, const int *chunkStart, int numJobs, int numChunks, cudaStream_t s);
// out-of-range accesses counted by the bounds-checked build since the last
// call (then reset); -1 in the normal build, -2 on a CUDA error
long long readBoundsViolations();
bool boundsCheckedBuild();

// No-allocation render: majorant grid, occupancy bitmap and counters in a
// static device array sized for kNoAllocMaxMacrocells macrocells (see
// bn_kernels.cu).
constexpr int64_t kNoAllocMaxMacrocells = 64 * 64 * 64;
cudaError_t launchRenderNoAlloc(VolumeDD v, FrameDD fr, int fmt, void *color, int roundUp, cudaStream_t s);

// The regrouped render kernel for a plain single-frame job (no isosurface,
// multi-scatter or principled volume; cudaErrorInvalidValue otherwise): the
// same frame and counters as launchRender, pixel slots advanced by
// phase-compacted lists in shared memory.  Launch shape from the occupancy.
cudaError_t launchRenderRegrouped(const VolumeDD &vol, const FrameDD &frame, LaunchCounters *counters, cudaStream_t s);

// Field samples and TF lookups (sampleAndMap) at n device points P into
// device arrays scalar (NaN outside the field) and rgba.
cudaError_t launchSampleProbe(const VolumeDD &vol, const float3 *P, int n, float *scalar, float4 *rgba, cudaStream_t s);

// The fast-math form (renderer parameter bnx.fastMath): the plain kernels
// (no isosurface, multi-scatter or principled volume) compiled with FMA
// contraction and approximate division and square root, except where a
// sample's texel coordinate and TF coordinate are formed (explicitly
// rounded there).  Same launch semantics as the exact launchers; a job that
// needs an extended kernel returns cudaErrorInvalidValue.
namespace fastmath {
cudaError_t launchRender(const VolumeDD &vol, const FrameDD &frame, LaunchCounters *counters, int blocksPerSM,
                         int threadsPerBlock, cudaStream_t s, const SchedDD &sd = SchedDD());
cudaError_t launchRenderBatch(const JobDD *jobs, const int *chunkStart, int numJobs, LaunchCounters *counters,
                              int blocksPerSM, int threadsPerBlock, cudaStream_t s, const SchedDD &sd = SchedDD(),
                              int extended = 0, int voxelType = -1, int compensated = 1);
cudaError_t launchRenderBatchParams(const JobDD *hostJobs, const int *hostChunkStart, int numJobs,
                                    LaunchCounters *counters, int blocksPerSM, int threadsPerBlock, cudaStream_t s,
                                    const SchedDD &sd, int voxelType, int compensated);
cudaError_t launchSampleProbe(const VolumeDD &vol, const float3 *P, int n, float *scalar, float4 *rgba, cudaStream_t s);
cudaError_t launchRenderRegrouped(const VolumeDD &vol, const FrameDD &frame, LaunchCounters *counters, cudaStream_t s);
long long readBoundsViolationsHere();  // bounds-checked build only
}  // namespace fastmath
long long readBoundsViolationsHere();  // bounds-checked build only

}  // namespace bnb
