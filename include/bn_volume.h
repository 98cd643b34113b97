/* bn_volume.h -- C ABI of barney_b200, a B200-native (sm_100a) replacement
 * for Barney's structured-volume path-tracing path.
 *
 * The bn* entry points below have the names, argument meanings and call
 * order of Barney's native API (barney/native/include/barney.h, where they
 * are C++ functions in namespace BARNEY_NS, deliberately not extern "C",
 * implemented in barney/native/barney.cu).  Here they are plain extern "C"
 * symbols over opaque handles, so any FFI (ctypes, cgo, JNI, N-API) or a C++
 * namespace shim (include/barney_shim.hpp) can bind them.  Each declaration
 * cites the reference entry point it replaces.
 *
 * Scope: one GPU; scalar fields of type "structured" (float32 / unorm8, plus
 * the float16 / bfloat16 storage forms added here); one volume per group,
 * identity instance transforms; pinhole ("perspective") camera; constant
 * environment (ambientRadiance) and "directional" lights; colour channel of
 * the frame buffer.  Anything else is rejected with an error.
 *
 * Errors: the reference throws C++ exceptions through its API
 * (barney.cu:23-37).  No exception crosses this ABI: every entry point
 * catches, records a thread-local error (bnGetLastError /
 * bnGetLastErrorString) and returns (0 / NULL for constructors).
 *
 * Threading: as in the reference, calls are expected from one thread per
 * context; bnRender is synchronous (returns after the frame is resolved).
 */
#ifndef BN_VOLUME_H
#define BN_VOLUME_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define BN_API __attribute__((visibility("default")))
#else
#define BN_API
#endif

typedef struct _BNContext *BNContext;
typedef struct _BNObject *BNObject;
typedef BNObject BNData;
typedef BNObject BNTextureData;
typedef BNObject BNScalarField;
typedef BNObject BNGeom;
typedef BNObject BNMaterial;
typedef BNObject BNSampler;
typedef BNObject BNTexture2D;
typedef BNObject BNTexture3D;
typedef BNObject BNVolume;
typedef BNObject BNGroup;
typedef BNObject BNModel;
typedef BNObject BNRenderer;
typedef BNObject BNFrameBuffer;
typedef BNObject BNLight;
typedef BNObject BNCamera;

typedef struct { float x, y; } bn_float2;
typedef struct { float x, y, z; } bn_float3;
typedef struct { float x, y, z, w; } bn_float4;

/* barney.h BNTransform: 3x3 linear part (columns vx, vy, vz) + translation */
typedef struct {
  struct { bn_float3 vx, vy, vz; } l;
  bn_float3 p;
} BNTransform;

/* barney.h BNFrameBufferChannel (values kept) */
typedef enum {
  BN_FB_COLOR = (1 << 0),
  BN_FB_DEPTH = (1 << 1),
  BN_FB_PRIMID = (1 << 2),
  BN_FB_INSTID = (1 << 3),
  BN_FB_OBJID = (1 << 4),
  BN_FB_NORMAL = (1 << 5)
} BNFrameBufferChannel;

/* barney.h BNDataType (values kept; only the ones this path uses listed) */
typedef enum {
  BN_DATA_UNDEFINED = 0,
  BN_DATA = 1,
  BN_OBJECT = 2,
  BN_UINT8 = 110,
  BN_FLOAT32 = 180,
  BN_FLOAT32_VEC4 = 183,
  BN_FLOAT = BN_FLOAT32,
  BN_FLOAT4 = BN_FLOAT32_VEC4,
  BN_UFIXED8 = 300,
  BN_UFIXED8_RGBA = 301,
  BN_UFIXED8_RGBA_SRGB = 302,
  BN_UFIXED16 = 303,
  /* storage forms with no reference counterpart (precision path) */
  BNX_FLOAT16 = 1000,
  BNX_BFLOAT16 = 1001
} BNDataType;

/* ---------------------------------------------------------------------- */
/* context                                                                 */
/* ---------------------------------------------------------------------- */

/* replaces barney.cu:58 bnContextCreate. Exactly one data group and at most
   one GPU; gpuIDs may be NULL (device 0). */
BN_API BNContext bnContextCreate(int numDataGroupsOnThisContext, const int *dataRanksInDataGroup,
                                 int numGPUs, const int *gpuIDs);
/* replaces barney.cu bnContextDestroy: frees every object of the context */
BN_API void bnContextDestroy(BNContext context);
/* replaces barney.cu bnPhysicalDeviceCount */
BN_API int bnPhysicalDeviceCount(void);

/* ---------------------------------------------------------------------- */
/* object lifetime and parameters (barney.h "general set/commit")          */
/* ---------------------------------------------------------------------- */
/* replaces barney.cu bnRelease (Context.cpp:250-261): drops the app's reference */
BN_API void bnRelease(BNObject object);
/* replaces barney.cu bnAddReference */
BN_API void bnAddReference(BNObject object);
/* replaces barney.cu bnCommit (Object::commit) */
BN_API void bnCommit(BNObject target);
/* replace barney.cu bnSet{1,2,3,4}{i,f} (Object::set*) */
BN_API void bnSet1i(BNObject target, const char *paramName, int value);
BN_API void bnSet2i(BNObject target, const char *paramName, int x, int y);
BN_API void bnSet3i(BNObject target, const char *paramName, int x, int y, int z);
BN_API void bnSet4i(BNObject target, const char *paramName, int x, int y, int z, int w);
BN_API void bnSet1f(BNObject target, const char *paramName, float value);
BN_API void bnSet2f(BNObject target, const char *paramName, float x, float y);
BN_API void bnSet3f(BNObject target, const char *paramName, float x, float y, float z);
BN_API void bnSet4f(BNObject target, const char *paramName, float x, float y, float z, float w);
/* replaces barney.cu bnSetObject (StructuredData::setObject "textureData") */
BN_API void bnSetObject(BNObject target, const char *paramName, BNObject value);
/* replaces barney.cu bnSetData (Group "lights", Group.cpp:50-51) */
BN_API void bnSetData(BNObject target, const char *paramName, BNData value);
/* replace barney.cu:559 bnSetString, :654 bnSet4x3fv, :662 bnSet4x4fv: no
   object of this path has string or matrix parameters (sampler- or
   attribute-mapped material inputs are not supported); each records
   "unsupported parameter" */
BN_API void bnSetString(BNObject target, const char *paramName, const char *value);
BN_API void bnSet4x3fv(BNObject target, const char *paramName, const BNTransform *affineMatrix);
BN_API void bnSet4x4fv(BNObject target, const char *paramName, const bn_float4 *xfm);

/* ---------------------------------------------------------------------- */
/* scene content                                                           */
/* ---------------------------------------------------------------------- */
/* replaces barney.cu bnDataCreate (BN_OBJECT arrays of lights) */
BN_API BNData bnDataCreate(BNContext context, int whichSlot, BNDataType dataType, size_t numItems,
                           const void *items);
/* replaces barney.cu:498 bnDataSet: new contents of a BN_OBJECT array */
BN_API void bnDataSet(BNData data, size_t numItems, const void *items);
/* barney.h texture and sampler objects (barney.h:203-223 enums; barney.cu:205
   bnTextureData2DCreate, :242 bnTexture2DCreate, :272 bnTexture3DCreate, :417
   bnSamplerCreate) feed surface materials, which this path does not map:
   each returns NULL and records "unsupported" */
typedef enum { BN_TEXTURE_NEAREST, BN_TEXTURE_LINEAR } BNTextureFilterMode;
typedef enum { BN_TEXTURE_WRAP, BN_TEXTURE_CLAMP, BN_TEXTURE_BORDER, BN_TEXTURE_MIRROR } BNTextureAddressMode;
typedef enum { BN_COLOR_SPACE_LINEAR, BN_COLOR_SPACE_SRGB } BNTextureColorSpace;
BN_API BNTextureData bnTextureData2DCreate(BNContext context, int whichSlot, BNDataType texelFormat, int width,
                                           int height, const void *items);
BN_API BNTexture2D bnTexture2DCreate(BNContext context, int whichSlot, BNDataType texelFormat, uint32_t sizeX,
                                     uint32_t sizeY, const void *texels, BNTextureFilterMode filterMode,
                                     BNTextureAddressMode addressModeX, BNTextureAddressMode addressModeY,
                                     BNTextureColorSpace colorSpace);
BN_API BNTexture3D bnTexture3DCreate(BNContext context, int whichSlot, BNDataType texelFormat, uint32_t sizeX,
                                     uint32_t sizeY, uint32_t sizeZ, const void *texels,
                                     BNTextureFilterMode filterMode, BNTextureAddressMode addressMode);
BN_API BNSampler bnSamplerCreate(BNContext context, int whichSlot, const char *type);
/* replaces barney.cu:223 bnTextureData3DCreate. texelFormat: BN_FLOAT32,
   BN_UFIXED8 / BN_UINT8 (unorm, x/255), BN_UFIXED16 (unorm, x/65535),
   BNX_FLOAT16, BNX_BFLOAT16. texels may be host or device memory; it is
   copied before return. */
BN_API BNTextureData bnTextureData3DCreate(BNContext context, int whichSlot, BNDataType texelFormat,
                                           int width, int height, int depth, const void *texels);
/* replaces barney.cu:382 bnScalarFieldCreate; type must be "structured" */
BN_API BNScalarField bnScalarFieldCreate(BNContext context, int whichSlot, const char *type);
/* replaces barney.cu:457 bnVolumeCreate.  Parameters (Volume.cpp:36-126):
   anisotropy (clamped to +-0.99), scatteringAlbedo, and the principled
   volume set -- principledVolume (int), principledDensity,
   principledDensityThreshold, principledDensityScale,
   principledEmissionStrength, principledBlackbodyIntensity,
   principledTemperature, principledValueRange (float2),
   principledScatterColor, principledAbsorptionColor, principledEmissionColor,
   principledBlackbodyTint (float3); extension bnx.majorantRoundUp. */
BN_API BNVolume bnVolumeCreate(BNContext context, int whichSlot, BNScalarField sf);
/* replaces barney.cu:442 bnVolumeSetXF (Volume::setXF, Volume.cpp:15-24) */
BN_API void bnVolumeSetXF(BNVolume volume, bn_float2 domain, const bn_float4 *colorMap,
                          int numColorMapValues, float densityAt1);
/* replaces barney.cu bnLightCreate; type "directional" */
BN_API BNLight bnLightCreate(BNContext context, int whichSlot, const char *type);
/* replaces barney.cu:394 bnGeometryCreate (Geometry::create, Geometry.cpp:33);
   type "iso_surface" only (IsoSurface.cpp): bnSet1f "isoValue", bnSetObject
   "scalarField" (a structured field) and "material" (a committed material),
   bnSetData "isoValues" (kept, unused, as by the reference's intersection
   program).  With a volume in the same group the isosurface must lie on the
   volume's field. */
BN_API BNGeom bnGeometryCreate(BNContext context, int whichSlot, const char *type);
/* replaces barney.cu:405 bnMaterialCreate (HostMaterial::create); type "matte" /
   "AnariMatte" with constant parameters: bnSet3f / bnSet4f "color" (default
   .8,.8,.8), bnSet1f "opacity" (default 1) */
BN_API BNMaterial bnMaterialCreate(BNContext context, int whichSlot, const char *type);
/* replaces barney.cu:510 bnGroupCreate; at most one iso_surface geometry and at
   most one volume, at least one of the two */
BN_API BNGroup bnGroupCreate(BNContext context, int whichSlot, BNGeom *geoms, int numGeoms,
                             BNVolume *volumes, int numVolumes);
/* replaces barney.cu bnGroupBuild (Group::build -> MCVolumeAccel::build):
   macrocell ranges + majorants are built here */
BN_API void bnGroupBuild(BNGroup group);
/* replaces barney.cu bnModelCreate */
BN_API BNModel bnModelCreate(BNContext ctx);
/* replaces barney.cu bnSetInstances; one group, transform NULL or identity */
BN_API void bnSetInstances(BNModel model, int whichSlot, BNGroup *groups, BNTransform *xfms,
                           int numInstances);
/* replaces barney.cu:352 bnUpdateInstanceTransforms: the transforms of the
   instances bnSetInstances set, which must stay identity */
BN_API void bnUpdateInstanceTransforms(BNModel model, int whichSlot, BNTransform *instanceTransforms,
                                       int numInstances);
/* replaces barney.cu:323 bnSetInstanceAttributes: instance attributes are not
   read by this path; a NULL array is accepted, any other records
   "unsupported" */
BN_API void bnSetInstanceAttributes(BNModel model, int whichSlot, const char *attributeName, BNData data);
/* replaces barney.cu:542 bnBuild */
BN_API void bnBuild(BNModel model, int whichSlot);

/* ---------------------------------------------------------------------- */
/* camera, renderer, frame buffer                                          */
/* ---------------------------------------------------------------------- */
/* replaces barney.cu bnCameraCreate; type "perspective" (or "pinhole") */
BN_API BNCamera bnCameraCreate(BNContext context, const char *type);
/* replaces barney.cu bnRendererCreate; type "default" / "pathTracer".
   Parameters (Renderer.cpp:42-95): bgColor, ambientRadiance, pathsPerPixel,
   cutPlane, maxVolumeBounces; extensions bnx.hgPhase, bnx.emissionAbsorption,
   bnx.exactLog, bnx.compensatedAccum.  maxVolumeBounces acts only together
   with bnx.hgPhase, which selects Barney's multi-scatter build: scattered
   rays continue for up to that many volume bounces (path depth at most 10,
   shadeRays.cu:749-878).  Without it, a volume scatter ends the path, as in
   Barney's default build. */
BN_API BNRenderer bnRendererCreate(BNContext ctx, const char *type);
/* replaces barney.cu bnFrameBufferCreate */
BN_API BNFrameBuffer bnFrameBufferCreate(BNContext context, int deprecated);
/* replaces barney.cu bnFrameBufferResize (FrameBuffer::resize); colorFormat
   BN_FLOAT4, BN_UFIXED8_RGBA or BN_UFIXED8_RGBA_SRGB. Resets accumulation. */
BN_API void bnFrameBufferResize(BNFrameBuffer fb, BNDataType colorFormat, int sizeX, int sizeY,
                                uint32_t requiredChannels);
/* replaces barney.cu:696 bnFrameBufferRead (FrameBuffer::read); BN_FB_COLOR
   only; pointer may be host or device memory */
BN_API void bnFrameBufferRead(BNFrameBuffer fb, BNFrameBufferChannel channelToRead,
                              void *pointerToReadDataInto, BNDataType requiredFormat);
/* replaces barney.cu bnFrameBufferGetSize */
BN_API void bnFrameBufferGetSize(BNFrameBuffer fb, int *sizeX, int *sizeY);
/* replaces barney.cu:721 bnAccumReset */
BN_API void bnAccumReset(BNFrameBuffer fb);
/* replaces barney.cu:727 bnRender (Context::renderTiles, Context.cpp:139-182):
   renders renderer.pathsPerPixel waves and resolves the colour channel */
BN_API void bnRender(BNRenderer renderer, BNModel model, BNCamera camera, BNFrameBuffer fb);

/* ---------------------------------------------------------------------- */
/* errors (no reference counterpart: the reference throws)                 */
/* ---------------------------------------------------------------------- */
BN_API int bnGetLastError(void);
BN_API const char *bnGetLastErrorString(void);
BN_API void bnClearLastError(void);

/* ---------------------------------------------------------------------- */
/* bnx: extensions with no reference counterpart                           */
/* ---------------------------------------------------------------------- */
/* Work done by the last bnRender / batch on this context and the device
   time of its render kernel. */
typedef struct {
  unsigned long long samples;       /* volume samples (sampleAndMap calls) */
  unsigned long long mcVisits;      /* macrocells whose majorant was read */
  unsigned long long rays;          /* primary + shadow rays traced */
  unsigned long long pixelSamples;  /* pixels x waves */
  unsigned long long errorFlags;    /* iteration caps hit, aborts */
  float renderMs;                   /* device time of the render kernel(s) */
  float resolveMs;                  /* device time of the resolve kernel */
} BNXStats;
BN_API void bnxGetStats(BNContext context, BNXStats *stats);
/* Launch all work of the context on this CUDA stream (cudaStream_t); NULL
   selects the context's own stream. */
BN_API void bnxSetStream(BNContext context, void *cudaStream);
BN_API void *bnxGetStream(BNContext context);
/* Deadline of bnRender and bnxRenderBatch (0: none), counted from the call.
   When a frame is still running at the deadline, the render kernel is told
   to stop (every warp quits at its next pixel chunk), the frame buffer's
   accumulation is reset and the call records error 8 (timeout); the context
   stays usable.  A frame that has finished by the time the deadline is
   checked is kept. */
BN_API void bnxSetRenderTimeout(BNContext context, int milliseconds);
/* Pixel-tile data parallelism (the reference deals tiles round-robin across
   GPUs, TiledFB.cu:230-261): bnRender on this context renders only the tiles
   of 1024 pixels whose index modulo `count` is `rank` (count 1: all).  The
   other pixels of the frame buffer are left as they were; a frame is
   assembled from each rank's owned pixels, which bnxPixelPartitionOwners
   lists.  Per-pixel results equal an unpartitioned render.  Batches reject a
   partition. */
BN_API void bnxSetPixelPartition(BNContext context, int rank, int count);
/* owners[y * width + x] = the rank that renders pixel (x, y) */
BN_API void bnxPixelPartitionOwners(int width, int height, int count, int *owners);
/* Launch parameters of the render kernel (0 = automatic). */
BN_API void bnxSetLaunchConfig(BNContext context, int blocksPerSM, int threadsPerBlock);
/* With enable != 0, plain jobs (no isosurface, multi-scatter or principled
   volume) of bnRender, and single-job batches without a graph, render with
   the regrouped kernel: pixel slots whose state lives in shared memory and
   which wait in ring queues there (new pixels, rays to trace, collisions to
   shade, rays that ended); each warp takes up to 32 slots from one queue at
   a time, with no block-wide barrier, so that every step runs with full
   warps.  The default (0) is the per-lane kernel (one pixel per lane;
   bnxSetLaunchConfig and bnxSetScheduling apply to it), which is faster on
   the workloads measured.  Both give the same frames and counters.  No
   reference counterpart. */
BN_API void bnxSetRegrouping(BNContext context, int enable);
/* Warp scheduling of the render kernel: a warp keeps stepping macrocells and
   Woodcock ranges until at least serviceBatch of its lanes (or all of its
   busy lanes) need service -- shading, accumulation, a new ray -- and then
   serves them together (1..32, default 22). */
BN_API void bnxSetScheduling(BNContext context, int serviceBatch);
/* Bounds-checked build (libbarney_b200_bc.so, python -m barney_b200.build
   --bounds-check): every indexed access of the render and macrocell kernels
   is checked; an out-of-range index is counted and the access skipped.
   Returns the count since the last call on this context's device (and resets
   it), -1 in the normal build, -2 on error. */
BN_API long long bnxBoundsViolations(BNContext context);
/* Host-side fault injection for tests: after afterAllocations more device
   allocations (frame buffers, textures, macrocell grids, server buffers), the
   next one fails once with error 6 (out of memory), made on the host; no CUDA
   call fails.  A negative count disables it. */
BN_API void bnxInjectAllocationFailure(int afterAllocations);

/* Checkpoint / resume of a frame buffer's progressive state (the reference's
   only resumable state: the accumulation tiles and accumID, FrameBuffer.h:147).
   Layout: a 32-byte header (uint32 magic 0x43584E42 "BNXC", version 1, width,
   height, accumID, compensation flag, 2 reserved), the width*height float4
   accumulation buffer and, with the flag set, its float4 compensation terms. */
BN_API size_t bnxFrameBufferCheckpointSize(BNFrameBuffer fb);
/* writes bnxFrameBufferCheckpointSize(fb) bytes to host memory */
BN_API void bnxFrameBufferCheckpoint(BNFrameBuffer fb, void *hostOut);
/* fb must be resized to the checkpoint's width and height; restores accumID
   and the buffers and resolves the colour buffer again, so that reads return
   the checkpointed frame and the next bnRender continues its accumulation
   exactly as if it had never stopped */
BN_API void bnxFrameBufferRestore(BNFrameBuffer fb, const void *hostIn, size_t bytes);
/* Render several jobs in one persistent launch (each job: renderer, model,
   camera, frame buffer of this context; distinct frame buffers).  Same
   result as one bnRender per job, bit for bit.  The launch sequence is
   captured into a CUDA graph per batch shape and replayed (see
   bnxSetBatchGraphs). */
typedef struct {
  BNRenderer renderer;
  BNModel model;
  BNCamera camera;
  BNFrameBuffer frameBuffer;
} BNXRenderJob;
BN_API void bnxRenderBatch(BNContext context, const BNXRenderJob *jobs, int numJobs);
BN_API void bnxSetBatchGraphs(BNContext context, int enable);
/* Times candidate launch shapes and scheduling thresholds on this batch,
   keeps the fastest for the context and reports it (blocksPerSM 0: as many
   blocks per SM as the batch's kernel fits).  The tuning frames are
   rendered into the jobs' frame buffers and discarded (accumulation reset). */
typedef struct {
  int threadsPerBlock, blocksPerSM, serviceBatch;
  float renderMs;
} BNXLaunchConfig;
BN_API void bnxAutotuneBatch(BNContext context, const BNXRenderJob *jobs, int numJobs, BNXLaunchConfig *best);
/* Device pointer of the resolved colour channel of a frame buffer. */
BN_API void *bnxFrameBufferDevicePointer(BNFrameBuffer fb);
/* Device copies of the macrocell grid of a volume after bnGroupBuild:
   ranges (2 floats per cell) and majorants (1 float per cell), x fastest. */
BN_API void bnxVolumeGetMacrocells(BNVolume volume, int *dims3, float *rangesHostOut,
                                   float *majorantsHostOut);
/* The volume's field and transfer function evaluated on the device at n
   world-space points (3 floats each, host or device memory): scalarsOut[i]
   is the trilinear field value (NaN outside the field, as
   StructuredDataSampler::DD::sample, StructuredData.h:101-112, returns) and
   rgbaOut[4i..4i+3] the mapped colour and density of Volume::DD::sampleAndMap
   (Volume.h:62-74), computed by the same device code as the render kernels'
   Woodcock step -- the fast-math kernels' with fastMath != 0 (principled
   volumes, which render with the exact kernels only, sample with those
   too).  A diagnostic
   with no reference counterpart; allocates temporary device memory. */
BN_API void bnxVolumeSample(BNVolume volume, const float *points, int n, float *scalarsOut, float *rgbaOut,
                            int fastMath);

/* No-allocation render (no reference counterpart).  For callers that cannot
   allocate device memory while rendering -- an application that reserves
   all of its GPU memory up front and hands this library only buffers it
   owns, or a real-time loop that must not stall a frame on cudaMalloc's
   implicit device synchronisation.  Renders pathsPerPixel waves of one
   structured volume into the caller's accumulation buffer and resolves the
   colour into the caller's output, launching asynchronously on cudaStream
   (NULL: the legacy default stream) and allocating nothing: the macrocell
   majorant grid, its occupancy bitmap and the launch counters live in a
   static device array sized for BNX_NOALLOC_MAX_MACROCELLS macrocells (64^3,
   i.e. grids up to 513^3 scalars; 1.03 MiB held by every GPU that loads the
   library until exit).
   Larger volumes are rejected with error 2 and a message.  All calls share
   that array, so calls whose work overlaps on the GPU (other streams, other
   host threads) race; serialise them.  Every call made while its stream is
   not capturing looks up the array's device address (cudaGetSymbolAddress,
   which allocates nothing); a call on a capturing stream reuses the address
   found by its device's last such call.  So make the first call on each
   device outside any stream capture, and again the first call after a
   cudaDeviceReset: a reset unloads the array, and the address remembered
   from before it is stale.  Returns 0 or the error code also recorded for
   bnGetLastError. */
#define BNX_NOALLOC_MAX_MACROCELLS (64 * 64 * 64)
typedef struct {
  const void *voxels;              /* device: x-fastest scalars, dims[0]*dims[1]*dims[2] */
  BNDataType voxelType;            /* BN_FLOAT32, BN_UFIXED8, BN_UFIXED16, BNX_FLOAT16, BNX_BFLOAT16 */
  int dims[3];
  bn_float3 gridOrigin, gridSpacing;
  const bn_float4 *transferFunction; /* device: numTFValues RGBA entries */
  int numTFValues;
  bn_float2 domain;
  float densityAt1;
  bn_float3 cameraPosition, cameraDirection, cameraUp;
  float fovy;
  bn_float4 bgColor;
  float ambientRadiance;
  int numDirLights;                /* at most 16 */
  const float *dirLights;          /* host: per light direction xyz, radiance, colour rgb */
  int hgPhase;                     /* as renderer parameter bnx.hgPhase */
  float anisotropy, scatteringAlbedo;
  int width, height;
  int accumID;                     /* accumulation index of the first wave; 0 starts a frame */
  int pathsPerPixel;
  bn_float4 *accum;                /* device: width*height accumulation buffer, in/out */
  void *color;                     /* device: width*height pixels of colorFormat */
  BNDataType colorFormat;          /* BN_FLOAT4, BN_UFIXED8_RGBA, BN_UFIXED8_RGBA_SRGB */
} BNXNoAllocFrame;
BN_API int bnxRenderStructuredNoAlloc(const BNXNoAllocFrame *frame, void *cudaStream);

/* ---------------------------------------------------------------------- */
/* render server: continuous batching (no reference counterpart)           */
/* ---------------------------------------------------------------------- */
/* A worker thread renders submitted requests in slices of at most
   sliceWaves waves per request, one persistent batch launch per slice.
   Requests are admitted in arrival order while their per-request device
   buffers (accumulation, compensation, colour) fit hbmBudgetBytes and fewer
   than maxSlots requests are admitted; later arrivals join the next slice.
   Volumes (built BNModels) stay resident and are shared by requests.  While
   a server runs, it alone launches work on its context. */
typedef struct _BNXServer *BNXServer;
typedef struct {
  size_t hbmBudgetBytes;  /* device memory for admitted requests' buffers */
  int maxSlots;           /* requests rendered together in one launch */
  int sliceWaves;         /* waves per request per launch */
  long long slicePixelWaves; /* at most this many pixel-waves (pixels x waves) per launch,
                                oldest requests first, others wait for the next launch; the
                                oldest request always runs.  0: no limit */
} BNXServerConfig;
typedef struct {
  BNModel model;          /* a built model of the server's context */
  BNRenderer renderer;    /* parameters copied at submission (pathsPerPixel ignored) */
  bn_float3 position, direction, up;
  float fovy;
  int width, height, spp;
  BNDataType colorFormat; /* BN_FLOAT4, BN_UFIXED8_RGBA, BN_UFIXED8_RGBA_SRGB */
} BNXRequest;
typedef struct {
  unsigned long long submitted, completed, rejected, launches, queued, active, samples;
  size_t peakBytes;
  double busySeconds, wallSeconds, framesPerSecond;
  double p50Ms, p99Ms, meanMs, maxMs;  /* submission to completion */
  double queueP99Ms;                   /* submission to admission */
  double maxSliceMs;                   /* longest launch (host time around it) */
} BNXServerStats;
BN_API BNXServer bnxServerCreate(BNContext context, const BNXServerConfig *config);
BN_API void bnxServerDestroy(BNXServer server);
/* Takes `bytes` (at most the HBM budget) of device memory for request
   buffers now, in 256 MiB chunks, so that admissions find buffers without a
   cudaMalloc, which inside a busy process took up to tens of milliseconds per
   chunk.  Without a reservation the chunks are taken as requests need them. */
BN_API void bnxServerReserve(BNXServer server, size_t bytes);
/* returns the request id (>= 0), or -1 on error; callable from any thread */
BN_API long long bnxServerSubmit(BNXServer server, const BNXRequest *request);
/* waits up to timeoutMs (< 0: forever) for a request; copies its colour
   channel into hostPixels (may be NULL) and forgets it.  Returns 1 when
   done, 0 on timeout, a negative error code on failure. */
BN_API int bnxServerWait(BNXServer server, long long id, int timeoutMs, void *hostPixels);
/* Setting the environment variable BNX_SERVER_TRACE to a file path makes
   every server created afterwards append one line per launch to that file:
   start and gap since the previous launch (ms from the server's creation),
   time spent taking device buffers for newly admitted requests, duration,
   requests in the launch, admitted and retired by it, queue length, waves and
   pixel-waves rendered. */
BN_API void bnxServerGetStats(BNXServer server, BNXServerStats *stats);
BN_API void bnxServerResetStats(BNXServer server);

/* ---------------------------------------------------------------------- */
/* ANARI parameter mapping (no native-API counterpart: the ANARI device      */
/* does this before calling bn*; restated from barney/anari)                */
/* ---------------------------------------------------------------------- */
/* "transferFunction1D" colour / opacity arrays -> the RGBA table passed to
   bnVolumeSetXF (Volume.cpp:178-234).  colors: numColors x colorChannels (3
   or 4) floats or NULL (uniformColor); opacities: numOpacities floats or NULL
   (uniformOpacity, multiplied by uniformColor.w as Volume.cpp:166-167 does).
   Returns the table size max(numColors, numOpacities) and, if out is not
   NULL, writes the table. */
BN_API int bnxAnariTransferFunction1D(const float *colors, int numColors, int colorChannels,
                                      const float *opacities, int numOpacities, bn_float4 uniformColor,
                                      float uniformOpacity, bn_float4 *out);
/* volume "unitDistance" -> densityAt1 of bnVolumeSetXF (Volume.cpp:99-107) */
BN_API float bnxAnariDensityScale(float unitDistance);
/* "structuredRegular" spatial field (SpatialField.cpp:74-140): texture data
   of float32 or uint8 / ufixed8 scalars + a "structured" field with dims,
   gridOrigin, gridSpacing, committed */
BN_API BNScalarField bnxAnariStructuredRegular(BNContext context, int slot, BNDataType elementType,
                                               const void *data, int nx, int ny, int nz, bn_float3 origin,
                                               bn_float3 spacing);

/* ANARI "renderer" parameters (Renderer.cpp:22-37).  set: the BNX_ANARI_*
   bits of the parameters the application set; the others take the ANARI
   device's defaults. */
#define BNX_ANARI_PIXEL_SAMPLES 0x1u
#define BNX_ANARI_AMBIENT_RADIANCE 0x2u
#define BNX_ANARI_BACKGROUND 0x4u
#define BNX_ANARI_CUT_PLANE 0x8u
#define BNX_ANARI_MAX_VOLUME_BOUNCES 0x10u
#define BNX_ANARI_CROSSHAIRS 0x20u
typedef struct {
  unsigned set;
  int pixelSamples;       /* default 1 */
  float ambientRadiance;  /* default 1 */
  bn_float4 background;   /* default (0, 0, 0, 1) */
  bn_float4 cutPlane;     /* default (0, 0, 0, 0): a zero normal clips nothing */
  int maxVolumeBounces;   /* default 0 */
  int crosshairs;         /* default 0 (accepted; the debug overlay is not built) */
} BNXAnariRenderer;
/* Fills the parameters in that are not set with the defaults
   (Renderer::commitParameters); out->set has every bit. */
BN_API void bnxAnariRendererParams(const BNXAnariRenderer *in, BNXAnariRenderer *out);
/* What the ANARI renderer's commit does to the Barney renderer
   (Renderer::finalize, Renderer.cpp:40-51): the parameters, with their
   defaults, as bgColor, crosshairs, pathsPerPixel, ambientRadiance,
   maxVolumeBounces and cutPlane, then bnCommit. */
BN_API void bnxAnariRendererCommit(BNRenderer renderer, const BNXAnariRenderer *params);
/* anariRenderFrame (Frame::renderFrame, Frame.cpp:165-262): if any object of
   the context was committed or built (bnCommit, bnGroupBuild, bnBuild,
   bnSetInstances, bnVolumeSetXF) since this frame buffer's last frame --
   or this is its first frame -- its accumulation starts over
   (bnAccumReset); then bnRender. */
BN_API void bnxAnariRenderFrame(BNRenderer renderer, BNModel model, BNCamera camera, BNFrameBuffer frameBuffer);

#ifdef __cplusplus
}
#endif
#endif /* BN_VOLUME_H */
