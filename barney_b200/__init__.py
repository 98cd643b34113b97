"""barney_b200: B200-native (sm_100a) structured-volume path tracing behind
Barney's native ``bn*`` API.

The product is ``libbarney_b200.so`` (CUDA kernels + C++ object model,
C ABI declared in ``include/bn_volume.h``).  This module is a thin ctypes
mirror of that ABI, used the way an application uses Barney's native API
(barney/native/include/barney.h): create a context, upload a structured
scalar field, attach a transfer function, build, render, read the frame.

There is no CPU fallback: importing works without a GPU, but every call that
needs the device fails loudly if the library or the GPU is missing.
"""
import ctypes
import os

import numpy as np

from . import build as _build

_HERE = os.path.dirname(os.path.abspath(__file__))
# BARNEY_B200_LIBRARY selects another build of the library, e.g. the
# bounds-checked libbarney_b200_bc.so; it is loaded as it is, never rebuilt
LIB_PATH = os.environ.get("BARNEY_B200_LIBRARY") or _build.LIB
_lib = None

# BNDataType values (include/bn_volume.h)
BN_OBJECT = 2
BN_UINT8 = 110
BN_FLOAT32 = 180
BN_FLOAT4 = 183
BN_UFIXED8 = 300
BN_UFIXED8_RGBA = 301
BN_UFIXED8_RGBA_SRGB = 302
BN_UFIXED16 = 303
BNX_FLOAT16 = 1000
BNX_BFLOAT16 = 1001
BN_FB_COLOR = 1

VOXEL_FORMATS = {"f32": BN_FLOAT32, "u8": BN_UFIXED8, "u16": BN_UFIXED16, "f16": BNX_FLOAT16, "bf16": BNX_BFLOAT16}
COLOR_FORMATS = {"float4": BN_FLOAT4, "rgba8": BN_UFIXED8_RGBA, "rgba8_srgb": BN_UFIXED8_RGBA_SRGB}

# every symbol include/bn_volume.h declares
EXPORTS = [
    "bnContextCreate", "bnContextDestroy", "bnPhysicalDeviceCount", "bnRelease", "bnAddReference", "bnCommit",
    "bnSet1i", "bnSet2i", "bnSet3i", "bnSet4i", "bnSet1f", "bnSet2f", "bnSet3f", "bnSet4f", "bnSetObject",
    "bnSetData", "bnSetString", "bnSet4x3fv", "bnSet4x4fv", "bnDataCreate", "bnDataSet",
    "bnTextureData2DCreate", "bnTexture2DCreate", "bnTexture3DCreate", "bnSamplerCreate", "bnTextureData3DCreate", "bnScalarFieldCreate", "bnVolumeCreate",
    "bnVolumeSetXF", "bnLightCreate", "bnGeometryCreate", "bnMaterialCreate", "bnGroupCreate", "bnGroupBuild", "bnModelCreate", "bnSetInstances",
    "bnUpdateInstanceTransforms", "bnSetInstanceAttributes",
    "bnBuild", "bnCameraCreate", "bnRendererCreate", "bnFrameBufferCreate", "bnFrameBufferResize",
    "bnFrameBufferRead", "bnFrameBufferGetSize", "bnAccumReset", "bnRender", "bnGetLastError",
    "bnGetLastErrorString", "bnClearLastError", "bnxGetStats", "bnxSetStream", "bnxGetStream",
    "bnxSetLaunchConfig", "bnxFrameBufferDevicePointer", "bnxVolumeGetMacrocells", "bnxVolumeSample", "bnxSetRegrouping",
    "bnxRenderStructuredNoAlloc", "bnxSetScheduling", "bnxBoundsViolations", "bnxInjectAllocationFailure", "bnxFrameBufferCheckpointSize",
    "bnxFrameBufferCheckpoint", "bnxFrameBufferRestore", "bnxRenderBatch", "bnxSetBatchGraphs", "bnxAutotuneBatch",
    "bnxServerCreate", "bnxServerDestroy", "bnxServerSubmit", "bnxServerWait", "bnxServerGetStats",
    "bnxServerResetStats", "bnxServerReserve", "bnxSetRenderTimeout", "bnxSetPixelPartition",
    "bnxPixelPartitionOwners", "bnxAnariTransferFunction1D", "bnxAnariDensityScale",
    "bnxAnariStructuredRegular", "bnxAnariRendererParams", "bnxAnariRendererCommit", "bnxAnariRenderFrame",
]


class bn_float2(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float)]


class bn_float3(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float), ("z", ctypes.c_float)]


class bn_float4(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float), ("z", ctypes.c_float), ("w", ctypes.c_float)]


def anari_transfer_function_1d(colors=None, opacities=None, uniform_color=(1.0, 1.0, 1.0, 1.0),
                               uniform_opacity=1.0):
    """ANARI transferFunction1D arrays -> the RGBA table for bnVolumeSetXF."""
    L = lib()
    c = None if colors is None else np.ascontiguousarray(colors, np.float32)
    o = None if opacities is None else np.ascontiguousarray(opacities, np.float32).reshape(-1)
    nc, ch = (0, 4) if c is None else (c.shape[0], c.shape[1])
    no = 0 if o is None else o.shape[0]
    uc = bn_float4(*uniform_color)
    n = L.bnxAnariTransferFunction1D(_void_p(c), nc, ch, _void_p(o), no, uc, uniform_opacity, None)
    check()
    out = np.zeros((n, 4), np.float32)
    L.bnxAnariTransferFunction1D(_void_p(c), nc, ch, _void_p(o), no, uc, uniform_opacity, out.ctypes.data)
    check()
    return out


# ANARI renderer parameters (BNXAnariRenderer; barney/anari/Renderer.cpp:22-37)
BNX_ANARI_BITS = {"pixelSamples": 0x1, "ambientRadiance": 0x2, "background": 0x4, "cutPlane": 0x8,
                  "maxVolumeBounces": 0x10, "crosshairs": 0x20}


class BNXAnariRenderer(ctypes.Structure):
    _fields_ = [("set", ctypes.c_uint), ("pixelSamples", ctypes.c_int), ("ambientRadiance", ctypes.c_float),
                ("background", bn_float4), ("cutPlane", bn_float4), ("maxVolumeBounces", ctypes.c_int),
                ("crosshairs", ctypes.c_int)]


def anari_renderer(**params):
    """A BNXAnariRenderer with the given ANARI renderer parameters set (the
    others take the ANARI device's defaults when it is committed)."""
    p = BNXAnariRenderer()
    for k, val in params.items():
        if k not in BNX_ANARI_BITS:
            raise ValueError(f"unknown ANARI renderer parameter {k!r}")
        p.set |= BNX_ANARI_BITS[k]
        setattr(p, k, bn_float4(*val) if k in ("background", "cutPlane") else val)
    return p


def anari_renderer_params(**params):
    """The parameters an ANARI renderer commit uses: the given ones, the
    defaults for the rest (bnxAnariRendererParams)."""
    out = BNXAnariRenderer()
    lib().bnxAnariRendererParams(ctypes.byref(anari_renderer(**params)), ctypes.byref(out))
    check()
    return {"set": out.set, "pixelSamples": out.pixelSamples, "ambientRadiance": out.ambientRadiance,
            "background": (out.background.x, out.background.y, out.background.z, out.background.w),
            "cutPlane": (out.cutPlane.x, out.cutPlane.y, out.cutPlane.z, out.cutPlane.w),
            "maxVolumeBounces": out.maxVolumeBounces, "crosshairs": out.crosshairs}


class BNXStats(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_ulonglong), ("mcVisits", ctypes.c_ulonglong), ("rays", ctypes.c_ulonglong),
                ("pixelSamples", ctypes.c_ulonglong), ("errorFlags", ctypes.c_ulonglong),
                ("renderMs", ctypes.c_float), ("resolveMs", ctypes.c_float)]


class BNXRenderJob(ctypes.Structure):
    _fields_ = [("renderer", ctypes.c_void_p), ("model", ctypes.c_void_p), ("camera", ctypes.c_void_p),
                ("frameBuffer", ctypes.c_void_p)]


class BNXLaunchConfig(ctypes.Structure):
    _fields_ = [("threadsPerBlock", ctypes.c_int), ("blocksPerSM", ctypes.c_int), ("serviceBatch", ctypes.c_int),
                ("renderMs", ctypes.c_float)]


class BNXServerConfig(ctypes.Structure):
    _fields_ = [("hbmBudgetBytes", ctypes.c_size_t), ("maxSlots", ctypes.c_int), ("sliceWaves", ctypes.c_int),
                ("slicePixelWaves", ctypes.c_longlong)]


_F3 = ctypes.c_float * 3


class BNXRequest(ctypes.Structure):
    _fields_ = [("model", ctypes.c_void_p), ("renderer", ctypes.c_void_p), ("position", _F3), ("direction", _F3),
                ("up", _F3), ("fovy", ctypes.c_float), ("width", ctypes.c_int), ("height", ctypes.c_int),
                ("spp", ctypes.c_int), ("colorFormat", ctypes.c_int)]


class BNXServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_ulonglong) for n in ("submitted", "completed", "rejected", "launches", "queued",
                                                  "active", "samples")] + \
               [("peakBytes", ctypes.c_size_t)] + \
               [(n, ctypes.c_double) for n in ("busySeconds", "wallSeconds", "framesPerSecond", "p50Ms", "p99Ms",
                                               "meanMs", "maxMs", "queueP99Ms", "maxSliceMs")]


class BarneyError(RuntimeError):
    pass


def lib(build_if_missing=True):
    """Load libbarney_b200.so (building it first if needed)."""
    global _lib
    if _lib is not None:
        return _lib
    if build_if_missing and LIB_PATH == _build.LIB and _build._stale():
        _build.build()
    if not os.path.exists(LIB_PATH):
        raise BarneyError("libbarney_b200.so is missing; run barney_b200.build.build()")
    L = ctypes.CDLL(LIB_PATH)
    P, I, F, S = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_char_p
    sig = {
        "bnContextCreate": ([I, P, I, P], P), "bnContextDestroy": ([P], None), "bnPhysicalDeviceCount": ([], I),
        "bnRelease": ([P], None), "bnAddReference": ([P], None), "bnCommit": ([P], None),
        "bnSet1i": ([P, S, I], None), "bnSet2i": ([P, S, I, I], None), "bnSet3i": ([P, S, I, I, I], None),
        "bnSet4i": ([P, S, I, I, I, I], None), "bnSet1f": ([P, S, F], None), "bnSet2f": ([P, S, F, F], None),
        "bnSet3f": ([P, S, F, F, F], None), "bnSet4f": ([P, S, F, F, F, F], None),
        "bnSetObject": ([P, S, P], None), "bnSetData": ([P, S, P], None), "bnSetString": ([P, S, S], None),
        "bnSet4x3fv": ([P, S, P], None), "bnSet4x4fv": ([P, S, P], None),
        "bnDataSet": ([P, ctypes.c_size_t, P], None),
        "bnTextureData2DCreate": ([P, I, I, I, I, P], P),
        "bnTexture2DCreate": ([P, I, I, ctypes.c_uint32, ctypes.c_uint32, P, I, I, I, I], P),
        "bnTexture3DCreate": ([P, I, I, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, P, I, I], P),
        "bnSamplerCreate": ([P, I, S], P),
        "bnUpdateInstanceTransforms": ([P, I, P, I], None), "bnSetInstanceAttributes": ([P, I, S, P], None),
        "bnDataCreate": ([P, I, I, ctypes.c_size_t, P], P),
        "bnTextureData3DCreate": ([P, I, I, I, I, I, P], P), "bnScalarFieldCreate": ([P, I, S], P),
        "bnVolumeCreate": ([P, I, P], P), "bnVolumeSetXF": ([P, bn_float2, P, I, F], None),
        "bnLightCreate": ([P, I, S], P), "bnGeometryCreate": ([P, I, S], P), "bnMaterialCreate": ([P, I, S], P),
        "bnGroupCreate": ([P, I, P, I, P, I], P), "bnGroupBuild": ([P], None),
        "bnModelCreate": ([P], P), "bnSetInstances": ([P, I, P, P, I], None), "bnBuild": ([P, I], None),
        "bnCameraCreate": ([P, S], P), "bnRendererCreate": ([P, S], P), "bnFrameBufferCreate": ([P, I], P),
        "bnFrameBufferResize": ([P, I, I, I, ctypes.c_uint32], None),
        "bnFrameBufferRead": ([P, I, P, I], None), "bnFrameBufferGetSize": ([P, P, P], None),
        "bnAccumReset": ([P], None), "bnRender": ([P, P, P, P], None), "bnGetLastError": ([], I),
        "bnGetLastErrorString": ([], S), "bnClearLastError": ([], None),
        "bnxGetStats": ([P, P], None), "bnxSetStream": ([P, P], None), "bnxGetStream": ([P], P),
        "bnxSetLaunchConfig": ([P, I, I], None), "bnxFrameBufferDevicePointer": ([P], P),
        "bnxVolumeGetMacrocells": ([P, P, P, P], None), "bnxVolumeSample": ([P, P, I, P, P, I], None),
        "bnxRenderStructuredNoAlloc": ([P, P], I),
        "bnxSetScheduling": ([P, I], None), "bnxSetRegrouping": ([P, I], None), "bnxBoundsViolations": ([P], ctypes.c_longlong),
        "bnxInjectAllocationFailure": ([I], None),
        "bnxFrameBufferCheckpointSize": ([P], ctypes.c_size_t), "bnxFrameBufferCheckpoint": ([P, P], None),
        "bnxFrameBufferRestore": ([P, P, ctypes.c_size_t], None),
        "bnxRenderBatch": ([P, P, I], None),
        "bnxSetBatchGraphs": ([P, I], None), "bnxAutotuneBatch": ([P, P, I, P], None),
        "bnxServerCreate": ([P, P], P), "bnxServerDestroy": ([P], None),
        "bnxServerSubmit": ([P, P], ctypes.c_longlong), "bnxServerWait": ([P, ctypes.c_longlong, I, P], I),
        "bnxServerGetStats": ([P, P], None), "bnxServerResetStats": ([P], None),
        "bnxServerReserve": ([P, ctypes.c_size_t], None),
        "bnxSetRenderTimeout": ([P, I], None),
        "bnxSetPixelPartition": ([P, I, I], None), "bnxPixelPartitionOwners": ([I, I, I, P], None),
        "bnxAnariTransferFunction1D": ([P, I, I, P, I, bn_float4, F, P], I),
        "bnxAnariDensityScale": ([F], F),
        "bnxAnariStructuredRegular": ([P, I, I, P, I, I, I, bn_float3, bn_float3], P),
        "bnxAnariRendererParams": ([P, P], None), "bnxAnariRendererCommit": ([P, P], None),
        "bnxAnariRenderFrame": ([P, P, P, P], None),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def check():
    """Raise BarneyError if the last bn* call on this thread recorded an error."""
    L = lib()
    code = L.bnGetLastError()
    if code:
        msg = L.bnGetLastErrorString().decode()
        L.bnClearLastError()
        raise BarneyError(f"barney error {code}: {msg}")


def _b(s):
    return s.encode() if isinstance(s, str) else s


def _void_p(x):
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    if hasattr(x, "data_ptr"):  # torch tensor (host or device)
        return x.data_ptr()
    return x


class Context:
    """A bn* context shared by several VolumeRenderers (batch rendering)."""

    def __init__(self, gpu=0, stream=None):
        L = lib()
        self.L = L
        ids = (ctypes.c_int * 1)(gpu)
        self.ctx = L.bnContextCreate(1, None, 1, ids)
        check()
        if stream is not None:
            L.bnxSetStream(self.ctx, stream)

    def render_batch(self, renderers):
        """One persistent launch for all renderers' frames (bnxRenderBatch)."""
        jobs = (BNXRenderJob * len(renderers))()
        for j, r in zip(jobs, renderers):
            j.renderer, j.model, j.camera, j.frameBuffer = r.renderer, r.model, r.camera, r.fb
        self.L.bnxRenderBatch(self.ctx, jobs, len(renderers))
        check()

    def autotune_batch(self, renderers):
        jobs = (BNXRenderJob * len(renderers))()
        for j, r in zip(jobs, renderers):
            j.renderer, j.model, j.camera, j.frameBuffer = r.renderer, r.model, r.camera, r.fb
        best = BNXLaunchConfig()
        self.L.bnxAutotuneBatch(self.ctx, jobs, len(renderers), ctypes.byref(best))
        check()
        return {f: getattr(best, f) for f, _ in BNXLaunchConfig._fields_}

    def set_graphs(self, enable):
        self.L.bnxSetBatchGraphs(self.ctx, int(enable))
        check()

    def stats(self):
        st = BNXStats()
        self.L.bnxGetStats(self.ctx, ctypes.byref(st))
        check()
        return {"samples": st.samples, "mc_visits": st.mcVisits, "rays": st.rays,
                "pixel_samples": st.pixelSamples, "error_flags": st.errorFlags,
                "render_ms": st.renderMs, "resolve_ms": st.resolveMs}

    def close(self):
        if self.ctx:
            self.L.bnContextDestroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class VolumeRenderer:
    """One structured volume rendered through the bn* API, in the call order
    of Barney's own clients (texture data -> structured field -> volume +
    transfer function -> group -> model -> build; camera, renderer, frame
    buffer -> bnRender -> bnFrameBufferRead).

    ``desc`` is the scene dict of ``barney_b200.synth`` (the same dict the
    oracle takes)."""

    def __init__(self, desc, color_format="float4", gpu=0, stream=None, context=None):
        L = lib()
        self.L = L
        self.desc = desc
        self.shared = context
        if context is not None:
            self.ctx = context.ctx
        else:
            ids = (ctypes.c_int * 1)(gpu)
            self.ctx = L.bnContextCreate(1, None, 1, ids)
            check()
            if stream is not None:
                L.bnxSetStream(self.ctx, stream)
        self._objects = []
        vox = desc["voxels"]
        nz, ny, nx = vox.shape
        self.td = self._keep(L.bnTextureData3DCreate(self.ctx, 0, VOXEL_FORMATS[desc["dtype"]], nx, ny, nz,
                                                     _void_p(vox)))
        check()
        sf = self._keep(L.bnScalarFieldCreate(self.ctx, 0, b"structured"))
        L.bnSetObject(sf, b"textureData", self.td)
        L.bnSet3i(sf, b"dims", nx, ny, nz)
        L.bnSet3f(sf, b"gridOrigin", *desc.get("origin", (0.0, 0.0, 0.0)))
        L.bnSet3f(sf, b"gridSpacing", *desc["spacing"])
        L.bnCommit(sf)
        check()
        self.sf = sf
        self.vol = self._keep(L.bnVolumeCreate(self.ctx, 0, sf))
        check()
        self.set_transfer_function(desc["tf"], desc.get("domain", (0.0, 1.0)), desc["density"])
        L.bnSet1f(self.vol, b"anisotropy", desc.get("anisotropy", 0.6))
        L.bnSet1f(self.vol, b"scatteringAlbedo", desc.get("scattering_albedo", 0.9))
        if desc.get("majorant_round_up"):
            L.bnSet1i(self.vol, b"bnx.majorantRoundUp", 1)
        pv = desc.get("principled")
        if pv:  # principled volume coefficients (Volume.cpp:36-126 parameter names)
            L.bnSet1i(self.vol, b"principledVolume", 1 if pv.get("enabled", True) else 0)
            for key, name in (("density", b"principledDensity"), ("density_threshold", b"principledDensityThreshold"),
                              ("density_scale", b"principledDensityScale"),
                              ("emission_strength", b"principledEmissionStrength"),
                              ("blackbody_intensity", b"principledBlackbodyIntensity"),
                              ("temperature", b"principledTemperature")):
                if key in pv:
                    L.bnSet1f(self.vol, name, float(pv[key]))
            if "value_range" in pv:
                L.bnSet2f(self.vol, b"principledValueRange", *map(float, pv["value_range"]))
            for key, name in (("scatter_color", b"principledScatterColor"),
                              ("absorption_color", b"principledAbsorptionColor"),
                              ("emission_color", b"principledEmissionColor"),
                              ("blackbody_tint", b"principledBlackbodyTint")):
                if key in pv:
                    L.bnSet3f(self.vol, name, *map(float, pv[key]))
        L.bnCommit(self.vol)
        check()
        # an iso_surface geometry with a matte material on the same field; with
        # desc["volume"] False the group holds the isosurface alone
        geoms, n_geoms = None, 0
        self.iso = self.material = None
        if desc.get("iso"):
            self.material = self._keep(L.bnMaterialCreate(self.ctx, 0, b"matte"))
            self.iso = self._keep(L.bnGeometryCreate(self.ctx, 0, b"iso_surface"))
            check()
            L.bnSetObject(self.iso, b"scalarField", sf)
            self.set_iso(**desc["iso"])
            geoms, n_geoms = (ctypes.c_void_p * 1)(self.iso), 1
        with_vol = desc.get("volume", True)
        vols = (ctypes.c_void_p * 1)(self.vol) if with_vol else None
        self.group = self._keep(L.bnGroupCreate(self.ctx, 0, geoms, n_geoms, vols, 1 if with_vol else 0))
        check()
        lights = desc.get("dir_lights", [])
        self.lights_data = None
        if lights:
            hs = []
            for l in lights:
                h = self._keep(L.bnLightCreate(self.ctx, 0, b"directional"))
                L.bnSet3f(h, b"direction", *l["direction"])
                L.bnSet1f(h, b"radiance", l.get("radiance", 1.0))
                if "color" in l:
                    L.bnSet3f(h, b"color", *l["color"])
                L.bnCommit(h)
                hs.append(h)
            arr = (ctypes.c_void_p * len(hs))(*hs)
            data = self._keep(L.bnDataCreate(self.ctx, 0, BN_OBJECT, len(hs), arr))
            self.lights_data = data
            L.bnSetData(self.group, b"lights", data)
        L.bnGroupBuild(self.group)
        check()
        self.model = self._keep(L.bnModelCreate(self.ctx))
        groups = (ctypes.c_void_p * 1)(self.group)
        L.bnSetInstances(self.model, 0, groups, None, 1)
        L.bnBuild(self.model, 0)
        check()
        self.camera = self._keep(L.bnCameraCreate(self.ctx, b"perspective"))
        self.set_camera(desc["camera"])
        self.renderer = self._keep(L.bnRendererCreate(self.ctx, b"default"))
        self.fb = self._keep(L.bnFrameBufferCreate(self.ctx, 0))
        self.color_format = color_format
        self.resize(desc["width"], desc["height"], color_format)
        self.set_renderer(desc, spp=desc.get("spp", 1))

    def _keep(self, h):
        self._objects.append(h)
        return h

    def set_iso(self, value=None, color=None, opacity=None):
        """Isosurface parameters: iso value; the matte material's "color" (rgb or
        rgba) and "opacity"."""
        L = self.L
        if color is not None:
            c = tuple(float(x) for x in color)
            (L.bnSet3f if len(c) == 3 else L.bnSet4f)(self.material, b"color", *c)
        if opacity is not None:
            L.bnSet1f(self.material, b"opacity", float(opacity))
        L.bnCommit(self.material)
        if value is not None:
            L.bnSet1f(self.iso, b"isoValue", float(value))
        L.bnSetObject(self.iso, b"material", self.material)
        L.bnCommit(self.iso)
        check()

    def set_transfer_function(self, tf, domain, density):
        tf = np.ascontiguousarray(tf, np.float32).reshape(-1, 4)
        self._tf = tf
        self.L.bnVolumeSetXF(self.vol, bn_float2(*domain), tf.ctypes.data, tf.shape[0], float(density))
        self.L.bnCommit(self.vol)
        check()

    def set_camera(self, cam):
        L = self.L
        L.bnSet3f(self.camera, b"position", *cam["position"])
        L.bnSet3f(self.camera, b"direction", *cam["direction"])
        L.bnSet3f(self.camera, b"up", *cam.get("up", (0.0, 1.0, 0.0)))
        L.bnSet1f(self.camera, b"fovy", cam.get("fovy", 60.0))
        L.bnCommit(self.camera)
        check()

    def set_renderer(self, desc, spp=1):
        L = self.L
        L.bnSet4f(self.renderer, b"bgColor", *desc.get("bg_color", (0.0, 0.0, 0.0, 1.0)))
        L.bnSet4f(self.renderer, b"cutPlane", *desc.get("cut_plane", (0.0, 0.0, 0.0, -1e30)))
        L.bnSet1f(self.renderer, b"ambientRadiance", desc.get("ambient", 1.0))
        L.bnSet1i(self.renderer, b"pathsPerPixel", int(spp))
        L.bnSet1i(self.renderer, b"maxVolumeBounces", int(desc.get("max_volume_bounces", 0)))
        L.bnSet1i(self.renderer, b"bnx.hgPhase", 1 if desc.get("phase", "simple") == "hg" else 0)
        L.bnSet1i(self.renderer, b"bnx.emissionAbsorption", int(desc.get("emission_absorption", False)))
        L.bnSet1i(self.renderer, b"bnx.exactLog", int(desc.get("exact_log", False)))
        L.bnSet1i(self.renderer, b"bnx.compensatedAccum", int(desc.get("compensated_accum", False)))
        L.bnSet1i(self.renderer, b"bnx.fastMath", int(desc.get("fast_math", False)))
        L.bnCommit(self.renderer)
        check()

    def set_spp(self, spp):
        self.L.bnSet1i(self.renderer, b"pathsPerPixel", int(spp))
        self.L.bnCommit(self.renderer)
        check()

    def resize(self, w, h, color_format=None):
        fmt = color_format or self.color_format
        self.color_format = fmt
        self.width, self.height = w, h
        self.L.bnFrameBufferResize(self.fb, COLOR_FORMATS[fmt], w, h, BN_FB_COLOR)
        check()

    def render(self):
        self.L.bnRender(self.renderer, self.model, self.camera, self.fb)
        check()

    def accum_reset(self):
        self.L.bnAccumReset(self.fb)
        check()

    def checkpoint(self):
        """The frame buffer's progressive state (bnxFrameBufferCheckpoint) as bytes."""
        n = self.L.bnxFrameBufferCheckpointSize(self.fb)
        check()
        buf = ctypes.create_string_buffer(n)
        self.L.bnxFrameBufferCheckpoint(self.fb, buf)
        check()
        return buf.raw

    def restore(self, data):
        """Continue from a checkpoint of a frame buffer of the same size."""
        self.L.bnxFrameBufferRestore(self.fb, data, len(data))
        check()

    def read(self, out=None):
        """Copy the resolved colour channel into `out` (host numpy array or
        device tensor) or a new numpy array."""
        if out is None:
            if self.color_format == "float4":
                out = np.zeros((self.height, self.width, 4), np.float32)
            else:
                out = np.zeros((self.height, self.width), np.uint32)
        self.L.bnFrameBufferRead(self.fb, BN_FB_COLOR, _void_p(out), COLOR_FORMATS[self.color_format])
        check()
        return out

    def stats(self):
        st = BNXStats()
        self.L.bnxGetStats(self.ctx, ctypes.byref(st))
        check()
        return {"samples": st.samples, "mc_visits": st.mcVisits, "rays": st.rays,
                "pixel_samples": st.pixelSamples, "error_flags": st.errorFlags,
                "render_ms": st.renderMs, "resolve_ms": st.resolveMs}

    def macrocells(self):
        dims = (ctypes.c_int * 3)()
        self.L.bnxVolumeGetMacrocells(self.vol, dims, None, None)
        check()
        d = tuple(dims)
        ranges = np.zeros((d[2], d[1], d[0], 2), np.float32)
        maj = np.zeros((d[2], d[1], d[0]), np.float32)
        self.L.bnxVolumeGetMacrocells(self.vol, None, ranges.ctypes.data, maj.ctypes.data)
        check()
        return ranges, maj

    def sample(self, points, fast_math=False):
        """The field (NaN outside) and sampleAndMap's rgba at world points,
        evaluated on the device by the render kernels' code (bnxVolumeSample)."""
        P = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        scal = np.zeros(P.shape[0], np.float32)
        rgba = np.zeros((P.shape[0], 4), np.float32)
        self.L.bnxVolumeSample(self.vol, P.ctypes.data, P.shape[0], scal.ctypes.data, rgba.ctypes.data,
                               1 if fast_math else 0)
        check()
        return scal, rgba

    def anari_commit_renderer(self, **params):
        """The ANARI renderer's commit (bnxAnariRendererCommit) on this renderer."""
        self.L.bnxAnariRendererCommit(self.renderer, ctypes.byref(anari_renderer(**params)))
        check()

    def anari_render_frame(self):
        """anariRenderFrame (bnxAnariRenderFrame): accumulation starts over
        after any commit or build of the context since the last frame."""
        self.L.bnxAnariRenderFrame(self.renderer, self.model, self.camera, self.fb)
        check()

    def set_regrouping(self, enable=True):
        """Regrouped kernel for plain jobs, or the per-lane kernel (default)."""
        self.L.bnxSetRegrouping(self.ctx, 1 if enable else 0)
        check()

    def set_scheduling(self, service_batch=22):
        self.L.bnxSetScheduling(self.ctx, service_batch)
        check()

    def set_partition(self, rank, count):
        """Render only this rank's pixel tiles (bnxSetPixelPartition)."""
        self.L.bnxSetPixelPartition(self.ctx, int(rank), int(count))
        check()

    def set_timeout(self, milliseconds):
        self.L.bnxSetRenderTimeout(self.ctx, int(milliseconds))
        check()

    def set_launch_config(self, blocks_per_sm=0, threads_per_block=0):
        self.L.bnxSetLaunchConfig(self.ctx, blocks_per_sm, threads_per_block)
        check()

    def close(self):
        if self.ctx and self.shared is None:
            self.L.bnContextDestroy(self.ctx)
        elif self.ctx:
            for h in self._objects:
                self.L.bnRelease(h)
            self._objects = []
        self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def partition_owners(width, height, count):
    """(height, width) int32 map: the rank that renders each pixel of a frame
    partitioned over `count` ranks (bnxPixelPartitionOwners)."""
    owners = np.zeros((height, width), np.int32)
    L = lib()
    L.bnxPixelPartitionOwners(int(width), int(height), int(count), owners.ctypes.data)
    check()
    return owners


def merge_partitions(frames, owners):
    """Assemble a frame from per-rank frames (stacked on axis 0; numpy or
    torch) by the owner map: pixel (y, x) is taken from frame owners[y, x]."""
    out = frames[0].clone() if hasattr(frames[0], "clone") else frames[0].copy()
    for r in range(1, len(frames)):
        sel = owners == r
        out[sel] = frames[r][sel]
    return out


class Server:
    """Continuous-batching render server over resident volumes (bnxServer*)."""

    def __init__(self, context, hbm_budget_bytes=150 << 30, max_slots=256, slice_waves=4, slice_pixel_waves=0):
        self.L = lib()
        self.context = context
        cfg = BNXServerConfig(hbm_budget_bytes, max_slots, slice_waves, slice_pixel_waves)
        self.h = self.L.bnxServerCreate(context.ctx, ctypes.byref(cfg))
        check()

    def reserve(self, nbytes):
        """Take device memory for request buffers now (bnxServerReserve)."""
        self.L.bnxServerReserve(self.h, ctypes.c_size_t(nbytes))
        check()

    def submit(self, renderer, camera, width, height, spp, color_format="rgba8"):
        """renderer: a VolumeRenderer of the server's context (its model and
        renderer parameters are used); camera: dict as in synth.look_at."""
        q = BNXRequest()
        q.model, q.renderer = renderer.model, renderer.renderer
        q.position[:] = camera["position"]
        q.direction[:] = camera["direction"]
        q.up[:] = camera.get("up", (0.0, 1.0, 0.0))
        q.fovy = camera.get("fovy", 60.0)
        q.width, q.height, q.spp = width, height, spp
        q.colorFormat = COLOR_FORMATS[color_format]
        rid = self.L.bnxServerSubmit(self.h, ctypes.byref(q))
        if rid < 0:
            check()
        return rid

    def wait(self, rid, out=None, timeout_ms=-1):
        rc = self.L.bnxServerWait(self.h, rid, timeout_ms, _void_p(out))
        if rc < 0:
            check()
        return rc == 1

    def stats(self):
        st = BNXServerStats()
        self.L.bnxServerGetStats(self.h, ctypes.byref(st))
        check()
        return {f: getattr(st, f) for f, _ in BNXServerStats._fields_}

    def reset_stats(self):
        self.L.bnxServerResetStats(self.h)

    def close(self):
        if self.h:
            self.L.bnxServerDestroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
