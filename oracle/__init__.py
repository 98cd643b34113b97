"""CPU oracle for Barney's structured-volume path -- TEST INFRASTRUCTURE ONLY.

ctypes bindings to ``liboracle.so`` (built from ``bn_oracle.cpp`` and
``bn_fp64.cpp`` by ``oracle/Makefile``).  The product (``barney_b200``) never
imports this package; only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline / reference legs of ``bench.py`` use it, and only as the checker
or the timed CPU baseline.

Pinned to the reference's own code: tests/test_ref_golden.py checks this
restatement bit for bit against golden vectors that the reference's own
sources produce (its RNG, hash, fastLog, DDA, trilinear texture sampler,
transfer function, Woodcock tracking and principled-volume functions,
compiled from where they lie by oracle/Makefile target `ref`;
tests/golden/make_ref_golden.py).  The shading, light sampling and
accumulation steps, which the reference cannot run outside its full
renderer, are pinned by hand-derived known answers
(tests/test_oracle_kat.py) and by frames rendered through the same compiled
traversal.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

DTYPE_CODES = {"f32": 0, "u8": 1, "f16": 2, "bf16": 3, "u16": 4}


class OrcScene(ctypes.Structure):
    _fields_ = [
        ("voxels", ctypes.c_void_p),
        ("dtype", ctypes.c_int),
        ("dims", ctypes.c_int * 3),
        ("origin", ctypes.c_float * 3),
        ("spacing", ctypes.c_float * 3),
        ("tf", ctypes.c_void_p),
        ("tfN", ctypes.c_int),
        ("domain", ctypes.c_float * 2),
        ("baseDensity", ctypes.c_float),
        ("camPos", ctypes.c_float * 3),
        ("camDir", ctypes.c_float * 3),
        ("camUp", ctypes.c_float * 3),
        ("fovy", ctypes.c_float),
        ("bgColor", ctypes.c_float * 4),
        ("ambientRadiance", ctypes.c_float),
        ("cutPlane", ctypes.c_float * 4),
        ("numDirLights", ctypes.c_int),
        ("dirLights", ctypes.c_void_p),
        ("phaseMode", ctypes.c_int),
        ("anisotropy", ctypes.c_float),
        ("scatteringAlbedo", ctypes.c_float),
        ("emissionAbsorption", ctypes.c_int),
        ("exactLog", ctypes.c_int),
        ("majorantRoundUp", ctypes.c_int),
        ("compensatedAccum", ctypes.c_int),
        ("maxVolumeBounces", ctypes.c_int),
        ("principled", ctypes.c_int),
        ("pDensity", ctypes.c_float), ("pDensityThreshold", ctypes.c_float), ("pDensityScale", ctypes.c_float),
        ("pValueRange", ctypes.c_float * 2),
        ("pEmissionStrength", ctypes.c_float), ("pBlackbodyIntensity", ctypes.c_float),
        ("pTemperature", ctypes.c_float),
        ("pScatterColor", ctypes.c_float * 3), ("pAbsorptionColor", ctypes.c_float * 3),
        ("pEmissionColor", ctypes.c_float * 3), ("pBlackbodyTint", ctypes.c_float * 3),
        ("iso", ctypes.c_int), ("isoValue", ctypes.c_float), ("isoColor", ctypes.c_float * 4),
        ("isoOpacity", ctypes.c_float), ("noVolume", ctypes.c_int),
        ("width", ctypes.c_int),
        ("height", ctypes.c_int),
    ]


class OrcStats(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_ulonglong), ("mcVisits", ctypes.c_ulonglong),
                ("rays", ctypes.c_ulonglong), ("pixelSamples", ctypes.c_ulonglong)]


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P, I, F, U32, U64, D = (ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_uint32,
                                ctypes.c_uint64, ctypes.c_double)
        L.orc_rng_stream.argtypes = [U32, U32, I, P]
        L.orc_rng_floats.argtypes = [U32, U32, I, P]
        L.orc_rng_derived.argtypes = [U64, U64, I, P, P]
        L.orc_hash3.argtypes = [U32, U32, U32]
        L.orc_hash3.restype = U64
        L.orc_fastlog.argtypes = [F]
        L.orc_fastlog.restype = F
        L.orc_f2h.argtypes = [F]
        L.orc_f2h.restype = ctypes.c_uint16
        L.orc_h2f.argtypes = [ctypes.c_uint16]
        L.orc_h2f.restype = F
        L.orc_mc_dims.argtypes = [P, P]
        L.orc_build_ranges.argtypes = [P, P]
        L.orc_map_majorants.argtypes = [P, P, ctypes.c_int64, P]
        L.orc_sample_points.argtypes = [P, I, P, P, P]
        L.orc_tf_map.argtypes = [P, I, P, P]
        L.orc_dda_cells.argtypes = [P, P, F, P, I, P, P]
        L.orc_dda_cells.restype = I
        L.orc_trace_primary.argtypes = [P, I, I, I, P, P, P]
        L.orc_tex3d.argtypes = [P, I, P, P]
        L.orc_trace_ray.argtypes = [P, P, P, F, U64, P, P, P, P]
        L.orc_principled.argtypes = [P, I, P, P, P]
        L.orc_render.argtypes = [P, I, I, P, P, I, I, I, I, I, P]
        L.orc_render.restype = D
        L.orc_resolve.argtypes = [P, P, ctypes.c_int64, I, I, P]
        L.orc64_render_expected.argtypes = [P, I, I, I, I, D, I, I, I, P]
        L.orc_sincos.argtypes = [I, P, P, P]
        L.orc_logp.argtypes = [I, P, P]
        L.orc_expp.argtypes = [I, P, P]
        L.orc_blackbody.argtypes = [F, P]
        L.orc_hg_sample.argtypes = [P, F, U64, I, P]
        L.orc_iso_trace.argtypes = [P, P, P, F, U64, P, P, P]
        L.orc_frame_xfm.argtypes = [P, P, P]
        _lib = L
    return _lib


def principled_params(p):
    """Principled volume parameters with the reference's defaults and the
    clamps of its setters (PrincipledVolume.h:17-30, Volume.cpp:36-126)."""
    p = dict(p or {})
    out = {"enabled": 1 if p.get("enabled", bool(p)) else 0,
           "density": float(p.get("density", 1.0)),
           "density_threshold": max(float(p.get("density_threshold", 0.0)), 0.0),
           "density_scale": float(p.get("density_scale", 1.0)),
           "value_range": tuple(float(x) for x in p.get("value_range", (0.0, 1.0))),
           "emission_strength": max(float(p.get("emission_strength", 0.0)), 0.0),
           "blackbody_intensity": max(float(p.get("blackbody_intensity", 0.0)), 0.0),
           "temperature": max(float(p.get("temperature", 0.0)), 0.0)}
    if not out["density_scale"] > 0.0:
        out["density_scale"] = 1.0
    for k, dflt in (("scatter_color", (0.8, 0.8, 0.8)), ("absorption_color", (0.0, 0.0, 0.0)),
                    ("emission_color", (1.0, 1.0, 1.0)), ("blackbody_tint", (1.0, 1.0, 1.0))):
        out[k] = tuple(max(float(x), 0.0) for x in p.get(k, dflt))
    return out


def iso_params(p):
    """Isosurface parameters: iso value and the AnariMatte material's constant
    color (rgb gives alpha 1) and opacity (AnariMatte.h:44-45 defaults .8 / 1)."""
    if not p:
        return {"enabled": 0, "value": 0.0, "color": (0.8, 0.8, 0.8, 1.0), "opacity": 1.0}
    c = tuple(float(x) for x in p.get("color", (0.8, 0.8, 0.8)))
    if len(c) == 3:
        c = c + (1.0,)
    return {"enabled": 1, "value": float(p["value"]), "color": c, "opacity": float(p.get("opacity", 1.0))}


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Scene:
    """Keeps the numpy arrays alive for the lifetime of the ctypes struct."""

    def __init__(self, desc):
        self.desc = desc
        vol = np.ascontiguousarray(desc["voxels"])
        self.vol = vol
        self.tf = np.ascontiguousarray(desc["tf"], dtype=np.float32).reshape(-1, 4)
        lights = desc.get("dir_lights", [])
        self.lights = np.array([[*l["direction"], l.get("radiance", 1.0), *l.get("color", (1, 1, 1))]
                                for l in lights], dtype=np.float32).reshape(-1, 7)
        s = OrcScene()
        s.voxels = vol.ctypes.data
        s.dtype = DTYPE_CODES[desc["dtype"]]
        nz, ny, nx = vol.shape  # numpy volumes are [z][y][x], x fastest
        s.dims[:] = (nx, ny, nz)
        s.origin[:] = desc.get("origin", (0.0, 0.0, 0.0))
        s.spacing[:] = desc["spacing"]
        s.tf = self.tf.ctypes.data
        s.tfN = self.tf.shape[0]
        s.domain[:] = desc.get("domain", (0.0, 1.0))
        s.baseDensity = desc["density"]
        cam = desc["camera"]
        s.camPos[:] = cam["position"]
        s.camDir[:] = cam["direction"]
        s.camUp[:] = cam.get("up", (0.0, 1.0, 0.0))
        s.fovy = cam.get("fovy", 60.0)
        s.bgColor[:] = desc.get("bg_color", (0.0, 0.0, 0.0, 1.0))
        s.ambientRadiance = desc.get("ambient", 1.0)
        s.cutPlane[:] = desc.get("cut_plane", (0.0, 0.0, 0.0, -1e30))
        s.numDirLights = self.lights.shape[0]
        s.dirLights = self.lights.ctypes.data if self.lights.size else None
        s.phaseMode = 1 if desc.get("phase", "simple") == "hg" else 0
        s.anisotropy = desc.get("anisotropy", 0.6)
        s.scatteringAlbedo = desc.get("scattering_albedo", 0.9)
        s.emissionAbsorption = int(desc.get("emission_absorption", False))
        s.exactLog = int(desc.get("exact_log", False))
        s.majorantRoundUp = int(desc.get("majorant_round_up", False))
        s.compensatedAccum = int(desc.get("compensated_accum", False))
        s.maxVolumeBounces = int(desc.get("max_volume_bounces", 0))
        pv = principled_params(desc.get("principled"))
        s.principled = pv["enabled"]
        s.pDensity, s.pDensityThreshold, s.pDensityScale = pv["density"], pv["density_threshold"], pv["density_scale"]
        s.pValueRange[:] = pv["value_range"]
        s.pEmissionStrength, s.pBlackbodyIntensity = pv["emission_strength"], pv["blackbody_intensity"]
        s.pTemperature = pv["temperature"]
        s.pScatterColor[:], s.pAbsorptionColor[:] = pv["scatter_color"], pv["absorption_color"]
        s.pEmissionColor[:], s.pBlackbodyTint[:] = pv["emission_color"], pv["blackbody_tint"]
        iso = iso_params(desc.get("iso"))
        s.iso = iso["enabled"]
        s.isoValue = iso["value"]
        s.isoColor[:] = iso["color"]
        s.isoOpacity = iso["opacity"]
        s.noVolume = 0 if desc.get("volume", True) else 1
        s.width, s.height = desc["width"], desc["height"]
        self.s = s

    @property
    def ref(self):
        return ctypes.byref(self.s)


def rng_stream(a, b, n):
    out = np.zeros(n, np.uint32)
    lib().orc_rng_stream(a, b, n, _ptr(out))
    return out


def rng_floats(a, b, n):
    out = np.zeros(n, np.float32)
    lib().orc_rng_floats(a, b, n, _ptr(out))
    return out


def rng_derived(parent_state, h, n):
    out = np.zeros(n, np.uint32)
    parent = ctypes.c_uint64(0)
    lib().orc_rng_derived(parent_state, h, n, _ptr(out), ctypes.byref(parent))
    return out, parent.value


def hash3(a, b, c):
    return lib().orc_hash3(a, b, c)


def fastlog(f):
    return lib().orc_fastlog(f)


def f2h(f):
    return lib().orc_f2h(f)


def sincos(x):
    """The portable binary32 sin/cos shared by the oracle and the kernels."""
    x = np.ascontiguousarray(x, np.float32)
    sn, cs = np.empty_like(x), np.empty_like(x)
    lib().orc_sincos(x.size, _ptr(x), _ptr(sn), _ptr(cs))
    return sn, cs


def logp(x):
    """The portable binary32 natural log shared by the oracle and the kernels."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    lib().orc_logp(x.size, _ptr(x), _ptr(out))
    return out


def expp(x):
    """The portable binary32 exponential shared by the oracle and the kernels."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    lib().orc_expp(x.size, _ptr(x), _ptr(out))
    return out


def blackbody(kelvin):
    out = np.empty(3, np.float32)
    lib().orc_blackbody(kelvin, _ptr(out))
    return out


def hg_sample(wi, g, seed_state, n):
    """n directions of HGPhase::sampleDirection from one RNG state."""
    wi = np.ascontiguousarray(wi, np.float32)
    out = np.empty((n, 3), np.float32)
    lib().orc_hg_sample(_ptr(wi), g, seed_state, n, _ptr(out))
    return out


def iso_trace(sc, org, dir, tmax=1e30, seed_state=0xcafef00dd15ea5e5):
    """One ray against the scene's isosurface: (hit, t, stored normal)."""
    org = np.ascontiguousarray(org, np.float32)
    dir = np.ascontiguousarray(dir, np.float32)
    hit, t = ctypes.c_int(0), ctypes.c_float(0.0)
    n = np.zeros(3, np.float32)
    lib().orc_iso_trace(sc.ref, _ptr(org), _ptr(dir), tmax, seed_state, ctypes.byref(hit), ctypes.byref(t), _ptr(n))
    return bool(hit.value), t.value, n


def frame_xfm(N, v):
    """owl::common::frame(N) applied to v (the Lambertian's local-to-world map)."""
    N = np.ascontiguousarray(N, np.float32)
    v = np.ascontiguousarray(v, np.float32)
    out = np.zeros(3, np.float32)
    lib().orc_frame_xfm(_ptr(N), _ptr(v), _ptr(out))
    return out


def mc_dims(sc):
    out = np.zeros(3, np.int32)
    lib().orc_mc_dims(sc.ref, _ptr(out))
    return tuple(int(v) for v in out)


def build_ranges(sc):
    d = mc_dims(sc)
    out = np.zeros((d[2], d[1], d[0], 2), np.float32)
    lib().orc_build_ranges(sc.ref, _ptr(out))
    return out


def map_majorants(sc, ranges):
    ranges = np.ascontiguousarray(ranges, np.float32)
    out = np.zeros(ranges.shape[:-1], np.float32)
    lib().orc_map_majorants(sc.ref, _ptr(ranges), out.size, _ptr(out))
    return out


def sample_points(sc, P):
    P = np.ascontiguousarray(P, np.float32).reshape(-1, 3)
    scal = np.zeros(P.shape[0], np.float32)
    rgba = np.zeros((P.shape[0], 4), np.float32)
    lib().orc_sample_points(sc.ref, P.shape[0], _ptr(P), _ptr(scal), _ptr(rgba))
    return scal, rgba


def tf_map(sc, v):
    v = np.ascontiguousarray(v, np.float32).reshape(-1)
    rgba = np.zeros((v.size, 4), np.float32)
    lib().orc_tf_map(sc.ref, v.size, _ptr(v), _ptr(rgba))
    return rgba


def tex3d(sc, tc):
    """LINEAR tex3D of the scene's field at unnormalized texel coordinates."""
    tc = np.ascontiguousarray(tc, np.float32).reshape(-1, 3)
    out = np.zeros(tc.shape[0], np.float32)
    lib().orc_tex3d(sc.ref, tc.shape[0], _ptr(tc), _ptr(out))
    return out


def trace_ray(sc, org, dir, tmax, seed_state):
    """One ray with an explicit RNG seed state through the volume: (hit, t,
    rgb at the collision, [samples, macrocell visits])."""
    org = np.ascontiguousarray(org, np.float32)
    dir = np.ascontiguousarray(dir, np.float32)
    hit, t = ctypes.c_int(0), ctypes.c_float(0.0)
    rgb = np.zeros(3, np.float32)
    counts = np.zeros(2, np.int32)
    lib().orc_trace_ray(sc.ref, _ptr(org), _ptr(dir), tmax, seed_state, ctypes.byref(hit), ctypes.byref(t),
                        _ptr(rgb), _ptr(counts))
    return bool(hit.value), t.value, rgb, counts


def trace_primary(sc, ix, iy, accum_id):
    """The primary ray of pixel (ix, iy) at accum_id: (hit, t, rgb)."""
    hit, t = ctypes.c_int(0), ctypes.c_float(0.0)
    rgb = np.zeros(3, np.float32)
    lib().orc_trace_primary(sc.ref, ix, iy, accum_id, ctypes.byref(hit), ctypes.byref(t), _ptr(rgb))
    return bool(hit.value), t.value, rgb


def principled(sc, v):
    """The principled volume's sampleMap (tint rgb, sigma_t) and emission."""
    v = np.ascontiguousarray(v, np.float32).reshape(-1)
    m = np.zeros((v.size, 4), np.float32)
    e = np.zeros((v.size, 3), np.float32)
    lib().orc_principled(sc.ref, v.size, _ptr(v), _ptr(m), _ptr(e))
    return m, e


def dda_cells(org, dir, tmax, grid, max_cells=4096):
    org = np.asarray(org, np.float32)
    dir = np.asarray(dir, np.float32)
    grid = np.asarray(grid, np.int32)
    cells = np.zeros((max_cells, 3), np.int32)
    ts = np.zeros((max_cells, 2), np.float32)
    n = lib().orc_dda_cells(_ptr(org), _ptr(dir), tmax, _ptr(grid), max_cells, _ptr(cells), _ptr(ts))
    return cells[:n], ts[:n]


def render(sc, accum_id0, spp, accum=None, rect=None, threads=0, comp=None):
    """Accumulate spp waves into a (H, W, 4) float32 buffer; returns (accum, seconds, stats).
    comp: (H, W, 4) compensation buffer of the compensated-accumulation form."""
    W, H = sc.s.width, sc.s.height
    if accum is None:
        accum = np.zeros((H, W, 4), np.float32)
    x0, y0, x1, y1 = rect if rect is not None else (0, 0, W, H)
    st = OrcStats()
    secs = lib().orc_render(sc.ref, accum_id0, spp, _ptr(accum), _ptr(comp) if comp is not None else None,
                            x0, y0, x1, y1, threads, ctypes.byref(st))
    return accum, secs, {"samples": st.samples, "mc_visits": st.mcVisits, "rays": st.rays,
                         "pixel_samples": st.pixelSamples}


def resolve(accum, accum_id, fmt="float4", comp=None):
    code = {"float4": 0, "rgba8": 1, "rgba8_srgb": 2}[fmt]
    n = accum.shape[0] * accum.shape[1]
    if code == 0:
        out = np.zeros(accum.shape, np.float32)
    else:
        out = np.zeros(accum.shape[:2], np.uint32)
    cp = _ptr(np.ascontiguousarray(comp)) if comp is not None else None
    lib().orc_resolve(_ptr(np.ascontiguousarray(accum)), cp, n, accum_id, code, _ptr(out))
    return out


def render_expected_fp64(sc, rect=None, step=None, subpix=2, env_dirs=64, threads=0):
    if sc.s.maxVolumeBounces > 0:
        raise ValueError("the FP64 expectation covers single scattering only")
    W, H = sc.s.width, sc.s.height
    x0, y0, x1, y1 = rect if rect is not None else (0, 0, W, H)
    if step is None:
        step = 0.5 * min(sc.s.spacing[:3])
    out = np.zeros((H, W, 4), np.float64)
    lib().orc64_render_expected(sc.ref, x0, y0, x1, y1, step, subpix, env_dirs, threads, _ptr(out))
    return out
