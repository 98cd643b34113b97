"""The reference's own hot-path code, compiled here -- TEST INFRASTRUCTURE ONLY.

ctypes bindings to ``oracle/_ref/libbnref.so``, which ``oracle/Makefile``
(target ``ref``) compiles from the reference's sources where they lie (its
RNG and hash, fastLog, Woodcock::sampleRange, sampleAndMap, dda3, the
transfer function's map and majorant, the principled-volume functions,
linear_to_srgb / make_rgba, and its CPU backend's texture samplers and
binary16 rounding), behind the stand-in include tree ``oracle/refshim`` and
the glue in ``oracle/ref_harness.cpp``.

Only ``tests/golden/make_ref_golden.py`` calls this module: the reference
exists in the build container, not on GPU machines, so its outputs are
committed as ``tests/golden/ref_*.npz`` and the tests read those.
"""
import ctypes
import os
import subprocess

import numpy as np

from . import Scene  # noqa: F401  (scene description shared with the oracle)

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_ref", "libbnref.so")
_lib = None


def build(ref_root="/root/reference"):
    """Compile oracle/_ref/libbnref.so from the reference tree at ref_root."""
    subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={ref_root}"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P, I, F, U32, U64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_uint32, ctypes.c_uint64
        L.ref_rng_stream.argtypes = [U32, U32, I, P]
        L.ref_rng_floats.argtypes = [U32, U32, I, P]
        L.ref_rng_derived.argtypes = [U64, U64, I, P, P]
        L.ref_ray_seed.argtypes = [U32, U32]
        L.ref_ray_seed.restype = U64
        L.ref_hash3.argtypes = [U32, U32, U32]
        L.ref_hash3.restype = U64
        L.ref_fastlog.argtypes = [I, P, P]
        L.ref_f2h.argtypes = [I, P, P]
        L.ref_h2f.argtypes = [I, P, P]
        L.ref_linear_to_srgb.argtypes = [I, P, P]
        L.ref_make_rgba.argtypes = [I, P, P]
        L.ref_tex3d.argtypes = [P, I, I, P, P]
        L.ref_sample_points.argtypes = [P, I, P, P, P]
        L.ref_tf_map.argtypes = [P, I, P, P]
        L.ref_mc_dims.argtypes = [P, P]
        L.ref_build_ranges.argtypes = [P, P]
        L.ref_map_majorants.argtypes = [P, P, ctypes.c_int64, P]
        L.ref_principled.argtypes = [P, I, P, P, P]
        L.ref_dda_cells.argtypes = [P, P, F, P, I, P, P]
        L.ref_dda_cells.restype = I
        L.ref_trace_ray.argtypes = [P, P, P, F, U64, P, P, P, P]
        L.ref_trace_frame.argtypes = [P, I, P, P, P, P]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f32(x):
    return np.ascontiguousarray(x, np.float32)


def rng_stream(a, b, n):
    out = np.zeros(n, np.uint32)
    lib().ref_rng_stream(a, b, n, _ptr(out))
    return out


def rng_floats(a, b, n):
    out = np.zeros(n, np.float32)
    lib().ref_rng_floats(a, b, n, _ptr(out))
    return out


def rng_derived(parent_state, h, n):
    out = np.zeros(n, np.uint32)
    parent = ctypes.c_uint64(0)
    lib().ref_rng_derived(parent_state, h, n, _ptr(out), ctypes.byref(parent))
    return out, parent.value


def ray_seed(a, b):
    return lib().ref_ray_seed(a, b)


def hash3(a, b, c):
    return lib().ref_hash3(a, b, c)


def _unary(fn, x, out_dtype=np.float32, in_dtype=np.float32):
    x = np.ascontiguousarray(x, in_dtype).reshape(-1)
    out = np.zeros(x.size, out_dtype)
    fn(x.size, _ptr(x), _ptr(out))
    return out


def fastlog(x):
    return _unary(lib().ref_fastlog, x)


def f2h(x):
    return _unary(lib().ref_f2h, x, np.uint16)


def h2f(bits):
    return _unary(lib().ref_h2f, bits, np.float32, np.uint16)


def linear_to_srgb(x):
    return _unary(lib().ref_linear_to_srgb, x)


def make_rgba(rgba):
    rgba = _f32(rgba).reshape(-1, 4)
    out = np.zeros(rgba.shape[0], np.uint32)
    lib().ref_make_rgba(rgba.shape[0], _ptr(rgba), _ptr(out))
    return out


def tex3d(sc, tc, linear=True):
    tc = _f32(tc).reshape(-1, 3)
    out = np.zeros(tc.shape[0], np.float32)
    lib().ref_tex3d(sc.ref, 1 if linear else 0, tc.shape[0], _ptr(tc), _ptr(out))
    return out


def sample_points(sc, P):
    P = _f32(P).reshape(-1, 3)
    scal = np.zeros(P.shape[0], np.float32)
    rgba = np.zeros((P.shape[0], 4), np.float32)
    lib().ref_sample_points(sc.ref, P.shape[0], _ptr(P), _ptr(scal), _ptr(rgba))
    return scal, rgba


def tf_map(sc, v):
    v = _f32(v).reshape(-1)
    rgba = np.zeros((v.size, 4), np.float32)
    lib().ref_tf_map(sc.ref, v.size, _ptr(v), _ptr(rgba))
    return rgba


def mc_dims(sc):
    out = np.zeros(3, np.int32)
    lib().ref_mc_dims(sc.ref, _ptr(out))
    return tuple(int(v) for v in out)


def build_ranges(sc):
    d = mc_dims(sc)
    out = np.zeros((d[2], d[1], d[0], 2), np.float32)
    lib().ref_build_ranges(sc.ref, _ptr(out))
    return out


def map_majorants(sc, ranges):
    ranges = _f32(ranges)
    out = np.zeros(ranges.shape[:-1], np.float32)
    lib().ref_map_majorants(sc.ref, _ptr(ranges), out.size, _ptr(out))
    return out


def principled(sc, v):
    v = _f32(v).reshape(-1)
    m = np.zeros((v.size, 4), np.float32)
    e = np.zeros((v.size, 3), np.float32)
    lib().ref_principled(sc.ref, v.size, _ptr(v), _ptr(m), _ptr(e))
    return m, e


def dda_cells(org, dir, tmax, grid, max_cells=4096):
    org, dir = _f32(org), _f32(dir)
    grid = np.ascontiguousarray(grid, np.int32)
    cells = np.zeros((max_cells, 3), np.int32)
    ts = np.zeros((max_cells, 2), np.float32)
    n = lib().ref_dda_cells(_ptr(org), _ptr(dir), tmax, _ptr(grid), max_cells, _ptr(cells), _ptr(ts))
    return cells[:n], ts[:n]


def trace_ray(sc, org, dir, tmax, seed_state):
    org, dir = _f32(org), _f32(dir)
    hit, t = ctypes.c_int(0), ctypes.c_float(0.0)
    rgb = np.zeros(3, np.float32)
    counts = np.zeros(2, np.int32)
    lib().ref_trace_ray(sc.ref, _ptr(org), _ptr(dir), tmax, seed_state, ctypes.byref(hit), ctypes.byref(t),
                        _ptr(rgb), _ptr(counts))
    return bool(hit.value), t.value, rgb, counts


def trace_frame(sc, accum_id):
    """Primary-ray first collisions of every pixel at accum_id: hit (H, W),
    t (H, W), rgb (H, W, 3), counts (H, W, 2) = samples, macrocell visits."""
    W, H = sc.s.width, sc.s.height
    hit = np.zeros((H, W), np.int32)
    t = np.zeros((H, W), np.float32)
    rgb = np.zeros((H, W, 3), np.float32)
    counts = np.zeros((H, W, 2), np.int32)
    lib().ref_trace_frame(sc.ref, accum_id, _ptr(hit), _ptr(t), _ptr(rgb), _ptr(counts))
    return hit, t, rgb, counts
