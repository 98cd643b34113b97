"""Seeded synthetic structured volumes, transfer functions and scenes.

These stand in for user data on the structured-volume path: a
``dims``-sized scalar grid on the unit cube (``gridOrigin`` 0,
``gridSpacing`` 1/(N-1)), a 1D RGBA transfer function and a camera.

Two field generators:

* ``blobs(n, seed)``: sum of 8 isotropic Gaussians, centres U[0,1]^3,
  sigma U[0.05, 0.2], amplitude U[0.2, 1], drawn from
  ``numpy.random.default_rng(seed)`` in that order; not clamped.
* ``value_noise(n, seed)``: 6-octave value noise.  Lattice values are the
  PCG hash of Jarzynski & Olano ("Hash Functions for GPU Rendering", JCGT
  2020) chained over (ix, iy, iz, octave, seed) divided by 2^32; quintic
  fade (6t^5 - 15t^4 + 10t^3) trilinear interpolation; base frequency 4
  lattice cells per unit, lacunarity 2, gain 0.5; the octave sum is divided
  by the amplitude sum 1.96875 so values lie in [0, 1].  All arithmetic is
  float64 and rounded once to float32, so the numpy path and the torch
  (CUDA) path give bit-identical volumes.

Both accept ``xp`` = numpy (default) or torch; with torch, tensors are made
on ``device`` and the field is generated slab by slab.
"""
import math

import numpy as np

_MASK = 0xFFFFFFFF


def _pcg(x):
    state = (x * 747796405 + 2891336453) & _MASK
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & _MASK
    return ((word >> 22) ^ word) & _MASK


def _lattice(ix, iy, iz, octave, seed):
    h = int(_pcg(octave + int(_pcg(seed))))
    return _pcg((ix + _pcg((iy + _pcg((iz + h) & _MASK)) & _MASK)) & _MASK)


def _fade(t):
    return t * t * t * (t * (t * 6.0 - 15.0) + 10.0)


def _noise_slab(xp, zc, yc, xc, seed, octaves=6, base=4.0):
    """zc, yc, xc: broadcastable float64 coordinate arrays in [0, 1]."""
    total = 0.0
    amp_sum = 0.0
    for k in range(octaves):
        f = base * (2.0 ** k)
        a = 0.5 ** k
        pz, py, px = zc * f, yc * f, xc * f
        fz, fy, fx = xp.floor(pz), xp.floor(py), xp.floor(px)
        tz, ty, tx = _fade(pz - fz), _fade(py - fy), _fade(px - fx)
        if xp is np:
            iz, iy, ix = fz.astype(np.int64), fy.astype(np.int64), fx.astype(np.int64)
        else:
            iz, iy, ix = fz.long(), fy.long(), fx.long()
        acc = None
        for dz in (0, 1):
            wz = tz if dz else (1.0 - tz)
            for dy in (0, 1):
                wy = ty if dy else (1.0 - ty)
                for dx in (0, 1):
                    wx = tx if dx else (1.0 - tx)
                    v = _lattice(ix + dx, iy + dy, iz + dz, k, seed)
                    v = v.astype(np.float64) if xp is np else v.double()
                    term = (wz * wy) * wx * (v * (1.0 / 4294967296.0))
                    acc = term if acc is None else acc + term
        total = total + a * acc
        amp_sum += a
    return total / amp_sum


def value_noise(n, seed, xp=np, device=None, slab=16, out_dtype=None):
    """n^3 float32 volume [z][y][x] of 6-octave value noise in [0,1]."""
    inv = 1.0 / (n - 1)
    if xp is np:
        out = np.empty((n, n, n), np.float32)
        x = (np.arange(n, dtype=np.float64) * inv)[None, None, :]
        y = (np.arange(n, dtype=np.float64) * inv)[None, :, None]
        for z0 in range(0, n, slab):
            z = (np.arange(z0, min(n, z0 + slab), dtype=np.float64) * inv)[:, None, None]
            out[z0:z0 + z.shape[0]] = _noise_slab(np, z, y, x, seed).astype(np.float32)
        return out
    import torch
    out = torch.empty((n, n, n), dtype=torch.float32, device=device)
    x = (torch.arange(n, dtype=torch.float64, device=device) * inv)[None, None, :]
    y = (torch.arange(n, dtype=torch.float64, device=device) * inv)[None, :, None]
    for z0 in range(0, n, slab):
        z = (torch.arange(z0, min(n, z0 + slab), dtype=torch.float64, device=device) * inv)[:, None, None]
        out[z0:z0 + z.shape[0]] = _noise_slab(torch, z, y, x, seed).float()
    return out


def blob_params(seed):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, 1.0, size=(8, 3))
    sigma = rng.uniform(0.05, 0.2, size=8)
    amp = rng.uniform(0.2, 1.0, size=8)
    return centres, sigma, amp


def blobs(n, seed=0, xp=np, device=None):
    """n^3 float32 volume [z][y][x]: sum of 8 Gaussian blobs (seeded)."""
    centres, sigma, amp = blob_params(seed)
    inv = 1.0 / (n - 1)
    if xp is np:
        c = np.arange(n, dtype=np.float64) * inv
        z, y, x = c[:, None, None], c[None, :, None], c[None, None, :]
        f = np.zeros((n, n, n), np.float64)
        for (cx, cy, cz), s, a in zip(centres, sigma, amp):
            d2 = (x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2
            f += a * np.exp(-d2 / (2.0 * s * s))
        return f.astype(np.float32)
    import torch
    c = torch.arange(n, dtype=torch.float64, device=device) * inv
    out = torch.empty((n, n, n), dtype=torch.float32, device=device)
    for z0 in range(0, n, 32):
        z = c[z0:z0 + 32][:, None, None]
        y, x = c[None, :, None], c[None, None, :]
        f = torch.zeros((z.shape[0], n, n), dtype=torch.float64, device=device)
        for (cx, cy, cz), s, a in zip(centres, sigma, amp):
            d2 = (x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2
            f += a * torch.exp(-d2 / (2.0 * s * s))
        out[z0:z0 + z.shape[0]] = f.float()
    return out


def to_storage(vol_f32, dtype):
    """Stored form of a [0,1] float32 field: f32 as is, u8 = round(255 v),
    u16 = round(65535 v), f16 / bf16 by round-to-nearest-even (returned as
    16-bit patterns)."""
    if dtype == "f32":
        return vol_f32
    if isinstance(vol_f32, np.ndarray):
        if dtype == "u8":
            return np.clip(np.rint(vol_f32.astype(np.float64) * 255.0), 0, 255).astype(np.uint8)
        if dtype == "u16":
            return np.clip(np.rint(vol_f32.astype(np.float64) * 65535.0), 0, 65535).astype(np.uint16)
        if dtype == "f16":
            return vol_f32.astype(np.float16).view(np.uint16)
        if dtype == "bf16":
            u = vol_f32.view(np.uint32).astype(np.uint64)
            r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
            return r
    import torch
    if dtype == "u8":
        return torch.clamp(torch.round(vol_f32.double() * 255.0), 0, 255).to(torch.uint8)
    if dtype == "u16":
        return torch.clamp(torch.round(vol_f32.double() * 65535.0), 0, 65535).to(torch.int32).to(torch.int16)
    if dtype == "f16":
        return vol_f32.half().view(torch.int16)
    if dtype == "bf16":
        return vol_f32.bfloat16().view(torch.int16)
    raise ValueError(dtype)


# ---------------------------------------------------------------------------
# transfer functions
# ---------------------------------------------------------------------------
def tf_linear_ramp(n):
    """Opacity ramp 0->1, colour ramp blue->red: rgba[i] = (t, 0, 1-t, t)."""
    t = np.arange(n, dtype=np.float64) / (n - 1)
    return np.stack([t, np.zeros_like(t), 1.0 - t, t], axis=1).astype(np.float32)


def tf_knots(n, seed=1, knots=4):
    """Piecewise-linear opacity through `knots` seeded knots (x sorted
    U[0,1], y U[0,1], constant extrapolation), colour ramp blue->red."""
    rng = np.random.default_rng(seed)
    kx = np.sort(rng.uniform(0.0, 1.0, size=knots))
    ky = rng.uniform(0.0, 1.0, size=knots)
    t = np.arange(n, dtype=np.float64) / (n - 1)
    op = np.interp(t, kx, ky)
    return np.stack([t, np.zeros_like(t), 1.0 - t, op], axis=1).astype(np.float32)


# ---------------------------------------------------------------------------
# cameras and scene descriptions
# ---------------------------------------------------------------------------
CUBE_CENTRE = (0.5, 0.5, 0.5)


def look_at(position, target=CUBE_CENTRE, fovy=45.0, up=(0.0, 1.0, 0.0)):
    d = tuple(float(t) - float(p) for p, t in zip(position, target))
    return {"position": tuple(float(v) for v in position), "direction": d, "up": up, "fovy": fovy}


def orbit_camera(rng, radius=2.5, fovy=45.0):
    az = rng.uniform(0.0, 2 * math.pi)
    el = math.radians(rng.uniform(-30.0, 60.0))
    p = (0.5 + radius * math.cos(el) * math.cos(az), 0.5 + radius * math.sin(el),
         0.5 + radius * math.cos(el) * math.sin(az))
    return look_at(p, fovy=fovy)


def scene(voxels, dtype, width, height, tf, density, camera, **kw):
    """Scene description dict consumed by the API wrapper and the oracle."""
    d = {"voxels": voxels, "dtype": dtype, "origin": (0.0, 0.0, 0.0),
         "spacing": (1.0 / (voxels.shape[2] - 1), 1.0 / (voxels.shape[1] - 1), 1.0 / (voxels.shape[0] - 1)),
         "tf": tf, "domain": (0.0, 1.0), "density": float(density), "camera": camera,
         "width": int(width), "height": int(height), "bg_color": (0.0, 0.0, 0.0, 1.0),
         "ambient": 1.0, "dir_lights": [], "phase": "simple"}
    d.update(kw)
    return d


DEFAULT_CAMERA = look_at((2.0, 1.5, 2.0))
CONFIG2_LIGHTS = [{"direction": (-1.0, -1.0, -1.0), "radiance": 1.0, "color": (1.0, 1.0, 1.0)}]


def config1(reference_semantics=True, spp=16):
    """64^3 f32 Gaussian blobs (seed 0), 256x256, 128-entry linear TF,
    density 50.  reference_semantics: ambient 1, no lights, default-build
    single scatter; otherwise the emission-absorption extension."""
    vol = blobs(64, 0)
    kw = {"ambient": 1.0} if reference_semantics else {"emission_absorption": True, "ambient": 0.0}
    d = scene(vol, "f32", 256, 256, tf_linear_ramp(128), 50.0, DEFAULT_CAMERA, **kw)
    d["spp"] = spp
    return d


def config2(n=512, width=1920, height=1080, spp=64, dtype="f32", vol=None, xp=np, device=None):
    """n^3 value noise (seed 0), 256-entry knot TF (seed 1), density 50,
    directional light normalize(-1,-1,-1) + ambient 0.25, isotropic HG
    phase with scattering albedo 0.8 (multi-scatter build semantics with
    maxVolumeBounces = 0)."""
    if vol is None:
        vol = to_storage(value_noise(n, 0, xp=xp, device=device), dtype)
    d = scene(vol, dtype, width, height, tf_knots(256, 1), 50.0, DEFAULT_CAMERA,
              ambient=0.25, dir_lights=CONFIG2_LIGHTS, phase="hg", anisotropy=0.0,
              scattering_albedo=0.8)
    d["spp"] = spp
    return d


def config4_jobs(n_jobs=64, xp=np, device=None):
    """The batching workload: job i draws from default_rng(i) a volume edge
    log-uniform in [32, 256], a field (Gaussian blobs or value noise, seeded
    by i), a storage type from {u8, f16, f32}, an image side log-uniform in
    [128, 1024], spp from {1, 4, 16, 32} and an orbit camera (azimuth
    U[0, 2pi), elevation U[-30, 60] degrees, radius 2.5 about the cube
    centre).  Blob jobs use the config-1 look (linear TF, ambient 1, default
    single scatter); noise jobs the config-2 look (knot TF, HG albedo 0.8,
    directional light + ambient 0.25)."""
    jobs = []
    for i in range(n_jobs):
        rng = np.random.default_rng(i)
        edge = int(round(math.exp(rng.uniform(math.log(32), math.log(256)))))
        field = "blobs" if rng.integers(2) == 0 else "noise"
        dtype = ["u8", "f16", "f32"][int(rng.integers(3))]
        side = int(round(math.exp(rng.uniform(math.log(128), math.log(1024)))))
        spp = [1, 4, 16, 32][int(rng.integers(4))]
        cam = orbit_camera(rng)
        if field == "blobs":
            vol = to_storage(blobs(edge, i, xp=xp, device=device), dtype)
            d = scene(vol, dtype, side, side, tf_linear_ramp(128), 50.0, cam, ambient=1.0)
        else:
            vol = to_storage(value_noise(edge, i, xp=xp, device=device), dtype)
            d = config2(vol=vol, dtype=dtype, width=side, height=side, spp=spp)
            d["camera"] = cam
        d["spp"] = spp
        d["field"] = field
        jobs.append(d)
    return jobs
