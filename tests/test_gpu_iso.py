"""Isosurfaces on the structured field (MCIsoSurfaceAccel::isProg with an
AnariMatte material): every pixel, every counter and every accumulated sum
equal the oracle's restatement -- the macrocell-range DDA with ten linear
steps per candidate cell, the central-difference normal stored in binary16,
the Lambertian shadow ray and the one diffuse bounce, next to a volume on
the same field or alone."""
import ctypes

import numpy as np
import pytest

from barney_b200 import synth
from tests.helpers import assert_bitexact, gpu_render, oracle_render, small_blob_scene, small_noise_scene
from tests.test_oracle_kat import ramp_scene

pytestmark = pytest.mark.gpu

ISO_SCENES = {
    "ramp_plane_light": lambda: ramp_scene(0.37, ambient=0.0,
                                           dir_lights=[{"direction": (-1.0, 0.0, 0.0), "radiance": 1.0}]),
    "ramp_plane_ambient": lambda: ramp_scene(0.61, ambient=0.7),
    "blobs_alone": lambda: small_blob_scene(n=32, w=48, h=40, volume=False, ambient=0.3,
                                            dir_lights=synth.CONFIG2_LIGHTS,
                                            iso={"value": 0.3, "color": (0.9, 0.5, 0.2)}),
    "blobs_rgba_half_opaque": lambda: small_blob_scene(n=32, w=48, h=40, volume=False, ambient=0.5,
                                                       iso={"value": 0.25, "color": (0.2, 0.9, 0.4, 0.8),
                                                            "opacity": 0.6}),
    "noise_with_volume_simple": lambda: small_noise_scene(phase="simple", iso={"value": 0.55}),
    "noise_with_volume_hg": lambda: small_noise_scene(iso={"value": 0.55, "color": (0.3, 0.6, 0.9)}),
    "noise_multiscatter": lambda: small_noise_scene(phase="hg", anisotropy=0.5, max_volume_bounces=3,
                                                    iso={"value": 0.5, "color": (0.8, 0.7, 0.2), "opacity": 0.8}),
    "noise_u8_cut_plane": lambda: small_noise_scene(dtype="u8", iso={"value": 0.45},
                                                    cut_plane=(0.0, 1.0, 0.0, -0.5)),
    "noise_f16_alone_exact_log": lambda: small_noise_scene(dtype="f16", volume=False, exact_log=True,
                                                           iso={"value": 0.6}),
    # edge cases: an iso value never set (NaN: no macrocell qualifies, the
    # walk still derives its RNG), an iso value on voxel values exactly, and
    # plateaus at the iso value (0/0 segments) on a clamped ramp
    "nan_iso_value": lambda: small_noise_scene(iso={"value": float("nan")}),
    "iso_on_voxel_values": lambda: ramp_scene(0.5, ambient=0.6),
    "iso_plateau": lambda: _plateau_scene(),
}


def _plateau_scene():
    d = ramp_scene(0.25, ambient=0.6, dir_lights=[{"direction": (-1.0, -0.2, 0.1), "radiance": 1.0}])
    d["voxels"] = np.clip(d["voxels"], np.float32(0.25), np.float32(0.75))
    d["camera"] = {"position": (1.8, 1.4, 1.6), "direction": (-1.3, -0.9, -1.1), "up": (0.0, 1.0, 0.0),
                   "fovy": 40.0}
    return d


@pytest.mark.parametrize("name", sorted(ISO_SCENES))
def test_iso_bitexact(name):
    d = ISO_SCENES[name]()
    for spp in (1, 4):
        img, st = gpu_render(d, spp)
        ref, _, ost = oracle_render(d, spp)
        assert_bitexact(img, ref, f"{name} spp={spp}")
        assert st["samples"] == ost["samples"]
        assert st["mc_visits"] == ost["mc_visits"]
        assert st["rays"] == ost["rays"]
        assert st["error_flags"] == 0


def test_iso_value_change_takes_effect_on_the_next_render():
    import barney_b200 as bn
    d = small_noise_scene(iso={"value": 0.55})
    r = bn.VolumeRenderer(d)
    try:
        r.set_spp(2)
        r.render()
        r.accum_reset()
        r.set_iso(value=0.4, color=(0.1, 0.2, 0.9))
        r.render()
        ref, _, _ = oracle_render(dict(d, iso={"value": 0.4, "color": (0.1, 0.2, 0.9)}), 2)
        assert_bitexact(r.read(), ref, "after set_iso")
    finally:
        r.close()


def test_iso_jobs_in_a_batch_equal_solo_renders():
    import barney_b200 as bn
    descs = [small_noise_scene(iso={"value": 0.5}),
             small_noise_scene(w=24, h=20),  # no isosurface in the same launch
             small_blob_scene(volume=False, iso={"value": 0.3}, ambient=0.6)]
    ctx = bn.Context()
    rs = [bn.VolumeRenderer(d, context=ctx) for d in descs]
    try:
        for r in rs:
            r.set_spp(2)
        ctx.render_batch(rs)
        for r, d in zip(rs, descs):
            ref, _, _ = oracle_render(d, 2)
            assert_bitexact(r.read(), ref, f"batch job {d['width']}x{d['height']}")
    finally:
        for r in rs:
            r.close()
        ctx.close()


def test_iso_api_errors():
    import barney_b200 as bn
    r = bn.VolumeRenderer(small_noise_scene(iso={"value": 0.5}))
    L = r.L
    try:
        L.bnClearLastError()
        assert not L.bnGeometryCreate(r.ctx, 0, b"triangles")
        assert L.bnGetLastError() == 3
        L.bnClearLastError()
        assert not L.bnMaterialCreate(r.ctx, 0, b"glass")
        assert L.bnGetLastError() == 3
        L.bnClearLastError()
        L.bnSetObject(r.iso, b"scalarField", r.vol)  # not a scalar field
        assert L.bnGetLastError() == 2
        L.bnClearLastError()
        L.bnSetData(r.iso, b"isoValues", None)  # as the ANARI device sets it; unused
        assert L.bnGetLastError() == 0
        # a material that was never committed
        m = L.bnMaterialCreate(r.ctx, 0, b"AnariMatte")
        L.bnSetObject(r.iso, b"material", m)
        L.bnRender(r.renderer, r.model, r.camera, r.fb)
        assert L.bnGetLastError() == 5
        L.bnClearLastError()
        L.bnCommit(m)
        L.bnRender(r.renderer, r.model, r.camera, r.fb)
        assert L.bnGetLastError() == 0
        # an isosurface on another field than the group's volume
        other = L.bnScalarFieldCreate(r.ctx, 0, b"structured")
        L.bnSetObject(other, b"textureData", r.td)
        nz, ny, nx = r.desc["voxels"].shape
        L.bnSet3i(other, b"dims", nx, ny, nz)
        L.bnCommit(other)
        L.bnSetObject(r.iso, b"scalarField", other)
        L.bnRender(r.renderer, r.model, r.camera, r.fb)
        assert L.bnGetLastError() == 3
        L.bnClearLastError()
        L.bnSetObject(r.iso, b"scalarField", r.sf)
        # emission-absorption mode has no isosurfaces
        L.bnSet1i(r.renderer, b"bnx.emissionAbsorption", 1)
        L.bnCommit(r.renderer)
        L.bnRender(r.renderer, r.model, r.camera, r.fb)
        assert L.bnGetLastError() == 3
        L.bnClearLastError()
        # a group needs a volume or a geometry, and takes one of each at most
        assert not L.bnGroupCreate(r.ctx, 0, None, 0, None, 0)
        assert L.bnGetLastError() == 3
        L.bnClearLastError()
        two = (ctypes.c_void_p * 2)(r.iso, r.iso)
        assert not L.bnGroupCreate(r.ctx, 0, two, 2, None, 0)
        assert L.bnGetLastError() == 3
        L.bnClearLastError()
    finally:
        r.close()
