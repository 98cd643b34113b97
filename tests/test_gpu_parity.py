"""Parity of the CUDA path (through the bn* C ABI) with the CPU oracle.

Bar: bit-exact.  Macrocell ranges and majorants, every accumulated float4
pixel, the work counters (volume samples, macrocell visits, rays) and the
rgba8 frames must be identical; the sRGB frame may differ by one 8-bit step
where powf of the two math libraries rounds differently (tolerance 1).
"""
import numpy as np
import pytest

import oracle
from barney_b200 import synth
from tests.helpers import (assert_bitexact, gpu_render, oracle_render, small_blob_scene,
                           small_noise_scene)

pytestmark = pytest.mark.gpu


def _bn():
    import barney_b200 as bn
    return bn


@pytest.mark.parametrize("dtype", ["f32", "u8", "u16", "f16", "bf16"])
@pytest.mark.parametrize("shape", [(33, 40, 17), (64, 64, 64), (2, 2, 2), (9, 9, 9), (3, 70, 5)])
def test_macrocells_bitexact(dtype, shape):
    rng = np.random.default_rng(hash((dtype, shape)) & 0xFFFF)
    vol = synth.to_storage(rng.random(shape).astype(np.float32), dtype)
    d = synth.scene(vol, dtype, 8, 8, synth.tf_knots(256, 1), 50.0, synth.DEFAULT_CAMERA)
    for round_up in (False, True):
        d["majorant_round_up"] = round_up
        r = _bn().VolumeRenderer(d)
        ranges, maj = r.macrocells()
        r.close()
        sc = oracle.Scene(d)
        o_ranges = oracle.build_ranges(sc)
        o_maj = oracle.map_majorants(sc, o_ranges)
        assert_bitexact(ranges, o_ranges, "ranges")
        assert_bitexact(maj, o_maj, "majorants")


SCENES = {
    "blobs_ambient": lambda: small_blob_scene(),
    "blobs_emission_absorption": lambda: small_blob_scene(emission_absorption=True, ambient=0.0),
    "noise_hg_dirlight": lambda: small_noise_scene(),
    "noise_simple_dirlight": lambda: small_noise_scene(phase="simple"),
    "noise_u8": lambda: small_noise_scene(dtype="u8"),
    "noise_f16": lambda: small_noise_scene(dtype="f16"),
    "noise_bf16": lambda: small_noise_scene(dtype="bf16"),
    "noise_u16": lambda: small_noise_scene(dtype="u16"),
    "noise_exact_log": lambda: small_noise_scene(exact_log=True),
    "two_lights_aniso": lambda: small_noise_scene(
        dir_lights=[{"direction": (-1, -1, -1), "radiance": 1.0},
                    {"direction": (0.3, -1, 0.2), "radiance": 2.0, "color": (1.0, 0.5, 0.25)}],
        anisotropy=0.5),
    "gradient_bg_cutplane": lambda: small_blob_scene(bg_color=(0, 0, 0, -1), cut_plane=(1.0, 0.0, 0.0, -0.5)),
    "camera_inside": lambda: small_blob_scene(camera=synth.look_at((0.5, 0.5, 0.45), (0.5, 0.5, 1.0), fovy=70)),
    "axis_aligned_view": lambda: small_blob_scene(w=41, h=41, camera={"position": (0.5, 0.5, -2.0), "direction": (0.0, 0.0, 1.0),
                                                         "up": (0.0, 1.0, 0.0), "fovy": 30.0}),
    "ragged_volume": lambda: synth.scene(synth.blobs(20, 0)[:, 3:17, 1:20].copy(), "f32", 37, 29,
                                         synth.tf_linear_ramp(64), 30.0, synth.DEFAULT_CAMERA,
                                         spacing=(1 / 18.0, 1 / 13.0, 1 / 19.0)),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_render_bitexact(name):
    d = SCENES[name]()
    for spp in (1, 5):
        img, st = gpu_render(d, spp)
        ref, _, ost = oracle_render(d, spp)
        assert_bitexact(img, ref, f"{name} spp={spp}")
        assert st["samples"] == ost["samples"]
        assert st["mc_visits"] == ost["mc_visits"]
        assert st["rays"] == ost["rays"]
        assert st["error_flags"] == 0


def test_accumulation_across_renders():
    d = small_noise_scene(w=32, h=24)
    img, _ = gpu_render(d, 2, renders=3)  # accumIDs 0..5 over three bnRender calls
    ref, _, _ = oracle_render(d, 6)
    assert_bitexact(img, ref, "3 x 2 waves")


@pytest.mark.parametrize("fmt", ["rgba8", "rgba8_srgb"])
def test_color_formats(fmt):
    d = small_blob_scene()
    img, _ = gpu_render(d, 3, fmt=fmt)
    ref, _, _ = oracle_render(d, 3, fmt=fmt)
    if fmt == "rgba8":
        assert_bitexact(img, ref, fmt)
    else:
        a = img.view(np.uint8).astype(int)
        b = ref.view(np.uint8).astype(int)
        assert np.abs(a - b).max() <= 1


def test_deterministic_and_launch_shape_invariant():
    bn = _bn()
    d = small_noise_scene(n=48, w=64, h=40)
    r = bn.VolumeRenderer(d)
    r.set_spp(3)
    r.render()
    a = r.read().copy()
    for bps, tpb in [(1, 32), (2, 64), (0, 128), (3, 96)]:
        r.accum_reset()
        r.set_launch_config(bps, tpb)
        r.render()
        assert_bitexact(r.read(), a, f"launch {bps}x{tpb}")
    r.close()


def test_invalid_calls_record_errors():
    bn = _bn()
    d = small_blob_scene()
    r = bn.VolumeRenderer(d)
    L = r.L
    L.bnClearLastError()
    L.bnFrameBufferRead(r.fb, 1, np.zeros(4, np.uint32).ctypes.data, bn.BN_UFIXED8_RGBA)  # wrong format
    assert L.bnGetLastError() != 0
    L.bnClearLastError()
    L.bnSet1i(r.renderer, b"maxVolumeBounces", 3)
    L.bnSet1i(r.renderer, b"bnx.hgPhase", 1)
    L.bnCommit(r.renderer)
    L.bnRender(r.renderer, r.model, r.camera, r.fb)
    assert L.bnGetLastError() == 0  # multiple scattering renders
    L.bnSet1f(r.camera, b"apertureRadius", 0.1)
    L.bnCommit(r.camera)
    L.bnRender(r.renderer, r.model, r.camera, r.fb)
    assert L.bnGetLastError() == 3  # unsupported: depth of field
    L.bnClearLastError()
    L.bnxSetLaunchConfig(r.ctx, 1, 256)  # beyond the kernel's launch bounds
    assert L.bnGetLastError() == 2
    L.bnClearLastError()
    r.close()


def test_scheduling_thresholds_do_not_change_results():
    bn = _bn()
    d = small_noise_scene(n=40, w=48, h=40)
    r = bn.VolumeRenderer(d)
    r.set_spp(3)
    r.render()
    a = r.read().copy()
    for service in (1, 32, 7):
        r.accum_reset()
        r.set_scheduling(service)
        r.render()
        assert_bitexact(r.read(), a, f"service batch {service}")
    r.close()


BATCH = [
    (lambda: small_noise_scene(n=40, w=48, h=32), 3),
    (lambda: small_blob_scene(n=24, w=40, h=36), 2),
    (lambda: small_noise_scene(n=33, w=37, h=29, dtype="u8", phase="simple"), 4),
    (lambda: small_blob_scene(n=20, w=20, h=52, emission_absorption=True, ambient=0.0), 1),
    (lambda: small_noise_scene(n=24, w=16, h=16, dtype="f16", compensated_accum=True), 5),
]


@pytest.mark.parametrize("graphs", [True, False])
def test_batch_equals_one_render_per_job(graphs):
    bn = _bn()
    descs = [f() for f, _ in BATCH]
    spps = [s for _, s in BATCH]
    ctx = bn.Context()
    rs = [bn.VolumeRenderer(d, context=ctx) for d in descs]
    try:
        ctx.set_graphs(graphs)
        for r, spp in zip(rs, spps):
            r.set_spp(spp)
        ctx.render_batch(rs)
        ctx.render_batch(rs)  # the second frame continues every job's accumulation
        total = 0
        for r, d, spp in zip(rs, descs, spps):
            sc = oracle.Scene(d)
            acc = np.zeros((d["height"], d["width"], 4), np.float32)
            comp = np.zeros_like(acc) if d.get("compensated_accum") else None
            _, _, st = oracle.render(sc, 0, 2 * spp, accum=acc, comp=comp)
            ref = oracle.resolve(acc, 2 * spp, comp=comp)
            assert_bitexact(r.read(), ref, f"batch job {d['width']}x{d['height']}")
            total += st["samples"]
        assert ctx.stats()["error_flags"] == 0
    finally:
        for r in rs:
            r.close()
        ctx.close()


def test_autotuned_batch_is_still_exact():
    bn = _bn()
    descs = [f() for f, _ in BATCH[:3]]
    ctx = bn.Context()
    rs = [bn.VolumeRenderer(d, context=ctx) for d in descs]
    try:
        for r in rs:
            r.set_spp(2)
        best = ctx.autotune_batch(rs)
        assert best["threadsPerBlock"] in (64, 128) and best["renderMs"] > 0
        ctx.render_batch(rs)
        for r, d in zip(rs, descs):
            ref, _, _ = oracle_render(d, 2)
            assert_bitexact(r.read(), ref, "after autotune")
    finally:
        for r in rs:
            r.close()
        ctx.close()


def test_compensated_accumulation_bitexact():
    d = small_noise_scene(w=32, h=24, compensated_accum=True)
    img, _ = gpu_render(d, 7, renders=2)
    sc = oracle.Scene(d)
    acc = np.zeros((24, 32, 4), np.float32)
    comp = np.zeros_like(acc)
    oracle.render(sc, 0, 14, accum=acc, comp=comp)
    assert_bitexact(img, oracle.resolve(acc, 14, comp=comp), "compensated")


def test_anari_structured_regular_field_renders_like_native_calls():
    """bnxAnariStructuredRegular + the ANARI TF mapping give the same frame as
    the native calls with the same data (SpatialField.cpp / Volume.cpp path)."""
    import ctypes
    bn = _bn()
    d = small_blob_scene(n=20, w=32, h=24)
    L = bn.lib()
    ctx = bn.Context()
    try:
        vol = np.ascontiguousarray(d["voxels"])
        sf = L.bnxAnariStructuredRegular(ctx.ctx, 0, bn.BN_FLOAT32, vol.ctypes.data, 20, 20, 20,
                                         bn.bn_float3(0, 0, 0), bn.bn_float3(*d["spacing"]))
        bn.check()
        assert sf
        table = bn.anari_transfer_function_1d(colors=d["tf"][:, :3].copy(), opacities=d["tf"][:, 3].copy())
        assert np.array_equal(table, d["tf"])  # same-length arrays resample to themselves
        v = L.bnVolumeCreate(ctx.ctx, 0, sf)
        dens = L.bnxAnariDensityScale(ctypes.c_float(1.0 / d["density"]))  # unitDistance -> densityAt1
        L.bnVolumeSetXF(v, bn.bn_float2(0.0, 1.0), table.ctypes.data, table.shape[0], dens)
        L.bnSet1f(v, b"anisotropy", 0.6)
        L.bnCommit(v)
        vols = (ctypes.c_void_p * 1)(v)
        g = L.bnGroupCreate(ctx.ctx, 0, None, 0, vols, 1)
        L.bnGroupBuild(g)
        m = L.bnModelCreate(ctx.ctx)
        groups = (ctypes.c_void_p * 1)(g)
        L.bnSetInstances(m, 0, groups, None, 1)
        L.bnBuild(m, 0)
        cam = L.bnCameraCreate(ctx.ctx, b"perspective")
        c = d["camera"]
        L.bnSet3f(cam, b"position", *c["position"])
        L.bnSet3f(cam, b"direction", *c["direction"])
        L.bnSet3f(cam, b"up", *c["up"])
        L.bnSet1f(cam, b"fovy", c["fovy"])
        L.bnCommit(cam)
        ren = L.bnRendererCreate(ctx.ctx, b"default")
        L.bnSet1i(ren, b"pathsPerPixel", 2)
        L.bnSet1f(ren, b"ambientRadiance", d["ambient"])
        L.bnSet4f(ren, b"bgColor", *d["bg_color"])
        L.bnCommit(ren)
        fb = L.bnFrameBufferCreate(ctx.ctx, 0)
        L.bnFrameBufferResize(fb, bn.BN_FLOAT4, 32, 24, 1)
        L.bnRender(ren, m, cam, fb)
        img = np.zeros((24, 32, 4), np.float32)
        L.bnFrameBufferRead(fb, 1, img.ctypes.data, bn.BN_FLOAT4)
        bn.check()
    finally:
        ctx.close()
    ref, _ = gpu_render(dict(d, density=dens), 2)
    assert_bitexact(img, ref, "ANARI-mapped field vs native calls")


@pytest.mark.parametrize("w,h", [(1, 1), (1, 37), (37, 1), (5, 9), (33, 7)])
def test_degenerate_frame_shapes(w, h):
    # single pixels, single rows / columns and heights that end in a partial
    # 4-row band exercise the chunk and band arithmetic of the pixel order
    d = small_noise_scene(w=w, h=h)
    img, st = gpu_render(d, 3)
    ref, _, ost = oracle_render(d, 3)
    assert_bitexact(img, ref, f"{w}x{h}")
    assert st["rays"] == ost["rays"]


def test_long_accumulation_in_a_thin_frame():
    d = small_blob_scene(w=3, h=11, bg_color=(0, 0, 0, -1))
    img, _ = gpu_render(d, 7, renders=3)  # accumIDs 0..20
    ref, _, _ = oracle_render(d, 21)
    assert_bitexact(img, ref, "3 x 7 waves")


def test_data_set_and_instance_transform_updates():
    """bnDataSet replaces the group's light list in place; bnUpdateInstanceTransforms
    accepts the identity for the one instance and rejects anything else."""
    import ctypes
    bn = _bn()
    d = small_noise_scene()
    r = bn.VolumeRenderer(d)
    L = r.L
    try:
        L.bnClearLastError()
        L.bnDataSet(r.lights_data, 0, None)  # no directional lights any more
        assert L.bnGetLastError() == 0
        r.set_spp(2)
        r.render()
        ref, _, _ = oracle_render(dict(d, dir_lights=[]), 2)
        assert_bitexact(r.read(), ref, "lights removed by bnDataSet")

        class BNTransform(ctypes.Structure):
            _fields_ = [("m", ctypes.c_float * 12)]
        ident = BNTransform()
        ident.m[:] = (1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0)
        L.bnUpdateInstanceTransforms(r.model, 0, ctypes.byref(ident), 1)
        assert L.bnGetLastError() == 0
        moved = BNTransform()
        moved.m[:] = (1, 0, 0, 0, 1, 0, 0, 0, 1, 0.5, 0, 0)
        L.bnUpdateInstanceTransforms(r.model, 0, ctypes.byref(moved), 1)
        assert L.bnGetLastError() == 3
        L.bnClearLastError()
        L.bnUpdateInstanceTransforms(r.model, 0, ctypes.byref(ident), 2)
        assert L.bnGetLastError() == 2
        L.bnClearLastError()
    finally:
        r.close()


@pytest.mark.parametrize("graphs", [False, True])
def test_one_job_batch_equals_bnrender(graphs):
    # without a graph a one-job batch runs the single-frame kernel; with one,
    # the batch kernel: the same frame either way
    bn = _bn()
    d = small_noise_scene(w=37, h=23, iso={"value": 0.5})
    ctx = bn.Context()
    r = bn.VolumeRenderer(d, context=ctx)
    try:
        ctx.set_graphs(graphs)
        r.set_spp(2)
        ctx.render_batch([r])
        ctx.render_batch([r])  # accumulates: 4 waves
        ref, _, _ = oracle_render(d, 4)
        assert_bitexact(r.read(), ref, f"one-job batch, graphs={graphs}")
    finally:
        r.close()
        ctx.close()
