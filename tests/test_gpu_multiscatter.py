"""Multi-scatter volumes (the multi-scatter build: HG phase, maxVolumeBounces
> 0): every pixel, every counter and every accumulated sum equal the oracle's
restatement of bounce() with HG direction sampling, path throughput in
binary16, environment MIS on escaped scattered rays and the path-depth cap."""
import numpy as np
import pytest

import oracle
from barney_b200 import synth
from tests.helpers import assert_bitexact, gpu_render, oracle_render, small_blob_scene, small_noise_scene

pytestmark = pytest.mark.gpu

MS_SCENES = {
    "iso_1_bounce": lambda: small_noise_scene(phase="hg", anisotropy=0.0, max_volume_bounces=1),
    "forward_3_bounces": lambda: small_noise_scene(phase="hg", anisotropy=0.6, max_volume_bounces=3),
    "backward_4_bounces": lambda: small_noise_scene(phase="hg", anisotropy=-0.5, max_volume_bounces=4),
    "depth_cap": lambda: small_noise_scene(phase="hg", anisotropy=0.3, max_volume_bounces=14),
    "env_only": lambda: small_blob_scene(phase="hg", anisotropy=0.4, max_volume_bounces=5, ambient=0.8),
    "two_lights_u8": lambda: small_noise_scene(
        dtype="u8", phase="hg", anisotropy=0.7, max_volume_bounces=2,
        dir_lights=[{"direction": (-1, -1, -1), "radiance": 1.0},
                    {"direction": (0.3, -1, 0.2), "radiance": 2.0, "color": (1.0, 0.5, 0.25)}]),
    "f16_exact_log": lambda: small_noise_scene(dtype="f16", phase="hg", anisotropy=0.5, max_volume_bounces=3,
                                               exact_log=True, majorant_round_up=True),
}


@pytest.mark.parametrize("name", sorted(MS_SCENES))
def test_multi_scatter_bitexact(name):
    d = MS_SCENES[name]()
    for spp in (1, 4):
        img, st = gpu_render(d, spp)
        ref, _, ost = oracle_render(d, spp)
        assert_bitexact(img, ref, f"{name} spp={spp}")
        assert st["samples"] == ost["samples"]
        assert st["mc_visits"] == ost["mc_visits"]
        assert st["rays"] == ost["rays"]
        assert st["error_flags"] == 0


def test_multi_scatter_accumulates_across_renders_and_compensates():
    d = small_noise_scene(w=32, h=24, phase="hg", anisotropy=0.6, max_volume_bounces=3, compensated_accum=True)
    img, _ = gpu_render(d, 3, renders=2)
    sc = oracle.Scene(d)
    acc = np.zeros((24, 32, 4), np.float32)
    comp = np.zeros_like(acc)
    oracle.render(sc, 0, 6, accum=acc, comp=comp)
    assert_bitexact(img, oracle.resolve(acc, 6, comp=comp), "2 x 3 waves, compensated")


def test_max_volume_bounces_is_inert_in_the_default_build():
    # SimplePhase (default build): a volume scatter ends the path, so
    # maxVolumeBounces changes nothing (shadeRays.cu:23-25, 789-796)
    base = small_noise_scene(phase="simple")
    a, _ = gpu_render(base, 3)
    b, _ = gpu_render(dict(base, max_volume_bounces=6), 3)
    assert_bitexact(a, b, "maxVolumeBounces with SimplePhase")


def test_multi_scatter_jobs_in_a_batch_equal_solo_renders():
    import barney_b200 as bn
    descs = [small_noise_scene(phase="hg", anisotropy=0.6, max_volume_bounces=3),
             small_noise_scene(w=24, h=20),  # single scatter in the same launch
             small_blob_scene(phase="hg", anisotropy=-0.3, max_volume_bounces=2)]
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


def test_more_bounces_add_light():
    d = small_noise_scene(w=40, h=30, phase="hg", anisotropy=0.6)
    means = []
    for mvb in (0, 1, 3):
        img, _ = gpu_render(dict(d, max_volume_bounces=mvb), 16)
        means.append(float(img[..., :3].mean()))
    assert means[0] < means[1] < means[2]
