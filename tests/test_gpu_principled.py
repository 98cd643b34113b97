"""Principled volumes (PrincipledVolume.h: density, scattering / absorption
colours, threshold, value range, emission, blackbody): sampling, majorants and
the multi-scatter build's hit tint / albedo / emission are bit-exact against
the oracle, with single and multiple scattering and in batches."""
import pytest

from tests.helpers import assert_bitexact, gpu_render, oracle_render, small_noise_scene

pytestmark = pytest.mark.gpu

PV_SCENES = {
    "default_build": lambda: small_noise_scene(phase="simple", principled={"enabled": 1, "scatter_color": (0.9, 0.6, 0.3)}),
    "hg_emission_absorption": lambda: small_noise_scene(
        phase="hg", anisotropy=0.4,
        principled={"enabled": 1, "emission_strength": 2.0, "emission_color": (1.0, 0.7, 0.4),
                    "absorption_color": (0.2, 0.1, 0.0), "density": 1.5}),
    "threshold_range": lambda: small_noise_scene(
        phase="hg", anisotropy=0.0,
        principled={"enabled": 1, "density_threshold": 0.35, "value_range": (0.2, 0.8), "density_scale": 2.0}),
    "blackbody_log_branch": lambda: small_noise_scene(
        phase="hg", principled={"enabled": 1, "blackbody_intensity": 1.5, "temperature": 3000.0}),
    "blackbody_pow_branch_ms": lambda: small_noise_scene(
        phase="hg", anisotropy=0.6, max_volume_bounces=3,
        principled={"enabled": 1, "blackbody_intensity": 1.0, "temperature": 8000.0, "emission_strength": 0.5}),
    "noise_u8_ms": lambda: small_noise_scene(
        dtype="u8", phase="hg", anisotropy=-0.3, max_volume_bounces=2,
        principled={"enabled": 1, "scatter_color": (0.5, 0.8, 1.0), "absorption_color": (0.3, 0.3, 0.3)}),
}


@pytest.mark.parametrize("name", sorted(PV_SCENES))
def test_principled_bitexact(name):
    d = PV_SCENES[name]()
    for spp in (1, 4):
        img, st = gpu_render(d, spp)
        ref, _, ost = oracle_render(d, spp)
        assert_bitexact(img, ref, f"{name} spp={spp}")
        assert st["samples"] == ost["samples"]
        assert st["mc_visits"] == ost["mc_visits"]
        assert st["rays"] == ost["rays"]


def test_principled_majorants_bitexact():
    import barney_b200 as bn
    import numpy as np
    import oracle
    d = PV_SCENES["threshold_range"]()
    r = bn.VolumeRenderer(d)
    try:
        ranges, maj = r.macrocells()
    finally:
        r.close()
    sc = oracle.Scene(d)
    oranges = oracle.build_ranges(sc)
    assert_bitexact(ranges, oranges, "ranges")
    assert_bitexact(maj, oracle.map_majorants(sc, oranges), "principled majorants")
    assert (maj > 0).any()


def test_principled_jobs_in_a_batch_equal_solo_renders():
    import barney_b200 as bn
    descs = [PV_SCENES["hg_emission_absorption"](), small_noise_scene(w=24, h=20), PV_SCENES["noise_u8_ms"]()]
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
