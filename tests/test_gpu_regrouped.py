"""The regrouped render kernel (bnxSetRegrouping): pixel slots in shared
memory, taken by warps from ring queues (new pixels, rays to trace,
collisions to shade, rays that ended).  It must give the
per-lane kernel's frames and work counters bit for bit (both are checked
against the CPU oracle here), over every plain scene of the parity tests,
accumulation across renders and compensated accumulation, pixel partitions,
degenerate frame shapes, the fast-math object's instance, and a render
deadline that aborts the frame and leaves the context usable.  (It is not
the default: on the workloads measured the per-lane kernel is faster.)"""
import numpy as np
import pytest

from tests.helpers import assert_bitexact, oracle_render, small_blob_scene, small_noise_scene
from test_gpu_parity import SCENES

pytestmark = pytest.mark.gpu


def regrouped_render(d, spp, renders=1, fmt="float4", regroup=True, partition=None):
    import barney_b200 as bn
    r = bn.VolumeRenderer(d, color_format=fmt)
    try:
        r.set_regrouping(regroup)
        if partition:
            r.set_partition(*partition)
        r.set_spp(spp)
        for _ in range(renders):
            r.render()
        return r.read().copy(), r.stats()
    finally:
        r.close()


@pytest.mark.parametrize("name", sorted(SCENES))
def test_regrouped_render_bitexact(name):
    d = SCENES[name]()
    for spp in (1, 5):
        img, st = regrouped_render(d, spp)
        ref, _, ost = oracle_render(d, spp)
        assert_bitexact(img, ref, f"{name} spp={spp}")
        assert (st["samples"], st["mc_visits"], st["rays"]) == (ost["samples"], ost["mc_visits"], ost["rays"])
        assert st["error_flags"] == 0


@pytest.mark.parametrize("compensated", [False, True])
def test_regrouped_accumulation_across_renders(compensated):
    d = small_noise_scene(w=45, h=31, compensated_accum=compensated)
    img, _ = regrouped_render(d, 2, renders=3)
    want, _ = regrouped_render(d, 2, renders=3, regroup=False)
    assert_bitexact(img, want, "3 x 2 waves, regrouped vs per-lane")
    if not compensated:
        ref, _, _ = oracle_render(d, 6)
        assert_bitexact(img, ref, "3 x 2 waves")


@pytest.mark.parametrize("w,h", [(1, 1), (1, 37), (37, 1), (33, 1), (500, 3)])
def test_regrouped_degenerate_frames(w, h):
    d = small_blob_scene(w=w, h=h)
    img, st = regrouped_render(d, 3)
    ref, _, ost = oracle_render(d, 3)
    assert_bitexact(img, ref, f"{w}x{h}")
    assert st["samples"] == ost["samples"]


def test_regrouped_partitions_and_fast_math():
    import barney_b200 as bn
    d = small_noise_scene(w=67, h=45)
    full, _ = regrouped_render(d, 3)
    parts = [regrouped_render(d, 3, partition=(r, 3))[0] for r in range(3)]
    owners = bn.partition_owners(67, 45, 3)
    assert_bitexact(bn.merge_partitions(np.stack(parts), owners), full, "3 partitions")
    # the fast-math object's regrouped kernel runs, close to the fast-math
    # per-lane kernel (the two are compiled separately, so fused operations
    # may differ between them)
    df = dict(d, fast_math=True)
    a, sa = regrouped_render(df, 16)
    b, sb = regrouped_render(df, 16, regroup=False)
    assert sa["error_flags"] == 0 and sa["samples"] > 0
    assert np.abs(a - b).mean() / np.abs(b).mean() < 0.05


def test_regrouped_deadline_aborts_and_context_recovers():
    import barney_b200 as bn
    from barney_b200 import synth
    big = synth.config2(n=96, width=1920, height=1080, spp=256)
    r = bn.VolumeRenderer(big, color_format="rgba8")
    try:
        r.set_regrouping(True)
        r.set_spp(1)
        r.render()
        r.set_spp(256)
        r.set_timeout(1)
        with pytest.raises(bn.BarneyError) as e:
            r.render()
        assert "error 8" in str(e.value)
        assert r.stats()["error_flags"] & 2
        r.set_timeout(0)
        r.set_spp(1)
        r.render()
        assert r.stats()["error_flags"] == 0
    finally:
        r.close()
