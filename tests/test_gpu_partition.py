"""Pixel-tile data parallelism on one GPU: every rank's partition of a frame,
rendered on its own, merges by the owner map into exactly the unpartitioned
frame, and the ranks' work counters add up to the whole frame's."""
import numpy as np
import pytest

from tests.helpers import assert_bitexact, small_blob_scene, small_noise_scene

pytestmark = pytest.mark.gpu


def _render(d, spp, rank, count, renders=1):
    import barney_b200 as bn
    r = bn.VolumeRenderer(d, color_format="float4")
    try:
        r.set_partition(rank, count)
        r.set_spp(spp)
        for _ in range(renders):
            r.render()
        return r.read(), r.stats()
    finally:
        r.close()


@pytest.mark.parametrize("count", [2, 3, 8])
def test_partitions_merge_into_the_full_frame(count):
    import barney_b200 as bn
    d = small_noise_scene(w=67, h=45)  # 3015 pixels: 2 full tiles and a partial one
    full, fst = _render(d, 3, 0, 1)
    parts, samples = [], 0
    for rank in range(count):
        img, st = _render(d, 3, rank, count)
        parts.append(img)
        samples += st["samples"]
        assert st["error_flags"] == 0
    owners = bn.partition_owners(d["width"], d["height"], count)
    assert_bitexact(bn.merge_partitions(np.stack(parts), owners), full, f"{count} partitions")
    assert samples == fst["samples"]


def test_partitions_accumulate_across_renders_with_compensation():
    import barney_b200 as bn
    d = small_blob_scene(w=80, h=50, compensated_accum=True)
    full, _ = _render(d, 2, 0, 1, renders=2)
    parts = [_render(d, 2, r, 2, renders=2)[0] for r in range(2)]
    assert_bitexact(bn.merge_partitions(np.stack(parts), bn.partition_owners(80, 50, 2)), full, "2 x 2 waves")


def test_partition_is_rejected_for_batches():
    import barney_b200 as bn
    ctx = bn.Context()
    r = bn.VolumeRenderer(small_noise_scene(w=16, h=16), context=ctx)
    try:
        r.set_partition(1, 2)
        with pytest.raises(bn.BarneyError):
            ctx.render_batch([r])
        with pytest.raises(bn.BarneyError):
            r.set_partition(2, 2)  # rank out of range
    finally:
        r.close()
        ctx.close()


def test_isosurface_partitions_merge_into_the_full_frame():
    import barney_b200 as bn
    d = small_noise_scene(w=67, h=45, iso={"value": 0.5, "opacity": 0.8}, max_volume_bounces=2)
    full, fst = _render(d, 2, 0, 1)
    parts, rays = [], 0
    for rank in range(3):
        img, st = _render(d, 2, rank, 3)
        parts.append(img)
        rays += st["rays"]
    owners = bn.partition_owners(d["width"], d["height"], 3)
    assert_bitexact(bn.merge_partitions(np.stack(parts), owners), full, "3 isosurface partitions")
    assert rays == fst["rays"]
